/*
 * ns3d_oracle.h -- CPU restatement of the ns3d_wcns right-hand side and RK3
 * time advance, used ONLY as the test oracle and as the CPU baseline port.
 *
 * Test infrastructure: the product (ns3d_wcns_b200) never links this file.
 * Every routine cites the reference file:line it restates; the restatement
 * keeps the reference's floating-point operation order so that it can be
 * pinned bit-for-bit against the reference itself (oracle/_ref).
 *
 * Storage follows field_structures.h: SoA arrays of sx*sy*sz doubles,
 * id = (k*sy + j)*sx + i, sx = nx + 2*3 (ghost layers = 3 for WENO5/MDCD,
 * initialization.cpp:175-192).
 */
#ifndef NS3D_ORACLE_H
#define NS3D_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* enum values follow the reference's enum order (field_structures.h:131-165) */
enum { ORC_WENO5 = 0, ORC_ZERO = 1, ORC_MDCD_LINEAR = 2, ORC_MDCD_HYBRID = 3 };
enum { ORC_ROE = 0, ORC_RUSANOV = 1, ORC_HLLC = 2, ORC_HLL = 3, ORC_HLLC_P = 4, ORC_AUSM = 5 };
enum { ORC_PERIODIC = 0, ORC_WALL = 1, ORC_SYMMETRY = 2, ORC_OUTFLOW = 3, ORC_INFLOW = 4 };

typedef struct orc_config {
    double gamma, Pr, Ma, Re, cfl, dt_fixed;
    double mdcd_diss, mdcd_disp;
    double sutherland_s;           /* S_ref, field_structures.h:95 */
    double Lx, Ly, Lz;
    int nx, ny, nz;
    int interpolation, riemann, char_recon;
    int bc[6];                     /* xmin xmax ymin ymax zmin zmax */
} orc_config;

/* Field names accepted by orc_get/orc_set (same spelling as Field3D members). */
int orc_init(const orc_config *cfg);           /* 0 ok, <0 invalid config */
void orc_free(void);
int orc_dims(int *out6);                         /* nx ny nz sx sy sz */
int orc_set_interior_prims(const double *rho, const double *u, const double *v,
                           const double *w, const double *p);
long orc_get(const char *name, double *dst, long cap);
int orc_set(const char *name, const double *src, long count);
void orc_compute_rhs(void);
void orc_apply_boundary(void);
void orc_prim_to_cons(void);
void orc_cons_to_prim(void);
void orc_rk3_step(double dt);
double orc_timestep(void);
double orc_total_energy(void);
void orc_residuals(double out[5]);

/* Scalar kernels, exported for known-answer tests against the reference. */
double orc_weno5(const double f[6]);
double orc_mdcd_linear(const double f[6], double disp, double diss);
double orc_mdcd_hybrid(const double f[6], double disp, double diss);
void orc_riemann(int solver, const double UL[5], const double UR[5], int dir, double gamma,
                 double F[5]);

#ifdef __cplusplus
}
#endif
#endif
