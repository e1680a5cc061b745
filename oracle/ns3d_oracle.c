/*
 * ns3d_oracle.c -- CPU restatement of ns3d_wcns's RHS + RK3 hot path.
 *
 * TEST INFRASTRUCTURE (the oracle).  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg may load it.  It restates the reference's
 * algorithm in plain C, keeping the reference's floating-point operation
 * order, and is pinned bit-for-bit against the reference sources compiled in
 * place (oracle/_ref) by tests/test_oracle_pin.py and the committed golden
 * fixtures under tests/golden/.
 *
 * Reference files cited as file:line (wylx-2/ns3d_wcns).
 */
#include "ns3d_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NG 3

typedef struct {
    orc_config c;
    int nx, ny, nz, sx, sy, sz;
    long ncell, nfx, nfy, nfz;
    double dx, dy, dz, Cv, Cp, Rgas, mu;
    int periodic[3];
    /* conserved, backup, primitives, rhs */
    double *U[5], *U0[5], *W[5], *T, *R[5];
    /* half-node fluxes per direction, 5 components each */
    double *FX[5], *FY[5], *FZ[5];
    /* gradients du,dv,dw,dT x (x,y,z) */
    double *G[12];
    /* node viscous fluxes: Fv(momx,momy,momz,E), Hv(...), Gv(...) */
    double *V[12];
} orc_state;

static orc_state *S = NULL;

static inline long I3(int i, int j, int k) { return ((long)k * S->sy + j) * S->sx + i; }
/* face indices, field_structures.h:73-82 */
static inline long IFX(int i, int j, int k) { return ((long)k * S->sy + j) * (S->sx - 1) + i; }
static inline long IFY(int i, int j, int k) { return ((long)k * (S->sy - 1) + j) * S->sx + i; }
static inline long IFZ(int i, int j, int k) { return ((long)k * S->sy + j) * S->sx + i; }

static double *zalloc(long n) { return (double *)calloc((size_t)n, sizeof(double)); }

void orc_free(void) {
    if (!S) return;
    for (int n = 0; n < 5; ++n) {
        free(S->U[n]); free(S->U0[n]); free(S->W[n]); free(S->R[n]);
        free(S->FX[n]); free(S->FY[n]); free(S->FZ[n]);
    }
    for (int n = 0; n < 12; ++n) { free(S->G[n]); free(S->V[n]); }
    free(S->T);
    free(S);
    S = NULL;
}

int orc_init(const orc_config *cfg) {
    orc_free();
    if (cfg->interpolation == ORC_ZERO) return -2; /* ghost_layers=1 makes a10/a11 read out of bounds */
    if (cfg->interpolation < 0 || cfg->interpolation > 3) return -2;
    if (cfg->riemann < 0 || cfg->riemann > 5) return -3;
    if (cfg->nx < 1 || cfg->ny < 1 || cfg->nz < 1) return -4;
    S = (orc_state *)calloc(1, sizeof(orc_state));
    S->c = *cfg;
    S->nx = cfg->nx; S->ny = cfg->ny; S->nz = cfg->nz;
    S->sx = S->nx + 2 * NG; S->sy = S->ny + 2 * NG; S->sz = S->nz + 2 * NG;
    S->ncell = (long)S->sx * S->sy * S->sz;
    S->nfx = (long)(S->sx - 1) * S->sy * S->sz;
    S->nfy = (long)S->sx * (S->sy - 1) * S->sz;
    S->nfz = (long)S->sx * S->sy * (S->sz - 1);
    /* derived constants, initialization.cpp:170-172, 194-197 */
    S->dx = cfg->Lx / (cfg->nx);
    S->dy = cfg->Ly / (cfg->ny);
    S->dz = cfg->Lz / (cfg->nz);
    S->Cv = 1.0 / (cfg->gamma * (cfg->gamma - 1.0) * cfg->Ma * cfg->Ma);
    S->Cp = S->Cv * cfg->gamma;
    S->Rgas = 1.0 / (cfg->Ma * cfg->Ma * cfg->gamma);
    S->mu = 1.0 / cfg->Re;
    /* periods[d] = 1 only when both sides are Periodic, initialization.cpp:161-169 */
    for (int d = 0; d < 3; ++d)
        S->periodic[d] = (cfg->bc[2 * d] == ORC_PERIODIC && cfg->bc[2 * d + 1] == ORC_PERIODIC);
    for (int n = 0; n < 5; ++n) {
        S->U[n] = zalloc(S->ncell); S->U0[n] = zalloc(S->ncell);
        S->W[n] = zalloc(S->ncell); S->R[n] = zalloc(S->ncell);
        S->FX[n] = zalloc(S->nfx); S->FY[n] = zalloc(S->nfy); S->FZ[n] = zalloc(S->nfz);
    }
    for (int n = 0; n < 12; ++n) { S->G[n] = zalloc(S->ncell); S->V[n] = zalloc(S->ncell); }
    S->T = zalloc(S->ncell);
    /* Field3D::allocate sets rho = 1 everywhere, field_structures.h:257 */
    for (long id = 0; id < S->ncell; ++id) S->U[0][id] = 1.0;
    return 0;
}

int orc_dims(int *o) {
    if (!S) return -1;
    o[0] = S->nx; o[1] = S->ny; o[2] = S->nz; o[3] = S->sx; o[4] = S->sy; o[5] = S->sz;
    return 0;
}

/* ---------------------------------------------------------------- c2p / p2c */

/* Field3D::conservedToPrimitive, field_structures.h:444-465 (all cells). */
void orc_cons_to_prim(void) {
    const double g = S->c.gamma;
    for (long id = 0; id < S->ncell; ++id) {
        double rr = S->U[0][id];
        if (rr <= 0.0) { rr = 1e-12; S->U[0][id] = rr; }
        double u = S->U[1][id] / rr, v = S->U[2][id] / rr, w = S->U[3][id] / rr;
        S->W[1][id] = u; S->W[2][id] = v; S->W[3][id] = w;
        double kinetic = 0.5 * (u * u + v * v + w * w);
        double e_internal = S->U[4][id] / rr - kinetic;
        double p = (g - 1.0) * rr * e_internal;
        S->W[4][id] = p;
        S->T[id] = p / (rr * S->Rgas);
        /* the reference keeps density in the conserved array only */
        S->W[0][id] = rr;
    }
}

/* Field3D::primitiveToConserved, field_structures.h:468-488 (all cells). */
void orc_prim_to_cons(void) {
    const double g = S->c.gamma;
    for (long id = 0; id < S->ncell; ++id) {
        double rr = S->U[0][id];
        if (rr <= 0.0) { rr = 1e-12; S->U[0][id] = rr; }
        double u = S->W[1][id], v = S->W[2][id], w = S->W[3][id], p = S->W[4][id];
        S->U[1][id] = rr * u; S->U[2][id] = rr * v; S->U[3][id] = rr * w;
        double kinetic = 0.5 * (u * u + v * v + w * w);
        double e_internal = p / ((g - 1.0) * rr);
        S->U[4][id] = rr * (e_internal + kinetic);
        S->T[id] = p / (rr * S->Rgas);
    }
}

/* ------------------------------------------------------------- boundaries */

/* Density lives in U[0]; the reference's primitive set is (rho,u,v,w,p) with
 * rho taken from the conserved array (field_structures.h:530-534). */
static inline void copy_prim(long dst, long src) {
    S->U[0][dst] = S->U[0][src];
    for (int n = 1; n < 5; ++n) S->W[n][dst] = S->W[n][src];
}

static inline void zero_prim(long dst) {
    for (int n = 0; n < 5; ++n) { if (n == 0) S->U[0][dst] = 0.0; else S->W[n][dst] = 0.0; }
}

/* Periodic self-exchange of rho,u,v,w,p over interior tangential extents,
 * field_structures.h:517-649, 936-994 (one rank, MPI_Cart_shift -> self).
 * In a non-periodic dimension the neighbour is MPI_PROC_NULL, nothing is
 * received, and the unpack still copies the zero-initialised receive buffers
 * into the ghost slabs (field_structures.h:945-950, 988-993).  The boundary
 * conditions overwrite those zeros except on a Periodic side whose partner is
 * not Periodic. */
static void exchange_prims(void) {
    const int nx = S->nx, ny = S->ny, nz = S->nz;
    if (!S->periodic[0])
        for (int k = NG; k < NG + nz; ++k)
            for (int j = NG; j < NG + ny; ++j)
                for (int g = 0; g < NG; ++g) { zero_prim(I3(g, j, k)); zero_prim(I3(NG + nx + g, j, k)); }
    if (!S->periodic[1])
        for (int k = NG; k < NG + nz; ++k)
            for (int g = 0; g < NG; ++g)
                for (int i = NG; i < NG + nx; ++i) { zero_prim(I3(i, g, k)); zero_prim(I3(i, NG + ny + g, k)); }
    if (!S->periodic[2])
        for (int g = 0; g < NG; ++g)
            for (int j = NG; j < NG + ny; ++j)
                for (int i = NG; i < NG + nx; ++i) { zero_prim(I3(i, j, g)); zero_prim(I3(i, j, NG + nz + g)); }
    if (S->periodic[0])
        for (int k = NG; k < NG + nz; ++k)
            for (int j = NG; j < NG + ny; ++j)
                for (int g = 0; g < NG; ++g) {
                    copy_prim(I3(g, j, k), I3(g + nx, j, k));
                    copy_prim(I3(NG + nx + g, j, k), I3(NG + g, j, k));
                }
    if (S->periodic[1])
        for (int k = NG; k < NG + nz; ++k)
            for (int g = 0; g < NG; ++g)
                for (int i = NG; i < NG + nx; ++i) {
                    copy_prim(I3(i, g, k), I3(i, g + ny, k));
                    copy_prim(I3(i, NG + ny + g, k), I3(i, NG + g, k));
                }
    if (S->periodic[2])
        for (int g = 0; g < NG; ++g)
            for (int j = NG; j < NG + ny; ++j)
                for (int i = NG; i < NG + nx; ++i) {
                    copy_prim(I3(i, j, g), I3(i, j, g + nz));
                    copy_prim(I3(i, j, NG + nz + g), I3(i, j, NG + g));
                }
}

/* apply_wall_bc (== apply_symmetry_bc), boundary.cpp:58-141: mirror with the
 * normal velocity negated, full tangential extents. */
static void wall_bc(int face) {
    const int sx = S->sx, sy = S->sy, sz = S->sz;
    const int d = face / 2, hi = face % 2;
    const int ext[3] = {sx, sy, sz};
    for (int k = 0; k < sz; ++k)
        for (int j = 0; j < sy; ++j)
            for (int i = 0; i < sx; ++i) {
                int c[3] = {i, j, k};
                int x = c[d];
                int m;
                if (!hi) { if (x >= NG) continue; m = 2 * NG - 1 - x; }
                else { if (x < ext[d] - NG) continue; m = 2 * (ext[d] - NG) - 1 - x; }
                int s[3] = {i, j, k};
                s[d] = m;
                long idg = I3(c[0], c[1], c[2]), idm = I3(s[0], s[1], s[2]);
                S->U[0][idg] = S->U[0][idm];
                for (int n = 1; n < 5; ++n) S->W[n][idg] = S->W[n][idm];
                S->W[1 + d][idg] = -S->W[1 + d][idm];
            }
}

/* apply_outflow_bc, boundary.cpp:144-182: zero-gradient copy of the first /
 * last interior plane, full tangential extents. */
static void outflow_bc(int face) {
    const int sx = S->sx, sy = S->sy, sz = S->sz;
    const int d = face / 2, hi = face % 2;
    const int ext[3] = {sx, sy, sz};
    for (int k = 0; k < sz; ++k)
        for (int j = 0; j < sy; ++j)
            for (int i = 0; i < sx; ++i) {
                int c[3] = {i, j, k};
                int x = c[d];
                int src;
                if (!hi) { if (x >= NG) continue; src = NG; }
                else { if (x < ext[d] - NG) continue; src = ext[d] - NG - 1; }
                int s[3] = {i, j, k};
                s[d] = src;
                copy_prim(I3(i, j, k), I3(s[0], s[1], s[2]));
            }
}

/* apply_inflow_bc, boundary.cpp:185-205: rho=1, u=1, v=w=0, p=1 and
 * E = p/(1.4-1) + 0.5 rho |u|^2 (gamma hard-coded there). */
static void inflow_bc(int face) {
    const int sx = S->sx, sy = S->sy, sz = S->sz;
    const int d = face / 2, hi = face % 2;
    const int ext[3] = {sx, sy, sz};
    const double rho0 = 1.0, u0 = 1.0, v0 = 0.0, w0 = 0.0, p0 = 1.0, gamma = 1.4;
    const double E0 = p0 / (gamma - 1.0) + 0.5 * rho0 * (u0 * u0 + v0 * v0 + w0 * w0);
    for (int k = 0; k < sz; ++k)
        for (int j = 0; j < sy; ++j)
            for (int i = 0; i < sx; ++i) {
                int c[3] = {i, j, k};
                int x = c[d];
                if (!hi) { if (x >= NG) continue; }
                else { if (x < ext[d] - NG) continue; }
                long id = I3(i, j, k);
                S->U[0][id] = rho0; S->W[1][id] = u0; S->W[2][id] = v0; S->W[3][id] = w0;
                S->W[4][id] = p0; S->U[4][id] = E0;
            }
}

/* apply_boundary, boundary.cpp:14-54. */
void orc_apply_boundary(void) {
    exchange_prims();
    for (int face = 0; face < 6; ++face) {
        if (S->periodic[face / 2]) continue;  /* neighbour exists -> exchanged */
        switch (S->c.bc[face]) {
            case ORC_WALL: case ORC_SYMMETRY: wall_bc(face); break;
            case ORC_OUTFLOW: outflow_bc(face); break;
            case ORC_INFLOW: inflow_bc(face); break;
            default: break; /* Periodic without a periodic partner: nothing */
        }
    }
}

/* -------------------------------------------------------- interpolation */

/* weno5_interpolate, interpolation.cpp:86-115 (WCNS-E5 midpoint weights). */
double orc_weno5(const double f[6]) {
    const double f0 = f[0], f1 = f[1], f2 = f[2], f3 = f[3], f4 = f[4];
    const double eps = 1e-6;
    double b0 = (13.0 / 12.0) * (f0 - 2 * f1 + f2) * (f0 - 2 * f1 + f2) +
                0.25 * (f0 - 4 * f1 + 3 * f2) * (f0 - 4 * f1 + 3 * f2);
    double b1 = (13.0 / 12.0) * (f1 - 2 * f2 + f3) * (f1 - 2 * f2 + f3) + 0.25 * (f1 - f3) * (f1 - f3);
    double b2 = (13.0 / 12.0) * (f2 - 2 * f3 + f4) * (f2 - 2 * f3 + f4) +
                0.25 * (3 * f2 - 4 * f3 + f4) * (3 * f2 - 4 * f3 + f4);
    double a0 = (1.0 / 16.0) / ((eps + b0) * (eps + b0));
    double a1 = (5.0 / 8.0) / ((eps + b1) * (eps + b1));
    double a2 = (5.0 / 16.0) / ((eps + b2) * (eps + b2));
    double as = a0 + a1 + a2;
    double w0 = a0 / as, w1 = a1 / as, w2 = a2 / as;
    double p0 = (3 * f0 - 10 * f1 + 15 * f2) / 8.0;
    double p1 = (-f1 + 6 * f2 + 3 * f3) / 8.0;
    double p2 = (3 * f2 + 6 * f3 - f4) / 8.0;
    return w0 * p0 + w1 * p1 + w2 * p2;
}

/* mdcd_linear_interpolate, interpolation.cpp:118-133. */
double orc_mdcd_linear(const double f[6], double disp, double diss) {
    return (3.0 * disp + 3.0 * diss) / 8.0 * f[0] + (-18.0 * disp - 30 * diss - 1.0) / 16.0 * f[1] +
           (12.0 * disp + 60.0 * diss + 9.0) / 16.0 * f[2] + (12.0 * disp - 60.0 * diss + 9.0) / 16.0 * f[3] +
           (-18.0 * disp + 30.0 * diss - 1.0) / 16.0 * f[4] + (3.0 * disp - 3.0 * diss) / 8.0 * f[5];
}

static inline double sq(double x) { return x * x; } /* std::pow(x,2) is exact x*x */

/* mdcd_hybrid_interpolate, interpolation.cpp:135-209. */
double orc_mdcd_hybrid(const double f[6], double disp, double diss) {
    const double eps_small = 1e-40;
    const double f0 = f[0], f1 = f[1], f2 = f[2], f3 = f[3], f4 = f[4], f5 = f[5];
    double eps = 0.9 * 0.4 / (1.0 - 0.9 * 0.4) * 1e-4;
    double a1 = fabs(f2 - f1) + fabs(f2 - 2 * f1 + f0);
    double b1 = fabs(f2 - f3) + fabs(f2 - 2 * f3 + f4);
    double a2 = fabs(f3 - f2) + fabs(f3 - 2 * f2 + f1);
    double b2 = fabs(f3 - f4) + fabs(f3 - 2 * f4 + f5);
    double s1 = (2 * a1 * b1 + eps) / (a1 * a1 + b1 * b1 + eps);
    double s2 = (2 * a2 * b2 + eps) / (a2 * a2 + b2 * b2 + eps);
    double s = s2 < s1 ? s2 : s1; /* std::min */
    if (s > 0.4) return orc_mdcd_linear(f, disp, diss);
    double q0 = (3 * f0 - 10 * f1 + 15 * f2) / 8.0;
    double q1 = (-f1 + 6 * f2 + 3 * f3) / 8.0;
    double q2 = (3 * f2 + 6 * f3 - f4) / 8.0;
    double q3 = (15 * f3 - 10 * f4 + 3 * f5) / 8.0;
    double d0 = 1.5 * (disp + diss);
    double d1 = 0.5 - 1.5 * (disp - 3 * diss);
    double d2 = 0.5 - 1.5 * (disp + 3 * diss);
    double d3 = 1.5 * (disp - diss);
    double be0 = 13.0 / 12.0 * sq(f0 - 2 * f1 + f2) + 0.25 * sq(f0 - 4 * f1 + 3 * f2);
    double be1 = 13.0 / 12.0 * sq(f1 - 2 * f2 + f3) + 0.25 * sq(f1 - f3);
    double be2 = 13.0 / 12.0 * sq(f2 - 2 * f3 + f4) + 0.25 * sq(3 * f2 - 4 * f3 + f4);
    double be3 = (271799 * sq(f0) +
                  f0 * (-2380800 * f1 + 4086352 * f2 - 3462252 * f3 + 1458762 * f4 - 245620 * f5) +
                  f1 * (5653317 * f1 - 20427884 * f2 + 17905032 * f3 - 7727988 * f4 + 1325006 * f5) +
                  f2 * (19510972 * f2 - 35817664 * f3 + 15929912 * f4 - 2792660 * f5) +
                  f3 * (17195652 * f3 - 15880404 * f4 + 2863984 * f5) + f4 * (3824847 * f4 - 1429976 * f5) +
                  139633 * sq(f5)) / 120960.0;
    double tau6 = fabs(be3 - (be0 + 4 * be1 + be2) / 6.0);
    double al0 = d0 * sq(20 + tau6 / (be0 + eps_small));
    double al1 = d1 * sq(20 + tau6 / (be1 + eps_small));
    double al2 = d2 * sq(20 + tau6 / (be2 + eps_small));
    double al3 = d3 * sq(20 + tau6 / (be3 + eps_small));
    return (al0 * q0 + al1 * q1 + al2 * q2 + al3 * q3) / (al0 + al1 + al2 + al3);
}

/* interpolate_select, interpolation.cpp:13-77: flag < 0 reverses the stencil. */
static double interp(const double v[6], int flag) {
    double a[6];
    for (int i = 0; i < 6; ++i) a[i] = flag < 0 ? v[5 - i] : v[i];
    switch (S->c.interpolation) {
        case ORC_WENO5: return orc_weno5(a);
        case ORC_MDCD_LINEAR: return orc_mdcd_linear(a, S->c.mdcd_disp, S->c.mdcd_diss);
        case ORC_MDCD_HYBRID: return orc_mdcd_hybrid(a, S->c.mdcd_disp, S->c.mdcd_diss);
        default: return v[0];
    }
}

/* ------------------------------------------------------ eigen-system (Roe) */

/* computeRoeAveragedState, InviscousFlux.cpp:849-884 (inputs are primitives). */
static void roe_avg(const double ul[5], const double ur[5], double g, double *rb, double *ub,
                    double *vb, double *wb, double *hb, double *ab) {
    double rL = ul[0], uL = ul[1], vL = ul[2], wL = ul[3], pL = ul[4];
    double EL = rL * (0.5 * (uL * uL + vL * vL + wL * wL) + pL / ((g - 1.0) * rL));
    double rR = ur[0], uR = ur[1], vR = ur[2], wR = ur[3], pR = ur[4];
    double ER = rR * (0.5 * (uR * uR + vR * vR + wR * wR) + pR / ((g - 1.0) * rR));
    double sL = sqrt(rL), sR = sqrt(rR);
    *rb = sL * sR;
    double den = 1.0 / (sL + sR);
    *ub = (sL * uL + sR * uR) * den;
    *vb = (sL * vL + sR * vR) * den;
    *wb = (sL * wL + sR * wR) * den;
    double HL = (EL + pL) / rL, HR = (ER + pR) / rR;
    *hb = (sL * HL + sR * HR) * den;
    double kin = 0.5 * (*ub * *ub + *vb * *vb + *wb * *wb);
    *ab = sqrt((g - 1.0) * (*hb - kin));
}

/* build_eigen_matrices, InviscousFlux.cpp:888-987 (Blazek form, sqrt(2) scaling). */
static void eigen(const double ul[5], const double ur[5], double nx, double ny, double nz, double g,
                  double L[5][5], double R[5][5], double lam[5]) {
    double rb, ub, vb, wb, Hb, c;
    roe_avg(ul, ur, g, &rb, &ub, &vb, &wb, &Hb, &c);
    double V = nx * ub + ny * vb + nz * wb;
    lam[0] = V - c; lam[1] = V; lam[2] = V; lam[3] = V; lam[4] = V + c;
    double phi = 0.5 * (g - 1.0) * (ub * ub + vb * vb + wb * wb);
    double a1 = g - 1.0;
    double a2 = 1.0 / (sqrt(2.0) * rb * c);
    double a3 = rb / (sqrt(2.0) * c);
    double a4 = (phi + c * c) / (g - 1.0);
    double a5 = 1.0 - phi / (c * c);
    double a6 = phi / (g - 1.0);
    L[0][0] = a2 * (phi + c * V);
    L[0][1] = -a2 * (a1 * ub + nx * c);
    L[0][2] = -a2 * (a1 * vb + ny * c);
    L[0][3] = -a2 * (a1 * wb + nz * c);
    L[0][4] = a1 * a2;
    L[1][0] = nx * a5 - (nz * vb - ny * wb) / rb;
    L[1][1] = nx * a1 * ub / (c * c);
    L[1][2] = nx * a1 * vb / (c * c) + nz / rb;
    L[1][3] = nx * a1 * wb / (c * c) - ny / rb;
    L[1][4] = -nx * a1 / (c * c);
    L[2][0] = nz * a5 - (ny * ub - nx * vb) / rb;
    L[2][1] = nz * a1 * ub / (c * c) + ny / rb;
    L[2][2] = nz * a1 * vb / (c * c) - nx / rb;
    L[2][3] = nz * a1 * wb / (c * c);
    L[2][4] = -nz * a1 / (c * c);
    L[3][0] = ny * a5 - (nx * wb - nz * ub) / rb;
    L[3][1] = ny * a1 * ub / (c * c) - nz / rb;
    L[3][2] = ny * a1 * vb / (c * c);
    L[3][3] = ny * a1 * wb / (c * c) + nx / rb;
    L[3][4] = -ny * a1 / (c * c);
    L[4][0] = a2 * (phi - c * V);
    L[4][1] = -a2 * (a1 * ub - nx * c);
    L[4][2] = -a2 * (a1 * vb - ny * c);
    L[4][3] = -a2 * (a1 * wb - nz * c);
    L[4][4] = a1 * a2;
    R[0][0] = a3; R[1][0] = a3 * (ub - nx * c); R[2][0] = a3 * (vb - ny * c);
    R[3][0] = a3 * (wb - nz * c); R[4][0] = a3 * (a4 - c * V);
    R[0][1] = nx; R[1][1] = nx * ub; R[2][1] = nx * vb + nz * rb; R[3][1] = nx * wb - ny * rb;
    R[4][1] = nx * a6 + rb * (nz * vb - ny * wb);
    R[0][2] = nz; R[1][2] = nz * ub + ny * rb; R[2][2] = nz * vb - nx * rb; R[3][2] = nz * wb;
    R[4][2] = nz * a6 + rb * (ny * ub - nx * vb);
    R[0][3] = ny; R[1][3] = ny * ub - nz * rb; R[2][3] = ny * vb; R[3][3] = ny * wb + nx * rb;
    R[4][3] = ny * a6 + rb * (nx * wb - nz * ub);
    R[0][4] = a3; R[1][4] = a3 * (ub + nx * c); R[2][4] = a3 * (vb + ny * c);
    R[3][4] = a3 * (wb + nz * c); R[4][4] = a3 * (a4 + c * V);
}

/* ----------------------------------------------------------- Riemann solvers */

typedef struct { double r, u, v, w, E, p, a, un; } side_t;

static inline side_t side(const double U[5], double nx, double ny, double nz, double g) {
    side_t s;
    s.r = U[0]; s.u = U[1] / s.r; s.v = U[2] / s.r; s.w = U[3] / s.r; s.E = U[4];
    s.p = (U[4] - 0.5 * s.r * (s.u * s.u + s.v * s.v + s.w * s.w)) * (g - 1.0);
    s.a = sqrt(g * s.p / s.r);
    s.un = s.u * nx + s.v * ny + s.w * nz;
    return s;
}

static inline void phys_flux(const side_t *s, double nx, double ny, double nz, double F[5]) {
    F[0] = s->r * s->un;
    F[1] = s->r * s->u * s->un + s->p * nx;
    F[2] = s->r * s->v * s->un + s->p * ny;
    F[3] = s->r * s->w * s->un + s->p * nz;
    F[4] = (s->E + s->p) * s->un;
}

/* Rusanov_Riemann_solver, InviscousFlux.cpp:270-311. */
static void rusanov(const double UL[5], const double UR[5], double nx, double ny, double nz, double g,
                    double F[5]) {
    side_t L = side(UL, nx, ny, nz, g), R = side(UR, nx, ny, nz, g);
    double FL[5], FR[5];
    phys_flux(&L, nx, ny, nz, FL);
    phys_flux(&R, nx, ny, nz, FR);
    double sl = fabs(L.u * nx + L.v * ny + L.w * nz) + L.a;
    double sr = fabs(R.u * nx + R.v * ny + R.w * nz) + R.a;
    double smax = sl < sr ? sr : sl; /* std::max */
    for (int n = 0; n < 5; ++n) F[n] = 0.5 * (FL[n] + FR[n]) - 0.5 * smax * (UR[n] - UL[n]);
}

/* Roe_Riemann_solver, InviscousFlux.cpp:313-382. */
static void roe(const double UL[5], const double UR[5], double nx, double ny, double nz, double g,
                double F[5]) {
    side_t L = side(UL, nx, ny, nz, g), R = side(UR, nx, ny, nz, g);
    double FL[5], FR[5];
    phys_flux(&L, nx, ny, nz, FL);
    phys_flux(&R, nx, ny, nz, FR);
    const double ul[5] = {L.r, L.u, L.v, L.w, L.p};
    const double ur[5] = {R.r, R.u, R.v, R.w, R.p};
    double Lm[5][5], Rm[5][5], lam[5];
    eigen(ul, ur, nx, ny, nz, g, Lm, Rm, lam);
    double alpha[5];
    for (int m = 0; m < 5; ++m) {
        alpha[m] = 0.0;
        for (int n = 0; n < 5; ++n) alpha[m] += Lm[m][n] * (UR[n] - UL[n]);
    }
    double mx = 0.0;
    for (int m = 0; m < 5; ++m) { double a = fabs(lam[m]); mx = mx < a ? a : mx; }
    double delta = 0.1 * mx;
    for (int m = 0; m < 5; ++m)
        if (fabs(lam[m]) < delta) lam[m] = (lam[m] * lam[m] + delta * delta) / (2.0 * delta);
    for (int n = 0; n < 5; ++n) {
        F[n] = 0.5 * (FL[n] + FR[n]);
        for (int m = 0; m < 5; ++m) F[n] -= 0.5 * fabs(lam[m]) * alpha[m] * Rm[n][m];
    }
}

/* HLL_Riemann_solver, InviscousFlux.cpp:384-447 (Davis wave speeds). */
static void hll(const double UL[5], const double UR[5], double nx, double ny, double nz, double g,
                double F[5]) {
    side_t L = side(UL, nx, ny, nz, g), R = side(UR, nx, ny, nz, g);
    double FL[5], FR[5];
    phys_flux(&L, nx, ny, nz, FL);
    phys_flux(&R, nx, ny, nz, FR);
    double a = L.un - L.a, b = R.un - R.a;
    double SL = b < a ? b : a;
    a = L.un + L.a; b = R.un + R.a;
    double SR = a < b ? b : a;
    if (SL >= 0.0) { for (int i = 0; i < 5; ++i) F[i] = FL[i]; }
    else if (SR <= 0.0) { for (int i = 0; i < 5; ++i) F[i] = FR[i]; }
    else {
        double den = SR - SL, f1 = SR / den, f2 = SL / den, f3 = SL * SR / den;
        for (int i = 0; i < 5; ++i) F[i] = (f1 * FL[i] - f2 * FR[i] + f3 * (UR[i] - UL[i]));
    }
}

/* HLLC star-state flux shared by HLLC and HLLC_p, InviscousFlux.cpp:537-591, 663-715. */
static void hllc_star(const side_t *L, const side_t *R, const double UL[5], const double UR[5],
                      const double FL[5], const double FR[5], double SL, double SR, double SM,
                      double nx, double ny, double nz, double F[5]) {
    if (SM >= 0.0) {
        double rs = L->r * (SL - L->un) / (SL - SM);
        double tx = L->u - L->un * nx, ty = L->v - L->un * ny, tz = L->w - L->un * nz;
        double ux = SM * nx + tx, uy = SM * ny + ty, uz = SM * nz + tz;
        double Es = L->E / L->r + (SM - L->un) * (SM + L->p / (L->r * (SL - L->un)));
        double Us[5] = {rs, rs * ux, rs * uy, rs * uz, rs * Es};
        for (int i = 0; i < 5; ++i) F[i] = FL[i] + SL * (Us[i] - UL[i]);
    } else {
        double rs = R->r * (SR - R->un) / (SR - SM);
        double tx = R->u - R->un * nx, ty = R->v - R->un * ny, tz = R->w - R->un * nz;
        double ux = SM * nx + tx, uy = SM * ny + ty, uz = SM * nz + tz;
        double Es = R->E / R->r + (SM - R->un) * (SM + R->p / (R->r * (SR - R->un)));
        double Us[5] = {rs, rs * ux, rs * uy, rs * uz, rs * Es};
        for (int i = 0; i < 5; ++i) F[i] = FR[i] + SR * (Us[i] - UR[i]);
    }
}

/* HLLC_Riemann_solver, InviscousFlux.cpp:449-592 (Davis S_L/S_R, Batten S_M). */
static void hllc(const double UL[5], const double UR[5], double nx, double ny, double nz, double g,
                 double F[5]) {
    side_t L = side(UL, nx, ny, nz, g), R = side(UR, nx, ny, nz, g);
    double FL[5], FR[5];
    phys_flux(&L, nx, ny, nz, FL);
    phys_flux(&R, nx, ny, nz, FR);
    double a = L.un - L.a, b = R.un - R.a;
    double SL = b < a ? b : a;
    a = L.un + L.a; b = R.un + R.a;
    double SR = a < b ? b : a;
    if (SL >= 0.0) { for (int i = 0; i < 5; ++i) F[i] = FL[i]; return; }
    if (SR <= 0.0) { for (int i = 0; i < 5; ++i) F[i] = FR[i]; return; }
    double sL = sqrt(L.r), sR = sqrt(R.r), ssum = sL + sR;
    double ur = (sL * L.u + sR * R.u) / ssum;
    double vr = (sL * L.v + sR * R.v) / ssum;
    double wr = (sL * L.w + sR * R.w) / ssum;
    double unr = ur * nx + vr * ny + wr * nz;
    double SM;
    double num = R.r * R.un * (SR - R.un) - L.r * L.un * (SL - L.un) + L.p - R.p;
    double den = R.r * (SR - R.un) - L.r * (SL - L.un);
    if (fabs(den) > 1e-12) SM = num / den; else SM = unr;
    hllc_star(&L, &R, UL, UR, FL, FR, SL, SR, SM, nx, ny, nz, F);
}

/* HLLC_p_Riemann_solver, InviscousFlux.cpp:594-717 (PVRS p*, Toro speeds). */
static void hllc_p(const double UL[5], const double UR[5], double nx, double ny, double nz, double g,
                   double F[5]) {
    side_t L = side(UL, nx, ny, nz, g), R = side(UR, nx, ny, nz, g);
    double FL[5], FR[5];
    phys_flux(&L, nx, ny, nz, FL);
    phys_flux(&R, nx, ny, nz, FR);
    double ps = 0.5 * (L.p + R.p) - 0.125 * (R.un - L.un) * (L.r + R.r) * (L.a + R.a);
    ps = (0.0 < ps) ? ps : 0.0; /* std::max(0.0, p_star) */
    double SL, SR;
    if (ps <= L.p) SL = L.un - L.a;
    else SL = L.un - L.a * sqrt((g + 1.0) * ps / (2.0 * g * L.p) + (g - 1.0) / (2.0 * g));
    if (ps <= R.p) SR = R.un + R.a;
    else SR = R.un + R.a * sqrt((g + 1.0) * ps / (2.0 * g * R.p) + (g - 1.0) / (2.0 * g));
    if (SL >= 0.0) { for (int i = 0; i < 5; ++i) F[i] = FL[i]; return; }
    if (SR <= 0.0) { for (int i = 0; i < 5; ++i) F[i] = FR[i]; return; }
    double SM = (R.p - L.p + L.r * L.un * (SL - L.un) - R.r * R.un * (SR - R.un)) /
                (L.r * (SL - L.un) - R.r * (SR - R.un));
    hllc_star(&L, &R, UL, UR, FL, FR, SL, SR, SM, nx, ny, nz, F);
}

static inline double m4p(double M) { return fabs(M) >= 1.0 ? 0.5 * (M + fabs(M)) : 0.25 * (M + 1.0) * (M + 1.0); }
static inline double m4m(double M) { return fabs(M) >= 1.0 ? 0.5 * (M - fabs(M)) : -0.25 * (M - 1.0) * (M - 1.0); }
static inline double p5p(double M) {
    return fabs(M) >= 1.0 ? 0.5 * (1.0 + (M > 0 ? 1.0 : -1.0)) : 0.25 * (M + 1.0) * (M + 1.0) * (2.0 - M);
}
static inline double p5m(double M) {
    return fabs(M) >= 1.0 ? 0.5 * (1.0 - (M > 0 ? 1.0 : -1.0)) : 0.25 * (M - 1.0) * (M - 1.0) * (2.0 + M);
}

/* AUSM_Riemann_solver, InviscousFlux.cpp:719-846 (AUSM+-up style, Kp=.25, Ku=.75). */
static void ausm(const double UL[5], const double UR[5], double nx, double ny, double nz, double g,
                 double F[5]) {
    const double Kp = 0.25, Ku = 0.75;
    double rL = UL[0], uL = UL[1] / rL, vL = UL[2] / rL, wL = UL[3] / rL, EL = UL[4];
    double pL = (EL - 0.5 * rL * (uL * uL + vL * vL + wL * wL)) * (g - 1.0);
    pL = pL < 1e-12 ? 1e-12 : pL;
    double aL = sqrt(g * pL / rL), HL = (EL + pL) / rL;
    double rR = UR[0], uR = UR[1] / rR, vR = UR[2] / rR, wR = UR[3] / rR, ER = UR[4];
    double pR = (ER - 0.5 * rR * (uR * uR + vR * vR + wR * wR)) * (g - 1.0);
    pR = pR < 1e-12 ? 1e-12 : pR;
    double aR = sqrt(g * pR / rR), HR = (ER + pR) / rR;
    double unL = uL * nx + vL * ny + wL * nz, unR = uR * nx + vR * ny + wR * nz;
    double ab = 0.5 * (aL + aR), rb = 0.5 * (rL + rR);
    double ML = unL / ab, MR = unR / ab;
    double Mb2 = (unL * unL + unR * unR) / (2.0 * ab * ab);
    double t = Mb2 < 0.5 ? 0.5 : Mb2;       /* std::max(M_bar2, 0.5) */
    double Mo2 = t < 1.0 ? t : 1.0;         /* std::min(1.0, .) */
    double fa = Mo2 * (2.0 - Mo2);
    double Mp = m4p(ML), Mm = m4m(MR);
    double om = 1.0 - Mb2;
    om = om < 0.0 ? 0.0 : om;
    double Mh = Mp + Mm - Kp / fa * om * ((pR - pL) / (rb * ab * ab));
    double md = ab * Mh * (Mh >= 0.0 ? rL : rR);
    double pp = p5p(ML), pm = p5m(MR);
    double ph = pp * pL + pm * pR - Ku * pm * pp * (rL + rR) * fa * (uR - uL) * ab;
    double uf, vf, wf, Hf;
    if (md >= 0.0) { uf = uL; vf = vL; wf = wL; Hf = HL; }
    else { uf = uR; vf = vR; wf = wR; Hf = HR; }
    F[0] = md;
    F[1] = md * uf + ph * nx;
    F[2] = md * vf + ph * ny;
    F[3] = md * wf + ph * nz;
    F[4] = md * Hf;
}

void orc_riemann(int solver, const double UL[5], const double UR[5], int dir, double g, double F[5]) {
    double nx = dir == 0 ? 1.0 : 0.0, ny = dir == 1 ? 1.0 : 0.0, nz = dir == 2 ? 1.0 : 0.0;
    switch (solver) {
        case ORC_ROE: roe(UL, UR, nx, ny, nz, g, F); break;
        case ORC_RUSANOV: rusanov(UL, UR, nx, ny, nz, g, F); break;
        case ORC_HLLC: hllc(UL, UR, nx, ny, nz, g, F); break;
        case ORC_HLL: hll(UL, UR, nx, ny, nz, g, F); break;
        case ORC_HLLC_P: hllc_p(UL, UR, nx, ny, nz, g, F); break;
        case ORC_AUSM: ausm(UL, UR, nx, ny, nz, g, F); break;
        default: for (int n = 0; n < 5; ++n) F[n] = 0.0;
    }
}

/* ---------------------------------------------------------- inviscid flux */

/* WCNS_Riemann_InviscidFlux, InviscousFlux.cpp:146-268.
 * Ut[n][m]: conserved stencil, ut[n][m]: primitive stencil, m = cell i-2 .. i+3. */
static void face_flux(const double Ut[5][6], const double ut[5][6], int dir, double F[5]) {
    const double g = S->c.gamma;
    double nx = dir == 0 ? 1.0 : 0.0, ny = dir == 1 ? 1.0 : 0.0, nz = dir == 2 ? 1.0 : 0.0;
    double UL[5], UR[5];
    if (S->c.char_recon) {
        double Lm[5][5], Rm[5][5], lam[5], LU[5][6], Q[5];
        for (int side_ = 0; side_ < 2; ++side_) {
            const int m0 = side_ == 0 ? 2 : 3; /* cell i for UL, cell i+1 for UR */
            const double st[5] = {ut[0][m0], ut[1][m0], ut[2][m0], ut[3][m0], ut[4][m0]};
            eigen(st, st, nx, ny, nz, g, Lm, Rm, lam);
            for (int m = 0; m < 6; ++m)
                for (int n = 0; n < 5; ++n) {
                    double s = 0.0;
                    for (int r = 0; r < 5; ++r) s += Lm[n][r] * Ut[r][m];
                    LU[n][m] = s;
                }
            for (int n = 0; n < 5; ++n) Q[n] = interp(LU[n], side_ == 0 ? +1 : -1);
            for (int n = 0; n < 5; ++n) {
                double s = 0.0;
                for (int r = 0; r < 5; ++r) s += Rm[n][r] * Q[r];
                if (side_ == 0) UL[n] = s; else UR[n] = s;
            }
        }
    } else {
        for (int n = 0; n < 5; ++n) {
            UL[n] = interp(Ut[n], +1);
            UR[n] = interp(Ut[n], -1);
        }
    }
    orc_riemann(S->c.riemann, UL, UR, dir, g, F);
}

static void gather_stencil(int i, int j, int k, int dir, double Ut[5][6], double ut[5][6]) {
    for (int m = 0; m < 6; ++m) {
        int o = m - 2;
        long id = dir == 0 ? I3(i + o, j, k) : dir == 1 ? I3(i, j + o, k) : I3(i, j, k + o);
        for (int n = 0; n < 5; ++n) Ut[n][m] = S->U[n][id];
        ut[0][m] = S->U[0][id];
        for (int n = 1; n < 5; ++n) ut[n][m] = S->W[n][id];
    }
}

/* compute_invis_flux, InviscousFlux.cpp:10-144: faces ng-1 .. ng+n-1 on interior lines. */
static void invis_flux(void) {
    const int nx = S->nx, ny = S->ny, nz = S->nz;
    double Ut[5][6], ut[5][6], F[5];
    for (int k = NG; k < NG + nz; ++k)
        for (int j = NG; j < NG + ny; ++j)
            for (int i = NG - 1; i < NG + nx; ++i) {
                gather_stencil(i, j, k, 0, Ut, ut);
                face_flux(Ut, ut, 0, F);
                for (int n = 0; n < 5; ++n) S->FX[n][IFX(i, j, k)] = F[n];
            }
    for (int k = NG; k < NG + nz; ++k)
        for (int i = NG; i < NG + nx; ++i)
            for (int j = NG - 1; j < NG + ny; ++j) {
                gather_stencil(i, j, k, 1, Ut, ut);
                face_flux(Ut, ut, 1, F);
                for (int n = 0; n < 5; ++n) S->FY[n][IFY(i, j, k)] = F[n];
            }
    for (int i = NG; i < NG + nx; ++i)
        for (int j = NG; j < NG + ny; ++j)
            for (int k = NG - 1; k < NG + nz; ++k) {
                gather_stencil(i, j, k, 2, Ut, ut);
                face_flux(Ut, ut, 2, F);
                for (int n = 0; n < 5; ++n) S->FZ[n][IFZ(i, j, k)] = F[n];
            }
}

/* apply_boundary_halfnode_flux, boundary.cpp:207-300 and
 * exchange_halos_halfnode_flux, field_structures.h:773-874, 998-1056:
 * periodic dims get wrapped faces (0,1 <- n,n+1; n+3,n+4 <- 3,4) on interior
 * tangential lines; Outflow copies the boundary face over full extents;
 * Wall/Symmetry/Inflow leave the ghost faces untouched. */
static void halfnode_boundary(void) {
    const int nx = S->nx, ny = S->ny, nz = S->nz, sx = S->sx, sy = S->sy, sz = S->sz;
    if (S->periodic[0])
        for (int k = NG; k < NG + nz; ++k)
            for (int j = NG; j < NG + ny; ++j)
                for (int g = 0; g < NG - 1; ++g)
                    for (int n = 0; n < 5; ++n) {
                        S->FX[n][IFX(g, j, k)] = S->FX[n][IFX(nx + g, j, k)];
                        S->FX[n][IFX(NG + nx + g, j, k)] = S->FX[n][IFX(NG + g, j, k)];
                    }
    if (S->periodic[1])
        for (int k = NG; k < NG + nz; ++k)
            for (int i = NG; i < NG + nx; ++i)
                for (int g = 0; g < NG - 1; ++g)
                    for (int n = 0; n < 5; ++n) {
                        S->FY[n][IFY(i, g, k)] = S->FY[n][IFY(i, ny + g, k)];
                        S->FY[n][IFY(i, NG + ny + g, k)] = S->FY[n][IFY(i, NG + g, k)];
                    }
    if (S->periodic[2])
        for (int i = NG; i < NG + nx; ++i)
            for (int j = NG; j < NG + ny; ++j)
                for (int g = 0; g < NG - 1; ++g)
                    for (int n = 0; n < 5; ++n) {
                        S->FZ[n][IFZ(i, j, g)] = S->FZ[n][IFZ(i, j, nz + g)];
                        S->FZ[n][IFZ(i, j, NG + nz + g)] = S->FZ[n][IFZ(i, j, NG + g)];
                    }
    for (int face = 0; face < 6; ++face) {
        int d = face / 2, hi = face % 2;
        if (S->periodic[d] || S->c.bc[face] != ORC_OUTFLOW) continue;
        for (int k = 0; k < sz; ++k)
            for (int j = 0; j < sy; ++j)
                for (int i = 0; i < sx; ++i) {
                    int c[3] = {i, j, k};
                    int ext = d == 0 ? sx : d == 1 ? sy : sz;
                    int x = c[d], src;
                    if (!hi) { if (x >= NG - 1) continue; src = NG - 1; }
                    else { if (x < ext - NG || x >= ext - 1) continue; src = ext - NG - 1; }
                    int s[3] = {i, j, k};
                    s[d] = src;
                    for (int n = 0; n < 5; ++n) {
                        if (d == 0) S->FX[n][IFX(i, j, k)] = S->FX[n][IFX(s[0], s[1], s[2])];
                        else if (d == 1) S->FY[n][IFY(i, j, k)] = S->FY[n][IFY(s[0], s[1], s[2])];
                        else S->FZ[n][IFZ(i, j, k)] = S->FZ[n][IFZ(s[0], s[1], s[2])];
                    }
                }
    }
}

/* diff_6th_central_half, InviscousFlux.cpp:990-992; faces i-3..i+2 around cell i (:996-1005). */
static inline double dhalf(const double f[6], double h) {
    return ((f[3] - f[2]) * (75.0 / 64.0) + (f[4] - f[1]) * (-25.0 / 384.0) + (f[5] - f[0]) * (3.0 / 640.0)) / h;
}

/* compute_invis_dflux, InviscousFlux.cpp:1027-1056: x, y, z differences per variable. */
static void invis_dflux(void) {
    const int nx = S->nx, ny = S->ny, nz = S->nz;
    double f[6];
    for (int k = NG; k < NG + nz; ++k)
        for (int j = NG; j < NG + ny; ++j)
            for (int i = NG; i < NG + nx; ++i) {
                long id = I3(i, j, k);
                for (int n = 0; n < 5; ++n) {
                    for (int q = 0; q < 6; ++q) f[q] = S->FX[n][IFX(i + q - 3, j, k)];
                    S->R[n][id] -= dhalf(f, S->dx);
                    for (int q = 0; q < 6; ++q) f[q] = S->FY[n][IFY(i, j + q - 3, k)];
                    S->R[n][id] -= dhalf(f, S->dy);
                    for (int q = 0; q < 6; ++q) f[q] = S->FZ[n][IFZ(i, j, k + q - 3)];
                    S->R[n][id] -= dhalf(f, S->dz);
                }
            }
}

/* ------------------------------------------------------------ viscous terms */

/* choose_scheme, ViscousFlux.cpp:33-50. */
static inline int choose(int idx, int n0, int n1, int periodic) {
    if (periodic) return 6;
    int dl = idx - n0;
    if (dl == 0) return 1;
    int dr = (n1 - 1) - idx;
    if (dr == 0) return -1;
    int dm = dl < dr ? dl : dr;
    return dm == 1 ? 2 : dm == 2 ? 4 : 6;
}

/* diff_x/y/z stencils, ViscousFlux.cpp:15-104 (7 points, centre at index 3).
 * order +-1 is the one-sided 2nd-order form; at the right boundary it yields
 * -df/dx, reproduced as in the reference. */
static inline double dstencil(const double f[7], double h, int order) {
    if (order == 1 || order == -1)
        return (-3.0 * f[3] + 4.0 * f[3 + order] - f[3 + 2 * order]) / (2.0 * h);
    if (order == 2) return (f[4] - f[2]) / (2.0 * h);
    if (order == 4) return (-f[5] + 8.0 * f[4] - 8.0 * f[2] + f[1]) / (12.0 * h);
    return (f[6] - 9.0 * f[5] + 45.0 * f[4] - 45.0 * f[2] + 9.0 * f[1] - f[0]) / (60.0 * h);
}

static inline double dgrad(const double *a, int i, int j, int k, int dir, double h, int order) {
    double f[7];
    for (int q = 0; q < 7; ++q) {
        int o = q - 3;
        f[q] = a[dir == 0 ? I3(i + o, j, k) : dir == 1 ? I3(i, j + o, k) : I3(i, j, k + o)];
    }
    return dstencil(f, h, order);
}

/* compute_gradients, ViscousFlux.cpp:109-148. */
static void gradients(void) {
    const int nx = S->nx, ny = S->ny, nz = S->nz;
    const double *fld[4] = {S->W[1], S->W[2], S->W[3], S->T};
    for (int k = NG; k < NG + nz; ++k)
        for (int j = NG; j < NG + ny; ++j)
            for (int i = NG; i < NG + nx; ++i) {
                long id = I3(i, j, k);
                int ox = choose(i, NG, NG + nx, S->periodic[0]);
                int oy = choose(j, NG, NG + ny, S->periodic[1]);
                int oz = choose(k, NG, NG + nz, S->periodic[2]);
                for (int q = 0; q < 4; ++q) {
                    S->G[3 * q + 0][id] = dgrad(fld[q], i, j, k, 0, S->dx, ox);
                    S->G[3 * q + 1][id] = dgrad(fld[q], i, j, k, 1, S->dy, oy);
                    S->G[3 * q + 2][id] = dgrad(fld[q], i, j, k, 2, S->dz, oz);
                }
            }
}

/* compute_viscous_flux, ViscousFlux.cpp:151-208 and SolverParams::get_mu
 * (Sutherland), field_structures.h:96-106. */
static void viscous_flux(void) {
    const int nx = S->nx, ny = S->ny, nz = S->nz;
    const double Sr = S->c.sutherland_s;
    for (int k = NG; k < NG + nz; ++k)
        for (int j = NG; j < NG + ny; ++j)
            for (int i = NG; i < NG + nx; ++i) {
                long id = I3(i, j, k);
                double T = S->T[id];
                double mu = S->mu * pow(T, 1.5) * (1.0 + Sr) / (T + Sr);
                double ux = S->G[0][id], uy = S->G[1][id], uz = S->G[2][id];
                double vx = S->G[3][id], vy = S->G[4][id], vz = S->G[5][id];
                double wx = S->G[6][id], wy = S->G[7][id], wz = S->G[8][id];
                double Tx = S->G[9][id], Ty = S->G[10][id], Tz = S->G[11][id];
                double divU = ux + vy + wz;
                double txx = 2.0 * mu * ux - (2.0 / 3.0) * mu * divU;
                double tyy = 2.0 * mu * vy - (2.0 / 3.0) * mu * divU;
                double tzz = 2.0 * mu * wz - (2.0 / 3.0) * mu * divU;
                double txy = mu * (uy + vx), txz = mu * (uz + wx), tyz = mu * (vz + wy);
                double qx = mu * S->Cp / S->c.Pr * Tx;
                double qy = mu * S->Cp / S->c.Pr * Ty;
                double qz = mu * S->Cp / S->c.Pr * Tz;
                double u = S->W[1][id], v = S->W[2][id], w = S->W[3][id];
                S->V[0][id] = txx; S->V[1][id] = txy; S->V[2][id] = txz;
                S->V[3][id] = u * txx + v * txy + w * txz + qx;
                S->V[4][id] = txy; S->V[5][id] = tyy; S->V[6][id] = tyz;
                S->V[7][id] = u * txy + v * tyy + w * tyz + qy;
                S->V[8][id] = txz; S->V[9][id] = tyz; S->V[10][id] = tzz;
                S->V[11][id] = u * txz + v * tyz + w * tzz + qz;
            }
}

/* exchange_halos_viscous_flux, field_structures.h:651-770, 877-932: wrapped
 * node viscous fluxes in periodic dims over interior tangential extents. */
static void exchange_viscous(void) {
    const int nx = S->nx, ny = S->ny, nz = S->nz;
    for (int q = 0; q < 12; ++q) {
        double *a = S->V[q];
        if (S->periodic[0])
            for (int k = NG; k < NG + nz; ++k)
                for (int j = NG; j < NG + ny; ++j)
                    for (int g = 0; g < NG; ++g) {
                        a[I3(g, j, k)] = a[I3(g + nx, j, k)];
                        a[I3(NG + nx + g, j, k)] = a[I3(NG + g, j, k)];
                    }
        if (S->periodic[1])
            for (int k = NG; k < NG + nz; ++k)
                for (int g = 0; g < NG; ++g)
                    for (int i = NG; i < NG + nx; ++i) {
                        a[I3(i, g, k)] = a[I3(i, g + ny, k)];
                        a[I3(i, NG + ny + g, k)] = a[I3(i, NG + g, k)];
                    }
        if (S->periodic[2])
            for (int g = 0; g < NG; ++g)
                for (int j = NG; j < NG + ny; ++j)
                    for (int i = NG; i < NG + nx; ++i) {
                        a[I3(i, j, g)] = a[I3(i, j, g + nz)];
                        a[I3(i, j, NG + nz + g)] = a[I3(i, j, NG + g)];
                    }
    }
}

/* compute_vis_flux, ViscousFlux.cpp:210-255 (mass skipped). */
static void vis_divergence(void) {
    const int nx = S->nx, ny = S->ny, nz = S->nz;
    for (int k = NG; k < NG + nz; ++k)
        for (int j = NG; j < NG + ny; ++j)
            for (int i = NG; i < NG + nx; ++i) {
                long id = I3(i, j, k);
                int ox = choose(i, NG, NG + nx, S->periodic[0]);
                int oy = choose(j, NG, NG + ny, S->periodic[1]);
                int oz = choose(k, NG, NG + nz, S->periodic[2]);
                for (int n = 0; n < 4; ++n) {
                    S->R[1 + n][id] += dgrad(S->V[n], i, j, k, 0, S->dx, ox);
                    S->R[1 + n][id] += dgrad(S->V[4 + n], i, j, k, 1, S->dy, oy);
                    S->R[1 + n][id] += dgrad(S->V[8 + n], i, j, k, 2, S->dz, oz);
                }
            }
}

/* compute_rhs, range_kutta.cpp:11-43. */
void orc_compute_rhs(void) {
    for (int n = 0; n < 5; ++n) memset(S->R[n], 0, sizeof(double) * (size_t)S->ncell);
    invis_flux();
    halfnode_boundary();
    invis_dflux();
    gradients();
    viscous_flux();
    exchange_viscous();
    vis_divergence();
}

/* recordConservedTo0 (field_structures.h:491-497) + runge_kutta_3
 * (range_kutta.cpp:46-92): stage updates over all cells, then c2p, boundary,
 * p2c after every stage. */
void orc_rk3_step(double dt) {
    for (int n = 0; n < 5; ++n) memcpy(S->U0[n], S->U[n], sizeof(double) * (size_t)S->ncell);
    for (int stage = 0; stage < 3; ++stage) {
        orc_compute_rhs();
        for (int n = 0; n < 5; ++n) {
            double *u = S->U[n], *u0 = S->U0[n], *r = S->R[n];
            for (long id = 0; id < S->ncell; ++id) {
                if (stage == 0) u[id] = u0[id] + dt * r[id];
                else if (stage == 1) u[id] = 0.75 * u0[id] + 0.25 * (u[id] + dt * r[id]);
                else u[id] = (1.0 / 3.0) * u0[id] + (2.0 / 3.0) * (u[id] + dt * r[id]);
            }
        }
        orc_cons_to_prim();
        orc_apply_boundary();
        orc_prim_to_cons();
    }
}

/* compute_timestep, timestep.cpp:5-23: x-direction CFL with |u| only. */
double orc_timestep(void) {
    double dtl = 1e9;
    const double g = S->c.gamma;
    for (int k = NG; k < NG + S->nz; ++k)
        for (int j = NG; j < NG + S->ny; ++j)
            for (int i = NG; i < NG + S->nx; ++i) {
                long id = I3(i, j, k);
                double rho = S->U[0][id];
                double u = S->U[1][id] / rho;
                double p = (g - 1.) * (S->U[4][id] - 0.5 * rho * u * u);
                double a = sqrt(g * p / rho);
                double c = S->dx / (fabs(u) + a);
                dtl = c < dtl ? c : dtl;
            }
    return S->c.cfl * dtl;
}

/* compute_total_energy, postprocess.cpp:103-128: sum of 0.5 rho |u|^2 dV
 * over the interior (internal energy deliberately 0). */
double orc_total_energy(void) {
    const double vol = S->dx * S->dy * S->dz;
    double sum = 0.0;
    for (int k = NG; k < NG + S->nz; ++k)
        for (int j = NG; j < NG + S->ny; ++j)
            for (int i = NG; i < NG + S->nx; ++i) {
                long id = I3(i, j, k);
                double rho = S->U[0][id], u = S->W[1][id], v = S->W[2][id], w = S->W[3][id];
                double kinetic = 0.5 * rho * (u * u + v * v + w * w);
                double eint = 0;
                sum += (kinetic + eint) * vol;
            }
    return sum;
}

/* compute_diagnostics, postprocess.cpp:7-98, with updateResiduals
 * (field_structures.h:500-508): per conserved variable sqrt(sum over the
 * interior of (U - U0)^2 dx^3) / max |U|, U0 the state recorded at the start
 * of the last step (orc_rk3_step).  Same loop and operation order. */
void orc_residuals(double out[5]) {
    const double dx3 = S->dx * S->dx * S->dx;
    double sq[5] = {0, 0, 0, 0, 0}, mx[5] = {0, 0, 0, 0, 0};
    for (int k = NG; k < NG + S->nz; ++k)
        for (int j = NG; j < NG + S->ny; ++j)
            for (int i = NG; i < NG + S->nx; ++i) {
                long id = I3(i, j, k);
                for (int n = 0; n < 5; ++n) {
                    double a = fabs(S->U[n][id]);
                    mx[n] = mx[n] < a ? a : mx[n];  /* std::max(max_abs, |x|) */
                }
                for (int n = 0; n < 5; ++n) {
                    double r = S->U[n][id] - S->U0[n][id];
                    sq[n] += r * r * dx3;
                }
            }
    for (int n = 0; n < 5; ++n) out[n] = sqrt(sq[n]) / mx[n];
}

/* main.cpp:98-99 after an initialiser: interior primitives -> ghosts -> conserved. */
int orc_set_interior_prims(const double *rho, const double *u, const double *v, const double *w,
                           const double *p) {
    if (!S) return -1;
    long n = 0;
    for (int k = 0; k < S->nz; ++k)
        for (int j = 0; j < S->ny; ++j)
            for (int i = 0; i < S->nx; ++i, ++n) {
                long id = I3(i + NG, j + NG, k + NG);
                S->U[0][id] = rho[n]; S->W[1][id] = u[n]; S->W[2][id] = v[n];
                S->W[3][id] = w[n]; S->W[4][id] = p[n];
            }
    orc_apply_boundary();
    orc_prim_to_cons();
    return 0;
}

/* ------------------------------------------------------------- field access */

static double *by_name(const char *name, long *count) {
    static const char *cn[] = {"rho", "rhou", "rhov", "rhow", "E"};
    static const char *c0[] = {"rho0", "rhou0", "rhov0", "rhow0", "E0"};
    static const char *rn[] = {"rhs_rho", "rhs_rhou", "rhs_rhov", "rhs_rhow", "rhs_E"};
    static const char *pn[] = {"u", "v", "w", "p"};
    static const char *fx[] = {"flux_fx_mass", "flux_fx_momx", "flux_fx_momy", "flux_fx_momz", "flux_fx_E"};
    static const char *fy[] = {"flux_fy_mass", "flux_fy_momx", "flux_fy_momy", "flux_fy_momz", "flux_fy_E"};
    static const char *fz[] = {"flux_fz_mass", "flux_fz_momx", "flux_fz_momy", "flux_fz_momz", "flux_fz_E"};
    static const char *gn[] = {"du_dx", "du_dy", "du_dz", "dv_dx", "dv_dy", "dv_dz",
                               "dw_dx", "dw_dy", "dw_dz", "dT_dx", "dT_dy", "dT_dz"};
    static const char *vn[] = {"Fvflux_momx", "Fvflux_momy", "Fvflux_momz", "Fvflux_E",
                               "Hvflux_momx", "Hvflux_momy", "Hvflux_momz", "Hvflux_E",
                               "Gvflux_momx", "Gvflux_momy", "Gvflux_momz", "Gvflux_E"};
    *count = S->ncell;
    for (int n = 0; n < 5; ++n) {
        if (!strcmp(name, cn[n])) return S->U[n];
        if (!strcmp(name, c0[n])) return S->U0[n];
        if (!strcmp(name, rn[n])) return S->R[n];
    }
    for (int n = 0; n < 4; ++n)
        if (!strcmp(name, pn[n])) return S->W[1 + n];
    if (!strcmp(name, "T")) return S->T;
    for (int n = 0; n < 12; ++n) {
        if (!strcmp(name, gn[n])) return S->G[n];
        if (!strcmp(name, vn[n])) return S->V[n];
    }
    for (int n = 0; n < 5; ++n) {
        if (!strcmp(name, fx[n])) { *count = S->nfx; return S->FX[n]; }
        if (!strcmp(name, fy[n])) { *count = S->nfy; return S->FY[n]; }
        if (!strcmp(name, fz[n])) { *count = S->nfz; return S->FZ[n]; }
    }
    return NULL;
}

long orc_get(const char *name, double *dst, long cap) {
    long n;
    if (!S) return -1;
    double *a = by_name(name, &n);
    if (!a) return -1;
    if (n > cap) return -2;
    memcpy(dst, a, sizeof(double) * (size_t)n);
    return n;
}

int orc_set(const char *name, const double *src, long count) {
    long n;
    if (!S) return -1;
    double *a = by_name(name, &n);
    if (!a) return -1;
    if (n != count) return -2;
    memcpy(a, src, sizeof(double) * (size_t)n);
    return 0;
}
