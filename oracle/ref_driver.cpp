/*
 * ref_driver.cpp -- C driver around the UNMODIFIED reference solver sources,
 * compiled in place (see oracle/Makefile) into oracle/_ref/libns3d_ref.so.
 *
 * TEST INFRASTRUCTURE ONLY.  It exists to pin the CPU restatement
 * (oracle/ns3d_oracle.c) and to serve as the timed CPU baseline; nothing in
 * the product links it.
 *
 * The call sequence mirrors the reference's own driver:
 *   read_solver_params_from_file            (main.cpp:16, initialization.cpp:36-200)
 *   build_cart_decomp / compute_local_desc  (main.cpp:17-20, field_structures.h:1062-1115)
 *   F.allocate                               (main.cpp:67, field_structures.h:250-373)
 *   interior primitives supplied by the caller (replaces the initialisers)
 *   apply_boundary; primitiveToConserved     (main.cpp:98-99)
 *   recordConservedTo0; runge_kutta_3        (maincycle.cpp:22,56)
 */
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "field_structures.h"
#include "ns3d_func.h"
#include <thread>

// Runs fn on a new thread.  The reference's isotropic initialiser draws from a
// thread_local std::mt19937_64 seeded on first use in a thread
// (isotropic_ini.cpp:16-20), so on a fresh thread every call starts from the
// seed, as the reference's first call in a process does.
template <class F>
static void on_fresh_thread(F fn) {
    std::thread t(fn);
    t.join();
}

// The reference's post-processing writers live in files that need FFTW/HDF5;
// the oracle build leaves those files out and supplies no-op definitions.
void write_tecplot_field(const Field3D &, const GridDesc &, const CartDecomp &, const SolverParams &, double) {}
void write_residuals_tecplot(const Field3D &, int, const std::string &) {}
void compute_energy_spectrum(const Field3D &, const GridDesc &, const CartDecomp &, const std::string &) {}
void compute_turbulence_statistics(Field3D &, const GridDesc &, const SolverParams &, const CartDecomp &, const double) {}

namespace {
struct RefState {
    SolverParams P;
    GridDesc G;
    CartDecomp C;
    Field3D F;
    HaloRequests reqs;
    bool ready = false;
};
RefState *S = nullptr;

std::vector<double> *field_by_name(const char *name) {
    if (!S) return nullptr;
    Field3D &F = S->F;
    static const char *names[] = {
        "rho", "rhou", "rhov", "rhow", "E", "rho0", "rhou0", "rhov0", "rhow0", "E0",
        "u", "v", "w", "p", "T", "rhs_rho", "rhs_rhou", "rhs_rhov", "rhs_rhow", "rhs_E",
        "flux_fx_mass", "flux_fx_momx", "flux_fx_momy", "flux_fx_momz", "flux_fx_E",
        "flux_fy_mass", "flux_fy_momx", "flux_fy_momy", "flux_fy_momz", "flux_fy_E",
        "flux_fz_mass", "flux_fz_momx", "flux_fz_momy", "flux_fz_momz", "flux_fz_E",
        "du_dx", "du_dy", "du_dz", "dv_dx", "dv_dy", "dv_dz", "dw_dx", "dw_dy", "dw_dz",
        "dT_dx", "dT_dy", "dT_dz",
        "Fvflux_momx", "Fvflux_momy", "Fvflux_momz", "Fvflux_E",
        "Hvflux_momx", "Hvflux_momy", "Hvflux_momz", "Hvflux_E",
        "Gvflux_momx", "Gvflux_momy", "Gvflux_momz", "Gvflux_E", nullptr};
    std::vector<double> *ptrs[] = {
        &F.rho, &F.rhou, &F.rhov, &F.rhow, &F.E, &F.rho0, &F.rhou0, &F.rhov0, &F.rhow0, &F.E0,
        &F.u, &F.v, &F.w, &F.p, &F.T, &F.rhs_rho, &F.rhs_rhou, &F.rhs_rhov, &F.rhs_rhow, &F.rhs_E,
        &F.flux_fx_mass, &F.flux_fx_momx, &F.flux_fx_momy, &F.flux_fx_momz, &F.flux_fx_E,
        &F.flux_fy_mass, &F.flux_fy_momx, &F.flux_fy_momy, &F.flux_fy_momz, &F.flux_fy_E,
        &F.flux_fz_mass, &F.flux_fz_momx, &F.flux_fz_momy, &F.flux_fz_momz, &F.flux_fz_E,
        &F.du_dx, &F.du_dy, &F.du_dz, &F.dv_dx, &F.dv_dy, &F.dv_dz, &F.dw_dx, &F.dw_dy, &F.dw_dz,
        &F.dT_dx, &F.dT_dy, &F.dT_dz,
        &F.Fvflux_momx, &F.Fvflux_momy, &F.Fvflux_momz, &F.Fvflux_E,
        &F.Hvflux_momx, &F.Hvflux_momy, &F.Hvflux_momz, &F.Hvflux_E,
        &F.Gvflux_momx, &F.Gvflux_momy, &F.Gvflux_momz, &F.Gvflux_E};
    for (int i = 0; names[i]; ++i)
        if (std::strcmp(names[i], name) == 0) return ptrs[i];
    return nullptr;
}
}  // namespace

extern "C" {

/* Parse a solver.in file with the reference parser and allocate the field.
 * s_ref > 0 overrides the hard-coded Sutherland constant (field_structures.h:95). */
int ref_init_file(const char *path, double s_ref) {
    delete S;
    S = new RefState();
    S->C = CartDecomp();
    if (!read_solver_params_from_file(path, S->P, S->G, S->C)) return -1;
    if (s_ref > 0.0) S->P.S_ref = s_ref;
    build_cart_decomp(S->C);
    LocalDesc L;
    compute_local_desc(S->G, S->C, L, S->P.ghost_layers, S->P.ghost_layers, S->P.ghost_layers);
    S->F.allocate(L);
    S->ready = true;
    return 0;
}

void ref_free(void) { delete S; S = nullptr; }

int ref_dims(int *out6) {
    if (!S) return -1;
    const LocalDesc &L = S->F.L;
    out6[0] = L.nx; out6[1] = L.ny; out6[2] = L.nz;
    out6[3] = L.ngx; out6[4] = L.ngy; out6[5] = L.ngz;
    return 0;
}

/* Scalars after parsing: gamma Pr Ma Re cfl dt_fixed mu S_ref Cv Cp Rgas dx dy dz
 * mdcd_diss mdcd_disp TotalTime output_Timefreq and ints. */
int ref_params(double *d18, int *i16) {
    if (!S) return -1;
    const SolverParams &P = S->P;
    const GridDesc &G = S->G;
    double d[18] = {P.gamma, P.Pr, P.Ma, P.Re, P.cfl, P.dt_fixed, P.mu, P.S_ref, P.Cv, P.Cp, P.Rgas,
                    G.dx, G.dy, G.dz, P.mdcd_diss, P.mdcd_disp, P.TotalTime, P.output_Timefreq};
    std::memcpy(d18, d, sizeof(d));
    int i[16] = {(int)P.interpolation, (int)P.riemann_solver, (int)P.char_recon,
                 (int)P.bc_xmin, (int)P.bc_xmax, (int)P.bc_ymin, (int)P.bc_ymax, (int)P.bc_zmin, (int)P.bc_zmax,
                 G.global_nx, G.global_ny, G.global_nz, P.max_steps, P.monitor_Stepfreq,
                 (int)P.fvs_type, (int)P.vis_scheme};
    std::memcpy(i16, i, sizeof(i));
    return 0;
}

/* Interior primitives (nx*ny*nz each, x fastest) -> ghost fill -> conserved,
 * exactly as main.cpp:98-99 does after an initialiser. */
int ref_set_interior_prims(const double *rho, const double *u, const double *v, const double *w,
                           const double *p) {
    if (!S) return -1;
    Field3D &F = S->F;
    const LocalDesc &L = F.L;
    size_t n = 0;
    for (int k = 0; k < L.nz; ++k)
        for (int j = 0; j < L.ny; ++j)
            for (int i = 0; i < L.nx; ++i, ++n) {
                int id = F.I(i + L.ngx, j + L.ngy, k + L.ngz);
                F.rho[id] = rho[n]; F.u[id] = u[n]; F.v[id] = v[n]; F.w[id] = w[n]; F.p[id] = p[n];
            }
    apply_boundary(F, S->G, S->C, S->P);
    F.primitiveToConserved(S->P);
    return 0;
}

int ref_get(const char *name, double *dst, long cap) {
    std::vector<double> *f = field_by_name(name);
    if (!f) return -1;
    if ((long)f->size() > cap) return -2;
    std::memcpy(dst, f->data(), f->size() * sizeof(double));
    return (int)f->size();
}

int ref_set(const char *name, const double *src, long count) {
    std::vector<double> *f = field_by_name(name);
    if (!f) return -1;
    if ((long)f->size() != count) return -2;
    std::memcpy(f->data(), src, f->size() * sizeof(double));
    return 0;
}

void ref_compute_rhs(void) { compute_rhs(S->F, S->C, S->G, S->P, S->reqs); }
void ref_apply_boundary(void) { apply_boundary(S->F, S->G, S->C, S->P); }
void ref_prim_to_cons(void) { S->F.primitiveToConserved(S->P); }
void ref_cons_to_prim(void) { S->F.conservedToPrimitive(S->P); }

/* One RK3 step as time_advance performs it (maincycle.cpp:22,56). */
void ref_rk3_step(double dt) {
    S->F.recordConservedTo0();
    runge_kutta_3(S->F, S->C, S->G, S->P, S->reqs, dt);
}

double ref_timestep(void) { return compute_timestep(S->F, S->G, S->P); }

double ref_total_energy(void) {
    compute_total_energy(S->F, S->G, S->C, S->P);
    return S->F.global_Etot;
}

/* One of the reference's built-in initialisers (initialization.cpp:516-638),
 * then apply_boundary + primitiveToConserved as main.cpp:85-99.  kind: 0
 * riemann_2d, 1 sod, 2 uniform, 3 sine_x. */
int ref_initialize(int kind) {
    if (!S) return -1;
    switch (kind) {
        case 0: initialize_riemann_2d(S->F, S->G, S->P); break;
        case 1: initialize_sod_shock_tube(S->F, S->G, S->P); break;
        case 2: initialize_uniform_field(S->F, S->G, S->P); break;
        case 3: initialize_sine_x_field(S->F, S->G, S->P); break;
        case 4: on_fresh_thread([] { init_isotropic_turbulence(S->F, S->G, S->C, S->P); }); break;
        default: return -1;
    }
    apply_boundary(S->F, S->G, S->C, S->P);
    S->F.primitiveToConserved(S->P);
    return 0;
}

/* compute_diagnostics (postprocess.cpp:7-98) after the last step: the
 * residual norms F.global_res_rho ... F.global_res_E. */
void ref_residuals(double *out5) {
    compute_diagnostics(S->F, S->P, S->G);
    const Field3D &F = S->F;
    out5[0] = F.global_res_rho; out5[1] = F.global_res_rhou; out5[2] = F.global_res_rhov;
    out5[3] = F.global_res_rhow; out5[4] = F.global_res_E;
}

/* F.global_Etot and the residual norms as the last time_advance left them. */
void ref_monitor_values(double *out6) {
    const Field3D &F = S->F;
    out6[0] = F.global_Etot; out6[1] = F.global_res_rho; out6[2] = F.global_res_rhou;
    out6[3] = F.global_res_rhov; out6[4] = F.global_res_rhow; out6[5] = F.global_res_E;
}

/* The reference's own step loop (maincycle.cpp:7-113) with the run-control
 * keys of the parsed solver.in; output writers are no-ops. */
void ref_time_advance(void) { time_advance(S->F, S->C, S->G, S->P); }

}  // extern "C"

/* ---- per-function known-answer wrappers around the reference's free
 * functions (ns3d_func.h:77-112), used to generate the scalar KAT fixtures. */
extern "C" {

double ref_weno5(const double *f) {
    std::array<double, 6> a;
    for (int i = 0; i < 6; ++i) a[i] = f[i];
    return weno5_interpolate(a);
}

double ref_mdcd_linear(const double *f, double disp, double diss) {
    std::array<double, 6> a;
    for (int i = 0; i < 6; ++i) a[i] = f[i];
    SolverParams P;
    P.mdcd_disp = disp; P.mdcd_diss = diss;
    return mdcd_linear_interpolate(a, P);
}

double ref_mdcd_hybrid(const double *f, double disp, double diss) {
    std::array<double, 6> a;
    for (int i = 0; i < 6; ++i) a[i] = f[i];
    SolverParams P;
    P.mdcd_disp = disp; P.mdcd_diss = diss;
    return mdcd_hybrid_interpolate(a, P);
}

void ref_riemann(int solver, const double *UL, const double *UR, int dir, double gamma, double *F) {
    std::vector<double> L(UL, UL + 5), R(UR, UR + 5), out(5, 0.0);
    double nx = dir == 0, ny = dir == 1, nz = dir == 2;
    switch (solver) {
        case 0: Roe_Riemann_solver(out, L, R, nx, ny, nz, gamma); break;
        case 1: Rusanov_Riemann_solver(out, L, R, nx, ny, nz, gamma); break;
        case 2: HLLC_Riemann_solver(out, L, R, nx, ny, nz, gamma); break;
        case 3: HLL_Riemann_solver(out, L, R, nx, ny, nz, gamma); break;
        case 4: HLLC_p_Riemann_solver(out, L, R, nx, ny, nz, gamma); break;
        case 5: AUSM_Riemann_solver(out, L, R, nx, ny, nz, gamma); break;
    }
    for (int i = 0; i < 5; ++i) F[i] = out[i];
}

// generate_full_turbulence (isotropic_ini.cpp:26-126): the velocity field in the
// reference's order, index (i*ny + j)*nz + k, from the generator's seed.
int ref_isotropic_field(int nx, int ny, int nz, double *u, double *v, double *w) {
    std::vector<double> U, V, W;
    on_fresh_thread([&] { generate_full_turbulence(nx, ny, nz, U, V, W); });
    for (size_t id = 0; id < U.size(); ++id) { u[id] = U[id]; v[id] = V[id]; w[id] = W[id]; }
    return 0;
}

}  // extern "C"
