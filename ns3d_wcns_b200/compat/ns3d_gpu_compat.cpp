// ns3d_gpu_compat.cpp -- reference-side drop-in: the hot-path entry points of
// ns3d_func.h implemented over the C ABI of libns3d_b200.so.
//
// Build it into the reference in place of range_kutta.cpp and timestep.cpp
// (which define these three functions on the CPU), with the reference's
// headers on the include path and -lns3d_b200:
//
//   compute_rhs      (ns3d_func.h:134, range_kutta.cpp:11-43)
//   runge_kutta_3    (ns3d_func.h:137, range_kutta.cpp:46-92)
//   compute_timestep (ns3d_func.h:140, timestep.cpp:5-23)
//
// Every call uploads the primitive state of the Field3D (rho,u,v,w,p: the
// arrays primitiveToConserved rebuilds the conserved state from), runs on the
// GPU and writes the conserved, primitive, temperature and RHS arrays back,
// so the host Field3D holds exactly what the CPU implementation leaves there
// and the rest of the reference (time_advance, diagnostics, output) is
// unchanged.  One GPU holds the whole domain: the CartDecomp and
// HaloRequests arguments are accepted and ignored (single rank).  A CUDA or
// configuration failure prints the library's message and aborts, where the
// reference would also stop (it has no error returns on this path).
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "field_structures.h"
#include "ns3d_b200.h"
#include "ns3d_func.h"

namespace {

struct Binding {
    ns3d_handle *h = nullptr;
    const Field3D *field = nullptr;
    int sx = 0, sy = 0, sz = 0;
};
Binding g_bind;

void check(int status, const char *what) {
    if (status == NS3D_OK) return;
    std::fprintf(stderr, "ns3d_b200: %s failed: %s (%s)\n", what, ns3d_status_string(status),
                 ns3d_last_error(g_bind.h));
    std::abort();
}

ns3d_handle *bind(Field3D &F, const GridDesc &G, const SolverParams &P) {
    const LocalDesc &L = F.L;
    if (g_bind.h && g_bind.field == &F && g_bind.sx == L.sx && g_bind.sy == L.sy && g_bind.sz == L.sz)
        return g_bind.h;
    if (g_bind.h) ns3d_destroy(g_bind.h);
    ns3d_params p;
    ns3d_params_default(&p);
    p.gamma = P.gamma; p.Pr = P.Pr; p.Ma = P.Ma; p.Re = P.Re; p.cfl = P.cfl; p.dt_fixed = P.dt_fixed;
    p.mdcd_diss = P.mdcd_diss; p.mdcd_disp = P.mdcd_disp; p.sutherland_s = P.S_ref;
    p.interpolation = (int)P.interpolation;
    p.riemann_solver = (int)P.riemann_solver;
    p.char_recon = P.char_recon ? 1 : 0;
    const SolverParams::BCType b[6] = {P.bc_xmin, P.bc_xmax, P.bc_ymin, P.bc_ymax, P.bc_zmin, P.bc_zmax};
    for (int f = 0; f < 6; ++f) p.bc[f] = (int)b[f];
    const char *dev = std::getenv("NS3D_DEVICE");
    p.device = dev ? std::atoi(dev) : 0;
    ns3d_grid g = {L.nx, L.ny, L.nz, G.x0, G.y0, G.z0, G.Lx, G.Ly, G.Lz};
    check(ns3d_create(&p, &g, &g_bind.h), "ns3d_create");
    g_bind.field = &F;
    g_bind.sx = L.sx; g_bind.sy = L.sy; g_bind.sz = L.sz;
    return g_bind.h;
}

void push(ns3d_handle *h, Field3D &F) {
    const double *w[5] = {F.rho.data(), F.u.data(), F.v.data(), F.w.data(), F.p.data()};
    check(ns3d_upload_primitives(h, w), "ns3d_upload_primitives");
}

void pull(ns3d_handle *h, Field3D &F, bool with_rhs) {
    double *u[5] = {F.rho.data(), F.rhou.data(), F.rhov.data(), F.rhow.data(), F.E.data()};
    check(ns3d_download(h, NS3D_CONSERVED, u), "ns3d_download(conserved)");
    std::vector<double> rho(F.rho.size());
    double *w[5] = {rho.data(), F.u.data(), F.v.data(), F.w.data(), F.p.data()};
    check(ns3d_download(h, NS3D_PRIMITIVE, w), "ns3d_download(primitive)");
    double *t[1] = {F.T.data()};
    check(ns3d_download(h, NS3D_TEMPERATURE, t), "ns3d_download(temperature)");
    if (with_rhs) {
        double *r[5] = {F.rhs_rho.data(), F.rhs_rhou.data(), F.rhs_rhov.data(), F.rhs_rhow.data(), F.rhs_E.data()};
        check(ns3d_download(h, NS3D_RHS, r), "ns3d_download(rhs)");
    }
}

}  // namespace

void compute_rhs(Field3D &F, CartDecomp &, GridDesc &G, SolverParams &P, HaloRequests &) {
    ns3d_handle *h = bind(F, G, P);
    push(h, F);
    check(ns3d_compute_rhs(h), "ns3d_compute_rhs");
    double *r[5] = {F.rhs_rho.data(), F.rhs_rhou.data(), F.rhs_rhov.data(), F.rhs_rhow.data(), F.rhs_E.data()};
    check(ns3d_download(h, NS3D_RHS, r), "ns3d_download(rhs)");
}

void runge_kutta_3(Field3D &F, CartDecomp &, GridDesc &G, SolverParams &P, HaloRequests &, double dt) {
    ns3d_handle *h = bind(F, G, P);
    push(h, F);
    check(ns3d_rk3_step(h, dt), "ns3d_rk3_step");
    pull(h, F, true);
}

double compute_timestep(Field3D &F, const GridDesc &G, const SolverParams &P) {
    ns3d_handle *h = bind(F, G, P);
    push(h, F);
    double dt = 0.0;
    check(ns3d_compute_timestep(h, &dt), "ns3d_compute_timestep");
    return dt;
}
