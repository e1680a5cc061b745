// ns3d_gpu_compat.cpp -- reference-side drop-in: the hot-path entry points of
// ns3d_func.h implemented over the C ABI of libns3d_b200.so.
//
// Build it into the reference in place of range_kutta.cpp and timestep.cpp
// (which define the first three functions on the CPU), with the reference's
// headers on the include path and -lns3d_b200:
//
//   compute_rhs      (ns3d_func.h:134, range_kutta.cpp:11-43)
//   runge_kutta_3    (ns3d_func.h:137, range_kutta.cpp:46-92)
//   compute_timestep (ns3d_func.h:140, timestep.cpp:5-23)
//
// Each of these uploads the primitive state of the Field3D (rho,u,v,w,p: the
// arrays primitiveToConserved rebuilds the conserved state from), runs on the
// GPU and writes the conserved, primitive, temperature and RHS arrays back
// (runge_kutta_3 leaves its last stage's right-hand side in F.rhs_*, as the
// reference does), so the host Field3D holds what the CPU implementation
// leaves there and the rest of the reference is unchanged.
//
// Built with -DNS3D_COMPAT_TIME_ADVANCE (and without maincycle.cpp) it also
// defines
//
//   time_advance     (ns3d_func.h:198, maincycle.cpp:7-113)
//
// with the state resident on the GPU for the whole run: one upload at the
// start, the reference's dt schedule, monitor output and output schedule on
// the host, compute_diagnostics' residual norms and compute_total_energy on
// the device (ns3d_residuals, ns3d_total_energy), and the host Field3D
// refreshed only where reference code reads it -- before write_tecplot_field
// and isotropic_post_process, and at the end.  recordConservedTo0's host copy
// of the conserved state is not made: the device keeps the step-start state
// itself (F.rho0 ... F.E0 are not refreshed).
//
// One GPU holds the whole domain: the CartDecomp and HaloRequests arguments
// are accepted and ignored (single rank).  A CUDA or configuration failure
// prints the library's message and aborts, where the reference would also
// stop (it has no error returns on this path).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <vector>

#include "field_structures.h"
#include "ns3d_b200.h"
#include "ns3d_func.h"

namespace {

struct Binding {
    ns3d_handle *h = nullptr;
    const Field3D *field = nullptr;
    int sx = 0, sy = 0, sz = 0;
    ns3d_params params{};  // what the handle was created with
    ns3d_grid grid{};
};
Binding g_bind;

void check(int status, const char *what) {
    if (status == NS3D_OK) return;
    std::fprintf(stderr, "ns3d_b200: %s failed: %s (%s)\n", what, ns3d_status_string(status),
                 ns3d_last_error(g_bind.h));
    std::abort();
}

ns3d_params params_of(const SolverParams &P) {
    ns3d_params p;
    ns3d_params_default(&p);  // zero-fills the whole struct first
    p.gamma = P.gamma; p.Pr = P.Pr; p.Ma = P.Ma; p.Re = P.Re; p.cfl = P.cfl; p.dt_fixed = P.dt_fixed;
    p.mdcd_diss = P.mdcd_diss; p.mdcd_disp = P.mdcd_disp; p.sutherland_s = P.S_ref;
    p.interpolation = (int)P.interpolation;
    p.riemann_solver = (int)P.riemann_solver;
    p.char_recon = P.char_recon ? 1 : 0;
    const SolverParams::BCType b[6] = {P.bc_xmin, P.bc_xmax, P.bc_ymin, P.bc_ymax, P.bc_zmin, P.bc_zmax};
    for (int f = 0; f < 6; ++f) p.bc[f] = (int)b[f];
    const char *dev = std::getenv("NS3D_DEVICE");
    p.device = dev ? std::atoi(dev) : 0;
    p.keep_rhs = 1;  // runge_kutta_3 leaves the last stage's RHS in F.rhs_*
    return p;
}

// The handle of this Field3D and configuration: reused while the field, its
// sizes, the grid and every solver parameter the GPU reads are unchanged,
// recreated otherwise (a host that changes SolverParams between calls gets a
// handle with the new ones).
ns3d_handle *bind(Field3D &F, const GridDesc &G, const SolverParams &P) {
    const LocalDesc &L = F.L;
    const ns3d_params p = params_of(P);
    const ns3d_grid g = {L.nx, L.ny, L.nz, G.x0, G.y0, G.z0, G.Lx, G.Ly, G.Lz};
    if (g_bind.h && g_bind.field == &F && g_bind.sx == L.sx && g_bind.sy == L.sy && g_bind.sz == L.sz &&
        std::memcmp(&g_bind.params, &p, sizeof(p)) == 0 && std::memcmp(&g_bind.grid, &g, sizeof(g)) == 0)
        return g_bind.h;
    if (g_bind.h) ns3d_destroy(g_bind.h);
    g_bind.h = nullptr;
    check(ns3d_create(&p, &g, &g_bind.h), "ns3d_create");
    g_bind.field = &F;
    g_bind.sx = L.sx; g_bind.sy = L.sy; g_bind.sz = L.sz;
    g_bind.params = p;
    g_bind.grid = g;
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

#ifdef NS3D_COMPAT_TIME_ADVANCE
// time_advance, maincycle.cpp:7-113: the same step loop, dt schedule, monitor
// lines and output calls, with the state on the GPU between them.
void time_advance(Field3D &F, CartDecomp &C, GridDesc &G, SolverParams &P) {
    ns3d_handle *h = bind(F, G, P);
    push(h, F);
    bool host_current = true;  // the host Field3D holds the device's state
    auto refresh_host = [&]() {
        if (!host_current) pull(h, F, true);
        host_current = true;
    };
    double t_start = MPI_Wtime();
    double t_last = t_start;
    double current_time = 0.0;
    const int max_steps = P.max_steps;
    const int monitor_Stepfreq = P.monitor_Stepfreq;
    double output_Timefreq = P.output_Timefreq;
    const double TotalTime = P.TotalTime;

    for (int step = 1; step <= max_steps; ++step) {
        double dt = P.dt_fixed;
        const double eps = 1e-12;
        if (std::abs(TotalTime - current_time) <= eps) break;
        if (P.dt_fixed < 0.0) check(ns3d_compute_timestep(h, &dt), "ns3d_compute_timestep");

        bool if_output = false;
        if (current_time >= output_Timefreq - eps) {
            if_output = true;
            output_Timefreq += P.output_Timefreq;
        }
        if (current_time + dt > TotalTime) dt = TotalTime - current_time;
        if (current_time + dt > output_Timefreq) {
            dt = output_Timefreq - current_time;
            output_Timefreq += P.output_Timefreq;
            if_output = true;
        }
        if (dt <= eps) {
            if (C.rank == 0)
                std::cerr << "dt too small or zero; aborting to avoid stall at Time=" << current_time << "\n";
            break;
        }
        current_time += dt;

        check(ns3d_rk3_step(h, dt), "ns3d_rk3_step");
        host_current = false;
        if (C.rank == 0)
            std::cout << "Completed step " << step << " / " << max_steps << ", Time = " << current_time << " / "
                      << TotalTime << "\n";

        if (step % monitor_Stepfreq == 0 || step == 1) {
            if (P.monitor_res) {
                double res[5];
                check(ns3d_residuals(h, res), "ns3d_residuals");
                F.global_res_rho = res[0]; F.global_res_rhou = res[1]; F.global_res_rhov = res[2];
                F.global_res_rhow = res[3]; F.global_res_E = res[4];
            }
            if (P.monitor_energy) check(ns3d_total_energy(h, &F.global_Etot), "ns3d_total_energy");

            double t_now = MPI_Wtime();
            double t_elapsed = t_now - t_start;
            double t_step = t_now - t_last;
            t_last = t_now;
            if (C.rank == 0) {
                std::cout << std::fixed << std::setprecision(6) << "[Step " << step << "] ";
                std::cout << "dt=" << dt << "  Time/step=" << t_step << "s  Elapsed=" << t_elapsed << "s";
                std::cout << "  Time=" << current_time << "/" << TotalTime;
                if (P.monitor_energy) std::cout << "  Ek_avg=" << F.global_Etot;
                std::cout << "\n";
                if (P.monitor_res) {
                    std::stringstream ss;
                    ss << "output_residuals.dat";
                    write_residuals_tecplot(F, step, ss.str());
                }
            }
            if (P.isotropic_analyse) {
                refresh_host();
                isotropic_post_process(F, G, C, P, current_time);
            }
        }

        if (if_output) {
            if (P.post_basicfield) {
                refresh_host();
                write_tecplot_field(F, G, C, P, current_time);
            }
            if (P.isotropic_analyse) {
                refresh_host();
                isotropic_post_process(F, G, C, P, current_time);
            }
        }
        if (current_time >= TotalTime) break;
    }
    refresh_host();

    if (C.rank == 0) {
        double total_time = MPI_Wtime() - t_start;
        std::cout << "Simulation complete. Total time: " << total_time << " s\n";
    }
}
#endif
