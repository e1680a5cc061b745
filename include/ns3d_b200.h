/*
 * ns3d_b200.h -- C ABI of the B200 (sm_100a) implementation of ns3d_wcns's
 * right-hand-side evaluation and RK3 time advance.
 *
 * The entry points replace the per-rank CPU loops behind the reference's
 * ns3d_func.h; each declaration names the reference interface it stands in
 * for.  Plain pointers and sizes only: no C++ or torch types cross this
 * boundary, no exceptions escape it, every call returns an int status
 * (NS3D_OK == 0, negative on error) and ns3d_last_error() describes the last
 * failure of a handle.
 *
 * Host arrays use the reference's Field3D layout (field_structures.h:64-67):
 * one array per variable of sx*sy*sz doubles, sx = nx + 6, sy = ny + 6,
 * sz = nz + 6 (3 ghost layers), id = (k*sy + j)*sx + i, x fastest.  Interior
 * cells are i in [3, nx+3) etc.  The device keeps its own padded layout; the
 * ABI converts on upload/download.
 *
 * Threading: one handle per host thread.  Calls are ordered on the handle's
 * CUDA stream; calls that return host values synchronise that stream.
 */
#ifndef NS3D_B200_H
#define NS3D_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status codes */
#define NS3D_OK 0
#define NS3D_ERR_INVALID_ARG (-1)   /* null pointer, bad enum, bad size */
#define NS3D_ERR_CONFIG (-2)        /* configuration the path does not support */
#define NS3D_ERR_OOM (-3)           /* device allocation failed */
#define NS3D_ERR_CUDA (-4)          /* CUDA runtime error (message in last_error) */
#define NS3D_ERR_NONFINITE (-5)     /* non-finite or non-positive state detected */
#define NS3D_ERR_NO_DEVICE (-6)     /* no usable CUDA device */
#define NS3D_ERR_STATE (-7)         /* call out of order (e.g. no state uploaded) */
#define NS3D_ERR_DT (-8)            /* time step <= 1e-12 (maincycle.cpp:46-52) */
#define NS3D_ERR_TIMEOUT (-9)       /* a bounded device wait expired */
#define NS3D_ERR_SIZE (-10)         /* grid larger than an entry point's stated maximum */

/* ------------------------------------------------------------ enumerations */
/* Same numbering as the reference enums (field_structures.h:131-165).
 * NS3D_STEGER_WARMING is this library's addition: the reference declares the
 * splitting (field_structures.h:113-119) without implementing it. */
enum { NS3D_WENO5 = 0, NS3D_ZERO = 1, NS3D_MDCD_LINEAR = 2, NS3D_MDCD_HYBRID = 3 };
enum { NS3D_ROE = 0, NS3D_RUSANOV = 1, NS3D_HLLC = 2, NS3D_HLL = 3, NS3D_HLLC_P = 4, NS3D_AUSM = 5,
       NS3D_STEGER_WARMING = 6 };
enum { NS3D_PERIODIC = 0, NS3D_WALL = 1, NS3D_SYMMETRY = 2, NS3D_OUTFLOW = 3, NS3D_INFLOW = 4 };
enum { NS3D_FP64 = 0, NS3D_MIXED = 1 };

/* Which group of arrays ns3d_download / ns3d_device_fields refer to. */
enum {
    NS3D_PRIMITIVE = 0,   /* rho, u, v, w, p          (Field3D rho,u,v,w,p)        */
    NS3D_CONSERVED = 1,   /* rho, rhou, rhov, rhow, E (Field3D rho,rhou,...,E)     */
    NS3D_RHS = 2,         /* rhs_rho ... rhs_E of the last compute_rhs              */
    NS3D_TEMPERATURE = 3  /* T = p / (rho Rgas)        (one array)                  */
};

/* SolverParams subset the hot path reads (field_structures.h:86-186) plus
 * this build's additions.  Fill with ns3d_params_default() first. */
typedef struct ns3d_params {
    double gamma, Pr, Ma, Re;
    double cfl, dt_fixed;           /* dt_fixed < 0 => adaptive (maincycle.cpp:30) */
    double mdcd_diss, mdcd_disp;
    double sutherland_s;            /* S/T_ref; reference value 110.4/288.15 */
    int interpolation;              /* NS3D_WENO5 | NS3D_MDCD_LINEAR | NS3D_MDCD_HYBRID */
    int riemann_solver;             /* NS3D_ROE ... NS3D_AUSM, NS3D_STEGER_WARMING */
    int char_recon;                 /* 0 component-wise, 1 characteristic-wise */
    int bc[6];                      /* xmin xmax ymin ymax zmin zmax */
    int precision;                  /* NS3D_FP64 (reference parity) | NS3D_MIXED */
    int device;                     /* CUDA device ordinal */
    int check_state;                /* 1: rk3 calls verify the state is finite */
    int keep_rhs;                   /* 1: an RK3 step also leaves its last stage's complete
                                       right-hand side in the RHS buffer, as runge_kutta_3
                                       leaves it in F.rhs_* (one more write per cell in the
                                       last stage); 0 (default): the last stage updates the
                                       state without storing its RHS, and NS3D_RHS can be
                                       downloaded only after ns3d_compute_rhs */
} ns3d_params;

/* GridDesc (field_structures.h:33-38). */
typedef struct ns3d_grid {
    int nx, ny, nz;                 /* interior cells (global_nx ...) */
    double x0, y0, z0;
    double Lx, Ly, Lz;              /* dx = Lx / nx (initialization.cpp:170-172) */
} ns3d_grid;

typedef struct ns3d_handle ns3d_handle;

/* Defaults of SolverParams (field_structures.h:86-186); bc all Periodic. */
void ns3d_params_default(ns3d_params *p);

const char *ns3d_status_string(int status);

/* Allocates every device buffer of the solver for this grid.
 * Replaces: Field3D::allocate (field_structures.h:250-373) and the MPI set-up
 * of main.cpp:16-20 (one GPU holds the whole domain). */
int ns3d_create(const ns3d_params *params, const ns3d_grid *grid, ns3d_handle **out);
int ns3d_destroy(ns3d_handle *h);
const char *ns3d_last_error(const ns3d_handle *h);

/* Field3D sizes: out[0..2] = sx, sy, sz. */
int ns3d_field_dims(const ns3d_handle *h, int out[3]);

/* Full-field upload of primitives (rho,u,v,w,p), all sx*sy*sz cells in Field3D
 * layout: the state the reference holds after apply_boundary +
 * primitiveToConserved (main.cpp:98-99).  Ghost cells are taken as given. */
int ns3d_upload_primitives(ns3d_handle *h, const double *const fields[5]);

/* Interior-only upload (nx*ny*nz per array, x fastest) followed by the device
 * ghost fill.  Replaces: an initialiser + apply_boundary + primitiveToConserved
 * (main.cpp:85-99). */
int ns3d_set_interior_primitives(ns3d_handle *h, const double *const fields[5]);

/* Built-in initial states on the device, followed by the ghost fill: the
 * state main.cpp:85-99 sets up with one of the reference's initialisers,
 * apply_boundary and primitiveToConserved.  Replaces:
 *   NS3D_INIT_RIEMANN_2D  initialize_riemann_2d     (initialization.cpp:516-566;
 *                         main.cpp's default; every cell, ghosts included)
 *   NS3D_INIT_SOD         initialize_sod_shock_tube (initialization.cpp:568-596)
 *   NS3D_INIT_UNIFORM     initialize_uniform_field  (initialization.cpp:598-617)
 *   NS3D_INIT_SINE_X      initialize_sine_x_field   (initialization.cpp:619-638)
 *   NS3D_INIT_ISOTROPIC   init_isotropic_turbulence (isotropic_ini.cpp:16-193):
 *                         the seed-123 std::mt19937_64 phases, the k0 = 8
 *                         spectrum, its inverse transform scaled to the
 *                         reference's energy; rho = 1, T = 1.  Allocates
 *                         scratch (three complex fields); at most 2048 cells
 *                         per axis.  Each call starts the generator afresh (the
 *                         reference's first call in a process).
 * Cells an initialiser does not write keep their current values (the
 * Field3D::allocate defaults on a new handle). */
enum { NS3D_INIT_RIEMANN_2D = 0, NS3D_INIT_SOD = 1, NS3D_INIT_UNIFORM = 2, NS3D_INIT_SINE_X = 3,
       NS3D_INIT_ISOTROPIC = 4 };
int ns3d_initialize(ns3d_handle *h, int kind);

/* Download one group (NS3D_PRIMITIVE/CONSERVED/RHS: 5 arrays; TEMPERATURE: 1)
 * in Field3D layout. */
int ns3d_download(ns3d_handle *h, int what, double *const out[]);

/* Ghost fill of the current state.  Replaces: apply_boundary
 * (boundary.cpp:14-54, ns3d_func.h:60), including exchange_halos_physical's
 * periodic wrap (field_structures.h:936-994). */
int ns3d_apply_boundary(ns3d_handle *h);

/* Right-hand side of the current state into the device RHS buffer.
 * Replaces: compute_rhs (range_kutta.cpp:11-43, ns3d_func.h:134) and the
 * functions it calls (compute_invis_flux, apply_boundary_halfnode_flux,
 * compute_invis_dflux, compute_gradients, compute_viscous_flux,
 * exchange_halos_viscous_flux, compute_vis_flux). */
int ns3d_compute_rhs(ns3d_handle *h);

/* One SSP-RK3 step: recordConservedTo0 + runge_kutta_3 with the c2p ->
 * boundary -> p2c round trip after every stage.
 * Replaces: runge_kutta_3 (range_kutta.cpp:46-92, ns3d_func.h:137) and
 * Field3D::recordConservedTo0 (field_structures.h:491-497). */
int ns3d_rk3_step(ns3d_handle *h, double dt);

/* nsteps fixed-dt RK3 steps in one call (one synchronisation at the end). */
int ns3d_rk3_steps(ns3d_handle *h, int nsteps, double dt);

/* CFL time step.  Replaces: compute_timestep (timestep.cpp:5-23,
 * ns3d_func.h:140): dt = cfl * min over the interior of dx/(|u|+a). */
int ns3d_compute_timestep(ns3d_handle *h, double *dt_out);

/* Sum of 0.5 rho |u|^2 dV over the interior.  Replaces: compute_total_energy
 * (postprocess.cpp:103-128, ns3d_func.h:195). */
int ns3d_total_energy(ns3d_handle *h, double *ke_out);

/* Turbulence reductions of the current state, one pass, FP64 accumulation:
 * out[0] = kinetic energy (as ns3d_total_energy),
 * out[1] = <|grad u|^2> = mean over the interior of sum_ij (du_i/dx_j)^2 with
 *          the viscous-gradient stencils (ViscousFlux.cpp:15-148),
 * out[2] = mean Sutherland mu, out[3] = mean rho,
 * out[4] = dissipation nu * <|grad u|^2>, nu = mean mu / mean rho: the
 *          physical-space counterpart of the spectral epsilon
 *          2 nu sum_k k^2 E(k) of ana_isotropic.cpp:271-305,
 * out[5] = u_rms = sqrt(<u^2+v^2+w^2>/3) (ana_isotropic.cpp:280). */
int ns3d_diagnostics(ns3d_handle *h, double out[6]);

/* Residual norms of the last step.  Replaces: compute_diagnostics
 * (postprocess.cpp:7-98, ns3d_func.h) with Field3D::updateResiduals
 * (field_structures.h:500-508): out[q] = sqrt(sum over the interior of
 * (U_q - U0_q)^2 dx^3) / max over the interior of |U_q| for q = rho, rhou,
 * rhov, rhow, E (F.global_res_rho ... F.global_res_E), U the state after the
 * step and U0 the state the step started from.  Valid right after
 * ns3d_rk3_step / ns3d_rk3_steps / ns3d_time_advance; a download, upload,
 * ghost fill or adjoint call in between reuses the step-start buffer, and the
 * call then returns NS3D_ERR_STATE. */
int ns3d_residuals(ns3d_handle *h, double out[5]);

/* The dt schedule of time_advance (maincycle.cpp:18-56) without I/O:
 * advances from *time until t_end or max_steps, adaptive dt when
 * dt_fixed < 0, last step clipped to hit t_end.  Returns NS3D_ERR_DT when the
 * step would be <= 1e-12 (the reference aborts the loop there). */
int ns3d_time_advance(ns3d_handle *h, double t_end, int max_steps, double *time,
                      int *steps_done);

/* Device pointers of a group (5 pointers, or 1 for TEMPERATURE) plus the
 * padded layout: layout[0..2] = sx, sy, sz, layout[3] = x pitch (elements),
 * layout[4] = x offset of i = 0 (elements), layout[5] = element size (bytes).
 * Pointers stay valid until the next ns3d_rk3_step / ns3d_destroy. */
int ns3d_device_fields(ns3d_handle *h, int what, void *ptrs[5], long layout[6]);

/* Bind the handle to a caller stream (cudaStream_t as void*).  NULL gives the
 * handle a private non-blocking stream of its own, not the legacy default
 * stream: a caller that orders its own work with the handle's (copies of
 * device_fields, NCCL operations, events) passes an explicit stream, e.g.
 * a torch.cuda.Stream(), never torch's default stream (whose handle is 0). */
int ns3d_set_stream(ns3d_handle *h, void *stream);
int ns3d_synchronize(ns3d_handle *h);

/* Kernel launches issued by the last call on this handle (launch accounting). */
int ns3d_last_launch_count(const ns3d_handle *h, long *count);

/* Per-kernel CUDA-event timing on the handle's stream (tracing; no
 * reference counterpart: the reference times with MPI_Wtime only,
 * maincycle.cpp:9,70-77).  enable != 0 starts a fresh record;
 * ns3d_profile_report writes one line per kernel:
 * "<name> <launches> <total milliseconds>". */
int ns3d_profile(ns3d_handle *h, int enable);
int ns3d_profile_report(ns3d_handle *h, char *buf, long len);

/* ------------------------------------------------------------- adjoint
 * Hand-written reverse mode of the RHS and of the RK3 step (no counterpart in
 * the reference).  Plain FP64 path, periodic boundaries, component-wise
 * WENO5 / MDCD_LINEAR / MDCD_HYBRID interpolation (interpolation.cpp:86-209;
 * the hybrid's detector is a switch with zero derivative, its active branch
 * is differentiated) with the Roe, Rusanov, HLL or HLLC flux
 * (InviscousFlux.cpp:449-592: the active arms of the wave-speed and star-state
 * branches); other configurations return NS3D_ERR_CONFIG.  The state differentiated is the
 * interior conserved field (the c2p/p2c round trip is the identity).
 * Host arrays are Field3D-sized (sx*sy*sz); only interior entries are read,
 * ghost entries of outputs are zero. */

/* ubar = (dR/dU)^T rbar at the current state (R = compute_rhs). */
int ns3d_vjp_rhs(ns3d_handle *h, const double *const rbar[5], double *const ubar[5]);

/* ubar = (dU^{n+1}/dU^n)^T ubar_next for one runge_kutta_3 step of size dt
 * from the current state (the state is left unchanged). */
int ns3d_vjp_rk3_step(ns3d_handle *h, double dt, const double *const ubar_next[5], double *const ubar[5]);

/* J = compute_total_energy after nsteps fixed-dt RK3 steps from the current
 * state, and dJ/d(u,v,w) of the initial velocity at fixed rho and p, by a
 * forward pass that keeps a checkpoint every checkpoint_every steps and a
 * backward pass that recomputes each segment's stage states.  grad: three
 * host arrays of nx*ny*nz (x fastest).  stats (nullable): [0] forward ms,
 * [1] backward ms (recompute + adjoint), [2] peak adjoint device bytes,
 * [3] recomputed steps.  The handle's state is the initial one on return. */
int ns3d_adjoint_kinetic_energy(ns3d_handle *h, int nsteps, double dt, int checkpoint_every, double *J,
                                double *const grad[3], double stats[4]);

/* ------------------------------------------------------------- batched
 * Many independent small problems of uneven size (e.g. quasi-1D shock tubes,
 * Nx x 4 x 4) in one persistent launch: each is a full time_advance run
 * (maincycle.cpp:18-56) of its own grid to its own end time with its own CFL
 * time step.  No counterpart in the reference (one problem per process).
 * Plain FP64, inviscid (Re = inf), y and z periodic, any x boundary types,
 * component-wise interpolation.  Thread-block clusters take problems from an
 * atomic work queue, largest first (the persistent schedule).  The
 * wavefront schedule (cluster 0) instead advances every active problem one
 * step per round of flat launches over all their cells, so uneven sizes
 * keep the whole GPU busy (faces and update fused per brick of 256/(ny nz)
 * x-cells by the cross-section when ny nz <= 64); the host drops finished
 * problems every 16 steps.
 * Both give the same bits for the compiled-in WENO5 + Roe instantiation (other
 * schemes agree to rounding).  ns3d_batch_autotune times the wavefront and the
 * persistent cluster size (1,2,4,8) x CTA width (128,256) x resident CTAs
 * per SM (1,2,3: the register budget of the kernel instantiation) choices
 * and keeps the fastest; config_out = {cluster (0: wavefront), width, CTAs
 * per SM}. */
typedef struct ns3d_batch ns3d_batch;
int ns3d_batch_create(const ns3d_params *params, int n_problems, const ns3d_grid *grids, const double *t_end,
                      ns3d_batch **out);
int ns3d_batch_destroy(ns3d_batch *b);
const char *ns3d_batch_last_error(const ns3d_batch *b);
/* interior primitives of problem i (nx*ny*nz each) + its ghost fill */
int ns3d_batch_set_interior_primitives(ns3d_batch *b, int problem, const double *const fields[5]);
/* every problem to its t_end (or max_steps steps) with the configured
 * schedule: the wavefront's rounds of launches, or one persistent launch
 * captured in a CUDA graph */
int ns3d_batch_run(ns3d_batch *b, int max_steps);
int ns3d_batch_autotune(ns3d_batch *b, int trial_steps, int config_out[3]);
int ns3d_batch_set_config(ns3d_batch *b, int cluster, int threads, int ctas_per_sm);
/* final time, steps taken, status (0 reached t_end, 1 dt <= 1e-12, 2 max_steps) */
int ns3d_batch_query(ns3d_batch *b, int problem, double *time, int *steps, int *status);
/* primitive Field3D arrays (rho,u,v,w,p; sx*sy*sz each) of problem i */
int ns3d_batch_download(ns3d_batch *b, int problem, double *const out[5]);

/* ------------------------------------------------- verification helpers
 * Host evaluation (no device needed) of the code the adjoint kernels run,
 * for finite-difference checks.  No counterpart in the reference.
 * ns3d_debug_face_vjp: U30 = conserved stencil U[q][m] (q = rho..E, m = cells
 * i-2..i+3), Fbar5 = adjoint of the face flux; out30 = dF/dU^T Fbar (same
 * indexing); flux5 (nullable) = the production face flux of that stencil.
 * interpolation: NS3D_WENO5 | NS3D_MDCD_LINEAR (lin = its six coefficients)
 * | NS3D_MDCD_HYBRID (lin = ten values: the six linear coefficients, then the
 * four of the WENO branch); riemann: NS3D_ROE | NS3D_RUSANOV | NS3D_HLLC |
 * NS3D_HLL.
 * ns3d_debug_visc_vjp: pointwise node viscous flux at x4 = (u,v,w,T) with
 * gradients g12 (d{u,v,w,T}/d{x,y,z}); V9 (nullable) = the nine fluxes
 * txx tyy tzz txy txz tyz ex ey ez, xb4/gb12 = their VJP with Vbar9. */
int ns3d_debug_face_vjp(int direction, int interpolation, int riemann, double gamma, const double *lin,
                        const double *U30, const double *Fbar5, double *out30, double *flux5);
int ns3d_debug_visc_vjp(double mu0, double S, double cp_over_pr, const double *x4, const double *g12,
                        const double *Vbar9, double *xb4, double *gb12, double *V9);
/* Host evaluation of the production face flux F(UL, UR) of one Riemann solver
 * (NS3D_ROE ... NS3D_STEGER_WARMING) along direction 0/1/2, FP64.  Replaces no
 * reference entry point (the reference's solvers are the static functions of
 * InviscousFlux.cpp:270-846); for unit tests of the flux functions. */
int ns3d_debug_riemann(int direction, int riemann, double gamma, const double UL[5], const double UR[5],
                       double F[5]);
/* The MDCD_HYBRID discontinuity detector of the FP64 sweeps evaluated on the
 * device: smooth_out[i] = 1 when sai(a, b) > 0.4 at the centre of the
 * five-point stencil stencils[5i .. 5i+4] (the reference's sigma test of one
 * centre, mdcd_hybrid_interpolate, interpolation.cpp:149-160), else 0.
 * n <= 2^26.  For tests of near-threshold decisions; allocates and frees its
 * own device buffers. */
int ns3d_debug_mdcd_detector(int device, long n, const double *stencils, int *smooth_out);
/* Runs the bounded mbarrier wait of the TMA kernels against a barrier that
 * never completes (armed for bytes no copy delivers): each block gives up
 * after `polls` polls, writes the device error word (returned in *code_out)
 * and exits.  Returns NS3D_ERR_TIMEOUT when that happened, as the solver
 * entry points do when one of their TMA waits runs out.  No counterpart in
 * the reference; for tests of the failure path. */
int ns3d_debug_wait_timeout(int device, unsigned polls, int *code_out);

/* ------------------------------------------------ z-slab decomposition
 * A handle holding one rank's z-slab of a domain split along z over several
 * GPUs.  Replaces the reference's per-rank decomposition (build_cart_decomp /
 * compute_local_desc, field_structures.h:1062-1115) and its three exchanges
 * per stage (exchange_halos_physical :936-994, exchange_halos_halfnode_flux
 * :998-1056, exchange_halos_viscous_flux :877-932) by one: the local grid
 * holds the rank's owned interior planes [z_begin, z_end) plus six halo
 * planes on every side that borders another rank, whose primitives and
 * temperature the caller refreshes after every stage; the face and node
 * viscous fluxes the owned cells need are then computed locally from the
 * same inputs, so the owned cells equal a single-domain run bit for bit.
 * ns3d_set_slab: the owned planes (local interior indices; six planes or
 * more, and six halo planes on each bordering side; the local z boundary
 * types must be non-periodic -- their treatment stays inside the halo) and,
 * when dz > 0, the global grid spacing (so the local dz is the global one bit
 * for bit); z_periodic = 1 when the whole domain is periodic in z (both of
 * the slab's z sides are then halos).  The x/y sweeps then run over the owned planes, the viscous
 * fluxes over the owned planes and three halo planes each side, the z-sweep
 * updates owned cells only, and every reduction (time step, kinetic energy,
 * diagnostics) counts owned cells only.  ns3d_rk3_step / _steps /
 * time_advance and the adjoint return NS3D_ERR_STATE / NS3D_ERR_CONFIG on a
 * slab.
 * ns3d_rk3_stage: one RK3 stage (1, 2, 3, in order) of a step, enqueued on
 * the handle's stream without synchronising; the halo planes of the stage's
 * result are then exchanged through the pointers of ns3d_device_fields
 * (NS3D_PRIMITIVE and NS3D_TEMPERATURE), as runge_kutta_3's apply_boundary
 * does after every stage (range_kutta.cpp:61-63). */
int ns3d_set_slab(ns3d_handle *h, int z_begin, int z_end, double dz, int z_periodic);
int ns3d_rk3_stage(ns3d_handle *h, int stage, double dt);

/* ---------------------------------------- scratch-free CFL time step
 * No counterpart in the reference.  For host codes that cannot let a library
 * allocate device memory -- solvers that hand out every device byte from
 * their own pre-sized pool, where a stray allocation breaks their memory
 * accounting or fails once the pool holds the GPU's memory -- this computes
 * what ns3d_compute_timestep computes
 * (compute_timestep, timestep.cpp:5-23) without a handle and without calling
 * cudaMalloc, cudaFree or any allocating routine.
 *   d_fields  five caller-owned device arrays rho, u, v, w, p in the unpadded
 *             Field3D layout (sx*sy*sz doubles, sx = nx+6, ...);
 *   d_dt_out  caller-owned device double receiving cfl * min dx/(|u|+a);
 *   stream    cudaStream_t as void* (NULL: the default stream); the call only
 *             enqueues work and returns before the result is ready.
 * Limit: nx*ny*nz <= NS3D_NOALLOC_MAX_CELLS (2^27, e.g. 512^3); larger grids
 * return NS3D_ERR_SIZE.  Its scratch is one fixed 128 KB device array of
 * per-block partials (NS3D_NOALLOC_MAX_BLOCKS doubles) that every GPU which
 * loads the library holds until the process exits.  All calls share that
 * array, so calls that overlap on a GPU (other streams or host threads) race
 * on it: serialise them.  The first call in a CUDA context looks up the
 * array's device address (cudaGetSymbolAddress) and caches it for that
 * context; make that first call before any stream capture, once per device,
 * and again after cudaDeviceReset or a switch to another context on the
 * device (each of which loads the library's module at a new address). */
#define NS3D_NOALLOC_MAX_BLOCKS 16384
#define NS3D_NOALLOC_MAX_CELLS (16384L * 256 * 32)
int ns3d_compute_timestep_noalloc(const double *const d_fields[5], int nx, int ny, int nz, double gamma,
                                  double cfl, double dx, double *d_dt_out, void *stream);

#ifdef __cplusplus
}
#endif
#endif
