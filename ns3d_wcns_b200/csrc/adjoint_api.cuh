// adjoint_api.cuh -- launch interface of the adjoint kernels (adjoint.cu).
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"

namespace ns3d {

struct AdjArgs {
    const double *W[5];   // primitive state the RHS is linearised at (padded layout)
    const double *Rb[5];  // adjoint of the RHS (interior layout), read as rbs * Rb
    double rbs;           // scale applied to Rb
    double *Ub[5];        // adjoint of the conserved state, accumulated (interior layout)
    double *G[30];        // face-VJP scratch: 6 stencil cells x 5 variables per face
    double *X[16];        // viscous scratch: (u,v,w,T) adjoints + 12 gradient adjoints per node
    Layout L;
    double inv_h[3];
    double gamma, Rgas, mu0, S, cpr;
    int interp, riemann;  // public values (NS3D_WENO5 ... ; NS3D_ROE ...)
    double lin[6];        // MDCD linear coefficients
    double hd[4];         // MDCD_HYBRID WENO weights d0..d3
    int first;            // 1: the x-direction gather overwrites Ub
};

cudaError_t adj_rhs_vjp(const AdjArgs &a, cudaStream_t st, long *launches);
cudaError_t adj_axpby(double *const *y, const double *const *x, double alpha, double beta, long n, cudaStream_t st);
// the linear combinations of one RK3 step's backward pass (see vjp_step_async)
cudaError_t adj_step_combine(int which, double *const *tab, double dt, long n, cudaStream_t st);
cudaError_t adj_ke_seed(const AdjArgs &a, double vol, double *const *Ub, cudaStream_t st);
cudaError_t adj_velocity_grad(const AdjArgs &a, const double *const *Ub, double *const *gvel, cudaStream_t st);

}  // namespace ns3d
