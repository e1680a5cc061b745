"""Adjoint (VJP) through the C ABI, against central finite differences.

* RHS and RK3-step VJPs: <rbar, (R(U + h dU) - R(U - h dU)) / 2h> = <VJP(rbar), dU>;
* the kinetic-energy gradient with checkpointing (ns3d_adjoint_kinetic_energy):
  (J(u + h d) - J(u - h d)) / 2h = <grad, d> for random directions d of the
  initial velocity at fixed rho and p;
* a torch.autograd.Function wrapper of compute_rhs / ns3d_vjp_rhs (test
  harness only) reproduces the same directional derivative through autograd.
"""
import numpy as np
import pytest

from ns3d_wcns_b200.config import make_params
from ns3d_wcns_b200.initial import isotropic_state

pytestmark = pytest.mark.gpu
GAMMA = 1.4


def c2p(U):
    rho = U[0]
    u, v, w = U[1] / rho, U[2] / rho, U[3] / rho
    p = (GAMMA - 1) * (U[4] - 0.5 * rho * (u * u + v * v + w * w))
    return rho, u, v, w, p


def p2c(rho, u, v, w, p):
    return np.stack([rho, rho * u, rho * v, rho * w, p / (GAMMA - 1) + 0.5 * rho * (u * u + v * v + w * w)])


def interior(x):
    return x[..., 3:-3, 3:-3, 3:-3]


def embed(x_int, shape):
    out = np.zeros((x_int.shape[0],) + shape)
    out[:, 3:-3, 3:-3, 3:-3] = x_int
    return out


# (interpolation, riemann): WENO5+Roe, MDCD_LINEAR+Rusanov, WENO5+HLL, and the benchmark
# scheme MDCD_HYBRID+HLLC (the detector a switch: zero derivative, active branch differentiated)
SCHEMES = [(0, 0), (2, 1), (0, 3), (3, 2), (2, 2)]


def setup(n, interp, rs, Re=200.0):
    from ns3d_wcns_b200.solver import Solver
    P, G = make_params(n=n, Ma=0.3, Re=Re, Pr=0.72, interpolation=interp, riemann=rs, dt_fixed=2e-3)
    st = isotropic_state(n, P.gamma, P.Ma, seed=11)
    return Solver(P, G), P, G, st


@pytest.mark.parametrize("scheme,n", [(sc, (16, 12, 10)) for sc in SCHEMES] +
                         # lines longer than 256 cells take the two-kernel face store path
                         [(SCHEMES[0], (260, 6, 5)), (SCHEMES[2], (5, 6, 260))])
def test_vjp_rhs_dot_product(gpu_lib, scheme, n):
    s, P, G, st = setup(n, *scheme)
    rng = np.random.default_rng(3)
    with s:
        U0 = p2c(*st)
        rbar = rng.standard_normal((5,) + n[::-1])
        dU = rng.standard_normal((5,) + n[::-1]) * np.abs(U0).mean(axis=(1, 2, 3))[:, None, None, None] * 1e-2
        s.set_interior_primitives(*st)
        ub = interior(s.vjp_rhs(embed(rbar, s.shape)))
        h = 1e-6
        Rs = []
        for sgn in (1, -1):
            s.set_interior_primitives(*c2p(U0 + sgn * h * dU))
            s.compute_rhs()
            Rs.append(interior(s.rhs()))
        fd = np.sum(rbar * (Rs[0] - Rs[1])) / (2 * h)
        ad = np.sum(ub * dU)
        assert abs(fd - ad) <= 1e-6 * abs(fd), (fd, ad)


@pytest.mark.parametrize("scheme", SCHEMES[:2] + SCHEMES[3:])
def test_vjp_rk3_step_dot_product(gpu_lib, scheme):
    n = (12, 12, 12)
    s, P, G, st = setup(n, *scheme)
    rng = np.random.default_rng(5)
    dt = 2e-3
    with s:
        U0 = p2c(*st)
        ubn = rng.standard_normal((5,) + n[::-1])
        dU = rng.standard_normal((5,) + n[::-1]) * np.abs(U0).mean(axis=(1, 2, 3))[:, None, None, None] * 1e-2
        s.set_interior_primitives(*st)
        ub = interior(s.vjp_rk3_step(dt, embed(ubn, s.shape)))
        # the state is unchanged by the VJP call
        np.testing.assert_allclose(interior(s.conserved()), U0, rtol=1e-14, atol=0)
        h = 1e-6
        Us = []
        for sgn in (1, -1):
            s.set_interior_primitives(*c2p(U0 + sgn * h * dU))
            s.rk3_step(dt)
            Us.append(interior(s.conserved()))
        fd = np.sum(ubn * (Us[0] - Us[1])) / (2 * h)
        ad = np.sum(ub * dU)
        assert abs(fd - ad) <= 1e-6 * abs(fd), (fd, ad)


@pytest.mark.parametrize("scheme", [(0, 0), (2, 2)], ids=["weno5_roe", "mdcd_linear_hllc"])
def test_kinetic_energy_gradient_against_fd(gpu_lib, scheme):
    """Config-4 shape at reduced size: Re 200, dt 2e-3, checkpoints + recompute."""
    n = (16, 16, 16)
    nsteps, ce = 30, 7
    s, P, G, st = setup(n, *scheme)
    rng = np.random.default_rng(9)
    with s:
        s.set_interior_primitives(*st)
        J, grad, stats = s.adjoint_kinetic_energy(nsteps, 2e-3, ce)
        # every segment but the last is recomputed from its checkpoint; the
        # last one keeps the stage states of the forward pass
        nck = -(-nsteps // ce)
        assert stats["recomputed_steps"] == (nck - 1) * ce
        # forward J agrees with a plain forward run
        s.set_interior_primitives(*st)
        s.rk3_steps(nsteps, 2e-3)
        assert abs(s.total_energy() - J) <= 1e-13 * J
        h = 1e-6
        for _ in range(3):
            d = rng.standard_normal((3,) + n[::-1])
            Jpm = []
            for sgn in (1, -1):
                rho, u, v, w, p = st
                s.set_interior_primitives(rho, u + sgn * h * d[0], v + sgn * h * d[1], w + sgn * h * d[2], p)
                s.rk3_steps(nsteps, 2e-3)
                Jpm.append(s.total_energy())
            fd = (Jpm[0] - Jpm[1]) / (2 * h)
            ad = float(np.sum(grad * d))
            assert abs(fd - ad) <= 1e-6 * abs(fd), (fd, ad)


def test_torch_autograd_function_wrapper(gpu_lib):
    torch = pytest.importorskip("torch")
    n = (12, 10, 8)
    s, P, G, st = setup(n, 0, 0)

    class RHS(torch.autograd.Function):
        """compute_rhs as an autograd op on the interior conserved state (test harness only)."""

        @staticmethod
        def forward(ctx, U):
            Un = U.detach().cpu().numpy()
            s.set_interior_primitives(*c2p(Un))
            s.compute_rhs()
            ctx.state = Un
            return torch.from_numpy(interior(s.rhs()).copy())

        @staticmethod
        def backward(ctx, rbar):
            s.set_interior_primitives(*c2p(ctx.state))
            ub = interior(s.vjp_rhs(embed(rbar.detach().cpu().numpy(), s.shape)))
            return torch.from_numpy(ub.copy())

    with s:
        U0 = torch.from_numpy(p2c(*st)).requires_grad_(True)
        R = RHS.apply(U0)
        rng = np.random.default_rng(1)
        rbar = torch.from_numpy(rng.standard_normal(R.shape))
        (g,) = torch.autograd.grad((R * rbar).sum(), U0)
        dU = torch.from_numpy(rng.standard_normal(U0.shape)) * 1e-2
        h = 1e-6
        with torch.no_grad():
            fd = ((RHS.apply(U0 + h * dU) - RHS.apply(U0 - h * dU)) * rbar).sum() / (2 * h)
        ad = (g * dU).sum()
        assert abs(float(fd - ad)) <= 1e-6 * abs(float(fd))


def test_checkpointed_gradient_equals_store_all_gradient(gpu_lib):
    """The plain backward pass (every stage state kept from the forward run:
    checkpoint interval = step count, nothing recomputed) and the checkpointed
    one with recompute give the same gradient bit for bit."""
    n = (12, 10, 8)
    nsteps = 24
    s, P, G, st = setup(n, 0, 0)
    with s:
        s.set_interior_primitives(*st)
        J1, g_plain, st1 = s.adjoint_kinetic_energy(nsteps, 2e-3, nsteps)
        assert st1["recomputed_steps"] == 0
        s.set_interior_primitives(*st)
        J2, g_ck, st2 = s.adjoint_kinetic_energy(nsteps, 2e-3, 5)
        assert st2["recomputed_steps"] == 20
    assert J1 == J2
    np.testing.assert_array_equal(g_plain, g_ck)
