"""The scratch-free CFL time step (ns3d_compute_timestep_noalloc).

Callers that cannot let the library allocate device memory -- codes that own
every device byte through their own pre-sized pool, where a library's
allocation breaks their accounting or fails -- pass their own device arrays
and a device result slot;
the entry point's only scratch is a fixed device array inside the library.
This file is collected last so that a failure here comes after every other
test has run.  Its result must equal ns3d_compute_timestep's on the same
state, on two calls in a row (the shared scratch keeps the previous call's
contents, which must not leak into the next result).
"""
import ctypes as C

import numpy as np
import pytest

from ns3d_wcns_b200 import _lib
from ns3d_wcns_b200.config import make_params
from ns3d_wcns_b200.initial import isotropic_state, random_state

pytestmark = pytest.mark.gpu


def _call(lib, fields, n, P, G, out, stream):
    ptrs = (C.c_void_p * 5)(*[f.data_ptr() for f in fields])
    return lib.ns3d_compute_timestep_noalloc(ptrs, n[0], n[1], n[2], P.gamma, P.cfl, G.dx,
                                             C.c_void_p(out.data_ptr()), C.c_void_p(stream))


@pytest.mark.parametrize("n,seed", [((24, 20, 16), 1), ((33, 17, 9), 2)])
def test_noalloc_timestep_matches_handle_entry_point(gpu_lib, n, seed):
    import torch
    from ns3d_wcns_b200.solver import Solver
    lib = _lib.load()
    P, G = make_params(n=n, Ma=0.3, cfl=0.5, dt_fixed=-1.0, bcs=(3, 3, 0, 0, 1, 1))
    st = isotropic_state(n, P.gamma, P.Ma, seed=seed) if n[0] == n[1] else random_state(n, seed=seed)
    with Solver(P, G) as s:
        s.set_interior_primitives(*st)
        expected = s.compute_timestep()
        W = s.primitives()                      # Field3D layout, (5, sz, sy, sx)
    torch.cuda.set_device(0)
    fields = [torch.from_numpy(np.ascontiguousarray(W[q])).cuda() for q in range(5)]
    stream = torch.cuda.current_stream().cuda_stream
    results = []
    for _ in range(2):
        out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
        assert _call(lib, fields, n, P, G, out, stream) == 0
        torch.cuda.synchronize()
        results.append(float(out.item()))
    for r in results:
        assert abs(r - expected) <= 1e-14 * expected
    assert results[0] == results[1]


def _handle_dt_and_fields(n, P, G, st):
    import torch
    from ns3d_wcns_b200.solver import Solver
    with Solver(P, G) as s:
        s.set_interior_primitives(*st)
        expected = s.compute_timestep()
        W = s.primitives()
    return expected, [torch.from_numpy(np.ascontiguousarray(W[q])).cuda() for q in range(5)]


def test_noalloc_multi_block_then_smaller_grid(gpu_lib):
    """64 x 48 x 40 needs 15 blocks of partials, so the combine reads several;
    a following call on a smaller grid whose minimum is larger writes fewer
    partials than the first call left behind, and must still return its own
    grid's time step (only the partials a call writes are read)."""
    import torch
    lib = _lib.load()
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream().cuda_stream
    big = (64, 48, 40)
    Pb, Gb = make_params(n=big, L=(2 * np.pi, 1.5 * np.pi, 1.25 * np.pi), Ma=0.3, cfl=0.5, dt_fixed=-1.0)
    st_big = random_state(big, seed=7, amp=0.3)
    small = (20, 12, 10)
    Ps, Gs = make_params(n=small, L=(2 * np.pi, 1.2 * np.pi, np.pi), Ma=0.3, cfl=0.5, dt_fixed=-1.0)
    st_small = random_state(small, seed=8, amp=0.05)
    # the small grid is coarser and its state slower (smaller |u| + a), so
    # its time step is larger than the big grid's: a leftover big-grid
    # partial would show
    st_small = [st_small[0], st_small[1] * 0.2, st_small[2] * 0.2, st_small[3] * 0.2, st_small[4]]
    exp_big, f_big = _handle_dt_and_fields(big, Pb, Gb, st_big)
    exp_small, f_small = _handle_dt_and_fields(small, Ps, Gs, st_small)
    assert exp_small > exp_big  # every big-grid partial is below the small grid's minimum
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    assert _call(lib, f_big, big, Pb, Gb, out, stream) == 0
    torch.cuda.synchronize()
    assert abs(float(out.item()) - exp_big) <= 1e-14 * exp_big
    out.fill_(-1.0)
    assert _call(lib, f_small, small, Ps, Gs, out, stream) == 0
    torch.cuda.synchronize()
    assert abs(float(out.item()) - exp_small) <= 1e-14 * exp_small
    # and the big grid once more, after the small one
    out.fill_(-1.0)
    assert _call(lib, f_big, big, Pb, Gb, out, stream) == 0
    torch.cuda.synchronize()
    assert abs(float(out.item()) - exp_big) <= 1e-14 * exp_big


def test_noalloc_rejects_grids_beyond_its_scratch(gpu_lib):
    import torch
    lib = _lib.load()
    P, G = make_params(n=(8, 8, 8))
    dummy = [torch.zeros(1, dtype=torch.float64, device="cuda") for _ in range(5)]
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    big = (1024, 512, 257)  # 2^27 + 2^19 cells > NS3D_NOALLOC_MAX_CELLS
    assert _call(lib, dummy, big, P, G, out, 0) == -10
