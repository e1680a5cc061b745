"""The scratch-free CFL time step (ns3d_compute_timestep_noalloc).

Callers that cannot let the library allocate device memory -- codes that own
every device byte through their own pool, or that capture their time loop
into a CUDA graph -- pass their own device arrays and a device result slot;
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


def test_noalloc_rejects_grids_beyond_its_scratch(gpu_lib):
    import torch
    lib = _lib.load()
    P, G = make_params(n=(8, 8, 8))
    dummy = [torch.zeros(1, dtype=torch.float64, device="cuda") for _ in range(5)]
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    big = (1024, 512, 257)  # 2^27 + 2^19 cells > NS3D_NOALLOC_MAX_CELLS
    assert _call(lib, dummy, big, P, G, out, 0) == -10
