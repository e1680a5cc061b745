"""ns3d_batch_create rejects what the batched solver does not run -- before
any device call, so these run without a GPU: viscous problems, non-periodic
y/z (the quasi-1D cross-section is periodic), the mixed path, characteristic
reconstruction and the ZERO interpolation."""
import math

import pytest

from ns3d_wcns_b200 import _lib
from ns3d_wcns_b200.batch import Batch
from ns3d_wcns_b200.config import GridDesc, make_params


def _params(**kw):
    base = dict(n=(8, 4, 4), Ma=1.0, Re=math.inf, cfl=0.5, dt_fixed=-1.0, interpolation=0, riemann=0,
                bcs=(3, 3, 0, 0, 0, 0))
    base.update(kw)
    P, _ = make_params(**base)
    return P


GRIDS = [GridDesc(global_nx=16, global_ny=4, global_nz=4, Lx=1.0, Ly=1.0, Lz=1.0)]


@pytest.mark.parametrize("kw", [dict(Re=400.0), dict(bcs=(3, 3, 1, 1, 0, 0)), dict(bcs=(3, 3, 0, 0, 3, 3)),
                                dict(precision=1), dict(char_recon=True), dict(interpolation=1)],
                         ids=["viscous", "wall_y", "outflow_z", "mixed", "char_recon", "zero_interp"])
def test_unsupported_batches_rejected_before_device(kw):
    with pytest.raises(_lib.Ns3dError) as e:
        Batch(_params(**kw), GRIDS, [0.1])
    assert e.value.status == -2  # NS3D_ERR_CONFIG
