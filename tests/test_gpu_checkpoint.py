"""Asynchronous checkpoint (cube_gpu_checkpoint_async) against the state it snapshots.

The files of one image (checkpoint.f90:11-39: info, xp, vp, np, id) are written by the
library's writer thread while the host keeps stepping (eager and graph steps); they must
hold the state of the moment of the call byte for byte, and read back with the
reference-layout reader (particle_initialization.f90:31-90)."""
import numpy as np
import pytest

from cube_nu_b200 import checkpoint
from cube_nu_b200.params import DEPOSIT_FIXED, config_small
from tests.helpers import lattice_state

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("graph", [False, True])
def test_checkpoint_async_matches_snapshot(tmp_path, graph):
    from cube_nu_b200._lib import Context

    p = config_small(ng=64, nnt=2, nns=2, np_nc=2, izipx=2)
    p.deposit_mode = DEPOSIT_FIXED
    p.step_graph = graph
    st = lattice_state(p, seed=5, disp=0.3, vscale=0.5)
    n = st[0].shape[0]
    p.mass_p_cdm = float(p.ng) ** 3 / n
    with Context(p) as ctx:
        ctx.upload(*st)
        vz = float(np.abs(st[1][:, 2]).max())
        so = ctx.step(0.3, 0.0, 0.05, vz)
        snap = ctx.download()
        h = checkpoint.new_header(nplocal=n, npglobal=n, izipx=2, izipv=2, a=0.05, mass_p_cdm=p.mass_p_cdm,
                                  timestep=1, box=p.box)
        ctx.checkpoint_async(str(tmp_path), 1, 19.0, h)
        # the run goes on while the files are written
        for k in range(3):
            so = ctx.step(0.3, 0.3, 0.06 + 0.01 * k, so.vz_max)
        after = ctx.download()
        ctx.checkpoint_wait()
    back = checkpoint.read(str(tmp_path), 1, 19.0, 2)
    for a, b, name in zip((back.xp, back.vp, back.pid, back.rhoc), snap, ("xp", "vp", "pid", "rhoc")):
        assert np.array_equal(a, b), name
    assert back.header.tobytes() == h.tobytes()
    assert not np.array_equal(after[1], snap[1])  # the state did move on meanwhile
