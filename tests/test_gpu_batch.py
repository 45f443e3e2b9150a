"""Batching form (oa_gpu_cp_run_batch): several independent systems of
different sizes advanced together, one CUDA graph per step with the systems
on concurrent streams.  Each system's energies and coefficients match its
own single-system run (oa_gpu_cp_run) bit for bit."""
import numpy as np
import pytest

from openatom_b200.system import make_system

pytestmark = pytest.mark.gpu

# (preset, states, seed): uneven sizes and grids (the whole step is one graph
# per system: even state counts, at most 128)
SYSTEMS = [("w2", None, 21), ("w2", 6, 22), ("w4", 12, 23), ("w8", 16, 24)]


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_batch_matches_single_runs(precision):
    from openatom_b200.gpu import CPDriver, run_batch
    nsteps = 4
    syss = [make_system(p, nstate=n, seed=sd, dt=0.5) for p, n, sd in SYSTEMS]
    single = [CPDriver(s, precision) for s in syss]
    ref = []
    for d in single:
        st = d.native_state(use_graph=True)
        ref.append(d.run_native(st, nsteps))
    batch = [CPDriver(s, precision) for s in syss]
    states = [d.native_state(use_graph=True) for d in batch]
    got = run_batch(batch, states, nsteps)
    for i in range(len(syss)):
        for k in range(nsteps):
            for key in ("EKE", "EHART", "EEXT", "EEXC", "ENL", "FICT_KE", "SMAX"):
                assert got[i][k][key] == ref[i][k][key], (i, k, key, got[i][k][key], ref[i][k][key])
        assert np.array_equal(batch[i].psi.cpu().numpy(), single[i].psi.cpu().numpy())
        assert np.array_equal(batch[i].v.cpu().numpy(), single[i].v.cpu().numpy())
    # one graph per steady step holds the kernels of every system
    assert states[0].last_kernels > 4 * 20


def test_batch_rejects_bad_input():
    """A context that appears twice is refused before anything runs."""
    import torch
    from openatom_b200.gpu import CPDriver, run_batch, OaError
    s = make_system("w2", seed=25, dt=0.5)
    d = CPDriver(s, "fp64")
    st = d.native_state()
    with pytest.raises(OaError):
        run_batch([d, d], [st, d.native_state()], 2)
