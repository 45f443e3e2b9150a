"""Full CP dynamics steps: the GPU host runner against the oracle's cp_step,
FP64 form; each energy term to 1e-10 relative, coefficients to 1e-9."""
import numpy as np
import pytest

from openatom_b200.system import make_system
from oracle import cp_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("preset,nst,nsteps", [("w2", None, 4), ("w8", 16, 3)])
def test_cp_steps_match_oracle(preset, nst, nsteps):
    from openatom_b200.gpu import CPDriver
    s = make_system(preset, nstate=nst, seed=11, dt=0.5)
    st = O.CPState(s)
    drv = CPDriver(s, "fp64", norb_tol=1e30)
    for i in range(nsteps):
        ref = O.cp_step(st, s)
        got = drv.step()
        for k in ("EKE", "EHART", "EEXT", "EEXC", "ENL", "FICT_KE"):
            tol = 1e-10 * max(1.0, abs(ref[k]))
            assert abs(got[k] - ref[k]) <= tol, (i, k, got[k], ref[k])
        assert got["ORTHO_ITERS"] == ref["ORTHO_ITERS"]
        psi = drv.psi.cpu().numpy()
        assert np.max(np.abs(psi - st.psi)) / np.max(np.abs(st.psi)) < 1e-9


@pytest.mark.parametrize("use_graph", [False, True])
def test_native_step_matches_host_runner(use_graph):
    """oa_gpu_cp_step (native sequencing, optional CUDA graph) reproduces the
    host-sequenced step bit for bit in the FP64 form."""
    from openatom_b200.gpu import CPDriver
    s = make_system("w8", nstate=16, seed=12, dt=0.5)
    a = CPDriver(s, "fp64")
    b = CPDriver(s, "fp64")
    st = b.native_state(use_graph=use_graph)
    for _ in range(4):
        ea = a.step()
        eb = b.step_native(st)
        for k in ("EKE", "EHART", "EEXT", "EEXC", "ENL", "FICT_KE"):
            assert eb[k] == ea[k], (k, ea[k], eb[k])
        assert np.array_equal(a.psi.cpu().numpy(), b.psi.cpu().numpy())
