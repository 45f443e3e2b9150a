"""Failure detection without a GPU fault (the reference ends such runs with
CkAbort / EXIT: ortho.C:129-133, cp_lowdin.C:246-252):

* a pipeline wait of a tcgen05 product runs out of time because a host-set
  hook made one block skip the loads of one stage: the block takes its
  error path (loads landed, TMEM freed), oa_gpu_check reports it once, and
  the context gives the right product on the next call;
* a non-finite coefficient and a singular overlap matrix injected from the
  host: the native run returns OA_ERR_NONFINITE / OA_ERR_NOT_CONVERGED and
  names the first failing step."""
import time

import numpy as np
import pytest

from openatom_b200.system import make_system

pytestmark = pytest.mark.gpu


def test_bounded_wait_runs_out_and_is_reported():
    import torch
    from openatom_b200.gpu import CPContext, OaError, OA_ERR_CUDA
    s = make_system("w8", nstate=16, seed=31)
    ctx = CPContext(s, "mixed")
    rng = np.random.default_rng(3)
    psi = torch.from_numpy(s.psi).cuda()
    F = torch.from_numpy((rng.standard_normal(s.psi.shape) + 1j * rng.standard_normal(s.psi.shape)) * 0.1).cuda()
    lam0 = torch.zeros(s.nstate, s.nstate, dtype=torch.float64, device="cuda")
    ctx.pc_forward_mixed(psi, F, 1.0, 1.0, lam0)
    ctx.check()
    ctx.fault_inject(1)
    lam1 = torch.zeros_like(lam0)
    t0 = time.perf_counter()
    ctx.pc_forward_mixed(psi, F, 1.0, 1.0, lam1)
    with pytest.raises(OaError) as ei:
        ctx.check()
    dt = time.perf_counter() - t0
    assert ei.value.status == OA_ERR_CUDA and "ran out of time" in str(ei.value)
    # one 200 ms wait (plus the bounded clean-up waits), not an iteration count
    assert 0.15 < dt < 10.0, dt
    # the failed block's partial was zeroed: the product differs, is finite
    got = lam1.cpu().numpy()
    assert np.all(np.isfinite(got)) and not np.array_equal(got, lam0.cpu().numpy())
    # reported once; the context is usable and the hook was consumed
    ctx.check()
    lam2 = torch.zeros_like(lam0)
    ctx.pc_forward_mixed(psi, F, 1.0, 1.0, lam2)
    ctx.check()
    assert np.array_equal(lam2.cpu().numpy(), lam0.cpu().numpy())
    ctx.close()


def test_nonfinite_coefficient_names_the_step():
    from openatom_b200.gpu import CPDriver, OaError, OA_ERR_NONFINITE
    s = make_system("w2", seed=32, dt=0.5)
    d = CPDriver(s, "fp64")
    d.psi[1, 7] = float("nan")
    d.psi_t[1, 7] = float("nan")
    st = d.native_state(use_graph=True)
    with pytest.raises(OaError) as ei:
        d.run_native(st, 3)
    assert ei.value.status == OA_ERR_NONFINITE
    assert "step 1 of 3" in str(ei.value)


def test_singular_overlap_names_the_step():
    """Two equal states make S singular: the Schulz iteration cannot reach
    its tolerance (it overflows), the run reports the first step."""
    from openatom_b200.gpu import CPDriver, OaError, OA_ERR_NONFINITE, OA_ERR_NOT_CONVERGED
    s = make_system("w2", seed=33, dt=0.5)
    p0 = s.psi.copy()
    p0[1] = p0[0]
    d = CPDriver(s, "fp64", psi0=p0)
    st = d.native_state(use_graph=True)
    with pytest.raises(OaError) as ei:
        d.run_native(st, 2)
    assert ei.value.status in (OA_ERR_NONFINITE, OA_ERR_NOT_CONVERGED)
    assert "step 1 of 2" in str(ei.value)
