"""BLYP gradient correction on the GPU (oa_gpu_set_xc functional 1): the
density path's grad rho transforms, the per-point Becke 88 / LYP functional
and the white-byrd divergence, against the oracle (pinned to compiled
cp_becke.C / cp_grad_rho_ctrl.C).

* vks_build: V_KS(r) to 1e-10 relative and every energy term (EGGA
  included) to 1e-10, on grids with two-pass kernels (24^3, 36^3, 64^3)
  and on one without (30^3: the runtime-plan transforms);
* the native graphed FP64 step: 8 waters with all 32 states, five CPMD
  steps at dt = 5, each energy term to 1e-10 and the coefficients to 1e-9;
* the mixed form from a quenched start: the total energy within 1e-6
  Ha/atom of the oracle;
* switching the functional back to PZ-LDA re-captures the step graph."""
import numpy as np
import pytest

from openatom_b200.system import make_system
from oracle import cp_oracle as O

pytestmark = pytest.mark.gpu

E_TOL = 1e-10
C_TOL = 1e-9
TERMS = ("EKE", "EHART", "EEXT", "EEXC", "ENL", "EGGA")


def _rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(np.asarray(b))), 1e-300))


@pytest.mark.parametrize("preset,nfft,nstate", [("w2", None, None), ("w4", None, None), ("w8", None, 16),
                                                 ("w2", (30, 30, 30), None)])
def test_vks_build_blyp(preset, nfft, nstate):
    import torch
    from openatom_b200.gpu import CPContext
    over = {} if nfft is None else {"nfft": nfft}
    s = make_system(preset, seed=11, nstate=nstate, xc="blyp", **over)
    ctx = CPContext(s, "fp64")
    nx, ny, nz = s.nfft
    psi = torch.from_numpy(s.psi).cuda()
    vks = torch.zeros(nz, ny, nx, dtype=torch.float64, device="cuda")
    ctx.state_fft_fwd(psi)
    ctx.vks_build(vks)
    en = ctx.energies()
    _, vref, eref = O.vks_build(O.state_g_to_r(s.psi, s), s)
    assert eref["EGGA"] < 0.0
    assert _rel(vks.cpu().numpy(), vref) < 1e-10
    for k in ("EHART", "EEXT", "EEXC", "EWALD_RECIP", "MUXC", "EGGA"):
        assert abs(en[k] - eref[k]) <= E_TOL * max(1.0, abs(eref[k])), (k, en[k], eref[k])
    # back to PZ-LDA on the same context: EGGA is 0 and V_KS is the LDA one
    ctx.set_xc("pz_lda")
    ctx.state_fft_fwd(psi)
    ctx.vks_build(vks)
    s.xc = "pz_lda"
    _, vlda, elda = O.vks_build(O.state_g_to_r(s.psi, s), s)
    assert ctx.energies()["EGGA"] == 0.0
    assert _rel(vks.cpu().numpy(), vlda) < 1e-10
    ctx.close()


def _blyp_w8():
    return make_system("w8", seed=2024, ecut_mass=2.0, cmass0=400.0, dt=5.0, xc="blyp")


def test_blyp_native_steps_fp64():
    from openatom_b200.gpu import CPDriver
    s = _blyp_w8()
    st = O.CPState(s)
    ref = [O.cp_step(st, s, norb_tol=0.003) for _ in range(5)]
    d = CPDriver(s, "fp64", norb_tol=0.003)
    got = d.run_native(d.native_state(use_graph=True), 5)
    for i, (g, r) in enumerate(zip(got, ref)):
        for k in TERMS + ("FICT_KE",):
            assert abs(g[k] - r[k]) <= E_TOL * max(1.0, abs(r[k])), (i, k, g[k], r[k])
    assert _rel(d.psi.cpu().numpy(), st.psi) < C_TOL
    assert _rel(d.v.cpu().numpy(), st.v) < C_TOL
    d.ctx.close()


def test_blyp_native_steps_mixed():
    """From a quenched start (three damped FP64 steps at dt = 5, then 27 at
    dt = 10 on the GPU; the FP64 form is pinned above), where the energy
    terms have their physical size, as in the mixed-form benchmark."""
    from openatom_b200.gpu import CPDriver
    s = _blyp_w8()
    q = CPDriver(s, "fp64")
    q.quench(3)
    q.quench(27, dt=10.0)
    psi0 = q.psi.cpu().numpy()
    q.ctx.close()
    st = O.CPState(s)
    st.psi_t = psi0.copy()
    st.psi = psi0.copy()
    ref = [O.cp_step(st, s, norb_tol=0.003) for _ in range(5)]
    d = CPDriver(s, "mixed", psi0=psi0, norb_tol=0.003)
    got = d.run_native(d.native_state(use_graph=True), 5)
    natm = s.natm
    for g, r in zip(got, ref):
        tot_g = sum(g[k] for k in TERMS)
        tot_r = sum(r[k] for k in TERMS)
        assert abs(tot_g - tot_r) / natm <= 1e-6, (tot_g, tot_r)
        assert abs(g["EGGA"] - r["EGGA"]) / natm <= 1e-6
    d.ctx.close()
