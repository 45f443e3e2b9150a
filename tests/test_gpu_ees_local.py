"""The EES local pseudopotential and reciprocal Ewald path
(oa_gpu_set_ees_local, cp_eext_ees_opt on) against the oracle's EES
restatement (hart_eext_ees, pinned to compiled cp_hart_ext.C): the density
pass energies and V_KS, and ion dynamics whose local and reciprocal Ewald
atom forces come from the back-transformed B-spline grids.

FP64 form: energies to 1e-10 relative, V_KS to 1e-10 of its scale,
positions and velocities to 1e-10 of their scale."""
import copy

import numpy as np
import pytest

from openatom_b200.system import make_system
from oracle import cp_oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("preset,nstate,order", [("w2", None, 4), ("w8", 16, 6), ("w32", 8, 4)])
def test_vks_build_ees_local(preset, nstate, order):
    import torch
    from openatom_b200.gpu import CPContext
    s = make_system(preset, nstate=nstate, seed=7, eext_ees_order=order)
    ctx = CPContext(s, "fp64")
    psi = torch.from_numpy(s.psi).cuda()
    nx, ny, nz = s.nfft
    vks = torch.zeros(nz, ny, nx, dtype=torch.float64, device="cuda")
    ctx.state_fft_fwd(psi)
    ctx.vks_build(vks)
    en = ctx.energies()
    _, vref, eref = O.vks_build(O.state_g_to_r(s.psi, s), s)
    assert rel(vks.cpu().numpy(), vref) < 1e-10
    for k in ("EHART", "EEXT", "EEXC", "EWALD_RECIP", "MUXC"):
        assert abs(en[k] - eref[k]) <= 1e-10 * max(1.0, abs(eref[k])), (k, en[k], eref[k])
    # and back to the structure-factor method on the same context
    ctx.set_ees_local(None)
    ctx.vks_build(vks)
    en2 = ctx.energies()
    s_sf = copy.copy(s)
    s_sf.eext_ees = None
    _, vsf, esf = O.vks_build(O.state_g_to_r(s.psi, s), s_sf)
    assert rel(vks.cpu().numpy(), vsf) < 1e-10
    assert abs(en2["EEXT"] - esf["EEXT"]) <= 1e-10 * abs(esf["EEXT"])
    ctx.close()


@pytest.mark.parametrize("preset,nstate,order", [("w2", None, 4), ("w8", 16, 6)])
def test_ion_dynamics_ees_local_fp64(preset, nstate, order):
    from openatom_b200.gpu import CPDriver
    s = make_system(preset, seed=41, nstate=nstate, ecut_mass=2.0, cmass0=400.0, dt=5.0, eext_ees_order=order)
    rng = np.random.default_rng(41)
    m = O.atom_masses(s)
    vel = rng.standard_normal(s.pos.shape) * np.sqrt(300.0 * 3.1668115634556e-6 / m)[:, None]
    d = CPDriver(s, "fp64", norb_tol=0.003)
    d.ctx.set_ions(m, vel)
    got = d.run_native(d.native_state(use_graph=True), 6)
    so = copy.deepcopy(s)
    st = O.CPState(so)
    ions = O.IonState(so, vel)
    ref = [O.cp_step(st, so, norb_tol=0.003, ions=ions) for _ in range(6)]
    for i, (g, r) in enumerate(zip(got, ref)):
        for k in ("EKE", "EHART", "EEXT", "EEXC", "ENL", "FICT_KE", "ION_KE"):
            assert abs(g[k] - r[k]) <= 1e-10 * max(1.0, abs(r[k])), (i, k, g[k], r[k])
    pos, v = d.ctx.get_ions()
    assert np.max(np.abs(pos - so.pos)) <= 1e-10 * np.max(np.abs(so.pos))
    assert np.max(np.abs(v - ions.v)) <= 1e-10 * np.max(np.abs(ions.v))
    assert np.max(np.abs(pos - s.pos)) > 1e-4
    d.ctx.close()


def test_ees_local_refuses_small_grid():
    from openatom_b200.gpu import CPContext, OaError
    s = make_system("w2", seed=3)
    ctx = CPContext(s, "fp64")
    with pytest.raises(OaError):
        ctx.set_ees_local((16, 16, 16), 4)     # smaller than the density sphere
    with pytest.raises(OaError):
        ctx.set_ees_local((98, 98, 98), 4)     # 98 = 2 * 7^2: no radix plan
    with pytest.raises(OaError):
        ctx.set_ees_local((64, 64, 64), 5)     # odd order
    ctx.close()
