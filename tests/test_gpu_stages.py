"""Stage-by-stage parity of the CUDA path (through the C ABI) with the CPU
oracle, FP64 form: energies to 1e-10 relative, coefficient forces to 1e-9
relative (max abs error over max abs value)."""
import math

import numpy as np
import pytest

from openatom_b200.system import make_system
from oracle import cp_oracle as O

pytestmark = pytest.mark.gpu

E_TOL = 1e-10
F_TOL = 1e-9


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture(scope="module", params=["w2", "w4", "w8", "w32"])
def case(request):
    import torch
    from openatom_b200.gpu import CPContext
    nst = {"w2": None, "w4": None, "w8": 16, "w32": 8}[request.param]
    s = make_system(request.param, nstate=nst, seed=7)
    ctx = CPContext(s, "fp64")
    psi = torch.from_numpy(s.psi).cuda()
    return s, ctx, psi


def test_density(case):
    import torch
    s, ctx, psi = case
    nx, ny, nz = s.nfft
    rho = torch.zeros(nz, ny, nx, dtype=torch.float64, device="cuda")
    ctx.state_fft_fwd(psi, rho)
    torch.cuda.synchronize()
    ref = O.density(O.state_g_to_r(s.psi, s), s)
    assert rel(rho.cpu().numpy(), ref) < 1e-11
    # total charge = 2 * nstate electrons
    assert abs(rho.sum().item() * s.vol / s.npts - 2.0 * s.nstate) < 1e-9


def test_vks_build_energies(case):
    import torch
    s, ctx, psi = case
    nx, ny, nz = s.nfft
    vks = torch.zeros(nz, ny, nx, dtype=torch.float64, device="cuda")
    ctx.state_fft_fwd(psi)
    ctx.vks_build(vks)
    en = ctx.energies()
    psir = O.state_g_to_r(s.psi, s)
    _, vref, eref = O.vks_build(psir, s)
    assert rel(vks.cpu().numpy(), vref) < 1e-10
    for k in ("EHART", "EEXT", "EEXC", "EWALD_RECIP", "MUXC"):
        assert abs(en[k] - eref[k]) <= E_TOL * max(1.0, abs(eref[k])), (k, en[k], eref[k])


def test_forces_eke(case):
    import torch
    s, ctx, psi = case
    nx, ny, nz = s.nfft
    rng = np.random.default_rng(3)
    v = rng.standard_normal((nz, ny, nx)) * 0.3
    ctx.set_vks(torch.from_numpy(v).cuda())
    f = torch.zeros_like(psi)
    eke = torch.zeros(s.nstate, dtype=torch.float64, device="cuda")
    ctx.vks_apply_fft_bwd(psi, f, recompute_fwd=True, eke_out=eke)
    torch.cuda.synchronize()
    psir = O.state_g_to_r(s.psi, s)
    fr = O.add_forces(O.vks_forces(psir, v, s), None, s)
    fr, ek = O.eke(s.psi, fr, s)
    assert rel(f.cpu().numpy(), fr) < F_TOL
    assert rel(eke.cpu().numpy(), ek) < E_TOL


def test_forces_from_stored_psi_r(case):
    """vks_apply_fft_bwd without recompute_fwd starts from the psi(r) the
    density pass stored; same forces as the recomputing path."""
    import torch
    s, ctx, psi = case
    nx, ny, nz = s.nfft
    rng = np.random.default_rng(6)
    v = rng.standard_normal((nz, ny, nx)) * 0.3
    ctx.state_fft_fwd(psi)
    ctx.set_vks(torch.from_numpy(v).cuda())
    f = torch.zeros_like(psi)
    eke = torch.zeros(s.nstate, dtype=torch.float64, device="cuda")
    ctx.vks_apply_fft_bwd(psi, f, recompute_fwd=False, eke_out=eke)
    torch.cuda.synchronize()
    psir = O.state_g_to_r(s.psi, s)
    fr = O.add_forces(O.vks_forces(psir, v, s), None, s)
    fr, ek = O.eke(s.psi, fr, s)
    assert rel(f.cpu().numpy(), fr) < F_TOL
    assert rel(eke.cpu().numpy(), ek) < E_TOL


def test_forces_with_nonlocal_input(case):
    import torch
    s, ctx, psi = case
    nx, ny, nz = s.nfft
    rng = np.random.default_rng(4)
    v = rng.standard_normal((nz, ny, nx)) * 0.1
    fnl = (rng.standard_normal(s.psi.shape) + 1j * rng.standard_normal(s.psi.shape)) * 1e-2
    ctx.set_vks(torch.from_numpy(v).cuda())
    f = torch.zeros_like(psi)
    ctx.vks_apply_fft_bwd(psi, f, fnl=torch.from_numpy(fnl).cuda(), recompute_fwd=True)
    torch.cuda.synchronize()
    psir = O.state_g_to_r(s.psi, s)
    fr, _ = O.eke(s.psi, O.add_forces(O.vks_forces(psir, v, s), fnl, s), s)
    assert rel(f.cpu().numpy(), fr) < F_TOL


def test_pc_forward_and_ortho(case):
    import torch
    s, ctx, psi = case
    rng = np.random.default_rng(5)
    pert = (rng.standard_normal(s.psi.shape) + 1j * rng.standard_normal(s.psi.shape)) * 2e-3 / (1 + s.g2())
    pt = O.sync_redundant(s.psi + pert, s)
    n = s.nstate
    S = torch.zeros(n, n, dtype=torch.float64, device="cuda")
    T = torch.zeros_like(S)
    ptg = torch.from_numpy(pt).cuda()
    ctx.pc_forward(ptg, ptg, 2.0, 0.5, S)
    torch.cuda.synchronize()
    new_ref, T_ref, S_ref, it_ref, err_ref = O.ortho_psi(pt, s)
    assert rel(S.cpu().numpy(), S_ref) < 1e-13
    it, err, ok = ctx.ortho_invsqrt(S, T, 1e-15, 1000)
    assert ok and it == it_ref
    assert rel(T.cpu().numpy(), T_ref) < 1e-12
    out = torch.zeros_like(ptg)
    ctx.pc_backward(T, ptg, 1.0, 1.0, out)
    torch.cuda.synchronize()
    o = out.cpu().numpy()
    assert rel(o, new_ref) < 1e-12
    from openatom_b200.system import gamma_overlap
    Snew = gamma_overlap(o, s.kx)
    assert np.max(np.abs(Snew - 2 * np.eye(n))) < 1e-12


def test_lambda_constraint(case):
    import torch
    s, ctx, psi = case
    rng = np.random.default_rng(6)
    n = s.nstate
    F = (rng.standard_normal(s.psi.shape) + 1j * rng.standard_normal(s.psi.shape)) * 0.1
    Tm = np.eye(n) + 1e-3 * rng.standard_normal((n, n))
    Tm = 0.5 * (Tm + Tm.T)
    fref, lref = O.lambda_step(s.psi, F, Tm, s)
    Fg = torch.from_numpy(F).cuda()
    Tg = torch.from_numpy(Tm).cuda()
    lam = torch.zeros(n, n, dtype=torch.float64, device="cuda")
    gam = torch.zeros_like(lam)
    out = torch.zeros_like(Fg)
    ctx.pc_forward(psi, Fg, 1.0, 1.0, lam)
    ctx.small_gemm(Tg, lam, 1.0, gam)
    ctx.pc_backward(gam, psi, -0.5, -1.0, out, M2=Tg, X2=Fg, a2=1.0)
    torch.cuda.synchronize()
    assert rel(lam.cpu().numpy(), lref) < 1e-12
    assert rel(out.cpu().numpy(), fref) < F_TOL


def test_integrate(case):
    import torch
    s, ctx, psi = case
    rng = np.random.default_rng(8)
    F = (rng.standard_normal(s.psi.shape) + 1j * rng.standard_normal(s.psi.shape)) * 0.01
    V = (rng.standard_normal(s.psi.shape) + 1j * rng.standard_normal(s.psi.shape)) * 0.001
    P = s.psi.copy()
    Fg, Vg, Pg = (torch.from_numpy(a.copy()).cuda() for a in (F, V, P))
    ctx.integrate(Fg, Vg, Pg, s.dt, True)
    en = ctx.energies()
    v1 = O.evolve_vel(F, V, s.cmass, s.dt, s)
    ke = O.fict_ke(v1, s.cmass, s).sum()
    v2 = O.evolve_vel(F, v1, s.cmass, s.dt, s)
    p2 = P.copy()
    p2[:, s.nkx0_red:] += v2[:, s.nkx0_red:] * s.dt
    p2 = O.sync_redundant(p2, s)
    v2 = O.sync_redundant(v2, s)
    assert rel(Vg.cpu().numpy(), v2) < 1e-13
    assert rel(Pg.cpu().numpy(), p2) < 1e-13
    assert abs(en["FICT_KE"] - ke) <= 1e-12 * max(ke, 1e-30)


def test_nonlocal_structure_factor(case):
    import torch
    s, ctx, psi = case
    f = torch.zeros_like(psi)
    enl = torch.zeros(s.nstate, dtype=torch.float64, device="cuda")
    ctx.nl_sf(psi, f, nterm=0, enl_out=enl)
    torch.cuda.synchronize()
    fr, er, _ = O.nl_energy_forces(s.psi, s)
    assert rel(f.cpu().numpy(), fr) < 1e-12
    assert rel(enl.cpu().numpy(), er) < 1e-12
    assert abs(ctx.energies()["ENL"] - er.sum()) <= 1e-12 * abs(er.sum())


@pytest.mark.parametrize("order,scale", [(6, 1.2), (4, 1.6)])
def test_nonlocal_ees(case, order, scale):
    """EES nonlocal path on the GPU against the oracle's EES restatement
    (FP64: energies 1e-10, forces 1e-9)."""
    import torch
    s, ctx, psi = case
    grid = ctx.ees_init(scale, order)
    ees = O.ees_setup(s, scale, order)
    assert tuple(grid) == tuple(ees["grid"])
    f = torch.zeros_like(psi)
    enl = torch.zeros(s.nstate, dtype=torch.float64, device="cuda")
    ctx.nl_ees(psi, f, enl_out=enl)
    torch.cuda.synchronize()
    fr, er, _ = O.nl_ees_energy_forces(s.psi, s, ees)
    assert rel(enl.cpu().numpy(), er) < 1e-10
    assert rel(f.cpu().numpy(), fr) < 1e-9
