"""Mixed-precision form of the state FFT path (FP32 pencils; FP64 packing,
accumulation and energies) against the FP64 oracle.  FP32 transforms of
length <= 160 carry a relative error of a few 1e-7 per pass; the bounds
below (density 2e-6, forces and EES 1e-5 of the largest entry) leave a
factor of a few above what the three chained transforms give."""
import numpy as np
import pytest

from openatom_b200.system import make_system
from oracle import cp_oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


# (preset, states): the odd state counts leave the last state pair of the
# state-pair plane kernels half empty
CASES = [("w2", None), ("w2", 7), ("w4", 9), ("w8", 16), ("w8", 15), ("w32", 8), ("w32", 11)]


@pytest.fixture(scope="module", params=CASES, ids=[f"{p}-{n}" for p, n in CASES])
def case(request):
    import torch
    from openatom_b200.gpu import CPContext
    preset, nst = request.param
    s = make_system(preset, nstate=nst, seed=11)
    ctx = CPContext(s, "mixed")
    psi = torch.from_numpy(s.psi).cuda()
    return s, ctx, psi


def test_pair_plane_kernels_in_use(case):
    """The mixed form runs the density and V_KS plane passes two states per
    x transform on every grid of the presets."""
    s, ctx, psi = case
    z = ctx.sizes()
    assert z["pair_planes"] == 1
    assert z["ngroup_pair"] >= 1


def test_density_mixed(case):
    import torch
    s, ctx, psi = case
    nx, ny, nz = s.nfft
    rho = torch.zeros(nz, ny, nx, dtype=torch.float64, device="cuda")
    ctx.state_fft_fwd(psi, rho)
    torch.cuda.synchronize()
    ref = O.density(O.state_g_to_r(s.psi, s), s)
    assert rel(rho.cpu().numpy(), ref) < 2e-6
    # renormalised to the exact electron count of the FP64 coefficients
    # (the FP32 transforms alone leave it about 1.4e-7 low)
    q_exact = float(np.sum(s.occ * np.sum(s.kx_weight()[None, :] * np.abs(s.psi) ** 2, axis=1)))
    q = rho.sum().item() * s.vol / s.npts
    assert abs(q - q_exact) <= 1e-12 * q_exact, (q, q_exact)


def test_forces_mixed(case):
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
    assert rel(f.cpu().numpy(), fr) < 1e-5
    # EKE is computed in FP64 from the FP64 coefficients
    assert rel(eke.cpu().numpy(), ek) < 1e-12


def test_forces_from_stored_psi_r_mixed(case):
    """V_KS pass from the psi(r) pairs the density pass stored: the same
    forces as the oracle, twice in a row (the stored psi(r) is read, not
    consumed), and with a V_KS that changes between the calls."""
    import torch
    s, ctx, psi = case
    nx, ny, nz = s.nfft
    rng = np.random.default_rng(8)
    psir = O.state_g_to_r(s.psi, s)
    ctx.state_fft_fwd(psi)
    for rep in range(2):
        v = rng.standard_normal((nz, ny, nx)) * 0.3
        ctx.set_vks(torch.from_numpy(v).cuda())
        f = torch.zeros_like(psi)
        eke = torch.zeros(s.nstate, dtype=torch.float64, device="cuda")
        ctx.vks_apply_fft_bwd(psi, f, recompute_fwd=False, eke_out=eke)
        torch.cuda.synchronize()
        fr = O.add_forces(O.vks_forces(psir, v, s), None, s)
        fr, ek = O.eke(s.psi, fr, s)
        assert rel(f.cpu().numpy(), fr) < 1e-5, rep
        assert rel(eke.cpu().numpy(), ek) < 1e-12


def test_density_after_recompute_mixed(case):
    """A recomputing V_KS pass in between leaves the next density pass and
    the V_KS pass after it consistent."""
    import torch
    s, ctx, psi = case
    nx, ny, nz = s.nfft
    rng = np.random.default_rng(9)
    v = rng.standard_normal((nz, ny, nx)) * 0.2
    ctx.set_vks(torch.from_numpy(v).cuda())
    f = torch.zeros_like(psi)
    ctx.vks_apply_fft_bwd(psi, f, recompute_fwd=True)
    rho = torch.zeros(nz, ny, nx, dtype=torch.float64, device="cuda")
    ctx.state_fft_fwd(psi, rho)
    f2 = torch.zeros_like(psi)
    ctx.vks_apply_fft_bwd(psi, f2, recompute_fwd=False)
    torch.cuda.synchronize()
    psir = O.state_g_to_r(s.psi, s)
    assert rel(rho.cpu().numpy(), O.density(psir, s)) < 2e-6
    fr = O.eke(s.psi, O.add_forces(O.vks_forces(psir, v, s), None, s), s)[0]
    assert rel(f2.cpu().numpy(), fr) < 1e-5
    assert rel(f.cpu().numpy(), fr) < 1e-5


def test_ees_mixed(case):
    import torch
    s, ctx, psi = case
    ctx.ees_init(1.2, 6)
    ees = O.ees_setup(s, 1.2, 6)
    f = torch.zeros_like(psi)
    enl = torch.zeros(s.nstate, dtype=torch.float64, device="cuda")
    ctx.nl_ees(psi, f, enl_out=enl)
    torch.cuda.synchronize()
    fr, er, _ = O.nl_ees_energy_forces(s.psi, s, ees)
    assert rel(enl.cpu().numpy(), er) < 1e-5
    assert rel(f.cpu().numpy(), fr) < 1e-5
