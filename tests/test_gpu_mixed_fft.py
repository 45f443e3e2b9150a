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


@pytest.fixture(scope="module", params=["w2", "w8", "w32"])
def case(request):
    import torch
    from openatom_b200.gpu import CPContext
    nst = {"w2": None, "w8": 16, "w32": 8}[request.param]
    s = make_system(request.param, nstate=nst, seed=11)
    ctx = CPContext(s, "mixed")
    psi = torch.from_numpy(s.psi).cuda()
    return s, ctx, psi


def test_density_mixed(case):
    import torch
    s, ctx, psi = case
    nx, ny, nz = s.nfft
    rho = torch.zeros(nz, ny, nx, dtype=torch.float64, device="cuda")
    ctx.state_fft_fwd(psi, rho)
    torch.cuda.synchronize()
    ref = O.density(O.state_g_to_r(s.psi, s), s)
    assert rel(rho.cpu().numpy(), ref) < 2e-6


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
