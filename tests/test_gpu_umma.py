"""Split-BF16 tcgen05 PairCalculator GEMMs against the FP64 form.

Tolerances (max |err| / max |ref|): 3-term split (6 products) 1e-5,
2-term split (3 products) 2e-4 -- the split depth sets the operand accuracy
(2^-24 / 2^-16); FP32 accumulation inside each K block adds up to a few
1e-6 when a CTA accumulates a long K range (few K blocks per output tile).
Above 160 states the output has 16 tiles or more sharing the SMs, so each
CTA sums a K range several times longer in FP32: twice the tolerance."""
import numpy as np
import pytest

from openatom_b200.system import make_system

pytestmark = pytest.mark.gpu

TOL = {3: 1e-5, 2: 2e-4}


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def tol(nterm, n):
    return TOL[nterm] * (2.0 if n > 160 else 1.0)


@pytest.fixture(scope="module", params=[("w4", None), ("w8", 32), ("w8", 48), ("w8", 100), ("w8", 128), ("w8", 160),
                                              ("w8", 512)])
def case(request):
    import torch
    from openatom_b200.gpu import CPContext
    preset, nst = request.param
    s = make_system(preset, nstate=nst, seed=17) if nst is None or nst <= 64 else None
    if s is None:
        # more states than the Loewdin start allows cheaply: random rows are fine here
        s = make_system(preset, nstate=32, seed=17)
        rng = np.random.default_rng(1)
        s.psi = (rng.standard_normal((nst, s.ng)) + 1j * rng.standard_normal((nst, s.ng))) / np.sqrt(s.ng)
        s.nstate = nst
        s.occ = np.ones(nst)
    ctx = CPContext(s, "mixed")
    return s, ctx


@pytest.mark.parametrize("nterm", [3, 2])
def test_forward_mixed(case, nterm):
    import torch
    s, ctx = case
    n = s.nstate
    rng = np.random.default_rng(2)
    F = (rng.standard_normal(s.psi.shape) + 1j * rng.standard_normal(s.psi.shape)) * 0.3
    P = torch.from_numpy(np.ascontiguousarray(s.psi)).cuda()
    Fg = torch.from_numpy(F).cuda()
    ref = torch.zeros(n, n, dtype=torch.float64, device="cuda")
    got = torch.zeros_like(ref)
    for (a, b, al, w) in ((P, P, 2.0, 0.5), (P, Fg, 1.0, 1.0)):
        ctx.pc_forward(a, b, al, w, ref)
        ctx.pc_forward_mixed(a, b, al, w, got, nterm=nterm)
        ctx.check()
        assert rel(got.cpu().numpy(), ref.cpu().numpy()) < tol(nterm, n)


@pytest.mark.parametrize("nterm", [3, 2])
def test_backward_mixed(case, nterm):
    import torch
    s, ctx = case
    n = s.nstate
    rng = np.random.default_rng(3)
    F = (rng.standard_normal(s.psi.shape) + 1j * rng.standard_normal(s.psi.shape)) * 0.3
    T = np.eye(n) + 0.01 * rng.standard_normal((n, n))
    G = 0.05 * rng.standard_normal((n, n))
    P = torch.from_numpy(np.ascontiguousarray(s.psi)).cuda()
    Fg = torch.from_numpy(F).cuda()
    Tg, Gg = torch.from_numpy(T).cuda(), torch.from_numpy(G).cuda()
    ref = torch.zeros_like(P)
    got = torch.zeros_like(P)
    ctx.pc_backward(Gg, P, -0.5, -1.0, ref, M2=Tg, X2=Fg, a2=1.0)
    ctx.pc_backward_mixed(Gg, P, -0.5, -1.0, got, M2=Tg, X2=Fg, a2=1.0, nterm=nterm)
    ctx.check()
    assert rel(got.cpu().numpy(), ref.cpu().numpy()) < tol(nterm, n)
    ctx.pc_backward(Tg, P, 1.0, 1.0, ref)
    ctx.pc_backward_mixed(Tg, P, 1.0, 1.0, got, nterm=nterm)
    ctx.check()
    assert rel(got.cpu().numpy(), ref.cpu().numpy()) < tol(nterm, n)


def test_nonlocal_mixed(case):
    import torch
    s, ctx = case
    P = torch.from_numpy(np.ascontiguousarray(s.psi)).cuda()
    ref = torch.zeros_like(P)
    got = torch.zeros_like(P)
    e_ref = torch.zeros(s.nstate, dtype=torch.float64, device="cuda")
    e_got = torch.zeros_like(e_ref)
    ctx.nl_sf(P, ref, nterm=0, enl_out=e_ref)
    ctx.nl_sf(P, got, nterm=3, enl_out=e_got)
    ctx.check()
    assert rel(got.cpu().numpy(), ref.cpu().numpy()) < TOL[3]
    assert rel(e_got.cpu().numpy(), e_ref.cpu().numpy()) < TOL[3]
