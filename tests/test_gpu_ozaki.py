"""The int8 digit products of the mixed form (Ozaki splitting on
tcgen05.mma.kind::i8): the overlap S = alpha sum w psi_t psi_t^T
(PairCalculator::multiplyForward, ckPairCalculator.C:821-893) and the
rotation psi_t T (bwMultiplyHelper, :1710-1946) against the FP64 DMMA
products and the oracle, for state counts that fill one or two 64-column
halves and for odd counts; a non-finite input propagates to the output.
Tolerances: S to 5e-13 of its largest entry (its K sums average the digit
cut-offs out); the rotation to 1e-12 of the largest coefficient (each output
is about one input coefficient, cut at 2^-41 of its K range's largest value);
the rotated set orthonormal to 1e-12."""
import numpy as np
import pytest

from openatom_b200.system import make_system
from oracle import cp_oracle as O

pytestmark = pytest.mark.gpu

TOL = 5e-13
TOL_ROT = 1e-12


def _case(preset, nst, seed):
    s = make_system(preset, nstate=nst, seed=seed)
    rng = np.random.default_rng(seed)
    # a non-orthogonal set near the orthonormal one, as after an integration step
    pt = s.psi + 1e-2 * (rng.standard_normal(s.psi.shape) + 1j * rng.standard_normal(s.psi.shape)) * np.abs(s.psi)
    return s, np.ascontiguousarray(pt)


@pytest.mark.parametrize("preset,nst", [("w8", 16), ("w8", 32), ("w4", 7), ("w32", 100), ("w32", 128)])
def test_overlap_and_rotation_match_fp64(preset, nst):
    import torch
    from openatom_b200.gpu import CPContext
    s, pt = _case(preset, nst, 61 + nst)
    ctx = CPContext(s, "mixed")
    assert ctx.has_i8()
    P = torch.from_numpy(pt).cuda()
    S8 = torch.zeros(nst, nst, dtype=torch.float64, device="cuda")
    S64 = torch.zeros_like(S8)
    ctx.pc_overlap_i8(P, 2.0, 0.5, S8)
    ctx.pc_forward(P, P, 2.0, 0.5, S64)
    torch.cuda.synchronize()
    s8, s64 = S8.cpu().numpy(), S64.cpu().numpy()
    ref = O.pc_forward(O.kx0_scale(pt, s, 2 ** -0.5), O.kx0_scale(pt, s, 2 ** -0.5), s, 2.0)
    assert np.max(np.abs(s8 - ref)) <= TOL * np.max(np.abs(ref))
    assert np.max(np.abs(s8 - s64)) <= TOL * np.max(np.abs(s64))
    assert np.array_equal(s8, s8.T)
    # T = (S/2)^-1/2 and the rotation
    w, V = np.linalg.eigh(ref / 2.0)
    T = (V * w ** -0.5) @ V.T
    Tg = torch.from_numpy(np.ascontiguousarray(T)).cuda()
    R8 = torch.zeros_like(P)
    R64 = torch.zeros_like(P)
    ctx.pc_rotate_i8(Tg, P, R8)
    ctx.pc_backward(Tg, P, 1.0, 1.0, R64)
    torch.cuda.synchronize()
    r8, r64 = R8.cpu().numpy(), R64.cpu().numpy()
    rref = T.T @ pt
    assert np.max(np.abs(r8 - rref)) <= TOL_ROT * np.max(np.abs(rref))
    assert np.max(np.abs(r8 - r64)) <= TOL_ROT * np.max(np.abs(r64))
    # the rotated set is orthonormal in FP64: S/2 = I
    q = O.pc_forward(O.kx0_scale(r8, s, 2 ** -0.5), O.kx0_scale(r8, s, 2 ** -0.5), s, 2.0) / 2.0
    assert np.max(np.abs(q - np.eye(nst))) < 1e-12
    ctx.check()
    ctx.close()


def test_nonfinite_and_operand_checks():
    import torch
    from openatom_b200.gpu import CPContext, OaError, OA_ERR_BAD_ARG
    s, pt = _case("w8", 16, 77)
    pt[3, 40] = np.nan
    ctx = CPContext(s, "mixed")
    P = torch.from_numpy(pt).cuda()
    S = torch.zeros(16, 16, dtype=torch.float64, device="cuda")
    ctx.pc_overlap_i8(P, 2.0, 0.5, S)
    got = S.cpu().numpy()
    assert np.all(np.isnan(got[3])) and np.all(np.isnan(got[:, 3]))
    assert np.all(np.isfinite(np.delete(np.delete(got, 3, 0), 3, 1)))
    # the rotation needs the operand of the last overlap
    other = torch.zeros_like(P)
    out = torch.zeros_like(P)
    with pytest.raises(OaError) as ei:
        ctx.pc_rotate_i8(torch.eye(16, dtype=torch.float64, device="cuda"), other, out)
    assert ei.value.status == OA_ERR_BAD_ARG
    ctx.close()
