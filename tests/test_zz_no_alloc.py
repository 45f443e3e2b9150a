"""The allocation-free PairCalculator forward product (oa_gpu_pc_forward_noalloc).

Callers that cannot allocate device memory -- a framework whose memory pool
already holds the device, or a latency-critical path that cannot take
cudaMalloc's device synchronisation -- call this entry point with their own
inputs and output; it keeps its split-K scratch in a fixed device array.
This test calls it through the C ABI twice in a row with different inputs
and compares each result with the context-based oa_gpu_pc_forward.  Both use
the FP64 DMMA kernel, but with different split-K partitions of the g-vectors
(the context path splits over about one CTA per SM, this one over 32 fixed
partials), so the sums round differently: the tolerance is 1e-13 relative.
It lives in its own file, collected last."""
import ctypes as C

import numpy as np
import pytest

from openatom_b200.system import make_system

pytestmark = pytest.mark.gpu

TOL = 1e-13


def test_pc_forward_noalloc_matches_context_entry():
    import torch
    from openatom_b200.gpu import CPContext, OA_ERR_BAD_ARG, OA_OK, load_library
    lib = load_library()
    s = make_system("w4", seed=31)
    ctx = CPContext(s, "fp64")
    n = s.nstate
    rng = np.random.default_rng(9)
    F = (rng.standard_normal(s.psi.shape) + 1j * rng.standard_normal(s.psi.shape)) * 0.2
    P = torch.from_numpy(np.ascontiguousarray(s.psi)).cuda()
    Fg = torch.from_numpy(F).cuda()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    # two calls in a row: S = 2 sum w psi psi (kx=0 weight 1/2), then Lambda
    for left, right, alpha, w in ((P, P, 2.0, 0.5), (P, Fg, 1.0, 1.0)):
        ref = torch.zeros(n, n, dtype=torch.float64, device="cuda")
        got = torch.full((n, n), float("nan"), dtype=torch.float64, device="cuda")
        ctx.pc_forward(left, right, alpha, w, ref)
        st = lib.oa_gpu_pc_forward_noalloc(stream, C.c_void_p(left.data_ptr()), C.c_void_p(right.data_ptr()),
                                           n, s.ng, s.nkx0, alpha, w, C.c_void_p(got.data_ptr()))
        assert st == OA_OK, lib.oa_gpu_last_error().decode()
        torch.cuda.synchronize()
        r = ref.cpu().numpy()
        g = got.cpu().numpy()
        assert np.max(np.abs(g - r)) <= TOL * np.max(np.abs(r))
    # sizes beyond the fixed scratch are refused with an error, not run
    st = lib.oa_gpu_pc_forward_noalloc(stream, C.c_void_p(P.data_ptr()), C.c_void_p(P.data_ptr()), 129, s.ng,
                                       s.nkx0, 1.0, 1.0, C.c_void_p(ref.data_ptr()))
    assert st == OA_ERR_BAD_ARG
    assert b"128" in lib.oa_gpu_last_error()
