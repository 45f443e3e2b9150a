"""Stage sequence of one CP step for profilers (ncu): builds a seeded system
and runs the state FFTs, V_KS, the force pass, the PairCalculator
products and the Newton-Schulz orthonormalisation a few times, each call
through the C ABI.

    python -m openatom_b200.profile_stages [--preset w32] [--precision mixed] [--reps 3]

It holds only one context's device memory (about 1.5 GB at w32), so that
full-metric captures of single launches stay small.
"""
import argparse
import sys


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--preset", default="w32")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--seed", type=int, default=3)
    a = ap.parse_args(argv)
    import numpy as np
    import torch
    from openatom_b200.gpu import CPContext
    from openatom_b200.system import make_system
    s = make_system(a.preset, seed=a.seed)
    ctx = CPContext(s, a.precision)
    psi = torch.from_numpy(s.psi).cuda()
    nx, ny, nz = s.nfft
    f = torch.zeros_like(psi)
    f2 = torch.zeros_like(psi)
    S = torch.zeros(s.nstate, s.nstate, dtype=torch.float64, device="cuda")
    T = torch.eye(s.nstate, dtype=torch.float64, device="cuda")
    v = torch.from_numpy(np.random.default_rng(1).standard_normal((nz, ny, nx)) * 0.1).cuda()
    # an overlap 2 I + a symmetric perturbation of size 1e-2, as after a
    # dynamics step (four Newton-Schulz iterations to 1e-15)
    E = np.random.default_rng(2).standard_normal((s.nstate, s.nstate)) * 1e-2
    S_ns = torch.from_numpy(2.0 * np.eye(s.nstate) + 0.5 * (E + E.T)).cuda()
    T_ns = torch.zeros_like(S_ns)
    ctx.set_vks(v)
    mixed = a.precision == "mixed"
    for _ in range(a.reps):
        ctx.state_fft_fwd(psi)
        ctx.vks_build()
        ctx.vks_apply_fft_bwd(psi, f)
        ctx.pc_forward(psi, psi, 2.0, 0.5, S)
        ctx.pc_backward(S, psi, 1.0, 1.0, f)
        if mixed:
            ctx.pc_forward_mixed(psi, f, 1.0, 1.0, S)
            ctx.pc_backward_mixed(S, psi, -0.5, -1.0, f2, M2=T, X2=f, a2=1.0)
        ctx.ortho_invsqrt(S_ns, T_ns)
    torch.cuda.synchronize()
    print("ok")
    return 0


if __name__ == "__main__":
    sys.exit(main())
