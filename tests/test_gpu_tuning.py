"""Runtime tile and schedule choices (oa_gpu_set_tuning): every choice
changes only the order of partial sums, so native CP steps agree with the
built-in choice to rounding -- FP64 each term to 1e-12 relative; mixed (FP32
density sums regrouped) each term to 1e-6 relative and the total to 1e-7
Ha/atom -- and the FP64 form with the runtime-plan transforms still matches
the oracle."""
import copy

import numpy as np
import pytest

from openatom_b200.system import make_system
from oracle import cp_oracle as O

pytestmark = pytest.mark.gpu

KEYS = ("EKE", "EHART", "EEXT", "EEXC", "ENL", "FICT_KE")


def _run(s, prec, steps, **choice):
    from openatom_b200.gpu import CPDriver
    d = CPDriver(s, prec, norb_tol=0.003, tuning="default")
    if choice:
        d.ctx.set_tuning(**choice)
    got = d.run_native(d.native_state(use_graph=True), steps)
    t = d.ctx.get_tuning()
    d.ctx.close()
    return got, t


@pytest.mark.parametrize("prec,choice,tol", [
    ("fp64", {"group_state": 3, "dgemm_kblocks": 48}, 1e-12),
    ("fp64", {"fft_path": 2}, 1e-12),
    ("mixed", {"group_pair": 7, "dgemm_kblocks": 96}, 1e-6),
])
def test_tuning_changes_rounding_only(prec, choice, tol):
    s = make_system("w8", nstate=32, seed=11)
    ref, t0 = _run(s, prec, 4)
    got, t1 = _run(s, prec, 4, **choice)
    for k, v in choice.items():
        assert t1[k] == v
    for g, r in zip(got, ref):
        for k in KEYS:
            assert abs(g[k] - r[k]) <= tol * max(1.0, abs(r[k])), (k, g[k], r[k])
        tot = sum(g[k] - r[k] for k in KEYS[:5])
        assert abs(tot) / s.natm <= (1e-12 if prec == "fp64" else 1e-7)


def test_runtime_fft_path_matches_oracle():
    s = make_system("w4", seed=12)
    got, _ = _run(s, "fp64", 3, fft_path=2)
    st = O.CPState(copy.deepcopy(s))
    so = copy.deepcopy(s)
    ref = [O.cp_step(st, so, norb_tol=0.003) for _ in range(3)]
    for g, r in zip(got, ref):
        for k in ("EKE", "EHART", "EEXT", "EEXC", "ENL"):
            assert abs(g[k] - r[k]) <= 1e-10 * max(1.0, abs(r[k])), (k, g[k], r[k])


def test_tuning_refusals():
    from openatom_b200.gpu import CPContext, OaError
    s = make_system("w2", seed=3)
    ctx = CPContext(s, "mixed", tuning="default")
    for bad in ({"group_state": 33}, {"group_pair": 99}, {"dgemm_kblocks": 1}, {"dgemm_kblocks": 161},
                {"tgemm_kblocks": 10 ** 6}, {"fft_path": 3}, {"fft_path": 2}):
        with pytest.raises(OaError):
            ctx.set_tuning(**bad)
    before = ctx.get_tuning()
    ctx.set_tuning()                     # all zero: nothing changes
    assert ctx.get_tuning() == before
    ctx.close()
