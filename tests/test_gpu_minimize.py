"""Electronic minimisation on the GPU (cp_min_opt: computeMinimization,
gspace.ci:85-196; CP_integrate_min_STD / CP_integrate_min_CG,
cp_min_std.C / cp_min_CG.C) against the oracle's loop, FP64 form: every
energy term and the force magnitude to 1e-10 relative over the iterations,
for steepest descent and conjugate gradients; conjugate gradients converge."""
import numpy as np
import pytest

from openatom_b200.system import make_system
from oracle import cp_oracle as O

pytestmark = pytest.mark.gpu

KEYS = ("EKE", "EHART", "EEXT", "EEXC", "ENL", "FMAG")


@pytest.mark.parametrize("method", ["sd", "cg"])
def test_minimizer_matches_oracle(method):
    from openatom_b200.gpu import CPDriver, CPMinimizer
    s = make_system("w8", nstate=16, seed=71, ecut_mass=2.0, dt=5.0)
    st = O.CPState(s)
    ref = O.minimize(st, s, 6, method=method, dt=10.0)
    d = CPDriver(s, "fp64")
    got = CPMinimizer(d, method, dt=10.0).run(6)
    for i, (g, r) in enumerate(zip(got, ref)):
        for k in KEYS:
            assert abs(g[k] - r[k]) <= 1e-10 * max(1.0, abs(r[k])), (i, k, g[k], r[k])
    psi = d.psi.cpu().numpy()
    assert np.max(np.abs(psi - st.psi)) / np.max(np.abs(st.psi)) < 1e-9
    d.ctx.close()


def test_cg_minimization_converges_mixed():
    """The mixed form minimises too: conjugate gradients on 8 waters / 32
    states cut the force magnitude tenfold and lower the energy."""
    from openatom_b200.gpu import CPDriver, CPMinimizer
    s = make_system("w8", seed=72, ecut_mass=2.0, dt=5.0)
    d = CPDriver(s, "mixed")
    recs = CPMinimizer(d, "cg", dt=10.0).run(40)
    e = [sum(r[k] for k in ("EKE", "EHART", "EEXT", "EEXC", "ENL")) for r in recs]
    assert e[-1] < e[0]
    assert recs[-1]["FMAG"] < 0.1 * recs[0]["FMAG"]
    d.ctx.close()
