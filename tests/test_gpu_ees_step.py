"""The EES nonlocal method inside the CP step (cp_nonloc_ees_opt on:
CP_State_ParticlePlane.C:867-1136, cp_ees_nonlocal.C:256-2079), B-spline
order 4 as in the 128-water configuration:

* the native graphed step in the FP64 form against the oracle's cp_step with
  its EES restatement (energies 1e-10 relative, coefficients 1e-9);
* the native step in the mixed form against the host-sequenced step, bit
  for bit (same kernels, captured into one graph)."""
import numpy as np
import pytest

from openatom_b200.system import make_system
from oracle import cp_oracle as O

pytestmark = pytest.mark.gpu

ORDER, SCALE = 4, 1.2


def test_native_step_ees_matches_oracle():
    from openatom_b200.gpu import CPDriver
    s = make_system("w8", nstate=16, seed=41, ecut_mass=2.0, cmass0=400.0, dt=5.0)
    ees = O.ees_setup(s, SCALE, ORDER)

    def nl(psi, sysm):
        f, enl, _ = O.nl_ees_energy_forces(psi, sysm, ees)
        return f, float(enl.sum())

    st = O.CPState(s)
    ref = [O.cp_step(st, s, nl=nl, norb_tol=0.003) for _ in range(4)]
    d = CPDriver(s, "fp64", norb_tol=0.003, nl_method="ees", ees_order=ORDER, ees_scale=SCALE)
    assert tuple(d.ctx.ees_grid) == tuple(ees["grid"])
    got = d.run_native(d.native_state(use_graph=True), 4)
    for i, (g, r) in enumerate(zip(got, ref)):
        for k in ("EKE", "EHART", "EEXT", "EEXC", "ENL", "FICT_KE"):
            assert abs(g[k] - r[k]) <= 1e-10 * max(1.0, abs(r[k])), (i, k, g[k], r[k])
    psi = d.psi.cpu().numpy()
    assert np.max(np.abs(psi - st.psi)) / np.max(np.abs(st.psi)) < 1e-9
    d.ctx.close()


def test_native_step_ees_mixed_matches_host_runner():
    from openatom_b200.gpu import CPDriver
    s = make_system("w8", nstate=16, seed=42, ecut_mass=2.0, cmass0=400.0, dt=5.0)
    a = CPDriver(s, "mixed", norb_tol=0.003, nl_method="ees", ees_order=ORDER, ees_scale=SCALE)
    c = CPDriver(s, "mixed", norb_tol=0.003, nl_method="ees", ees_order=ORDER, ees_scale=SCALE)
    ea = [a.step() for _ in range(3)]
    ec = c.run_native(c.native_state(use_graph=True), 3)
    for i in range(3):
        for k in ("EKE", "EHART", "EEXT", "EEXC", "ENL", "FICT_KE", "SMAX"):
            assert ec[i][k] == ea[i][k], (i, k, ea[i][k], ec[i][k])
    assert np.array_equal(a.psi.cpu().numpy(), c.psi.cpu().numpy())
    assert ec[0]["ENL"] != 0.0
