"""Ion dynamics in the native graphed step (oa_gpu_set_ions): the local
pseudopotential and reciprocal Ewald atom forces of the density z pass, the
nonlocal atom forces (structure-factor and EES methods), the real-space Ewald
sum and the NVE atom integration, against the oracle's CP step with an IonState (whose
forces are pinned to compiled cp_hart_ext.C, cp_nl_energy_forc.C and
cp_rspace_ion.C).

FP64 form: every energy term (the ionic kinetic energy and the real-space
Ewald energy included) to 1e-10 relative, positions and velocities to 1e-10
of their scale, coefficients to 1e-9."""
import copy

import numpy as np
import pytest

from openatom_b200.system import make_system
from oracle import cp_oracle as O

pytestmark = pytest.mark.gpu

TERMS = ("EKE", "EHART", "EEXT", "EEXC", "ENL", "FICT_KE", "ION_KE")


def _start(preset, nstate, seed):
    s = make_system(preset, seed=seed, nstate=nstate, ecut_mass=2.0, cmass0=400.0, dt=5.0)
    rng = np.random.default_rng(seed)
    m = O.atom_masses(s)
    kT = 300.0 * 3.1668115634556e-6   # 300 K in Hartree
    vel = rng.standard_normal(s.pos.shape) * np.sqrt(kT / m)[:, None]
    return s, m, vel


def _oracle(s, vel, nsteps):
    so = copy.deepcopy(s)
    st = O.CPState(so)
    ions = O.IonState(so, vel)
    recs = [O.cp_step(st, so, norb_tol=0.003, ions=ions) for _ in range(nsteps)]
    return so, st, ions, recs


@pytest.mark.parametrize("preset,nstate", [("w2", None), ("w8", 16)])
def test_ion_dynamics_fp64_matches_oracle(preset, nstate):
    from openatom_b200.gpu import CPDriver
    s, m, vel = _start(preset, nstate, 41)
    d = CPDriver(s, "fp64", norb_tol=0.003)
    d.ctx.set_ions(m, vel)
    got = d.run_native(d.native_state(use_graph=True), 6)
    so, st, ions, ref = _oracle(s, vel, 6)
    for i, (g, r) in enumerate(zip(got, ref)):
        for k in TERMS:
            assert abs(g[k] - r[k]) <= 1e-10 * max(1.0, abs(r[k])), (i, k, g[k], r[k])
        ew = r["EWALD_REAL"] + r["EWALD_SELF"] + r["EWALD_BGR"]
        assert abs(g["EWALD_REAL"] - ew) <= 1e-10 * max(1.0, abs(ew)), (i, g["EWALD_REAL"], ew)
    pos, v = d.ctx.get_ions()
    assert np.max(np.abs(pos - so.pos)) <= 1e-10 * np.max(np.abs(so.pos))
    assert np.max(np.abs(v - ions.v)) <= 1e-10 * np.max(np.abs(ions.v))
    assert np.max(np.abs(d.psi.cpu().numpy() - st.psi)) <= 1e-9 * np.max(np.abs(st.psi))
    # the atoms moved
    assert np.max(np.abs(pos - s.pos)) > 1e-4
    d.ctx.close()


def test_ion_dynamics_mixed_total_energy():
    """Mixed form from a quenched start (30 damped FP64 steps on the GPU), as
    in the mixed-form benchmark: the total energy within 1e-6 Ha/atom."""
    from openatom_b200.gpu import CPDriver
    s, m, vel = _start("w8", 16, 43)
    q = CPDriver(s, "fp64")
    q.quench(3)
    q.quench(27, dt=10.0)
    psi0 = q.psi.cpu().numpy()
    q.ctx.close()
    d = CPDriver(s, "mixed", psi0=psi0, norb_tol=0.003)
    d.ctx.set_ions(m, vel)
    got = d.run_native(d.native_state(use_graph=True), 5)
    so = copy.deepcopy(s)
    st = O.CPState(so)
    st.psi_t = psi0.copy()
    st.psi = psi0.copy()
    ions = O.IonState(so, vel)
    ref = [O.cp_step(st, so, norb_tol=0.003, ions=ions) for _ in range(5)]
    keys = ("EKE", "EHART", "EEXT", "EEXC", "ENL")
    for g, r in zip(got, ref):
        assert abs(sum(g[k] for k in keys) - sum(r[k] for k in keys)) / s.natm <= 1e-6
        assert abs(g["ION_KE"] - r["ION_KE"]) <= 1e-6 * max(1e-3, abs(r["ION_KE"]))
    pos, _ = d.ctx.get_ions()
    assert np.max(np.abs(pos - so.pos)) <= 1e-7
    d.ctx.close()


@pytest.mark.parametrize("preset,nstate,order", [("w2", None, 4), ("w8", 16, 6)])
def test_ion_dynamics_ees_nonlocal_fp64(preset, nstate, order):
    """EES nonlocal method with moving atoms: the B-splines follow the atoms
    every step and the nonlocal atom forces come from the gathered stencil
    sums (eesEnergyAtmForcRchare's force loop)."""
    from openatom_b200.gpu import CPDriver
    s, m, vel = _start(preset, nstate, 45)
    d = CPDriver(s, "fp64", norb_tol=0.003, nl_method="ees", ees_order=order)
    d.ctx.set_ions(m, vel)
    got = d.run_native(d.native_state(use_graph=True), 6)
    so = copy.deepcopy(s)
    st = O.CPState(so)
    ions = O.IonState(so, vel)
    ees = O.ees_setup(so, 1.2, order)

    def nl(psi, sysm):
        f, enl, _ = O.nl_ees_energy_forces(psi, sysm, ees)
        return f, float(enl.sum())

    ref = [O.cp_step(st, so, nl=nl, norb_tol=0.003, ions=ions, ees=ees) for _ in range(6)]
    for i, (g, r) in enumerate(zip(got, ref)):
        for k in TERMS:
            assert abs(g[k] - r[k]) <= 1e-10 * max(1.0, abs(r[k])), (i, k, g[k], r[k])
    pos, v = d.ctx.get_ions()
    assert np.max(np.abs(pos - so.pos)) <= 1e-10 * np.max(np.abs(so.pos))
    assert np.max(np.abs(v - ions.v)) <= 1e-10 * np.max(np.abs(ions.v))
    assert np.max(np.abs(d.psi.cpu().numpy() - st.psi)) <= 1e-9 * np.max(np.abs(st.psi))
    d.ctx.close()


def test_ion_dynamics_refuses_host_positions():
    from openatom_b200.gpu import CPDriver, OaError
    s, m, vel = _start("w2", None, 44)
    d = CPDriver(s, "fp64")
    d.ctx.set_ions(m, vel)
    with pytest.raises(OaError):
        d.run_native(d.native_state(use_graph=True), 2, pos_host=np.repeat(s.pos[None], 2, axis=0))
    d.ctx.close()
