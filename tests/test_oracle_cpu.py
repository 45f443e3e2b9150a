"""CPU checks of the oracle itself (no GPU): transforms, physics identities and
energy conservation of the CP dynamics it restates."""
import math

import numpy as np
import pytest

from openatom_b200.system import gamma_overlap, make_system
from oracle import cp_oracle as O


@pytest.fixture(scope="module")
def w2():
    return make_system("w2", seed=3, dt=0.25)


def test_layout(w2):
    s = w2
    assert np.all(s.kx[:s.nkx0] == 0)
    assert s.nkx0 == s.nkx0_red + s.nkx0_uni and s.nkx0_zero == 1
    assert int(np.sum(s.line_nneg + s.line_npos)) == s.ng
    assert np.all(np.diff(s.line_off) == (s.line_nneg + s.line_npos)[:-1])


def test_orthonormal_start(w2):
    S = gamma_overlap(w2.psi, w2.kx)
    assert np.max(np.abs(S - 2 * np.eye(w2.nstate))) < 1e-12


def test_expand_pack_roundtrip(w2):
    z = O.expand_gspace(w2.psi, w2)
    assert np.array_equal(O.pack_gspace(z, w2), w2.psi)


def test_psi_r_real_and_parseval(w2):
    s = w2
    full = O._full_grid(s.psi, s.kx, s.ky, s.kz, s.nfft)
    pr = np.fft.fftn(full, axes=(-3, -2, -1))
    assert np.max(np.abs(pr.imag)) < 1e-12 * np.max(np.abs(pr.real))
    psir = O.state_g_to_r(s.psi, s)
    # sum_r psi^2 = N * sum_full |c|^2 = 2 N
    assert np.allclose((psir ** 2).sum(axis=(1, 2, 3)), 2.0 * s.npts, rtol=1e-12)


def test_round_trip_r_to_g(w2):
    s = w2
    psir = O.state_g_to_r(s.psi, s)
    back = O.state_r_to_g(psir, s) / s.npts
    assert np.max(np.abs(back - s.psi)) < 1e-13


def test_hartree_real_space(w2):
    s = w2
    rho = O.density(O.state_g_to_r(s.psi, s), s)
    vr, eh, ee, ew = O.hart_eext(rho, s)
    assert eh > 0 and ew > 0
    # E_H + E_ext = integral of rho * (V_H + V_loc) minus E_H (V_H counted twice)
    tot = float(np.sum(rho * vr)) * s.vol / s.npts
    assert abs(tot - (2 * eh + ee)) < 1e-9 * max(1.0, abs(tot))


def test_eke_direct(w2):
    s = w2
    f, e = O.eke(s.psi, np.zeros_like(s.psi), s)
    g2 = s.g2()
    w = np.where(s.kx == 0, 1.0, 2.0)
    assert np.allclose(e, 0.5 * (w * g2 * np.abs(s.psi) ** 2).sum(1), rtol=1e-13)


def test_newton_schulz_vs_eigen():
    rng = np.random.default_rng(1)
    n = 24
    a = rng.standard_normal((n, n)) * 0.05
    S = 2 * np.eye(n) + a + a.T
    T, it, err = O.newton_schulz(S, tol=1e-15, max_iter=100)
    w, v = np.linalg.eigh(S / 2)
    Tex = (v / np.sqrt(w)) @ v.T
    assert np.max(np.abs(T - Tex)) < 1e-13 and err <= 1e-15


def test_newton_schulz_reports_non_convergence():
    S = 2 * np.diag([3.5, 0.5, 1.0, 1.2])  # an eigenvalue of S/2 above 3: no convergence
    T, it, err = O.newton_schulz(S, tol=1e-15, max_iter=7)
    assert it == 7 and not (err <= 1e-15)


def test_energy_conservation(w2):
    """E_KS + fictitious KE is conserved to O(dt^2) by the restated dynamics."""
    drifts = []
    for dt in (0.25, 0.125):
        s = make_system("w2", seed=3, dt=dt)
        st = O.CPState(s)
        tot = []
        for _ in range(int(round(1.0 / dt))):
            en = O.cp_step(st, s)
            tot.append(en["EKE"] + en["EHART"] + en["EEXC"] + en["EEXT"] + en["ENL"] + en["FICT_KE"])
        drifts.append(abs(tot[-1] - tot[0]))
    assert drifts[0] < 1e-3
    assert drifts[1] < drifts[0] / 2.5  # second order in dt


def test_psiv_reset_restores_orthonormal_frame(w2):
    """finiteDifferencePsiV: psi_t = psi (orthonormal), T = I, v = (psi(t) -
    psi(t - dt)) / dt, and the next step completes no half kick."""
    s = make_system("w2", seed=3, dt=0.5)
    st = O.CPState(s)
    for _ in range(3):
        O.cp_step(st, s)
    prev = st.psi.copy()
    O.cp_step(st, s)
    O.psiv_reset(st, s, prev, s.dt)
    S = gamma_overlap(st.psi_t, s.kx)
    assert np.max(np.abs(S - 2 * np.eye(s.nstate))) < 1e-12
    assert np.array_equal(st.T, np.eye(s.nstate))
    assert np.allclose(st.v, (st.psi - prev) / s.dt, rtol=0, atol=1e-15)
    # the next step's fictitious KE is that of v itself (no completing half kick)
    v0 = st.v.copy()
    en = O.cp_step(st, s)
    assert abs(en["FICT_KE"] - float(O.fict_ke(v0, s.cmass, s).sum())) <= 1e-12 * en["FICT_KE"]


def test_nonlocal_force_is_energy_gradient(w2):
    """F_nl = -dE_nl/d(Re c, Im c) (kx > 0) checked by finite differences."""
    s = w2
    f, enl, _ = O.nl_energy_forces(s.psi, s)
    rng = np.random.default_rng(4)
    d = (rng.standard_normal(s.psi.shape) + 1j * rng.standard_normal(s.psi.shape)) * 1e-6
    d[:, :s.nkx0] = 0.0
    e1 = O.nl_energy_forces(s.psi + d, s)[1].sum()
    e0 = O.nl_energy_forces(s.psi - d, s)[1].sum()
    pred = -2.0 * np.sum(f.real * d.real + f.imag * d.imag)
    assert abs((e1 - e0) - pred) < 1e-6 * abs(pred)


def test_ees_nonlocal_matches_structure_factor():
    """The EES interpolation (cp_ees_nonlocal.C) converges to the
    structure-factor result (cp_struct_fact.C / cp_nlmat.C) as the spline
    order and grid grow: an independent check of the EES conventions."""
    s = make_system("w4", seed=3)
    f1, e1, z1 = O.nl_energy_forces(s.psi, s)
    errs = []
    for order, scale in ((4, 1.2), (6, 1.2), (8, 2.0)):
        ees = O.ees_setup(s, scale, order)
        f2, e2, z2 = O.nl_ees_energy_forces(s.psi, s, ees)
        errs.append(abs(e2.sum() - e1.sum()) / abs(e1.sum()))
    assert errs[0] > errs[1] > errs[2]
    assert errs[2] < 1e-5


def test_ees_atom_forces_are_energy_gradient():
    """EES nonlocal atom forces (eesEnergyAtmForcRchare, the B-spline
    derivative weights of eesAtmBsplineRgrp) against a central finite
    difference of the EES nonlocal energy in each atom coordinate."""
    s = make_system("w4", seed=21)
    ees = O.ees_setup(s, scale=1.2, order=4)
    fa = O.nl_ees_energy_forces(s.psi, s, ees, atom_forces=True)[3]
    a = int(s.nl_atoms()[0])
    h = 1e-5
    for ax in range(3):
        es = []
        for sg in (1.0, -1.0):
            s.pos[a, ax] += sg * h
            es.append(O.nl_ees_energy_forces(s.psi, s, O.ees_setup(s, scale=1.2, order=4))[1].sum())
            s.pos[a, ax] -= sg * h
        assert abs(-(es[0] - es[1]) / (2 * h) - fa[a, ax]) < 1e-7 * np.max(np.abs(fa[a]))


def test_gga_potential_is_energy_derivative():
    """The BLYP gradient-correction potential (df/drho minus the white-byrd
    divergence term) is the functional derivative of EGGA: a central
    finite difference of EGGA along a density perturbation equals
    sum_r V_gga(r) drho(r) V/N."""
    s = make_system("w2", seed=3, xc="blyp")
    rho = O.density(O.state_g_to_r(s.psi, s), s)
    v, egga = O.gga_blyp(rho, s)
    assert egga < 0.0
    d = np.random.default_rng(7).standard_normal(rho.shape) * 1e-3 * rho
    e = 1e-3
    fd = (O.gga_blyp(rho + e * d, s)[1] - O.gga_blyp(rho - e * d, s)[1]) / (2 * e)
    pred = float(np.sum(v * d)) * s.vol / s.npts
    assert abs(fd - pred) < 1e-6 * abs(pred)


def test_ion_forces_are_energy_gradient():
    """The forces on the ions (local pseudopotential and reciprocal Ewald of
    CP_hart_eext_calc, the structure-factor nonlocal part, the real-space
    Ewald sum) are minus the gradient of EEXT + ENL + the Ewald energy at
    fixed coefficients, by central finite differences."""
    s = make_system("w2", seed=3)
    psi = s.psi

    def e_ion():
        rho = O.density(O.state_g_to_r(psi, s), s)
        _, _, ee, ew = O.hart_eext(rho, s)
        er, es, eb, _ = O.ewald_rspace(s)
        return ee + ew + float(O.nl_energy_forces(psi, s)[1].sum()) + er + es + eb

    F, _ = O.ion_forces(psi, s, O.density(O.state_g_to_r(psi, s), s))
    h = 1e-5
    for a in (0, 1, 4):
        for ax in range(3):
            s.pos[a, ax] += h
            ep = e_ion()
            s.pos[a, ax] -= 2 * h
            em = e_ion()
            s.pos[a, ax] += h
            assert abs(-(ep - em) / (2 * h) - F[a, ax]) < 1e-7 * np.max(np.abs(F))


def test_cg_minimisation_beats_steepest_descent():
    """The oracle's minimisation loop (computeMinimization): both methods
    lower the energy; conjugate gradients lower it further and reduce the
    constraint-projected force more in the same number of iterations."""
    s = make_system("w2", seed=5, ecut_mass=2.0, dt=5.0)
    out = {}
    for method in ("sd", "cg"):
        st = O.CPState(s)
        recs = O.minimize(st, s, 25, method=method, dt=10.0)
        e = [sum(r[k] for k in ("EKE", "EHART", "EEXT", "EEXC", "ENL")) for r in recs]
        assert e[-1] < e[0]
        out[method] = (e[-1], recs[-1]["FMAG"], recs[0]["FMAG"])
        # the result stays orthonormal
        S = O.pc_forward(O.kx0_scale(st.psi, s, 2 ** -0.5), O.kx0_scale(st.psi, s, 2 ** -0.5), s, 2.0)
        assert np.max(np.abs(S / 2.0 - np.eye(s.nstate))) < 1e-12
    assert out["cg"][0] < out["sd"][0] and out["cg"][1] < out["sd"][1] < out["sd"][2]


def test_ees_local_converges_to_structure_factor():
    """The EES local pseudopotential / reciprocal Ewald path approaches the
    structure-factor path as the B-spline order grows, and its atom forces
    are the negative gradient of E_ext + E_ewald(recip) at fixed density."""
    import copy
    s = make_system("w4", seed=21)
    rho = O.density(O.state_g_to_r(s.psi, s), s)
    ref = O.hart_eext(rho, s, want_forces=True)
    errs = []
    for order in (4, 8):
        s2 = copy.copy(s)
        s2.eext_ees = O.eesl_grid(s, 1.2, order) + (order,)
        out = O.hart_eext(rho, s2, want_forces=True)
        assert out[1] == ref[1]                                   # Hartree does not change
        errs.append((abs(out[2] - ref[2]) / abs(ref[2]), abs(out[3] - ref[3]) / abs(ref[3]),
                     np.max(np.abs(out[4] - ref[4])) / np.max(np.abs(ref[4]))))
    assert errs[1][0] < 1e-5 and errs[1][1] < 1e-7 and errs[1][2] < 1e-5
    assert all(b < a for a, b in zip(errs[0], errs[1]))
    s2 = copy.copy(s)
    s2.pos = s.pos.copy()
    s2.eext_ees = O.eesl_grid(s, 1.2, 6) + (6,)
    F = O.hart_eext(rho, s2, want_forces=True)[4]
    h = 1e-4
    for a, c in ((0, 0), (1, 2), (s.natm - 1, 1)):
        e = []
        for sgn in (1, -1):
            s3 = copy.copy(s2)
            s3.pos = s2.pos.copy()
            s3.pos[a, c] += sgn * h
            o = O.hart_eext(rho, s3)
            e.append(o[2] + o[3])
        assert abs(-(e[0] - e[1]) / (2 * h) - F[a, c]) <= 1e-6 * max(1.0, abs(F[a, c]))
