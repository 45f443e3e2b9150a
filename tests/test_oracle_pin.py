"""Pin the numpy oracle against the reference's own PINY physics routines,
compiled from the reference sources into oracle/_ref/libpiny_ref.so by
oracle/build_ref.sh (CPU only).

Pinned: CPNONLOCAL::CP_eke_calc (cp_eke.C), CPXCFNCTS::CP_exc_calc
(cp_pz_lda.C), CPLOCAL::CP_hart_eext_calc (cp_hart_ext.C),
CPORTHOG::get_iter_Tmat (cp_lowdin.C), the structure-factor nonlocal path
(cp_struct_fact.C, cp_nlmat.C, cp_nl_energy_forc.C), the EES nonlocal path
(cp_ees_nonlocal.C with get_bspline_wght1d of set_cp_ewald.C), the CP
integrator (cp_dynamics.C), the minimisers (cp_min_std.C, cp_min_CG.C), the
BLYP functional (cp_becke.C, cp_grad_rho_ctrl.C), the real-space Ewald
sum (cp_rspace_ion.C), the EES local pseudopotential and reciprocal Ewald
path (cp_hart_ext.C) and the pseudopotential splines (control_vps_params.C,
friend_lib.C).
The FFT and GEMM boundaries have no reference implementation here (FFTW2 /
Fortran BLAS are absent) and are pinned by mathematics in test_oracle_cpu.py.
"""
import copy
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from openatom_b200.system import make_system
from oracle import cp_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "libpiny_ref.so")

dp = C.POINTER(C.c_double)
ip = C.POINTER(C.c_int)


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(LIB) and os.path.isdir("/root/reference"):
        subprocess.run(["bash", os.path.join(ROOT, "oracle", "build_ref.sh")], check=True,
                       capture_output=True)
    if not os.path.exists(LIB):
        pytest.skip("oracle/_ref not built (reference sources absent)")
    lib = C.CDLL(LIB)
    lib.ref_eke.argtypes = [C.c_int, dp, dp, ip, ip, ip, dp, C.c_double, C.c_double, C.c_int, C.c_double, dp]
    lib.ref_pz_lda.argtypes = [C.c_int, C.c_int, C.c_int, dp, dp, C.c_double, dp, dp, C.c_int]
    lib.ref_gga.argtypes = [C.c_int, C.c_int, C.c_int, dp, dp, dp, dp, dp, C.c_double, C.c_double, C.c_int, C.c_int]
    lib.ref_gga.restype = C.c_double
    lib.ref_hart_eext.argtypes = [C.c_int, ip, ip, ip, dp, dp, C.c_int, dp, ip, dp, C.c_int, C.c_int, C.c_double,
                                  C.c_double, dp, dp, C.c_double, C.c_double, C.c_double, dp, dp, dp, dp]
    lib.ref_iter_tmat.argtypes = [dp, dp, C.c_int]
    return lib


def _d(a):
    return a.ctypes.data_as(dp)


def _i(a):
    return a.ctypes.data_as(ip)


@pytest.fixture(scope="module")
def sysm():
    return make_system("w4", seed=21)


def test_eke_pinned(ref, sysm):
    s = sysm
    rng = np.random.default_rng(0)
    f0 = (rng.standard_normal(s.psi.shape) + 1j * rng.standard_normal(s.psi.shape)) * 0.1
    f_or, e_or = O.eke(s.psi, f0, s)
    kx, ky, kz = (np.ascontiguousarray(a, dtype=np.int32) for a in (s.kx, s.ky, s.kz))
    f = 2.0 * np.pi / s.box
    g2 = np.ascontiguousarray((f * kx) ** 2 + (f * ky) ** 2 + (f * kz) ** 2, dtype=np.float64)
    for st in range(s.nstate):
        psi = np.ascontiguousarray(s.psi[st])
        fr = np.ascontiguousarray(f0[st].copy())
        e = C.c_double(0.0)
        ref.ref_eke(s.ng, _d(psi.view(np.float64)), _d(fr.view(np.float64)), _i(kx), _i(ky), _i(kz), _d(g2),
                    s.ecut_ry, float(s.occ[st]), s.nkx0, s.box, C.byref(e))
        assert abs(e.value - e_or[st]) <= 1e-12 * abs(e_or[st])
        assert np.max(np.abs(fr - f_or[st])) <= 1e-12 * np.max(np.abs(f_or[st]))


@pytest.mark.parametrize("lyp", [0, 1])
def test_pz_lda_pinned(ref, sysm, lyp):
    s = sysm
    nx, ny, nz = s.nfft
    rho = O.density(O.state_g_to_r(s.psi, s), s)
    v_or, exc_or, muxc_or = O.pz_lda(rho, s.vol, s.npts, lyp=bool(lyp))
    xl = 2 * (nx // 2 + 1)
    pad = np.zeros((nz, ny, xl))
    pad[:, :, :nx] = rho
    res = np.zeros_like(pad)
    exc, muxc = C.c_double(), C.c_double()
    ref.ref_pz_lda(nx, ny, nz, _d(pad), _d(res), s.box, C.byref(exc), C.byref(muxc), lyp)
    assert abs(exc.value - exc_or) <= 1e-12 * abs(exc_or)
    assert abs(muxc.value - muxc_or) <= 1e-12 * abs(muxc_or)
    assert np.max(np.abs(res[:, :, :nx] - v_or)) <= 1e-13 * np.max(np.abs(v_or))


def test_hart_eext_pinned(ref, sysm):
    s = sysm
    nx, ny, nz = s.nfft
    rho_r = O.density(O.state_g_to_r(s.psi, s), s)
    _, eh_or, ee_or, ew_or, f_or = O.hart_eext(rho_r, s, want_forces=True)
    kx, ky, kz, g2 = O.rho_sphere(s)
    # order points as z-lines (kz fastest) so the reference's incremental phases apply
    order = np.lexsort((kz, ky, kx))
    kx, ky, kz = kx[order], ky[order], kz[order]
    rhog = np.fft.fftn(rho_r * (s.vol / s.npts))[kz % nz, ky % ny, kx % nx]
    rhog = np.ascontiguousarray(rhog)
    vks = np.zeros_like(rhog)
    kx_, ky_, kz_ = (np.ascontiguousarray(a, dtype=np.int32) for a in (kx, ky, kz))
    typ = np.ascontiguousarray(s.atm_type, dtype=np.int32)
    pos = np.ascontiguousarray(s.pos)
    q = np.ascontiguousarray(s.q)
    spl = np.ascontiguousarray(s.vloc.coef)
    gz = np.ascontiguousarray(s.gzvps)
    fatm = np.zeros((s.natm, 3))
    eh, ee, ew = C.c_double(), C.c_double(), C.c_double()
    ref.ref_hart_eext(len(kx), _i(kx_), _i(ky_), _i(kz_), _d(rhog.view(np.float64)), _d(vks.view(np.float64)),
                      s.natm, _d(pos), _i(typ), _d(q), len(s.type_names), s.vloc.n, s.vloc.gmin, s.vloc.dg,
                      _d(spl), _d(gz), s.alp_ewd, s.ecut_ry, s.box, C.byref(eh), C.byref(ee), C.byref(ew),
                      _d(fatm))
    assert abs(eh.value - eh_or) <= 1e-11 * abs(eh_or)
    assert abs(ee.value - ee_or) <= 1e-11 * abs(ee_or)
    assert abs(ew.value - ew_or) <= 1e-11 * abs(ew_or)
    assert np.max(np.abs(fatm - f_or)) <= 1e-10 * np.max(np.abs(f_or))


def test_iter_tmat_pinned(ref):
    rng = np.random.default_rng(2)
    n = 16
    a = rng.standard_normal((n, n)) * 0.02
    S = np.ascontiguousarray(2 * np.eye(n) + a + a.T)
    T = np.zeros_like(S)
    ref.ref_iter_tmat(_d(S), _d(T), n)
    T_or, it, err = O.newton_schulz(S, tol=1e-15, max_iter=10)
    assert np.max(np.abs(T - T_or)) < 1e-14


def _nl_inputs(s):
    nl = s.nl_atoms()
    return dict(nl=np.ascontiguousarray(nl, dtype=np.int32),
                kx=np.ascontiguousarray(s.kx, dtype=np.int32), ky=np.ascontiguousarray(s.ky, dtype=np.int32),
                kz=np.ascontiguousarray(s.kz, dtype=np.int32), typ=np.ascontiguousarray(s.atm_type, dtype=np.int32),
                pos=np.ascontiguousarray(s.pos), spl=np.ascontiguousarray(s.nl_proj.coef),
                vn=np.ascontiguousarray(s.nl_vnorm, dtype=np.float64), gz=np.ascontiguousarray(s.nl_gz0, dtype=np.float64))


def test_nl_struct_fact_pinned(ref, sysm):
    """Structure-factor nonlocal energy and coefficient forces of every
    state: CP_calc_Struct_Fact, CP_enl_matrix_calc, CP_enl_atm_forc_calc and
    CP_enl_force_calc against oracle.struct_fact / nl_energy_forces."""
    s = sysm
    ref.ref_nl_sf.argtypes = [C.c_int, ip, ip, ip, C.c_int, dp, dp, C.c_int, dp, ip, C.c_int, C.c_int, ip, C.c_int,
                              C.c_double, C.c_double, dp, dp, dp, C.c_double, C.c_double, dp, dp, dp, dp, dp]
    a = _nl_inputs(s)
    nnl = len(a["nl"])
    assert nnl > 0
    psi = np.ascontiguousarray(s.psi)
    occ = np.ascontiguousarray(s.occ, dtype=np.float64)
    sf = np.zeros((nnl, s.ng), dtype=np.complex128)
    fnl = np.zeros((s.nstate, s.ng), dtype=np.complex128)
    zmat = np.zeros((s.nstate, nnl))
    enl = np.zeros(s.nstate)
    fatm = np.zeros((s.natm, 3))
    ref.ref_nl_sf(s.ng, _i(a["kx"]), _i(a["ky"]), _i(a["kz"]), s.nstate, _d(psi.view(np.float64)), _d(occ), s.natm,
                  _d(a["pos"]), _i(a["typ"]), len(s.type_names), nnl, _i(a["nl"]), s.nl_proj.n, s.nl_proj.gmin,
                  s.nl_proj.dg, _d(a["spl"]), _d(a["vn"]), _d(a["gz"]), s.ecut_ry, s.box,
                  _d(sf.view(np.float64)), _d(fnl.view(np.float64)), _d(zmat), _d(enl), _d(fatm))
    sf_or, _ = O.struct_fact(s)
    f_or, e_or, z_or = O.nl_energy_forces(s.psi, s, sf_or)
    assert np.max(np.abs(sf - sf_or)) <= 1e-13 * np.max(np.abs(sf_or))
    assert np.max(np.abs(enl - e_or)) <= 1e-12 * np.max(np.abs(e_or))
    assert np.max(np.abs(fnl - f_or)) <= 1e-12 * np.max(np.abs(f_or))
    vn = s.nl_vnorm[s.atm_type[a["nl"]]] / s.vol
    assert np.max(np.abs(zmat - 2.0 * vn[None, :] * z_or)) <= 1e-12 * np.max(np.abs(zmat))
    fa_or = O.nl_sf_atom_forces(s.psi, s, sf_or)
    assert np.max(np.abs(fatm - fa_or)) <= 1e-11 * np.max(np.abs(fa_or))


@pytest.mark.parametrize("iteration", [1, 2])
def test_integrate_dyn_pinned(ref, sysm, iteration):
    """CP_integrate_dyn (thermostat off) against oracle.integrate_dyn: the
    half kicks with the g = 0 / kx = 0 conventions, the fictitious KE and the
    drift, per state, bit for bit up to rounding."""
    s = sysm
    rng = np.random.default_rng(5 + iteration)
    shape = s.psi.shape
    f = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) * 0.1
    v = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) * 1e-3
    dt = 5.0
    v_or, p_or, ke_or = O.integrate_dyn(f, v, s.psi, s, iteration, dt)
    ref.ref_integrate_dyn.argtypes = [C.c_int, C.c_int, C.c_double, dp, dp, dp, dp, C.c_int, C.c_int, C.c_int, dp]
    cm = np.ascontiguousarray(s.cmass, dtype=np.float64)
    for st in range(s.nstate):
        ff = np.ascontiguousarray(f[st].copy())
        vv = np.ascontiguousarray(v[st].copy())
        pp = np.ascontiguousarray(s.psi[st].copy())
        ke = C.c_double()
        ref.ref_integrate_dyn(s.ng, iteration, dt, _d(ff.view(np.float64)), _d(vv.view(np.float64)),
                              _d(pp.view(np.float64)), _d(cm), s.nkx0_red, s.nkx0_uni, s.nkx0_zero, C.byref(ke))
        r0 = s.nkx0_red
        assert np.max(np.abs(vv[r0:] - v_or[st, r0:])) <= 1e-14 * np.max(np.abs(v_or[st]))
        assert np.max(np.abs(pp[r0:] - p_or[st, r0:])) <= 1e-14 * np.max(np.abs(p_or[st]))
        assert abs(ke.value - ke_or[st]) <= 1e-13 * abs(ke_or[st])


@pytest.mark.parametrize("cg", [False, True])
def test_min_step_pinned(ref, sysm, cg):
    """CP_integrate_min_STD / CP_integrate_min_CG and CP_fovlap_calc against
    oracle.min_step / fovlap, per state."""
    s = sysm
    ref.ref_min_step.argtypes = [C.c_int, dp, dp, dp, ip, ip, ip, dp, C.c_double, C.c_double, C.c_double, C.c_double]
    ref.ref_fovlap.argtypes = [C.c_int, dp]
    ref.ref_fovlap.restype = C.c_double
    rng = np.random.default_rng(8)
    shape = s.psi.shape
    f = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) * 0.1
    conj0 = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) * 0.05 if cg else None
    gamma, dt = 0.37, 5.0
    p_or, c_or = O.min_step(s.psi, f, s, dt, conj0, gamma)
    kx, ky, kz = (np.ascontiguousarray(a, dtype=np.int32) for a in (s.kx, s.ky, s.kz))
    cm = np.ascontiguousarray(s.cmass, dtype=np.float64)
    for st in range(s.nstate):
        ff = np.ascontiguousarray(f[st].copy())
        pp = np.ascontiguousarray(s.psi[st].copy())
        cc = np.ascontiguousarray(conj0[st].copy()) if cg else None
        ref.ref_min_step(s.ng, _d(ff.view(np.float64)), _d(cc.view(np.float64)) if cg else None,
                         _d(pp.view(np.float64)), _i(kx), _i(ky), _i(kz), _d(cm), dt, gamma, s.box, s.ecut_ry)
        assert np.max(np.abs(pp - p_or[st])) <= 1e-14 * np.max(np.abs(p_or[st]))
        if cg:
            assert np.max(np.abs(cc - c_or[st])) <= 1e-14 * np.max(np.abs(c_or[st]))
        fv = ref.ref_fovlap(s.ng, _d(np.ascontiguousarray(f[st]).view(np.float64)))
        assert abs(fv - O.fovlap(f[st:st + 1])) <= 1e-13 * fv


@pytest.mark.parametrize("order", [4, 6])
def test_ees_nonlocal_pinned(ref, sysm, order):
    """EES nonlocal (cp_ees_nonlocal.C), l = 0 channel, in the three phases
    the reference runs on G-space and real-space chares, with the oracle's
    nonlocal-grid transforms in between: eesSetEesWghtGgrp (d(g)),
    eesProjGchare / eesYlmOnD (dyp, projPsiG), eesAtmBsplineRgrp +
    eesZmatRchare summed over planes (zmat), eesEnergyAtmForcRchare (ENL,
    atom forces, the scattered grid) and eesPsiForcGspace (F_NL), against
    oracle.ees_setup / ees_dyp / nl_ees_energy_forces."""
    s = sysm
    a = _nl_inputs(s)
    nnl = len(a["nl"])
    ees = O.ees_setup(s, scale=1.2, order=order)
    na, nb, nc = ees["grid"]
    occ = np.ascontiguousarray(s.occ, dtype=np.float64)
    ref.ref_ees_config.argtypes = [C.c_int, ip, ip, ip, C.c_int, dp, C.c_int, dp, ip, C.c_int, C.c_int, ip, C.c_int,
                                   C.c_double, C.c_double, dp, dp, dp, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int]
    ref.ref_ees_gproj.argtypes = [C.c_int, dp, dp, dp, dp]
    ref.ref_ees_gproj.restype = C.c_int
    ref.ref_ees_rspace.argtypes = [C.c_int, dp, dp, dp, dp, dp]
    ref.ref_ees_psi_forc.argtypes = [C.c_int, dp, dp]
    ref.ref_ees_config(s.ng, _i(a["kx"]), _i(a["ky"]), _i(a["kz"]), s.nstate, _d(occ), s.natm, _d(a["pos"]),
                       _i(a["typ"]), len(s.type_names), nnl, _i(a["nl"]), s.nl_proj.n, s.nl_proj.gmin, s.nl_proj.dg,
                       _d(a["spl"]), _d(a["vn"]), _d(a["gz"]), s.box, na, nb, nc, order)
    psi = np.ascontiguousarray(s.psi)
    d = np.zeros(s.ng, dtype=np.complex128)
    dyp = np.zeros((1, s.ng), dtype=np.complex128)
    proj = np.zeros((1, s.nstate, s.ng), dtype=np.complex128)
    assert ref.ref_ees_gproj(s.nstate, _d(psi.view(np.float64)), _d(d.view(np.float64)), _d(dyp.view(np.float64)),
                             _d(proj.view(np.float64))) == 1
    assert np.max(np.abs(d - ees["d"])) <= 1e-13 * np.max(np.abs(ees["d"]))
    dyp_or = O.ees_dyp(s, ees)
    assert np.max(np.abs(dyp[0] - dyp_or)) <= 1e-13 * np.max(np.abs(dyp_or))
    assert np.max(np.abs(proj[0] - np.conj(dyp_or[None, :] * s.psi))) <= 1e-13 * np.max(np.abs(proj))
    # phase 2 on the real-space grid: x padded to na + 2 as the reference stores it
    pr = O._nl_grid_g_to_r(proj[0], s, ees["grid"])                       # [nstate, nc, nb, na]
    prr = np.zeros((1, s.nstate, nc, nb, na + 2))
    prr[0, ..., :na] = pr
    zmat = np.zeros((s.nstate, nnl))
    enl = np.zeros(s.nstate)
    scr = np.zeros_like(prr)
    fatm = np.zeros((s.natm, 3))
    ref.ref_ees_rspace(s.nstate, _d(prr), _d(zmat), _d(enl), _d(scr), _d(fatm))
    f_or, e_or, z_or, fa_or = O.nl_ees_energy_forces(s.psi, s, ees, atom_forces=True)
    assert np.max(np.abs(zmat - z_or)) <= 1e-12 * np.max(np.abs(z_or))
    assert np.max(np.abs(enl - e_or)) <= 1e-12 * np.max(np.abs(e_or))
    assert np.max(np.abs(fatm - fa_or)) <= 1e-11 * np.max(np.abs(fa_or))
    assert np.max(np.abs(scr[0, ..., na:])) == 0.0
    # phase 3 back in G space
    P = O._nl_grid_r_to_g(scr[0, ..., :na], s, ees["grid"])
    fpsi = np.zeros((s.nstate, s.ng), dtype=np.complex128)
    ref.ref_ees_psi_forc(s.nstate, _d(np.ascontiguousarray(P).view(np.float64)), _d(fpsi.view(np.float64)))
    assert np.max(np.abs(fpsi - f_or)) <= 1e-12 * np.max(np.abs(f_or))


def test_gga_functional_pinned(ref, sysm):
    """CP_getGGAFunctional with Becke 88 and LYP (cp_grad_rho_ctrl.C,
    cp_becke.C) on the oracle's density and density gradient, with a dilute
    region so that the switching function and the rho_cut branch both run:
    df/drho, the h = df/d|grad rho| unit(grad rho) fields and EGGA against
    oracle.gga_point."""
    s = sysm
    nx, ny, nz = s.nfft
    rho = O.density(O.state_g_to_r(s.psi, s), s)
    # scale a slab down into the switching range (rho_cut = 5e-6, full on at ~2e-4)
    rho = rho.copy()
    slab = rho[: nz // 3]
    rho[: nz // 3] = 2e-4 * (slab / slab.max()) ** 4
    grad = O.density_gradient(rho, s)
    fx, fc, v_or, h_or = O.gga_point(rho, grad, s.gga_cut)
    e_or = float(np.sum(fx) + np.sum(fc)) * s.vol / s.npts
    sw = (rho > 0.1 * s.gga_cut) & (rho < 0.1 * s.gga_cut + 3.9 * s.gga_cut)
    assert sw.sum() > 100 and (rho <= 0.1 * s.gga_cut).sum() > 100
    xl = 2 * (nx // 2 + 1)

    def pad(a):
        p = np.zeros((nz, ny, xl))
        p[:, :, :nx] = a
        return p

    dpad, vks = pad(rho), pad(np.zeros_like(rho))
    g = [pad(grad[a]) for a in range(3)]
    e = ref.ref_gga(nx, ny, nz, _d(dpad), _d(g[0]), _d(g[1]), _d(g[2]), _d(vks), s.box, s.gga_cut, 1, 1)
    assert abs(e - e_or) <= 1e-12 * abs(e_or)
    assert np.max(np.abs(vks[:, :, :nx] - v_or)) <= 1e-12 * np.max(np.abs(v_or))
    for a in range(3):
        assert np.max(np.abs(g[a][:, :, :nx] - h_or[a])) <= 1e-12 * np.max(np.abs(h_or))


def test_rspace_ewald_pinned(ref, sysm):
    """CPRSPACEION::CP_getionforce (cp_rspace_ion.C): real-space Ewald energy
    and forces at the minimum image within half the box, the self term with
    the erf factor of the finite reciprocal sum and the background term,
    against oracle.ewald_rspace."""
    s = sysm
    ref.ref_rspace_ion.argtypes = [C.c_int, dp, dp, C.c_double, C.c_double, C.c_double, dp, dp, dp, dp]
    pos = np.ascontiguousarray(s.pos)
    q = np.ascontiguousarray(s.q, dtype=np.float64)
    er, es, eb = C.c_double(), C.c_double(), C.c_double()
    fatm = np.zeros((s.natm, 3))
    # reciprocal cutoff of the density sphere in Hartree: k_cut^2 = 2 ecut
    ref.ref_rspace_ion(s.natm, _d(pos), _d(q), s.alp_ewd, 0.5 * s.ecut_rho_g2, s.box, C.byref(er), C.byref(es),
                       C.byref(eb), _d(fatm))
    e_r, e_s, e_b, f_or = O.ewald_rspace(s)
    assert abs(er.value - e_r) <= 1e-12 * abs(e_r)
    assert abs(es.value - e_s) <= 1e-13 * abs(e_s)
    assert abs(eb.value - e_b) <= 1e-13 * abs(e_b)
    assert np.max(np.abs(fatm - f_or)) <= 1e-12 * np.max(np.abs(f_or))


@pytest.mark.parametrize("name,loc_opt,n_ang,label", [("O", 1, 1, 1), ("H", 0, 0, 0)])
def test_pseudopotential_splines_pinned(ref, name, loc_opt, n_ang, label):
    """make_vps_splin / slow_bess_vps / spline_fit (control_vps_params.C,
    friend_lib.C) on the shipped O (KB, s nonlocal, p local) and H (local)
    BLYP pseudopotentials, on the spline grid of the 8-water box at 70 Ry,
    against openatom_b200.pseudo: the tabulated values, the spline
    evaluated between the knots, the g = 0 limits, the charge and the KB
    norm.  Also checks that the packaged radial data equal the files."""
    from openatom_b200 import pseudo as P
    path = f"/root/reference/data/DATABASE/{name}_BLYP_PP30.pseud"
    if not os.path.exists(path):
        pytest.skip("reference pseudopotential files absent")
    ref.ref_vps_splin.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                  C.c_double, C.c_double, dp, dp, dp, dp, dp]
    grid = P.spline_grid(11.7, 70.0)
    gmin, gmin_spl, dg, nspl = grid
    vps = np.zeros((n_ang + 1, nspl, 4))
    gz, gz0, q = C.c_double(), C.c_double(), C.c_double()
    nrm = np.zeros(n_ang + 1)
    ref.ref_vps_splin(path.encode(), loc_opt, n_ang, label, nspl, dg, gmin_spl, gmin_spl + dg * nspl, gmin,
                      _d(vps), C.byref(gz), C.byref(gz0), C.byref(q), _d(nrm))
    pp = P.read_pseud(path)
    packed = np.load(P._DATA)
    assert np.array_equal(packed[f"{name}_v"], pp["v"]) and np.array_equal(packed[f"{name}_rphi"], pp["rphi"])
    tab = P.vps_tables(pp, loc_opt, label == 1, grid)
    rng = np.random.default_rng(1)
    gs = gmin_spl + dg * (nspl - 1) * rng.random(2000)

    def ev(c):
        i = np.clip(((gs - gmin_spl) / dg + 1.0).astype(np.int64), 1, nspl)
        h = gs - ((i - 1) * dg + gmin_spl)
        cc = c[i - 1]
        return ((cc[:, 3] * h + cc[:, 2]) * h + cc[:, 1]) * h + cc[:, 0]

    pairs = [(tab["vloc"], vps[loc_opt])]
    if label == 1:
        pairs.append((tab["proj"], vps[0]))
        assert abs(tab["vpsnorm"] - nrm[0]) <= 1e-13 * abs(nrm[0])
        assert abs(tab["gzvps0"] - gz0.value) <= 1e-13 * abs(gz0.value)
    for mine, theirs in pairs:
        scale = np.max(np.abs(theirs[:, 0]))
        assert np.max(np.abs(mine[:, 0] - theirs[:, 0])) <= 1e-13 * scale
        assert np.max(np.abs(ev(mine) - ev(theirs))) <= 1e-12 * scale
    assert abs(tab["gzvps"] - gz.value) <= 1e-12 * max(1.0, abs(gz.value))
    assert tab["q"] == q.value


@pytest.mark.parametrize("order", [4, 6])
def test_ees_local_pinned(ref, sysm, order):
    """The EES local pseudopotential and reciprocal Ewald path
    (cp_eext_ees_opt on, cp_hart_ext.C:492-1470) against the oracle's
    eesl_* restatement, phase by phase with the oracle's transforms between:
    the per-type B-spline grids (eesAtmBsplineRgrp + eesPackGridRchare),
    the g-space energies / vks / force transforms (eesSetEesWghtGgrp,
    eesHartEextGchare over the types, eesEwaldGchare), and the atom forces
    (eesAtmForceRchare, types and Ewald)."""
    s = sysm
    ntyp = len(s.type_names)
    grid = O.eesl_grid(s, 1.2, order)
    na, nb, nc = grid
    lda = 2 * (na // 2 + 1)
    ref.ref_eesl_pack.argtypes = [C.c_int, dp, ip, dp, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, dp]
    ref.ref_eesl_gspace.argtypes = [C.c_int, ip, ip, ip, dp, dp, C.c_int, C.c_double, C.c_double, dp, dp,
                                    C.c_double, C.c_double, dp, dp, dp, dp, dp, dp]
    ref.ref_eesl_force.argtypes = [dp, dp, dp]
    typ = np.ascontiguousarray(s.atm_type, dtype=np.int32)
    pos = np.ascontiguousarray(s.pos)
    q = np.ascontiguousarray(s.q)
    grids = np.zeros((ntyp, nc, nb, lda))
    ref.ref_eesl_pack(s.natm, _d(pos), _i(typ), _d(q), ntyp, s.box, na, nb, nc, order, _d(grids))
    Q, bs = O.eesl_pack(s, grid, order)
    assert np.max(np.abs(grids[..., :na] - Q)) <= 1e-14
    assert not np.any(grids[..., na:])
    # g-space on the density sphere, rho of the seeded states
    rho_r = O.density(O.state_g_to_r(s.psi, s), s)
    kx, ky, kz, g2 = O.rho_sphere(s)
    nx, ny, nz = s.nfft
    rho = np.ascontiguousarray(np.fft.rfftn(rho_r * (s.vol / s.npts))[kz % nz, ky % ny, kx])
    qhat = O.eesl_sf(Q, kx, ky, kz)
    b_or = O.eesl_bfactor(kx, ky, kz, grid, order)
    vks_or, eh_or, ee_or, ew_or, Y_or, Yt_or = O.eesl_gspace(rho, kx, ky, kz, g2, qhat, b_or, s)
    kx_, ky_, kz_ = (np.ascontiguousarray(a, dtype=np.int32) for a in (kx, ky, kz))
    sfg = np.ascontiguousarray(O.eesl_sf(grids[..., :na], kx, ky, kz))
    vks = np.zeros_like(rho)
    sftot = np.zeros_like(rho)
    b = np.zeros_like(rho)
    eh, ee, ew = C.c_double(), C.c_double(), C.c_double()
    ref.ref_eesl_gspace(len(kx), _i(kx_), _i(ky_), _i(kz_), _d(rho.view(np.float64)), _d(vks.view(np.float64)),
                        s.vloc.n, s.vloc.gmin, s.vloc.dg, _d(np.ascontiguousarray(s.vloc.coef)),
                        _d(np.ascontiguousarray(s.gzvps)), s.alp_ewd, s.ecut_ry, _d(sfg.view(np.float64)),
                        _d(sftot.view(np.float64)), _d(b.view(np.float64)), C.byref(eh), C.byref(ee), C.byref(ew))
    assert np.max(np.abs(b - b_or)) <= 1e-13
    assert abs(eh.value - eh_or) <= 1e-12 * abs(eh_or)
    assert abs(ee.value - ee_or) <= 1e-12 * abs(ee_or)
    assert abs(ew.value - ew_or) <= 1e-12 * abs(ew_or)
    assert np.max(np.abs(vks - vks_or)) <= 1e-12 * np.max(np.abs(vks_or))
    assert np.max(np.abs(sfg - Y_or)) <= 1e-12 * np.max(np.abs(Y_or))
    assert np.max(np.abs(sftot - Yt_or)) <= 1e-12 * np.max(np.abs(Yt_or))
    # forces from the back-transformed grids (x-padded for the reference)
    P = O.eesl_backtransform(sfg, kx, ky, kz, grid)
    Pt = O.eesl_backtransform(sftot, kx, ky, kz, grid)
    Pg = np.zeros((ntyp, nc, nb, lda))
    Pg[..., :na] = P
    Ptg = np.zeros((nc, nb, lda))
    Ptg[..., :na] = Pt
    fatm = np.zeros((s.natm, 3))
    ref.ref_eesl_force(_d(Pg), _d(Ptg), _d(fatm))
    f_or = O.eesl_forces(P, Pt, s, bs, grid)
    assert np.max(np.abs(fatm - f_or)) <= 1e-11 * np.max(np.abs(f_or))
    # and the composed oracle path equals the pieces
    s2 = copy.copy(s)
    s2.eext_ees = grid + (order,)
    _, eh2, ee2, ew2, f2 = O.hart_eext(rho_r, s2, want_forces=True)
    assert (eh2, ee2, ew2) == (eh_or, ee_or, ew_or)
    assert np.max(np.abs(f2 - f_or)) <= 1e-13 * np.max(np.abs(f_or))
