"""Seeded Gamma-point water systems in the layout OpenAtom's state chares use.

Everything a CP electronic step needs as input is generated here from a seed:
cell, atoms, the state g-sphere with its z-line run layout, fictitious masses,
local-pseudopotential spline tables and Löwdin-orthonormalised coefficients.

Layout conventions (all follow the reference):

* Gamma-point double packing: only kx >= 0 is stored.  The kx = 0 plane is
  stored completely (both (ky,kz) and (-ky,-kz)), kx > 0 points carry weight 2
  (``src_piny_physics_v1.0/abinito_physics/cp_nonlocal/cp_eke.C:72-110``).
* kx = 0 points come first; inside them the redundant half (ky < 0, or ky = 0
  and kz < 0) precedes g = 0, which precedes the unique half
  (``src_charm_driver/fft_slab_ctrl/stateSlab.C:299-370``).
* Points are grouped in z-lines of constant (kx, ky); every line holds a
  negative-kz run followed by a non-negative-kz run, which is how
  ``RunDescriptor`` pairs describe it (``include/RunDescriptor.h:17-24``,
  ``src_charm_driver/utility/util.C:936-990``).  The FFT index of kz < 0 is
  kz + nz (``src_charm_driver/fft_slab_ctrl/fftCache.C:460-507``).
* Coefficients are normalised so that S = Psi^T Psi = 2 I (closed shell, the
  occupation 2 folded into the norm; occupations are 1), which is the
  convention ``src_charm_driver/orthog_ctrl/ortho.C:233-244`` divides out.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

BOHR_PER_ANG = 1.0 / 0.529177210903
TWO_PI = 2.0 * math.pi


@dataclasses.dataclass
class SplineTable:
    """Cubic spline of a radial G-space function on a uniform |g| grid.

    Evaluated the way ``CPLOCAL::CP_get_vpsnow`` does
    (``abinito_physics/cp_local/cp_hart_ext.C:433-480``):
    i = clamp(int((g-gmin)/dg + 1), 1, n); h = g - ((i-1) dg + gmin);
    v = ((c3 h + c2) h + c1) h + c0, using coefficients of interval i-1.
    """
    gmin: float
    dg: float
    coef: np.ndarray  # [ntype, n, 4] float64 (c0, c1, c2, c3)

    @property
    def n(self) -> int:
        return self.coef.shape[1]

    def eval(self, itype: np.ndarray, g: np.ndarray) -> np.ndarray:
        i = ((g - self.gmin) / self.dg + 1.0).astype(np.int64)
        i = np.clip(i, 1, self.n)
        h = g - ((i - 1) * self.dg + self.gmin)
        c = self.coef[itype, i - 1]
        return ((c[..., 3] * h + c[..., 2]) * h + c[..., 1]) * h + c[..., 0]


@dataclasses.dataclass
class CPSystem:
    name: str
    seed: int
    box: float                      # cubic cell edge (bohr)
    nfft: tuple                     # (nx, ny, nz) state = density grid
    ecut_ry: float                  # state cutoff in Ry, compared with g^2
    nstate: int
    # atoms
    pos: np.ndarray                 # [natm, 3] bohr
    atm_type: np.ndarray            # [natm] int, 0 = O, 1 = H
    q: np.ndarray                   # [natm] valence charges
    type_names: tuple
    gzvps: np.ndarray               # [ntype] g=0 limit of the non-Coulomb local part
    vloc: SplineTable
    alp_ewd: float
    # g-sphere
    kx: np.ndarray
    ky: np.ndarray
    kz: np.ndarray
    line_kx: np.ndarray
    line_ky: np.ndarray
    line_off: np.ndarray
    line_nneg: np.ndarray
    line_npos: np.ndarray
    nkx0: int
    nkx0_red: int
    nkx0_uni: int
    nkx0_zero: int
    occ: np.ndarray
    cmass: np.ndarray
    psi: np.ndarray                 # [nstate, ng] complex128, S = 2 I
    dt: float = 5.0
    cmass0: float = 400.0
    # nonlocal (Kleinman-Bylander, l = 0) projector per type; vnorm = 0 for
    # types without a nonlocal channel (H in the shipped tables: local only)
    nl_proj: SplineTable | None = None
    nl_vnorm: np.ndarray | None = None
    nl_gz0: np.ndarray | None = None
    # exchange-correlation: "pz_lda" (Perdew-Zunger LDA, cp_pz_lda.C) or
    # "blyp" (Slater exchange + Becke 88 gradient correction + LYP
    # correlation, cp_becke.C / cp_grad_rho_ctrl.C: \cp_ggax_typ{becke}
    # \cp_ggac_typ{lyp}); gga_cut is \gradient_cutoff (default 5e-5)
    xc: str = "pz_lda"
    gga_cut: float = 5.0e-5
    # local pseudopotential and reciprocal Ewald sum by the EES method
    # (\cp_eext_ees_opt{on}): (na, nb, nc, order) of its B-spline grid, or
    # None for the structure-factor method
    eext_ees: tuple | None = None

    @property
    def vol(self) -> float:
        return self.box ** 3

    @property
    def ng(self) -> int:
        return int(self.kx.shape[0])

    @property
    def nlines(self) -> int:
        return int(self.line_kx.shape[0])

    @property
    def npts(self) -> int:
        return int(np.prod(self.nfft))

    @property
    def natm(self) -> int:
        return int(self.pos.shape[0])

    @property
    def ecut_rho_g2(self) -> float:
        """Density cutoff on g^2: 4x the state cutoff
        (``cp_hart_ext.C:113``: ecut4 = 8 * ecut[Ha])."""
        return 4.0 * self.ecut_ry

    def g2(self) -> np.ndarray:
        f = TWO_PI / self.box
        return (f * f) * (self.kx.astype(np.float64) ** 2 + self.ky ** 2 + self.kz ** 2)

    def kx_weight(self) -> np.ndarray:
        return np.where(self.kx == 0, 1.0, 2.0)

    def nl_atoms(self) -> np.ndarray:
        """Atoms with a nonlocal channel, grouped by type in type order (the
        order of cppseudo->nonlocal.map_nl)."""
        if self.nl_vnorm is None:
            return np.zeros(0, dtype=np.int64)
        out = [np.nonzero(self.atm_type == t)[0] for t in range(len(self.type_names)) if self.nl_vnorm[t] != 0.0]
        return np.concatenate(out) if out else np.zeros(0, dtype=np.int64)


# ----------------------------------------------------------------------------
# geometry
# ----------------------------------------------------------------------------

def _rotation(rng: np.random.Generator) -> np.ndarray:
    q, r = np.linalg.qr(rng.standard_normal((3, 3)))
    q = q * np.sign(np.diag(r))
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q


def water_box(nmol: int, box: float, rng: np.random.Generator,
              min_oo_ang: float = 2.6, oh_ang: float = 0.96,
              hoh_deg: float = 104.5):
    """Random sequential placement of rigid waters with O-O >= min_oo (periodic).

    The H-O-H angle is 104.5 degrees (gas-phase value; not given by the
    reference's water.parm).  Returns positions [3*nmol, 3] ordered
    O1 H1 H1 O2 H2 H2 ... and types (0 = O, 1 = H).
    """
    d_oo = min_oo_ang * BOHR_PER_ANG
    r_oh = oh_ang * BOHR_PER_ANG
    half = math.radians(hoh_deg) / 2.0
    local_h = np.array([[r_oh * math.sin(half), 0.0, r_oh * math.cos(half)],
                        [-r_oh * math.sin(half), 0.0, r_oh * math.cos(half)]])
    oxy = []
    for _ in range(nmol):
        for _attempt in range(200000):
            p = rng.random(3) * box
            ok = True
            for o in oxy:
                d = p - o
                d -= box * np.round(d / box)
                if d @ d < d_oo * d_oo:
                    ok = False
                    break
            if ok:
                oxy.append(p)
                break
        else:
            raise RuntimeError("could not place water molecule; box too dense")
    pos, typ = [], []
    for o in oxy:
        rot = _rotation(rng)
        pos.append(o)
        typ.append(0)
        for h in local_h:
            pos.append(o + rot @ h)
            typ.append(1)
    return np.array(pos), np.array(typ, dtype=np.int32)


# ----------------------------------------------------------------------------
# g-sphere and run layout
# ----------------------------------------------------------------------------

def state_sphere(box: float, ecut_ry: float, nfft):
    """Half sphere g^2 <= ecut (Ry) in the reference order (see module doc)."""
    f = TWO_PI / box
    kmax = int(math.floor(math.sqrt(ecut_ry) / f)) + 1
    nx, ny, nz = nfft
    if 2 * kmax + 1 > min(nfft):
        raise ValueError("FFT grid too small for the state cutoff")
    kx_l, ky_l, kz_l = [], [], []
    lkx, lky, loff, lneg, lpos = [], [], [], [], []
    for ax in range(0, kmax + 1):
        for ay in range(-kmax, kmax + 1):
            rem = ecut_ry / (f * f) - ax * ax - ay * ay
            if rem < 0:
                continue
            a = int(math.floor(math.sqrt(rem) + 1e-12))
            zs = [z for z in range(-a, a + 1) if (ax * ax + ay * ay + z * z) * f * f <= ecut_ry]
            if not zs:
                continue
            lkx.append(ax)
            lky.append(ay)
            loff.append(len(kx_l))
            neg = [z for z in zs if z < 0]
            pos = [z for z in zs if z >= 0]
            lneg.append(len(neg))
            lpos.append(len(pos))
            for z in neg + pos:
                kx_l.append(ax)
                ky_l.append(ay)
                kz_l.append(z)
    kx = np.array(kx_l, dtype=np.int32)
    ky = np.array(ky_l, dtype=np.int32)
    kz = np.array(kz_l, dtype=np.int32)
    k0 = kx == 0
    red = k0 & ((ky < 0) | ((ky == 0) & (kz < 0)))
    zero = k0 & (ky == 0) & (kz == 0)
    nkx0 = int(k0.sum())
    nkx0_red = int(red.sum())
    nkx0_zero = int(zero.sum())
    nkx0_uni = nkx0 - nkx0_red
    # layout check the reference makes (stateSlab.C:330-370)
    assert np.all(kx[:nkx0] == 0)
    assert np.all(red[:nkx0_red]) and not np.any(red[nkx0_red:])
    return (kx, ky, kz, np.array(lkx, np.int32), np.array(lky, np.int32),
            np.array(loff, np.int32), np.array(lneg, np.int32), np.array(lpos, np.int32),
            nkx0, nkx0_red, nkx0_uni, nkx0_zero)


def create_mass(kx, g2, cmass0: float, ecut_mass: float) -> np.ndarray:
    """``CPINTEGRATE::CP_create_mass`` (``cp_control_integrate.C:136-210``)
    with cmass0 given directly in a.u.: m = w*cmass0 below the mass cutoff,
    w*g2*cmass0/ecut_mass above it, w = 1 for kx = 0 and 2 otherwise."""
    w = np.where(kx == 0, 1.0, 2.0)
    return np.where(g2 > ecut_mass, w * g2 * (cmass0 / ecut_mass), w * cmass0)


# ----------------------------------------------------------------------------
# local pseudopotential (analytic stand-in, tabulated as the reference's spline)
# ----------------------------------------------------------------------------

def _cubic_coeffs(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    from scipy.interpolate import CubicSpline
    cs = CubicSpline(x, y, bc_type="natural")
    c = cs.c  # [4, n-1] highest power first
    out = np.zeros((x.shape[0], 4))
    out[:-1, 0] = c[3]
    out[:-1, 1] = c[2]
    out[:-1, 2] = c[1]
    out[:-1, 3] = c[0]
    out[-1, 0] = y[-1]
    return out


def gaussian_nl_table(amp, rnl, gmax: float, nspl: int = 4000):
    """l = 0 KB projector p(g) = amp exp(-g^2 rnl^2 / 2) per type on the same
    kind of grid as the local table; p(0) = amp is the gzvps0 term
    (cp_struct_fact.C:get_rad_proj)."""
    gmin = gmax / nspl
    g = gmin + np.arange(nspl) * ((gmax - gmin) / (nspl - 1))
    dg = g[1] - g[0]
    coef = np.zeros((len(amp), nspl, 4))
    for t, (a, r) in enumerate(zip(amp, rnl)):
        coef[t] = _cubic_coeffs(g, a * np.exp(-0.5 * (g * r) ** 2))
    return SplineTable(gmin=float(gmin), dg=float(dg), coef=coef), np.array(amp, dtype=np.float64)


def gaussian_vloc_table(zval, rloc, gmax: float, nspl: int = 4000):
    """Local pseudopotential v(g) = -4 pi Z exp(-g^2 rloc^2 / 2) / g^2 per type
    (a Goedecker-style Gaussian-smeared ion core), tabulated on a uniform grid
    from gmin = dg to gmax.  gzvps is its non-Coulomb g -> 0 limit
    2 pi Z rloc^2, which the reference adds at g = 0 (cp_hart_ext.C:366-390).
    """
    gmin = gmax / nspl
    g = gmin + np.arange(nspl) * ((gmax - gmin) / (nspl - 1))
    dg = g[1] - g[0]
    coef = np.zeros((len(zval), nspl, 4))
    gz = np.zeros(len(zval))
    for t, (z, r) in enumerate(zip(zval, rloc)):
        v = -4.0 * math.pi * z * np.exp(-0.5 * (g * r) ** 2) / (g * g)
        coef[t] = _cubic_coeffs(g, v)
        gz[t] = 2.0 * math.pi * z * r * r
    return SplineTable(gmin=float(gmin), dg=float(dg), coef=coef), gz


# ----------------------------------------------------------------------------
# coefficients
# ----------------------------------------------------------------------------

def gamma_overlap(psi: np.ndarray, kx: np.ndarray) -> np.ndarray:
    """S_ij = sum over the full sphere of Re(c_i^* c_j), evaluated on the half
    sphere as 2*Re(sum_{kx>0}) + Re(sum_{kx=0}) -- the PairCalculator result
    with alpha = 2 and the kx = 0 rows scaled by 1/sqrt(2)
    (``src_charm_driver/paircalc/ckPairCalculator.C:821-893``)."""
    w = np.where(kx == 0, 1.0, 2.0)
    a = np.concatenate([psi.real, psi.imag], axis=1)
    ww = np.concatenate([w, w])
    return (a * ww) @ a.T


def symmetrize_kx0(psi, kx, ky, kz):
    """Make the redundant kx=0 half the conjugate of the unique half and zero
    Im c(g=0), so psi(r) is real."""
    k0 = np.nonzero(kx == 0)[0]
    key = {(int(ky[i]), int(kz[i])): i for i in k0}
    for i in k0:
        a, b = int(ky[i]), int(kz[i])
        red = a < 0 or (a == 0 and b < 0)
        if red:
            j = key[(-a, -b)]
            psi[..., i] = np.conj(psi[..., j])
        elif a == 0 and b == 0:
            psi[..., i] = psi[..., i].real
    return psi


def lowdin_normalize(psi, kx, occ_norm: float = 2.0):
    s = gamma_overlap(psi, kx) / occ_norm
    w, v = np.linalg.eigh(s)
    t = (v / np.sqrt(w)) @ v.T
    return t @ psi


def random_coefficients(nstate, kx, ky, kz, g2, rng):
    """c(g) ~ N(0,1) (1 + i N(0,1)) / (1 + g^2), then Gamma-symmetrised and
    Löwdin-orthonormalised in FP64 to S = 2 I."""
    ng = kx.shape[0]
    amp = 1.0 / (1.0 + g2)
    psi = (rng.standard_normal((nstate, ng)) + 1j * rng.standard_normal((nstate, ng))) * amp
    psi = symmetrize_kx0(psi, kx, ky, kz)
    psi = lowdin_normalize(psi, kx)
    return symmetrize_kx0(psi, kx, ky, kz)


# ----------------------------------------------------------------------------
# presets
# ----------------------------------------------------------------------------

PRESETS = {
    # 8 H2O, 11.7 bohr, 70 Ry, 64^3, 32 states
    "w8": dict(nmol=8, box=11.7, ecut_ry=70.0, nfft=(64, 64, 64)),
    # 32 H2O, 18.6 bohr, 80 Ry, 108^3, 128 states
    "w32": dict(nmol=32, box=18.6, ecut_ry=80.0, nfft=(108, 108, 108)),
    # 128 H2O, 29.6 bohr, 70 Ry, 160^3, 512 states
    "w128": dict(nmol=128, box=29.6, ecut_ry=70.0, nfft=(160, 160, 160)),
    # tiny case for fast tests: 2 H2O, 7 bohr, 20 Ry, 24^3, 8 states
    "w2": dict(nmol=2, box=7.0, ecut_ry=20.0, nfft=(24, 24, 24)),
    # small odd-radix case: 4 H2O, 9 bohr, 30 Ry, 36^3 (36 = 4*3*3), 16 states
    "w4": dict(nmol=4, box=9.0, ecut_ry=30.0, nfft=(36, 36, 36)),
}


# atom masses in amu (O, H as in the reference's water examples) and the
# amu -> electron-mass factor of PINY (piny_constants.h:55)
ATOM_MASS_AMU = {"O": 15.9994, "H": 1.00794}
PROT_MASS = 1822.8885


def atom_masses(sysm) -> np.ndarray:
    """[natm] atom masses in electron masses, for oa_gpu_set_ions."""
    return np.array([ATOM_MASS_AMU[sysm.type_names[int(t)]] for t in sysm.atm_type]) * PROT_MASS


def make_system(preset: str = "w8", seed: int = 1234, nstate: int | None = None,
                ecut_mass: float = 1.0e30, cmass0: float = 400.0, dt: float = 5.0,
                xc: str = "pz_lda", pseudo: str = "shipped", eext_ees_order: int | None = None,
                ees_scale: float = 1.2, **over) -> CPSystem:
    """A seeded water system of a preset.  pseudo: "shipped" splines the
    reference's O / H BLYP pseudopotentials (openatom_b200.pseudo, the
    make_vps_splin algorithm) on this box's spline grid; "analytic" uses
    Gaussian stand-ins (a Gaussian-smeared ion core and a Gaussian s
    projector).  eext_ees_order: the local pseudopotential and reciprocal
    Ewald sum by the EES method with B-splines of this order on the grid of
    ees.local_grid(ees_scale) (cp_eext_ees_opt on); None: structure factors."""
    if xc not in ("pz_lda", "blyp"):
        raise ValueError("xc must be 'pz_lda' or 'blyp'")
    if pseudo not in ("shipped", "analytic"):
        raise ValueError("pseudo must be 'shipped' or 'analytic'")
    p = dict(PRESETS[preset])
    p.update(over)
    nmol, box, ecut_ry, nfft = p["nmol"], p["box"], p["ecut_ry"], tuple(p["nfft"])
    if nstate is None:
        nstate = 4 * nmol  # 8 valence electrons per water, 2 per state
    rng = np.random.default_rng(seed)
    pos, typ = water_box(nmol, box, rng)
    q = np.where(typ == 0, 6.0, 1.0)
    (kx, ky, kz, lkx, lky, loff, lneg, lpos, nkx0, nred, nuni, nzero) = state_sphere(box, ecut_ry, nfft)
    f = TWO_PI / box
    g2 = f * f * (kx.astype(np.float64) ** 2 + ky ** 2 + kz ** 2)
    if pseudo == "shipped":
        # O: one s-channel KB projector (p local); H: local only (data/DATABASE/pi_md.vps)
        from .pseudo import shipped_water_tables
        gmin_s, dg_s, vl, gz, pj, nl_vnorm, nl_gz0 = shipped_water_tables(box, ecut_ry)
        vloc = SplineTable(gmin=float(gmin_s), dg=float(dg_s), coef=vl)
        nl_proj = SplineTable(gmin=float(gmin_s), dg=float(dg_s), coef=pj)
    else:
        gmax = math.sqrt(4.0 * ecut_ry) * 1.05 + 0.5
        vloc, gz = gaussian_vloc_table([6.0, 1.0], [0.247, 0.2], gmax)
        nl_proj, nl_gz0 = gaussian_nl_table([12.0, 0.0], [0.35, 0.35], gmax)
        nl_vnorm = np.array([0.9, 0.0])
    psi = random_coefficients(nstate, kx, ky, kz, g2, rng)
    cmass = create_mass(kx, g2, cmass0, ecut_mass)
    # Ewald splitting parameter: alpha = 3.5 / (L/2) style default (screening
    # length well inside the box)
    alp_ewd = 7.0 / box
    sysm = CPSystem(name=preset, seed=seed, box=box, nfft=nfft, ecut_ry=ecut_ry,
                    nstate=nstate, pos=pos, atm_type=typ, q=q, type_names=("O", "H"),
                    gzvps=gz, vloc=vloc, alp_ewd=alp_ewd, kx=kx, ky=ky, kz=kz,
                    line_kx=lkx, line_ky=lky, line_off=loff, line_nneg=lneg, line_npos=lpos,
                    nkx0=nkx0, nkx0_red=nred, nkx0_uni=nuni, nkx0_zero=nzero,
                    occ=np.ones(nstate), cmass=cmass, psi=psi, dt=dt, cmass0=cmass0,
                    nl_proj=nl_proj, nl_vnorm=nl_vnorm, nl_gz0=nl_gz0, xc=xc)
    if eext_ees_order is not None:
        from .ees import local_grid
        sysm.eext_ees = local_grid(sysm, ees_scale, int(eext_ees_order)) + (int(eext_ees_order),)
    return sysm


def batch_systems(seed, nsys):
    """Seeded set of uneven water systems for the batching form: 8-32 H2O at
    about 1 g/cc, 4 states per molecule (32-128), 60/70/80 Ry, each on the
    smallest two-pass grid that holds its density sphere (4 kmax)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(nsys):
        nmol = int(rng.integers(8, 33))
        ecut = float(rng.choice([60.0, 70.0, 80.0]))
        box = 18.6 * (nmol / 32.0) ** (1.0 / 3.0)
        kmax = int(math.floor(math.sqrt(ecut) / (2.0 * math.pi / box))) + 1
        grid = next(g for g in (64, 96, 108, 160) if g >= 4 * kmax)
        out.append(make_system("w32", seed=seed + 101 * i, nmol=nmol, box=box, ecut_ry=ecut,
                               nfft=(grid, grid, grid), ecut_mass=2.0, cmass0=400.0, dt=5.0))
    return out
