"""G-space spline tables of the shipped real-space pseudopotentials.

The reference builds its local and Kleinman-Bylander (KB) nonlocal tables
from the ``.pseud`` files of ``data/DATABASE`` with ``make_vps_splin``
(``src_piny_physics_v1.0/interface/vps_params/control_vps_params.C:690-1262``),
``slow_bess_vps`` (``:1266-1527``) and the cubic ``spline_fit`` of
``friend_lib/friend_lib.C:134-200``, on the spline grid that
``set_cp_ewald.C:250-347`` derives from the density sphere.  This module does
the same for the l = 0 channels the GPU path uses:

* ``.pseud`` layout: ``nr rmax n_ang``, then ``z1 alpha1 z2 alpha2`` and
  ``zpol gamma`` (read as free-format numbers), then one block of nr rows
  ``v_l(r) r phi_l(r)`` per angular channel l = 0 .. n_ang on the grid
  r_i = (i - 1) rmax / nr;
* the local part is the channel loc_opt: f(g) = sum_{i >= 2} 4 pi dr
  j0(g r_i) r_i^2 v_loc(r_i) minus the Coulomb tails
  4 pi z_k exp(-g^2 / 4 alpha_k^2) / g^2, and its g -> 0 limit
  gzvps = 4 pi dr sum r_i^2 v_loc + 4 pi sum z_k / (4 alpha_k^2);
* each KB channel l != loc_opt: dv_l = v_l - v_loc, the projector
  p(g) = sum_{i >= 2} 4 pi dr j_l(g r_i) r_i (dv_l r phi_l)(r_i), its norm
  vpsnorm = 1 / (sum_i dr (r phi_l)^2 dv_l), and for l = 0 its g = 0 value
  gzvps0 = 4 pi dr sum_i r_i (dv_l r phi_l)(r_i);
* each table is a cubic spline on g_j = gmin_spl + (j - 1) dg_spl,
  j = 1 .. nsplin, with gmin_spl = 0.75 |g|_min and gmax_spl = 4/3 |g|_max of
  the density sphere and dg_spl = (gmax_spl - gmin_spl) / nsplin.
"""
from __future__ import annotations

import math
import os

import numpy as np

FOUR_PI = 4.0 * math.pi


def read_pseud(path: str) -> dict:
    """The header and the radial channels of a ``.pseud`` file."""
    with open(path) as f:
        tok = f.read().split()
    nr, rmax, nang = int(tok[0]), float(tok[1]), int(tok[2])
    z1, a1, z2, a2, zpol, gam = (float(t) for t in tok[3:9])
    body = np.array(tok[9:9 + 2 * nr * (nang + 1)], dtype=np.float64)
    if body.size != 2 * nr * (nang + 1):
        raise ValueError(f"{path}: {body.size // 2} radial rows, expected {nr * (nang + 1)}")
    body = body.reshape(nang + 1, nr, 2)
    return dict(nr=nr, rmax=rmax, nang=nang, z1=z1, a1=a1, z2=z2, a2=a2, zpol=zpol, gamma=gam,
                v=body[:, :, 0].copy(), rphi=body[:, :, 1].copy())


def spline_grid(box: float, ecut_ry: float, nsplin: int = 4000):
    """(gmin_true, gmin_spl, dg_spl, nsplin) of a cubic box: |g| over the
    nonzero points of the density sphere g^2 <= 4 Ecut[Ry]."""
    f = 2.0 * math.pi / box
    kmax = int(math.sqrt(4.0 * ecut_ry) / f) + 1
    k = np.arange(-kmax, kmax + 1, dtype=np.float64)
    g2 = f * f * (k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2)
    g2 = g2[(g2 > 0.0) & (g2 <= 4.0 * ecut_ry)]
    gmin, gmax = math.sqrt(float(g2.min())), math.sqrt(float(g2.max()))
    gmin_spl, gmax_spl = 0.75 * gmin, gmax * (4.0 / 3.0)
    return gmin, gmin_spl, (gmax_spl - gmin_spl) / nsplin, nsplin


def spline_fit(y: np.ndarray, x: np.ndarray) -> np.ndarray:
    """Cubic spline coefficients [n, 4] (c0 = y) with the end slopes taken
    from the first and last differences and the interior slopes from the
    tridiagonal continuity system, solved by forward elimination and back
    substitution (``spline_fit``, ``friend_lib.C:134-200``); c2 = c3 = 0 on
    the last point."""
    n = y.size
    c1 = np.zeros(n)
    c2 = np.zeros(n)
    c3 = np.zeros(n)
    d = np.zeros(n)
    diag = np.zeros(n)
    c1[0] = (y[1] - y[0]) / (x[1] - x[0])
    c1[n - 1] = (y[n - 1] - y[n - 2]) / (x[n - 1] - x[n - 2])
    diag[0] = 1.0
    d[1:] = x[1:] - x[:-1]
    diag[1:] = (y[1:] - y[:-1]) / d[1:]
    # interior right-hand sides and diagonals (m = 1 .. n-2, 0-based)
    m = np.arange(1, n - 1)
    c1[m] = 3.0 * (d[m] * diag[m + 1] + d[m + 1] * diag[m])
    diag[m] = 2.0 * (d[m] + d[m + 1])
    for i in range(1, n - 1):
        gq = -d[i + 1] / diag[i - 1]
        diag[i] += gq * d[i - 1]
        c1[i] += gq * c1[i - 1]
    for i in range(n - 2, 0, -1):
        c1[i] = (c1[i] - d[i] * c1[i + 1]) / diag[i]
    dx = x[1:] - x[:-1]
    dd1 = (y[1:] - y[:-1]) / dx
    dd3 = c1[:-1] + c1[1:] - 2.0 * dd1
    c2[:-1] = (dd1 - c1[:-1] - dd3) / dx
    c3[:-1] = dd3 / (dx * dx)
    return np.stack([y, c1, c2, c3], axis=1)


def _bessel_l0(vr: np.ndarray, r: np.ndarray, dr: float, g: np.ndarray, chunk: int = 256) -> np.ndarray:
    """sum_{i >= 2} 4 pi dr (sin(g r_i) / (g r_i)) r_i vr_i for every g."""
    out = np.zeros(g.size)
    rr, v = r[1:], vr[1:]
    for j0 in range(0, g.size, chunk):
        arg = np.outer(g[j0:j0 + chunk], rr)
        out[j0:j0 + chunk] = (FOUR_PI * dr) * ((np.sin(arg) / arg) * rr[None, :]) @ v
    return out


def vps_tables(pp: dict, loc_opt: int, kb: bool, grid) -> dict:
    """Local and (kb) l = 0 KB tables of one atom type on the spline grid
    ``grid`` = spline_grid(...): dict with vloc [nsplin, 4], gzvps, q, and
    for KB types proj [nsplin, 4], vpsnorm, gzvps0."""
    _, gmin_spl, dg, nspl = grid
    g = gmin_spl + dg * np.arange(nspl, dtype=np.float64)
    nr, rmax = pp["nr"], pp["rmax"]
    dr = rmax / nr
    r = dr * np.arange(nr, dtype=np.float64)
    vloc = pp["v"][loc_opt]
    # local part (ilong = 1): short-range Bessel transform minus the Coulomb tails
    vr = vloc * r
    f = _bessel_l0(vr, r, dr, g)
    gzvps = FOUR_PI * dr * float(np.sum(r[1:] * vr[1:]))
    z1, a1, z2, a2 = pp["z1"], pp["a1"], pp["z2"], pp["a2"]
    if z1 != 0.0 or z2 != 0.0:
        g2 = g * g
        f -= z1 * FOUR_PI * np.exp(-0.25 * g2 / (a1 * a1)) / g2 + z2 * FOUR_PI * np.exp(-0.25 * g2 / (a2 * a2)) / g2
        gzvps += FOUR_PI * (z1 / (4.0 * a1 * a1) + z2 / (4.0 * a2 * a2))
    if pp["zpol"] != 0.0:
        raise ValueError("polarisation corrections (zpol != 0) are not supported")
    out = dict(vloc=spline_fit(f, g), gzvps=gzvps, q=z1 + z2)
    if kb:
        if loc_opt == 0:
            raise ValueError("an l = 0 KB projector needs a local channel other than l = 0")
        # channel l = 0: dv r phi, its norm and its l = 0 Bessel transform (ilong = 0)
        rphi = pp["rphi"][0]
        vr0 = (pp["v"][0] - vloc) * rphi
        out["vpsnorm"] = 1.0 / float(np.sum(rphi * vr0 * dr))
        out["proj"] = spline_fit(_bessel_l0(vr0, r, dr, g), g)
        out["gzvps0"] = FOUR_PI * dr * float(np.sum(r[1:] * vr0[1:]))
    return out


_DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "blyp_pp30.npz")
# O: KB with the s channel nonlocal, p local (pi_md.vps: N_ANG 1, LOC_OPT 1);
# H: local only (N_ANG 0, LOC_OPT 0)
_WATER_TYPES = (("O", 1, True), ("H", 0, False))
_cache: dict = {}


def shipped_water_tables(box: float, ecut_ry: float, nsplin: int = 4000):
    """Spline tables of the shipped O / H BLYP pseudopotentials (type order O,
    H) on the spline grid of a cubic box at this cutoff: (gmin_spl, dg_spl,
    vloc [2, nsplin, 4], gzvps [2], proj [2, nsplin, 4] (zero for H),
    vpsnorm [2] (0 for H), gzvps0 [2]).  Cached per (box, cutoff)."""
    key = (float(box), float(ecut_ry), int(nsplin))
    if key in _cache:
        return _cache[key]
    d = np.load(_DATA)
    grid = spline_grid(box, ecut_ry, nsplin)
    vloc = np.zeros((2, nsplin, 4))
    proj = np.zeros((2, nsplin, 4))
    gz = np.zeros(2)
    vn = np.zeros(2)
    gz0 = np.zeros(2)
    for t, (name, loc, kb) in enumerate(_WATER_TYPES):
        pp = {k: d[f"{name}_{k}"][()] for k in ("nr", "rmax", "nang", "z1", "a1", "z2", "a2", "zpol", "gamma")}
        pp["nr"], pp["nang"] = int(pp["nr"]), int(pp["nang"])
        pp["v"], pp["rphi"] = d[f"{name}_v"], d[f"{name}_rphi"]
        tab = vps_tables(pp, loc, kb, grid)
        vloc[t], gz[t] = tab["vloc"], tab["gzvps"]
        if kb:
            proj[t], vn[t], gz0[t] = tab["proj"], tab["vpsnorm"], tab["gzvps0"]
    out = (grid[1], grid[2], vloc, gz, proj, vn, gz0)
    _cache[key] = out
    return out
