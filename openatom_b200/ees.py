"""Host-side setup of the EES (Euler exponential spline) nonlocal path.

Computed once per system, the way the reference's eesCache does at start-up:
the nonlocal grid size (``init_nonlocal_ees``,
``src_piny_physics_v1.0/interface/cp_ewald/set_cp_ewald.C:1329-1410``), the
complex B-spline factor of every g-vector (``get_bspline_wght1d``
``set_cp_ewald.C:1237-1325`` and ``CPNONLOCAL::eesSetEesWghtGgrp``
``abinito_physics/cp_nonlocal/cp_ees_nonlocal.C:60-160``) and the l = 0
projector factor dyp(g) = d(g) y00 p(|g|) of ``eesProjGchare`` (594-727).
The per-step work (atom B-splines, grid FFTs, Z, ENL, forces) runs on the GPU.
``local_grid`` gives the grid of the EES local pseudopotential path
(``init_eext_ees``), whose setup is otherwise done by the library.
"""
from __future__ import annotations

import math

import numpy as np

TWO_PI = 2.0 * math.pi


def _fft_size(n: int) -> int:
    """Smallest 2^a 3^b 5^c >= n (the radix rule of the GPU FFTs)."""
    while True:
        m = n
        for p in (2, 3, 5):
            while m % p == 0:
                m //= p
        if m == 1:
            return n
        n += 1


def nonlocal_grid(sysm, scale: float = 1.2, order: int = 6):
    """n = int(2 scale (kmax + 1)) per axis, at least 2 (kmax + 1), rounded up
    to an FFT size (cp_pseudo_ees_scale default 1.2, order default 6)."""
    grid = []
    for k in (sysm.kx, sysm.ky, sysm.kz):
        nk = int(np.max(np.abs(k))) + 1
        n = int(2.0 * scale * nk)
        if n < 2 * nk:
            n += 1
        grid.append(_fft_size(n))
    if min(grid) < order:
        raise ValueError("nonlocal grid smaller than the spline order")
    return tuple(grid)


def local_grid(sysm, scale: float = 1.2, order: int = 6):
    """EES grid of the local pseudopotential (``init_eext_ees``,
    ``set_cp_ewald.C:1419-1500``): n = int(2 scale (2 kmax + 1)) per axis, one
    more if below 2 (2 kmax + 1), rounded up to an FFT size; kmax of the
    state sphere.  The same scale and order keys as the nonlocal grid
    (cp_pseudo_ees_scale, cp_pseudo_ees_order)."""
    grid = []
    for k in (sysm.kx, sysm.ky, sysm.kz):
        nk = 2 * int(np.max(np.abs(k))) + 1
        n = int(2.0 * scale * nk)
        if n < 2 * nk:
            n += 1
        grid.append(_fft_size(n))
    if min(grid) < order:
        raise ValueError("EES local grid smaller than the spline order")
    return tuple(grid)


def _bspline_factor_1d(order: int, ngrid: int) -> np.ndarray:
    mk = np.zeros(order + 1)
    uk = np.arange(order + 1, dtype=np.float64)
    mk[1] = 1.0
    uk[1] = 1.0
    for n in range(3, order + 1):
        for k in range(n, 1, -1):
            mk[k] = (uk[k] * mk[k] + (n - uk[k]) * mk[k - 1]) / (n - 1)
        mk[1] = uk[1] * mk[1] / (n - 1)
    m = np.arange(ngrid)[:, None]
    k = np.arange(1, order)[None, :]
    ang = (TWO_PI / ngrid) * m * (k - 1)
    den = np.sum(np.cos(ang) * mk[1:order], axis=1) + 1j * np.sum(np.sin(ang) * mk[1:order], axis=1)
    num = np.exp(1j * (TWO_PI * (order - 1) / ngrid) * np.arange(ngrid))
    return num / den


def projector_factor(sysm, grid, order: int) -> np.ndarray:
    """dyp(g) = d(g) y00 p_t(|g|) for the (single) nonlocal atom type, as
    complex128 [ng]; at g = 0 the real part with p_t(0) = gzvps0."""
    nl = sysm.nl_atoms()
    if len(nl) == 0:
        raise ValueError("system has no nonlocal atoms")
    types = set(int(t) for t in sysm.atm_type[nl])
    if len(types) != 1:
        raise ValueError("the EES path here handles one nonlocal atom type")
    t = types.pop()
    na, nb, nc = grid
    ba, bb, bc = (_bspline_factor_1d(order, n) for n in grid)
    d = ba[sysm.kx % na] * bb[sysm.ky % nb] * bc[sysm.kz % nc]
    f = TWO_PI / sysm.box
    g = f * np.sqrt(sysm.kx.astype(np.float64) ** 2 + sysm.ky ** 2 + sysm.kz ** 2)
    g0 = g == 0.0
    p = sysm.nl_proj.eval(np.full(g.shape, t), np.where(g0, 1.0, g))
    p = np.where(g0, sysm.nl_gz0[t], p)
    y00 = 1.0 / math.sqrt(4.0 * math.pi)
    dyp = d * y00 * p
    dyp[g0] = (ba[0] * bb[0] * bc[0]).real * y00 * sysm.nl_gz0[t]
    return dyp
