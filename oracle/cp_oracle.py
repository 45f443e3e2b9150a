"""CPU oracle for the OpenAtom Gamma-point CP electronic step (FP64, numpy).

TEST INFRASTRUCTURE ONLY.  This module is the checker: only the tests, the
smoke check in ``__graft_entry__`` and the ``cpu_baseline`` / ``--impl
reference`` legs of ``bench.py`` may import it.  The product path
(``openatom_b200``) never calls it and fails loudly without its CUDA library.

Each function restates one reference routine and cites it.  FFTs use numpy's
pocketfft, GEMMs use numpy BLAS: FFTW2 / Fortran BLAS / the Charm-FFT library
of the reference are not present, so parity at those boundaries is pinned by
mathematics (any correct FP64 FFT/GEMM), while the physics kernels
(cp_eke, cp_pz_lda, cp_hart_ext, Newton-Schulz, cp_dynamics) are pinned
against the reference's own source compiled into ``oracle/_ref`` (see
``oracle/build_ref.sh`` and ``tests/test_oracle_pin.py``).

Sign conventions (``src_charm_driver/fft_slab_ctrl/fftCache.C:100-160``):
state "forward" plans are FFTW_FORWARD (exp(-i g.r)) and the c2r x-transform
is preceded by conjugation (``fftCache.C:1206-1212``), so
psi(r) = sum_{full sphere} c(g) exp(-i g.r); the backward path uses
exp(+i g.r).  The density forward transform is exp(-i g.r) with the V/N
volume factor (``CP_Rho_RealSpacePlane.C:846-851``).
"""
from __future__ import annotations

import math

import numpy as np

TWO_PI = 2.0 * math.pi

_FFT_WORKERS = 1


def set_fft_workers(n: int):
    """Threads for the oracle's FFTs (scipy.fft workers); 1 = numpy."""
    global _FFT_WORKERS
    _FFT_WORKERS = max(1, int(n))


def _fftn(a, axes=None):
    if _FFT_WORKERS > 1:
        import scipy.fft as sf
        return sf.fftn(a, axes=axes, workers=_FFT_WORKERS)
    return np.fft.fftn(a, axes=axes)


def _ifftn(a, axes=None):
    if _FFT_WORKERS > 1:
        import scipy.fft as sf
        return sf.ifftn(a, axes=axes, workers=_FFT_WORKERS)
    return np.fft.ifftn(a, axes=axes)


def _rfftn(a, axes=None):
    if _FFT_WORKERS > 1:
        import scipy.fft as sf
        return sf.rfftn(a, axes=axes, workers=_FFT_WORKERS)
    return np.fft.rfftn(a, axes=axes)


def _irfftn(a, s, axes=None):
    if _FFT_WORKERS > 1:
        import scipy.fft as sf
        return sf.irfftn(a, s=s, axes=axes, workers=_FFT_WORKERS)
    return np.fft.irfftn(a, s=s, axes=axes)


# ----------------------------------------------------------------------------
# sphere <-> grid
# ----------------------------------------------------------------------------

def expand_gspace(packed, sysm):
    """``FFTcache::expandGSpace`` (``fftCache.C:460-507``): packed runs ->
    zero-filled z-lines [.., nlines, nz]; kz < 0 goes to index kz + nz."""
    nz = sysm.nfft[2]
    out = np.zeros(packed.shape[:-1] + (sysm.nlines, nz), dtype=packed.dtype)
    line = np.repeat(np.arange(sysm.nlines), sysm.line_nneg + sysm.line_npos)
    out[..., line, sysm.kz % nz] = packed
    return out


def pack_gspace(lines, sysm):
    """``FFTcache::packGSpace`` (``fftCache.C:517-553``)."""
    nz = sysm.nfft[2]
    line = np.repeat(np.arange(sysm.nlines), sysm.line_nneg + sysm.line_npos)
    return lines[..., line, sysm.kz % nz]


def _full_grid(coef, kx, ky, kz, nfft, hermitian_partner=True):
    """Scatter half-sphere coefficients onto a full [.., nz, ny, nx] grid and
    add the Hermitian partner c(-g) = conj(c(g)) for kx > 0."""
    nx, ny, nz = nfft
    out = np.zeros(coef.shape[:-1] + (nz, ny, nx), dtype=np.complex128)
    out[..., kz % nz, ky % ny, kx % nx] = coef
    if hermitian_partner:
        m = kx > 0
        out[..., (-kz[m]) % nz, (-ky[m]) % ny, (-kx[m]) % nx] = np.conj(coef[..., m])
    return out


def _half_grid(coef, kx, ky, kz, nfft):
    """Scatter half-sphere coefficients (kx >= 0, the whole kx = 0 plane) onto
    the r2c half grid [.., nz, ny, nx/2 + 1]."""
    nx, ny, nz = nfft
    out = np.zeros(coef.shape[:-1] + (nz, ny, nx // 2 + 1), dtype=np.complex128)
    out[..., kz % nz, ky % ny, kx] = coef
    return out


def state_g_to_r(psi, sysm):
    """G-sphere -> real space for each state: the composition of
    ``doStpFFTGtoR_Gchare`` (expand + z FFT, ``fftCache.C:1133-1159``), the
    z->R transpose (``CP_State_GSpacePlane.C:1448-1517``,
    ``CP_State_RealSpacePlane.C:186-271``) and ``doStpFFTGtoR_Rchare``
    (y FFT, conjugate, c2r x FFT, ``fftCache.C:1167-1243``).
    psi(r) = sum_{full sphere} c(g) exp(-i g.r) is real, so it equals
    N * c2r[conj(c)] on the kx >= 0 half grid (the Hermitian partners
    c(-g) = conj(c(g)) are implied, as in the reference's c2r x transform).
    Returns psi(r) as float64 [nstate, nz, ny, nx]."""
    nx, ny, nz = sysm.nfft
    npts = nx * ny * nz
    out = np.empty(psi.shape[:-1] + (nz, ny, nx))
    flat_in = psi.reshape(-1, psi.shape[-1])
    flat_out = out.reshape(-1, nz, ny, nx)
    for c0 in range(0, flat_in.shape[0], 16):
        half = _half_grid(np.conj(flat_in[c0:c0 + 16]), sysm.kx, sysm.ky, sysm.kz, sysm.nfft)
        flat_out[c0:c0 + 16] = _irfftn(half, s=(nz, ny, nx), axes=(-3, -2, -1)) * npts
    return out


def state_r_to_g(fr, sysm):
    """Real space -> g-sphere, unnormalised exp(+i g.r): ``doStpFFTRtoG_Rchare``
    (r2c x, conjugate, y FFT, ``fftCache.C:1252-1319``), transpose back, and
    ``doStpFFTRtoG_Gchare`` (z FFT + pack, ``fftCache.C:1099-1123``).
    For real f(r), sum_r f(r) exp(+i g.r) = conj(r2c[f](g)) on kx >= 0."""
    nx, ny, nz = sysm.nfft
    flat = fr.reshape(-1, nz, ny, nx)
    out = np.empty((flat.shape[0], sysm.ng), dtype=np.complex128)
    for c0 in range(0, flat.shape[0], 16):
        half = _rfftn(flat[c0:c0 + 16], axes=(-3, -2, -1))
        out[c0:c0 + 16] = np.conj(half[:, sysm.kz % nz, sysm.ky % ny, sysm.kx])
    return out.reshape(fr.shape[:-3] + (sysm.ng,))


# ----------------------------------------------------------------------------
# density, XC, Hartree + local
# ----------------------------------------------------------------------------

def density(psir, sysm):
    """rho(r) = sum_s occ_s w_k psi_s(r)^2 / V
    (``CP_State_RealSpacePlane.C:349-363`` then the probScale = 1/V scaling
    of ``CP_Rho_RealSpacePlane.C:136-138,500``)."""
    return np.einsum("s,szyx->zyx", sysm.occ, psir * psir) / sysm.vol


def pz_lda(rho, vol, npts, lyp=False):
    """``CPXCFNCTS::CP_exc_calc`` (``abinito_physics/cp_xc_fnctl/cp_pz_lda.C:23-175``):
    Perdew-Zunger LDA.  With LYP correlation on (``cp_lyp``, ``:66``) the PZ
    correlation is dropped and only Slater exchange remains.  Returns
    (vxc(r), exc, muxc)."""
    gamma, beta1, beta2 = -0.14230, 1.05290, 0.33340
    au, bu, cu, du = 0.03110, -0.0480, 0.00200, -0.01160
    power = 1.0 / 3.0
    rat1 = (7.0 / 6.0) * beta1
    rat2 = (4.0 / 3.0) * beta2
    fpin = 4.0 * math.pi * rho
    rs = np.power(3.0 / fpin, power)
    sqtrs = np.sqrt(rs)
    xfact = -np.power(3.0 * rho / math.pi, power)
    hi = rs >= 1.0
    cf1 = 1.0 + beta1 * sqtrs + beta2 * rs
    cf2 = 1.0 + rat1 * sqtrs + rat2 * rs
    c_hi = gamma / cf1
    m_hi = c_hi * (cf2 / cf1)
    with np.errstate(divide="ignore", invalid="ignore"):
        lnrs = np.log(rs)
    c_lo = au * lnrs + bu + cu * rs * lnrs + du * rs
    m_lo = (au * lnrs + (bu - power * au) + 2.0 * power * cu * rs * lnrs
            + power * (2.0 * du - cu) * rs)
    cfact = np.where(hi, c_hi, c_lo)
    mufact = np.where(hi, m_hi, m_lo)
    if lyp:
        cfact = cfact * 0.0
        mufact = mufact * 0.0
    ex = float(np.sum(xfact * rho)) * 0.75
    ec = float(np.sum(cfact * rho))
    v = xfact + mufact
    vxc_sum = float(np.sum(v * rho))
    vscale = vol / npts
    return v, (ex + ec) * vscale, vxc_sum * vscale


def rho_sphere(sysm):
    """Density g-points: kx >= 0 half of g^2 <= 4 Ecut with the whole kx = 0
    plane (weight 1 on kx = 0, 2 elsewhere, ``cp_hart_ext.C:196-205``)."""
    nx, ny, nz = sysm.nfft
    f = TWO_PI / sysm.box
    kxs = np.arange(0, nx // 2 + 1)
    kys = np.arange(-(ny // 2), ny - ny // 2)
    kzs = np.arange(-(nz // 2), nz - nz // 2)
    KX, KY, KZ = np.meshgrid(kxs, kys, kzs, indexing="ij")
    g2 = f * f * (KX ** 2 + KY ** 2 + KZ ** 2)
    m = (g2 <= sysm.ecut_rho_g2)
    return KX[m], KY[m], KZ[m], g2[m]


def _phase_sums(sysm, kx, ky, kz, weights):
    """sum_a weights[k, a] exp(i g.R_a) at the g-points (kx, ky, kz), one row
    per weight vector, with the phase factorised per axis
    exp(i g.R) = exp(i gx x) exp(i gy y) exp(i gz z): the (kx, ky) products of
    the atoms times the kz phases is one complex GEMM per weight vector."""
    f = TWO_PI / sysm.box
    pos = sysm.pos
    ax = [np.arange(int(k.min()), int(k.max()) + 1) for k in (kx, ky, kz)]
    ex, ey, ez = (np.exp(1j * f * np.outer(pos[:, d], ax[d])) for d in range(3))
    nxy = ax[0].size * ax[1].size
    exy = (ex[:, :, None] * ey[:, None, :]).reshape(pos.shape[0], nxy)
    ix, iy, iz = kx - ax[0][0], ky - ax[1][0], kz - ax[2][0]
    out = []
    for w in weights:
        full = ((exy * w[:, None]).T @ ez).reshape(ax[0].size, ax[1].size, ax[2].size)
        out.append(full[ix, iy, iz])
    return out


def hart_eext(rho_r, sysm, want_forces=False):
    """``CPLOCAL::CP_hart_eext_calc`` (``abinito_physics/cp_local/cp_hart_ext.C:56-431``)
    on rho(g) = FFT_-[rho(r) V/N] (``CP_Rho_RealSpacePlane.C:846-851``).
    Returns (vks_hart_ext(r), ehart, eext, ewald_recip[, fatm]).  A system
    with eext_ees set takes the EES method (hart_eext_ees)."""
    if getattr(sysm, "eext_ees", None) is not None:
        return hart_eext_ees(rho_r, sysm, want_forces)
    nx, ny, nz = sysm.nfft
    n = nx * ny * nz
    vol = sysm.vol
    rhog_half = _rfftn(rho_r * (vol / n))
    kx, ky, kz, g2 = rho_sphere(sysm)
    rho = rhog_half[kz % nz, ky % ny, kx]
    f = TWO_PI / sysm.box
    gx, gy, gz = f * kx, f * ky, f * kz
    nz0 = g2 != 0
    w = np.where(kx == 0, 1.0, 2.0)
    # Hartree
    hf = np.zeros_like(g2)
    hf[nz0] = 4.0 * math.pi / (g2[nz0] * vol)
    ehart = float(np.sum(hf * np.abs(rho) ** 2 * w)) / 2.0
    vks = rho * hf
    # structure factors sum_a exp(i g.R_a) per atom type and with the ion
    # charges, and the local pseudopotential
    g = np.sqrt(g2)
    ntyp = len(sysm.type_names)
    vtyp = np.stack([sysm.vloc.eval(np.full(g.shape, t), g) for t in range(ntyp)], axis=1) / vol
    sums = _phase_sums(sysm, kx, ky, kz,
                       [(sysm.atm_type == t).astype(np.float64) for t in range(ntyp)] + [np.asarray(sysm.q, float)])
    vext = sum(vtyp[:, t] * sums[t] for t in range(ntyp))
    sewd = sums[ntyp]
    falp2 = 4.0 * sysm.alp_ewd ** 2
    ewf = np.zeros_like(g2)
    ewf[nz0] = 4.0 * math.pi * np.exp(-g2[nz0] / falp2) / (g2[nz0] * vol)
    ewald = float(np.sum(ewf * np.abs(sewd) ** 2 * w)) / 2.0
    vks = np.where(nz0, vks + np.conj(vext), 0.0)
    eext = float(np.sum(np.where(nz0, (rho * vext).real * w, 0.0)))
    fatm = None
    if want_forces:
        arg = np.outer(gx, sysm.pos[:, 0]) + np.outer(gy, sysm.pos[:, 1]) + np.outer(gz, sysm.pos[:, 2])
        h = np.exp(1j * arg)                                  # [ng, natm]
        vtemp = vtyp[:, sysm.atm_type]                        # [ng, natm]
        rr = (rho.real * w)[:, None] * vtemp + ((sewd.real * ewf * w)[:, None] * sysm.q[None, :])
        ri = (-rho.imag * w)[:, None] * vtemp + ((sewd.imag * ewf * w)[:, None] * sysm.q[None, :])
        comp = rr * h.imag - ri * h.real
        fatm = np.stack([(gx[:, None] * comp).sum(0), (gy[:, None] * comp).sum(0), (gz[:, None] * comp).sum(0)], axis=1)
    # g = 0 term (cp_hart_ext.C:366-395)
    iz = np.nonzero(~nz0)[0]
    if iz.size:
        v0 = float(np.sum(sysm.gzvps[sysm.atm_type])) / vol
        vks[iz[0]] = v0
        eext += v0 * rho[iz[0]].real
    # V(r) = sum_{full sphere} vks(g) exp(+i g.r): c2r of the kx >= 0 half
    # (the whole kx = 0 plane is in the density sphere)
    half = np.zeros((nz, ny, nx // 2 + 1), dtype=np.complex128)
    half[kz % nz, ky % ny, kx] = vks
    vr = _irfftn(half, s=(nz, ny, nx), axes=(0, 1, 2)) * n
    out = (vr, ehart, eext, ewald)
    return out + (fatm,) if want_forces else out


BECKE_BETA = 0.0042
LYP_A, LYP_B, LYP_C, LYP_D = 0.049180, 0.1320, 0.25330, 0.3490


def becke88(rho, g):
    """Becke 88 gradient correction to the LDA exchange (``becke_gcx_lda``,
    ``cp_becke.C:21-88``), spin-unpolarised: per spin rho_s = rho / 2,
    x = |grad rho_s| / rho_s^(4/3), b(x) = x^2 / (1 + 6 beta x asinh x),
    f = -2 beta rho_s^(4/3) b(x).  g = |grad rho|.  Returns
    (f, df/drho, df/dg)."""
    beta = BECKE_BETA
    rs = 0.5 * rho
    r13 = np.cbrt(rs)
    r43 = rs * r13
    x = 0.5 * g / r43
    root = np.sqrt(1.0 + x * x)
    ash = np.log(x + root)
    den = 1.0 + 6.0 * beta * x * ash
    b = x * x / den
    q = x / den
    bp = 2.0 * q - 6.0 * beta * q * q * (ash + x / root)       # db/dx
    return -2.0 * beta * r43 * b, -beta * (4.0 / 3.0) * r13 * (b - x * bp), -beta * bp


def lyp(rho, g):
    """Lee-Yang-Parr correlation, closed shell, with its local part
    (``lyp_gcc``, ``cp_becke.C:91-172``): with u = rho^(-1/3), D = 1 + d u,
    omega = exp(-c u) u^11 / D, delta = c u + d u / D and
    A = C_F rho^(8/3) + (5/12 - 7 delta / 72) g^2 - 11 g^2 / 24,
    f = -a rho / D - a b omega A rho^2.  Returns (f, df/drho, df/dg)."""
    a, b, c, d = LYP_A, LYP_B, LYP_C, LYP_D
    cf = 0.3 * (3.0 * math.pi * math.pi) ** (2.0 / 3.0)
    u = 1.0 / np.cbrt(rho)
    den = 1.0 + d * u
    om = np.exp(-c * u) * u ** 11 / den
    dl = c * u + d * u / den
    g2 = g * g
    A = cf * rho ** (8.0 / 3.0) + (5.0 / 12.0 - 7.0 * dl / 72.0) * g2 - 11.0 * g2 / 24.0
    f = -a * rho / den - a * b * om * A * rho * rho
    # derivatives in rho: du/drho = -u / (3 rho)
    dom = om * (c * u + d * u / den - 11.0) / (3.0 * rho)
    ddl = -(u / (3.0 * rho)) * (c + d / (den * den))
    dA = (8.0 / 3.0) * cf * rho ** (5.0 / 3.0) - (7.0 / 72.0) * ddl * g2
    dfr = -a * (1.0 + (4.0 / 3.0) * d * u) / (den * den) - a * b * (dom * A * rho * rho + om * (dA * rho * rho + 2.0 * A * rho))
    dfg = -a * b * om * rho * rho * 2.0 * g * (5.0 / 12.0 - 7.0 * dl / 72.0 - 11.0 / 24.0)
    return f, dfr, dfg


def gga_point(rho, grad, gga_cut, becke=True, lyp_on=True):
    """The per-point part of ``CPXCFNCTS::CP_getGGAFunctional``
    (``cp_grad_rho_ctrl.C:32-190``) on points with rho > rho_cut = gga_cut / 10:
    Becke and LYP times the switching function s(rho) = r^2 (3 - 2 r),
    r = clamp((rho - rho_cut) / (3.9 gga_cut), 0, 1).  grad: [3, ...].
    Returns (fx, fc, v = d(fx + fc)/drho, h = d(fx + fc)/d|grad rho| grad rho / |grad rho|),
    all zero where rho <= rho_cut."""
    rho_cut = 0.1 * gga_cut
    heal = 1.0 / (3.9 * gga_cut)
    on = rho > rho_cut
    r = np.where(on, rho, 1.0)
    g2 = grad[0] ** 2 + grad[1] ** 2 + grad[2] ** 2
    g = np.sqrt(g2)
    t = np.clip((r - rho_cut) * heal, 0.0, 1.0)
    sw = t * t * (3.0 - 2.0 * t)
    dsw = 6.0 * t * (1.0 - t) * heal
    zero = np.zeros_like(r)
    fx, dxr, dxg = becke88(r, g) if becke else (zero, zero, zero)
    fc, dcr, dcg = lyp(r, g) if lyp_on else (zero, zero, zero)
    v = (dxr + dcr) * sw + (fx + fc) * dsw
    dg = (dxg + dcg) * sw
    with np.errstate(divide="ignore", invalid="ignore"):
        unit = np.where(g2 > 0.0, 1.0 / g, 0.0)
    h = grad * (dg * unit)[None]
    fx, fc, v = fx * sw, fc * sw, v
    return (np.where(on, fx, 0.0), np.where(on, fc, 0.0), np.where(on, v, 0.0),
            np.where(on[None], h, 0.0))


def _sphere_to_r(vals, kx, ky, kz, sysm):
    """sum over the full density sphere of vals(g) exp(+i g.r) from the
    kx >= 0 half (the whole kx = 0 plane in it): a c2r transform."""
    nx, ny, nz = sysm.nfft
    half = np.zeros((nz, ny, nx // 2 + 1), dtype=np.complex128)
    half[kz % nz, ky % ny, kx] = vals
    return _irfftn(half, s=(nz, ny, nx), axes=(0, 1, 2)) * (nx * ny * nz)


def density_gradient(rho_r, sysm):
    """grad rho(r) = sum_sphere i g rho(g) / V exp(i g.r) with
    rho(g) = FFT_-[rho(r) V/N] (``divRhoVksGspace``, ``CP_Rho_GSpacePlane.C:278-320``,
    and its backward transforms scaled by 1/V).  Returns [3, nz, ny, nx]."""
    nx, ny, nz = sysm.nfft
    n = nx * ny * nz
    kx, ky, kz, g2 = rho_sphere(sysm)
    rhog = _rfftn(rho_r * (sysm.vol / n))[kz % nz, ky % ny, kx]
    f = TWO_PI / sysm.box
    return np.stack([_sphere_to_r(1j * (f * k) * rhog / sysm.vol, kx, ky, kz, sysm) for k in (kx, ky, kz)])


def gga_blyp(rho_r, sysm):
    """BLYP gradient correction (``CP_Rho_GSpacePlane::divRhoVksGspace``
    ``CP_Rho_GSpacePlane.C:278-320``, ``CP_Rho_RealSpacePlane::acceptGradRhoVks``
    ``CP_Rho_RealSpacePlane.C:1061-1215`` -> ``CP_getGGAFunctional``,
    ``whiteByrdFFT`` 1237-1300, ``CP_Rho_GSpacePlane::acceptWhiteByrd``
    330-380, ``CP_Rho_RealSpacePlane::acceptWhiteByrd`` 1314-1350):
    grad rho(r) from i g rho(g) on the density sphere, the per-point
    functional, h(g) = FFT(h(r)) / N and the white-byrd correction
    V -= sum_sphere (i g . h(g)) exp(i g.r).  Returns (V_gga(r), EGGA)."""
    nx, ny, nz = sysm.nfft
    n = nx * ny * nz
    vol = sysm.vol
    kx, ky, kz, g2 = rho_sphere(sysm)
    f = TWO_PI / sysm.box
    gv = (f * kx, f * ky, f * kz)
    grad = density_gradient(rho_r, sysm)
    fx, fc, v, h = gga_point(rho_r, grad, sysm.gga_cut)
    egga = float(np.sum(fx) + np.sum(fc)) * vol / n
    hg = [_rfftn(h[a] / n)[kz % nz, ky % ny, kx] for a in range(3)]
    div = 1j * (gv[0] * hg[0] + gv[1] * hg[1] + gv[2] * hg[2])
    return v - _sphere_to_r(div, kx, ky, kz, sysm), egga


def vks_build(psir, sysm):
    """Density -> V_KS(r) = V_xc + V_H + V_loc with the energy terms
    (``CP_Rho_RealSpacePlane::energyComputation`` 739-800, ``HartExtVksG``
    ``CP_Rho_GHartExt.C:461-510``, ``acceptHartVks`` 1365-1390), and the BLYP
    gradient correction when the system asks for it (EGGA)."""
    rho = density(psir, sysm)
    blyp = getattr(sysm, "xc", "pz_lda") == "blyp"
    vxc, exc, muxc = pz_lda(rho, sysm.vol, sysm.npts, lyp=blyp)
    vh, ehart, eext, ewald = hart_eext(rho, sysm)
    en = dict(EEXC=exc, MUXC=muxc, EHART=ehart, EEXT=eext, EWALD_RECIP=ewald, EGGA=0.0)
    if blyp:
        vg, en["EGGA"] = gga_blyp(rho, sysm)
        vxc = vxc + vg
    return rho, vxc + vh, en


# ----------------------------------------------------------------------------
# forces, EKE
# ----------------------------------------------------------------------------

def vks_forces(psir, vks, sysm):
    """psi(r) *= V_KS(r) occ w_k (``CP_State_RealSpacePlane::unpackVks`` 580-596),
    back-transform, F = -2/N * result (``CP_State_GSpacePlane::doIFFT``
    1581-1612)."""
    prod = psir * (vks[None] * sysm.occ[:, None, None, None])
    g = state_r_to_g(prod, sysm)
    return g * (-2.0 / sysm.npts)


def add_forces(fks, fnl, sysm):
    """``GStateSlab::addForces`` (``fft_slab_ctrl/stateSlab.C:239-268``):
    kx > 0 FFT forces are doubled before the nonlocal forces are added."""
    f = np.where(sysm.kx == 0, 1.0, 2.0) * fks
    return f + fnl if fnl is not None else f


def eke(psi, forces, sysm, kpt_weight=1.0):
    """``CPNONLOCAL::CP_eke_calc`` (``abinito_physics/cp_nonlocal/cp_eke.C:30-140``).
    Returns (new forces, per-state EKE)."""
    g2 = sysm.g2()
    ecut = sysm.ecut_ry
    w = np.where(sysm.kx == 0, 1.0, 2.0)
    wt = (sysm.occ * kpt_weight)[:, None] * w[None, :]
    inside = g2 <= ecut
    f = np.where(inside[None, :], forces - psi * (wt * g2[None, :]), 0.0)
    e = np.sum(np.where(inside[None, :], wt * g2[None, :] * np.abs(psi) ** 2, 0.0), axis=1) / 2.0
    return f, e


# ----------------------------------------------------------------------------
# nonlocal pseudopotential, structure-factor (N^2) method, l = 0 KB
# ----------------------------------------------------------------------------

def struct_fact(sysm):
    """``CPNONLOCAL::CP_calc_Struct_Fact`` (``cp_nonlocal/cp_struct_fact.C:37-255``)
    for l = 0: SF[a][g] = w_g p_t(|g|) y00 conj(exp(i g.R_a)), w_g = 1 on
    kx = 0 and 2 elsewhere, y00 = 1/sqrt(4 pi), p_t(0) = gzvps0
    (``get_rad_proj`` 260-285); the conjugation is the doublePack im flip
    at the end of the routine.  Returns ([natm_nl, ng] complex, atom list)."""
    nl = sysm.nl_atoms()
    f = TWO_PI / sysm.box
    gx, gy, gz = f * sysm.kx, f * sysm.ky, f * sysm.kz
    g = np.sqrt(gx * gx + gy * gy + gz * gz)
    w = np.where(sysm.kx == 0, 1.0, 2.0)
    y00 = 1.0 / math.sqrt(4.0 * math.pi)
    out = np.zeros((len(nl), sysm.ng), dtype=np.complex128)
    for ia, a in enumerate(nl):
        t = int(sysm.atm_type[a])
        p = sysm.nl_proj.eval(np.full(g.shape, t), np.where(g == 0, 1.0, g))
        p = np.where(g == 0, sysm.nl_gz0[t], p)
        x, y, z = sysm.pos[a]
        arg = x * gx + y * gy + z * gz
        out[ia] = np.conj(np.exp(1j * arg)) * (w * p * y00)
    return out, nl


def nl_energy_forces(psi, sysm, sf=None):
    """Z matrix, ENL and the nonlocal coefficient forces of the N^2 method:
    ``CPNONLOCAL::CP_enl_matrix_calc`` (``cp_nlmat.C:24-100``, DGEMV over the
    2 ng real view), ``CP_enl_atm_forc_calc`` (``cp_nl_energy_forc.C:178-235``,
    ENL = occ sum_a Z^2 vnorm / V, Z <- 2 vnorm / V Z) and
    ``CP_enl_force_calc`` (``cp_nl_energy_forc.C:29-110``, F -= sum_a Z SF_a).
    Returns (F_nl [nstate, ng] complex, per-state ENL, Z)."""
    if sf is None:
        sf, nl = struct_fact(sysm)
    else:
        nl = sysm.nl_atoms()
    vn = sysm.nl_vnorm[sysm.atm_type[nl]] / sysm.vol
    Z = real_view(psi) @ real_view(sf).T                 # [nstate, natm_nl]
    enl = sysm.occ * np.sum(Z * Z * vn[None, :], axis=1)
    Zp = 2.0 * vn[None, :] * Z
    f = -(Zp @ sf)
    return f, enl, Z


# ----------------------------------------------------------------------------
# nonlocal pseudopotential, EES (Euler exponential spline) method, l = 0
# ----------------------------------------------------------------------------

def _smooth235(n):
    while True:
        m = n
        for p in (2, 3, 5):
            while m % p == 0:
                m //= p
        if m == 1:
            return n
        n += 1


def ees_grid(sysm, scale=1.2, order=6):
    """Nonlocal EES grid (``init_nonlocal_ees``, ``interface/cp_ewald/set_cp_ewald.C:1329-1410``):
    n = int(2 scale (kmax+1)), at least 2 (kmax+1), rounded up to an FFT size
    (here: the next 2^a 3^b 5^c)."""
    kmax = [int(np.max(np.abs(k))) for k in (sysm.kx, sysm.ky, sysm.kz)]
    out = []
    for km in kmax:
        nk = km + 1
        n = int(2.0 * scale * nk)
        if n < 2 * nk:
            n += 1
        out.append(_smooth235(n))
    if min(out) < order:
        raise ValueError("EES grid smaller than the interpolation order")
    return tuple(out)


def bspline_weight_1d(order, ngrid):
    """``get_bspline_wght1d`` (``set_cp_ewald.C:1237-1325``): the complex
    Euler-exponential-spline factor 1/b(m) for m = 0..ngrid-1."""
    mn = np.zeros(order + 1)
    uk = np.zeros(order + 1)
    mn[1] = 1.0
    uk[1] = 1.0
    for k in range(2, order + 1):
        uk[k] = float(k)
    for n in range(3, order + 1):
        for k in range(n, 1, -1):
            mn[k] = (uk[k] * mn[k] + (n - uk[k]) * mn[k - 1]) / (n - 1)
        mn[1] = uk[1] * mn[1] / (n - 1)
    m = np.arange(ngrid)
    k = np.arange(1, order)
    arg = (2.0 * math.pi / ngrid) * np.outer(m, k - 1)
    den = (np.cos(arg) * mn[k]).sum(1) + 1j * (np.sin(arg) * mn[k]).sum(1)
    num = np.exp(1j * (2.0 * math.pi * (order - 1) / ngrid) * m)
    return num / den


def ees_dfactor(sysm, grid, order):
    """``eesSetEesWghtGgrp`` (``cp_ees_nonlocal.C:60-160``): d(g) = b_a(kx) b_b(ky) b_c(kz),
    negative k at index k + n; g = 0 keeps the real part."""
    na, nb, nc = grid
    ba, bb, bc = (bspline_weight_1d(order, n) for n in grid)
    d = ba[sysm.kx % na] * bb[sysm.ky % nb] * bc[sysm.kz % nc]
    g0 = (sysm.kx == 0) & (sysm.ky == 0) & (sysm.kz == 0)
    d[g0] = (ba[0] * bb[0] * bc[0]).real
    return d


def ees_bsplines(sysm, grid, order):
    """``eesAtmBsplineRgrp`` (``cp_ees_nonlocal.C:256-593``): for each nonlocal
    atom the order^3 grid points (ia, ib, ic) and weights M_a M_b M_c of its
    cardinal B-spline, and the derivative weights dM = M_{n-1}(u) - M_{n-1}(u - 1)
    taken from the recursion at n = order - 1 (``:436-449``).  Returns
    (idx [natm_nl, 3, order] int, mn [natm_nl, 3, order], dmn [natm_nl, 3, order])."""
    return atom_bsplines(sysm.pos[sysm.nl_atoms()], sysm.box, grid, order)


def atom_bsplines(pos, box, grid, order):
    """Per atom and axis the B-spline stencil of ``eesAtmBsplineRgrp``
    (nonlocal: ``cp_ees_nonlocal.C:256-593``; local: ``cp_hart_ext.C:641-860``,
    the same recursion): grid indices, M_n and dM_n, [natm, 3, order] each."""
    natm = pos.shape[0]
    idx = np.zeros((natm, 3, order), dtype=np.int64)
    mn = np.zeros((natm, 3, order))
    dmn = np.zeros((natm, 3, order))
    for ia_ in range(natm):
        for ax in range(3):
            ng = grid[ax]
            t = pos[ia_, ax] / box
            t -= round(t - 0.5)
            if t == 1.0:
                t = 0.0
            t *= ng
            it = int(t)
            frac = t - it
            u = frac + np.arange(order, dtype=np.float64)          # ua[j], j = 1..order
            m = np.zeros(order + 1)
            m[1] = 1.0 - abs(u[0] - 1.0)
            m[2] = 1.0 - abs(u[1] - 1.0)
            for n in range(3, order + 1):
                for j in range(n, 1, -1):
                    m[j] = (u[j - 1] * m[j] + (n - u[j - 1]) * m[j - 1]) / (n - 1)
                m[1] = u[0] * m[1] / (n - 1)
                if n == order - 1:
                    dmn[ia_, ax, 0] = m[1]
                    dmn[ia_, ax, 1:] = m[2:order + 1] - m[1:order]
            for j in range(1, order + 1):
                g = it - (j - 2)
                g = g if g > 0 else ng + g
                g = g if g <= ng else g - ng
                idx[ia_, ax, j - 1] = g - 1
                mn[ia_, ax, j - 1] = m[j]
    return idx, mn, dmn


def ees_setup(sysm, scale=1.2, order=6):
    grid = ees_grid(sysm, scale, order)
    return dict(grid=grid, order=order, d=ees_dfactor(sysm, grid, order),
                bspl=ees_bsplines(sysm, grid, order))


def _nl_grid_g_to_r(coef, sysm, grid):
    """State-convention transform on the nonlocal grid: sum over the full
    sphere of coef(g) exp(-i g.r) (``doNlFFTGtoR_Gchare``/``_Rchare``,
    ``fftCache.C:562-700``, same plans and signs as the state transforms)."""
    full = _full_grid(coef, sysm.kx, sysm.ky, sysm.kz, grid)
    return _fftn(full, axes=(-3, -2, -1)).real


def _nl_grid_r_to_g(fr, sysm, grid):
    na, nb, nc = grid
    full = _ifftn(fr, axes=(-3, -2, -1)) * (na * nb * nc)
    return full[..., sysm.kz % nc, sysm.ky % nb, sysm.kx % na]


def ees_dyp(sysm, ees):
    """``eesProjGchare`` + ``eesYlmOnD`` (``cp_ees_nonlocal.C:594-735``), l = 0:
    dyp(g) = d(g) y00 p(|g|) with y00 = 1/sqrt(4 pi), the projector spline p of
    the nonlocal atom type and its g = 0 value (``gzvps0``) at g = 0, where
    dyp is real."""
    d = ees["d"]
    nl = sysm.nl_atoms()
    f = TWO_PI / sysm.box
    g = f * np.sqrt(sysm.kx.astype(np.float64) ** 2 + sysm.ky ** 2 + sysm.kz ** 2)
    y00 = 1.0 / math.sqrt(4.0 * math.pi)
    t = int(sysm.atm_type[nl[0]]) if len(nl) else 0
    p = sysm.nl_proj.eval(np.full(g.shape, t), np.where(g == 0, 1.0, g))
    p = np.where(g == 0, sysm.nl_gz0[t], p)
    dyp = d * y00 * p
    return np.where(g == 0, dyp.real, dyp)


def nl_ees_energy_forces(psi, sysm, ees, atom_forces=False):
    """EES nonlocal energy and coefficient forces, l = 0 channel:
    ``eesProjGchare`` (``cp_ees_nonlocal.C:594-727``: dyp = d y00 p(|g|),
    projPsiG = conj(dyp psi)), the nonlocal-grid FFT, ``eesZmatRchare``
    (1238-1352: zmat = sum projPsiR M over the B-spline stencil),
    ``eesEnergyAtmForcRchare`` (1480-1720: ENL = occ vnorm/V sum zmat^2,
    zmat <- 2 vnorm/V occ zmat, scatter zmat M onto the grid; atom force
    F -= zmat sum projPsiR dM, dM_x = dMa Mb Mc n_a / L and so on), the inverse
    nonlocal-grid FFT and ``eesPsiForcGspace`` (2000-2079:
    F -= w conj(dyp P), w = 1 on kx = 0, 2 elsewhere; at g = 0 the
    imaginary parts of P and dyp are dropped).  Returns (F_nl, per-state ENL,
    zmat), and the atom forces [natm, 3] as a fourth item when atom_forces."""
    grid, order = ees["grid"], ees["order"]
    idx, mn, dmn = ees["bspl"]
    na, nb, nc = grid
    nl = sysm.nl_atoms()
    t = int(sysm.atm_type[nl[0]]) if len(nl) else 0
    dyp = ees_dyp(sysm, ees)
    g0 = (sysm.kx == 0) & (sysm.ky == 0) & (sysm.kz == 0)
    vn = sysm.nl_vnorm[t] / sysm.vol
    proj = np.conj(dyp[None, :] * psi)
    pr = _nl_grid_g_to_r(proj, sysm, grid)                     # [nstate, nc, nb, na]
    # stencil gather: zmat[s, a] = sum_{ja, jb, jc} pr[s, ic, ib, ia] Ma Mb Mc
    nst = psi.shape[0]
    zmat = np.zeros((nst, len(nl)))
    scr = np.zeros_like(pr)
    w3 = []
    subs = []
    for a in range(len(nl)):
        ia, ib, ic = idx[a]
        ma, mb, mc = mn[a]
        W = np.einsum("i,j,k->kji", ma, mb, mc)                 # [jc, jb, ja]
        sub = pr[:, ic][:, :, ib][:, :, :, ia]                   # [s, jc, jb, ja]
        zmat[:, a] = np.einsum("skji,kji->s", sub, W)
        w3.append(W)
        subs.append(sub)
    enl = sysm.occ * vn * np.sum(zmat * zmat, axis=1)
    zs = zmat * (2.0 * vn) * sysm.occ[:, None]
    for a in range(len(nl)):
        ia, ib, ic = idx[a]
        contrib = zs[:, a][:, None, None, None] * w3[a][None]
        np.add.at(scr, (slice(None), ic[:, None, None], ib[None, :, None], ia[None, None, :]), contrib)
    P = _nl_grid_r_to_g(scr, sysm, grid)
    P = np.where(g0[None, :], P.real, P)
    w = np.where(sysm.kx == 0, 1.0, 2.0)
    fnl = -w[None, :] * np.conj(dyp[None, :] * P)
    if not atom_forces:
        return fnl, enl, zmat
    fatm = np.zeros((sysm.natm, 3))
    for a, atom in enumerate(nl):
        ma, mb, mc = mn[a]
        da, db, dc = dmn[a]
        dw = (np.einsum("i,j,k->kji", da, mb, mc) * (na / sysm.box),
              np.einsum("i,j,k->kji", ma, db, mc) * (nb / sysm.box),
              np.einsum("i,j,k->kji", ma, mb, dc) * (nc / sysm.box))
        for ax in range(3):
            fatm[atom, ax] -= np.sum(zs[:, a] * np.einsum("skji,kji->s", subs[a], dw[ax]))
    return fnl, enl, zmat, fatm


# ----------------------------------------------------------------------------
# local pseudopotential and reciprocal Ewald sum, EES method
# (\cp_eext_ees_opt{on}: CP_Rho_RHartExt / CP_Rho_GHartExt)
# ----------------------------------------------------------------------------

def eesl_grid(sysm, scale=1.2, order=6):
    """EES local-pseudopotential grid (``init_eext_ees``,
    ``interface/cp_ewald/set_cp_ewald.C:1419-1500``): per axis
    n = int(2 scale (2 kmax + 1)), one more if below 2 (2 kmax + 1), rounded
    up to an FFT size (here: the next 2^a 3^b 5^c); kmax of the state sphere."""
    out = []
    for k in (sysm.kx, sysm.ky, sysm.kz):
        nk = 2 * int(np.max(np.abs(k))) + 1
        n = int(2.0 * scale * nk)
        if n < 2 * nk:
            n += 1
        out.append(_smooth235(n))
    if min(out) < order:
        raise ValueError("EES grid smaller than the interpolation order")
    return tuple(out)


def eesl_pack(sysm, grid, order):
    """``eesAtmBsplineRgrp`` + ``eesPackGridRchare`` (``cp_hart_ext.C:641-990``):
    per atom type the real grid Q_t[c, b, a] = sum over the type's atoms of
    M_a M_b M_c on their order^3 stencils.  Returns (Q [ntype, nc, nb, na],
    (idx, mn, dmn) of atom_bsplines)."""
    na, nb, nc = grid
    bs = atom_bsplines(sysm.pos, sysm.box, grid, order)
    idx, mn, _ = bs
    ntyp = len(sysm.type_names)
    Q = np.zeros((ntyp, nc, nb, na))
    for a in range(sysm.natm):
        w = np.einsum("i,j,k->kji", mn[a, 0], mn[a, 1], mn[a, 2])      # [jc, jb, ja]
        np.add.at(Q[int(sysm.atm_type[a])], np.ix_(idx[a, 2], idx[a, 1], idx[a, 0]), w)
    return Q, bs


def eesl_sf(Q, kx, ky, kz):
    """sfAtmTypG: Qhat_t(g) = sum_k Q_t(k) exp(+2 pi i m.k / n) at the density
    g-points (the R -> G transform of ``CP_Rho_RHartExt.C:300-330``; with
    this sign b(g) Qhat(g) approximates the structure factor
    sum_a exp(+i g.R_a) of ``CP_hart_eext_calc``)."""
    nc, nb, na = Q.shape[1:]
    full = _ifftn(Q, axes=(1, 2, 3)) * (na * nb * nc)
    return full[:, kz % nc, ky % nb, kx % na]


def eesl_bfactor(kx, ky, kz, grid, order):
    """``CPLOCAL::eesSetEesWghtGgrp`` (``cp_hart_ext.C:521-635``):
    b(g) = b_a(kx) b_b(ky) b_c(kz); at g = 0 the real product."""
    na, nb, nc = grid
    ba, bb, bc = (bspline_weight_1d(order, n) for n in grid)
    b = ba[kx % na] * bb[ky % nb] * bc[kz % nc]
    g0 = (kx == 0) & (ky == 0) & (kz == 0)
    b[g0] = (ba[0] * bb[0] * bc[0]).real
    return b


def eesl_gspace(rho, kx, ky, kz, g2, qhat, b, sysm):
    """``eesHartEextGchare`` over the atom types then ``eesEwaldGchare``
    (``cp_hart_ext.C:1005-1330``) on the density g-points.  Returns
    (vks(g), ehart, eext, ewald, Y [ntype, npts], Ytot [npts]) with Y the
    per-type atom-force transforms v_t conj(rho b) (g = 0: v_t(0) rho b) and
    Ytot = prep sfAtmTotG = 4 pi e^{-g^2/4 alpha^2} / (g^2 V) |b|^2 sum_t q_t Qhat_t."""
    vol = sysm.vol
    ntyp = qhat.shape[0]
    w = np.where(kx == 0, 1.0, 2.0)
    g0 = g2 == 0.0
    ins = (g2 <= sysm.ecut_rho_g2) & ~g0
    hf = np.zeros_like(g2)
    hf[ins] = 4.0 * math.pi / (g2[ins] * vol)
    ehart = float(np.sum(hf * np.abs(rho) ** 2 * w)) / 2.0
    vks = rho * hf
    g = np.sqrt(g2)
    qt = np.array([float(sysm.q[sysm.atm_type == t][0]) if np.any(sysm.atm_type == t) else 0.0 for t in range(ntyp)])
    Y = np.zeros((ntyp, g.size), dtype=np.complex128)
    eext = 0.0
    for t in range(ntyp):
        vt = np.where(ins, sysm.vloc.eval(np.full(g.shape, t), np.where(ins, g, 1.0)), 0.0) / vol
        vext = b * qhat[t] * vt
        eext += float(np.sum(np.where(ins, (rho * vext).real * w, 0.0)))
        vks = vks + np.where(ins, np.conj(vext), 0.0)
        Y[t] = np.where(ins, vt * np.conj(rho * b), 0.0)
        if g0.any():
            i0 = int(np.nonzero(g0)[0][0])
            v0 = sysm.gzvps[t] / vol
            vx = v0 * qhat[t][i0].real * b[i0].real
            eext += rho[i0].real * vx
            vks[i0] = vks[i0].real + vx
            Y[t][i0] = v0 * rho[i0].real * b[i0].real
    sq = np.where(ins, np.tensordot(qt, qhat, axes=1), 0.0)
    falp2 = 4.0 * sysm.alp_ewd ** 2
    preg = np.zeros_like(g2)
    preg[ins] = 4.0 * math.pi * np.exp(-g2[ins] / falp2) / (g2[ins] * vol)
    bmag = np.abs(b) ** 2
    ewald = float(np.sum(bmag * np.abs(sq) ** 2 * preg * w)) / 2.0
    vks = np.where(ins | g0, vks, 0.0)
    return vks, ehart, eext, ewald, Y, sq * preg * bmag


def eesl_backtransform(Y, kx, ky, kz, grid):
    """The G -> R transform of the atom-force grids (``FFTEesFwd``,
    ``CP_Rho_GHartExt.C:1018-1060``): P(k) = sum over the full sphere of
    Y(g) exp(-2 pi i m.k / n), the kx > 0 half entering with its conjugate
    partner.  Y [..., npts] -> real [..., nc, nb, na]."""
    na, nb, nc = grid
    lead = Y.shape[:-1]
    full = np.zeros(lead + (nc, nb, na), dtype=np.complex128)
    full[..., kz % nc, ky % nb, kx % na] = Y
    h = kx > 0
    full[..., (-kz[h]) % nc, (-ky[h]) % nb, (-kx[h]) % na] = np.conj(Y[..., h])
    return _fftn(full, axes=(-3, -2, -1)).real


def eesl_forces(P, Ptot, sysm, bs, grid):
    """``eesAtmForceRchare`` (``cp_hart_ext.C:1357-1470``): for each atom
    f -= sum over its stencil of grad(M_a M_b M_c) P_type, then with the
    atom's charge the same with Ptot (the Ewald part)."""
    na, nb, nc = grid
    idx, mn, dmn = bs
    f = np.zeros((sysm.natm, 3))
    for a in range(sysm.natm):
        ma, mb, mc = mn[a]
        da, db, dc = dmn[a]
        sl = np.ix_(idx[a, 2], idx[a, 1], idx[a, 0])
        pt = P[int(sysm.atm_type[a])][sl]
        pq = Ptot[sl]
        for comp, dw in enumerate((np.einsum("i,j,k->kji", da, mb, mc) * (na / sysm.box),
                                   np.einsum("i,j,k->kji", ma, db, mc) * (nb / sysm.box),
                                   np.einsum("i,j,k->kji", ma, mb, dc) * (nc / sysm.box))):
            f[a, comp] -= float(np.sum(dw * pt)) + sysm.q[a] * float(np.sum(dw * pq))
    return f


def hart_eext_ees(rho_r, sysm, want_forces=False):
    """``CP_hart_eext_calc`` with the EES structure factors
    (cp_eext_ees_opt on; ``CP_Rho_RHartExt`` -> ``CP_Rho_GHartExt``):
    the per-type B-spline grids, their transform, b(g), the Hartree / local
    / reciprocal Ewald terms and V_KS(g), then the atom forces by the
    back-transformed grids.  sysm.eext_ees = (na, nb, nc, order).  Returns
    like hart_eext."""
    na, nb, nc, order = sysm.eext_ees
    grid = (na, nb, nc)
    nx, ny, nz = sysm.nfft
    n = nx * ny * nz
    rhog_half = _rfftn(rho_r * (sysm.vol / n))
    kx, ky, kz, g2 = rho_sphere(sysm)
    rho = rhog_half[kz % nz, ky % ny, kx]
    Q, bs = eesl_pack(sysm, grid, order)
    qhat = eesl_sf(Q, kx, ky, kz)
    b = eesl_bfactor(kx, ky, kz, grid, order)
    vks, ehart, eext, ewald, Y, Ytot = eesl_gspace(rho, kx, ky, kz, g2, qhat, b, sysm)
    half = np.zeros((nz, ny, nx // 2 + 1), dtype=np.complex128)
    half[kz % nz, ky % ny, kx] = vks
    vr = _irfftn(half, s=(nz, ny, nx), axes=(0, 1, 2)) * n
    out = (vr, ehart, eext, ewald)
    if not want_forces:
        return out
    P = eesl_backtransform(Y, kx, ky, kz, grid)
    Ptot = eesl_backtransform(Ytot, kx, ky, kz, grid)
    return out + (eesl_forces(P, Ptot, sysm, bs, grid),)


def nl_sf_atom_forces(psi, sysm, sf=None):
    """Nonlocal atom forces of the N^2 method (``CP_enl_atm_forc_calc``,
    ``cp_nl_energy_forc.C:178-235``, doublePack branch): with
    Z = real_view(psi) real_view(SF)^T and dSF/dR_a = -i g SF_a
    (``CP_calc_Struct_Fact``'s derivative structure factors,
    ``cp_struct_fact.C:37-255``), F_a -= sum_s (2 vnorm / V Z_sa) dZ_sa/dR_a.
    As in the reference, the occupation scales the energy, not this force
    (the seeded systems have occupation 1).  Returns [natm, 3]."""
    if sf is None:
        sf, nl = struct_fact(sysm)
    else:
        nl = sysm.nl_atoms()
    vn = sysm.nl_vnorm[sysm.atm_type[nl]] / sysm.vol
    Z = real_view(psi) @ real_view(sf).T
    Zp = 2.0 * vn[None, :] * Z
    f = TWO_PI / sysm.box
    fatm = np.zeros((sysm.natm, 3))
    for ax, k in enumerate((sysm.kx, sysm.ky, sysm.kz)):
        dsf = np.ascontiguousarray(-1j * (f * k)[None, :] * sf)
        dZ = real_view(psi) @ real_view(dsf).T
        np.add.at(fatm[:, ax], nl, -np.sum(Zp * dZ, axis=0))
    return fatm


# ----------------------------------------------------------------------------
# ion side: real-space Ewald, atom integration
# ----------------------------------------------------------------------------

PROT_MASS = 1822.8885                         # piny_constants.h:55: amu -> electron masses
ATOM_MASS_AMU = {"O": 15.9994, "H": 1.00794}
# erfc(x) exp(-x^2)-form approximation of CPRSPACEION::CP_getionforce
# (cp_ions/cp_rspace_ion.C:36-45): erfc(x) = t P(t) exp(-x^2), t = 1/(1 + p x)
EWALD_P = 0.3614
EWALD_E = (0.2041422096422003, 0.1997535956961481, 0.2213176596405576, 0.03360430734640255,
           0.4732592578721755, -0.509078520069735, 0.6772631491947646, -0.369912979092217,
           0.06965131976970335)


def _erfc_poly(x):
    """(erfc(x), t^2 exp(-x^2) sum_k k e_k t^(k-1)) of the reference's approximation."""
    t = 1.0 / (1.0 + EWALD_P * x)
    eee = np.exp(-x * x)
    poly = 0.0
    dpoly = 0.0
    for k in range(len(EWALD_E), 0, -1):
        poly = poly * t + EWALD_E[k - 1]
        dpoly = dpoly * t + k * EWALD_E[k - 1]
    return poly * t * eee, dpoly * t * t * eee


def atom_masses(sysm):
    return np.array([ATOM_MASS_AMU[sysm.type_names[t]] * PROT_MASS for t in sysm.atm_type])


def ewald_rspace(sysm):
    """``CPRSPACEION::CP_getionforce`` (``cp_rspace_ion.C:25-251``), cubic
    periodic cell: pairs at the minimum image within half the box,
    q_i q_j erfc(alpha r) / r and its force; the self term
    -alpha sum q^2 / sqrt(pi) times erf(k_cut / 2 alpha) of the finite
    reciprocal sum (k_cut = the density-sphere radius) and the neutralising
    background -pi (sum q)^2 / (2 alpha^2 V).  Returns (E_real, E_self,
    E_bgr, F [natm, 3])."""
    pos, q, L, alp = sysm.pos, np.asarray(sysm.q, float), sysm.box, sysm.alp_ewd
    natm = pos.shape[0]
    F = np.zeros((natm, 3))
    e_real = 0.0
    palp = EWALD_P * alp
    talp2 = 2.0 * alp * alp
    for i in range(natm - 1):
        d = pos[i] - pos[i + 1:]
        d -= L * np.rint(d / L)
        r2 = np.sum(d * d, axis=1)
        r = np.sqrt(r2)
        m = r <= 0.5 * L
        qij = q[i] * q[i + 1:]
        ge, dg = _erfc_poly(r * alp)
        dge = dg * palp + talp2 * ge * r
        v = np.where(m, qij * ge / r, 0.0)
        dv = np.where(m, (ge / r2 + dge / r) * qij / r, 0.0)
        e_real += float(np.sum(v))
        fij = d * dv[:, None]
        F[i] += fij.sum(0)
        F[i + 1:] -= fij
    kcut = math.sqrt(sysm.ecut_rho_g2)
    self_erfc, _ = _erfc_poly(np.array(kcut / (2.0 * alp)))
    e_self = -(float(np.sum(q * q)) * alp) / math.sqrt(math.pi) * (1.0 - float(self_erfc))
    e_bgr = -(0.5 * float(np.sum(q)) ** 2 * math.pi) / (alp * alp * sysm.vol)
    return e_real, e_self, e_bgr, F


class IonState:
    """Atom velocities and masses of a CPMD run with moving ions."""

    def __init__(self, sysm, vel=None):
        self.m = atom_masses(sysm)
        self.v = np.zeros_like(sysm.pos) if vel is None else np.array(vel, dtype=np.float64)


def ion_forces(psi, sysm, rho_r, nl="sf", ees=None):
    """Forces on the ions at the current positions: local pseudopotential and
    reciprocal Ewald (``CP_hart_eext_calc``), the nonlocal part (structure
    factor or EES) and the real-space Ewald sum.  Returns (F [natm, 3],
    dict of the ion-side energies)."""
    _, _, _, _, f_loc = hart_eext(rho_r, sysm, want_forces=True)
    if nl == "ees":
        f_nl = nl_ees_energy_forces(psi, sysm, ees, atom_forces=True)[3]
    elif nl == "sf":
        f_nl = nl_sf_atom_forces(psi, sysm)
    else:
        f_nl = 0.0
    e_real, e_self, e_bgr, f_r = ewald_rspace(sysm)
    return f_loc + f_nl + f_r, {"EWALD_REAL": e_real, "EWALD_SELF": e_self, "EWALD_BGR": e_bgr}


def integrate_ions(ions, F, sysm, iteration, dt):
    """NVE atom integration (``ATOMINTEGRATE::integrate_nve_2nd_half`` /
    ``integrate_nve_1st_half``, ``classical_physics/integrate/integration_drivers.C:17-85``,
    in the order of ``ctrl_atom_integrate``, ``control_integrate.C:22-160``):
    the second half kick of the previous step (not on the first step), the
    kinetic energy, then the first half kick and the drift.  Moves
    sysm.pos in place; returns the ionic kinetic energy."""
    a = F / ions.m[:, None]
    if iteration > 1:
        ions.v += 0.5 * dt * a
    ke = 0.5 * float(np.sum(ions.m[:, None] * ions.v * ions.v))
    ions.v += 0.5 * dt * a
    sysm.pos += dt * ions.v
    return ke


# ----------------------------------------------------------------------------
# PairCalculator / Ortho
# ----------------------------------------------------------------------------

def real_view(a):
    """complex [nstate, ng] -> real [nstate, 2 ng] (re, im interleaved),
    the DGEMM view of ``ckPairCalculator.C:866-871``."""
    return a.view(np.float64).reshape(a.shape[0], -1)


def kx0_scale(a, sysm, s):
    out = a.copy()
    out[:, :sysm.nkx0] *= s
    return out


def pc_forward(left, right, sysm, alpha):
    """``PairCalculator::multiplyForward`` (``ckPairCalculator.C:821-893``):
    DGEMM('T','N') over the real view; C[x][y] = alpha * <left_x | right_y>."""
    return alpha * (real_view(left) @ real_view(right).T)


def newton_schulz(S, tol=1e-15, max_iter=1000, lsda=False):
    """``Ortho::start_calc``/``do_iteration``/``step_2``/``step_3``/
    ``tolerance_check``/``collect_error`` (``orthog_ctrl/ortho.C:109-146,
    233-262, 848-971``); same iteration as ``CPORTHOG::get_iter_Tmat``
    (``cp_orthog/cp_lowdin.C:180-265``):
    A = I, B = S/2; loop C = 3I - A B; B <- B C / 2; A <- C A / 2;
    err = sqrt(sum((A_old - A)^2) / N^2) until err <= tol.
    Returns (T, iterations, err)."""
    n = S.shape[0]
    B = S.copy() if lsda else S / 2.0
    A = np.eye(n)
    it = 0
    err = 1.0
    while True:
        C = 3.0 * np.eye(n) - A @ B
        Bn = 0.5 * (B @ C)
        An = 0.5 * (C @ A)
        err = math.sqrt(float(np.sum((A - An) ** 2)) / (n * n))
        A, B = An, Bn
        it += 1
        if not (err > tol and it < max_iter):
            break
    return A, it, err


def ortho_psi(psi_nonorth, sysm, tol=1e-15, max_iter=1000):
    """Orthonormalisation step (``computeNewPsi``, ``gspace.ci:710-730``):
    kx=0 rows scaled by 1/sqrt(2) (``CP_State_GSpacePlane::sendPsi``
    2975-3070), S = 2 Psi^T Psi (symmetric PC, alpha = 2), T by
    Newton-Schulz, Psi_new = Psi T (``bwMultiplyHelper``, 'N','N'), kx=0
    rows rescaled by sqrt(2) (``doNewPsi`` 3232-3281).  Returns
    (psi_orth, T, S, iters, err)."""
    r2i = 1.0 / math.sqrt(2.0)
    ps = kx0_scale(psi_nonorth, sysm, r2i)
    S = pc_forward(ps, ps, sysm, 2.0)
    T, it, err = newton_schulz(S, tol, max_iter)
    new = T.T @ ps
    new = kx0_scale(new, sysm, math.sqrt(2.0))
    return new, T, S, it, err


def lambda_step(psi, force, T, sysm):
    """Constraint force in dynamics (``computeLambdaAndCg``, ``gspace.ci:667-690``):
    kx=0: psi/sqrt2, F*sqrt2 (``sendLambda`` 1817-2007); Lambda[x][y] =
    <psi_x|F_y> (asymmetric PC, alpha = 1); Gamma = T Lambda
    (``ortho.C:565-570``); PC backward R = Psi Gamma^T - F T
    (``bwMultiplyHelper`` 1842 + ``bwMultiplyDynOrthoT`` 1965-2031);
    F = -R (``unpackLambda`` 2067-2072); kx=0 F/sqrt2 (``doLambda`` 2237-2242).
    Returns (F_new, Lambda)."""
    r2 = math.sqrt(2.0)
    ps = kx0_scale(psi, sysm, 1.0 / r2)
    fs = kx0_scale(force, sysm, r2)
    lam = pc_forward(ps, fs, sysm, 1.0)
    gam = T @ lam
    # Column-major (state = column) R = Psi Gamma - F T; as state rows:
    # R_j = sum_k Gamma[k][j] psi_k - sum_k T[k][j] F_k
    r = gam.T @ ps - T.T @ fs
    fnew = -r
    fnew = kx0_scale(fnew, sysm, 1.0 / r2)
    return fnew, lam


# ----------------------------------------------------------------------------
# integrator
# ----------------------------------------------------------------------------

def evolve_vel(force, vpsi, cmass, dt, sysm):
    """``CPINTEGRATE::cp_evolve_vel`` without NHC (``cp_dynamics.C:97-210``):
    on [nkx0_red, ng): g=0 imaginary parts zeroed, kx=0 unique points use
    F*2 / m*2, v += F dt/2 / m."""
    v = vpsi.copy()
    f = force.copy()
    r0 = sysm.nkx0_red
    r1 = r0 + sysm.nkx0_zero
    f[:, r0:r1] = f[:, r0:r1].real
    v[:, r0:r1] = v[:, r0:r1].real
    v[:, r0:] += f[:, r0:] * (0.5 * dt / cmass[None, r0:])
    v[:, r0:r1] = v[:, r0:r1].real
    return v


def fict_ke(vpsi, cmass, sysm):
    """``CPINTEGRATE::get_fictKE`` (``cp_dynamics.C:218-270``): sum m|v|^2 / 2
    over kx>0 plus the unique kx=0 points with mass doubled, g=0 real part."""
    r0 = sysm.nkx0_red
    r1 = r0 + sysm.nkx0_zero
    iend = sysm.nkx0_red + sysm.nkx0_uni
    m = cmass.copy()
    m[r1:iend] *= 2.0
    e = np.sum(m[None, r0:] * np.abs(vpsi[:, r0:]) ** 2, axis=1)
    return 0.5 * e


def integrate_dyn(force, vpsi, psi_t, sysm, iteration, dt):
    """``CPINTEGRATE::CP_integrate_dyn`` (``cp_dynamics.C:29-88``) with the
    coefficient thermostat off: complete the previous half kick
    (iteration > 1), the fictitious KE at time t, the next half kick, and
    the drift psi += v dt on [nkx0_red, ng).  Returns (v, psi_t, per-state
    fictitious KE); the inputs are not modified."""
    v = vpsi
    if iteration > 1:
        v = evolve_vel(force, v, sysm.cmass, dt, sysm)
    fict = fict_ke(v, sysm.cmass, sysm)
    v = evolve_vel(force, v, sysm.cmass, dt, sysm)
    r0 = sysm.nkx0_red
    p = psi_t.copy()
    p[:, r0:] = p[:, r0:] + v[:, r0:] * dt
    return v, p, fict


def sync_redundant(a, sysm):
    """Gamma redundancy sync (``gspace.ci:692-708``, ``CP_State_GSpacePlane.C:2829-2970``):
    the redundant kx=0 half is the conjugate of the unique half."""
    idx = redundant_partner(sysm)
    out = a.copy()
    out[:, :sysm.nkx0_red] = np.conj(a[:, idx])
    return out


def redundant_partner(sysm):
    k0 = np.arange(sysm.nkx0)
    key = {(int(sysm.ky[i]), int(sysm.kz[i])): i for i in k0}
    return np.array([key[(-int(sysm.ky[i]), -int(sysm.kz[i]))] for i in range(sysm.nkx0_red)], dtype=np.int64)


# ----------------------------------------------------------------------------
# one CP dynamics step (gspace.ci:199-324), electrons only, ions fixed
# ----------------------------------------------------------------------------

class CPState:
    """psi_t: non-orthogonal coefficients integrated by Verlet; psi: the
    orthonormal set psi_t T; T: last Newton-Schulz result; v: velocities."""

    def __init__(self, sysm):
        self.psi_t = sysm.psi.copy()
        self.psi = sysm.psi.copy()
        self.T = np.eye(sysm.nstate)
        self.v = np.zeros_like(sysm.psi)
        self.iteration = 0
        self.half_step = True    # False after a PsiV reset: v is at t, the next step completes no half kick


def electronic_forces(psi, sysm, fnl=None, enl=0.0):
    psir = state_g_to_r(psi, sysm)
    rho, vks, en = vks_build(psir, sysm)
    fks = vks_forces(psir, vks, sysm)
    f = add_forces(fks, fnl, sysm)
    f, ek = eke(psi, f, sysm)
    en = dict(en)
    en["EKE"] = float(ek.sum())
    en["ENL"] = enl
    return f, en


def psiv_reset(st, sysm, psi_prev, dt):
    """PsiV tolerance reset of the reference's default build
    (``Ortho::maxCheck``, ``ortho.C:455-475`` -> ``computeNewPsiVFiniteDifference``,
    ``gspace.ci:290-301``; ``CP_State_GSpacePlane::finiteDifferencePsiV``,
    ``CP_State_GSpacePlane.C:3741-3800``, ``norb_fin_diff_order`` 0): the
    non-orthogonal set is replaced by the orthonormal one (psi_t <- psi,
    T <- I) and the velocities by the first-order finite difference of the
    orthonormal states, v = (psi(t) - psi(t - dt)) / dt, taken as the
    velocity at t (``halfStepEvolve = 0``: the next integration does not
    complete a half kick)."""
    st.v = (st.psi - psi_prev) / dt
    st.psi_t = st.psi.copy()
    st.T = np.eye(sysm.nstate)
    st.half_step = False


def _nl_default(psi, sysm):
    f, enl, _ = nl_energy_forces(psi, sysm)
    return f, float(enl.sum())


def cp_step(st, sysm, tol=1e-15, max_iter=1000, nl="auto", norb_tol=None, dt=None, ions=None, ees=None):
    """One CPAIMD electronic step.  Order: forces on the orthonormal psi
    (computePsiFandVKS + NL, combineForcesGetEke), constraint force
    (computeLambdaAndCg), integrate (integrateModForce ->
    CPINTEGRATE::CP_integrate_dyn, cp_dynamics.C:29-88), orthonormalise
    (computeNewPsi).  With ions (an IonState) the atoms move too: their
    forces at the positions of this step (ion_forces) and the NVE atom
    integration (integrate_ions, AtomsCompute::integrateAtoms,
    drv/main/AtomsCompute.C:461-640), after which the next step's structure
    factors see the new positions.  ees: the EES nonlocal setup (ees_setup)
    that nl evaluates with; with ions its B-splines follow the atoms and the
    nonlocal atom forces come from it.  Returns the energy record of the psi
    the forces were evaluated on."""
    st.iteration += 1
    dt_now = sysm.dt if dt is None else dt
    psi_prev = st.psi.copy()       # the orthonormal psi(t) (sendLambda keeps it, CP_State_GSpacePlane.C:1838-1858)
    if ees is not None and ions is not None:
        ees["bspl"] = ees_bsplines(sysm, ees["grid"], ees["order"])
    if nl == "auto":
        nl = _nl_default if len(sysm.nl_atoms()) else None
    fnl, enl = (None, 0.0) if nl is None else nl(st.psi, sysm)
    if ions is not None:
        rho_r = density(state_g_to_r(st.psi, sysm), sysm)
        nl_ion = None if nl is None else ("ees" if ees is not None else "sf")
        fion, eion = ion_forces(st.psi, sysm, rho_r, nl=nl_ion, ees=ees)
    f, en = electronic_forces(st.psi, sysm, fnl, enl)
    if ions is not None:
        en.update(eion)
        en["ION_KE"] = integrate_ions(ions, fion, sysm, st.iteration, sysm.dt if dt is None else dt)
    f, lam = lambda_step(st.psi, f, st.T, sysm)
    # after a PsiV reset the velocity is already at t (halfStepEvolve = 0)
    it_int = st.iteration if getattr(st, "half_step", True) else 1
    st.v, st.psi_t, fict = integrate_dyn(f, st.v, st.psi_t, sysm, it_int, dt_now)
    st.half_step = True
    en["FICT_KE"] = float(fict.sum())
    st.psi_t = sync_redundant(st.psi_t, sysm)
    st.v = sync_redundant(st.v, sysm)
    st.psi, st.T, S, it, err = ortho_psi(st.psi_t, sysm, tol, max_iter)
    en["ORTHO_ITERS"] = it
    en["ORTHO_ERR"] = err
    en["SMAX"] = float(np.max(np.abs(S - 2.0 * np.eye(sysm.nstate))))
    if norb_tol is not None and en["SMAX"] > norb_tol:
        psiv_reset(st, sysm, psi_prev, dt_now)
    return en


def quench(st, sysm, nsteps, tol=1e-15, max_iter=1000, dt=None):
    """Damped CP from a random start: each step is ``cp_step`` with the
    velocities zeroed after the integration and the non-orthogonal set reset
    to the orthonormal one (psi_t <- psi, T <- I, v = 0), the iteration count
    restarting every step -- steepest descent on the orthonormal states with
    step dt^2 / (2 m) (dt: the system's time step unless given).  The same
    procedure as ``CPDriver.quench`` on the GPU; it brings the start near the
    Born-Oppenheimer surface before CPMD.  Returns the energy record of every
    step."""
    out = []
    for _ in range(nsteps):
        st.iteration = 0
        st.v = np.zeros_like(st.v)
        en = cp_step(st, sysm, tol, max_iter, dt=dt)
        st.v = np.zeros_like(st.v)
        st.psi_t = st.psi.copy()
        st.T = np.eye(sysm.nstate)
        st.half_step = True
        out.append(en)
    st.iteration = 0
    return out


# ----------------------------------------------------------------------------
# minimisation (cp_min_opt), fixed ions
# ----------------------------------------------------------------------------

def fovlap(force):
    """``CPINTEGRATE::CP_fovlap_calc`` (``cp_integrate/cp_min_CG.C:128-140``):
    sum |F|^2 over every stored point of every state."""
    return float(np.sum(force.real ** 2 + force.imag ** 2))


def min_step(psi, force, sysm, dt, conj=None, gamma=0.0):
    """``CP_integrate_min_STD`` (``cp_min_std.C:17-60``): psi += F dt / m, or
    ``CP_integrate_min_CG`` (``cp_min_CG.C:29-120``): conj = conj gamma + F
    for g^2 <= ecut, psi += conj dt / m.  Returns (psi, conj)."""
    if conj is not None:
        inside = (sysm.g2() <= sysm.ecut_ry)[None, :]
        conj = np.where(inside, conj * gamma + force, conj)
        d = conj
    else:
        d = force
    return psi + d * (dt / sysm.cmass[None, :]), conj


def minimize(st, sysm, nsteps, method="cg", dt=None, tol=1e-15, max_iter=1000, nl="auto"):
    """Electronic minimisation at fixed ions, the loop of
    ``GSpaceDriver::computeMinimization`` (``gspace.ci:85-196``): forces on
    the orthonormal psi, F' = F - Psi Lambda (Lambda handed back unchanged by
    Ortho in minimisation, ``ortho.C:497-608``), |F'|^2, the steepest-descent
    or conjugate-gradient step with the resets of
    ``CP_State_GSpacePlane.C:2636-2660``, the Gamma redundancy sync and the
    orthonormalisation.  Returns one record per iteration (energies of the
    psi the forces were evaluated on, FMAG = |F'|)."""
    dt = sysm.dt if dt is None else dt
    if nl == "auto":
        nl = _nl_default if len(sysm.nl_atoms()) else None
    conj = np.zeros_like(st.psi) if method == "cg" else None
    out = []
    fov = fmag = 0.0
    nreset = 0
    for it in range(1, nsteps + 1):
        fnl, enl = (None, 0.0) if nl is None else nl(st.psi, sysm)
        f, en = electronic_forces(st.psi, sysm, fnl, enl)
        f, _ = lambda_step(st.psi, f, np.eye(sysm.nstate), sysm)
        fov_old, fmag_old = fov, fmag
        fov = fovlap(f)
        fmag = math.sqrt(fov)
        gamma = 0.0
        if method == "cg":
            reset = it == 1 or (fmag > 1.05 * fmag_old and nreset >= 5) or fmag > 2.0 * fmag_old
            if reset:
                nreset = 0
            else:
                gamma = fov / fov_old
            nreset += 1
        p, conj = min_step(st.psi, f, sysm, dt, conj, gamma)
        p = sync_redundant(p, sysm)
        st.psi, st.T, S, its, err = ortho_psi(p, sysm, tol, max_iter)
        st.psi_t = st.psi.copy()
        en["FMAG"] = fmag
        en["ORTHO_ITERS"] = its
        out.append(en)
    return out
