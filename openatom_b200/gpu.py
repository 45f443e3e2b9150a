"""ctypes binding of liboa_gpu and the host-side CP step driver.

``CPContext`` exposes one method per C-ABI entry point (include/oa_gpu.h);
``CPDriver`` sequences one Car-Parrinello dynamics step the way
``GSpaceDriver::computeDynamics`` does (src_charm_driver/cp_state_ctrl/gspace.ci:199-324):
forces on the orthonormal states (computePsiFandVKS + combineForcesGetEke),
the constraint force (computeLambdaAndCg), integration (integrateModForce)
and orthonormalisation (computeNewPsi).

Device memory and streams come from torch; there is no CPU fallback: every
method raises if the CUDA library or a GPU is missing.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboa_gpu.so")

OA_OK, OA_ERR_BAD_ARG, OA_ERR_CUDA, OA_ERR_NOT_CONVERGED, OA_ERR_NONFINITE, OA_ERR_UNSUPPORTED = range(6)
OA_FP64, OA_MIXED = 0, 1

_ip = C.POINTER(C.c_int)
_dp = C.POINTER(C.c_double)


class SystemDesc(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("nstate", C.c_int), ("ng", C.c_int), ("nlines", C.c_int),
        ("line_kx", _ip), ("line_ky", _ip), ("line_off", _ip), ("line_nneg", _ip), ("line_npos", _ip),
        ("kx", _ip), ("ky", _ip), ("kz", _ip),
        ("nkx0", C.c_int), ("nkx0_red", C.c_int), ("nkx0_uni", C.c_int), ("nkx0_zero", C.c_int),
        ("red_partner", _ip),
        ("box", C.c_double), ("ecut_psi", C.c_double), ("ecut_rho", C.c_double),
        ("occ", _dp), ("cmass", _dp),
        ("natm", C.c_int), ("ntype", C.c_int),
        ("pos", _dp), ("atm_type", _ip), ("q_type", _dp), ("gzvps", _dp),
        ("alp_ewd", C.c_double),
        ("nspl", C.c_int), ("spl_gmin", C.c_double), ("spl_dg", C.c_double), ("spl", _dp),
        ("natm_nl", C.c_int), ("nl_atm", _ip), ("nl_spl", _dp), ("nl_vnorm", _dp), ("nl_gz0", _dp),
    ]


STEP_KEYS = ("EKE", "EHART", "EEXT", "EWALD_RECIP", "EEXC", "MUXC", "FICT_KE", "ENL", "ORTHO_ITERS",
             "ORTHO_ERR", "SMAX", "EGGA", "ION_KE", "EWALD_REAL")
NREC = len(STEP_KEYS)
XC_FUNCTIONALS = {"pz_lda": 0, "blyp": 1}


class CPState(C.Structure):
    _fields_ = [
        ("psi_t", _dp), ("psi", _dp), ("vpsi", _dp), ("T", _dp),
        ("iteration", C.c_int), ("dt", C.c_double), ("ns_tol", C.c_double), ("norb_tol", C.c_double),
        ("ns_max_iter", C.c_int), ("mixed_nterm", C.c_int), ("use_graph", C.c_int),
        ("last_ns_iters", C.c_int), ("last_ns_err", C.c_double), ("last_smax", C.c_double),
        ("last_kernels", C.c_int), ("psiv_pending", C.c_int),
    ]


class Tuning(C.Structure):
    """oa_tuning: the runtime tile and schedule choices of a context."""
    _fields_ = [("group_state", C.c_int), ("group_pair", C.c_int), ("dgemm_kblocks", C.c_int),
                ("tgemm_kblocks", C.c_int), ("fft_path", C.c_int)]


TUNING_FIELDS = tuple(f for f, _ in Tuning._fields_)


# name -> (restype, argtypes); the exported surface of include/oa_gpu.h
_vp = C.c_void_p
SIGNATURES = {
    "oa_gpu_init": (C.c_int, [C.POINTER(SystemDesc), C.c_int, C.POINTER(_vp)]),
    "oa_gpu_destroy": (C.c_int, [_vp]),
    "oa_gpu_last_error": (C.c_char_p, []),
    "oa_gpu_scratch_bytes": (C.c_size_t, [_vp]),
    "oa_gpu_state_fft_fwd": (C.c_int, [_vp, _vp, _vp, _vp]),
    "oa_gpu_vks_build": (C.c_int, [_vp, _vp, _vp]),
    "oa_gpu_set_vks": (C.c_int, [_vp, _vp, _vp]),
    "oa_gpu_vks_apply_fft_bwd": (C.c_int, [_vp, _vp, _vp, C.c_int, _vp, _vp, _vp]),
    "oa_gpu_pc_forward": (C.c_int, [_vp, _vp, _vp, _vp, C.c_double, C.c_double, _vp]),
    "oa_gpu_pc_overlap_i8": (C.c_int, [_vp, _vp, _vp, C.c_double, C.c_double, _vp]),
    "oa_gpu_min_fovlap": (C.c_int, [_vp, _vp, _vp, _dp]),
    "oa_gpu_min_step": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_double, C.c_double]),
    "oa_gpu_pc_rotate_i8": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "oa_gpu_ortho_invsqrt": (C.c_int, [_vp, _vp, _vp, _vp, C.c_double, C.c_int, _ip, _dp, _dp]),
    "oa_gpu_pc_backward": (C.c_int, [_vp, _vp, _vp, _vp, C.c_double, C.c_double, _vp, _vp, C.c_double, _vp]),
    "oa_gpu_small_gemm": (C.c_int, [_vp, _vp, _vp, _vp, C.c_double, _vp]),
    "oa_gpu_integrate": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_double, C.c_int, _vp]),
    "oa_gpu_energies": (C.c_int, [_vp, _vp, _dp]),
    "oa_gpu_set_xc": (C.c_int, [_vp, C.c_int, C.c_double]),
    "oa_gpu_set_ions": (C.c_int, [_vp, _dp, _dp]),
    "oa_gpu_get_ions": (C.c_int, [_vp, _vp, _dp, _dp]),
    "oa_gpu_psiv_reset": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, C.c_double]),
    "oa_gpu_cp_run_batch": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_int, _vp, C.c_int,
                                      C.POINTER(C.c_double)]),
    "oa_gpu_set_atoms": (C.c_int, [_vp, _vp, _dp]),
    "oa_gpu_time_kernels": (C.c_int, [_vp, _vp, _vp, C.c_int, _dp]),
    "oa_gpu_sizes": (C.c_int, [_vp, C.POINTER(C.c_long)]),
    "oa_gpu_pc_forward_mixed": (C.c_int, [_vp, _vp, _vp, _vp, C.c_double, C.c_double, C.c_int, _vp]),
    "oa_gpu_pc_backward_mixed": (C.c_int, [_vp, _vp, _vp, _vp, C.c_double, C.c_double, _vp, _vp, C.c_double,
                                           C.c_int, _vp]),
    "oa_gpu_check": (C.c_int, [_vp, _vp]),
    "oa_gpu_fault_inject": (C.c_int, [_vp, C.c_int]),
    "oa_gpu_nl_sf": (C.c_int, [_vp, _vp, _vp, C.c_int, _vp, _vp]),
    "oa_gpu_cp_step": (C.c_int, [_vp, _vp, C.POINTER(CPState), _dp]),
    "oa_gpu_cp_run": (C.c_int, [_vp, _vp, C.POINTER(CPState), C.c_int, _dp, _dp]),
    "oa_gpu_ees_init": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int, _dp]),
    "oa_gpu_nl_ees": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "oa_gpu_set_ees_local": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int]),
    "oa_gpu_get_tuning": (C.c_int, [_vp, C.POINTER(Tuning)]),
    "oa_gpu_set_tuning": (C.c_int, [_vp, C.POINTER(Tuning)]),
    "oa_gpu_pc_forward_noalloc": (C.c_int, [_vp, _vp, _vp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                            _vp]),
}

KERNEL_NAMES = ("state_zfwd", "state_plane_density", "rho_xc", "vks_build", "state_plane_vks",
                "state_zbwd", "pc_forward_S", "pc_backward", "ortho_ns", "pc_rotate", "pc_forward_lambda",
                "pc_overlap_i8", "pc_rotate_i8")

_lib = None


class OaError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"liboa_gpu status {status}: {msg}")
        self.status = status


def load_library(path: str = LIB_PATH):
    """Load liboa_gpu.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise OSError(f"{path} not found: build it with `python -m openatom_b200.build`")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _check(st):
    if st != OA_OK:
        raise OaError(st, _lib.oa_gpu_last_error().decode())


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _iarr(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _darr(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def redundant_partner(sysm) -> np.ndarray:
    key = {(int(sysm.ky[i]), int(sysm.kz[i])): i for i in range(sysm.nkx0)}
    return np.array([key[(-int(sysm.ky[i]), -int(sysm.kz[i]))] for i in range(sysm.nkx0_red)], dtype=np.int32)


class CPContext:
    """One system on the current CUDA device (one ``oa_ctx``)."""

    def __init__(self, sysm, precision: str = "fp64", tuning: str = "table"):
        """tuning: "table" applies the autotuner's recorded choices for this
        system's sizes and precision when the table has them
        (openatom_b200/tuning/b200.json, openatom_b200.tuner); "default"
        keeps the library's built-in heuristics."""
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("CPContext needs a CUDA device; there is no CPU path")
        lib = load_library()
        self.sys = sysm
        self.precision = OA_FP64 if precision == "fp64" else OA_MIXED
        keep = dict(
            line_kx=_iarr(sysm.line_kx), line_ky=_iarr(sysm.line_ky), line_off=_iarr(sysm.line_off),
            line_nneg=_iarr(sysm.line_nneg), line_npos=_iarr(sysm.line_npos),
            kx=_iarr(sysm.kx), ky=_iarr(sysm.ky), kz=_iarr(sysm.kz), red=_iarr(redundant_partner(sysm)),
            occ=_darr(sysm.occ), cmass=_darr(sysm.cmass), pos=_darr(sysm.pos), atm_type=_iarr(sysm.atm_type),
            q_type=_darr([6.0, 1.0][: len(sysm.type_names)]), gzvps=_darr(sysm.gzvps),
            spl=_darr(sysm.vloc.coef))
        # per-type valence charge from the atoms
        qt = np.zeros(len(sysm.type_names))
        for t in range(len(sysm.type_names)):
            m = sysm.atm_type == t
            if m.any():
                qt[t] = sysm.q[m][0]
        keep["q_type"] = _darr(qt)
        nl = sysm.nl_atoms()
        keep["nl_atm"] = _iarr(nl)
        ntyp = len(sysm.type_names)
        keep["nl_spl"] = _darr(sysm.nl_proj.coef if sysm.nl_proj is not None else np.zeros((ntyp, sysm.vloc.n, 4)))
        keep["nl_vnorm"] = _darr(sysm.nl_vnorm if sysm.nl_vnorm is not None else np.zeros(ntyp))
        keep["nl_gz0"] = _darr(sysm.nl_gz0 if sysm.nl_gz0 is not None else np.zeros(ntyp))
        if sysm.nl_proj is not None and (sysm.nl_proj.n != sysm.vloc.n or sysm.nl_proj.dg != sysm.vloc.dg
                                         or sysm.nl_proj.gmin != sysm.vloc.gmin):
            raise ValueError("nonlocal and local spline tables must share one g grid")

        def ip(a):
            return a.ctypes.data_as(_ip)

        def dp(a):
            return a.ctypes.data_as(_dp)

        d = SystemDesc()
        d.nx, d.ny, d.nz = sysm.nfft
        d.nstate, d.ng, d.nlines = sysm.nstate, sysm.ng, sysm.nlines
        d.line_kx, d.line_ky, d.line_off = ip(keep["line_kx"]), ip(keep["line_ky"]), ip(keep["line_off"])
        d.line_nneg, d.line_npos = ip(keep["line_nneg"]), ip(keep["line_npos"])
        d.kx, d.ky, d.kz = ip(keep["kx"]), ip(keep["ky"]), ip(keep["kz"])
        d.nkx0, d.nkx0_red, d.nkx0_uni, d.nkx0_zero = sysm.nkx0, sysm.nkx0_red, sysm.nkx0_uni, sysm.nkx0_zero
        d.red_partner = ip(keep["red"])
        d.box, d.ecut_psi, d.ecut_rho = sysm.box, sysm.ecut_ry, sysm.ecut_rho_g2
        d.occ, d.cmass = dp(keep["occ"]), dp(keep["cmass"])
        d.natm, d.ntype = sysm.natm, len(sysm.type_names)
        d.pos, d.atm_type, d.q_type, d.gzvps = dp(keep["pos"]), ip(keep["atm_type"]), dp(keep["q_type"]), dp(keep["gzvps"])
        d.alp_ewd = sysm.alp_ewd
        d.nspl, d.spl_gmin, d.spl_dg, d.spl = sysm.vloc.n, sysm.vloc.gmin, sysm.vloc.dg, dp(keep["spl"])
        d.natm_nl, d.nl_atm = len(nl), ip(keep["nl_atm"])
        d.nl_spl, d.nl_vnorm, d.nl_gz0 = dp(keep["nl_spl"]), dp(keep["nl_vnorm"]), dp(keep["nl_gz0"])
        h = C.c_void_p()
        _check(lib.oa_gpu_init(C.byref(d), self.precision, C.byref(h)))
        self._h = h
        self._lib = lib
        xc = getattr(sysm, "xc", "pz_lda")
        if xc != "pz_lda":
            self.set_xc(xc, getattr(sysm, "gga_cut", 5.0e-5))
        if getattr(sysm, "eext_ees", None) is not None:
            na, nb, nc, order = sysm.eext_ees
            self.set_ees_local((na, nb, nc), order)
        self.tuning_source = "default"
        if tuning == "table":
            from .tuner import lookup
            choice = lookup(sysm, precision)
            if choice is not None:
                self.set_tuning(**choice)
                self.tuning_source = "table"
        elif tuning != "default":
            raise ValueError("tuning must be 'table' or 'default'")

    def set_ions(self, masses, vel=None):
        """Turn on ion dynamics in the native step (oa_gpu_set_ions): masses
        [natm] in electron masses, velocities [natm, 3] (None: zero)."""
        m = np.ascontiguousarray(masses, dtype=np.float64)
        if m.shape != (self.sys.natm,):
            raise ValueError("masses must have shape (natm,)")
        v = None
        if vel is not None:
            v = np.ascontiguousarray(vel, dtype=np.float64)
            if v.shape != (self.sys.natm, 3):
                raise ValueError("vel must have shape (natm, 3)")
        _check(self._lib.oa_gpu_set_ions(self._h, m.ctypes.data_as(_dp), None if v is None else v.ctypes.data_as(_dp)))

    def get_ions(self):
        """(positions, velocities) of the atoms, host arrays [natm, 3]."""
        pos = np.zeros((self.sys.natm, 3))
        vel = np.zeros((self.sys.natm, 3))
        _check(self._lib.oa_gpu_get_ions(self._h, self._stream(), pos.ctypes.data_as(_dp), vel.ctypes.data_as(_dp)))
        return pos, vel

    def get_tuning(self) -> dict:
        """The context's tile and schedule choices (oa_gpu_get_tuning)."""
        t = Tuning()
        _check(self._lib.oa_gpu_get_tuning(self._h, C.byref(t)))
        return {f: int(getattr(t, f)) for f in TUNING_FIELDS}

    def set_tuning(self, **choice):
        """Set some of the choices (oa_gpu_set_tuning); the others are kept."""
        bad = set(choice) - set(TUNING_FIELDS)
        if bad:
            raise ValueError(f"unknown tuning fields {sorted(bad)}")
        t = Tuning(**{f: int(choice.get(f, 0)) for f in TUNING_FIELDS})
        _check(self._lib.oa_gpu_set_tuning(self._h, C.byref(t)))

    def set_ees_local(self, grid, order: int = 6):
        """Local pseudopotential and reciprocal Ewald sum by the EES method
        (cp_eext_ees_opt on; oa_gpu_set_ees_local) on grid (na, nb, nc) with
        B-splines of this order; grid None: the structure-factor method."""
        na, nb, nc = (0, 0, 0) if grid is None else (int(g) for g in grid)
        _check(self._lib.oa_gpu_set_ees_local(self._h, na, nb, nc, int(order)))

    def set_xc(self, functional: str, gradient_cutoff: float = 5.0e-5):
        """Exchange-correlation of the density path: "pz_lda" or "blyp"
        (oa_gpu_set_xc)."""
        if functional not in XC_FUNCTIONALS:
            raise ValueError(f"functional must be one of {sorted(XC_FUNCTIONALS)}")
        _check(self._lib.oa_gpu_set_xc(self._h, XC_FUNCTIONALS[functional], float(gradient_cutoff)))

    def close(self):
        if getattr(self, "_h", None):
            self._lib.oa_gpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _stream():
        import torch
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def scratch_bytes(self) -> int:
        return int(self._lib.oa_gpu_scratch_bytes(self._h))

    # -- entry points -------------------------------------------------------
    def state_fft_fwd(self, psi, rho_out=None):
        _check(self._lib.oa_gpu_state_fft_fwd(self._h, self._stream(), _ptr(psi), _ptr(rho_out)))

    def vks_build(self, vks_out=None):
        _check(self._lib.oa_gpu_vks_build(self._h, self._stream(), _ptr(vks_out)))

    def set_vks(self, vks):
        _check(self._lib.oa_gpu_set_vks(self._h, self._stream(), _ptr(vks)))

    def vks_apply_fft_bwd(self, psi, force, fnl=None, recompute_fwd=False, eke_out=None):
        _check(self._lib.oa_gpu_vks_apply_fft_bwd(self._h, self._stream(), _ptr(psi), int(recompute_fwd),
                                                  _ptr(fnl), _ptr(force), _ptr(eke_out)))

    def pc_forward(self, left, right, alpha, w_kx0, out):
        _check(self._lib.oa_gpu_pc_forward(self._h, self._stream(), _ptr(left), _ptr(right),
                                           float(alpha), float(w_kx0), _ptr(out)))

    def pc_overlap_i8(self, psi_t, alpha, w_kx0, out):
        """S = alpha sum w psi_t psi_t^T on the int8 tensor cores (FP64 accuracy)."""
        _check(self._lib.oa_gpu_pc_overlap_i8(self._h, self._stream(), _ptr(psi_t), float(alpha), float(w_kx0),
                                              _ptr(out)))

    def pc_rotate_i8(self, T, psi_t, out):
        """out = psi_t T from the digits of the last pc_overlap_i8 (FP64 accuracy)."""
        _check(self._lib.oa_gpu_pc_rotate_i8(self._h, self._stream(), _ptr(T), _ptr(psi_t), _ptr(out)))

    def min_fovlap(self, force) -> float:
        """sum |force|^2 over every stored point (CP_fovlap_calc)."""
        out = C.c_double(0.0)
        _check(self._lib.oa_gpu_min_fovlap(self._h, self._stream(), _ptr(force), C.byref(out)))
        return out.value

    def min_step(self, force, psi, dt, conj=None, gamma=0.0):
        """One steepest-descent (conj None) or conjugate-gradient step on psi."""
        _check(self._lib.oa_gpu_min_step(self._h, self._stream(), _ptr(force), _ptr(conj), _ptr(psi),
                                         float(gamma), float(dt)))

    def has_i8(self) -> bool:
        """True when the int8 overlap / rotation are available (mixed form, <= 128 states)."""
        return bool(self.sizes()["int8_products"])

    def ortho_invsqrt(self, S, T, tol=1e-15, max_iter=1000, with_smax=False):
        it = C.c_int(0)
        err = C.c_double(0.0)
        smax = C.c_double(0.0)
        st = self._lib.oa_gpu_ortho_invsqrt(self._h, self._stream(), _ptr(S), _ptr(T), float(tol), int(max_iter),
                                            C.byref(it), C.byref(err), C.byref(smax))
        if st not in (OA_OK, OA_ERR_NOT_CONVERGED):
            _check(st)
        if with_smax:
            return it.value, err.value, st == OA_OK, smax.value
        return it.value, err.value, st == OA_OK

    def pc_backward(self, M1, X1, a1_kx0, a1_rest, out, M2=None, X2=None, a2=0.0):
        _check(self._lib.oa_gpu_pc_backward(self._h, self._stream(), _ptr(M1), _ptr(X1), float(a1_kx0),
                                            float(a1_rest), _ptr(M2), _ptr(X2), float(a2), _ptr(out)))

    def pc_forward_mixed(self, left, right, alpha, w_kx0, out, nterm=3):
        _check(self._lib.oa_gpu_pc_forward_mixed(self._h, self._stream(), _ptr(left), _ptr(right), float(alpha),
                                                 float(w_kx0), int(nterm), _ptr(out)))

    def pc_backward_mixed(self, M1, X1, a1_kx0, a1_rest, out, M2=None, X2=None, a2=0.0, nterm=3):
        _check(self._lib.oa_gpu_pc_backward_mixed(self._h, self._stream(), _ptr(M1), _ptr(X1), float(a1_kx0),
                                                  float(a1_rest), _ptr(M2), _ptr(X2), float(a2), int(nterm),
                                                  _ptr(out)))

    def check(self):
        _check(self._lib.oa_gpu_check(self._h, self._stream()))

    def fault_inject(self, kind: int):
        """Test hook: kind 1 makes the next split-BF16 forward product skip
        one stage's loads in one block (its bounded wait runs out); 0 clears."""
        _check(self._lib.oa_gpu_fault_inject(self._h, int(kind)))

    def small_gemm(self, A, B, alpha, out):
        _check(self._lib.oa_gpu_small_gemm(self._h, self._stream(), _ptr(A), _ptr(B), float(alpha), _ptr(out)))

    def integrate(self, force, vpsi, psi, dt, complete_prev, fict_out=None):
        _check(self._lib.oa_gpu_integrate(self._h, self._stream(), _ptr(force), _ptr(vpsi), _ptr(psi), float(dt),
                                          int(complete_prev), _ptr(fict_out)))

    def psiv_reset(self, psi, psi_prev, psi_t, vpsi, dt: float):
        """psi_t <- psi, v <- (psi - psi_prev) / dt (oa_gpu_psiv_reset)."""
        _check(self._lib.oa_gpu_psiv_reset(self._h, self._stream(), _ptr(psi), _ptr(psi_prev), _ptr(psi_t),
                                           _ptr(vpsi), float(dt)))

    def set_atoms(self, pos_host: np.ndarray):
        a = np.ascontiguousarray(pos_host, dtype=np.float64)
        _check(self._lib.oa_gpu_set_atoms(self._h, self._stream(), a.ctypes.data_as(_dp)))

    def sizes(self) -> dict:
        out = (C.c_long * 13)()
        _check(self._lib.oa_gpu_sizes(self._h, out))
        keys = ("nstate", "ng", "nlines", "nz", "ldl", "ngroup", "npts", "rbytes", "nlines_d", "launches_per_step",
                "pair_planes", "ngroup_pair", "int8_products")
        return {k: int(v) for k, v in zip(keys, out)}

    def time_kernels(self, psi, reps: int = 5) -> dict:
        out = (C.c_double * len(KERNEL_NAMES))()
        _check(self._lib.oa_gpu_time_kernels(self._h, self._stream(), _ptr(psi), int(reps), out))
        return {k: float(v) for k, v in zip(KERNEL_NAMES, out)}

    def algorithmic_bytes(self) -> dict:
        """Compulsory HBM bytes per launch of each kernel (inputs read once,
        outputs written once) -- the numerator of the roofline."""
        z = self.sizes()
        n, ng, nl, nz, npts = z["nstate"], z["ng"], z["nlines"], z["nz"], z["npts"]
        # density partials: one per state group of the plane kernels (state pairs in the mixed form)
        g = z["ngroup_pair"] if z["pair_planes"] else z["ngroup"]
        cb = 2 * z["rbytes"]
        zrow = n * nz * nl * cb          # the z-line buffer
        coef = n * ng * 16               # one coefficient array
        psir = n * npts * z["rbytes"]    # psi(r) of all states
        return {
            "state_zfwd": coef + zrow,
            # reads the z-line buffer, writes the density partials and psi(r)
            "state_plane_density": zrow + g * npts * 8 + psir,
            "rho_xc": g * npts * 8 + 2 * npts * 8,
            "vks_build": npts * 8 * 2 + npts * z["rbytes"],
            # reads psi(r) and V_KS, writes the z-line buffer
            "state_plane_vks": psir + npts * z["rbytes"] + zrow,
            "state_zbwd": zrow + 2 * coef + ng * 8,
            "pc_forward_S": coef + n * n * 8,
            "pc_backward": 3 * coef,
            "ortho_ns": 2 * n * n * 8,
        }

    def nl_sf(self, psi, fnl_out, nterm=0, enl_out=None):
        _check(self._lib.oa_gpu_nl_sf(self._h, self._stream(), _ptr(psi), int(nterm), _ptr(fnl_out),
                                      _ptr(enl_out)))

    def cp_step(self, state: CPState) -> dict:
        out = (C.c_double * NREC)()
        _check(self._lib.oa_gpu_cp_step(self._h, self._stream(), C.byref(state), out))
        return {k: float(v) for k, v in zip(STEP_KEYS, out)}

    def cp_run(self, state: CPState, nsteps: int, pos_host=None) -> list:
        """nsteps CP steps enqueued back to back with one synchronisation
        (oa_gpu_cp_run); pos_host: optional host array [nsteps][natm][3]
        copied in before each step.  Returns one record per step."""
        out = np.zeros((nsteps, NREC))
        pp = None
        if pos_host is not None:
            pp = np.ascontiguousarray(pos_host, dtype=np.float64)
            if pp.shape != (nsteps, self.sys.natm, 3):
                raise ValueError("pos_host must have shape (nsteps, natm, 3)")
            pp = pp.ctypes.data_as(_dp)
        _check(self._lib.oa_gpu_cp_run(self._h, self._stream(), C.byref(state), int(nsteps), pp,
                                       out.ctypes.data_as(_dp)))
        return [{k: float(v) for k, v in zip(STEP_KEYS, row)} for row in out]

    def ees_init(self, scale: float = 1.2, order: int = 6):
        """Enable the EES nonlocal path (grid and dyp from openatom_b200.ees)."""
        from . import ees
        grid = ees.nonlocal_grid(self.sys, scale, order)
        dyp = np.ascontiguousarray(ees.projector_factor(self.sys, grid, order))
        _check(self._lib.oa_gpu_ees_init(self._h, grid[0], grid[1], grid[2], int(order),
                                         dyp.view(np.float64).ctypes.data_as(_dp)))
        self.ees_grid = grid
        return grid

    def nl_ees(self, psi, fnl_out, enl_out=None):
        _check(self._lib.oa_gpu_nl_ees(self._h, self._stream(), _ptr(psi), _ptr(fnl_out), _ptr(enl_out)))

    def energies(self) -> dict:
        out = (C.c_double * 11)()
        _check(self._lib.oa_gpu_energies(self._h, self._stream(), out))
        keys = ("EKE", "EHART", "EEXT", "EWALD_RECIP", "EEXC", "MUXC", "FICT_KE", "ENL", "EGGA", "ION_KE",
                "EWALD_REAL")
        return {k: float(v) for k, v in zip(keys, out)}


class CPDriver:
    """Host runner of the CP dynamics step on one GPU (electrons; ions fixed)."""

    def __init__(self, sysm, precision: str = "fp64", tol: float = 1e-15, max_iter: int = 1000,
                 psi0=None, norb_tol: float = 0.003, nl_method: str = "sf", ees_order: int = 6,
                 ees_scale: float = 1.2, v0=None, tuning: str = "table"):
        import torch
        self.torch = torch
        self.sys = sysm
        self.ctx = CPContext(sysm, precision, tuning=tuning)
        # nonlocal method (cp_nonloc_ees_opt): "sf" structure factor (N^2) or
        # "ees" (Euler exponential splines of order ees_order on the
        # nonlocal grid); the native step follows the context's choice
        if nl_method not in ("sf", "ees"):
            raise ValueError("nl_method must be 'sf' or 'ees'")
        self.nl_method = nl_method
        if nl_method == "ees":
            self.ctx.ees_init(ees_scale, ees_order)
        dev = torch.device("cuda")
        n, ng = sysm.nstate, sysm.ng
        p0 = sysm.psi if psi0 is None else psi0
        self.psi_t = torch.from_numpy(np.ascontiguousarray(p0)).to(dev)   # non-orthogonal, integrated
        self.psi = self.psi_t.clone()                                     # orthonormal psi_t T
        self.v = torch.zeros_like(self.psi) if v0 is None else torch.from_numpy(np.ascontiguousarray(v0)).to(dev)
        self.F = torch.zeros_like(self.psi)
        self.F2 = torch.zeros_like(self.psi)
        self.psi_prev = torch.zeros_like(self.psi)   # psi(t - dt) for the PsiV finite difference
        self.half_step = True
        self.Fnl = torch.zeros_like(self.psi)
        # mixed form: split-BF16 tcgen05 GEMMs for Lambda, the constraint
        # force and the nonlocal Z / force products; FP64 for S and Psi T
        self.mixed = precision != "fp64"
        self.nterm_nl = 3 if self.mixed else 0
        self.T = torch.eye(n, dtype=torch.float64, device=dev)
        self.S = torch.zeros(n, n, dtype=torch.float64, device=dev)
        self.lam = torch.zeros_like(self.S)
        self.gam = torch.zeros_like(self.S)
        self.tol, self.max_iter = tol, max_iter
        # native steps run on their own stream (the legacy default stream
        # cannot be captured into a CUDA graph)
        self.stream = torch.cuda.Stream()
        # PsiV tolerance (cp_norb_tol, default 0.003; Ortho::maxCheck every step)
        self.norb_tol = norb_tol
        self.n_psiv = 0
        self.iteration = 0
        self.last_ortho = (0, 0.0, True)

    def forces(self):
        """computePsiFandVKS + nonlocal forces + combineForcesGetEke on the
        orthonormal psi."""
        c = self.ctx
        c.state_fft_fwd(self.psi)
        c.vks_build()
        if self.nl_method == "ees":
            c.nl_ees(self.psi, self.Fnl)
        else:
            c.nl_sf(self.psi, self.Fnl, nterm=self.nterm_nl)
        c.vks_apply_fft_bwd(self.psi, self.F, fnl=self.Fnl)

    def native_state(self, use_graph: bool = True) -> CPState:
        """The C-ABI run state pointing at this driver's device buffers."""
        self.torch.cuda.synchronize()
        st = CPState()
        st.psi_t = C.cast(C.c_void_p(self.psi_t.data_ptr()), _dp)
        st.psi = C.cast(C.c_void_p(self.psi.data_ptr()), _dp)
        st.vpsi = C.cast(C.c_void_p(self.v.data_ptr()), _dp)
        st.T = C.cast(C.c_void_p(self.T.data_ptr()), _dp)
        st.iteration = self.iteration
        st.dt = self.sys.dt
        st.ns_tol, st.norb_tol, st.ns_max_iter = self.tol, self.norb_tol, self.max_iter
        st.mixed_nterm = self.nterm_nl
        st.use_graph = int(use_graph)
        st.psiv_pending = 0 if self.half_step else 1
        return st

    def step_native(self, state: CPState) -> dict:
        """One CP step through oa_gpu_cp_step (native sequencing, one sync),
        on the driver's own stream."""
        with self.torch.cuda.stream(self.stream):
            en = self.ctx.cp_step(state)
        self.iteration = state.iteration
        self.half_step = not state.psiv_pending
        self.last_ortho = (int(en["ORTHO_ITERS"]), en["ORTHO_ERR"], True)
        return en

    def run_native(self, state: CPState, nsteps: int, pos_host=None) -> list:
        """nsteps native CP steps with one synchronisation (oa_gpu_cp_run),
        on the driver's own stream."""
        with self.torch.cuda.stream(self.stream):
            ens = self.ctx.cp_run(state, nsteps, pos_host)
        self.iteration = state.iteration
        self.half_step = not state.psiv_pending
        self.last_ortho = (int(ens[-1]["ORTHO_ITERS"]), ens[-1]["ORTHO_ERR"], True)
        return ens

    def launches_per_step(self) -> int:
        return self.ctx.sizes()["launches_per_step"]

    def psiv_reset(self, dt: float):
        """PsiV tolerance reset of the reference's default build
        (finiteDifferencePsiV; oracle.psiv_reset restates it): psi_t = psi,
        T = I, v = (psi - psi_prev) / dt, and the next integration completes
        no half kick."""
        self.ctx.psiv_reset(self.psi, self.psi_prev, self.psi_t, self.v, dt)
        self.T.copy_(self.torch.eye(self.sys.nstate, dtype=self.torch.float64, device=self.T.device))
        self.half_step = False

    def _restart_frame(self):
        """psi_t = psi, T = I (the quench's reset, velocities zero)."""
        self.psi_t.copy_(self.psi)
        self.T.copy_(self.torch.eye(self.sys.nstate, dtype=self.torch.float64, device=self.T.device))
        self.half_step = True

    def quench(self, nsteps: int, dt: float | None = None):
        """Damped CP (steepest descent on the orthonormal states): each step
        zeroes the velocities and resets psi_t to psi.  Used to bring a random
        start near the Born-Oppenheimer surface before dynamics."""
        out = []
        for _ in range(nsteps):
            out.append(self.step(damp_velocity=True, dt=dt))
            self._restart_frame()
            self.iteration = 0
        return out

    def step(self, damp_velocity: bool = False, dt: float | None = None) -> dict:
        c, s = self.ctx, self.sys
        dt = s.dt if dt is None else dt
        self.iteration += 1
        self.forces()
        en = c.energies()
        # Lambda = <psi_x | F_y>, Gamma = T Lambda, F' = F T - Psi Gamma (kx0 psi term halved)
        if self.mixed:
            c.pc_forward_mixed(self.psi, self.F, 1.0, 1.0, self.lam)
            c.small_gemm(self.T, self.lam, 1.0, self.gam)
            c.pc_backward_mixed(self.gam, self.psi, -0.5, -1.0, self.F2, M2=self.T, X2=self.F, a2=1.0)
        else:
            c.pc_forward(self.psi, self.F, 1.0, 1.0, self.lam)
            c.small_gemm(self.T, self.lam, 1.0, self.gam)
            c.pc_backward(self.gam, self.psi, -0.5, -1.0, self.F2, M2=self.T, X2=self.F, a2=1.0)
        # integrate psi_t (after a PsiV reset the velocity is already at t)
        c.integrate(self.F2, self.v, self.psi_t, dt, self.iteration > 1 and self.half_step)
        self.half_step = True
        en["FICT_KE"] = c.energies()["FICT_KE"]
        if damp_velocity:
            self.v.zero_()
        # orthonormalise: S = 2 sum w psi psi (kx0 weight 1/2), T = (S/2)^-1/2, psi = psi_t T
        c.pc_forward(self.psi_t, self.psi_t, 2.0, 0.5, self.S)
        it, err, ok, smax = c.ortho_invsqrt(self.S, self.T, self.tol, self.max_iter, with_smax=True)
        self.last_ortho = (it, err, ok)
        if not ok:
            raise RuntimeError(f"Newton-Schulz did not converge: {it} iterations, residual {err:g}")
        self.psi_prev.copy_(self.psi)
        c.pc_backward(self.T, self.psi_t, 1.0, 1.0, self.psi)
        if smax > self.norb_tol and not damp_velocity:
            # Ortho::maxCheck -> PsiV: restart the non-orthogonal set from psi
            self.psiv_reset(dt)
            self.n_psiv += 1
        en["ORTHO_ITERS"] = it
        en["ORTHO_ERR"] = err
        en["SMAX"] = smax
        return en


class CPMinimizer:
    """Electronic minimisation at fixed ions (cp_min_opt): the loop of
    GSpaceDriver::computeMinimization (gspace.ci:85-196).  Every iteration:
    forces on the orthonormal psi (KS, nonlocal, EKE), the Lagrange
    multipliers Lambda = <psi|F> and F' = F - Psi Lambda (Ortho hands Lambda
    back unchanged in minimisation, ortho.C:497-608), |F'|^2
    (CP_fovlap_calc), the steepest-descent or conjugate-gradient step
    (CP_integrate_min_STD / CP_integrate_min_CG) with the reference's
    conjugate-gradient resets (CP_State_GSpacePlane.C:2636-2660), and the
    orthonormalisation S, Newton-Schulz, psi = psi T (computeNewPsi).  Stops
    when |F'| = sqrt(sum |F'|^2) <= tol (tol_cp_min)."""

    def __init__(self, driver: "CPDriver", method: str = "cg", dt: float | None = None):
        if method not in ("cg", "sd"):
            raise ValueError("method must be 'cg' or 'sd'")
        self.d = driver
        self.method = method
        self.dt = driver.sys.dt if dt is None else dt
        self.conj = driver.torch.zeros_like(driver.psi) if method == "cg" else None
        self.iteration = 0
        self.fovlap = 0.0
        self.fmag = 0.0
        self.num_reset = 0

    def step(self) -> dict:
        d, c = self.d, self.d.ctx
        self.iteration += 1
        d.forces()
        en = c.energies()
        if d.mixed:
            c.pc_forward_mixed(d.psi, d.F, 1.0, 1.0, d.lam)
        else:
            c.pc_forward(d.psi, d.F, 1.0, 1.0, d.lam)
        eye = d.torch.eye(d.sys.nstate, dtype=d.torch.float64, device=d.psi.device)
        c.pc_backward(d.lam, d.psi, -0.5, -1.0, d.F2, M2=eye, X2=d.F, a2=1.0)
        fov_old, fmag_old = self.fovlap, self.fmag
        self.fovlap = c.min_fovlap(d.F2)
        self.fmag = math.sqrt(self.fovlap)
        gamma = 0.0
        if self.method == "cg":
            reset = self.iteration == 1
            if self.iteration > 1 and ((self.fmag > 1.05 * fmag_old and self.num_reset >= 5)
                                       or self.fmag > 2.0 * fmag_old):
                reset = True
            if reset:
                self.num_reset = 0
            else:
                gamma = self.fovlap / fov_old
            self.num_reset += 1
        c.min_step(d.F2, d.psi, self.dt, conj=self.conj, gamma=gamma)
        # computeNewPsi: S, T = (S/2)^-1/2, psi = psi_t T
        d.psi_t.copy_(d.psi)
        c.pc_forward(d.psi_t, d.psi_t, 2.0, 0.5, d.S)
        it, err, ok = c.ortho_invsqrt(d.S, d.T, d.tol, d.max_iter)
        if not ok:
            raise RuntimeError(f"Newton-Schulz did not converge: {it} iterations, residual {err:g}")
        c.pc_backward(d.T, d.psi_t, 1.0, 1.0, d.psi)
        d.psi_t.copy_(d.psi)
        en["FMAG"] = self.fmag
        en["ORTHO_ITERS"] = it
        return en

    def run(self, max_iter: int, tol: float = 0.0) -> list:
        out = []
        for _ in range(max_iter):
            out.append(self.step())
            if self.fmag <= tol:
                break
        return out


def run_batch(drivers, states, nsteps: int, stream=None) -> list:
    """nsteps CP steps of several independent systems in one call
    (oa_gpu_cp_run_batch): after each system's first step, one step of all
    systems is one CUDA graph with the systems on concurrent streams.
    drivers: CPDriver per system; states: their native_state().  Returns,
    per system, one record per step (as CPContext.cp_run)."""
    import torch
    n = len(drivers)
    if n != len(states) or n < 1:
        raise ValueError("one state per driver")
    lib = load_library()
    ctxs = (C.c_void_p * n)(*[d.ctx._h.value for d in drivers])
    sts = (C.c_void_p * n)(*[C.cast(C.pointer(s), C.c_void_p).value for s in states])
    out = np.zeros((n, nsteps, NREC))
    st = stream if stream is not None else drivers[0].stream
    torch.cuda.synchronize()
    _check(lib.oa_gpu_cp_run_batch(ctxs, sts, n, C.c_void_p(st.cuda_stream), int(nsteps),
                                   out.ctypes.data_as(_dp)))
    for d, s in zip(drivers, states):
        d.iteration = s.iteration
        d.half_step = not s.psiv_pending
    return [[{k: float(v) for k, v in zip(STEP_KEYS, row)} for row in sysrows] for sysrows in out]
