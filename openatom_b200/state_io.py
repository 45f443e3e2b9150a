"""State-file reader and writer in the reference's format, so GPU runs can
start from and restart into reference-format coefficient files.

Files (one per state, N = state index + 1)::

    <data_path>/Spin.<s>_Kpt.<k>_Bead.<b>_Temper.<t>/state<N>.out[.gz]   coefficients
    <data_path>/Spin.<s>_Kpt.<k>_Bead.<b>_Temper.<t>/vState<N>.out[.gz]  velocities

(``CP_State_GSpacePlane.C:697-876``).  Content, Gamma point, double packing:

* a header ``ncoef nx ny nz``: the number of points in the file and the FFT
  grid;
* one point per line, ``re im kx ky kz``: the kx = 0 unique half without
  g = 0 (it starts at (0, 0, 1)), then every kx > 0 point, sorted by
  (kx, ky, kz), and g = 0 last (``writeStateFile``, ``util.C:1955-2175``,
  with ``sort_psi_output``).

Four encodings, the reference's ``ibinary_opt``: 0 text, 1 binary (int32
header, then per point float64 re, im and int32 kx, ky, kz, packed), 2 text
gzipped, 3 binary gzipped (``.gz`` appended to the name).  The reference
writes text with ``%g`` (six significant digits); ``write_state`` does the
same unless ``digits`` asks for more, and binary is exact.

Reading follows ``readState`` (``util.C:1107-1330``) and the double-pack
expansion ``ParaGrpParse::flip_data_set`` (``para_grp_parse.C:178-260``): the
points are read up to g = 0, the redundant kx = 0 half is rebuilt as
c(0, -ky, -kz) = conj(c(0, ky, kz)), and the points are mapped onto the
system's own point order (z-line runs, the doublePack layout the GPU path
uses).  Malformed files raise ``StateFileError`` (the reference aborts).
"""
from __future__ import annotations

import gzip
import io
import os
import struct

import numpy as np

ENCODINGS = {"text": 0, "binary": 1, "text.gz": 2, "binary.gz": 3}


class StateFileError(ValueError):
    """A state file that does not parse or does not fit the system."""


def state_path(data_path: str, istate: int, velocity: bool = False, encoding: str = "text", spin: int = 0,
               kpt: int = 0, bead: int = 0, temper: int = 0) -> str:
    """Path of state istate (0-based) as the reference names it."""
    name = f"{'vState' if velocity else 'state'}{istate + 1}.out"
    if encoding.endswith(".gz"):
        name += ".gz"
    return os.path.join(data_path, f"Spin.{spin}_Kpt.{kpt}_Bead.{bead}_Temper.{temper}", name)


def file_order(sysm) -> np.ndarray:
    """Indices into the system's points in file order: the kx = 0 unique half
    without g = 0 and the kx > 0 points sorted by (kx, ky, kz), then g = 0."""
    kx, ky, kz = (np.asarray(a, dtype=np.int64) for a in (sysm.kx, sysm.ky, sysm.kz))
    red = (kx == 0) & ((ky < 0) | ((ky == 0) & (kz < 0)))
    g0 = (kx == 0) & (ky == 0) & (kz == 0)
    keep = np.nonzero(~red & ~g0)[0]
    keep = keep[np.lexsort((kz[keep], ky[keep], kx[keep]))]
    z = np.nonzero(g0)[0]
    if z.size != 1:
        raise StateFileError("the g-sphere has no g = 0 point")
    return np.concatenate([keep, z])


def _open(path: str, mode: str, gz: bool):
    return gzip.open(path, mode) if gz else open(path, mode)


def write_state(path: str, coef: np.ndarray, sysm, encoding: str = "text", digits: int | None = None) -> None:
    """Write one state's coefficients (complex [ng], the system's point order)."""
    if encoding not in ENCODINGS:
        raise ValueError(f"encoding must be one of {sorted(ENCODINGS)}")
    c = np.asarray(coef, dtype=np.complex128)
    if c.shape != (sysm.ng,):
        raise ValueError(f"coefficients must have shape ({sysm.ng},)")
    order = file_order(sysm)
    nx, ny, nz = sysm.nfft
    kx, ky, kz = sysm.kx[order], sysm.ky[order], sysm.kz[order]
    v = c[order]
    gz = encoding.endswith(".gz")
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    if encoding.startswith("binary"):
        rec = np.zeros(order.size, dtype=np.dtype([("re", "<f8"), ("im", "<f8"), ("kx", "<i4"), ("ky", "<i4"),
                                                   ("kz", "<i4")]))
        rec["re"], rec["im"], rec["kx"], rec["ky"], rec["kz"] = v.real, v.imag, kx, ky, kz
        with _open(path, "wb", gz) as f:
            f.write(struct.pack("<4i", order.size, nx, ny, nz))
            f.write(rec.tobytes())
    else:
        fmt = "%g" if digits is None else f"%.{int(digits)}g"
        lines = [f"{order.size} {nx} {ny} {nz}\n"]
        lines += [f"{fmt % a} {fmt % b} {x} {y} {z} \n" for a, b, x, y, z in zip(v.real, v.imag, kx, ky, kz)]
        with _open(path, "wt" if gz else "w", gz) as f:
            f.writelines(lines)


def _read_points(path: str, encoding: str):
    gz = encoding.endswith(".gz")
    if not os.path.exists(path):
        raise StateFileError(f"can't open state file {path}")
    if encoding.startswith("binary"):
        with _open(path, "rb", gz) as f:
            raw = f.read()
        if len(raw) < 16:
            raise StateFileError(f"can't parse size line of file {path}")
        n, nx, ny, nz = struct.unpack("<4i", raw[:16])
        rec = np.dtype([("re", "<f8"), ("im", "<f8"), ("kx", "<i4"), ("ky", "<i4"), ("kz", "<i4")])
        body = raw[16:]
        if n < 1 or len(body) < n * rec.itemsize:
            raise StateFileError(f"can't parse packed state location {path}")
        r = np.frombuffer(body[:n * rec.itemsize], dtype=rec)
        return (nx, ny, nz), r["re"] + 1j * r["im"], r["kx"].astype(np.int64), r["ky"].astype(np.int64), \
            r["kz"].astype(np.int64)
    with _open(path, "rt" if gz else "r", gz) as f:
        text = f.read()
    tok = text.split()
    if len(tok) < 4:
        raise StateFileError(f"can't parse size line of file {path}")
    try:
        n, nx, ny, nz = (int(t) for t in tok[:4])
        body = np.array(tok[4:4 + 5 * n], dtype=object)
        if body.size < 5 * n:
            raise ValueError
        body = body.reshape(n, 5)
        re = body[:, 0].astype(np.float64)
        im = body[:, 1].astype(np.float64)
        ks = body[:, 2:].astype(np.int64)
    except ValueError:
        raise StateFileError(f"can't parse packed state location {path}") from None
    return (nx, ny, nz), re + 1j * im, ks[:, 0], ks[:, 1], ks[:, 2]


def read_state(path: str, sysm, encoding: str = "text") -> np.ndarray:
    """Read one state file into the system's point order (complex [ng])."""
    if encoding not in ENCODINGS:
        raise ValueError(f"encoding must be one of {sorted(ENCODINGS)}")
    grid, val, kx, ky, kz = _read_points(path, encoding)
    if tuple(grid) != tuple(sysm.nfft):
        raise StateFileError(f"{path}: FFT grid {grid} does not match the system's {tuple(sysm.nfft)}")
    # readState stops at g = 0 under double packing
    z = np.nonzero((kx == 0) & (ky == 0) & (kz == 0))[0]
    if z.size == 0:
        raise StateFileError(f"{path}: no g = 0 point (double-packed files end with it)")
    n = int(z[0]) + 1
    val, kx, ky, kz = val[:n], kx[:n], ky[:n], kz[:n]
    # flip_data_set: the kx = 0 points come first, g = 0 is last
    nplane0 = int(np.count_nonzero(kx == 0))
    if np.any(kx[:nplane0 - 1] != 0):
        raise StateFileError(f"{path}: error while flipping the double-packed data set")
    if nplane0 > 1 and (ky[0], kz[0]) != (0, 1):
        raise StateFileError(f"{path}: the kx = 0 half must start at (0, 0, 1)")
    full = {}
    for c, a, b, d in zip(val, kx, ky, kz):
        full[(int(a), int(b), int(d))] = c
    for c, a, b, d in zip(val[:nplane0 - 1], kx[:nplane0 - 1], ky[:nplane0 - 1], kz[:nplane0 - 1]):
        full[(0, -int(b), -int(d))] = np.conj(c)
    out = np.empty(sysm.ng, dtype=np.complex128)
    try:
        for i, key in enumerate(zip(sysm.kx.tolist(), sysm.ky.tolist(), sysm.kz.tolist())):
            out[i] = full[key]
    except KeyError as e:
        raise StateFileError(f"{path}: g-point {e.args[0]} of the system's sphere is missing") from None
    if len(full) != sysm.ng:
        raise StateFileError(f"{path}: {len(full)} points, the system's sphere has {sysm.ng}")
    return out


def write_states(data_path: str, psi: np.ndarray, sysm, vpsi: np.ndarray | None = None, encoding: str = "text",
                 digits: int | None = None, **where) -> list:
    """state<N>.out for every state (and vState<N>.out when vpsi is given)."""
    paths = []
    for i in range(psi.shape[0]):
        p = state_path(data_path, i, False, encoding, **where)
        write_state(p, psi[i], sysm, encoding, digits)
        paths.append(p)
        if vpsi is not None:
            write_state(state_path(data_path, i, True, encoding, **where), vpsi[i], sysm, encoding, digits)
    return paths


def read_states(data_path: str, sysm, nstate: int | None = None, velocity: bool = False, encoding: str = "text",
                **where) -> np.ndarray:
    """All states (or velocities) of a run directory, [nstate][ng] complex."""
    n = sysm.nstate if nstate is None else nstate
    return np.stack([read_state(state_path(data_path, i, velocity, encoding, **where), sysm, encoding)
                     for i in range(n)])


def dumps_header(path: str, encoding: str = "text") -> tuple:
    """(ncoef, nx, ny, nz) of a state file."""
    gz = encoding.endswith(".gz")
    if encoding.startswith("binary"):
        with _open(path, "rb", gz) as f:
            return struct.unpack("<4i", f.read(16))
    with _open(path, "rt" if gz else "r", gz) as f:
        return tuple(int(t) for t in io.StringIO(f.readline()).read().split()[:4])
