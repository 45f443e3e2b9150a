"""State files in the reference's format (readState / writeStateFile,
util.C:1107-1330 and 1955-2175; flip_data_set, para_grp_parse.C:178-260):
layout of a written file, exact round trips in the binary encodings and in
text with enough digits, the reference's six-digit text, and refusal of
files that do not fit the system."""
import os

import numpy as np
import pytest

from openatom_b200 import state_io as S
from openatom_b200.system import make_system


@pytest.fixture(scope="module")
def sysm():
    return make_system("w4", seed=51)


def test_file_layout(sysm, tmp_path):
    s = sysm
    p = str(tmp_path / "state1.out")
    S.write_state(p, s.psi[0], s, "text", digits=17)
    lines = open(p).read().splitlines()
    n, nx, ny, nz = (int(t) for t in lines[0].split())
    assert (nx, ny, nz) == tuple(s.nfft)
    # the unique half: everything but the redundant kx = 0 points
    assert n == s.ng - s.nkx0_red == len(lines) - 1
    first = [int(t) for t in lines[1].split()[2:]]
    last = [int(t) for t in lines[-1].split()[2:]]
    assert first == [0, 0, 1] and last == [0, 0, 0]
    ks = np.array([[int(t) for t in ln.split()[2:]] for ln in lines[1:-1]])
    # sorted by (kx, ky, kz), kz consecutive inside a line (processState's checks)
    key = (ks[:, 0] * 1000 + ks[:, 1]) * 1000 + ks[:, 2]
    assert np.all(np.diff(key) > 0)


@pytest.mark.parametrize("enc", ["binary", "binary.gz"])
def test_binary_round_trip_is_exact(sysm, tmp_path, enc):
    s = sysm
    rng = np.random.default_rng(1)
    v = (rng.standard_normal(s.psi.shape) + 1j * rng.standard_normal(s.psi.shape)) * 1e-3
    from openatom_b200.system import symmetrize_kx0
    v = symmetrize_kx0(v, s.kx, s.ky, s.kz)
    paths = S.write_states(str(tmp_path), s.psi, s, vpsi=v, encoding=enc)
    assert paths[0].endswith(os.path.join("Spin.0_Kpt.0_Bead.0_Temper.0", "state1.out" + (".gz" if "gz" in enc else "")))
    got = S.read_states(str(tmp_path), s, encoding=enc)
    gotv = S.read_states(str(tmp_path), s, velocity=True, encoding=enc)
    assert np.array_equal(got, s.psi)
    assert np.array_equal(gotv, v)


@pytest.mark.parametrize("enc", ["text", "text.gz"])
def test_text_round_trip(sysm, tmp_path, enc):
    s = sysm
    S.write_states(str(tmp_path / "a"), s.psi, s, encoding=enc, digits=17)
    assert np.array_equal(S.read_states(str(tmp_path / "a"), s, encoding=enc), s.psi)
    # the reference's own text (%g): six significant digits
    S.write_states(str(tmp_path / "b"), s.psi, s, encoding=enc)
    got = S.read_states(str(tmp_path / "b"), s, encoding=enc)
    assert np.max(np.abs(got - s.psi) / np.maximum(np.abs(s.psi), 1e-300)) < 1e-5


def test_redundant_half_is_rebuilt(sysm, tmp_path):
    """The file holds one half of the kx = 0 plane; the reader rebuilds the
    other as conjugates (c(0,-ky,-kz) = conj c(0,ky,kz))."""
    s = sysm
    p = str(tmp_path / "s.out")
    S.write_state(p, s.psi[1], s, "binary")
    got = S.read_state(p, s, "binary")
    red = np.arange(s.nkx0_red)
    key = {(int(s.ky[i]), int(s.kz[i])): i for i in range(s.nkx0)}
    partner = np.array([key[(-int(s.ky[i]), -int(s.kz[i]))] for i in red])
    assert np.array_equal(got[red], np.conj(got[partner]))


def test_bad_files_are_refused(sysm, tmp_path):
    s = sysm
    p = str(tmp_path / "s.out")
    S.write_state(p, s.psi[0], s, "text", digits=17)
    other = make_system("w4", seed=51, nfft=(40, 40, 40))
    with pytest.raises(S.StateFileError, match="grid"):
        S.read_state(p, other, "text")
    smaller = make_system("w4", seed=51, ecut_ry=20.0)
    with pytest.raises(S.StateFileError):
        S.read_state(p, smaller, "text")
    lines = open(p).read().splitlines()
    open(p, "w").write("\n".join(lines[:-1]) + "\n")   # g = 0 missing, header unchanged
    with pytest.raises(S.StateFileError, match="can't parse"):
        S.read_state(p, s, "text")
    n, nx, ny, nz = lines[0].split()
    open(p, "w").write("\n".join([f"{int(n) - 1} {nx} {ny} {nz}"] + lines[1:-1]) + "\n")
    with pytest.raises(S.StateFileError, match="g = 0"):
        S.read_state(p, s, "text")
    with pytest.raises(S.StateFileError, match="can't open"):
        S.read_state(str(tmp_path / "none.out"), s, "text")
