"""A GPU run restarted from reference-format state files (state<N>.out and
vState<N>.out, CP_State_GSpacePlane.C:697-876): the native step from the
files read back reproduces the native step from the same arrays in memory,
bit for bit in the binary encoding, and to the six digits of the
reference's text encoding."""
import numpy as np
import pytest

from openatom_b200 import state_io as S
from openatom_b200.system import make_system

pytestmark = pytest.mark.gpu


def test_restart_from_state_files(tmp_path):
    from openatom_b200.gpu import CPDriver
    s = make_system("w8", nstate=16, seed=52, ecut_mass=2.0, cmass0=400.0, dt=5.0)
    a = CPDriver(s, "fp64", norb_tol=0.003)
    a.run_native(a.native_state(use_graph=True), 3)
    psi = a.psi.cpu().numpy()
    v = a.v.cpu().numpy()
    a.ctx.close()
    S.write_states(str(tmp_path / "bin"), psi, s, vpsi=v, encoding="binary")
    S.write_states(str(tmp_path / "txt"), psi, s, vpsi=v, encoding="text")
    out = {}
    for tag, p0, v0 in (("mem", psi, v),
                        ("bin", S.read_states(str(tmp_path / "bin"), s, encoding="binary"),
                         S.read_states(str(tmp_path / "bin"), s, velocity=True, encoding="binary")),
                        ("txt", S.read_states(str(tmp_path / "txt"), s, encoding="text"),
                         S.read_states(str(tmp_path / "txt"), s, velocity=True, encoding="text"))):
        d = CPDriver(s, "fp64", psi0=p0, v0=v0, norb_tol=0.003)
        out[tag] = (d.run_native(d.native_state(use_graph=True), 3), d.psi.cpu().numpy())
        d.ctx.close()
    for i in range(3):
        for k in ("EKE", "EHART", "EEXT", "EEXC", "ENL", "FICT_KE"):
            assert out["bin"][0][i][k] == out["mem"][0][i][k], (i, k)
            assert abs(out["txt"][0][i][k] - out["mem"][0][i][k]) <= 1e-4 * max(1.0, abs(out["mem"][0][i][k]))
    assert np.array_equal(out["bin"][1], out["mem"][1])
