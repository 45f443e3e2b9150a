"""State counts of the large single-system configuration (up to 512
states): the cooperative Newton-Schulz kernel that runs above 128 states,
against an eigendecomposition in FP64, and the native step's general-kernel
path above 128 states against the host runner."""
import numpy as np
import pytest

from openatom_b200.system import make_system

pytestmark = pytest.mark.gpu


def _ctx_with_states(nst):
    from openatom_b200.gpu import CPContext
    s = make_system("w8", nstate=32, seed=21)
    rng = np.random.default_rng(4)
    s.psi = (rng.standard_normal((nst, s.ng)) + 1j * rng.standard_normal((nst, s.ng))) / np.sqrt(s.ng)
    s.nstate = nst
    s.occ = np.ones(nst)
    return CPContext(s, "fp64")


@pytest.mark.parametrize("nst", [130, 512])
def test_ortho_invsqrt_many_states(nst):
    """T = (S/2)^(-1/2) for S = 2 I + a symmetric perturbation of 1e-2
    (ortho.C:153-266 with the S = 2I occupation convention), to 1e-12."""
    import torch
    ctx = _ctx_with_states(nst)
    rng = np.random.default_rng(nst)
    E = rng.standard_normal((nst, nst)) * 1e-2
    S = 2.0 * np.eye(nst) + 0.5 * (E + E.T)
    w, V = np.linalg.eigh(S / 2.0)
    T_ref = (V * w ** -0.5) @ V.T
    Sg = torch.from_numpy(S).cuda()
    T = torch.zeros_like(Sg)
    it, err, ok = ctx.ortho_invsqrt(Sg, T, 1e-15, 1000)
    assert ok and it < 20
    Tn = T.cpu().numpy()
    assert float(np.max(np.abs(Tn - T_ref)) / np.max(np.abs(T_ref))) < 1e-12
    # T S T = 2 I
    assert float(np.max(np.abs(Tn @ S @ Tn - 2.0 * np.eye(nst)))) < 1e-12
    ctx.close()


def test_native_run_many_states():
    """Above 128 states the native step runs Psi T and the PsiV projection
    through the general FP64 kernels (the projection computed whole and kept
    under the device flag): it reproduces the host runner bit for bit, with
    a reset in every step."""
    from openatom_b200.gpu import CPDriver
    s = make_system("w8", nstate=130, seed=22, dt=0.5)
    a = CPDriver(s, "fp64", norb_tol=1e-14)
    c = CPDriver(s, "fp64", norb_tol=1e-14)
    sc = c.native_state(use_graph=True)
    ea = [a.step() for _ in range(3)]
    ec = c.run_native(sc, 3)
    assert a.n_psiv == 3
    for i in range(3):
        for k in ("EKE", "EHART", "EEXC", "ENL", "FICT_KE", "SMAX"):
            assert ec[i][k] == ea[i][k], (i, k, ea[i][k], ec[i][k])
    assert np.array_equal(a.psi.cpu().numpy(), c.psi.cpu().numpy())
    assert np.array_equal(a.psi_t.cpu().numpy(), c.psi_t.cpu().numpy())
    assert np.array_equal(a.v.cpu().numpy(), c.v.cpu().numpy())
