"""Finite-difference Poisson stand-in (electrostatics.FDPoissonGAA), on CPU.

Checks on a small gate-all-around case: the coupling matrix is symmetric
(deposit and gather use the same trilinear weights and the stencil is
symmetric), positive and decaying along the tube; a gate that wraps
everything gives U_ext = -Vg exactly; the couplings between distinct rings
agree with the analytic Bessel-series operator to the discretisation error;
the self-consistent loop of the oracle runs with it.
"""
import numpy as np
import pytest


def _rings(uc, acc=1.42e-10):
    N = 4 * uc
    y0 = -(uc / 2.0) * 3.0 * acc - acc / 2.0
    ring = np.array([acc, 1.5 * acc, 2.5 * acc, 3.0 * acc])
    r = np.arange(N)
    return (ring[r % 4] + 3 * acc * (r // 4) + y0) / 1e-9


@pytest.fixture(scope="module")
def fd_case():
    from electrostatic_b200.electrostatics import FDPoissonGAA, GateAllAround
    y = _rings(5)
    R = 1.42e-10 * np.sqrt(3.0) * 17 / (2 * np.pi)
    fd = FDPoissonGAA(y, R, R + 1.0e-9, 17, shape=(36, 36, 64), h_xy=0.1e-9, device="cpu", tol=1e-9)
    ga = GateAllAround(y, R, R + 1.0e-9)
    return fd, ga, y


def test_fd_coupling_symmetric_positive_decaying(fd_case):
    fd, _, y = fd_case
    K = fd.K
    assert np.max(np.abs(K - K.T)) <= 1e-6 * np.max(np.abs(K))
    assert np.all(np.linalg.eigvalsh(0.5 * (K + K.T)) > 0)
    mid = len(y) // 2
    assert K[mid, mid] > K[mid, mid + 4] > K[mid, mid + 8] > 0


def test_fd_closed_gate_external_and_contacts(fd_case):
    fd, _, y = fd_case
    np.testing.assert_allclose(fd.external(0.37), -0.37, rtol=0, atol=1e-7)
    from electrostatic_b200.electrostatics import FDPoissonGAA
    R = 1.42e-10 * np.sqrt(3.0) * 17 / (2 * np.pi)
    fc = FDPoissonGAA(y, R, R + 1.0e-9, 17, shape=(36, 36, 64), h_xy=0.1e-9, device="cpu", tol=1e-9,
                      contact_length=0.4e-9, Vds=0.3)
    U = fc.external(0.5)
    mid = len(y) // 2
    # source at 0 V, gate at 0.5 V, drain at 0.3 V (U = -phi): the source end is
    # highest, the channel lies between -Vg and -Vds, the drain end below the source
    assert U[0] > U[mid] and U[-1] < U[0] and -0.5 <= U[mid] <= -0.3
    # linear in the electrode potentials
    d1, d2 = fc.external(0.5) - fc.external(0.1), fc.external(0.9) - fc.external(0.5)
    np.testing.assert_allclose(d1, d2, rtol=1e-6, atol=1e-9)


def test_fd_matches_analytic_couplings(fd_case):
    fd, ga, y = fd_case
    K, Ka = fd.K, ga.K
    mid = len(y) // 2
    off = [d for d in range(2, 8)]
    rel = [abs(K[mid, mid + d] - Ka[mid, mid + d]) / Ka[mid, mid + d] for d in off]
    assert max(rel) < 0.12, rel


def test_oracle_scf_with_fd_operator(fd_case, oracle):
    from oracle.scf_oracle import run_scf_oracle
    fd, _, y = fd_case
    t = oracle.OracleTube(type_id=(17, 0), num_unitcells=5, num_modes=2, contact_mu=(-1.0, -1.0),
                          contact_T=(300.0, 300.0), eq_integration_pts=(24, 24, 24), E_pole_max=3.0)
    res = run_scf_oracle(t, fd, [0.0, 0.2], nthreads=4)
    for s in res.steps:
        assert s.norm <= 1e-6 and s.iterations < 100
        np.testing.assert_allclose(s.U, fd.potential(s.Q, s.Vg), rtol=0, atol=1e-5)
