"""Self-consistent loop: electrostatics stand-in (CPU), oracle SCF (CPU), and
the device SCF against the oracle SCF (GPU)."""
import numpy as np
import pytest


def _ring_y(unitcells, acc=1.42e-10):
    y0 = -(unitcells / 2.0) * 3 * acc - acc / 2
    ring = np.array([acc, 1.5 * acc, 2.5 * acc, 3 * acc])
    r = np.arange(4 * unitcells)
    return (ring[r % 4] + 3 * acc * (r // 4) + y0) / 1e-9


def test_coupling_matrix_properties():
    from electrostatic_b200.electrostatics import ring_coupling_matrix
    y = _ring_y(20)
    K = ring_coupling_matrix(y, 0.6655e-9, 2.2e-9)
    assert np.allclose(K, K.T)
    assert np.all(K > 0)
    # screened by the grounded gate: decays with distance, positive definite
    assert K[0, 79] < 1e-3 * K[0, 0]  # 8.4 nm = 3.8 gate radii away
    assert np.all(np.linalg.eigvalsh(K) > 0)


def test_coupling_matrix_far_field_is_exponential():
    """Beyond a few gate radii only the first Bessel term survives: exp(-x1 dz / a)."""
    from electrostatic_b200.electrostatics import ring_coupling_matrix
    a = 2.0e-9
    y = np.array([0.0, 6.0, 7.0])  # nm
    K = ring_coupling_matrix(y, 0.6655e-9, a)
    x1 = 2.404825557695773
    np.testing.assert_allclose(K[0, 2] / K[0, 1], np.exp(-x1 * 1e-9 / a), rtol=1e-4)  # next term ~1e-5


SMALL = dict(type_id=(17, 0), num_unitcells=10, num_modes=2, contact_mu=(-1.0, -1.0), contact_T=(300.0, 300.0),
             eq_integration_pts=(24, 24, 24), E_valence_min=-10.0, E_pole_max=3.0)


def test_oracle_scf_converges(oracle):
    from electrostatic_b200.electrostatics import ring_coupling_matrix
    from oracle.scf_oracle import run_scf_oracle
    t = oracle.OracleTube(**SMALL)
    K = ring_coupling_matrix(_ring_y(10), t.radius, t.radius + 1.5e-9)
    res = run_scf_oracle(t, K, [0.0, 0.2], nthreads=4)
    for s in res.steps:
        assert s.norm <= 1e-6 and s.iterations < 60
    # a positive gate voltage removes holes (mu = -1 eV: p-type tube)
    assert res.steps[1].Q.sum() < res.steps[0].Q.sum()


@pytest.mark.gpu
@pytest.mark.parametrize("keep", [False, True])
def test_device_scf_follows_oracle_scf(oracle, keep):
    from electrostatic_b200.electrostatics import GateAllAround
    from electrostatic_b200.negf import CNT
    from electrostatic_b200.scf import run_scf
    from oracle.scf_oracle import run_scf_oracle
    g = CNT(**SMALL)
    y = g.site_positions()
    np.testing.assert_allclose(y, _ring_y(10), rtol=1e-12)
    ga = GateAllAround(y, 0.6655e-9, 0.6655e-9 + 1.5e-9)
    Vg = [0.0, 0.15, 0.3]
    rg = run_scf(g, ga, Vg, reset_with_previous_charge=keep)
    ro = run_scf_oracle(oracle.OracleTube(**SMALL), ga.K, Vg, reset_with_previous_charge=keep, nthreads=8)
    for sg, so in zip(rg.steps, ro.steps):
        assert sg.norm <= 1e-6
        assert sg.iterations == so.iterations, (sg.iterations, so.iterations)
        np.testing.assert_allclose(sg.Q, so.Q, rtol=0, atol=1e-9)
        np.testing.assert_allclose(sg.U, so.U, rtol=0, atol=1e-9)


def test_step_response_properties():
    """Wall-potential step inside the gate cylinder: s(0) = 1/2, s(dz) + s(-dz) = 1,
    monotonic, bare step far away, and a contacted stand-in pins the tube ends."""
    from electrostatic_b200.electrostatics import step_response
    a, r = 2.17e-9, 0.67e-9
    dz = np.linspace(-40e-9, 40e-9, 801)
    s = step_response(dz, r, a)
    assert abs(s[400] - 0.5) < 1e-12
    assert np.max(np.abs(s + s[::-1] - 1.0)) < 1e-12
    assert np.all(np.diff(s) >= -1e-12)
    assert s[0] < 1e-12 and s[-1] > 1 - 1e-12
    from electrostatic_b200.workloads import gate_with_contacts
    y = np.linspace(0, 60, 600)
    g = gate_with_contacts(y, r, vds=0.4)
    U = g.external(0.3)
    assert abs(U[0]) < 1e-3 and abs(U[-1] + 0.4) < 1e-3 and abs(U[300] + 0.3) < 1e-6
