"""Both RGF schedules against the FP64 oracle, through the C-ABI.

The fused schedule (one kernel: forward and backward sweeps meet in the
middle, each integrates the half it crosses second) has separate code for
one segment, the middle segment of an odd count, the contact segments and
the interior; the lengths below cover segment counts 1, 2, 3, 4, 5, 13 and
larger, with and without a partial last segment, on contour and real-axis
chains, in FP64 and mixed precision.  The two-pass schedule runs the same
cases, and both must agree with the oracle to the usual bounds.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-8
MIXED_TOL = 1e-5


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.fixture
def schedule():
    from electrostatic_b200.negf import TUNE_SCHEDULE, set_tuning
    yield lambda v: set_tuning(TUNE_SCHEDULE, v)
    set_tuning(TUNE_SCHEDULE, 0)


# (type_id, unit cells): N = 4 * cells for zigzag, 2 * cells for the chiral (13, 2)
LENGTHS = [((17, 0), 1), ((17, 0), 3), ((17, 0), 5), ((17, 0), 6), ((17, 0), 8), ((17, 0), 9), ((13, 2), 17),
           ((17, 0), 25), ((19, 0), 51), ((17, 0), 300)]


@pytest.mark.parametrize("sched", ["fused", "two_pass"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("tid,cells", LENGTHS)
def test_schedule_matches_oracle(oracle, schedule, sched, precision, tid, cells):
    from electrostatic_b200.negf import CNT, SCHEDULE_FUSED, SCHEDULE_TWO_PASS, last_stats
    from electrostatic_b200.workloads import site_potential
    kw = dict(type_id=tid, num_unitcells=cells, num_modes=3, contact_mu=(0.05, -0.35), contact_T=(300.0, 300.0),
              eq_integration_pts=(24, 24, 40), noneq_integration_pts=(40, 80, 40),
              noneq_percent_intercuts=(30.0, 70.0), E_zPlus_imag=2e-3, precision=precision,
              mixed_realaxis_fp32=True)
    schedule(SCHEDULE_FUSED if sched == "fused" else SCHEDULE_TWO_PASS)
    g = CNT(**kw)
    U = site_potential(g.site_positions(), 1000 + cells, amp=0.3, ramp=0.35)
    g.set_potential(U, (U[0], U[-1]))
    Qg = g.Solve_NEGF()
    st = last_stats()
    assert st["schedule"] == (2 if sched == "fused" else 1)
    okw = {k: v for k, v in kw.items() if k not in ("precision", "mixed_realaxis_fp32")}
    o = oracle.OracleTube(**okw)
    o.set_potential(U, (U[0], U[-1]))
    Qo = o.charge(nthreads=8)
    assert np.all(np.isfinite(Qg))
    tol = FP64_TOL if precision == "fp64" else MIXED_TOL
    assert _rel(Qg, Qo) <= tol, (_rel(Qg, Qo), g.num_field_sites)


def test_fused_equilibrium_poles_and_decimation(oracle, schedule):
    from electrostatic_b200.negf import CNT, SCHEDULE_FUSED
    schedule(SCHEDULE_FUSED)
    for kw in (dict(type_id=(17, 0), num_unitcells=40, num_modes=2, contact_mu=(-1.0, -1.0), contact_T=(300.0, 300.0),
                    eq_integration_pts=(32, 32, 32), E_pole_max=3.0),
               dict(type_id=(17, 0), num_unitcells=12, num_modes=2, contact_mu=(0.0, -0.3), contact_T=(300.0, 300.0),
                    eq_integration_pts=(16, 16, 16), noneq_integration_pts=(48,), use_decimation=1)):
        g = CNT(**kw)
        y = g.site_positions()
        U = 0.2 * np.exp(-((y - y.mean()) ** 2) / 10.0) + 0.05 * (y - y[0]) / (y[-1] - y[0])
        g.set_potential(U, (U[0], U[-1]))
        o = oracle.OracleTube(**kw)
        o.set_potential(U, (U[0], U[-1]))
        assert _rel(g.Solve_NEGF(), o.charge(nthreads=8)) <= FP64_TOL


def test_schedules_agree_on_config2_shape(schedule):
    """The benchmark tube with a quarter of its energies: fused vs two-pass."""
    from electrostatic_b200.negf import CNT, SCHEDULE_FUSED, SCHEDULE_TWO_PASS
    from electrostatic_b200.workloads import SEED_BASE, config2_kwargs, site_potential
    g = CNT(**config2_kwargs(small=True))
    U = site_potential(g.site_positions(), SEED_BASE + 2)
    g.set_potential(U, (U[0], U[-1]))
    schedule(SCHEDULE_FUSED)
    a = g.Solve_NEGF()
    schedule(SCHEDULE_TWO_PASS)
    b = g.Solve_NEGF()
    assert _rel(a, b) <= 1e-11
