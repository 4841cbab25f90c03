"""GPU parity of the transport characteristics (DOS, transmission,
conductance, LDOS, terminal current, integrand probes) through the C-ABI.

References: the reference engine's committed DOS_Compare output
(tests/golden/dos_compare_gpu_*.txt, 6 printed digits) and the FP64 oracle
(Compute_DensityOfStates / Compute_Current restated with the per-site contact
walks).  Bar: norm-wise relative error <= 1e-8 against the oracle.
"""
import os

import numpy as np
import pytest

from test_gpu_parity import _pair, _rel

pytestmark = pytest.mark.gpu

TOL = 1e-8
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_dos_transmission_against_reference_output(oracle):
    from electrostatic_b200.negf import CNT
    kw = dict(type_id=(17, 0), num_unitcells=1, num_modes=2, contact_mu=(0.0, -1e-4),
              realaxis_window=(-1.0, 1.0, 200, 0), E_zPlus_imag=1e-8)
    g = CNT(**kw)
    g.set_potential(np.zeros(g.num_field_sites), (0.0, 0.0))
    d = g.Compute_DensityOfStates()
    gT = np.loadtxt(os.path.join(GOLDEN, "dos_compare_gpu_Transmission.txt"), skiprows=1)
    gD = np.loadtxt(os.path.join(GOLDEN, "dos_compare_gpu_LDOS.txt"), skiprows=1)
    assert np.allclose(d["E"].real, gT[:, 0], rtol=0, atol=1e-6)
    assert np.max(np.abs(d["T"] - gT[:, 1]) / np.abs(gT[:, 1])) < 1e-5
    assert np.max(np.abs(d["dos"] - gD[:, 1]) / np.abs(gD[:, 1])) < 1e-5
    # and element-wise against the oracle, gap values (~1e-15) included
    o = oracle.OracleTube(**kw)
    o.set_potential(np.zeros(o.N), (0.0, 0.0))
    od = o.dos(faithful=True, nthreads=8)
    assert np.max(np.abs(d["T"] - od["T"]) / np.abs(od["T"])) < 1e-7
    assert np.max(np.abs(d["dos"] - od["dos"]) / np.abs(od["dos"])) < 1e-7


TRANSPORT_CASES = {
    # biased: DOS path = the non-equilibrium paths (two GL paths with an intercut)
    "bias": dict(type_id=(17, 0), num_unitcells=12, num_modes=3, contact_mu=(0.0, -0.4), contact_T=(300.0, 300.0),
                 noneq_integration_pts=(40, 60), noneq_percent_intercuts=(40.0,), E_zPlus_imag=1e-6),
    # zero bias: flat-band GL DOS path, 3 unit cells (a partial 8-site segment)
    "zero_bias": dict(type_id=(17, 0), num_unitcells=3, num_modes=2, contact_mu=(-1.0, -1.0),
                      contact_T=(300.0, 300.0), flatband_dos_integration_pts=64),
    # decimation leads, unequal temperatures, uniform real-axis window
    "decimation": dict(type_id=(17, 0), num_unitcells=5, num_modes=2, contact_mu=(-0.1, -0.3),
                       contact_T=(300.0, 350.0), use_decimation=1, realaxis_window=(-1.2, 0.8, 96, 0),
                       E_zPlus_imag=1e-5),
    # chiral tube with 4 modes, long enough for several pass-2 units
    "chiral_long": dict(type_id=(13, 0), num_unitcells=90, num_modes=4, contact_mu=(0.1, -0.3),
                        contact_T=(300.0, 300.0), noneq_integration_pts=(80,), E_zPlus_imag=1e-5),
}


@pytest.mark.parametrize("case", sorted(TRANSPORT_CASES))
def test_dos_against_oracle(oracle, case):
    kw = TRANSPORT_CASES[case]
    okw = {k: v for k, v in kw.items() if k != "flatband_dos_integration_pts"}
    g, o = _pair(oracle, seed=11, **okw)
    if "flatband_dos_integration_pts" in kw:
        from electrostatic_b200.negf import CNT
        g = CNT(**kw)
        U = np.zeros(g.num_field_sites)
        g.set_potential(U, (0.0, 0.0))
        o.set_potential(U, (0.0, 0.0))
        od = o.dos(faithful=True, nthreads=8, ldos=True, flatband_pts=kw["flatband_dos_integration_pts"])
    else:
        od = o.dos(faithful=True, nthreads=8, ldos=True)
    d = g.Compute_DensityOfStates(ldos=True)
    assert len(d["E"]) == len(od["E"])
    assert np.max(np.abs(d["E"] - od["E"])) < 1e-12
    for key in ("dos", "T", "conductance"):
        assert _rel(d[key], od[key]) <= TOL, key
    assert _rel(d["ldos"], od["ldos"]) <= TOL
    assert abs(d["total_conductance"] - od["total_conductance"]) <= TOL * max(1.0, abs(od["total_conductance"]))
    if case == "zero_bias":
        # flat band: the transmission plateaus at the open-channel count (2 modes, degeneracy 2)
        assert set(np.round(d["T"][d["T"] > 0.5]).astype(int)) <= {2, 4}


@pytest.mark.parametrize("case", ["bias", "decimation", "chiral_long"])
def test_current_against_oracle(oracle, case):
    kw = TRANSPORT_CASES[case]
    g, o = _pair(oracle, seed=12, **kw)
    I, probes, E = g.Compute_Current(integrand=True)
    oI, oprobes = o.current(nthreads=8, probes=True)
    assert np.all(np.abs(I - oI) <= TOL * np.abs(oI).max())
    assert abs(I[0] + I[1]) <= 1e-6 * abs(I[0])  # current conservation
    assert _rel(probes, oprobes) <= TOL
    assert len(E) == probes.shape[1]


def test_current_zero_at_equilibrium():
    from electrostatic_b200.negf import CNT
    g = CNT(type_id=(17, 0), num_unitcells=4, num_modes=2, contact_mu=(-1.0, -1.0))
    g.set_potential(np.zeros(g.num_field_sites), (0.0, 0.0))
    assert np.all(g.Compute_Current() == 0.0)


def test_transport_writers(tmp_path):
    from electrostatic_b200.negf import CNT, write_current, write_current_header
    g = CNT(**TRANSPORT_CASES["bias"])
    g.set_potential(np.zeros(g.num_field_sites), (0.0, 0.0))
    d = g.Compute_DensityOfStates()
    I, probes, E = g.Compute_Current(integrand=True)
    tc = str(tmp_path / "transport_char.dat")
    g.Write_Eql_Characteristics(tc, d)
    lines = open(tc).read().splitlines()
    assert lines[0] == " E_r, Fermi_Contact1, Fermi_Contact2, DOS_r, Transmission_r, Conductance_r "
    assert len(lines) == len(d["E"]) + 1
    row = np.array(lines[1].split(), dtype=float)
    assert row.shape == (6,) and abs(row[4] - d["T"][0]) <= 1e-5 * abs(d["T"][0])
    Ipath = str(tmp_path / "I.dat")
    write_current_header(Ipath)
    write_current(Ipath, 1, 0.4, 0.1, I, 100.0, 12, d["total_conductance"])
    il = open(Ipath).read().splitlines()
    assert il[0].startswith("'step', 'Vds' , 'Vgs', , 'I at contact_1',, 'I at contact_2','Avg_intg_pts'")
    vals = il[1].split()
    assert len(vals) == 8 and int(vals[0]) == 1 and abs(float(vals[3]) - I[0]) <= 1e-5 * abs(I[0])
    ip = str(tmp_path / "step0001_integrand.dat")
    g.Write_Integrand(ip, E, probes)
    rows = np.loadtxt(ip, skiprows=1)
    assert rows.shape == (len(E), 6)
    assert np.allclose(rows[:, 1], probes[0], rtol=1e-14, atol=0)


@pytest.mark.parametrize("paths", [2, 3])
def test_adaptive_intercuts_against_oracle(oracle, paths):
    """Update_IntegrationPaths with flag_correct_integration_limits: the
    charge integrand (sites N/2, N/4, 3N/4), E* and the corrected intercuts
    and point counts match the oracle over two corrections, then the charge."""
    pts, cuts = ((30, 50), (40.0,)) if paths == 2 else ((20, 40, 20), (30.0, 70.0))
    kw = dict(type_id=(17, 0), num_unitcells=12, num_modes=2, contact_mu=(0.0, -0.4), contact_T=(300.0, 300.0),
              noneq_integration_pts=pts, noneq_percent_intercuts=cuts, E_zPlus_imag=1e-6)
    g, o = _pair(oracle, seed=21, **kw)
    assert _rel(g.noneq_integrand(), o.noneq_integrand(nthreads=8)) <= TOL
    for _ in range(2):
        g.correct_integration_limits()
        o.correct_limits(nthreads=8)
        gp, gc, gE = g.noneq_layout()
        op, oc, oE = o.noneq_layout()
        assert list(gp) == list(op) and gE == oE
        assert np.allclose(gc, oc, rtol=0, atol=1e-9)
    assert _rel(g.Solve_NEGF(), o.charge(nthreads=8)) <= TOL


def test_solve_negf_adaptive_schedule():
    """Solve_NEGF(iter) corrects only on multiples of the interval."""
    from electrostatic_b200.negf import CNT
    g = CNT(type_id=(17, 0), num_unitcells=8, num_modes=2, contact_mu=(0.0, -0.4), noneq_integration_pts=(20, 40, 20),
            noneq_percent_intercuts=(30.0, 70.0), flag_adaptive_integration_limits=1, integrand_correction_interval=3)
    g.set_potential(np.zeros(g.num_field_sites), (0.0, 0.0))
    g.Solve_NEGF(iter=1)
    assert list(g.noneq_layout()[0]) == [20, 40, 20]
    g.Solve_NEGF(iter=3)
    assert list(g.noneq_layout()[0]) != [20, 40, 20]
