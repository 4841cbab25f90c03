"""C-ABI library checks that need no GPU: every declared symbol is exported,
compute calls fail loudly without a device, and the host-side path logic
(energy limits, Gauss-Legendre paths, poles, real-axis windows, shards)
matches the oracle's restatement of the reference."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    src = open(os.path.join(ROOT, "include", "negf_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(negf_\w+)\s*\(", src, flags=re.M)))


def test_every_declared_symbol_is_exported(negf_lib):
    from electrostatic_b200 import _lib
    decl = _declared_functions()
    assert len(decl) >= 25
    assert sorted(_lib.EXPORTED) == decl
    for name in decl:
        assert hasattr(negf_lib, name), name


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device error path")
def test_compute_fails_loudly_without_device(negf_lib):
    from electrostatic_b200 import _lib
    d = _lib.TubeDesc()
    assert negf_lib.negf_tube_desc_init(C.byref(d)) == 0
    h = C.c_void_p()
    rc = negf_lib.negf_tube_create(C.byref(d), C.byref(h))
    assert rc == -2  # NEGF_ERR_CUDA
    assert b"CUDA" in negf_lib.negf_last_error() or b"device" in negf_lib.negf_last_error()
    b = C.c_void_p()
    assert negf_lib.negf_broyden_create(10, 20, 0.1, 0, C.byref(b)) == -2
    assert negf_lib.negf_release_scratch(None) == -2


def test_argument_errors(negf_lib):
    from electrostatic_b200 import _lib
    d = _lib.TubeDesc()
    negf_lib.negf_tube_desc_init(C.byref(d))
    d.num_noneq_paths = 0
    h = C.c_void_p()
    assert negf_lib.negf_tube_create(C.byref(d), C.byref(h)) == -1
    assert b"num_noneq_paths" in negf_lib.negf_last_error()
    lo, hi = C.c_int(), C.c_int()
    assert negf_lib.negf_shard_range(10, 3, 2, C.byref(lo), C.byref(hi)) == -1
    # argument checks that run before any device work (through the declared ctypes signatures)
    null1 = (C.c_void_p * 1)(None)
    zero1 = (C.c_int * 1)(0)
    assert negf_lib.negf_potential_batch_create(0, null1, zero1, null1, null1, null1, null1, zero1, C.byref(h)) == -1
    assert negf_lib.negf_affine_potential_toeplitz(None, 0, None, None, None, None, 0, None, None) == -1
    assert negf_lib.negf_broyden_set_segments(None, 2, None, None) == -1


def test_shard_ranges_partition(negf_lib):
    for P in (0, 1, 7, 100, 4096):
        for W in (1, 2, 3, 8):
            covered = []
            for r in range(W):
                lo, hi = C.c_int(), C.c_int()
                assert negf_lib.negf_shard_range(P, r, W, C.byref(lo), C.byref(hi)) == 0
                covered += list(range(lo.value, hi.value))
                assert hi.value - lo.value in (P // W, P // W + 1)
            assert covered == list(range(P))


def _desc(**kw):
    from electrostatic_b200 import _lib
    d = _lib.TubeDesc()
    _lib.load().negf_tube_desc_init(C.byref(d))
    for k, v in kw.items():
        if isinstance(v, (list, tuple)):
            arr = getattr(d, k)
            for i, x in enumerate(v):
                arr[i] = x
        else:
            setattr(d, k, v)
    return d


def _lib_points(d, kind):
    from electrostatic_b200 import _lib
    L = _lib.load()
    n = C.c_int()
    assert L.negf_desc_energy_points(C.byref(d), kind, None, C.byref(n)) == 0
    buf = np.zeros(6 * max(1, n.value))
    assert L.negf_desc_energy_points(C.byref(d), kind, buf.ctypes.data_as(C.POINTER(C.c_double)), C.byref(n)) == 0
    b = buf[: 6 * n.value].reshape(-1, 6)
    return b[:, 0] + 1j * b[:, 1], b[:, 2] + 1j * b[:, 3], b[:, 4] + 1j * b[:, 5]


CASES = [
    dict(name="equilibrium", mu=(0.0, 0.0), T=(298.0, 298.0), eq=(30, 30, 30), ne=(100,), cuts=None, win=None),
    dict(name="equilibrium_Ef", mu=(-1.0, -1.0), T=(300.0, 300.0), eq=(32, 32, 32), ne=(100,), cuts=None, win=None),
    dict(name="bias", mu=(0.0, -0.4), T=(300.0, 300.0), eq=(24, 24, 40), ne=(60,), cuts=None, win=None),
    dict(name="bias_3paths", mu=(0.1, -0.3), T=(298.0, 298.0), eq=(10, 20, 30), ne=(20, 40, 20), cuts=(30.0, 60.0),
         win=None),
    dict(name="bias_3paths_uniform", mu=(0.1, -0.3), T=(298.0, 298.0), eq=(10, 20, 30), ne=(20, 40, 20), cuts=None,
         win=None),
    dict(name="temperature", mu=(0.0, 0.0), T=(300.0, 500.0), eq=(16, 16, 16), ne=(50,), cuts=None, win=None),
    dict(name="window_regular", mu=(0.0, -0.5), T=(300.0, 300.0), eq=(256, 256, 512), ne=(100,), cuts=None,
         win=(-1.5, 1.5, 3072, 0)),
    dict(name="window_gl", mu=(-1.0, -1.0), T=(300.0, 300.0), eq=(64, 32, 32), ne=(100,), cuts=None,
         win=(-1.3, -0.7, 256, 1)),
]


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_paths_match_oracle(oracle, case):
    kw = dict(contact_mu=case["mu"], contact_T=case["T"], eq_integration_pts=case["eq"],
              num_noneq_paths=len(case["ne"]), noneq_integration_pts=case["ne"], E_zPlus_imag=1e-8)
    if case["cuts"] is not None:
        kw["noneq_percent_intercuts"] = case["cuts"]
    if case["win"] is not None:
        lo, hi, pts, kind = case["win"]
        kw.update(realaxis_min=lo, realaxis_max=hi, realaxis_pts=pts, realaxis_kind=kind, E_zPlus_imag=1e-4)
    d = _desc(**kw)
    t = oracle.OracleTube(num_unitcells=2, contact_mu=case["mu"], contact_T=case["T"],
                          eq_integration_pts=case["eq"], noneq_integration_pts=case["ne"],
                          noneq_percent_intercuts=case["cuts"], E_zPlus_imag=kw["E_zPlus_imag"],
                          realaxis_window=case["win"])
    for kind in (0, 1, 2, 3):
        E, w, J = _lib_points(d, kind)
        Eo, wo, Jo = t.paths(kind)
        assert len(E) == len(Eo), (kind, len(E), len(Eo))
        np.testing.assert_allclose(E, Eo, rtol=1e-13, atol=1e-13)
        np.testing.assert_allclose(w, wo, rtol=1e-13, atol=1e-15)
        np.testing.assert_allclose(J, Jo, rtol=1e-13, atol=1e-15)


def test_poles_count_equilibrium():
    d = _desc(contact_mu=(0.0, 0.0), contact_T=(298.0, 298.0), E_pole_max=3.0)
    E, _, _ = _lib_points(d, 2)
    kT = 8.617333262e-5 * 298.0
    assert len(E) == int((3.0 - np.pi * kT) / (2 * np.pi * kT) + 1) == 19
    np.testing.assert_allclose(E.imag, np.pi * kT * (2 * np.arange(len(E)) + 1))


def test_read_table1d(negf_lib, tmp_path):
    """Read_Table1D restated: header + n lines, size assertion, missing file."""
    from electrostatic_b200 import negf
    from electrostatic_b200._lib import NEGFError
    p = tmp_path / "step0003_Qout.dat"
    vals = np.linspace(-1e-3, 2e-3, 7)
    with open(p, "w") as f:
        f.write("'axial location / (nm)', 'Induced charge per site / (e)'\n")
        for i, v in enumerate(vals):
            f.write("%35.15g%35.15g\n" % (0.1 * i, v))
    assert np.array_equal(negf.read_table1d(str(p), 7), vals)
    with pytest.raises(NEGFError, match="Assert size, 8, is not equal to the filesize-1, 7 !"):
        negf.read_table1d(str(p), 8)
    with pytest.raises(NEGFError, match="Failed to read file"):
        negf.read_table1d(str(tmp_path / "missing.dat"), 7)
    assert negf.restart_charge_filename("output/negf", "cnt", 4) == "output/negf/cnt/step0003_Qout.dat"
    assert negf.iter_filename(negf.step_filename("out", "cnt", 1), 12) == "out/cnt/step0001_iter/iter0012"
