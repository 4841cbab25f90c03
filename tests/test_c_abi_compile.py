"""The C-ABI from a C and a C++ compiler, host only.

A caller of the boundary is compiled code (the reference is C++), so the
header must compile as strict C99 and as C++17 with warnings as errors, the
library must link from plain C, and the struct layouts that the C compiler
sees must be the ones the ctypes mirror (electrostatic_b200._lib) assumes.
The C program below prints sizeof/offsetof of every field of negf_tube_desc
and negf_stats and runs the calls that need no device (descriptor defaults,
the energy-point tables of a descriptor, shard ranges, an argument error);
its output must equal the same calls made through ctypes.  Without a GPU,
negf_tube_create must fail with NEGF_ERR_CUDA rather than crash.
"""
import ctypes as C
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")


def _program(desc_fields, stats_fields):
    lines = [
        "#include <stddef.h>",
        "#include <stdio.h>",
        "#include <stdlib.h>",
        '#include "negf_b200.h"',
        "",
        "int main(void) {",
        "    negf_tube_desc d;",
        "    double* buf;",
        "    int count = 0, lo = 0, hi = 0, rc, k;",
        "    negf_tube* t = NULL;",
        '    printf("sizeof desc %d\\n", (int)sizeof(negf_tube_desc));',
        '    printf("sizeof stats %d\\n", (int)sizeof(negf_stats));',
    ]
    for f in desc_fields:
        lines.append(f'    printf("desc {f} %d\\n", (int)offsetof(negf_tube_desc, {f}));')
    for f in stats_fields:
        lines.append(f'    printf("stats {f} %d\\n", (int)offsetof(negf_stats, {f}));')
    lines += [
        "    if (negf_tube_desc_init(&d) != NEGF_OK) return 10;",
        '    printf("default %d %d %d %.17g %.17g %.17g\\n", d.type_id[0], d.type_id[1], d.eq_integration_pts[2],',
        "           d.gamma, d.E_zPlus_imag, d.E_valence_min);",
        "    d.num_unitcells = 10;",
        "    d.num_modes = 2;",
        "    d.contact_mu[0] = 0.0;",
        "    d.contact_mu[1] = -0.3;",
        "    for (k = 0; k <= 3; ++k) {",
        "        if (negf_desc_energy_points(&d, k, NULL, &count) != NEGF_OK) return 11;",
        "        buf = (double*)malloc(sizeof(double) * 6 * (size_t)(count > 0 ? count : 1));",
        "        if (!buf || negf_desc_energy_points(&d, k, buf, &count) != NEGF_OK) return 12;",
        '        printf("points %d %d %.17g %.17g %.17g\\n", k, count, count ? buf[0] : 0.0, count ? buf[1] : 0.0,',
        "               count ? buf[6 * (count - 1) + 2] : 0.0);",
        "        free(buf);",
        "    }",
        "    if (negf_shard_range(100, 1, 4, &lo, &hi) != NEGF_OK) return 13;",
        '    printf("shard %d %d\\n", lo, hi);',
        "    rc = negf_shard_range(10, 3, 2, &lo, &hi);",
        '    printf("bad_shard %d\\n", rc);',
        "    rc = negf_tube_create(&d, &t);",
        '    printf("create %d\\n", rc);',
        "    if (rc == NEGF_OK) negf_tube_destroy(t);",
        "    return 0;",
        "}",
    ]
    return "\n".join(lines) + "\n"


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(shutil.which("gcc") is None or shutil.which("g++") is None, reason="needs gcc and g++")
def test_header_compiles_links_and_matches_ctypes_layout(negf_lib, tmp_path):
    from electrostatic_b200 import _lib
    desc_fields = [f for f, _ in _lib.TubeDesc._fields_]
    stats_fields = [f for f, _ in _lib.Stats._fields_]
    src = tmp_path / "abi.c"
    src.write_text(_program(desc_fields, stats_fields))
    libdir = os.path.dirname(_lib.LIB_PATH)
    exe = tmp_path / "abi"
    c_cmd = ["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I", INCLUDE, str(src),
             "-L", libdir, "-lnegf_b200", f"-Wl,-rpath,{libdir}", "-o", str(exe)]
    r = subprocess.run(c_cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    # the same file as C++ (extern "C" guards, no C-only constructs)
    r = subprocess.run(["g++", "-x", "c++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-I", INCLUDE, "-c",
                        str(src), "-o", str(tmp_path / "abi_cxx.o")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    out = {}
    for line in r.stdout.splitlines():
        parts = line.split()
        if parts[0] in ("sizeof", "desc", "stats", "points"):
            out[" ".join(parts[:2])] = parts[2:]
        else:
            out[parts[0]] = parts[1:]

    # layouts: the C compiler's view equals the ctypes mirror
    assert int(out["sizeof desc"][0]) == C.sizeof(_lib.TubeDesc)
    assert int(out["sizeof stats"][0]) == C.sizeof(_lib.Stats)
    for f in desc_fields:
        assert int(out[f"desc {f}"][0]) == getattr(_lib.TubeDesc, f).offset, f
    for f in stats_fields:
        assert int(out[f"stats {f}"][0]) == getattr(_lib.Stats, f).offset, f

    # host-only calls: the C program and ctypes see the same library state
    d = _lib.TubeDesc()
    assert negf_lib.negf_tube_desc_init(C.byref(d)) == 0
    dflt = out["default"]
    assert [int(dflt[0]), int(dflt[1]), int(dflt[2])] == [d.type_id[0], d.type_id[1], d.eq_integration_pts[2]]
    assert [float(x) for x in dflt[3:6]] == [d.gamma, d.E_zPlus_imag, d.E_valence_min]
    d.num_unitcells, d.num_modes = 10, 2
    d.contact_mu[0], d.contact_mu[1] = 0.0, -0.3
    for k in range(4):
        n = C.c_int()
        assert negf_lib.negf_desc_energy_points(C.byref(d), k, None, C.byref(n)) == 0
        buf = (C.c_double * (6 * max(n.value, 1)))()
        assert negf_lib.negf_desc_energy_points(C.byref(d), k, buf, C.byref(n)) == 0
        got = out[f"points {k}"]
        assert int(got[0]) == n.value, k
        if n.value:
            assert float(got[1]) == buf[0] and float(got[2]) == buf[1], k
            assert float(got[3]) == buf[6 * (n.value - 1) + 2], k
    assert out["points 1"][0] != "0"  # the equilibrium contour is never empty
    lo, hi = C.c_int(), C.c_int()
    assert negf_lib.negf_shard_range(100, 1, 4, C.byref(lo), C.byref(hi)) == 0
    assert out["shard"] == [str(lo.value), str(hi.value)]
    assert out["bad_shard"] == ["-1"]  # NEGF_ERR_ARG
    if not _has_gpu():
        assert out["create"] == ["-2"]  # NEGF_ERR_CUDA, no CPU fallback
