"""Seeded synthetic workloads of the benchmark configurations.

No dataset is involved: every input is drawn from numpy's generator seeded
with 20261203 + config id.  Shapes follow the configurations the engine is
measured on:

* uneven multi-tube batch (config id 4): 16 tubes of chirality (13,0),
  (17,0) or (19,0) drawn uniformly, length log-uniform in [200, 2000] unit
  cells, 2-10 modes (at most the m//2 + 1 distinct modes of (m,0)), log-uniform 512-8192 energy points per tube
  (equilibrium contour 1/8 + 1/8 + 1/4 of them, the rest on three real-axis
  paths), Vds = 0.4 V (contact mu 0 and -0.4 eV), 300 K, mixed precision,
  real-axis broadening E_zPlus_imag = 2 meV (with these point counts a
  smaller broadening leaves the resonances of the longer tubes unresolved
  and the biased self-consistency does not settle at 1e-6);
  each tube inside its own gate-all-around stand-in (gate radius R + 1.5 nm,
  permittivity 3.9, source/drain electrodes over the first and last
  min(5 nm, L/10)); gate swept 0 -> 0.6 V in 0.05 V steps.
"""
from __future__ import annotations

import numpy as np

SEED_BASE = 20261203


def site_potential(y_nm, seed, amp=0.4, ramp=0.5):
    """Seeded sum of 5 Gaussian bumps (amplitude U(-amp, amp) V, width
    U(2, 10) nm, centre U(0, L)) plus a linear ramp 0 -> ramp, as U in eV."""
    rng = np.random.default_rng(seed)
    y_nm = np.asarray(y_nm, dtype=np.float64)
    L = y_nm[-1] - y_nm[0]
    U = np.zeros_like(y_nm)
    for _ in range(5):
        A = rng.uniform(-amp, amp)
        w = rng.uniform(2.0, 10.0)
        c = rng.uniform(0.0, L)
        U += A * np.exp(-((y_nm - y_nm[0] - c) ** 2) / (2 * w * w))
    return U + ramp * (y_nm - y_nm[0]) / L


def uneven_batch(num_tubes=16, precision="mixed", vds=0.4, seed=SEED_BASE + 4, scale=1.0, realaxis_fp32=False):
    """Tube descriptors (CNT keyword dicts) of the uneven batch; `scale`
    shrinks lengths and energy counts for tests (1.0 = the benchmark);
    realaxis_fp32: mixed mode also runs the real-axis chains (broadening
    2 meV, above the 1 meV FP64 band) in FP32."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(num_tubes):
        m = int(rng.choice([13, 17, 19]))
        uc = int(round(np.exp(rng.uniform(np.log(200), np.log(2000)))))
        M = min(int(rng.integers(2, 11)), m // 2 + 1)  # (m,0) has m//2 + 1 distinct modes
        E = int(round(np.exp(rng.uniform(np.log(512), np.log(8192)))))
        uc = max(2, int(round(uc * scale)))
        E = max(16, int(round(E * scale)))
        eq = (max(2, E // 8), max(2, E // 8), max(2, E // 4))
        ne_total = max(6, E - sum(eq))
        ne = (ne_total // 4, ne_total // 2, ne_total - ne_total // 4 - ne_total // 2)
        out.append(dict(type_id=(m, 0), num_unitcells=uc, num_modes=M, contact_mu=(0.0, -float(vds)),
                        contact_T=(300.0, 300.0), eq_integration_pts=eq, noneq_integration_pts=ne,
                        noneq_percent_intercuts=(30.0, 70.0), E_zPlus_imag=2e-3, precision=precision,
                        mixed_realaxis_fp32=bool(realaxis_fp32)))
    return out


GATE_SWEEP = [round(0.05 * i, 2) for i in range(13)]  # 0 -> 0.6 V


def config2_kwargs(precision="fp64", small=False):
    """Batched mode-space benchmark tube (config id 2): (17,0), 1000 unit
    cells (N = 4000), 8 modes, 1024 equilibrium-contour points (256 + 256
    line, 512 arc) + 3072 real-axis points uniform on [-1.5, 1.5] eV with
    eta = 1e-4 eV, contacts mu = (0, -0.5) eV at 300 K.  small: a quarter of
    the energies (the profiling case)."""
    eq, rt = ((64, 64, 128), 768) if small else ((256, 256, 512), 3072)
    return dict(type_id=(17, 0), num_unitcells=1000, num_modes=8, contact_mu=(0.0, -0.5), contact_T=(300.0, 300.0),
                eq_integration_pts=eq, E_zPlus_imag=1e-4, realaxis_window=(-1.5, 1.5, rt, 0), precision=precision)


def config3_kwargs(precision="fp64", small=False):
    """Real-space benchmark tube (config id 3): (13,0), 300 unit cells = 600
    ring blocks of 26 atoms, 2048 equilibrium-contour points (512 + 512
    line, 1024 arc) plus the Matsubara poles up to 3 eV, mu = -0.8 eV at
    300 K; the leads' exact surface Green's function (what Sancho-Rubio
    decimation of the 26-atom lead cell converges to).  small: 200 blocks and
    256 contour points (the profiling case)."""
    return dict(type_id=(13, 0), num_unitcells=100 if small else 300, num_modes=7, contact_mu=(-0.8, -0.8),
                contact_T=(300.0, 300.0), eq_integration_pts=(64, 64, 128) if small else (512, 512, 1024),
                E_pole_max=3.0, E_zPlus_imag=1e-6, precision=precision)


def gate_with_contacts(y_nm, r_tube, vds=0.4, gate_gap=1.5e-9, contact_nm=5.0):
    """Gate-all-around stand-in of a batch tube: gate radius r_tube + 1.5 nm,
    source (0 V) and drain (Vds) electrodes over the first and last
    min(5 nm, L/10) of the tube."""
    from .electrostatics import GateAllAround
    y = np.asarray(y_nm)
    Lc = min(contact_nm, 0.1 * (y.max() - y.min())) * 1e-9
    return GateAllAround(y, r_tube, r_tube + gate_gap, contact_length=Lc, Vds=vds)
