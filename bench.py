"""Benchmark: site*energy RGF updates/s of the NEGF induced-charge pass.

Workload (one step = one full induced-charge pass over resident inputs):
  (17,0) CNT, 1000 unit cells -> N = 4000 sites, M = 8 lowest distinct modes,
  E = 4096 energies = 1024 equilibrium-contour points (Gauss-Legendre 256 + 256
  line, 512 arc) + 3072 real-axis points uniform on [-1.5, 1.5] eV with
  eta = 1e-4 eV; contacts mu = (0, -0.5) eV at 300 K; site potential = seeded
  sum of 5 Gaussian bumps (amplitude U(-0.4, 0.4) V, width U(2, 10) nm) plus a
  0-0.5 V linear ramp.  Updates per pass = N * M * E = 131,072,000.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--precision fp64|mixed]

Multi-GPU (torchrun, one rank per GPU): the ranks split the one tube's energy
points into contiguous shards (negf_tube_set_energy_shard; Rho0 subtracted on
rank 0 only) and sum their partial site charges with one NCCL all-reduce of
N doubles per pass, inside the timed region: the total work is fixed as the
GPU count grows (strong scaling).  The step time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_UNITCELLS = 1000
N_MODES = 8
EQ_PTS = (256, 256, 512)
RT_PTS = 3072
ETA = 1e-4
MU = (0.0, -0.5)
TEMP = (300.0, 300.0)
SEED = 20261203 + 2
FLOP_CONTOUR = 53  # per contour update: forward 15 + backward 15 + G_nn 15 + accumulate 8
FLOP_REALAXIS = 76  # + two running products 12, two |G|^2 Gamma f terms 8, accumulate 3
MIXED_RULE = ("FP32 recursions for contour/pole chains at least 1e-3 eV above the real axis (Kahan FP64 "
              "sums); real-axis chains, chains within 1e-3 eV of a lead band edge, leads and Rho0 in FP64")
WORKLOAD = (f"mode-space RGF induced-charge pass: (17,0) CNT N={4 * N_UNITCELLS} sites, M={N_MODES} modes, "
            f"E={sum(EQ_PTS) + RT_PTS} energies ({sum(EQ_PTS)} contour GL + {RT_PTS} real-axis uniform on "
            f"[-1.5,1.5] eV, eta={ETA} eV), mu=(0,-0.5) eV, 300 K")


def tube_kwargs(precision="fp64"):
    from electrostatic_b200.workloads import config2_kwargs
    kw = config2_kwargs(precision, small=RT_PTS != 3072)
    assert kw["num_unitcells"] == N_UNITCELLS and kw["num_modes"] == N_MODES and kw["eq_integration_pts"] == EQ_PTS
    return kw


def site_potential(y_nm, seed):
    """Seeded sum of 5 Gaussian bumps + linear ramp 0-0.5 V (as U in eV = -phi)."""
    from electrostatic_b200.workloads import site_potential as sp
    return sp(y_nm, seed)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def wait_first(self, timeout=5.0):
        t0 = time.time()
        while self.proc and not self.rows and time.time() - t0 < timeout:
            time.sleep(0.02)

    def mark(self):
        return len(self.rows)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self, lo=0, hi=None):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows[lo:hi]:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except Exception:
                continue
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_fp64_peak(torch):
    """FP64 throughput of a cuBLAS DGEMM (8192^3, best of 5) on this GPU [TFLOP/s]."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.mm(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.mm(a, b)
        e.record()
        e.synchronize()
        best = max(best, 2 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def load_profile_traffic(name):
    p = os.path.join(ROOT, "profiles", name)
    if os.path.exists(p):
        try:
            return json.load(open(p))
        except Exception:
            return None
    return None


def run_reference_arm(args, rank, world):
    """Reference arm: the reference path's CPU implementation (oracle port,
    faithful walk) on the host cores, each step a bounded strided sample."""
    if rank != 0:
        return
    from oracle import oracle as O
    O.build()
    kw = tube_kwargs()
    kw.pop("precision")
    t = O.OracleTube(**kw)
    y = ring_positions_nm(N_UNITCELLS)
    U = site_potential(y, SEED)
    t.set_potential(U, (U[0], U[-1]))
    threads = len(os.sched_getaffinity(0))
    # 8 energy points per step (about 1 s on 16 threads) for short runs; for
    # many steps fewer points per step keep the whole run within minutes
    stride = 512 if args.steps <= 20 else (1024 if args.steps <= 60 else 4096)
    # offsets hop by 1031 (coprime to 4096): the samples mix contour and real-axis points as the grid does
    for i in range(args.warmup):
        t.sample(stride, (i * 1031) % stride, faithful=True, nthreads=threads)
    tot_upd, tot_t = 0, 0.0
    for i in range(args.steps):
        t0 = time.perf_counter()
        _, n = t.sample(stride, ((args.warmup + i) * 1031) % stride, faithful=True, nthreads=threads)
        tot_t += time.perf_counter() - t0
        tot_upd += n
    v = tot_upd / tot_t
    sample = (f"every {stride}th of the 4096 energy points per step ({4096 // stride} point(s), offsets rotating "
              f"over contour and real-axis points, all 8 modes, N=4000), faithful O(N)-per-site contact walk as in "
              f"NEGF_Common.cpp:3418-3426")
    line = {"impl": "reference", "metric": "site*energy RGF updates/s", "value": v, "unit": "updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "precision": "fp64", "implementation": "oracle port of the reference "
                       "CPU path (reference not buildable here: AMReX and MPI absent)"},
            "cpu_baseline": {"value": v, "unit": "updates/s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


SCF_KW = dict(type_id=(17, 0), num_unitcells=100, num_modes=2, contact_mu=(-1.0, -1.0), contact_T=(300.0, 300.0),
              eq_integration_pts=(32, 32, 32), E_valence_min=-10.0, E_pole_max=3.0)
SCF_VG = [0.0, 0.1, 0.2, 0.3]
SCF_WORKLOAD = ("config-1 self-consistent sweep: (17,0) CNT N=400, M=2, mu=(-1,-1) eV, 300 K, contour 32+32+32 "
                "GL + Matsubara poles (E_pole_max 3 eV), gate-all-around stand-in (gate radius R+1.5 nm, eps 3.9), "
                "Vg 0..0.3 V step 0.1, Broyden alpha=0.1 to 1e-6 absolute max-norm")


def scf_measure(threads):
    """Config-1 SCF sweep: device loop (FP64) vs the same loop on the CPU oracle."""
    from electrostatic_b200.electrostatics import GateAllAround
    from electrostatic_b200.negf import CNT
    from electrostatic_b200.scf import run_scf, run_scf_batch
    from oracle.scf_oracle import run_scf_oracle
    from oracle import oracle as O
    tube = CNT(**SCF_KW)
    y = tube.site_positions()
    ot = O.OracleTube(**SCF_KW)
    ga = GateAllAround(y, ot.radius, ot.radius + 1.5e-9)
    run_scf(tube, ga, [0.0])  # warm-up (tables, caches)
    rg = run_scf(tube, ga, SCF_VG)
    rgraph = run_scf_batch([tube], [ga], SCF_VG, use_graph=True, iters_per_graph=8, autotune=False)
    ro = run_scf_oracle(ot, ga.K, SCF_VG, nthreads=threads)
    dq = max(float(np.max(np.abs(a.Q - b.Q))) for a, b in zip(rg.steps, ro.steps))
    return {"workload": SCF_WORKLOAD, "gpu_seconds": rg.seconds, "gpu_iterations": [s.iterations for s in rg.steps],
            "cpu_seconds": ro.seconds, "cpu_iterations": [s.iterations for s in ro.steps], "cpu_cores": threads,
            "cpu_kind": "port (oracle, O(N) walk; the reference path at Vds=0 has no real-axis walk)",
            "max_abs_dQ_gpu_vs_cpu": dq, "speedup": ro.seconds / rg.seconds,
            "gpu_graph_seconds": rgraph.seconds, "gpu_graph_iterations": [s.iterations for s in rgraph.steps],
            "graph_speedup_vs_cpu": ro.seconds / rgraph.seconds,
            "max_abs_dQ_graph_vs_loop": max(float(np.max(np.abs(a.Q - b.Q))) for a, b in zip(rgraph.steps, rg.steps))}


def config4_measure(torch, passes=5):
    """Uneven 16-tube batch (seeded): batched charge pass (autotuned plan)
    throughput and the self-consistent gate sweep replayed as CUDA graphs,
    in mixed precision (FP32 contour chains; and with the real-axis chains
    at 2 meV broadening in FP32 too) and in FP64."""
    from electrostatic_b200.electrostatics import GateAllAround
    from electrostatic_b200.negf import CNT, ChargePlan
    from electrostatic_b200.scf import run_scf_batch
    from electrostatic_b200.workloads import GATE_SWEEP, SEED_BASE, gate_with_contacts, site_potential, uneven_batch
    out = {"workload": "16 tubes (13,0)/(17,0)/(19,0), 200-2000 unit cells, 2-10 modes, 512-8192 energies each, "
                       "Vds 0.4 V, 300 K; gate-all-around stand-in per tube with source/drain electrodes over the first/last "
                       "min(5 nm, L/10); Vg 0..0.6 V step 0.05, "
                       "Broyden alpha 0.1 to 1e-6 absolute max-norm; seeded (%d)" % (SEED_BASE + 4)}
    electros = None
    Qs = {}
    for prec in ("mixed", "mixed_realaxis_fp32", "fp64"):
        descs = uneven_batch(precision="fp64" if prec == "fp64" else "mixed",
                             realaxis_fp32=prec == "mixed_realaxis_fp32")
        tubes = [CNT(**d) for d in descs]
        if electros is None:
            electros = []
            for d, t in zip(descs, tubes):
                R = 1.42e-10 * np.sqrt(3.0) * d["type_id"][0] / (2 * np.pi)  # CNT.cpp:23-41
                electros.append(gate_with_contacts(t.site_positions(), R))
        for i, t in enumerate(tubes):
            U = site_potential(t.site_positions(), SEED_BASE + 4 + 100 * i)
            t.set_potential(U, (U[0], U[-1]))
        S = sum(t.num_field_sites for t in tubes)
        Q = torch.zeros(S, dtype=torch.float64, device="cuda")
        plan = ChargePlan(tubes, Q, autotune=True)
        info = plan.info()
        for _ in range(2):
            plan.launch()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(passes):
            plan.launch(stream=torch.cuda.current_stream())
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / passes
        plan.close()
        entry = {"updates_per_pass": info["updates"], "ms_per_pass": ms, "updates_per_s": info["updates"] / (ms * 1e-3),
                 "schedule": {"pass2_warps_per_block": info["pass2_warps_per_block"],
                              "segs_per_unit": info["segs_per_unit"]}}
        try:
            sw = 1e-4 if prec != "fp64" else None
            r = run_scf_batch(tubes, electros, GATE_SWEEP, use_graph=True, iters_per_graph=4, switch_norm=sw)
            entry.update({"scf_seconds": r.seconds, "scf_iterations": [s.iterations for s in r.steps]})
            if sw:
                entry["switch_norm"] = sw
                entry["scf_lowprec_iterations"] = [s.lowprec_iterations for s in r.steps]
            Qs[prec] = [s.Q for s in r.steps]
        except RuntimeError as e:
            entry["scf_error"] = str(e)
        out[prec] = entry
        del tubes
    for name in ("mixed", "mixed_realaxis_fp32"):
        if name in Qs and "fp64" in Qs:
            out[name + "_vs_fp64_rel"] = max(float(np.max(np.abs(a - b)) / np.max(np.abs(b)))
                                             for a, b in zip(Qs[name], Qs["fp64"]))
    return out


def config4_pass_only(prec, ntubes, passes, warmup, autotune=False):
    """Profiling case: the charge pass of the first ntubes tubes of the
    config-4 batch (seeded potentials as in config4_measure), one plan without
    autotuning, warm-up then CUDA-event timing; prints one JSON line with the
    error against the FP64 pass of the same potentials."""
    import torch
    from electrostatic_b200 import build
    from electrostatic_b200.negf import CNT, ChargePlan
    from electrostatic_b200.workloads import SEED_BASE, site_potential, uneven_batch
    build.build()

    def batch(p):
        descs = uneven_batch(precision="fp64" if p == "fp64" else "mixed",
                             realaxis_fp32=p == "mixed_realaxis_fp32")[:ntubes]
        tubes = [CNT(**d) for d in descs]
        for i, t in enumerate(tubes):
            U = site_potential(t.site_positions(), SEED_BASE + 4 + 100 * i)
            t.set_potential(U, (U[0], U[-1]))
        Q = torch.zeros(sum(t.num_field_sites for t in tubes), dtype=torch.float64, device="cuda")
        return tubes, Q, ChargePlan(tubes, Q, autotune=autotune and p == prec)

    tubes, Q, plan = batch(prec)
    s = torch.cuda.current_stream()
    for _ in range(max(1, warmup)):
        plan.launch(stream=s)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(passes):
        plan.launch(stream=s)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / passes
    info = plan.info()
    out = {"config4_pass": prec, "tubes": ntubes, "autotune": bool(autotune), "ms_per_pass": ms,
           "updates": info["updates"], "updates_per_s": info["updates"] / (ms * 1e-3),
           "schedule": {"pass2_warps_per_block": info["pass2_warps_per_block"],
                        "segs_per_unit": info["segs_per_unit"], "tuned_ms": info["tuned_ms"]}}
    if prec != "fp64":
        t64, Q64, p64 = batch("fp64")
        p64.launch(stream=s)
        torch.cuda.synchronize()
        out["max_rel_vs_fp64"] = float((Q - Q64).abs().max() / Q64.abs().max())
        p64.close()
        for t in t64:
            t.close()
    plan.close()
    for t in tubes:
        t.close()
    print(json.dumps(out))


def surrogate_gemm_only(reps, warmup):
    """Profiling case: the BF16 GEMMs of one training step of the tube-set
    operator (batch 64 on the 7424-site canvas) through negf_nn_gemm, on the
    tcgen05 path (TMA-fed where the operands allow), the register-staged
    tcgen05 kernel and the mma.sync path; one JSON line per shape."""
    import ctypes as C
    import torch
    from electrostatic_b200 import _lib, build
    from electrostatic_b200.negf import TUNE_NN_GEMM, set_tuning
    build.build()
    L = _lib.load()
    vp = lambda t: C.c_void_p(t.data_ptr())
    R, S = 64 * 7424, 7424
    shapes = [("pointwise h W: R x 128 x 128", 0, 0, R, 128, 128, 1),
              ("spectral analysis F h: 64 x 128 x S, batch 64", 0, 0, 64, 128, S, 64),
              ("synthesis G z: S x 128 x 64, batch 64", 0, 0, S, 128, 64, 64),
              ("weight gradient h^T d: 128 x 128 x R", 1, 0, 128, 128, R, 1)]
    g = torch.Generator(device="cuda").manual_seed(0)
    for name, at, bt, M, N, K, batch in shapes:
        A = torch.randn(batch, *((K, M) if at else (M, K)), device="cuda", generator=g).to(torch.bfloat16)
        B = torch.randn(batch, *((N, K) if bt else (K, N)), device="cuda", generator=g).to(torch.bfloat16)
        Cm = torch.zeros(batch, M, N, device="cuda")
        lda, ldb = (M if at else K), (K if bt else N)
        res = {"shape": name}
        outs = []
        for path, key in ((1, "tcgen05"), (3, "tcgen05_staged"), (2, "mma_sync")):
            set_tuning(TUNE_NN_GEMM, path)

            def f():
                rc = L.negf_nn_gemm(at, bt, M, N, K, batch, vp(A), lda, A[0].numel(), vp(B), ldb, B[0].numel(),
                                    vp(Cm), N, M * N, None, 0, None)
                if rc != 0:
                    raise RuntimeError(L.negf_last_error().decode())

            for _ in range(max(1, warmup)):
                f()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            for _ in range(reps):
                f()
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / reps
            res[key] = {"ms": ms, "tflops": 2.0 * M * N * K * batch / ms / 1e9}
            outs.append(Cm.clone())
        set_tuning(TUNE_NN_GEMM, 0)
        res["max_abs_diff_paths"] = max(float((o - outs[0]).abs().max()) for o in outs[1:])
        print(json.dumps(res))


def config3_measure(torch, passes=2, small=False):
    """Real-space ring blocks: (13,0), 600 blocks of 26 atoms, 2048 contour
    energies + poles, FP64 and mixed; against the mode-space pass of the same
    tube with all 7 modes (equal for this ring-uniform potential).  small:
    the profiling case, 200 blocks and 256 contour energies."""
    from electrostatic_b200.negf import CNT, last_stats, set_timing
    from electrostatic_b200.workloads import SEED_BASE, config3_kwargs, site_potential
    kw = config3_kwargs(small=small)
    kw.pop("precision")
    t = CNT(**kw)
    U = site_potential(t.site_positions(), SEED_BASE + 3)
    t.set_potential(U, (U[0], U[-1]))
    Q = torch.zeros(t.num_field_sites, dtype=torch.float64, device="cuda")
    t.realspace_charge(out=Q)  # warm-up (buffers, lazy loading)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(passes):
        t.realspace_charge(out=Q)
    torch.cuda.synchronize()
    sec = (time.perf_counter() - t0) / passes
    Qm = t.Solve_NEGF()
    # mixed precision: FP32 chains with tensor-core products away from the real axis
    tm = CNT(**kw, precision="mixed")
    tm.set_potential(U, (U[0], U[-1]))
    Qx = torch.zeros_like(Q)
    tm.realspace_charge(out=Qx)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(passes):
        tm.realspace_charge(out=Qx)
    torch.cuda.synchronize()
    sec_mixed = (time.perf_counter() - t0) / passes
    Eall = np.concatenate([t.energy_points(1)[0], t.energy_points(2)[0]])
    n32 = int(np.sum(np.abs(Eall.imag) >= 1e-3))
    E = len(t.energy_points(1)[0]) + len(t.energy_points(2)[0])
    E0 = len(t.energy_points(0)[0])
    K, m = t.num_field_sites // 2, 13
    # ring-corner algorithm: one m x m inverse (8m^3) and three m x m complex
    # products (8m^3 each) per block update; the lead decimation (stopped at
    # convergence, data-dependent) is not counted
    flops = E * K * 32 * m ** 3  # timed passes: the tube's Rho0 comes from the warm-up call
    Qr = Q.cpu().numpy()
    return {"workload": "(13,0) CNT, %d blocks of 2 rings (26 atoms), %d contour+pole energies per pass (the "
                        "%d-energy Rho0 pass at U = 0 runs once per tube, in the warm-up call, as the mode-space "
                        "Rho0 does at tube creation), the leads' exact surface Green's function (ring Fourier modes, "
                        "analytic per mode; what Sancho-Rubio decimation of the lead cell converges to), FP64, "
                        "seeded config-2 ring potential" % (K, E, E0),
            "seconds_per_pass": sec, "block_updates_per_s": E * K / sec,
            "achieved_tflops": flops / sec / 1e12, "flops_per_pass": flops,
            "flop_convention": "ring corners m=13: inverse 8m^3 + three complex products 8m^3 per block update "
                               "(leads not counted)",
            "dense_convention": {"flops_per_pass": E * K * 56 * (2 * m) ** 3,
                                 "effective_tflops": E * K * 56 * (2 * m) ** 3 / sec / 1e12,
                                 "note": "the dense 2m x 2m block algorithm's count (56 n^3 per block update, n = 26: "
                                         "forward inverse + 2 GEMM, backward the same, G_nn inverse), which the "
                                         "ring-corner algebra replaces with 1/14 of the operations (32 m^3 per update)"},
            "path": "negf_rs_compute_charge (FP64 CUDA cores, one warp per energy, Schur complements on ring corners)",
            "max_rel_vs_mode_space_all_modes": float(np.max(np.abs(Qr - Qm)) / np.max(np.abs(Qm))),
            "mixed": {"seconds_per_pass": sec_mixed, "block_updates_per_s": E * K / sec_mixed,
                      "fp32_energies": n32, "fp64_energies": E - n32,
                      "path": "FP32 chains: TF32 tensor-core products (high/remainder split, 3 real products per "
                              "complex product), FP32 inversion; FP64 leads and near-axis chains",
                      "max_rel_vs_fp64": float(np.max(np.abs(Qx.cpu().numpy() - Qr)) / np.max(np.abs(Qr)))},
            "biased": config3_biased(torch, kw, U, passes)}


def config3_biased(torch, kw, U, passes):
    """The config-3 tube at a 0.3 V drain bias: the contour and poles of the
    lower contact plus the real-axis points of the non-equilibrium term
    (source and drain spectral functions carried through the ring-corner
    sweeps, FP64), against the mode-space pass with all 7 modes."""
    from electrostatic_b200.negf import CNT
    try:
        kb = dict(kw, contact_mu=(-0.8, -1.1), noneq_integration_pts=(3072,), E_zPlus_imag=1e-4)
        t = CNT(**kb)
        t.set_potential(U, (U[0], U[-1]))
        Q = torch.zeros(t.num_field_sites, dtype=torch.float64, device="cuda")
        t.realspace_charge(out=Q)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(passes):
            t.realspace_charge(out=Q)
        torch.cuda.synchronize()
        sec = (time.perf_counter() - t0) / passes
        Qm = t.Solve_NEGF()
        Qr = Q.cpu().numpy()
        ne = len(t.energy_points(3)[0])
        E = len(t.energy_points(1)[0]) + len(t.energy_points(2)[0])
        return {"workload": "(13,0) CNT, %d blocks, %d contour+pole and %d real-axis energies per pass, contact "
                            "potentials -0.8 / -1.1 eV, 1e-4 eV broadening, FP64" % (t.num_field_sites // 2, E, ne),
                "seconds_per_pass": sec,
                "max_rel_vs_mode_space_all_modes": float(np.max(np.abs(Qr - Qm)) / np.max(np.abs(Qm)))}
    except Exception as exc:  # reported, not fatal: the headline metric does not depend on it
        return {"error": str(exc)}


def long_tube_measure(torch, reps=10):
    """Parallel in length: a 64000-site (17,0) tube with 2 modes and 96
    energies (few chains for a whole GPU), pass-1 sweeps as one piece per
    chain against the automatic split into pieces; device times by CUDA
    events of the charge pass."""
    from electrostatic_b200 import _lib
    from electrostatic_b200.negf import CNT, last_stats, set_timing
    from electrostatic_b200.workloads import SEED_BASE, site_potential
    t = CNT(type_id=(17, 0), num_unitcells=16000, num_modes=2, contact_mu=(0.0, -0.2), contact_T=(300.0, 300.0),
            eq_integration_pts=(8, 8, 16), noneq_integration_pts=(64,), E_zPlus_imag=1e-3)
    U = site_potential(t.site_positions(), SEED_BASE + 4)
    U = 0.5 * (U - U.mean())
    t.set_potential(U, (U[0], U[-1]))
    L = _lib.load()
    set_timing(True)
    res = {}
    try:
        for name, P in (("one_piece", 1), ("automatic", 0)):
            L.negf_set_tuning(4, P)
            for _ in range(3):
                Q = t.Solve_NEGF()
            ms = []
            for _ in range(reps):
                Q = t.Solve_NEGF()
                ms.append(last_stats()["rgf_kernel_ms"] + last_stats()["reduce_kernel_ms"])
            st = last_stats()
            res[name] = {"ms_per_pass": float(np.median(ms)), "pieces": st["pieces"],
                         "updates_per_s": st["updates"] / (float(np.median(ms)) * 1e-3), "Q": Q}
    finally:
        L.negf_set_tuning(4, 0)
        set_timing(False)
    Q1, Qa = res["one_piece"].pop("Q"), res["automatic"].pop("Q")
    return {"workload": "(17,0) CNT, N=64000 sites, 2 modes, 96 energies (contour+poles+real axis), FP64",
            "one_piece": res["one_piece"], "automatic": res["automatic"],
            "speedup": res["one_piece"]["ms_per_pass"] / res["automatic"]["ms_per_pass"],
            "max_rel_automatic_vs_one_piece": float(np.max(np.abs(Qa - Q1)) / np.max(np.abs(Q1)))}


# config 5 in the default run: fewer training pairs and epochs than the stated 20k / 20
CONFIG5_COMPACT = dict(n_pairs=6000, epochs=12)


def config5_measure(torch, n_pairs=20000, epochs=20, batch=64, oracle_check=True, ablation=True,
                    keep_arrays=False):
    """Surrogate-assisted self-consistency on the config-4 tube set (16
    tubes): one neural operator for the whole set (6 layers, width 128, 64
    cosine modes of each tube's length, BF16 weights, FP32 accumulation)
    trained on n_pairs (external potential, self-consistent charge) pairs
    that the engine's own batched solves produce; then the Vds = 0.4 V gate
    sweep 0 -> 0.6 V: plain (FP64 tubes, one Broyden over the set with
    fraction 0.1 from zero charge at every gate point: the reference's
    defaults) and surrogate-started (mixed-precision tubes, start from the
    operator, fraction from the operator's Jacobian, one secant update per
    tube, FP64 finish), with the same solver from other starts beside it.
    Per-step times exclude the one-off plans and graph captures of every
    sweep; data generation and training are reported separately."""
    from electrostatic_b200.negf import CNT
    from electrostatic_b200.scf import run_scf_batch
    from electrostatic_b200.surrogate_set import (TubeSetOperator, fixed_point_sweep, generate_fixed_points,
                                                  tube_descriptor)
    from electrostatic_b200.workloads import GATE_SWEEP, gate_with_contacts, uneven_batch
    descs = uneven_batch(precision="fp64")
    vds = 0.4

    def make(lv, precision="fp64", realaxis_fp32=False):
        return [CNT(**dict(d, contact_mu=(0.0, -float(lv)), precision=precision, mixed_realaxis_fp32=realaxis_fp32))
                for d in descs]

    tubes64 = make(vds)
    electros = []
    for d, t in zip(descs, tubes64):
        R = 1.42e-10 * np.sqrt(3.0) * d["type_id"][0] / (2 * np.pi)  # CNT.cpp:23-41
        electros.append(gate_with_contacts(t.site_positions(), R, vds=vds))
    t0 = time.perf_counter()
    U, Vg, Vds, tid, Q, eng, data_iters = generate_fixed_points(make, electros, n_pairs)
    t_data = time.perf_counter() - t0
    for e in electros:
        e.Vds = vds
    model = TubeSetOperator([tube_descriptor(t) for t in tubes64], seed=0)
    ntr = int(0.9 * n_pairs)
    fit = model.fit_set(U[:ntr], Vg[:ntr], Vds[:ntr], tid[:ntr], Q[:ntr], epochs=epochs, batch=batch)
    pred = model.predict_set(U[ntr:], Vg[ntr:], Vds[ntr:], tid[ntr:])
    qt = Q[ntr:].double()
    qmax = qt.abs().max(dim=1).values.clamp_min(1e-30)
    err = ((pred - qt).abs().max(dim=1).values / qmax).cpu().numpy()
    rms = ((pred - qt).pow(2).sum(dim=1) / model._mask_set[tid[ntr:]].sum(dim=1)).sqrt().div(qmax).cpu().numpy()
    del U, Q, pred, qt
    torch.cuda.empty_cache()
    # plain FP64 sweep (warm-up on one gate point first: plans, graphs, lazy loading)
    run_scf_batch(tubes64, electros, [0.0], use_graph=True, iters_per_graph=4)
    plain = run_scf_batch(tubes64, electros, GATE_SWEEP, use_graph=True, iters_per_graph=4)
    # the same with the charge carried between gate points (the validation decks'
    # reset_with_previous_charge_distribution = 1)
    cont = run_scf_batch(tubes64, electros, GATE_SWEEP, use_graph=True, iters_per_graph=4,
                         reset_with_previous_charge=True)
    # surrogate-started, mixed precision (contour and real-axis chains in FP32 at 2 meV broadening)
    tubesmx = make(vds, precision="mixed", realaxis_fp32=True)
    fixed_point_sweep(tubesmx, electros, [0.0], model)  # warm-up
    sur, alpha, lam, t_setup = fixed_point_sweep(tubesmx, electros, GATE_SWEEP, model)
    t_plain = sum(s_.seconds for s_ in plain.steps)
    t_cont = sum(s_.seconds for s_ in cont.steps)
    t_sur = sum(r["seconds"] for r in sur)
    qref = [s_.Q for s_ in plain.steps]
    dq = max(float(np.max(np.abs(r["Q"] - q))) / float(np.max(np.abs(q))) for r, q in zip(sur, qref))

    def rel(a, q):
        return float(np.max(np.abs(a - q)) / np.max(np.abs(q)))

    res = {"workload": "config-4 tube set (16 tubes), Vds 0.4 V, Vg 0..0.6 V step 0.05, 1e-6 absolute max-norm; "
                       "operator 6 layers x width 128 x 64 cosine modes of each tube's length (32 mixing pairs), "
                       "BF16 weights, FP32 accumulation, trained on self-consistent fixed points",
           "pairs": n_pairs, "data_seconds": t_data, "data_solve_seconds": eng,
           "data_mean_iterations": float(np.mean([i for i in data_iters if i > 0])),
           "data_failed_solves": int(sum(1 for i in data_iters if i < 0)), "train_seconds": fit["seconds"],
           "epochs": epochs, "batch": batch, "final_loss": fit["loss"][-1],
           "test_rel_err_median": float(np.median(err)), "test_rel_err_p90": float(np.percentile(err, 90)),
           "test_rms_rel_err_median": float(np.median(rms)),
           "plain": {"iterations": [s_.iterations for s_ in plain.steps], "seconds": t_plain,
                     "method": "FP64 tubes, one Broyden over the set, fraction 0.1, n = 0 at every gate point "
                               "(reference defaults)"},
           "plain_continuation": {"iterations": [s_.iterations for s_ in cont.steps], "seconds": t_cont,
                                  "method": "as plain, n_in carried from the previous gate point"},
           "surrogate_started": {"negf_iterations": [r["negf_iterations"] for r in sur],
                                 "fp32_iterations": [r["lowprec_iterations"] for r in sur], "seconds": t_sur,
                                 "start_rel_err": [rel(r["start"], q) for r, q in zip(sur, qref)],
                                 "surrogate_rel_err": [rel(r["surrogate"], q) for r, q in zip(sur, qref)],
                                 "fraction": alpha, "lambda_max": lam, "setup_seconds_excluded": t_setup,
                                 "method": "mixed-precision tubes (FP32 contour and real-axis chains, FP64 finish "
                                           "below 3e-6); start = linear extrapolation of the previous two converged "
                                           "charges plus the operator's second difference (the operator's change at "
                                           "the second gate point, its charge at the first); initial inverse "
                                           "Jacobian 0.2 * I; one secant update per tube"},
           "speedup": t_plain / t_sur, "speedup_vs_plain_continuation": t_cont / t_sur,
           "max_rel_dQ_vs_plain_fp64": dq}
    if ablation:
        # the same solver with other starts (with and without the operator), with the secant
        # rows carried between gate points, and with the fraction from the operator's Jacobian
        variants = [(m, dict(start=m)) for m in ("difference", "surrogate", "extrapolation", "continuation", "zero")]
        variants += [("extrapolated_carry_rows", dict(carry_rows=True)),
                     ("extrapolated_fraction_from_operator", dict(fraction=None)),
                     ("extrapolated_fraction_0.15", dict(fraction=0.15)),
                     ("extrapolated_fraction_0.25", dict(fraction=0.25, max_fraction=0.25))]
        # the design rule's mixed mode (real-axis chains in FP64, contour chains in FP32)
        tubesrule = make(vds, precision="mixed")
        variants.append(("extrapolated_realaxis_fp64", dict(tubes=tubesrule)))
        for name, kw in variants:
            kw = dict(kw)
            tset = kw.pop("tubes", tubesmx)
            try:
                o, a_, l_, _ = fixed_point_sweep(tset, electros, GATE_SWEEP, model, **kw)
            except RuntimeError as e:  # a variant that does not converge is reported, not fatal
                res["same_solver_" + name] = {"error": str(e)}
                continue
            res["same_solver_" + name] = {"negf_iterations": [r["negf_iterations"] for r in o],
                                          "seconds": sum(r["seconds"] for r in o), "fraction": a_, "lambda_max": l_,
                                          "start_rel_err": [rel(r["start"], q) for r, q in zip(o, qref)]}
    if keep_arrays:
        res["_arrays"] = {"plain_Q": np.array(qref), "surrogate": np.array([r["surrogate"] for r in sur]),
                          "start": np.array([r["start"] for r in sur]), "n_conv": np.array([r["n_in"] for r in sur])}
    if oracle_check:
        # the FP64 oracle's charge at the converged potential of the last gate point (fixed-point check)
        from oracle import oracle as O
        O.build()
        threads = len(os.sched_getaffinity(0))
        r = sur[-1]
        n_conv = r["n_in"]
        offs = np.concatenate([[0], np.cumsum([t.num_field_sites for t in tubesmx])]).astype(int)
        worst, worst_mx, worst_rule, t1 = 0.0, 0.0, 0.0, time.perf_counter()
        qmx = float(np.max(np.abs(n_conv)))
        rule = tubesrule if ablation else [None] * len(descs)
        for d, e, a, b, tm, tr in zip(descs, electros, offs[:-1], offs[1:], tubesmx, rule):
            kw = {k: v for k, v in d.items() if k not in ("precision", "mixed_realaxis_fp32")}
            ot = O.OracleTube(**dict(kw, contact_mu=(0.0, -vds)))
            Uc = e.potential(n_conv[a:b], GATE_SWEEP[-1])
            ot.set_potential(Uc, (Uc[0], Uc[-1]))
            qo = ot.charge(nthreads=threads)
            worst = max(worst, float(np.max(np.abs(qo - n_conv[a:b]))))
            # the mixed-precision engine's charge at the same potential against the oracle's
            qm = tm.Solve_NEGF(Uc, (Uc[0], Uc[-1]))
            worst_mx = max(worst_mx, float(np.max(np.abs(qm - qo))))
            if tr is not None:
                worst_rule = max(worst_rule, float(np.max(np.abs(tr.Solve_NEGF(Uc, (Uc[0], Uc[-1])) - qo))))
        res["oracle_fixed_point"] = {"Vg": GATE_SWEEP[-1], "max_abs_Qoracle_minus_n": worst,
                                     "relative": worst / qmx, "residual_bar_abs": 1e-6,
                                     "within_residual_bar": bool(worst <= 1e-6),
                                     "mixed_charge_max_rel_vs_oracle": worst_mx / qmx,
                                     "mixed_realaxis_fp64_charge_max_rel_vs_oracle": (worst_rule / qmx
                                                                                      if ablation else None),
                                     "seconds": time.perf_counter() - t1,
                                     "check": "|Q_oracle(U(n)) - n| of the surrogate sweep's converged charge n (the "
                                              "FP64 oracle's residual of the fixed point; the loop's bar is 1e-6 "
                                              "absolute), and the mixed-precision engine's charge at U(n) against "
                                              "the oracle's"}
    for t in tubes64 + tubesmx + (tubesrule if ablation else []):
        t.close()
    return res


def ring_positions_nm(unitcells, acc=1.42e-10):
    """Axial ring positions [nm] of a zigzag tube (CNT.cpp:93-132)."""
    y0 = -(unitcells / 2.0) * 3.0 * acc - acc / 2.0
    ring = np.array([acc, 1.5 * acc, 2.5 * acc, 3.0 * acc])
    r = np.arange(4 * unitcells)
    return (ring[r % 4] + 3 * acc * (r // 4) + y0) / 1e-9


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-scf", action="store_true")
    ap.add_argument("--no-config4", action="store_true")
    ap.add_argument("--no-config3", action="store_true")
    ap.add_argument("--no-long-tube", action="store_true")
    ap.add_argument("--config5", action="store_true",
                    help="surrogate-assisted sweep of the config-4 set at the stated size (20k pairs, 20 epochs); "
                         "without it the default run measures the compact variant")
    ap.add_argument("--no-config5", action="store_true")
    ap.add_argument("--schedule", default="auto", choices=["auto", "fused", "two_pass"],
                    help="RGF schedule of the timed passes (automatic by default)")
    ap.add_argument("--small", action="store_true",
                    help="profiling case: same tube, E = 1024 (256 contour + 768 real-axis); "
                         "real-space case of 200 blocks and 256 contour energies")
    ap.add_argument("--config4-pass", default=None, choices=["fp64", "mixed", "mixed_realaxis_fp32"],
                    help="profiling case: only the config-4 batch charge pass in this precision (one JSON line)")
    ap.add_argument("--tubes", type=int, default=16, help="with --config4-pass: the first TUBES tubes of the batch")
    ap.add_argument("--autotune", action="store_true", help="with --config4-pass: an autotuned plan")
    ap.add_argument("--surrogate-gemm", action="store_true",
                    help="profiling case: negf_nn_gemm on the surrogate's shapes, both tensor-core paths")
    args = ap.parse_args()
    if args.small:
        global EQ_PTS, RT_PTS, WORKLOAD
        EQ_PTS, RT_PTS = (64, 64, 128), 768
        WORKLOAD = WORKLOAD.replace("E=4096", "E=1024").replace("1024 contour", "256 contour").replace(
            "3072 real-axis", "768 real-axis")
    args.warmup = max(3, args.warmup)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return
    if args.config4_pass:
        config4_pass_only(args.config4_pass, args.tubes, args.steps, args.warmup, args.autotune)
        return
    if args.surrogate_gemm:
        surrogate_gemm_only(args.steps, args.warmup)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    from electrostatic_b200 import build
    build.build()
    from electrostatic_b200.negf import CNT, TUNE_SCHEDULE, compute_charge, last_stats, set_timing, set_tuning
    set_tuning(TUNE_SCHEDULE, {"auto": 0, "two_pass": 1, "fused": 2}[args.schedule])

    tube = CNT(**tube_kwargs(args.precision))
    y = tube.site_positions()
    U = site_potential(y, SEED)
    Uc = (U[0], U[-1])
    tube.set_potential(U, Uc)
    if world > 1:
        tube.set_energy_shard(rank, world)  # contiguous energy ranges; Rho0 on rank 0 only
    N = tube.num_field_sites
    Q = torch.zeros(N, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")  # 256 MiB > 126 MB L2
    stream = torch.cuda.current_stream()

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def charge_pass(out):
        """One step: this rank's energy shard, then (N > 1) the sum of the
        partial site charges over the ranks (NCCL, N doubles)."""
        compute_charge([tube], out=out, stream=stream)
        if dist is not None:
            dist.all_reduce(out)

    clk = ClockSampler(local).__enter__()
    # ---- warm-up
    for _ in range(args.warmup):
        charge_pass(Q)
    torch.cuda.synchronize()
    clk.wait_first()
    # updates of the whole tube (every rank's shard)
    upd = torch.tensor([float(last_stats()["updates"])], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(upd)
    updates = int(upd.item())

    # ---- timed: K passes over resident inputs, L2 flushed between passes
    set_timing(True)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    rgf_ms, red_ms, p1_ms, p2_ms = [], [], [], []
    barrier()
    clk_lo = clk.mark()
    for i in range(args.steps):
        flush.zero_()
        ev[i][0].record(stream)
        charge_pass(Q)
        ev[i][1].record(stream)
        st = last_stats()  # waits for this pass's kernel events
        rgf_ms.append(st["rgf_kernel_ms"])
        red_ms.append(st["reduce_kernel_ms"])
        p1_ms.append(st["pass1_kernel_ms"])
        p2_ms.append(st["pass2_kernel_ms"])
    barrier()
    clk_hi = clk.mark() + 1
    set_timing(False)
    step_ms = [a.elapsed_time(b) for a, b in ev]
    t_local = float(np.sum(step_ms))
    t_all = torch.tensor([t_local], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(t_all, op=dist.ReduceOp.MAX)
    t_max = float(t_all.item())
    value = updates * args.steps / (t_max * 1e-3)
    Q_dev = Q.cpu().numpy()

    # ---- end to end through the public API with host buffers: H2D of U
    # (negf_tube_set_potential), the charge pass, and D2H of Q
    U_pinned = torch.from_numpy(U).pin_memory()
    Uh = U_pinned.numpy()
    e2e_ev = []
    barrier()
    for i in range(args.steps):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        flush.zero_()
        s.record(stream)
        tube.set_potential(Uh, Uc)
        if dist is None:
            Qh = compute_charge([tube], stream=stream)  # host Q through the C-ABI
        else:
            charge_pass(Q)
            Qh = Q.cpu().numpy()
        e.record(stream)
        e2e_ev.append((s, e))
    barrier()
    e2e_local = float(np.sum([s.elapsed_time(e) for s, e in e2e_ev]))
    e2e_all = torch.tensor([e2e_local], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(e2e_all, op=dist.ReduceOp.MAX)
    e2e_value = updates * args.steps / (float(e2e_all.item()) * 1e-3)
    assert np.all(np.isfinite(Qh))

    # ---- the same workload in the mixed path
    mixed = None
    Q_mixed = Q_mixed_all = None
    if args.precision == "fp64" and world == 1:
        tm = CNT(**tube_kwargs("mixed"))
        tm.set_potential(U, Uc)
        Qm = torch.zeros_like(Q)
        for _ in range(3):
            compute_charge([tm], out=Qm, stream=stream)
        nm = min(args.steps, 50)
        mev = []
        for i in range(nm):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            flush.zero_()
            a.record(stream)
            compute_charge([tm], out=Qm, stream=stream)
            b.record(stream)
            mev.append((a, b))
        torch.cuda.synchronize()
        sm = last_stats()
        mms = float(np.mean([a.elapsed_time(b) for a, b in mev]))
        Q_mixed = Qm.cpu().numpy()
        mixed = {"ms_per_pass": mms, "updates_per_s": sm["updates"] / (mms * 1e-3),
                 "speedup_vs_fp64": (t_max / args.steps) / mms,
                 "updates_fp32": sm["updates_fp32"], "updates": sm["updates"],
                 "rule": MIXED_RULE,
                 "max_rel_vs_fp64": float(np.max(np.abs(Q_mixed - Q_dev)) / np.max(np.abs(Q_dev)))}
        # opt-in outside that rule: the band lowered to the 1e-4 eV broadening, so the
        # real-axis chains run in FP32 as well (all but the lead band-edge chains)
        ta = CNT(**dict(tube_kwargs("mixed"), mixed_fp64_band=ETA, mixed_realaxis_fp32=True))
        ta.set_potential(U, Uc)
        for _ in range(3):
            compute_charge([ta], out=Qm, stream=stream)
        mev = []
        for i in range(nm):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            flush.zero_()
            a.record(stream)
            compute_charge([ta], out=Qm, stream=stream)
            b.record(stream)
            mev.append((a, b))
        torch.cuda.synchronize()
        sa = last_stats()
        ams = float(np.mean([a.elapsed_time(b) for a, b in mev]))
        Q_mixed_all = Qm.cpu().numpy()
        mixed["realaxis_fp32_opt_in"] = {
            "ms_per_pass": ams, "speedup_vs_fp64": (t_max / args.steps) / ams, "updates_fp32": sa["updates_fp32"],
            "rule": "mixed_fp64_band = 1e-4 eV (the broadening) and mixed_realaxis_fp32: every chain in FP32 but "
                    "those within 1e-4 eV of a lead band edge (outside the 1e-3 eV FP64 band of the design rule)",
            "max_rel_vs_fp64": float(np.max(np.abs(Q_mixed_all - Q_dev)) / np.max(np.abs(Q_dev)))}
        ta.close()
        tm.close()

    # ---- both RGF schedules on the same tube (kernel time per pass, CUDA events)
    schedules = None
    if world == 1:
        from electrostatic_b200.negf import SCHEDULE_FUSED, SCHEDULE_TWO_PASS
        schedules = {"chosen": {1: "two_pass", 2: "fused"}.get(st["schedule"], "?")}
        set_timing(True)
        try:
            for name, v in (("fused", SCHEDULE_FUSED), ("two_pass", SCHEDULE_TWO_PASS)):
                set_tuning(TUNE_SCHEDULE, v)
                Qs = torch.zeros_like(Q)
                for _ in range(3):
                    compute_charge([tube], out=Qs, stream=stream)
                kms = []
                for _ in range(min(args.steps, 30)):
                    flush.zero_()
                    compute_charge([tube], out=Qs, stream=stream)
                    kms.append(last_stats()["rgf_kernel_ms"])
                ss = last_stats()
                schedules[name] = {"rgf_kernel_ms": float(np.mean(kms)), "kernel_launches": ss["kernel_launches"],
                                   "checkpoint_bytes": ss["checkpoint_bytes"],
                                   "max_rel_vs_timed": float((Qs - Q).abs().max() / Q.abs().max())}
        finally:
            set_tuning(TUNE_SCHEDULE, {"auto": 0, "two_pass": 1, "fused": 2}[args.schedule])
            set_timing(False)

    # ---- roofline of the dominant kernel (the RGF sweep kernel)
    flops = st["contour_updates"] * FLOP_CONTOUR + st["realaxis_updates"] * FLOP_REALAXIS
    k_ms = float(np.mean(rgf_ms))
    achieved_tf = flops / (k_ms * 1e-3) / 1e12
    peak_tf = measured_fp64_peak(torch) if rank == 0 else None
    prof = load_profile_traffic("rgf_kernel_config2_ncu.json") or {}
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    scratch_gbs = st["checkpoint_bytes"] / (k_ms * 1e-3) / 1e9

    line = None
    if rank == 0:
        cpu = None
        parity = None
        if not args.no_cpu_baseline and world == 1:
            from oracle import oracle as O
            O.build()
            kw = tube_kwargs()
            kw.pop("precision")
            ot = O.OracleTube(**kw)
            ot.set_potential(U, Uc)
            threads = len(os.sched_getaffinity(0))
            t0 = time.perf_counter()
            _, n = ot.sample(512, 0, faithful=True, nthreads=threads)
            dt = time.perf_counter() - t0
            # one thread (one rank of the reference): energies 0 and 2048 (1 contour + 1 real-axis)
            t1 = time.perf_counter()
            _, n1 = ot.sample(2048, 0, faithful=True, nthreads=1)
            dt1 = time.perf_counter() - t1
            cpu = {"value": n / dt, "unit": "updates/s", "cores": threads, "kind": "port",
                   "sample": "8 of the 4096 energy points (every 512th: 2 contour + 6 real-axis), all 8 modes, "
                             "N=4000, faithful O(N)-per-site contact walk (NEGF_Common.cpp:3418-3426), "
                             f"{threads} threads over energies; {dt:.2f} s",
                   "single_thread": {"value": n1 / dt1, "unit": "updates/s", "cores": 1,
                                     "sample": f"energies 0 and 2048 (1 contour + 1 real-axis), 1 thread; {dt1:.2f} s"}}
            # the oracle as the checker: the whole workload (all 4096 energies, O(N) sweeps), outside the timing
            t2 = time.perf_counter()
            Qo = ot.charge(nthreads=threads)
            dto = time.perf_counter() - t2
            qmax = float(np.max(np.abs(Qo)))
            parity = {"oracle": f"FP64 CPU restatement, whole config-2 pass, {threads} threads, {dto:.1f} s",
                      "fp64_max_rel_vs_oracle": float(np.max(np.abs(Q_dev - Qo)) / qmax),
                      "e2e_max_rel_vs_oracle": float(np.max(np.abs(Qh - Qo)) / qmax),
                      "bars": {"fp64": 1e-8, "mixed": 1e-5}}
            if Q_mixed is not None:
                parity["mixed_max_rel_vs_oracle"] = float(np.max(np.abs(Q_mixed - Qo)) / qmax)
                parity["mixed_realaxis_fp32_opt_in_max_rel_vs_oracle"] = float(np.max(np.abs(Q_mixed_all - Qo)) / qmax)
        scf = None if (args.no_scf or world > 1) else scf_measure(len(os.sched_getaffinity(0)))
        cfg4 = None if (args.no_config4 or world > 1) else config4_measure(torch)
        cfg3 = None if (args.no_config3 or world > 1) else config3_measure(torch, small=args.small)
        longt = None if (args.no_long_tube or world > 1) else long_tube_measure(torch)
        cfg5 = None
        if world == 1 and not args.no_config5:
            cfg5 = config5_measure(torch, **({} if args.config5 else CONFIG5_COMPACT))
            cfg5["size"] = "stated (20k pairs, 20 epochs)" if args.config5 else "compact (%d pairs, %d epochs)" % (
                CONFIG5_COMPACT["n_pairs"], CONFIG5_COMPACT["epochs"])
        clk.__exit__()
        roof = {"bound": "fp64", "achieved": achieved_tf, "peak": peak_tf, "unit": "TFLOP/s",
                "frac": achieved_tf / peak_tf if peak_tf else None,
                "traffic": prof.get("dram_bytes_per_launch"),
                "peak_source": "measured in this run: cuBLAS DGEMM 8192^3 (MEASURED_PEAKS.json has no FP64 figure)",
                "flops_per_launch": flops, "kernel_ms": k_ms,
                "flop_convention": "complex add 2, mul 6, real*complex 2, div 11, |z|^2 3; "
                                   f"{FLOP_CONTOUR}/contour update, {FLOP_REALAXIS}/real-axis update",
                "hbm": {"scratch_bytes_per_launch": st["checkpoint_bytes"], "achieved_gbs": scratch_gbs,
                        "peak_gbs": hbm_peak, "frac": scratch_gbs / hbm_peak}}
        clocks = clk.summary()
        clocks["window"] = "whole GPU phase of the run (warm-up through the last measurement)"
        clocks["timed_region"] = clk.summary(clk_lo, clk_hi)
        line = {"metric": "site*energy RGF updates/s", "value": value, "unit": "updates/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max / args.steps,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
                "dtype": "f64" if args.precision == "fp64" else "f32+f64",
                "data": "synthetic (seeded potential; no dataset)",
                "config": {"workload": WORKLOAD, "precision": args.precision, "updates_per_pass": updates,
                           "updates_fp32": st["updates_fp32"],
                           "parallelism": ("one tube on one GPU" if world == 1 else
                                           f"energy shards of one tube over {world} GPUs, one NCCL all-reduce of "
                                           f"{N} doubles per pass"),
                           "l2": "flushed between passes (256 MiB write), flush outside the per-pass events"},
                "roofline": roof, "cpu_baseline": cpu, "parity": parity, "schedules": schedules, "scf": scf,
                "mixed": mixed,
                "config3": cfg3, "config4": cfg4, "long_tube": longt, "config5": cfg5,
                "e2e": {"value": e2e_value, "unit": "updates/s", "h2d_bytes_per_step": 8 * N + 16,
                        "d2h_bytes_per_step": 8 * N,
                        "path": "negf_tube_set_potential (host U) + negf_compute_charge (host Q)" if world == 1 else
                                "negf_tube_set_potential (host U) + negf_compute_charge + NCCL all-reduce + D2H of Q"},
                "gpu_launches": int(st["kernel_launches"]) * args.steps, "clocks": clocks,
                "kernel_ms_per_pass": {"rgf": k_ms, "rgf_pass1": float(np.mean(p1_ms)),
                                       "rgf_pass2": float(np.mean(p2_ms)), "reduce": float(np.mean(red_ms))}}
        print(json.dumps(line), flush=True)
    else:
        clk.__exit__()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
