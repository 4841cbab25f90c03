"""Self-consistent NEGF-Poisson loop (the transport driver around the engine).

Mirrors c_TransportSolver::Solve (Source/Solver/Transport/Transport.cpp:385-505):
each iteration computes the site potential from the current input charge
(the electrostatics stand-in of electrostatics.py replaces MLMG + gather),
sets U_contact to the end-site potentials (Nanostructure.cpp:500-504), runs the
NEGF charge pass and one Broyden modified-second step; the loop ends when the
Broyden max-norm of the iteration's residual is <= Broyden_max_norm, and
Broyden is reset between bias steps (Reset_ForNextBiasStep,
Transport.cpp:713-717; Broyden_Parallel_General.cpp:250-355).  Every vector
stays on the device; per iteration the host reads the two contact potentials
and the Broyden norm.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import check


@dataclass
class StepResult:
    Vg: float
    iterations: int
    norm: float
    Q: np.ndarray
    U: np.ndarray
    seconds: float


@dataclass
class SCFResult:
    steps: list = field(default_factory=list)

    @property
    def total_iterations(self):
        return sum(s.iterations for s in self.steps)

    @property
    def seconds(self):
        return sum(s.seconds for s in self.steps)


def device_view(ptr: int, n: int):
    """Zero-copy float64 torch view of n doubles of device memory at ptr."""
    import torch

    class _Array:
        __cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (int(ptr), False), "version": 3}

    return torch.as_tensor(_Array(), device="cuda")


def run_scf(tube, electro, Vg_list, fraction=0.1, max_norm=1e-6, max_step=200, norm_type="absolute",
            initial_charge=0.0, reset_with_previous_charge=False, stream=None):
    """Bias sweep of self-consistent solves for one tube on the current device.
    initial_charge: a value for every site, or the path of a _Qout.dat table
    (restart, read with Read_Table1D's rules)."""
    import torch
    from .negf import Broyden, compute_charge

    from .negf import read_table1d

    L = _lib.load()
    N = tube.num_field_sites
    dev = torch.device("cuda")
    if isinstance(initial_charge, str):
        # Initialize_ChargeAtFieldSites with a charge table (NEGF_Common.cpp:178-235)
        n_in = torch.tensor(read_table1d(initial_charge, N), dtype=torch.float64, device=dev)
        initial_charge = 0.0
    else:
        n_in = torch.full((N,), float(initial_charge), dtype=torch.float64, device=dev)
    Q = torch.zeros(N, dtype=torch.float64, device=dev)
    br = Broyden(n_in, max_step=max_step, fraction=fraction, norm_type=norm_type)
    U_ptr = tube.potential_device_ptr()
    U_view = device_view(U_ptr, N)
    s_ptr = None if stream is None else C.c_void_p(stream.cuda_stream)
    res = SCFResult()
    for Vg in Vg_list:
        Kd, U0 = electro.device_operator(Vg)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        it, nrm = 0, float("inf")
        while True:
            if br.step_number > max_step:  # Transport.cpp:389-393
                raise RuntimeError("Broyden_Step has exceeded the Broyden_Threshold_MaxStep")
            check(L.negf_affine_potential(C.c_void_p(Kd.data_ptr()), C.c_void_p(U0.data_ptr()),
                                          C.c_void_p(n_in.data_ptr()), C.c_void_p(U_ptr), N, s_ptr),
                  "negf_affine_potential")
            ends = U_view[[0, N - 1]].cpu().numpy()
            tube.set_potential_device(U_ptr, (float(ends[0]), float(ends[1])), stream=stream)
            compute_charge([tube], out=Q, stream=stream)
            nrm = br.step(Q, n_in_out=n_in, stream=stream)
            it += 1
            if not (nrm > max_norm):
                break
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        res.steps.append(StepResult(Vg, it, nrm, Q.cpu().numpy().copy(), U_view.cpu().numpy().copy(), dt))
        br.reset(keep_charge=reset_with_previous_charge, init_value=initial_charge)
        if reset_with_previous_charge:
            n_in.copy_(device_view(br.input_device_ptr(), N))
        else:
            n_in.fill_(float(initial_charge))
    br.close()
    return res


class BatchSCF:
    """One self-consistent solver over a batch of tubes, kept between solves.

    Each iteration: U_t = U0_t + K_t n_in[t] for every tube (its electrostatics
    operator), one charge-plan launch for the whole batch, one device-resident
    Broyden step over all the tubes' sites (the all-tubes n_in of
    Broyden_Parallel_General.cpp:42-66).  With use_graph, iters_per_graph
    iterations are captured in one CUDA graph and replayed until the device
    flags say converged (or failed); the host reads the flag ints once per
    replay.  With switch_norm (mixed-precision tubes), the iterations run on
    the tubes' own plan until the residual falls below switch_norm and on an
    FP64 plan from then on; only an FP64 charge ends a solve.  segments: one
    secant update per tube (negf_broyden_set_segments) instead of one over the
    whole batch.  Every solve runs on the solver's own stream."""

    def __init__(self, tubes, electros, fraction=0.1, max_norm=1e-6, max_step=200, norm_type="absolute",
                 initial_charge=0.0, use_graph=True, iters_per_graph=8, autotune=True, switch_norm=None,
                 segments=False):
        import torch
        from .negf import Broyden, ChargePlan, PotentialBatch, affine_potential_masked

        dev = torch.device("cuda")
        self.tubes, self.electros = list(tubes), list(electros)
        self.Ns = [t.num_field_sites for t in tubes]
        self.offs = np.concatenate([[0], np.cumsum(self.Ns)]).astype(int)
        S = self.S = int(self.offs[-1])
        self.stream = stream = torch.cuda.Stream()
        self.initial_charge = float(initial_charge)
        with torch.cuda.stream(stream):
            self.Q = Q = torch.zeros(S, dtype=torch.float64, device=dev)
            n0 = torch.full((S,), self.initial_charge, dtype=torch.float64, device=dev)
            self.br = br = Broyden(n0, max_step=max_step, fraction=fraction, norm_type=norm_type, stream=stream)
            if segments and len(tubes) > 1:
                br.set_segments(self.offs, stream=stream)
            nin = br.input_device_ptr()
            self.n_in = device_view(nin, S)
            self.U_ptrs = U_ptrs = [t.potential_device_ptr() for t in tubes]
            self.ops = ops = []
            for e in electros:
                Kd, U0 = e.device_operator(0.0)
                ops.append((Kd, U0.clone()))
            # lattice-distance kernels (every zigzag tube of the gate-all-around stand-in) are
            # applied from their tables, all tubes in one launch, instead of the n x n matrices
            toes = [e.device_toeplitz() if hasattr(e, "device_toeplitz") else None for e in electros]
            self.potbatch = None
            if all(t is not None for t in toes):
                self.potbatch = PotentialBatch([t[0] for t in toes], [t[1] for t in toes], [U0 for _, U0 in ops],
                                               [nin + 8 * int(o) for o in self.offs[:-1]], list(self.U_ptrs),
                                               self.Ns)

            def potentials(skip_ptr, s):
                if self.potbatch is not None:
                    self.potbatch.launch(skip=skip_ptr, stream=s)
                    return
                for (Kd, U0), o, N, Up in zip(ops, self.offs, self.Ns, self.U_ptrs):
                    affine_potential_masked(Kd, U0, nin + 8 * int(o), Up, N, skip_ptr, stream=s)

            self.flags = flags = torch.zeros(8, dtype=torch.int32, device=dev)
            skip = flags.data_ptr() + 3 * 4
            self.switch = switch = switch_norm is not None and switch_norm > 0
            # the initial potential (paths do not depend on it; contact potentials are read on the device)
            potentials(None, stream)
            self.plan = plan = ChargePlan(tubes, Q, autotune=autotune)
            self.plan64 = plan64 = ChargePlan(tubes, Q, autotune=autotune, fp64=True) if switch else None

            def body(s):
                potentials(skip, s)
                if switch:
                    plan.launch(skip=flags.data_ptr() + 5 * 4, stream=s)
                    plan64.launch(skip=flags.data_ptr() + 6 * 4, stream=s)
                    br.step_device_switch(Q, max_norm, switch_norm, flags, stream=s)
                else:
                    plan.launch(skip=skip, stream=s)
                    br.step_device(Q, max_norm, flags, stream=s)

            self._body = body
            self.graph = None
            if use_graph:
                flags[3] = 1  # load every kernel once, all skipped
                body(stream)
                stream.synchronize()
                self.graph = torch.cuda.CUDAGraph()
                with torch.cuda.graph(self.graph, stream=stream):
                    for _ in range(iters_per_graph):
                        body(torch.cuda.current_stream())
            stream.synchronize()

    def set_external(self, Vg=None, U0=None):
        """The external potential of the next solve: the electrostatics' at
        gate voltage Vg, or U0 (one array per tube: host arrays, or float64
        device tensors copied on the solver's stream)."""
        import torch
        with torch.cuda.stream(self.stream):
            for t_, ((Kd, U0d), e) in enumerate(zip(self.ops, self.electros)):
                if U0 is None:
                    U0d.copy_(e.device_operator(Vg)[1])
                elif isinstance(U0[t_], torch.Tensor):
                    U0d.copy_(U0[t_])
                else:
                    U0d.copy_(torch.as_tensor(np.asarray(U0[t_], dtype=np.float64)), non_blocking=False)

    def solve(self):
        """Iterate to convergence from the current n_in; returns (steps,
        low-precision steps).  Raises on MaxStep or a non-finite norm."""
        import torch
        with torch.cuda.stream(self.stream):
            self.flags.zero_()
            if self.switch:
                self.flags[6] = 1  # the FP64 plan waits for the switch
            while True:
                if self.graph is not None:
                    self.graph.replay()
                else:
                    self._body(self.stream)
                f = self.flags.cpu().numpy()
                if f[3]:
                    break
        if f[2] == 1:
            raise RuntimeError("Broyden_Step has exceeded the Broyden_Threshold_MaxStep")
        if f[2] == 2:
            raise RuntimeError("non-finite Broyden norm")
        return int(f[1]), int(f[7])

    def reset(self, keep_charge=False, init_value=None):
        """Reset_ForNextBiasStep: clear the secant rows; n_in stays (keep_charge)
        or becomes init_value (default: the initial charge)."""
        v = self.initial_charge if init_value is None else float(init_value)
        self.br.reset(keep_charge=keep_charge, init_value=v, stream=self.stream)

    def potentials(self):
        return np.concatenate([device_view(Up, N).cpu().numpy() for Up, N in zip(self.U_ptrs, self.Ns)])

    def close(self):
        self.stream.synchronize()
        self.graph = None
        if self.potbatch is not None:
            self.potbatch.close()
        self.plan.close()
        if self.plan64 is not None:
            self.plan64.close()
        self.br.close()


def run_scf_batch(tubes, electros, Vg_list, fraction=0.1, max_norm=1e-6, max_step=200, norm_type="absolute",
                  initial_charge=0.0, reset_with_previous_charge=False, use_graph=True, iters_per_graph=8,
                  autotune=True, switch_norm=None, segments=False):
    """Self-consistent bias sweep of a batch of tubes (BatchSCF) with one
    Broyden over all their sites, reset between bias points
    (Reset_ForNextBiasStep, Transport.cpp:713-717).  Returns an SCFResult
    plus the plan's schedule."""
    import torch
    scf = BatchSCF(tubes, electros, fraction=fraction, max_norm=max_norm, max_step=max_step, norm_type=norm_type,
                   initial_charge=initial_charge, use_graph=use_graph, iters_per_graph=iters_per_graph,
                   autotune=autotune, switch_norm=switch_norm, segments=segments)
    res = SCFResult()
    for Vg in Vg_list:
        scf.set_external(Vg=Vg)
        scf.stream.synchronize()
        t0 = time.perf_counter()
        it, low = scf.solve()
        dt = time.perf_counter() - t0
        with torch.cuda.stream(scf.stream):
            st = StepResult(Vg, it, float("nan"), scf.Q.cpu().numpy().copy(), scf.potentials(), dt)
        st.lowprec_iterations = low
        res.steps.append(st)
        scf.reset(keep_charge=reset_with_previous_charge)
    info = scf.plan.info()
    scf.close()
    res.schedule = info
    return res
