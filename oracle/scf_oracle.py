"""ORACLE — test infrastructure only.

The self-consistent NEGF-Poisson loops of ``electrostatic_b200.scf`` restated
on the CPU oracle: the single-tube sweep and the batched sweep with one
Broyden over all tubes' sites.  They follow the loop predicate of
Source/Solver/Transport/Transport.cpp:385-505 and the Broyden reset of
Broyden_Parallel_General.cpp:250-355.  Only ``tests/`` and the CPU-baseline
leg of ``bench.py`` call them, as the checker; the product package never
imports this module.
"""
from __future__ import annotations

import time

import numpy as np

from electrostatic_b200.scf import SCFResult, StepResult

from . import oracle as O


def run_scf_oracle(oracle_tube, K, Vg_list, fraction=0.1, max_norm=1e-6, max_step=200, norm_type="absolute",
                   initial_charge=0.0, reset_with_previous_charge=False, nthreads=8):
    """The same loop on the CPU oracle (test infrastructure and CPU baseline).
    K: the coupling matrix (U = -Vg - K Q) or an electrostatics object with
    potential(Q, Vg)."""
    pot = K.potential if hasattr(K, "potential") else (lambda q, vg: -float(vg) - K @ q)

    N = oracle_tube.N
    n_in = np.full(N, float(initial_charge))
    br = O.OracleBroyden(n_in, max_step=max_step, fraction=fraction, norm_type=norm_type)
    res = SCFResult()
    for Vg in Vg_list:
        t0 = time.perf_counter()
        it, nrm = 0, float("inf")
        while True:
            U = pot(n_in, Vg)
            oracle_tube.set_potential(U, (U[0], U[-1]))
            Q = oracle_tube.charge(nthreads=nthreads)
            nrm, n_in, _ = br.step(Q)
            it += 1
            if not (nrm > max_norm):
                break
        res.steps.append(StepResult(Vg, it, nrm, Q, U, time.perf_counter() - t0))
        br.reset(keep_charge=reset_with_previous_charge, init_value=initial_charge)
        if not reset_with_previous_charge:
            n_in = np.full(N, float(initial_charge))
    return res



def run_scf_batch_oracle(oracle_tubes, Ks, Vg_list, fraction=0.1, max_norm=1e-6, max_step=200,
                         norm_type="absolute", initial_charge=0.0, nthreads=8):
    """The batched loop on the CPU oracle: one Broyden over all tubes' sites.
    Ks: per tube a coupling matrix or an electrostatics object."""

    Ns = [t.N for t in oracle_tubes]
    offs = np.concatenate([[0], np.cumsum(Ns)]).astype(int)
    S = int(offs[-1])
    n_in = np.full(S, float(initial_charge))
    br = O.OracleBroyden(n_in, max_step=max_step, fraction=fraction, norm_type=norm_type)
    res = SCFResult()
    for Vg in Vg_list:
        t0 = time.perf_counter()
        it = 0
        while True:
            Q = np.zeros(S)
            for t, K, a, b in zip(oracle_tubes, Ks, offs[:-1], offs[1:]):
                U = K.potential(n_in[a:b], Vg) if hasattr(K, "potential") else -float(Vg) - K @ n_in[a:b]
                t.set_potential(U, (U[0], U[-1]))
                Q[a:b] = t.charge(nthreads=nthreads)
            nrm, n_in, _ = br.step(Q)
            it += 1
            if not (nrm > max_norm):
                break
            if it >= max_step:
                raise RuntimeError("Broyden_Step has exceeded the Broyden_Threshold_MaxStep")
        res.steps.append(StepResult(Vg, it, nrm, Q, None, time.perf_counter() - t0))
        br.reset(keep_charge=False, init_value=initial_charge)
        n_in = np.full(S, float(initial_charge))
    return res
