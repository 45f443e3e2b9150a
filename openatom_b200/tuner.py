"""Autotuner of the runtime tile and schedule choices of a context
(oa_tuning: state groups of the per-state and state-pair plane kernels,
split-K blocks of the FP64 products, the FFT path) per system size and
precision.

For each system it runs coordinate descent over the knobs: every candidate
value is set (oa_gpu_set_tuning) on a fresh context started from the same
quenched coefficients and timed as whole native CP steps (one
oa_gpu_cp_run call of ``steps`` steps after a warm-up call, CUDA events on
the context's stream, best of ``reps``).  A value is
kept only when it beats the current choice by more than ``margin``.  The
result is recorded in a JSON table keyed by the system's sizes and
precision (``tuning/b200.json``), which CPContext applies at creation.

Run on a B200:  python -m openatom_b200.tuner --presets w8 w32 w128 --batch 48
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.path.join(HERE, "tuning", "b200.json")
_table_cache: dict | None = None


def system_key(sysm, precision: str) -> str:
    """Sizes that set the kernels' shapes: precision, FFT grid, states,
    g-points, nonlocal atoms."""
    nx, ny, nz = sysm.nfft
    return f"{precision}/{nx}x{ny}x{nz}/s{sysm.nstate}/g{sysm.ng}/nl{len(sysm.nl_atoms())}"


def load_table(path: str = TABLE) -> dict:
    global _table_cache
    if path == TABLE and _table_cache is not None:
        return _table_cache
    tab = {}
    if os.path.exists(path):
        with open(path) as f:
            tab = json.load(f).get("entries", {})
    if path == TABLE:
        _table_cache = tab
    return tab


def lookup(sysm, precision: str, path: str = TABLE):
    """The recorded choice for this system, or None."""
    e = load_table(path).get(system_key(sysm, precision))
    return None if e is None else dict(e["choice"])


def candidates(knob: str, sysm, precision: str, current: dict, caps: dict) -> list:
    """Values of one knob worth timing for this system."""
    npair = (sysm.nstate + 1) // 2
    if knob == "group_pair":
        return [g for g in (1, 2, 3, 4, 5, 6, 8, 10, 12, 16) if g <= min(32, npair)]
    if knob == "group_state":
        return [g for g in (1, 2, 3, 4, 6, 8, 12, 16, 24, 32) if g <= min(32, sysm.nstate)]
    if knob == "dgemm_kblocks":
        return [k for k in (16, 32, 64, 96, 128, 148, 160) if 2 <= k <= caps["dgemm_kblocks"]]
    if knob == "tgemm_kblocks":
        c = caps["tgemm_kblocks"]
        return sorted({k for k in (max(1, c // 8), max(1, c // 4), max(1, c // 2), max(1, 3 * c // 4), c)})
    if knob == "fft_path":
        return [1, 2] if precision == "fp64" else [1]
    raise ValueError(knob)


def knobs_for(precision: str) -> tuple:
    """Knobs searched: the ones that change only the order of partial sums
    (tgemm_kblocks also lengthens the FP32 tensor-core accumulations, so it
    stays at the built-in choice, the largest the partials allow)."""
    if precision == "mixed":
        return ("group_pair", "dgemm_kblocks")
    return ("group_state", "dgemm_kblocks", "fft_path")


def _time_steps(torch, drv, st, steps: int, reps: int) -> float:
    """Best-of-reps ms per step of native CP steps (one call of `steps`)."""
    stream = torch.cuda.current_stream()
    best = float("inf")
    for _ in range(reps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        drv.run_native(st, steps)
        b.record(stream)
        torch.cuda.synchronize()
        best = min(best, a.elapsed_time(b) / steps)
    return best


def _quenched_psi(sysm, large: bool):
    """Coefficients off the random start: damped FP64 CP, three steps at
    the system's dt then more at dt = 10 (as the benchmark's start)."""
    from .gpu import CPDriver
    q = CPDriver(sysm, "fp64", tuning="default")
    q.quench(3)
    q.quench(3 if large else 27, dt=10.0)
    psi0 = q.psi.cpu().numpy()
    q.ctx.close()
    return psi0


def _measure(torch, sysm, precision: str, psi0, choice: dict, steps: int, reps: int) -> float:
    """ms per native CP step with these choices, on a fresh context from psi0."""
    from .gpu import CPDriver
    drv = CPDriver(sysm, precision, psi0=psi0, norb_tol=0.003, tuning="default")
    try:
        if choice:
            drv.ctx.set_tuning(**choice)
        st = drv.native_state(use_graph=True)
        drv.run_native(st, 3)
        return _time_steps(torch, drv, st, steps, reps)
    finally:
        drv.ctx.close()


def tune_system(sysm, precision: str, steps: int = 10, reps: int = 3, margin: float = 0.015, log=None) -> dict:
    """Coordinate descent over knobs_for(precision) on one system, every
    candidate timed on a fresh context from the same quenched coefficients;
    returns the table entry {"choice", "default", "ms_default", "ms_tuned",
    "trials"}."""
    import torch
    from .gpu import CPContext, OaError
    ctx = CPContext(sysm, precision, tuning="default")
    default = ctx.get_tuning()
    ctx.close()
    caps = dict(default)
    caps["dgemm_kblocks"] = 160
    psi0 = _quenched_psi(sysm, sysm.nstate > 128)
    ms_default = _measure(torch, sysm, precision, psi0, {}, steps, reps)
    cur, cur_ms = dict(default), ms_default
    trials = []
    for knob in knobs_for(precision):
        for v in candidates(knob, sysm, precision, cur, caps):
            if v == cur[knob]:
                continue
            trial = dict(cur)
            trial[knob] = v
            try:
                ms = _measure(torch, sysm, precision, psi0, trial, steps, reps)
            except OaError as e:
                trials.append({knob: v, "error": str(e)[:120]})
                continue
            trials.append({knob: v, "ms": ms})
            if ms < cur_ms * (1.0 - margin):
                cur, cur_ms = trial, ms
        if log:
            log(f"  {knob}: {cur[knob]} ({cur_ms:.4f} ms)")
    # confirm against the built-in choice with fresh timings of both
    ms_d2 = _measure(torch, sysm, precision, psi0, {}, steps, reps)
    ms_t2 = _measure(torch, sysm, precision, psi0, cur, steps, reps) if cur != default else ms_d2
    choice = cur if ms_t2 < ms_d2 * (1.0 - margin) else dict(default)
    torch.cuda.empty_cache()
    return {"choice": choice, "default": default, "ms_default": min(ms_default, ms_d2),
            "ms_tuned": ms_t2 if choice != default else min(ms_default, ms_d2), "trials": trials}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--presets", nargs="*", default=["w8", "w32", "w128"])
    ap.add_argument("--precisions", nargs="*", default=["mixed", "fp64"])
    ap.add_argument("--batch", type=int, default=0,
                    help="also tune N systems of system.batch_systems (mixed form only)")
    ap.add_argument("--batch-seed", type=int, default=2031,
                    help="seed of the batch systems (the benchmark's batching form uses 2031)")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--out", default=TABLE)
    ap.add_argument("--only-missing", action="store_true", help="skip systems the table already holds")
    a = ap.parse_args(argv)
    from .system import make_system
    import torch
    # the benchmark's systems: mass preconditioning at 2 Ry, mu = 400, dt = 5
    jobs = [(make_system(p, seed=a.seed, ecut_mass=2.0, cmass0=400.0, dt=5.0), prec)
            for p in a.presets for prec in a.precisions]
    if a.batch:
        from .system import batch_systems
        jobs += [(sy, "mixed") for sy in batch_systems(a.batch_seed, a.batch)]
    tab = {}
    if os.path.exists(a.out):
        with open(a.out) as f:
            tab = json.load(f).get("entries", {})
    t0 = time.time()
    for sysm, prec in jobs:
        key = system_key(sysm, prec)
        if key in tab and (tab[key].get("seen_this_run") or a.only_missing):
            continue
        print(f"{key}", flush=True)
        steps = a.steps if sysm.nstate <= 128 else max(2, a.steps // 4)
        try:
            e = tune_system(sysm, prec, steps=steps, reps=a.reps, log=lambda m: print(m, flush=True))
        except Exception as exc:  # record and go on with the other systems
            print(f"  failed: {exc}", flush=True)
            continue
        e["seen_this_run"] = True
        tab[key] = e
        print(f"  -> {e['choice']}  {e['ms_default']:.4f} -> {e['ms_tuned']:.4f} ms/step", flush=True)
    for e in tab.values():
        e.pop("seen_this_run", None)
    meta = {"device": torch.cuda.get_device_name(0), "tuned_s": round(time.time() - t0, 1),
            "method": "coordinate descent over oa_tuning, native CP steps timed with CUDA events, "
                      f"best of {a.reps}, {a.steps} steps (fewer above 128 states), 1.5% margin"}
    os.makedirs(os.path.dirname(a.out), exist_ok=True)
    with open(a.out, "w") as f:
        json.dump({"meta": meta, "entries": tab}, f, indent=1, sort_keys=True)
    print(f"wrote {a.out}: {len(tab)} entries")


if __name__ == "__main__":
    main()
