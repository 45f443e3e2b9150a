#!/usr/bin/env python
"""Benchmark: CP steps/s of the Gamma-point CP electronic step on B200.

Workload (default): 32 H2O (96 atoms) in an 18.6 bohr cubic box, 80 Ry state
cutoff, 108^3 grid, 128 doubly occupied states, dt = 5 a.u., fictitious mass
400 a.u. (mass cutoff 2 on g^2), synthetic seeded coefficients.  The random
start is quenched (damped CP, untimed) before the timed dynamics steps.

A "step" is one CP dynamics step: state FFTs + density, V_KS (XC, Hartree,
local), V_KS psi back to forces + EKE, Lambda / Gamma constraint force,
Verlet integration, S, Newton-Schulz S^-1/2 and Psi T.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  N > 1 runs independent replicas (one system
per rank, no data-path collective): scaling "weak".  Beside the headline the
line carries the FP64 form on the same start, the batching form (48 uneven
systems, `batch`) and the 128 H2O / 512-state / 160^3 system (`large`).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "CP steps/s at 128 states: mixed vs FP64 on 1 B200, |dE|<=1e-6 Ha/atom"
UNIT = "CP steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="w32")
    ap.add_argument("--quench", type=int, default=30)
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline sample")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--batch", type=int, default=48,
                    help="systems of the batching form measured beside the headline (0: skip)")
    ap.add_argument("--large", type=int, default=1,
                    help="also time the 128 H2O / 512-state / 160^3 system in the mixed form (0: skip)")
    ap.add_argument("--large-min-iter", type=int, default=80,
                    help="CG iterations of the large system's start")
    ap.add_argument("--blyp", type=int, default=1,
                    help="also time the 32-water step with the BLYP gradient correction (0: skip)")
    ap.add_argument("--ground", type=int, default=1,
                    help="also time the headline system from its CG-minimised ground state (0: skip)")
    ap.add_argument("--ions", type=int, default=1,
                    help="also time the 32-water step with moving atoms (structure factors, EES local; 0: skip)")
    ap.add_argument("--drift-steps", type=int, default=1000,
                    help="steps of the 8-water precision run (energy drift, mixed vs FP64; 0: skip)")
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rk = int(os.environ.get("RANK", "0"))
    lr = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rk, lr


def max_over_ranks(values, ws, device="cuda"):
    """The per-rank timings reduced to their maximum over the ranks (the
    slowest replica sets the step time); one all-reduce, every rank takes
    part."""
    if ws <= 1:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def replica_seed(seed, rank):
    """Seed of a rank's independent system (replicas only: no data-path
    collective between ranks)."""
    return seed + rank


def make_sys(cfg, seed):
    from openatom_b200.system import make_system
    return make_system(cfg, seed=seed, ecut_mass=2.0, cmass0=400.0, dt=5.0)


def batch_form(torch, args):
    """Batching form: args.batch independent systems advanced together, one
    CUDA graph per step (oa_gpu_cp_run_batch), against the same systems run
    one after the other (oa_gpu_cp_run each)."""
    from openatom_b200.gpu import CPDriver, run_batch
    from openatom_b200.system import batch_systems
    syss = batch_systems(args.seed + 7, args.batch)
    drv = [CPDriver(s, "mixed") for s in syss]
    for d in drv:
        d.quench(3)
    sts = [d.native_state(use_graph=True) for d in drv]
    stream = torch.cuda.Stream()
    run_batch(drv, sts, 3, stream)
    k = max(args.steps // 2, 3)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    run_batch(drv, sts, k, stream)
    ev1.record(stream)
    torch.cuda.synchronize()
    ms_batch = ev0.elapsed_time(ev1) / k
    batch_kernels = sts[0].last_kernels
    for d, st in zip(drv, sts):
        d.run_native(st, 2)
    ms_seq = 0.0
    for d, st in zip(drv, sts):
        ms, _ = time_steps(torch, d, st, k)
        ms_seq += ms
    n = len(drv)
    out = {"systems": n, "states": [min(s.nstate for s in syss), max(s.nstate for s in syss)],
           "grids": sorted({s.nfft[0] for s in syss}), "ecut_ry": sorted({s.ecut_ry for s in syss}),
           "steps": k, "ms_per_batch_step": ms_batch, "system_steps_per_s": n * 1e3 / ms_batch,
           "sequential_ms_per_batch_step": ms_seq, "speedup_vs_sequential": ms_seq / ms_batch,
           "graph_kernels_per_step": batch_kernels, "precision": "mixed",
           "tuned_systems": sum(1 for d in drv if d.ctx.tuning_source == "table")}
    del drv
    return out


def large_form(torch, args):
    """The large single system (128 H2O, 512 states, 70 Ry, 160^3) with the
    EES nonlocal projectors of B-spline order 4: mixed CP steps/s from a
    start minimised by conjugate gradients (mixed form, a capped number of
    iterations), then the FP64 form from the same start (its plane passes
    keep the FP64 density / V_KS plane in global memory at this size) and
    the total-energy difference of the two forms per atom."""
    from openatom_b200.gpu import CPDriver
    sysm = make_sys("w128", args.seed + 11)
    psi0, start = minimized_start(sysm, iters=args.large_min_iter, prec="mixed", nl_method="ees", ees_order=4)
    from openatom_b200 import ees as ees_mod
    grid = list(ees_mod.nonlocal_grid(sysm, 1.2, 4))
    torch.cuda.empty_cache()
    k = 4
    res, ens, first = {}, {}, {}
    for prec in ("mixed", "fp64"):
        d = CPDriver(sysm, prec, nl_method="ees", ees_order=4, norb_tol=NORB_TOL, psi0=psi0)
        st = d.native_state(use_graph=True)
        # the first step's record: the energies of the same psi0 in both forms
        first[prec] = d.run_native(st, 1)[0]
        d.run_native(st, 1)
        res[prec], ens[prec] = time_steps(torch, d, st, k)
        ortho = d.last_ortho[1]
        d.ctx.close()
        del d
        torch.cuda.empty_cache()
    de = max(abs(total_energy(a) - total_energy(b)) for a, b in zip(ens["mixed"], ens["fp64"])) / sysm.natm
    de0 = abs(total_energy(first["mixed"]) - total_energy(first["fp64"])) / sysm.natm
    return {"workload": f"w128: 128 H2O, {sysm.nstate} states, 70 Ry, 160^3, ng={sysm.ng}",
            "dE_per_atom_same_psi": de0,
            "per_term_same_psi": {t: abs(first["mixed"][t] - first["fp64"][t]) for t in TERMS},
            "nonlocal": "ees4", "ees_grid": grid, "precision": "mixed", "steps": k,
            "ms_per_step": res["mixed"], "value": 1e3 / res["mixed"], "unit": UNIT,
            "fp64": {"ms_per_step": res["fp64"], "value": 1e3 / res["fp64"]},
            "mixed_over_fp64": res["fp64"] / res["mixed"], "dE_per_atom_max_steps_3_to_6": de,
            "ortho_residual": ortho, "smax_max": max(e["SMAX"] for e in ens["mixed"]), "start": start}


def blyp_form(torch, args):
    """The 32-water workload with the BLYP functional (Becke 88 + LYP
    gradient correction, its six extra density-grid transforms per step):
    mixed and FP64 CP steps/s from the same CG-minimised start, the total-energy
    difference of the two forms, EGGA, and the density path's kernel time
    with and without the correction."""
    from openatom_b200.gpu import CPDriver
    sysm = make_sys(args.config, args.seed)
    sysm.xc = "blyp"
    psi0, start = minimized_start(sysm, iters=300)
    res = {}
    ens = {}
    kt = {}
    for prec in ("mixed", "fp64"):
        d = CPDriver(sysm, prec, psi0=psi0, norb_tol=NORB_TOL)
        st = d.native_state(use_graph=True)
        d.run_native(st, 3)
        k = 10
        ms, en = time_steps(torch, d, st, k)
        res[prec] = ms
        ens[prec] = en
        if prec == "mixed":
            kt["blyp"] = d.ctx.time_kernels(d.psi, reps=5)["vks_build"]
            d.ctx.set_xc("pz_lda")
            kt["pz_lda"] = d.ctx.time_kernels(d.psi, reps=5)["vks_build"]
        d.ctx.close()
        del d
    de = max(abs(total_energy(a) - total_energy(b)) for a, b in zip(ens["mixed"], ens["fp64"])) / sysm.natm
    torch.cuda.empty_cache()
    return {"workload": f"{args.config} with BLYP: {sysm.natm // 3} H2O, {sysm.nstate} states, "
                        f"{sysm.ecut_ry:g} Ry, {sysm.nfft[0]}^3, gradient_cutoff {sysm.gga_cut:g}",
            "steps": 10, "mixed": {"value": 1e3 / res["mixed"], "ms_per_step": res["mixed"]},
            "fp64": {"value": 1e3 / res["fp64"], "ms_per_step": res["fp64"]},
            "mixed_over_fp64": res["fp64"] / res["mixed"], "dE_per_atom_max_steps_3_to_6": de,
            "egga": ens["fp64"][-1]["EGGA"], "start": start,
            "density_path_ms": {"blyp": kt["blyp"], "pz_lda": kt["pz_lda"]}}


def ground_state_form(torch, sysm, k):
    """Mixed and FP64 CP steps/s from the CG-minimised ground state of the
    headline system (beside the quenched start the headline uses, which the
    reference arm can reproduce on the host), the PsiV resets in the timed
    steps and the largest total-energy difference of the two forms."""
    from openatom_b200.gpu import CPDriver
    psi0, start = minimized_start(sysm)
    out = {"start": start, "steps": k}
    ens = {}
    for prec in ("mixed", "fp64"):
        d = CPDriver(sysm, prec, psi0=psi0, norb_tol=NORB_TOL)
        st = d.native_state(use_graph=True)
        d.run_native(st, 5)
        ms, en = time_steps(torch, d, st, k)
        ens[prec] = en
        out[prec] = {"value": 1e3 / ms, "ms_per_step": ms, "psiv_resets": sum(1 for e in en if e["SMAX"] > NORB_TOL)}
        d.ctx.close()
    out["mixed_over_fp64"] = out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"]
    out["dE_per_atom_max"] = max(abs(total_energy(a) - total_energy(b))
                                 for a, b in zip(ens["mixed"], ens["fp64"])) / sysm.natm
    return out


def force_call_form(torch, drv, k):
    """The force half of a CP step as a chare would call it through the C
    ABI with host buffers: psi copied in from pinned host memory,
    state_fft_fwd + vks_build + nl_sf + vks_apply_fft_bwd (computePsiFandVKS,
    the ParticlePlane forces, combineForcesGetEke), F copied back to pinned
    host memory; CUDA events around k such calls."""
    psi_h = drv.psi.cpu().pin_memory()
    f_h = torch.empty_like(psi_h).pin_memory()

    def call():
        drv.psi.copy_(psi_h, non_blocking=True)
        drv.forces()
        f_h.copy_(drv.F, non_blocking=True)

    for _ in range(2):
        call()
    stream = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(k):
        call()
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / k
    nb = psi_h.numel() * psi_h.element_size()
    return {"value": 1e3 / ms, "unit": "force calls/s", "ms_per_call": ms, "h2d_bytes_per_call": nb,
            "d2h_bytes_per_call": nb, "precision": "mixed"}


def ion_form(torch, args):
    """Ion dynamics on the 32-water workload (NVE, atoms starting at 300 K):
    mixed-form CP steps/s with the structure-factor local and nonlocal atom
    forces and with the EES local path (order 6, cp_eext_ees_opt on), beside
    the fixed-ion step, all from one CG-minimised start."""
    import copy
    from openatom_b200.ees import local_grid
    from openatom_b200.gpu import CPDriver
    from openatom_b200.system import atom_masses
    sysm = make_sys(args.config, args.seed)
    psi0, _ = minimized_start(sysm, iters=300)
    m = atom_masses(sysm)
    rng = np.random.default_rng(args.seed)
    vel = rng.standard_normal(sysm.pos.shape) * np.sqrt(300.0 * 3.1668115634556e-6 / m)[:, None]
    out = {}
    k = 10
    variants = (("fixed_ions", None, False), ("ions_sf", None, True), ("ions_ees_local6", 6, True))
    for name, order, moving in variants:
        s2 = copy.copy(sysm)
        s2.pos = sysm.pos.copy()
        if order:
            s2.eext_ees = local_grid(s2, 1.2, order) + (order,)
        d = CPDriver(s2, "mixed", psi0=psi0, norb_tol=NORB_TOL)
        if moving:
            d.ctx.set_ions(m, vel)
        st = d.native_state(use_graph=True)
        d.run_native(st, 3)
        ms, _ = time_steps(torch, d, st, k)
        out[name] = {"value": 1e3 / ms, "ms_per_step": ms}
        if order:
            out[name]["grid"] = list(s2.eext_ees[:3])
        d.ctx.close()
        del d
    torch.cuda.empty_cache()
    return {"workload": f"{args.config} with moving atoms: {sysm.natm // 3} H2O, {sysm.nstate} states, "
                        f"NVE from 300 K", "steps": k, "precision": "mixed", **out}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    def __init__(self, idx):
        self.idx = idx
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                f = [x.strip() for x in out.stdout.strip().split(",")]
                if len(f) >= 7:
                    self.samples.append(f)
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


TERMS = ("EKE", "EHART", "EEXT", "EEXC", "ENL", "EGGA")
NORB_TOL = 0.003


def total_energy(en):
    """E_KS + E_NL of the orthonormal states (the Ewald energy of the fixed
    ions is a constant and left out)."""
    return sum(en[k] for k in TERMS)


def conserved_energy(en):
    """The CP constant of motion with fixed ions: E_KS + E_NL + fictitious KE."""
    return total_energy(en) + en["FICT_KE"]


QUENCH_DT = 10.0   # damped steps after the first three (steepest-descent step dt^2 / 2m)


def quench_schedule(nq):
    """(steps, dt) of the damped quench of the random start: three steps at
    the system's dt, then the rest at QUENCH_DT."""
    first = min(3, nq)
    return [(first, None), (nq - first, QUENCH_DT)]


def workload_config(args, sysm):
    """The config object both arms print for the headline workload."""
    return {"workload": f"{args.config}: {sysm.natm // 3} H2O, {sysm.nstate} states, {sysm.ecut_ry:g} Ry, "
                        f"{sysm.nfft[0]}^3, ng={sysm.ng}",
            "nstate": sysm.nstate, "grid": list(sysm.nfft), "dt": sysm.dt, "fict_mass": sysm.cmass0,
            "quench_steps": args.quench, "quench_dt": [sysm.dt, QUENCH_DT], "norb_tol": NORB_TOL,
            "seed": args.seed,
            "l2": "per-step working set > 126 MB L2 (z-line buffer alone 244 MB in FP32); no explicit flush",
            "parallelism": f"replicas x{args.gpus}"}


# ----------------------------------------------------------------------------
# CPU arm: the oracle port on the host cores (only here and in the reference
# arm does bench.py execute oracle code)
# ----------------------------------------------------------------------------

def cpu_info():
    model = ""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"cpu_model": model, "threads": os.cpu_count() or 1,
            "fft": "scipy.fft (pocketfft/ducc, r2c/c2r) with all host threads", "gemm": "numpy BLAS"}


def oracle_steps(sysm, psi0, nsteps, warm=0):
    """nsteps oracle CP steps from psi0 (None: the seeded start) with the
    PsiV tolerance of the GPU arm.  Returns (steps/s, seconds, records)."""
    from oracle import cp_oracle as O
    O.set_fft_workers(os.cpu_count() or 1)
    st = O.CPState(sysm)
    if psi0 is not None:
        st.psi_t = psi0.copy()
        st.psi = psi0.copy()
    for _ in range(warm):
        O.cp_step(st, sysm, norb_tol=NORB_TOL)
    t0 = time.perf_counter()
    recs = [O.cp_step(st, sysm, norb_tol=NORB_TOL) for _ in range(nsteps)]
    dt = time.perf_counter() - t0
    return nsteps / dt, dt, recs


def per_term_errors(got, ref, natm):
    """max over steps of |got - ref| per energy term (Ha) and of the total per atom."""
    out = {k: max(abs(g[k] - r[k]) for g, r in zip(got, ref)) for k in TERMS}
    out["total_per_atom"] = max(abs(total_energy(g) - total_energy(r)) for g, r in zip(got, ref)) / natm
    out["steps"] = min(len(got), len(ref))
    return out


def run_reference(args):
    """The reference arm: the FP64 oracle port of the CP step on the host
    cores, from the same seeded start quenched the same way (damped CP,
    args.quench steps), then W + K CPMD steps with the same PsiV tolerance."""
    ws, rk, lr = dist_env()
    if rk != 0:
        return 0
    from oracle import cp_oracle as O
    sysm = make_sys(args.config, args.seed)
    O.set_fft_workers(os.cpu_count() or 1)
    st = O.CPState(sysm)
    tq = time.perf_counter()
    for n, dtq in quench_schedule(args.quench):
        O.quench(st, sysm, n, dt=dtq)
    tq = time.perf_counter() - tq
    for _ in range(args.warmup):
        O.cp_step(st, sysm, norb_tol=NORB_TOL)
    t0 = time.perf_counter()
    recs = [O.cp_step(st, sysm, norb_tol=NORB_TOL) for _ in range(args.steps)]
    dt = time.perf_counter() - t0
    finite = all(math.isfinite(r[k]) for r in recs for k in TERMS + ("FICT_KE", "SMAX"))
    if not finite:
        print(json.dumps({"impl": "reference", "unavailable": "the oracle produced non-finite energies"}))
        return 0
    rate = args.steps / dt
    info = cpu_info()
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded water box, random Loewdin start quenched by damped CP)",
        "config": workload_config(args, sysm),
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": info["threads"], "kind": "port",
                         "sample": f"{args.steps} full CPMD steps of the FP64 oracle after {args.warmup} warm-up "
                                   f"steps and a {args.quench}-step damped quench ({tq:.0f} s, untimed)",
                         **info},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "energies_last": {k: recs[-1][k] for k in TERMS + ("FICT_KE", "SMAX")},
        "psiv_resets": sum(1 for r in recs if r["SMAX"] > NORB_TOL),
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------
# GPU arm
# ----------------------------------------------------------------------------

def time_steps(torch, drv, state, k, pos_host=None, sync_each=False):
    """K native CP steps between two CUDA events on the launching stream:
    one oa_gpu_cp_run call (steps enqueued back to back, CUDA-graph replay,
    one synchronisation), or K oa_gpu_cp_step calls (one synchronisation per
    step) when sync_each."""
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(drv.stream)
    if sync_each:
        ens = [drv.step_native(state) for _ in range(k)]
    else:
        ens = drv.run_native(state, k, pos_host)
    ev1.record(drv.stream)
    torch.cuda.synchronize()
    return ev0.elapsed_time(ev1) / k, ens


def quenched_start(sysm, nq):
    """The random start after nq damped FP64 CP steps on the GPU (host array)."""
    from openatom_b200.gpu import CPDriver
    d = CPDriver(sysm, "fp64")
    for n, dtq in quench_schedule(nq):
        d.quench(n, dt=dtq)
    psi0 = d.psi.cpu().numpy()
    d.ctx.close()
    return psi0


def minimized_start(sysm, iters=600, tol=1e-3, prec="fp64", **drv_kw):
    """The electronic ground state the reference reaches before dynamics
    (cp_min_opt): three damped steps off the random start, then
    conjugate-gradient minimisation (CPMinimizer, dt = 20) until |F| <= tol
    or iters iterations.  Returns (psi, info)."""
    from openatom_b200.gpu import CPDriver, CPMinimizer
    d = CPDriver(sysm, prec, **drv_kw)
    d.quench(3)
    m = CPMinimizer(d, "cg", dt=20.0)
    recs = m.run(iters, tol=tol)
    psi0 = d.psi.cpu().numpy()
    d.ctx.close()
    return psi0, {"method": "CG minimisation (cp_min_opt), dt 20", "iterations": len(recs),
                  "fmag": recs[-1]["FMAG"], "e_ks": total_energy(recs[-1])}


def native_records(sysm, psi0, prec, nsteps, norb_tol=NORB_TOL):
    from openatom_b200.gpu import CPDriver
    d = CPDriver(sysm, prec, psi0=psi0, norb_tol=norb_tol)
    recs = d.run_native(d.native_state(use_graph=True), nsteps)
    d.ctx.close()
    return recs


def drift_form(torch, args, want_oracle):
    """The precision configuration on 8 H2O (32 states, 70 Ry, 64^3, dt = 5,
    mu = 400): the mixed and the FP64 form for args.drift_steps CPMD steps
    from the same start, the electronic ground state (CG minimisation, as the
    reference runs cp_min_opt before dynamics).  Reports the drift of the CP
    constant of motion of each form, each energy term's largest difference
    between the two forms over the run, and (CPU leg) each term against the
    FP64 oracle over the first 20 steps."""
    sysm = make_sys("w8", args.seed + 3)
    psi0, start = minimized_start(sysm)
    n = args.drift_steps
    recs = {p: native_records(sysm, psi0, p, n) for p in ("fp64", "mixed")}
    # the same runs without the PsiV tolerance reset: the integrator and the
    # orthonormality constraint alone
    from openatom_b200.gpu import OaError
    free = {}
    out = {"workload": f"w8: 8 H2O, {sysm.nstate} states, 70 Ry, 64^3, ng={sysm.ng}", "steps": n,
           "start": start}
    for p in ("fp64", "mixed"):
        try:
            free[p] = native_records(sysm, psi0, p, n, norb_tol=1e30)
        except OaError as ex:
            # without the reset the states leave the Newton-Schulz convergence
            # region: the run is not stable, which is what this records
            out[f"no_psiv_{p}"] = f"unstable: {ex}"
    for tag, rr in (("", recs), ("_no_psiv", free)):
        for p, r in rr.items():
            e = np.array([conserved_energy(x) for x in r])
            out[f"drift_{p}{tag}_per_atom"] = float(e[-1] - e[0]) / sysm.natm
            out[f"drift_{p}{tag}_max_per_atom"] = float(np.max(np.abs(e - e[0]))) / sysm.natm
            out[f"psiv_resets_{p}{tag}"] = sum(1 for x in r if x["SMAX"] > NORB_TOL)
            out[f"smax_max_{p}{tag}"] = max(x["SMAX"] for x in r)
    out["mixed_vs_fp64"] = per_term_errors(recs["mixed"], recs["fp64"], sysm.natm)
    if want_oracle:
        k = min(20, n)
        _, _, ref = oracle_steps(sysm, psi0, k)
        out["fp64_vs_oracle"] = per_term_errors(recs["fp64"][:k], ref, sysm.natm)
        out["mixed_vs_oracle"] = per_term_errors(recs["mixed"][:k], ref, sysm.natm)
    return out


def run_ours(args):
    import torch
    from openatom_b200.gpu import CPDriver
    ws, rk, lr = dist_env()
    torch.cuda.set_device(lr)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    sysm = make_sys(args.config, replica_seed(args.seed, rk))
    natm = sysm.natm

    # quench the random start (untimed), FP64
    psi0 = quenched_start(sysm, args.quench)
    # two drivers from the same quenched state
    d64 = CPDriver(sysm, "fp64", psi0=psi0, norb_tol=NORB_TOL)
    dmx = CPDriver(sysm, "mixed", psi0=psi0, norb_tol=NORB_TOL)
    st64 = d64.native_state(use_graph=True)
    stmx = dmx.native_state(use_graph=True)
    for _ in range(args.warmup):
        d64.step_native(st64)
        dmx.step_native(stmx)

    def barrier():
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    with ClockSampler(lr) as clk:
        barrier()
        ms_mx, en_mx = time_steps(torch, dmx, stmx, args.steps)
        barrier()
        ms_64, en_64 = time_steps(torch, d64, st64, args.steps)
        barrier()
        # end-to-end through the public API: host atom positions copied in
        # before every step, the per-step energy records copied out
        pos_host = torch.from_numpy(np.repeat(np.ascontiguousarray(sysm.pos)[None], args.steps, axis=0)
                                    ).pin_memory().numpy()
        ms_e2e, _ = time_steps(torch, dmx, stmx, args.steps, pos_host=pos_host)
        barrier()
        # the same steps with a host synchronisation after each one
        ms_sync, _ = time_steps(torch, dmx, stmx, args.steps, sync_each=True)
        barrier()
    ms_mx, ms_64, ms_e2e, ms_sync = max_over_ranks([ms_mx, ms_64, ms_e2e, ms_sync], ws)

    # accuracy of the mixed form against FP64 on the same trajectory start
    de = max(abs(total_energy(a) - total_energy(b)) for a, b in zip(en_mx, en_64)) / natm
    s_err = dmx.last_ortho

    # the force half of the step with host psi in and host F out, per call
    force_call = force_call_form(torch, dmx, args.steps)
    # the same timing from the electronic ground state (CG minimisation):
    # the reference's cp_min_opt start, where the PsiV reset fires rarely
    ground = ground_state_form(torch, sysm, args.steps) if (rk == 0 and args.ground > 0) else None
    # per-kernel timing (CUDA events on the launch stream) for the roofline
    kt = dmx.ctx.time_kernels(dmx.psi, reps=5)
    kt64 = d64.ctx.time_kernels(d64.psi, reps=5)
    roof = roofline(sysm, dmx, kt, args.config)
    tuning = {"table": "openatom_b200/tuning/b200.json (openatom_b200.tuner)",
              "mixed": {"source": dmx.ctx.tuning_source, **dmx.ctx.get_tuning()},
              "fp64": {"source": d64.ctx.tuning_source, **d64.ctx.get_tuning()}}
    d64.ctx.close()
    dmx.ctx.close()
    del d64, dmx
    torch.cuda.empty_cache()

    cpu = None
    per_term = None
    if rk == 0 and not args.no_cpu:
        # the first steps from the quenched start in both GPU forms and in the
        # oracle on the host cores: per-term errors against the FP64 oracle,
        # and the oracle's rate (cpu_baseline)
        k = 2
        g64 = native_records(sysm, psi0, "fp64", k)
        gmx = native_records(sysm, psi0, "mixed", k)
        rate, dt, ref = oracle_steps(sysm, psi0, k)
        per_term = {"steps": k, "fp64_vs_oracle": per_term_errors(g64, ref, natm),
                    "mixed_vs_oracle": per_term_errors(gmx, ref, natm)}
        info = cpu_info()
        cpu = {"value": rate, "unit": UNIT, "cores": info["threads"], "kind": "port",
               "sample": f"{k} full CPMD steps of the FP64 oracle from the quenched start ({dt:.1f} s)", **info}

    drift = drift_form(torch, args, rk == 0 and not args.no_cpu) if (rk == 0 and args.drift_steps > 0) else None
    batch = batch_form(torch, args) if (rk == 0 and args.batch > 0) else None
    large = large_form(torch, args) if (rk == 0 and args.large > 0) else None
    blyp = blyp_form(torch, args) if (rk == 0 and args.blyp > 0) else None
    ions = ion_form(torch, args) if (rk == 0 and args.ions > 0) else None

    if rk == 0:
        # kernel launches of one mixed step, counted in its captured CUDA graph
        launches_per_step = stmx.last_kernels
        line = {
            "metric": METRIC, "value": ws * 1e3 / ms_mx, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_mx, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 FFT path + f64 GEMM/ortho/energies (mixed form)",
            "data": "synthetic (seeded water box, random Loewdin start quenched by damped CP)",
            "config": workload_config(args, sysm),
            "fp64": {"value": ws * 1e3 / ms_64, "ms_per_step": ms_64},
            "mixed_over_fp64": ms_64 / ms_mx,
            "dE_per_atom_max": de,
            "per_term_err": per_term,
            "ortho": {"iters": s_err[0], "residual": s_err[1],
                      "smax_max": max(e["SMAX"] for e in en_mx),
                      "psiv_resets": sum(1 for e in en_mx if e["SMAX"] > NORB_TOL),
                      "psiv_resets_fp64": sum(1 for e in en_64 if e["SMAX"] > NORB_TOL)},
            "kernel_ms": kt, "kernel_ms_fp64": kt64,
            "tuning": tuning,
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": {"value": ws * 1e3 / ms_e2e, "unit": UNIT, "h2d_bytes_per_step": 3 * 8 * natm,
                    "d2h_bytes_per_step": 20 * 8},
            "sync_every_step": {"value": ws * 1e3 / ms_sync, "ms_per_step": ms_sync},
            "e2e_force_call": force_call,
            "ground_state_start": ground,
            "gpu_launches": launches_per_step * args.steps,
            "clocks": clk.summary(),
            "drift_1000": drift,
            "batch": batch,
            "large": large,
            "blyp": blyp,
            "ions": ions,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


# DRAM traffic per launch (dram__bytes_read.sum + dram__bytes_write.sum) of
# the plane kernels on the 32-water workload, copied from one ncu capture of
# the same kernels (the run itself cannot read DRAM counters); None for other
# workloads.
TRAFFIC_W32 = {"state_plane_density": 755.4e6, "state_plane_vks": 748.0e6}


def roofline(sysm, drv, kt, config=None):
    """Roofline of the dominant kernel from its algorithmic bytes
    (CPContext.algorithmic_bytes states the per-kernel formulas) and its
    CUDA-event time."""
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    src = "measured" if "hbm_gbs" in peaks else "fallback"
    bytes_per = drv.ctx.algorithmic_bytes()
    # the kernels of the step (the int8 products are timed beside, not in the step)
    name = max((k for k in kt if k in bytes_per), key=lambda k: kt[k])
    b = bytes_per.get(name)
    if b is None:
        return {"kernel": name, "bound": "hbm", "achieved": None, "peak": hbm, "unit": "GB/s", "frac": None,
                "traffic": None, "peak_source": src}
    ach = b / (kt[name] * 1e-3) / 1e9
    traffic = TRAFFIC_W32.get(name) if config == "w32" else None
    return {"kernel": name, "bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
            "traffic": traffic, "traffic_source": "copied from an ncu capture of this kernel on this workload"
            if traffic is not None else None, "algorithmic_bytes": b, "peak_source": src}


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
