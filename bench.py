#!/usr/bin/env python
"""Benchmark: ns/day of full leapfrog steps on the 41,472-atom water box.

A step is one LeapfrogIntegrator iteration (kick + drift with the waters held
rigid by SETTLE, then the periodic cutoff LJ(C2) + Coulomb(C1) force with its
cell-list rebuild) at dt = 1 fs on 13,824 rigid TIP3P-geometry waters (24^3
lattice, box 74.496 A, rc 10, C2 from 9).

Default arm (libpmb200 on B200):
  value  -- device-resident steps (positions/velocities/forces in HBM, one
            CUDA-graph replay per step) that evaluate the LJ and Coulomb
            energies every step, as the reference's leapfrog does; L2 flushed
            (256 MiB write) before every timed step, each step timed with CUDA
            events on the stream it runs on; sum over K steps, max over ranks.
            The same steps without energies are reported as forces_only.
  e2e    -- the same steps through the reference-facing host-buffer C-ABI
            call (pmb200_eval: positions and forces copied host->device, forces
            and energies device->host, every step) with the kick/drift done
            on the host as ProtoMol's integrator does; wall clock per step.
  fp64   -- the same device-resident steps with the plain FP64 pair kernel.
  roofline -- the pair kernel of those steps (dominant, energy launch): 81
            algorithmic flops per unique
            in-cutoff pair over its CUDA-event duration, against the FP32 FMA
            peak measured in-run (the kernel runs on the FP32 pipe; tensor
            cores and HBM are not its bound); traffic from the committed ncu
            summary.
  cpu_baseline -- the reference's own CPU force (oracle/_ref, compiled from
            the reference sources) driving the same leapfrog on one host core.

--workload large: the 327,352-atom ion box (one force evaluation per step)
with both pair kernels, LJ+C1 and the real-space Ewald term; its line's
value is Gpairs/s of whole LJ+C1 evaluations.

--workload batch: 512 independent boxes of 300-6,000 atoms evaluated by one
persistent, graph-captured batched launch with the autotuned schedule,
against one launch sequence per system.

--workload diff: the differentiable form -- Hessian-vector products by
double backward, parameter gradients and a force-matching loss gradient on
the 648- and 41,472-atom boxes.

--impl reference: the reference CPU implementation alone, one independent
replica per host core (the reference force is serial), bounded sample.

Multi-GPU (torchrun): independent replicas, one per GPU (the path has no
exchange step for a single box at this size); value sums ranks' ns/day.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DT_FS = 1.0
FLOPS_PER_PAIR = 81          # algorithmic flops per unique in-cutoff pair
BYTES_PER_ATOM = 84          # algorithmic HBM bytes per atom per evaluation
KERNELS_PER_STEP = 7         # kick_drift_settle, cell_index, scan, scatter, rank_gather,
                             # pair, finalize_reduce (forces and energy sums)
KERNELS_PER_STEP_CLUSTERS = 13  # kick_drift_settle, sc_index, scan, scatter, rank_gather,
                             # sc_columns, sc_build, sc_list, sc_tasks, sc_pair,
                             # sc_finalize, sc_reduce1, reduce2
# ncu summaries holding each energy launch's DRAM bytes (traffic_bytes_per_launch)
TRAFFIC_PROFILE = {"search": "pair_mixed_water41k.md", "clusters": "pair_clusters_water41k.md",
                   "tiles": None}
WORKLOAD = ("water box: 41,472 atoms (13,824 TIP3P-geometry waters, 24^3 lattice, "
            "box 74.496 A), LJ C2 switch 9-10 A + Coulomb C1 cutoff 10 A, leapfrog 1 fs")
METRIC = "ns/day & Gpairs/s, 41k-atom water box: mixed vs FP64 on B200 @<=1e-5 force err"


def ns_per_day(sec_per_step):
    return 0.0864 * DT_FS / sec_per_step


def env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms in the background."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.p = None
        self.out = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader",
                                       "-lms", "200", "-i", str(self.idx)],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.out, _ = self.p.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()
                self.out, _ = self.p.communicate()

    def summary(self):
        if not self.out:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1].split()[0]))
                mx = float(f[2].split()[0])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
def committed_traffic(name="pair_mixed_water41k.md"):
    """Pair-kernel DRAM bytes per launch from a committed ncu summary."""
    path = os.path.join(ROOT, "profiles", name)  # ncu summary
    try:
        txt = open(path).read()
    except OSError:
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", txt)
    return float(m.group(1)) if m else None


def cpu_reference_time(sysd, steps, warmup=0):
    """Seconds per leapfrog step of the reference CPU force on this host, one
    core, after `warmup` untimed steps; (seconds, kind).  The reference's
    force evaluates energies every step, as its integrator asks."""
    from oracle import oracle as O
    if O.ref_available():
        R = O.RefForce(sysd)
        if warmup:
            R.leapfrog(sysd["pos"], sysd["vel"], DT_FS, warmup)
        t0 = time.perf_counter()
        R.leapfrog(sysd["pos"], sysd["vel"], DT_FS, steps)
        dt = time.perf_counter() - t0
        R.close()
        kind = "reference"
    else:
        if warmup:
            O.restate_leapfrog(sysd, sysd["pos"], sysd["vel"], DT_FS, warmup)
        t0 = time.perf_counter()
        O.restate_leapfrog(sysd, sysd["pos"], sysd["vel"], DT_FS, steps)
        dt = time.perf_counter() - t0
        kind = "port"
    return dt / (steps + 1), kind  # steps + 1 force evaluations


def _ref_replica(args):
    steps, warmup, seed = args
    sys.path.insert(0, ROOT)
    from protomoladdon_b200 import water
    s = water.medium_41k(seed=seed)
    t, kind = cpu_reference_time(s, steps, warmup)
    return t, kind


REF_MAX_STEPS = 20   # bounded sample: about 9 s of CPU time per replica


def run_reference(args):
    rank = env_int("RANK", 0)
    if rank != 0:
        return 0
    import multiprocessing as mp
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    steps = max(1, min(args.steps, REF_MAX_STEPS))
    warmup = min(args.warmup, 3)
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(cores) as pool:
        res = pool.map(_ref_replica, [(steps, warmup, 1234 + r) for r in range(cores)])
    wall = time.perf_counter() - t0
    per_step = statistics.mean(t for t, _ in res)
    kind = res[0][1]
    value = cores * ns_per_day(per_step)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "ns/day",
        "n_gpus": args.gpus, "steps": steps, "warmup": warmup, "steps_requested": args.steps,
        "ms_per_step": per_step * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "atoms": 41472, "replicas": cores,
                   "parallelism": f"{cores} independent single-core replicas",
                   "step": "leapfrog step with the reference force (forces and energies)"},
        "cpu_baseline": {"value": value, "unit": "ns/day", "cores": cores, "kind": kind,
                         "sample": f"{steps} timed leapfrog steps (+1 initial force) after "
                                   f"{warmup} untimed ones per replica, {cores} replicas in "
                                   f"parallel, wall {wall:.1f} s"},
        "e2e": {"value": value, "unit": "ns/day", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
def run_ours(args):
    import torch
    from protomoladdon_b200 import _lib, replicas, water
    from protomoladdon_b200.force import (NonbondedCutoffB200SystemForce, PeriodicTopology,
                                          ScalarStructure)
    world = env_int("WORLD_SIZE", 1)
    rank = env_int("RANK", 0)
    local = env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    s = water.medium_41k(seed=replicas.replica_seed(1234, rank))
    n = s["n"]
    widx = water.rigid_waters(s)
    topo = PeriodicTopology.from_dict(s)
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MiB > L2

    def make(prec):
        f = NonbondedCutoffB200SystemForce(s["ron"], s["rc_lj"], s["rc_coul"], s["rc_alg"],
                                           precision=prec, device=local)
        f.set_rigid_waters(topo, widx, water.D_OH, water.D_HH)
        return f

    def device_run(force, flags):
        """W warm-up + K timed device-resident steps, the force evaluated with
        `flags` (PMB200_ENERGY: energies every step, as the reference's
        integrator asks); returns per-step ms list, pair-kernel ms list (the
        same flags), pair count."""
        pos = torch.tensor(s["pos"], dtype=torch.float64, device=dev)
        vel = torch.tensor(s["vel"], dtype=torch.float64, device=dev)
        frc = torch.zeros_like(pos)
        out = torch.zeros(20, dtype=torch.float64, device=dev)
        with torch.cuda.stream(stream):
            force.evaluate_device(topo, pos.data_ptr(), frc.data_ptr(), out.data_ptr(),
                                  _lib.PMB200_ENERGY, stream.cuda_stream)
        stream.synchronize()
        force.sync()
        pairs = force.last_pair_count()
        sp = stream.cuda_stream
        optr = out.data_ptr() if flags else None
        for _ in range(args.warmup):
            force.step_device(topo, pos.data_ptr(), vel.data_ptr(), frc.data_ptr(), DT_FS, sp,
                              out_ptr=optr, flags=flags)
        stream.synchronize()
        e0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        e1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        kms = []
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                e0[k].record(stream)
            force.step_device(topo, pos.data_ptr(), vel.data_ptr(), frc.data_ptr(), DT_FS, sp,
                              out_ptr=optr, flags=flags)
            e1[k].record(stream)
        torch.cuda.synchronize(dev)
        if dist is not None:
            dist.barrier()
        force.sync()
        step_ms = [a.elapsed_time(b) for a, b in zip(e0, e1)]
        # the dominant kernel alone: CUDA events around each directly
        # launched pair kernel on its stream, L2 flushed before each
        force.set_kernel_timing(True)
        for k in range(min(args.steps, 50)):
            with torch.cuda.stream(stream):
                flush.zero_()
            force.evaluate_device(topo, pos.data_ptr(), frc.data_ptr(), optr, flags, sp)
            stream.synchronize()
            kms.append(force.last_kernel_ms())
        force.set_kernel_timing(False)
        force.sync()
        return step_ms, kms, pairs

    # accuracy of the mixed force vs the FP64 CPU oracle at the start positions
    acc = {}
    if rank == 0 and not args.skip_accuracy:
        from oracle import oracle as O
        fo, eo, vo, _ = O.restate_eval(s, s["pos"], virial_mode=0)
        fm = make("mixed")
        F = np.zeros_like(s["pos"])
        E = ScalarStructure()
        fm.evaluate(topo, s["pos"], F, E)
        fm.close()
        acc = {"force_rms_rel_err": float(np.sqrt(((F - fo) ** 2).sum() / (fo ** 2).sum())),
               "energy_rel_err_coulomb": float(abs(E[0] - eo[0]) / abs(eo[0])),
               "energy_rel_err_lj": float(abs(E[1] - eo[1]) / abs(eo[1]))}

    def tune(force):
        """pmb200_autotune on the start positions: the grid's cell size, the
        pair kernel and its warps per i-cell, applied to the context (or the
        pair kernel --pair-kernel names, untuned)."""
        pos = torch.tensor(s["pos"], dtype=torch.float64, device=dev)
        if args.pair_kernel != "auto" and force.precision == "mixed":
            force.set_pair_kernel(args.pair_kernel)
            return {"tuned": False, "kernel_energy": args.pair_kernel,
                    "kernel_forces": args.pair_kernel}
        if args.autotune_reps <= 0:
            return {"tuned": False}
        choice = force.autotune(topo, pos.data_ptr(), reps=args.autotune_reps,
                                stream=stream.cuda_stream)
        choice["grid"] = list(force.grid()[0])
        return choice

    fmix = make(args.precision)
    tuned = {args.precision: tune(fmix)}
    with ClockSampler(local) as clk:
        step_ms, kms, pairs = device_run(fmix, _lib.PMB200_ENERGY)
    clocks = clk.summary()
    # the same steps without energies (the forces an integrator needs when no
    # energy is asked for), reported beside the headline
    fo_ms, fo_kms, _ = device_run(fmix, 0)
    fp64 = None
    if args.precision == "mixed" and not args.skip_fp64:
        f64 = make("fp64")
        tuned["fp64"] = tune(f64)
        s64, k64, _ = device_run(f64, _lib.PMB200_ENERGY)
        f64.close()
        fp64 = (sum(s64), statistics.mean(k64))
    # the other pair kernel of mixed contexts, the supercluster kernel, on
    # the same steps (the autotuner's choice is the headline; this is its
    # alternative, reported beside it)
    other = None
    if (args.precision == "mixed" and not args.skip_alternative and args.pair_kernel == "auto"
            and tuned["mixed"].get("kernel_energy") != "clusters"):
        fc = make("mixed")
        fc.set_pair_kernel("clusters")
        ce_ms, ce_k, _ = device_run(fc, _lib.PMB200_ENERGY)
        cf_ms, cf_k, _ = device_run(fc, 0)
        fc.close()
        other = (statistics.mean(ce_ms), statistics.mean(ce_k), statistics.mean(cf_ms),
                 statistics.mean(cf_k))

    # end to end through the host-buffer C-ABI call (SystemForce::evaluate's
    # replacement): the host integrator does kick + drift + SETTLE, as
    # ProtoMol's leapfrog with a constraint modifier does, and calls the force
    from protomoladdon_b200 import rigid
    # the integrator's arrays in page-locked host memory (the library then
    # transfers positions without a staging copy)
    def pinned_copy(a):
        t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
        v = t.numpy()
        v[...] = a
        return t, v
    _xt, xh = pinned_copy(s["pos"])
    _vt, vh = pinned_copy(s["vel"])
    _ft, F = pinned_copy(np.zeros_like(s["pos"]))
    E = ScalarStructure()
    fmix.evaluate(topo, xh, F, E)
    e2e_steps = min(args.steps, 500)
    e2e_t, integ_t, call_t = [], [], []

    def host_step():
        t0 = time.perf_counter()
        # kick, drift, SETTLE, and the force array zeroed for the next
        # evaluation to add into (StandardIntegrator::calculateForces), in one pass
        rigid.host_kick_drift(xh, vh, F, s["mass"], DT_FS, widx, water.D_OH, water.D_HH,
                              clear_forces=True)
        E.clear()
        t1 = time.perf_counter()
        fmix.evaluate(topo, xh, F, E)
        return t1 - t0, time.perf_counter() - t1

    for _ in range(min(args.warmup, 3)):
        host_step()
    if dist is not None:
        dist.barrier()
    for _ in range(e2e_steps):
        flush.zero_()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        ti, tc = host_step()
        e2e_t.append(time.perf_counter() - t0)
        integ_t.append(ti)
        call_t.append(tc)

    # where an e2e step's force call goes, device-timed with CUDA events on
    # the same buffers: the pinned host->device copy of the positions, the
    # evaluation (cell build, pair kernel, finalize, energy reduction), the
    # device->host copy of forces and energies; the rest of the call is host
    # work (launch, synchronisation, adding the forces into the caller's array)
    def ev_ms(fn, reps=20):
        a = [torch.cuda.Event(enable_timing=True) for _ in range(reps)]
        b = [torch.cuda.Event(enable_timing=True) for _ in range(reps)]
        for k in range(reps):
            with torch.cuda.stream(stream):
                flush.zero_()
                a[k].record(stream)
                fn()
                b[k].record(stream)
        torch.cuda.synchronize(dev)
        return statistics.mean(x.elapsed_time(y) for x, y in zip(a, b))
    dpos = torch.empty((n, 3), dtype=torch.float64, device=dev)
    dfrc = torch.zeros_like(dpos)
    dout = torch.zeros(20, dtype=torch.float64, device=dev)
    # a mixed context reads the forces back in FP32 (pmb200_eval)
    compact = args.precision == "mixed"
    h2d_ms = ev_ms(lambda: dpos.copy_(_xt, non_blocking=True))
    eval_ms = ev_ms(lambda: fmix.evaluate_device(topo, dpos.data_ptr(), dfrc.data_ptr(),
                                                 dout.data_ptr(), _lib.PMB200_ENERGY,
                                                 stream.cuda_stream))

    # the call reads back forces, results and error flag in one copy (3n
    # doubles, or 3n floats to a double boundary, then 21 doubles)
    out_bytes = (4 * ((3 * n + 1) // 2 * 2) if compact else 8 * 3 * n) + 8 * 21
    dres = torch.zeros(out_bytes // 8, dtype=torch.float64, device=dev)
    hres = torch.empty(out_bytes // 8, dtype=torch.float64, pin_memory=True)
    d2h_ms = ev_ms(lambda: hres.copy_(dres, non_blocking=True))
    fmix.close()

    tot_ms = sum(step_ms)
    mean_k = statistics.mean(kms)
    e2e_s = sum(e2e_t) / len(e2e_t)
    tot_ms, e2e_s, mean_k = replicas.max_over_ranks([tot_ms, e2e_s, mean_k], dist, dev)
    ms_step = tot_ms / args.steps
    value = replicas.aggregate_ns_per_day(ms_step, world, DT_FS)

    if rank == 0:
        peak = ctypes_peak(local)
        achieved = FLOPS_PER_PAIR * pairs / (mean_k * 1e-3) / 1e12
        kern_e = tuned.get(args.precision, {}).get("kernel_energy", "search")
        prof = TRAFFIC_PROFILE.get(kern_e)
        traffic = committed_traffic(prof) if prof else None
        line = {
            "metric": METRIC, "value": value, "unit": "ns/day", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.precision == "mixed" else "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "atoms": n, "pairs_per_eval": pairs,
                       "precision": args.precision,
                       "step": "kick + drift + SETTLE + cell rebuild + force with LJ and "
                               "Coulomb energies (every step, as the reference's leapfrog)",
                       "l2": "flushed before every timed step (256 MiB write)",
                       "parallelism": f"{world} independent replica(s), one per GPU"},
            "gpairs_per_s": world * pairs / (ms_step * 1e-3) / 1e9,
            "pair_kernel_ms": mean_k,
            "gpairs_per_s_pair_kernel": pairs / (mean_k * 1e-3) / 1e9,
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak if peak else None,
                         "traffic": traffic,
                         "peak_source": "FP32 FMA throughput measured in this run "
                                        "(pmb200_measure_fp32_peak)",
                         "hbm": {"achieved_gbs": BYTES_PER_ATOM * n / (mean_k * 1e-3) / 1e9,
                                 "peak_gbs": measured_hbm()}},
            "e2e": {"value": world * ns_per_day(e2e_s), "unit": "ns/day",
                    "ms_per_step": e2e_s * 1e3,
                    "h2d_bytes_per_step": 24 * n,
                    "d2h_bytes_per_step": out_bytes},
            "e2e_breakdown": {
                "host_integrator_ms": statistics.mean(integ_t) * 1e3,
                "force_call_ms": statistics.mean(call_t) * 1e3,
                "of_which_device": {"h2d_ms": h2d_ms, "evaluation_ms": eval_ms,
                                    "d2h_ms": d2h_ms},
                "host_side_of_call_ms": statistics.mean(call_t) * 1e3 - (h2d_ms + eval_ms
                                                                         + d2h_ms),
                "note": "host kick/drift/SETTLE on the host's cores; the force call is one "
                        "CUDA-graph replay (copy in, evaluate with energies, copy out) and "
                        "a synchronisation; a mixed context's forces come back in FP32"},
            "forces_only": {"ns_per_day": world * ns_per_day(statistics.mean(fo_ms) * 1e-3),
                            "ms_per_step": statistics.mean(fo_ms),
                            "pair_kernel_ms": statistics.mean(fo_kms),
                            "note": "the same device steps without energies"},
            "autotune": tuned,
            **({"alternative_pair_kernel": {
                "kernel": "clusters (k_sc_pair: device-built supercluster lists, 4x4 tiles)",
                "ms_per_step": other[0], "pair_kernel_ms": other[1],
                "forces_only_ms_per_step": other[2], "forces_only_pair_kernel_ms": other[3],
                "pair_kernel_fp32_frac": (FLOPS_PER_PAIR * pairs / (other[1] * 1e-3) / 1e12
                                          / peak) if peak else None,
                "note": "the same device steps on the supercluster kernel: its pair kernel is "
                        "faster, its per-step list build costs more; the autotuner keeps "
                        "the faster whole step"}} if other else {}),
            "gpu_launches": (KERNELS_PER_STEP_CLUSTERS if kern_e == "clusters"
                             else KERNELS_PER_STEP) * args.steps,
            "clocks": clocks,
        }
        line.update(acc)
        if fp64 is not None:
            t64 = fp64[0] / args.steps
            line["fp64"] = {"ns_per_day": world * ns_per_day(t64 * 1e-3), "ms_per_step": t64,
                            "pair_kernel_ms": fp64[1],
                            "mixed_speedup": t64 / ms_step,
                            "pair_kernel_speedup": fp64[1] / mean_k,
                            "kernel": "k_pair_fp64_half: the mixed kernel's half-shell task "
                                      "split and box culling in FP64, each pair once, exact "
                                      "fixed-point force sums; the same device steps"}
        if world == 1 and not args.skip_cpu:
            cpu_steps = args.cpu_steps
            t_cpu, kind = cpu_reference_time(s, cpu_steps)
            line["cpu_baseline"] = {
                "value": ns_per_day(t_cpu), "unit": "ns/day", "cores": 1, "kind": kind,
                "sample": f"{cpu_steps} leapfrog steps (+1 initial force) of the same box, "
                          f"{t_cpu * 1e3:.0f} ms per step, serial reference force with "
                          f"energies"}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


LARGE_WORKLOAD = ("ion water box: 327,352 atoms (110,592 lattice sites, 48^3 lattice, box "
                  "148.992 A, 2% of waters replaced by Na+/Cl-), rc 12: LJ C2 11-12 A + "
                  "Coulomb C1 12 A, and the Ewald real-space term erfc(0.30 r)/r")
LARGE_METRIC = "Gpairs/s, 331k-atom ion box: LJ+C1 and Ewald real-space kernels, mixed vs FP64"


def run_large(args):
    """The large system's two pair kernels, one evaluation per step.  value =
    unique in-cutoff pairs per second of whole device-resident evaluations
    (cell build + pair kernel + fixed-point finalize) of the LJ+C1 force;
    the Ewald real-space kernel, the FP64 kernels, the pair kernels alone and
    the host-buffer C-ABI call (e2e) are reported beside it."""
    import torch
    from protomoladdon_b200 import water
    from protomoladdon_b200.force import (EwaldRealB200SystemForce,
                                          NonbondedCutoffB200SystemForce, PeriodicTopology,
                                          ScalarStructure)
    if env_int("WORLD_SIZE", 1) > 1 and env_int("RANK", 0) != 0:
        return 0  # one box, one GPU: replicas are the medium workload's business
    dev = torch.device("cuda", env_int("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    s = water.large_331k()
    n = s["n"]
    topo = PeriodicTopology.from_dict(s)
    acc = float(np.exp(-(0.30 * 12.0) ** 2))  # rc = sqrt(-log acc) / alpha = 12 A
    makers = {
        "cutoff": lambda p: NonbondedCutoffB200SystemForce(s["ron"], s["rc_lj"], s["rc_coul"],
                                                           s["rc_alg"], precision=p),
        "ewald_real": lambda p: EwaldRealB200SystemForce(0.30, acc, precision=p),
    }
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    pos = torch.tensor(s["pos"], dtype=torch.float64, device=dev)
    frc = torch.zeros_like(pos)
    out = torch.zeros(20, dtype=torch.float64, device=dev)
    sp = stream.cuda_stream

    def device_times(f):
        f.evaluate_device(topo, pos.data_ptr(), frc.data_ptr(), out.data_ptr(), 1, sp)
        stream.synchronize()
        f.sync()
        pairs = f.last_pair_count()
        for _ in range(args.warmup):
            f.evaluate_device(topo, pos.data_ptr(), frc.data_ptr(), None, 0, sp)
        e0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        e1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        torch.cuda.synchronize(dev)
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                e0[k].record(stream)
            f.evaluate_device(topo, pos.data_ptr(), frc.data_ptr(), None, 0, sp)
            e1[k].record(stream)
        torch.cuda.synchronize(dev)
        f.sync()
        eval_ms = statistics.mean(a.elapsed_time(b) for a, b in zip(e0, e1))
        f.set_kernel_timing(True)
        kms = []
        for _ in range(min(args.steps, 20)):
            with torch.cuda.stream(stream):
                flush.zero_()
            f.evaluate_device(topo, pos.data_ptr(), frc.data_ptr(), None, 0, sp)
            stream.synchronize()
            kms.append(f.last_kernel_ms())
        f.set_kernel_timing(False)
        f.sync()
        return eval_ms, statistics.mean(kms), pairs

    def host_eval(f, reps):
        F = np.zeros_like(s["pos"])
        E = ScalarStructure()
        f.evaluate(topo, s["pos"], F, E)
        ts = []
        for _ in range(reps):
            F[:] = 0.0
            E.clear()
            flush.zero_()
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            f.evaluate(topo, s["pos"], F, E)
            ts.append(time.perf_counter() - t0)
        return statistics.mean(ts), F, E

    peak = ctypes_peak(dev.index)
    res = {}
    with ClockSampler(dev.index) as clk:
        for name, mk in makers.items():
            for prec in ("mixed", "fp64"):
                f = mk(prec)
                eval_ms, k_ms, pairs = device_times(f)
                e2e_s, F, E = host_eval(f, min(args.steps, 20))
                f.close()
                res[(name, prec)] = dict(eval_ms=eval_ms, pair_kernel_ms=k_ms, pairs=pairs,
                                         e2e_ms=e2e_s * 1e3, F=F, E=E)
    clocks = clk.summary()

    def kernel_obj(name, prec):
        r = res[(name, prec)]
        achieved = FLOPS_PER_PAIR * r["pairs"] / (r["pair_kernel_ms"] * 1e-3) / 1e12
        o = {"eval_ms": r["eval_ms"], "pair_kernel_ms": r["pair_kernel_ms"],
             "pairs_per_eval": r["pairs"],
             "gpairs_per_s": r["pairs"] / (r["eval_ms"] * 1e-3) / 1e9,
             "gpairs_per_s_pair_kernel": r["pairs"] / (r["pair_kernel_ms"] * 1e-3) / 1e9,
             "e2e_ms": r["e2e_ms"],
             "roofline": {"bound": "fp32" if prec == "mixed" else "fp64",
                          "achieved": achieved,
                          "peak": peak if prec == "mixed" else None, "unit": "TFLOP/s",
                          "frac": achieved / peak if (peak and prec == "mixed") else None}}
        return o

    line = {
        "metric": LARGE_METRIC, "unit": "Gpairs/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": LARGE_WORKLOAD, "atoms": n,
                   "l2": "flushed before every timed evaluation (256 MiB write)",
                   "step": "one force evaluation (cell build + pair kernel + finalize)"},
    }
    cut = kernel_obj("cutoff", "mixed")
    line["value"] = cut["gpairs_per_s"]
    line["ms_per_step"] = cut["eval_ms"]
    line["roofline"] = dict(cut["roofline"], traffic=None,
                            peak_source="FP32 FMA throughput measured in this run")
    line["kernels"] = {f"{nm}_{p}": kernel_obj(nm, p) for nm in makers for p in ("mixed", "fp64")}
    line["mixed_speedup_vs_fp64"] = {
        nm: res[(nm, "fp64")]["eval_ms"] / res[(nm, "mixed")]["eval_ms"] for nm in makers}
    line["e2e"] = {"value": cut["pairs_per_eval"] / (cut["e2e_ms"] * 1e-3) / 1e9,
                   "unit": "Gpairs/s", "ms_per_step": cut["e2e_ms"],
                   "h2d_bytes_per_step": 24 * n, "d2h_bytes_per_step": 24 * n + 168}
    line["gpu_launches"] = 6 * args.steps  # cell_index, scan, scatter, rank_gather, pair, finalize
    line["clocks"] = clocks
    if not args.skip_accuracy:
        from oracle import oracle as O
        fo, eo, _, _ = O.restate_eval(s, s["pos"], virial_mode=0)
        fe, ee, _, _ = O.restate_ewald_real(s, s["pos"], 0.30, acc, False, virial_mode=0)
        acc_o = {}
        for nm, (fref, eref) in (("cutoff", (fo, eo[0] + eo[1])), ("ewald_real", (fe, ee))):
            for p in ("mixed", "fp64"):
                r = res[(nm, p)]
                acc_o[f"{nm}_{p}"] = {
                    "force_rms_rel_err": float(np.sqrt(((r["F"] - fref) ** 2).sum()
                                                       / (fref ** 2).sum())),
                    "energy_abs_err": float(abs(r["E"][0] + r["E"][1] - eref))}
        line["accuracy_vs_fp64_oracle"] = acc_o
    if not args.skip_cpu:
        from oracle import oracle as O
        t0 = time.perf_counter()
        if O.ref_available():
            R = O.RefForce(s)
            R.evaluate(s["pos"], 0)
            R.close()
            kind = "reference"
        else:
            O.restate_eval(s, s["pos"], virial_mode=0)
            kind = "port"
        t_cpu = time.perf_counter() - t0
        line["cpu_baseline"] = {
            "value": cut["pairs_per_eval"] / t_cpu / 1e9, "unit": "Gpairs/s", "cores": 1,
            "kind": kind, "sample": f"one LJ+C1 evaluation of the same box, {t_cpu:.1f} s"}
    print(json.dumps(line), flush=True)
    return 0


BATCH_WORKLOAD = ("512 independent periodic water boxes, atom counts log-uniform in "
                  "[300, 6000] rounded to whole waters at 0.0334 molecules/A^3 (boxes below "
                  "2 rc grown to 2 rc), rc 9: LJ C2 8-9 A + Coulomb C1 9 A")
BATCH_METRIC = ("Gpairs/s, 512 uneven water boxes: one persistent graph-captured batched "
                "launch (autotuned schedule) vs one launch per system")


def run_sharded(args):
    """--workload sharded: the 327,352-atom ion box's LJ+C1 force split over the
    N GPUs of the job (one process per GPU) by runs of i-cells
    (pmb200_shard_eval_device), the int64 fixed-point accumulators summed by one
    NCCL all-reduce, then converted on every rank (pmb200_shard_finalize).
    value = unique in-cutoff pairs per second of whole evaluations (cell build,
    shard pair kernel, all-reduce, finalize), device-timed, max over ranks;
    strong scaling (the box is the same at every N).  Rank 0 also checks that
    the summed forces equal a one-GPU evaluation bit for bit."""
    import datetime
    import torch
    import torch.distributed as dist
    from protomoladdon_b200 import water
    from protomoladdon_b200.force import NonbondedCutoffB200SystemForce, PeriodicTopology
    from protomoladdon_b200.shard import sharded_evaluate
    world = env_int("WORLD_SIZE", 1)
    rank = env_int("RANK", 0)
    dev = torch.device("cuda", env_int("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    if not dist.is_initialized():
        if "MASTER_ADDR" not in os.environ:  # a plain one-process run
            os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT="29511", RANK="0",
                              WORLD_SIZE="1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)
    s = water.large_331k()
    topo = PeriodicTopology.from_dict(s)
    f = NonbondedCutoffB200SystemForce(s["ron"], s["rc_lj"], s["rc_coul"], s["rc_alg"])
    pos = torch.tensor(s["pos"], dtype=torch.float64, device=dev)
    frc = torch.zeros_like(pos)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    # the reference result and the pair count: one whole evaluation on this GPU
    one = torch.zeros_like(pos)
    out = torch.zeros(20, dtype=torch.float64, device=dev)
    f.evaluate_device(topo, pos.data_ptr(), one.data_ptr(), out.data_ptr(), 1, 1)
    torch.cuda.synchronize(dev)
    f.sync()
    pairs = f.last_pair_count()

    def step():
        frc.zero_()
        sharded_evaluate(f, topo, pos, frc)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    identical = bool(torch.equal(frc, one))
    steps = min(args.steps, 50)
    e0 = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    e1 = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    dist.barrier()
    torch.cuda.synchronize(dev)
    for k in range(steps):
        flush.zero_()
        e0[k].record()
        step()
        e1[k].record()
    torch.cuda.synchronize(dev)
    dist.barrier()
    ms = statistics.mean(a.elapsed_time(b) for a, b in zip(e0, e1))
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    f.sync()
    f.close()
    dist.destroy_process_group()
    if rank == 0:
        print(json.dumps({
            "metric": "Gpairs/s, 327k-atom ion box split over N GPUs (LJ+C1, mixed)",
            "value": pairs / (ms * 1e-3) / 1e9, "unit": "Gpairs/s", "n_gpus": world,
            "steps": steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": "327,352-atom water box with 2% Na+/Cl-, rc 12 A, one force "
                                   "evaluation per step split by i-cell runs over the ranks",
                       "pairs_per_eval": pairs, "l2": "flushed before every timed step",
                       "parallelism": f"force decomposition over {world} GPU(s)"},
            "bit_identical_to_one_gpu": identical,
        }), flush=True)
    return 0


def _batch_cpu_worker(indices):
    """Seconds the reference's CPU force takes for the given systems of the
    512-box batch, evaluated one after another in this process."""
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    from protomoladdon_b200 import water
    boxes = water.batch_boxes(count=512, seed=1234)
    ref = O.ref_available()
    t = 0.0  # evaluations only (the topology set-up is not timed)
    for k in indices:
        s = boxes[k]
        if ref:
            R = O.RefForce(s)
            t0 = time.perf_counter()
            R.evaluate(s["pos"], 0)
            t += time.perf_counter() - t0
            R.close()
        else:
            t0 = time.perf_counter()
            O.restate_eval(s, s["pos"], virial_mode=0)
            t += time.perf_counter() - t0
    return t, "reference" if ref else "port"


def run_batch(args):
    """All 512 systems' forces per step.  value = unique in-cutoff pairs per
    second over the whole batch, device-resident, one CUDA-graph replay per
    step (L2 flushed before each); beside it the same step as one
    evaluation launch sequence per system, the pair kernel alone, the
    autotuner's choice, and an end-to-end step with positions copied in and
    forces copied out through pinned host buffers."""
    import torch
    from protomoladdon_b200 import _lib, water
    from protomoladdon_b200.batch import SystemBatch
    from protomoladdon_b200.force import NonbondedCutoffB200SystemForce, PeriodicTopology
    if env_int("WORLD_SIZE", 1) > 1 and env_int("RANK", 0) != 0:
        return 0
    dev = torch.device("cuda", env_int("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    boxes = water.batch_boxes(count=512, seed=1234)
    members = [(NonbondedCutoffB200SystemForce(s["ron"], s["rc_lj"], s["rc_coul"], s["rc_alg"]),
                PeriodicTopology.from_dict(s)) for s in boxes]
    batch = SystemBatch(members)
    N = batch.n_atoms
    stream = torch.cuda.Stream(device=dev)
    sp = stream.cuda_stream
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    pos = torch.tensor(np.concatenate([s["pos"] for s in boxes]), dtype=torch.float64,
                       device=dev)
    frc = torch.zeros_like(pos)
    out = torch.zeros((len(boxes), 20), dtype=torch.float64, device=dev)
    # pair counts (one evaluation with energies)
    batch.eval_device(pos.data_ptr(), frc.data_ptr(), out.data_ptr(), _lib.PMB200_ENERGY, sp)
    stream.synchronize()
    counts = batch.pair_counts()
    pairs = int(counts.sum())
    default_sched = batch.schedule()
    tune = batch.autotune(pos.data_ptr(), sp, reps=3)

    def timed(fn, steps):
        e0 = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        e1 = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        torch.cuda.synchronize(dev)
        for k in range(steps):
            with torch.cuda.stream(stream):
                flush.zero_()
                e0[k].record(stream)
            fn()
            e1[k].record(stream)
        torch.cuda.synchronize(dev)
        return [a.elapsed_time(b) for a, b in zip(e0, e1)]

    def batched():
        batch.eval_device(pos.data_ptr(), frc.data_ptr(), None, 0, sp)

    offs = batch.offsets
    views = [(pos[offs[k]:offs[k + 1]], frc[offs[k]:offs[k + 1]]) for k in range(len(boxes))]

    def one_by_one():
        for (f, t), (p, fr) in zip(members, views):
            f.evaluate_device(t, p.data_ptr(), fr.data_ptr(), None, 0, sp)

    with ClockSampler(dev.index) as clk:
        for _ in range(args.warmup):
            batched()
        ms_batch = timed(batched, args.steps)
        for _ in range(args.warmup):
            one_by_one()
        ms_loop = timed(one_by_one, min(args.steps, 20))
        batch.set_kernel_timing(True)
        kms = []
        for _ in range(min(args.steps, 20)):
            with torch.cuda.stream(stream):
                flush.zero_()
            batched()
            stream.synchronize()
            kms.append(batch.last_kernel_ms())
        batch.set_kernel_timing(False)
        # end to end: pinned host positions in, forces out, every step
        hpos = torch.empty(pos.shape, dtype=torch.float64, pin_memory=True)
        hpos.copy_(pos)
        hfrc = torch.empty(pos.shape, dtype=torch.float64, pin_memory=True)
        e2e = []
        for k in range(min(args.steps, 20) + 2):
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            with torch.cuda.stream(stream):
                pos.copy_(hpos, non_blocking=True)
                frc.zero_()
            batched()
            with torch.cuda.stream(stream):
                hfrc.copy_(frc, non_blocking=True)
            stream.synchronize()
            if k >= 2:
                e2e.append(time.perf_counter() - t0)
    clocks = clk.summary()
    t_batch = statistics.mean(ms_batch)
    t_loop = statistics.mean(ms_loop)
    k_ms = statistics.mean(kms)
    peak = ctypes_peak(dev.index)
    achieved = FLOPS_PER_PAIR * pairs / (k_ms * 1e-3) / 1e12
    line = {
        "metric": BATCH_METRIC, "value": pairs / (t_batch * 1e-3) / 1e9, "unit": "Gpairs/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_batch,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": BATCH_WORKLOAD, "systems": len(boxes), "atoms": N,
                   "atoms_min": int(batch.sizes.min()), "atoms_max": int(batch.sizes.max()),
                   "pairs_per_step": pairs,
                   "l2": "flushed before every timed step (256 MiB write)",
                   "step": "forces of every system (no energies)"},
        "schedule": {"default": default_sched, "autotuned": tune},
        "one_launch_per_system": {"ms_per_step": t_loop,
                                  "gpairs_per_s": pairs / (t_loop * 1e-3) / 1e9,
                                  "batched_speedup": t_loop / t_batch},
        "pair_kernel_ms": k_ms,
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak if peak else None,
                     "traffic": committed_traffic("pair_mixed_batch_512boxes.md"),
                     "peak_source": "FP32 FMA throughput measured in this run"},
        "e2e": {"value": pairs / statistics.mean(e2e) / 1e9, "unit": "Gpairs/s",
                "ms_per_step": statistics.mean(e2e) * 1e3,
                "h2d_bytes_per_step": 24 * N, "d2h_bytes_per_step": 24 * N},
        "gpu_launches": 6 * args.steps,  # cell_index, scan, scatter, rank_gather, pair, finalize
        "clocks": clocks,
    }
    if not args.skip_cpu:
        # the reference's force on every host core: one process per core, the
        # sample's systems dealt round-robin, throughput over the slowest
        import multiprocessing as mp
        cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
        nsample = len(boxes)  # every system: about a second per process
        shares = [list(range(w, nsample, cores)) for w in range(cores)]
        with mp.get_context("spawn").Pool(cores) as pool:
            res = pool.map(_batch_cpu_worker, shares)
        t_cpu = max(t for t, _ in res)
        npair = int(sum(int(c) for c in counts[:nsample]))
        line["cpu_baseline"] = {
            "value": npair / t_cpu / 1e9, "unit": "Gpairs/s", "cores": cores, "kind": res[0][1],
            "sample": f"all {nsample} systems, {cores} processes (one per core, systems "
                      f"dealt round-robin), slowest process {t_cpu:.2f} s"}
    batch.close()
    for f, _ in members:
        f.close()
    print(json.dumps(line), flush=True)
    return 0


DIFF_WORKLOAD = ("differentiable form on the 648- and 41,472-atom water boxes: 32 seeded unit "
                 "Hessian-vector products by double backward, dE/dq and dE/dsigma, dE/depsilon "
                 "per type, and the force-matching loss sum |F(theta) - F_target|^2 "
                 "(targets from 5% seeded Gaussian parameter perturbations) with its gradient")
DIFF_METRIC = "Hessian-vector products per second, 41k-atom water box (FP64 derivative kernel)"


def run_diff(args):
    """The differentiable form, timed with CUDA events through the torch
    autograd API (positions resident on the device): Hessian-vector products
    (value, on the 41k box), parameter gradients and the force-matching loss
    gradient, with the accuracy of one product against central differences
    of the FP64 oracle."""
    import torch
    from protomoladdon_b200 import water
    from protomoladdon_b200.autograd import NonbondedEnergy, lj_table
    if env_int("WORLD_SIZE", 1) > 1 and env_int("RANK", 0) != 0:
        return 0
    dev = torch.device("cuda", env_int("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    res = {}
    with ClockSampler(dev.index) as clk:
        for name, s in (("water648", water.small_648()), ("water41k", water.medium_41k())):
            m = NonbondedEnergy.from_system(s, precision="fp64")
            q, t = m.initial_params(device=dev)
            pos = torch.tensor(s["pos"], dtype=torch.float64, device=dev, requires_grad=True)
            rng = np.random.default_rng(2024)
            vs = []
            for _ in range(32):
                v = rng.standard_normal(s["pos"].shape)
                vs.append(torch.tensor(v / np.linalg.norm(v), device=dev))
            E = m.energy(pos, q, t)
            (g,) = torch.autograd.grad(E, pos, create_graph=True)

            def timed(fn, reps):
                for _ in range(max(args.warmup, 3)):
                    fn(0)
                torch.cuda.synchronize(dev)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                for k in range(reps):
                    fn(k)
                e1.record()
                torch.cuda.synchronize(dev)
                return e0.elapsed_time(e1) / reps

            hv_ms = timed(lambda k: torch.autograd.grad(g, pos, grad_outputs=vs[k % 32],
                                                        retain_graph=True), 32)
            sig = torch.tensor([3.1507, 0.0], dtype=torch.float64, device=dev, requires_grad=True)
            eps = torch.tensor([0.1521, 0.0], dtype=torch.float64, device=dev, requires_grad=True)
            qq = q.clone().requires_grad_(True)

            def param_grad(k):
                torch.autograd.grad(m.energy(pos.detach(), qq, lj_table(sig, eps)), (qq, sig, eps))
            pg_ms = timed(param_grad, 10)
            F_t = (-m.gradient(pos.detach(), q * 1.03, lj_table(sig * 1.02, eps * 0.97))).detach()

            def loss_grad(k):
                F = m.forces(pos.detach(), qq, lj_table(sig, eps))
                torch.autograd.grad(((F - F_t) ** 2).sum(), (qq, sig, eps))
            lg_ms = timed(loss_grad, 10)
            acc = None
            if not args.skip_accuracy:
                from oracle import oracle as O
                v = vs[0].cpu().numpy()
                (hv,) = torch.autograd.grad(g, pos, grad_outputs=vs[0], retain_graph=True)
                h = 1e-4
                fp, _, _, _ = O.restate_eval(s, s["pos"] + h * v, virial_mode=0)
                fm, _, _, _ = O.restate_eval(s, s["pos"] - h * v, virial_mode=0)
                fd = -(fp - fm) / (2 * h)
                acc = float(np.linalg.norm(hv.cpu().numpy() - fd) / np.linalg.norm(fd))
            m.close()
            res[name] = {"atoms": s["n"], "hvp_ms": hv_ms, "hvp_per_s": 1e3 / hv_ms,
                         "param_grad_ms": pg_ms, "loss_grad_ms": lg_ms,
                         "hvp_rel_err_vs_fd": acc}
    clocks = clk.summary()
    big = res["water41k"]
    line = {
        "metric": DIFF_METRIC, "value": big["hvp_per_s"], "unit": "HVP/s", "n_gpus": 1,
        "steps": 32, "warmup": max(args.warmup, 3), "ms_per_step": big["hvp_ms"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": DIFF_WORKLOAD, "step": "one Hessian-vector product (41k box)",
                   "l2": "not flushed: derivative passes run back to back as in an "
                         "optimizer loop, the ~6 MB working set staying in L2"},
        "systems": res, "gpu_launches": 32 * 6, "clocks": clocks,
        "e2e": {"value": big["hvp_per_s"], "unit": "HVP/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def ctypes_peak(device):
    import ctypes
    from protomoladdon_b200 import _lib
    v = ctypes.c_double()
    rc = _lib.lib().pmb200_measure_fp32_peak(int(device), ctypes.byref(v))
    return v.value if rc == 0 else None


def measured_hbm():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]
    except Exception:
        return 6650.0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--cpu-steps", type=int, default=20)
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-fp64", action="store_true")
    ap.add_argument("--skip-alternative", action="store_true",
                    help="do not time the supercluster kernel beside the autotuned one")
    ap.add_argument("--skip-accuracy", action="store_true")
    ap.add_argument("--pair-kernel", default="auto", choices=["auto", "search", "clusters"],
                    help="mixed pair kernel: auto (pmb200_autotune) or a fixed one")
    ap.add_argument("--autotune-reps", type=int, default=10,
                    help="timed launches per configuration of pmb200_autotune (0: no tuning, "
                         "the library's default grid and kernel)")
    ap.add_argument("--workload", default="medium",
                    choices=["medium", "large", "batch", "diff", "sharded"],
                    help="medium: the 41,472-atom water box (the headline); large: the "
                         "327,352-atom ion box's LJ+C1 and Ewald real-space kernels; batch: "
                         "512 uneven boxes in one batched launch; diff: the differentiable "
                         "form (Hessian-vector products, parameter gradients); sharded: "
                         "the 327k-atom box's force split over the job's GPUs")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "large":
        return run_large(args)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "diff":
        return run_diff(args)
    if args.workload == "sharded":
        return run_sharded(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
