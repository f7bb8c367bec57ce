#!/usr/bin/env python
"""Throughput benchmark of the per-step MHD hot path on B200.

Metric: zone-cycles/s (one cell advanced by one full SSP-RK3 step) and the
fraction of the measured HBM peak.  Default workload (one GPU): the MHD rotor,
1024^2, outflow on every side, HLLE + MC + MOOD, plain FP64 -- the drop-in
configuration.  Synthetic seeded / analytic initial states; no dataset.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl chimera|reference]

N > 1 (launched by torch.distributed.run): every rank advances its own replica
(the single-grid path does not shard; weak scaling, no data-path collective);
timing is the max over ranks.  --impl reference times the reference algorithm's
CPU implementation (the FP64 restatement, OpenMP on all host threads) on the
same workload.
"""
from __future__ import annotations

import argparse
import glob
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_ZC_FP64 = 384      # 8 accesses x 6 fields x 8 B over the three stages
STAGE_ACCESSES = {1: 12, 2: 18, 3: 18}   # field accesses per cell per stage launch
WORKLOAD = "MHD rotor 1024x1024, outflow all sides, HLLE + MC + MOOD, gamma 1.4, FP64 plain"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=40)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=("chimera", "reference"), default="chimera")
    p.add_argument("--n", type=int, default=1024, help="grid size (default: the rotor workload)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--precision", choices=("fp64", "fp32"), default="fp64",
                   help="precision form of the rotor measurement")
    p.add_argument("--ensemble", choices=("on", "off", "only"), default="on",
                   help="also measure the FP32-batched GRF ensemble against the FP64 form")
    p.add_argument("--ens-scale", type=int, default=1,
                   help="divide the ensemble member counts (1 = 256x128^2 + 192x256^2 + 64x512^2)")
    p.add_argument("--ens-steps", type=int, default=200)
    p.add_argument("--ens-variant", type=int, default=-1,
                   help="force a tile variant for the FP32-batched ensemble (-1: autotune)")
    p.add_argument("--ens-forms", default="fp32,fp32mixed,fp64",
                   help="ensemble forms to measure (the L1 comparison needs both)")
    p.add_argument("--kh", choices=("on", "off"), default="on",
                   help="also measure the Kelvin-Helmholtz HLLD comparison (FP32-bulk vs FP64)")
    p.add_argument("--kh-n", type=int, default=4096)
    p.add_argument("--kh-steps", type=int, default=1000)
    p.add_argument("--kh-variant", type=int, default=-1,
                   help="force a tile variant for the FP64 form of the Kelvin-Helmholtz leg (-1: autotune)")
    p.add_argument("--adjoint", choices=("on", "off"), default="on",
                   help="also measure the field-loop adjoint (forward + backward, central differences)")
    p.add_argument("--adj-steps", type=int, default=400, help="RK3 steps of the field-loop adjoint leg")
    p.add_argument("--adj-k", type=int, default=20, help="checkpoint interval of the adjoint leg")
    p.add_argument("--slabs", type=int, default=0,
                   help="also run the FP64 Kelvin-Helmholtz grid as this many y-slabs on one GPU "
                        "(ghost-row exchange by device copies) against the undivided grid (0: off)")
    p.add_argument("--ref-seconds", type=float, default=10.0,
                   help="seconds of CPU work per timed sample of the CPU restatement (reference arm and "
                        "cpu_baseline)")
    p.add_argument("--variant", type=int, default=-1,
                   help="force a tile variant for the single-grid measurement (-1: autotune)")
    return p.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_value(kind, key):
    """A per-kernel figure from a committed ncu summary: ``profiles/*.md``
    lines of the form ``<kind>[<key>]: <number>`` (kind ``traffic``: DRAM
    bytes per launch; kind ``instructions``: thread instructions per cell)."""
    pat = re.compile(r"\s*" + re.escape(kind) + r"\[(.+?)\]:\s*([0-9.eE+]+)")
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        with open(path) as f:
            for line in f:
                m = pat.match(line)
                if m and m.group(1) == key:
                    return float(m.group(2))
    return None


def profile_traffic(key):
    return profile_value("traffic", key)


def issue_roofline(inst_per_cell, cells, launch_ms, sm_mhz, n_sms):
    """The instruction-issue roofline of a compute-bound kernel: warp
    instructions issued per second (the ncu instruction count per cell x cells
    / 32, over the live launch time) against 4 warp instructions per clock per
    SM (one per scheduler) at the SM clock sampled during the timed region."""
    if inst_per_cell is None or not sm_mhz:
        return None
    achieved = inst_per_cell * cells / 32.0 / (launch_ms * 1e-3) / 1e9
    peak = 4.0 * n_sms * sm_mhz * 1e6 / 1e9
    return {"bound": "issue", "achieved": achieved, "peak": peak, "unit": "G warp-instructions/s",
            "frac": achieved / peak, "instructions_per_cell": inst_per_cell,
            "peak_kind": f"4 per clock per SM x {n_sms} SMs at the sampled {sm_mhz:.0f} MHz"}


class Clocks:
    """SM clock and clock-event reasons sampled DURING the timed region: an
    NVML poll every ~2 ms on a background thread (read-only queries), so that
    even short regions get samples; nvidia-smi (200 ms) if NVML is missing."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.smax = None
        self._stop = None
        self._thread = None
        self._smi = None

    def start(self):
        import threading
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.smax = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            bits = {"hw_slowdown": pynvml.nvmlClocksEventReasonHwSlowdown,
                    "hw_thermal_slowdown": pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                    "sw_thermal_slowdown": pynvml.nvmlClocksEventReasonSwThermalSlowdown,
                    "sw_power_cap": pynvml.nvmlClocksEventReasonSwPowerCap}
            self._stop = threading.Event()

            def poll():
                while not self._stop.is_set():
                    try:
                        sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                        r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                        self.samples.append((float(sm), [k for k, b in bits.items() if r & b]))
                    except Exception:
                        pass
                    self._stop.wait(0.002)

            self._thread = threading.Thread(target=poll, daemon=True)
            self._thread.start()
        except Exception:
            self._smi = _SmiClocks(self.index)
            self._smi.start()

    def stop(self):
        if self._smi is not None:
            return self._smi.stop()
        if self._thread is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        self._stop.set()
        self._thread.join(timeout=2)
        sm = [x for x, _ in self.samples]
        reasons = sorted({r for _, rs in self.samples for r in rs})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.smax,
                "reasons": reasons, "samples": len(sm), "source": "nvml"}


class _SmiClocks:
    """nvidia-smi samples (200 ms) during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax = float(parts[2])
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi"}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def dist_max(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_model():
    """The host CPU's model name (first /proc/cpuinfo entry), or the platform's."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def cpu_reference_rate(n, repeats=3, seconds=10.0, omp_mode=2):
    """The CPU restatement of the reference on the same workload, all host
    threads: zone-cycles/s of ``repeats`` timed samples of at least
    ``seconds`` each, all from one warm state (two untimed steps first).  Each
    sample is one oracle call of k steps, k calibrated from one timed step, so
    the per-call set-up of the oracle's work arrays is amortised.  omp_mode 2
    threads every loop; 1 threads only the three loops the reference threads.
    Returns a dict with the median rate, the spread, the per-sample rates, the
    cores used and the CPU model."""
    from chimera_b200 import problems
    from oracle import oracle
    oracle.build()
    oracle.set_omp_mode(omp_mode)
    # every core this process may run on, also under torchrun (which sets
    # OMP_NUM_THREADS=1 for its ranks)
    oracle.set_threads(len(os.sched_getaffinity(0)))
    cfg, st = problems.rotor(n)
    cfg = cfg.replace(t_end=1e30)
    s = oracle.State(st)
    oracle.run(cfg, s, 2)                      # warm-up (page-in, thread start)
    t0 = time.perf_counter()
    oracle.run(cfg, s, 1)                      # calibration step
    t1 = time.perf_counter() - t0
    k = max(1, int(seconds / max(t1, 1e-6) + 0.999))
    rates, steps, total = [], 0, 0.0
    for _ in range(repeats):
        t0 = time.perf_counter()
        oracle.run(cfg, s, k)
        el = time.perf_counter() - t0
        rates.append(n * n * k / el)
        steps += k
        total += el
    cores = oracle.max_threads()
    oracle.set_omp_mode(0)
    med = statistics.median(rates)
    return {"value": med, "rates": rates, "spread": (max(rates) - min(rates)) / med, "cores": cores,
            "steps": steps, "seconds": total, "steps_per_sample": k, "cpu_model": cpu_model(),
            "ms_per_step": 1e3 * n * n / med}


def run_reference(args, world, rank):
    if rank != 0:
        return
    # three timed samples of >= 10 s each, as cpu_baseline takes them: the host's all-core
    # clock settles over the first minute of load, so both take the same number
    r = cpu_reference_rate(args.n, repeats=3, seconds=args.ref_seconds)
    rate = r["value"]
    line = {
        "impl": "reference",
        "metric": "zone-cycles/s", "value": rate, "unit": "zone-cycles/s", "n_gpus": args.gpus,
        "steps": r["steps"], "warmup": 3, "ms_per_step": r["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD.replace("FP64 plain", "FP64, CPU"), "cells": args.n * args.n},
        "cpu_baseline": {"value": rate, "unit": "zone-cycles/s", "cores": r["cores"], "kind": "port",
                         "cpu_model": r["cpu_model"], "spread": r["spread"], "rates": r["rates"],
                         "sample": f"median of {len(r['rates'])} samples of {r['steps_per_sample']} RK3 steps "
                                   f"({r['seconds']:.1f} s in all) of the {args.n}^2 rotor from one warm state "
                                   f"(FP64 C restatement of the reference Fortran, OpenMP on every loop)"},
        "e2e": {"value": rate, "unit": "zone-cycles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_chimera(args, world, rank, local):
    import torch
    from chimera_b200 import gpu, problems
    from chimera_b200.config import FP32_BULK, FP64

    torch.cuda.set_device(local)
    ens = None
    if args.ensemble != "off":
        ens = run_ensemble(args, world)
        if args.ensemble == "only":
            if rank == 0:
                print(json.dumps({"ensemble": ens}), flush=True)
            return
    n = args.n
    cells = n * n
    cfg, st = problems.rotor(n)
    prec = FP32_BULK if args.precision == "fp32" else FP64
    esize = 4 if prec == FP32_BULK else 8
    cfg = cfg.replace(t_end=1e30, precision=prec)   # keep stepping past t=0.15; per-step work is unchanged
    s = gpu.Solver(cfg)
    s.set_state(st)
    ext = torch.cuda.ExternalStream(s.stream)
    s.step(args.warmup)
    if args.variant >= 0:
        s.set_variant(args.variant)
    else:
        s.autotune(reps=3)                      # tile shape for this problem (cached per shape)
    vinfo = s.variant()
    torch.cuda.synchronize()

    # --- device-resident throughput (inputs resident in HBM; the three state sets,
    #     3 x 48 MB, exceed the 126 MB L2, so no flush is needed between steps)
    clocks = Clocks(local)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    e0.record(ext)
    s.step(args.steps)
    e1.record(ext)
    e1.synchronize()
    ck = clocks.stop()
    torch.cuda.synchronize()
    barrier(world)
    ms = dist_max(e0.elapsed_time(e1), world)
    d = s.diag()
    if d["status"] != 0:
        raise RuntimeError(f"device status {d['status']} after the timed steps")
    value = world * cells * args.steps / (ms * 1e-3)

    # --- per-kernel device time (CUDA events around each launch, eager path)
    s.set_profiling(True)
    s.get_profile(reset=True)
    s.step(min(args.steps, 20))
    prof = s.get_profile(reset=True)
    s.set_profiling(False)
    avg = {k: v["ms"] / v["launches"] for k, v in prof.items() if v["launches"]}
    dom = max((k for k in avg if k.startswith("stage")), key=lambda k: avg[k])
    kidx = int(dom[-1])
    alg_bytes = STAGE_ACCESSES[kidx] * esize * cells
    hbm, peak_kind = peaks()
    achieved = alg_bytes / (avg[dom] * 1e-3) / 1e9
    # the committed ncu figures of the tile variant this run uses (key suffix _v<variant>),
    # else of the problem's profiled variant
    pkey = f"{args.precision}_hlle_{dom}_rotor{n}"
    vkey = f"{pkey}_v{s.variant()['variant']}"
    traffic = profile_traffic(vkey) or profile_traffic(pkey)
    inst_per_cell = profile_value("instructions", vkey) or profile_value("instructions", pkey)

    # --- end to end through the C-ABI with host buffers: every step copies the
    #     state in from pinned host memory, advances one step, copies it out.
    e2e = None
    if not args.no_e2e:
        host_in = [torch.from_numpy(a).pin_memory() for a in st]
        host_out = [torch.empty((n, n), dtype=torch.float64).pin_memory() for _ in range(6)]
        k2 = max(3, min(args.steps, 20))
        s2 = gpu.Solver(cfg)
        for _ in range(2):
            s2.step_host(host_in, out=host_out)
        ext2 = torch.cuda.ExternalStream(s2.stream)
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        barrier(world)
        f0.record(ext2)
        for _ in range(k2):
            s2.step_host(host_in, out=host_out)   # H2D, CFL dt, three stages, D2H (chimera_step_host)
        f1.record(ext2)
        f1.synchronize()
        ms2 = dist_max(f0.elapsed_time(f1), world)
        s2.close()
        e2e = {"value": world * cells * k2 / (ms2 * 1e-3), "unit": "zone-cycles/s",
               "h2d_bytes_per_step": 6 * 8 * cells, "d2h_bytes_per_step": 6 * 8 * cells,
               "steps": k2, "mode": "state copied host->device and back around every RK3 step "
                       "(chimera_step_host: the three stages run as a wavefront over chunks of tile rows "
                       "and each finished chunk goes back while later chunks compute)"}

    kh = adj_leg = None
    if world == 1 and args.kh == "on":
        kh = run_kh(args)
    if world == 1 and args.adjoint == "on":
        adj_leg = run_adjoint_leg(args)
    slab_leg = run_slab_leg(args) if world == 1 and args.slabs > 1 else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = cpu_reference_rate(n, repeats=3, seconds=args.ref_seconds)
        r1 = cpu_reference_rate(n, repeats=3, seconds=args.ref_seconds, omp_mode=1)
        cpu = {"value": r["value"], "unit": "zone-cycles/s", "cores": r["cores"], "kind": "port",
               "cpu_model": r["cpu_model"], "spread": r["spread"], "rates": r["rates"],
               "sample": f"median of {len(r['rates'])} samples of {r['steps_per_sample']} RK3 steps "
                         f"({r['seconds']:.1f} s in all) of the {n}^2 rotor from one warm state on the host "
                         f"cores (FP64 C restatement, OpenMP on every loop)",
               "reference_threading": {
                   "value": r1["value"], "unit": "zone-cycles/s", "spread": r1["spread"], "rates": r1["rates"],
                   "sample": f"median of {len(r1['rates'])} samples of {r1['steps_per_sample']} RK3 steps, "
                             f"OpenMP only on the three loops the reference threads "
                             f"(src/mhd_derivatives.f90:79,105,186)"}}

    if rank == 0:
        line = {
            "metric": "zone-cycles/s", "value": value, "unit": "zone-cycles/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if prec == FP32_BULK else "f64",
            "data": "synthetic (analytic rotor initial state)",
            "config": {"workload": WORKLOAD, "cells": cells, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (3 state sets x 48 MB > 126 MB)",
                       "hbm_fraction": value / world * 48 * esize / (hbm * 1e9),
                       "tile": vinfo,
                       "bytes_per_zone_cycle": 48 * esize},
            "roofline": {"bound": "hbm", "kernel": f"stage kernel ({args.precision}, HLLE, stage {kidx})",
                         "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "peak_kind": peak_kind, "traffic": traffic,
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "avg_launch_ms": avg[dom], "per_kernel_avg_ms": avg,
                         "issue": issue_roofline(inst_per_cell, cells, avg[dom], ck.get("sm_mhz"),
                                                 torch.cuda.get_device_properties(local).multi_processor_count)},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": 3 * args.steps,
            "clocks": ck,
            "forms": ens,
            "kelvin_helmholtz": kh,
            "adjoint": adj_leg,
            "slabs": slab_leg,
        }
        print(json.dumps(line), flush=True)
    s.close()


def run_ensemble(args, world):
    """The batched GRF ensemble (one persistent launch per stage over all
    members of uneven sizes, CUDA-graph replay) in the FP32-bulk form, the
    FP32-arithmetic form on FP64 storage and the plain FP64 form from the same
    seeded states.  The FP64 GPU form reproduces the FP64 oracle bit for bit
    (tests/test_gpu_parity.py, test_gpu_batch.py), so the FP32 forms' L1 errors
    are measured against it on the full ensemble, in all and per member size."""
    import numpy as np
    import torch
    from chimera_b200 import ensemble
    from chimera_b200.config import FP32_BULK, FP32_MIXED, FP64

    from chimera_b200 import problems
    from chimera_b200.shard import shard_members

    steps = args.ens_steps
    graph = 10 if steps % 10 == 0 else 1
    res = {}
    finals = {}
    hbm, _ = peaks()
    rank = int(os.environ.get("RANK", "0"))
    sizes = problems.grf_ensemble_sizes(args.ens_scale)
    all_cells = sum(n * n for n in sizes)
    mine = set(shard_members([n * n for n in sizes], world, rank))   # members are independent: no exchange
    forms = [(n, p) for n, p in (("fp32_batched", FP32_BULK), ("fp32mixed_batched", FP32_MIXED),
                                 ("fp64_batched", FP64))
             if n.split("_")[0] in args.ens_forms.split(",")]
    for name, prec in forms:
        cfgs, states = ensemble.grf_ensemble(args.ens_scale, prec, members=mine)
        cells = all_cells
        s = ensemble.make_batch(cfgs, states)
        s.step(1)
        if args.ens_variant >= 0 and prec == FP32_BULK:
            s.set_variant(args.ens_variant)
        else:
            s.autotune(reps=2)
        # restart from the initial states so both forms take the same steps
        for m, st in enumerate(states):
            s.set_state(st, member=m)
            s.set_time(0.0, 1, member=m)
        s.set_graph_steps(graph)
        ext = torch.cuda.ExternalStream(s.stream)
        s.step(graph)                         # capture the graph (not timed)
        for m, st in enumerate(states):
            s.set_state(st, member=m)
            s.set_time(0.0, 1, member=m)
        s.step(0)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        barrier(world)
        e0.record(ext)
        for _ in range(steps // graph):
            s.step(graph)
        e1.record(ext)
        e1.synchronize()
        ms = dist_max(e0.elapsed_time(e1), world)
        esize = 4 if prec == FP32_BULK else 8
        member_sizes = [c.nx for c in cfgs]
        zcs = cells * steps / (ms * 1e-3)
        res[name] = {"value": zcs, "unit": "zone-cycles/s", "ms": ms, "steps": steps,
                     "members": len(sizes), "members_per_rank_max": len(cfgs), "cells": cells,
                     "tile": s.variant(),
                     "bytes_per_zone_cycle": 48 * esize,
                     "hbm_fraction": zcs / world * 48 * esize / (hbm * 1e9),
                     "scaling": "strong (members sharded across ranks)",
                     "graph_steps": graph}
        finals[name] = [s.get_state(member=m) for m in range(len(cfgs))]
        if prec == FP64 and "fp32_batched" in finals:
            # conditioning of the ensemble: the same FP64 run from the initial states
            # rounded to FP32 (untimed); the FP32 form cannot be closer than this floor
            for m, st in enumerate(states):
                s.set_state([a.astype(np.float32).astype(np.float64) for a in st], member=m)
                s.set_time(0.0, 1, member=m)
            s.step(0)
            for _ in range(steps // graph):
                s.step(graph)
            finals["fp64_ic_rounded"] = [s.get_state(member=m) for m in range(len(cfgs))]
        s.close()
    if "fp32_batched" not in finals or "fp64_batched" not in finals:
        return res

    def l1_vs_fp64(key, size=None):
        num = np.zeros(6)
        den = np.zeros(6)
        for n, a, b in zip(member_sizes, finals[key], finals["fp64_batched"]):
            if size is not None and n != size:
                continue
            for q in range(6):
                num[q] += np.sum(np.abs(a[q] - b[q]))
                den[q] += np.sum(np.abs(b[q]))
        if world > 1:   # diagnostics only
            import torch.distributed as dist
            t = torch.tensor(np.concatenate([num, den]), dtype=torch.float64, device="cuda")
            dist.all_reduce(t)
            num, den = t[:6].cpu().numpy(), t[6:].cpu().numpy()
        return dict(zip(("Mass", "Momx", "Momy", "Energy", "b_x", "b_y"), (num / np.maximum(den, 1e-300)).tolist()))

    res["fp32_l1_vs_fp64"] = l1_vs_fp64("fp32_batched")
    res["fp64_from_fp32_rounded_ic_l1_vs_fp64"] = l1_vs_fp64("fp64_ic_rounded")
    res["fp32_over_fp64"] = res["fp32_batched"]["value"] / res["fp64_batched"]["value"]
    sizes_present = sorted(set(sizes))
    res["l1_vs_fp64_by_member_size"] = {
        key: {str(n): max(l1_vs_fp64(k, n).values()) for n in sizes_present}
        for key, k in (("fp32_bulk", "fp32_batched"), ("fp32_mixed", "fp32mixed_batched"),
                       ("fp64_from_fp32_rounded_ic", "fp64_ic_rounded")) if k in finals}
    if "fp32mixed_batched" in finals:
        res["fp32mixed_l1_vs_fp64"] = l1_vs_fp64("fp32mixed_batched")
        res["fp32mixed_over_fp64"] = res["fp32mixed_batched"]["value"] / res["fp64_batched"]["value"]
    res["workload"] = (f"GRF ensemble, {res['fp32_batched']['members']} members of uneven sizes "
                       f"(128^2/256^2/512^2), periodic, Rusanov + MC + MOOD, {steps} RK3 steps")
    return res


def _timed_run(s, steps, graph):
    """Device time (ms) of `steps` steps on the solver's stream, replayed
    from a graph of `graph` steps (captured by the caller beforehand)."""
    import torch
    ext = torch.cuda.ExternalStream(s.stream)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(ext)
    for _ in range(steps // graph):
        s.step(graph)
    e1.record(ext)
    e1.synchronize()
    return e0.elapsed_time(e1)


def run_kh(args):
    """Kelvin-Helmholtz n^2 on [0,1]x[-1,1] (HLLD + MC + MOOD), the FP32-bulk
    form and the FP32-arithmetic form on FP64 storage against the plain FP64
    form on the same GPU from the same state: zone-cycles/s of each (graph
    replay), L1 error per field and div B."""
    import numpy as np
    from chimera_b200 import gpu, problems
    from chimera_b200.config import FP32_BULK, FP32_MIXED, FP64
    n, steps = args.kh_n, args.kh_steps
    graph = 10 if steps % 10 == 0 else 1
    cfg, st = problems.kelvin_helmholtz(n)
    res, finals = {}, {}
    for name, prec in (("fp32_bulk", FP32_BULK), ("fp32_mixed", FP32_MIXED), ("fp64", FP64)):
        s = gpu.Solver(cfg.replace(precision=prec))
        s.set_state(st)
        if prec == FP64 and args.kh_variant >= 0:
            s.set_variant(args.kh_variant)
        else:
            s.autotune(reps=1)
        s.set_graph_steps(graph)
        s.step(graph)                                   # capture (not timed)
        s.set_state(st)
        s.set_time(0.0, 1)
        s.step(0)
        ms = _timed_run(s, steps, graph)
        d = s.diag()
        finals[name] = s.get_state()
        res[name] = {"value": n * n * steps / (ms * 1e-3), "unit": "zone-cycles/s", "ms": ms,
                     "divb_rel": d["divb_rel"], "tile": s.variant()}
        s.close()
    for key, form in (("fp32_l1_vs_fp64", "fp32_bulk"), ("fp32mixed_l1_vs_fp64", "fp32_mixed")):
        l1 = {}
        for q, f in enumerate(("Mass", "Momx", "Momy", "Energy", "b_x", "b_y")):
            a, b = finals[form][q], finals["fp64"][q]
            l1[f] = float(np.sum(np.abs(a - b)) / np.sum(np.abs(b)))
        res[key] = l1
    res["fp32_over_fp64"] = res["fp32_bulk"]["value"] / res["fp64"]["value"]
    res["fp32mixed_over_fp64"] = res["fp32_mixed"]["value"] / res["fp64"]["value"]
    res["workload"] = (f"Kelvin-Helmholtz {n}^2 on [0,1]x[-1,1], periodic, HLLD + MC + MOOD, gamma 1.4, "
                       f"{steps} RK3 steps from the same state")
    return res


def run_slab_leg(args):
    """The FP64 Kelvin-Helmholtz grid (HLLD + MC + MOOD) as ``args.slabs``
    y-slabs on one GPU -- separate handles on one stream, 7 ghost rows moved
    by device copies and the dt minimum taken every step (chimera_b200.slab)
    -- against the undivided grid stepped eagerly from the same state: device
    time per step of each, the overhead of the decomposition (redundant ghost
    rows, pack / unpack, the dt hand-off, smaller launches) and whether the
    results are bitwise equal."""
    import numpy as np
    import torch
    from chimera_b200 import gpu, problems
    from chimera_b200.slab import LocalTransport, SlabSolver, gather_interior, slab_step
    n, k, steps = args.kh_n, args.slabs, 50
    cfg, st = problems.kelvin_helmholtz(n)
    whole = gpu.Solver(cfg)
    whole.set_state(st)
    whole.step(3)                                         # warm-up (not timed)
    whole.set_state(st)
    whole.set_time(0.0, 1)
    whole.step(0)
    ms_whole = _timed_run(whole, steps, 1)
    ref = whole.get_state()
    whole.close()
    stream = torch.cuda.Stream()
    slabs = [SlabSolver(cfg, r, k, stream=stream) for r in range(k)]
    for sl in slabs:
        sl.set_global_state(st)
    slab_step(slabs, LocalTransport(), 3)                  # warm-up (not timed)
    for sl in slabs:
        sl.set_global_state(st)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    slab_step(slabs, LocalTransport(), steps)
    e1.record(stream)
    e1.synchronize()
    ms_slabs = e0.elapsed_time(e1)
    got = gather_interior(slabs)
    for sl in slabs:
        sl.close()
    return {"workload": f"Kelvin-Helmholtz {n}^2 FP64, HLLD + MC + MOOD, {steps} RK3 steps, "
                        f"{k} y-slabs of about {n // k} rows + 7 ghost rows per neighbour, on one GPU",
            "slabs": k, "ms_per_step_slabs": ms_slabs / steps, "ms_per_step_whole": ms_whole / steps,
            "overhead": ms_slabs / ms_whole - 1.0,
            "bitwise_equal": all(bool(np.array_equal(got[q], ref[q])) for q in range(6))}


def run_adjoint_leg(args):
    """The field-loop adjoint (512^2 on [0,2]x[0,1], v = (2, 1), HLLE + Van
    Leer, 400 RK3 steps, checkpoints every 20, loss = final magnetic energy,
    gradient w.r.t. the initial rho, vx, vy): forward and forward + backward
    times, and central differences on two smooth random directions."""
    import time
    import numpy as np
    import torch
    from chimera_b200 import adjoint, problems
    from chimera_b200.config import FP32_BULK, FP32_MIXED, FP64, HLLE, VAN_LEER
    n, steps, K = 512, args.adj_steps, args.adj_k
    cfg, st = problems.field_loop(n, n, 2.0, 1.0, v=(2.0, 1.0), riemann=HLLE, limiter=VAN_LEER)
    vol = cfg.dx * cfg.dy
    M, Mx, My, E, bx, by = st
    Bx, By = problems.face_to_cell(bx, by)
    rho, vx, vy = M / vol, Mx / M, My / M
    p = (E / vol - 0.5 * rho * (vx * vx + vy * vy) - 0.5 * (Bx * Bx + By * By)) * (cfg.gamma - 1.0)
    prims = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (rho, vx, vy, p, bx, by)]
    U0 = [u.contiguous() for u in adjoint.conserved_from_primitive(cfg, *prims)]
    dts = adjoint.cfl_dts(cfg, U0, steps)
    adj = adjoint.Adjoint(cfg)

    def loss_of(pr, grad, precision=FP64):
        U = [u.contiguous() for u in adjoint.conserved_from_primitive(cfg, *pr)]
        if not grad:
            for dt in dts:
                U = adj.forward_step(U, dt)
            return adjoint.magnetic_energy(cfg, U)
        return adjoint.magnetic_energy(cfg, adjoint.run(adj, U, dts, K=K, precision=precision))

    with torch.no_grad():
        loss_of(prims, False)                           # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    with torch.no_grad():
        base = float(loss_of(prims, False))
    torch.cuda.synchronize()
    t_fwd = time.perf_counter() - t0
    g_in = [x.clone().requires_grad_(k < 3) for k, x in enumerate(prims)]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    loss = loss_of(g_in, True)
    loss.backward()
    torch.cuda.synchronize()
    t_fb = time.perf_counter() - t0
    gen = torch.Generator(device="cuda").manual_seed(7)
    kx = 2 * np.pi * torch.fft.fftfreq(n, d=cfg.dx, device="cuda", dtype=torch.float64)
    ky = 2 * np.pi * torch.fft.fftfreq(n, d=cfg.dy, device="cuda", dtype=torch.float64)
    filt = torch.exp(-0.5 * 0.25 ** 2 * (ky[:, None] ** 2 + kx[None, :] ** 2))
    worst = 0.0
    for _ in range(2):
        dirs = []
        for k in range(3):
            w = torch.fft.ifft2(torch.fft.fft2(torch.randn((n, n), generator=gen, device="cuda",
                                                           dtype=torch.float64)) * filt).real
            dirs.append(w / torch.max(torch.abs(w)) * (float(torch.max(torch.abs(prims[k]))) or 1.0))
        eps = 1e-6
        with torch.no_grad():
            lp = float(loss_of([prims[k] + eps * dirs[k] if k < 3 else prims[k] for k in range(6)], False))
            lm = float(loss_of([prims[k] - eps * dirs[k] if k < 3 else prims[k] for k in range(6)], False))
        fd = (lp - lm) / (2 * eps)
        an = sum(float(torch.sum(g_in[k].grad * dirs[k])) for k in range(3))
        worst = max(worst, abs(fd - an) / abs(an))
    # the forward in the reduced-precision forms (fused FP32 solver, same frozen dts),
    # the adjoint in FP64 from their checkpoints
    forms = {}
    g64 = [g_in[k].grad for k in range(3)]
    for name, prec in (("fp32_bulk", FP32_BULK), ("fp32_mixed", FP32_MIXED)):
        warm = [x.clone().requires_grad_(k < 3) for k, x in enumerate(prims)]
        loss_of(warm, True, prec).backward()            # untimed: first use of the form in the process
        gp = [x.clone().requires_grad_(k < 3) for k, x in enumerate(prims)]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        lossp = loss_of(gp, True, prec)
        torch.cuda.synchronize()
        t_f = time.perf_counter() - t0
        lossp.backward()
        torch.cuda.synchronize()
        t_all = time.perf_counter() - t0
        rel = max(float(torch.max(torch.abs(gp[k].grad - g64[k])) / torch.max(torch.abs(g64[k]))) for k in range(3))
        forms[name] = {"forward_s": t_f, "forward_backward_s": t_all, "loss": float(lossp),
                       "loss_rel_vs_fp64": abs(float(lossp) - base) / abs(base),
                       "gradient_max_rel_vs_fp64_forward": rel}
    return {"workload": f"field-loop adjoint 512^2 on [0,2]x[0,1], v = (2, 1), HLLE + Van Leer, {steps} RK3 steps, "
                        f"K = {K}, loss = final magnetic energy, gradient w.r.t. initial rho, vx, vy",
            "forward_s": t_fwd, "forward_backward_s": t_fb, "loss": base,
            "gradient_zone_cycles_per_s": n * n * steps / t_fb,
            "central_difference_rel_err_2_dirs": worst,
            "reduced_precision_forward": forms,
            "note": "rho and v start exactly uniform, so every rho / v limiter starts at its kink: central "
                    "differences agree with the stated one-sided convention to about 3e-3 here, and to 1e-6 "
                    "on a generic state (tests/test_gpu_adjoint.py)"}


def main():
    args = parse()
    if args.impl == "reference":
        # the CPU reference arm: rank 0 alone times it, the other ranks exit at
        # once; no rank takes a collective step, so no process group is made
        run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")))
        return
    world, rank, local = dist_setup(args)
    try:
        run_chimera(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
