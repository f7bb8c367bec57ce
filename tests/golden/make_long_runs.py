"""Generate tests/golden/long_runs.json: the FP64 oracle run to the stated end
of each benchmark workload, recorded as SHA-256 digests of the final state.

The GPU parity tests of tests/test_gpu_long_runs.py advance the same initial
states on the device and compare digests, so a single flipped bit anywhere in
the final state -- a MOOD, floor or HLLD-guard branch taken differently in
any of the ~1,300 steps of a run -- fails the comparison.  The oracle
(oracle/chimera_oracle.c) is the checker; it runs here with OpenMP on every
loop, which changes no result (each loop iteration writes its own cells and the
reductions are exact maxima or are left to the final min over the dt array).

Workloads (each the configuration named in the benchmark specification):

* ``ot256_t05``       Orszag-Tang 256^2 periodic, Rusanov + MC + MOOD, to t = 0.5
* ``rotor1024_t015``  rotor 1024^2 outflow, HLLE + MC + MOOD, to t = 0.15
* ``kh4096_20``       Kelvin-Helmholtz 4096^2 periodic, HLLD + MC + MOOD, 20 steps
* ``grf128_200`` / ``grf256_200`` / ``grf512_200``  the first 128^2, 256^2
  and 512^2 members of the GRF ensemble (seeds 1000, 1256, 1448), Rusanov +
  MC + MOOD, 200 steps

Each record holds the digest of the initial state (so a host whose set-up
arithmetic differs is told apart from a kernel that differs), the digests of
the six final fields, t and dt as exact hex floats, the step and output counts,
and per-field sums and maxima of |value| (to locate a difference).

    python tests/golden/make_long_runs.py [case ...]

takes about 15 minutes on 8 cores (the rotor is most of it).
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from chimera_b200 import problems as P  # noqa: E402
from chimera_b200.config import HLLD, HLLE, MC, RUSANOV  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "long_runs.json")
FIELDS = ("Mass", "Momx", "Momy", "Energy", "b_x", "b_y")


def cases():
    """name -> (set-up callable, max steps).  A run stops at t_end or after
    max steps, whichever comes first (src/main.f90:65)."""
    return {
        "ot256_t05": (lambda: P.orszag_tang(256, riemann=RUSANOV, limiter=MC, mood=True, t_end=0.5), 10 ** 6),
        "rotor1024_t015": (lambda: P.rotor(1024, riemann=HLLE, limiter=MC, mood=True, t_end=0.15), 10 ** 6),
        "kh4096_20": (lambda: P.kelvin_helmholtz(4096, riemann=HLLD, limiter=MC, mood=True, seed=0), 20),
        "grf128_200": (lambda: P.grf_member(128, 1000), 200),
        "grf256_200": (lambda: P.grf_member(256, 1256), 200),
        "grf512_200": (lambda: P.grf_member(512, 1448), 200),
    }


def state_digest(arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    return h.hexdigest()


def field_digests(arrays) -> dict:
    return {f: hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()
            for f, a in zip(FIELDS, arrays)}


def field_stats(arrays) -> dict:
    return {f: {"sum": float(np.sum(a)), "max_abs": float(np.max(np.abs(a)))} for f, a in zip(FIELDS, arrays)}


def record(cfg, ic, final, t, output_count, steps, last_dt) -> dict:
    return {
        "config": {"nx": cfg.nx, "ny": cfg.ny, "dx": cfg.dx.hex(), "dy": cfg.dy.hex(),
                   "gamma": float(cfg.gamma).hex(), "riemann": cfg.riemann, "limiter": cfg.limiter,
                   "mood": bool(cfg.mood), "bc": list(cfg.bc), "t_out": cfg.t_out, "t_end": cfg.t_end},
        "initial_sha256": state_digest(ic),
        "final_sha256": field_digests(final),
        "t": float(t).hex(),
        "last_dt": float(last_dt).hex(),
        "steps": int(steps),
        "output_count": int(output_count),
        "stats": field_stats(final),
    }


def main(names):
    from oracle import oracle
    oracle.set_omp_mode(2)
    oracle.set_threads(os.cpu_count() or 1)
    data = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            data = json.load(f)
    table = cases()
    for name in names or list(table):
        make, max_steps = table[name]
        cfg, ic = make()
        st = oracle.State(ic)
        t0 = time.time()
        dts = oracle.run(cfg, st, max_steps)
        el = time.time() - t0
        data[name] = record(cfg, ic, st.a, st.t, st.output_count, len(dts), dts[-1])
        print(f"{name}: {len(dts)} steps to t={st.t:.6f} in {el:.1f} s", flush=True)
        with open(OUT, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
    oracle.set_omp_mode(0)


if __name__ == "__main__":
    main(sys.argv[1:])
