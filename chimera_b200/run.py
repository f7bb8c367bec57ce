"""Whole runs the way the reference program makes them, on the GPU.

``run_sim(problem_type, N, seed, out_dir, name)`` mirrors the reference's
command line (``./chimera <problem_type> <N> <seed> [output_path]
[h5_filename]``, src/mhd_init.f90:167-256): it sets up the problem, advances it
with the fused stage kernels to tEnd, collects the snapshot the reference
writes after every step that reaches the next output time (primitives with the
THERMAL pressure, src/main.f90:279-292) and writes them with the layout of
``write_prims_to_hdf5`` (src/mhd_write_h5.f90:13-194): groups ``rho``, ``P``,
``Bx``, ``By``, ``Vx``, ``Vy`` holding ``SNAPSHOT1``, ``SNAPSHOT2``, ... as
(ny, nx) arrays, ``time/sim_time`` and ``parameters/{gamma, M_s, beta}``.  No
HDF5 library exists in this environment, so the file is a NumPy ``.npz``
archive whose keys are those HDF5 paths (``"rho/SNAPSHOT1"``);
``read_snapshots`` returns a mapping with the same paths and ``to_hdf5``
converts when h5py is available.

Snapshot primitives are computed on the device with the per-routine kernels
(``average_face_to_cell_B``, ``get_primitive``), bit for bit as the reference
routines compute them.
"""
from __future__ import annotations

import os

import numpy as np

from . import problems as P
from .config import FP64, MC, RUSANOV

FIELDS = ("rho", "P", "Bx", "By", "Vx", "Vy")
PROBLEMS = {1: "Orszag-Tang", 2: "Kelvin-Helmholtz", 3: "Field loop", 4: "Rotor", 5: "GRF"}


def reference_problem(problem_type: int, n: int, seed: int = 0, t_end: float = 1.0):
    """(cfg, conserved state, parameters) of the reference's problem numbering
    (src/mhd_init.f90:172-174): 1 Orszag-Tang, 2 Kelvin-Helmholtz, 3 field loop,
    4 rotor, 5 Monte-Carlo GRF member.  tEnd defaults to the reference's
    compile-time 1.0 (src/mhd_config.f90:16).  Problem 2 is the
    Kelvin-Helmholtz set-up of this project's workload (periodic, [0,1]x[-1,1],
    Bx = 0.1), problem 5 the GRF member of the ensemble workload; the others
    are the reference's set-ups."""
    if problem_type == 1:
        cfg, st = P.orszag_tang(n, t_end=t_end)
    elif problem_type == 2:
        cfg, st = P.kelvin_helmholtz(n, seed=seed, t_end=t_end)
    elif problem_type == 3:   # the reference's field loop: unit square, v = (-2, -1) (src/mhd_init.f90:360-391)
        cfg, st = P.field_loop(n, n, 1.0, 1.0, v=(-2.0, -1.0), riemann=RUSANOV, limiter=MC, t_end=t_end)
    elif problem_type == 4:
        cfg, st = P.rotor(n, t_end=t_end)
    elif problem_type == 5:
        cfg, st = P.grf_member(n, seed)
        cfg = cfg.replace(t_end=t_end)
    else:
        raise ValueError(f"problem_type must be 1-5, got {problem_type}")
    return cfg, st, initial_parameters(cfg, st, problem_type)


def initial_parameters(cfg, st, problem_type: int) -> dict:
    """gamma, and for the GRF problem the sonic Mach number v_rms / <c_s> and
    the plasma beta 2 <p> / B_rms^2 of the initial state (the definitions of
    src/mhd_init.f90:839-841); 0 for the other problems, whose set-up does not
    compute them."""
    M_s = beta = 0.0
    if problem_type == 5:
        Bx, By = P.face_to_cell(st[4], st[5], cfg.bc[0] == 1, cfg.bc[2] == 1)
        vol = cfg.dx * cfg.dy
        rho = st[0] / vol
        vx, vy = st[1] / st[0], st[2] / st[0]
        p = (st[3] / vol - 0.5 * rho * (vx * vx + vy * vy) - 0.5 * (Bx * Bx + By * By)) * (cfg.gamma - 1.0)
        v_rms = np.sqrt(np.mean(vx * vx + vy * vy))
        c_s = np.mean(np.sqrt(cfg.gamma * p / rho))
        B_rms = np.sqrt(np.mean(Bx * Bx + By * By))
        M_s = float(v_rms / (c_s + 1e-16))
        beta = float(2.0 * np.mean(p) / (B_rms ** 2 + 1e-16))
    return {"gamma": float(cfg.gamma), "M_s": M_s, "beta": beta}


def run(cfg, state, precision: int = FP64, max_steps: int = 10 ** 7):
    """Advance ``state`` from t = 0 to cfg.t_end on the GPU and return the
    reference's snapshots: a list of dicts with t, rho, Vx, Vy, P (thermal),
    Bx, By (float64 numpy arrays, (ny, nx))."""
    import torch

    from . import gpu, ops

    c = cfg.replace(precision=precision)
    c64 = cfg.replace(precision=FP64)
    s = gpu.Solver(c)
    snaps = []
    try:
        s.set_state(state)
        dev = [torch.empty((cfg.ny, cfg.nx), dtype=torch.float64, device="cuda") for _ in range(6)]
        d = s.diag()
        oc, taken = d["output_count"], 0
        while d["active"] and taken < max_steps:
            # the time loop runs on the device up to the step that reaches the next
            # output time (src/main.f90:279), where the reference writes a snapshot
            taken += s.advance_output(max_steps - taken)
            d = s.diag()
            if d["output_count"] != oc:
                oc = d["output_count"]
                s.get_state(out=dev)
                Bx, By = ops.average_face_to_cell_B(c64, dev[4], dev[5])
                rho, vx, vy, Ptot = ops.get_primitive(c64, dev[0], dev[1], dev[2], dev[3], Bx, By)
                p_th = Ptot - 0.5 * (Bx * Bx + By * By)
                snaps.append(dict(t=d["t"], rho=rho.cpu().numpy(), Vx=vx.cpu().numpy(), Vy=vy.cpu().numpy(),
                                  P=p_th.cpu().numpy(), Bx=Bx.cpu().numpy(), By=By.cpu().numpy()))
    finally:
        s.close()
    return snaps


def write_snapshots(path: str, snaps, parameters: dict) -> str:
    """Write snapshots with the HDF5 paths of src/mhd_write_h5.f90 as keys of
    an .npz archive; returns the path written."""
    arrays = {}
    for k, snap in enumerate(snaps, start=1):
        for f in FIELDS:
            arrays[f"{f}/SNAPSHOT{k}"] = np.ascontiguousarray(snap[f])
    arrays["time/sim_time"] = np.array([snap["t"] for snap in snaps], dtype=np.float64)
    for name in ("gamma", "M_s", "beta"):
        arrays[f"parameters/{name}"] = np.array([parameters[name]], dtype=np.float64)
    if not path.endswith(".npz"):
        path = path + ".npz"
    np.savez(path, **arrays)
    return path


def read_snapshots(path: str) -> dict:
    """The archive as a dict of HDF5-style paths -> arrays."""
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


def snapshot_keys(data: dict, field: str = "rho"):
    """SNAPSHOT names of one group in output order (as the reference's tests
    sort them: tests/physics/test_rk3.py:47)."""
    keys = [k.split("/", 1)[1] for k in data if k.startswith(field + "/")]
    return sorted(keys, key=lambda k: int(k.replace("SNAPSHOT", "")))


def to_hdf5(npz_path: str, h5_path: str) -> None:
    """Convert an archive to the reference's HDF5 file (needs h5py)."""
    import h5py   # not installed in this environment

    data = read_snapshots(npz_path)
    with h5py.File(h5_path, "w") as f:
        for key, arr in data.items():
            f.create_dataset(key, data=arr)


def run_sim(problem_type: int, N: int, seed: int = 0, out_dir: str = ".", h5_name: str | None = None,
            t_end: float = 1.0, precision: int = FP64) -> str:
    """The reference program's run (set-up, time loop, snapshot file) on the
    GPU; returns the path of the snapshot archive."""
    cfg, st, params = reference_problem(problem_type, N, seed, t_end)
    snaps = run(cfg, st, precision)
    name = h5_name or f"test_p{problem_type}_N{N}_s{seed}.h5"
    stem = name[:-3] if name.endswith(".h5") else name
    return write_snapshots(os.path.join(out_dir, stem + ".npz"), snaps, params)


__all__ = ["reference_problem", "initial_parameters", "run", "write_snapshots", "read_snapshots",
           "snapshot_keys", "to_hdf5", "run_sim", "FIELDS", "PROBLEMS"]
