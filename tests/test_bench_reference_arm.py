"""bench.py --impl reference (the CPU restatement of the reference timed on the
host cores) needs no GPU: its JSON line has the keys the measurement contract
names, and under torchrun rank 0 alone prints it while the other ranks exit 0
-- with every host core in use, although torchrun sets OMP_NUM_THREADS=1."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ARGS = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1", "--ref-seconds", "0.5"]


def _lines(out):
    return [json.loads(x) for x in out.splitlines() if x.startswith("{")]


def _check(line, n_gpus):
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["n_gpus"] == n_gpus
    assert line["metric"] == "zone-cycles/s" and line["value"] > 0 and line["higher_is_better"] is True
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["kind"] == "port" and cb["sample"]
    assert cb["cores"] == len(os.sched_getaffinity(0))
    assert len(cb["rates"]) >= 3 and cb["spread"] >= 0 and cb["cpu_model"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_single_process():
    r = subprocess.run([sys.executable, *ARGS], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _lines(r.stdout)
    assert len(lines) == 1
    _check(lines[0], 1)


def test_reference_arm_under_torchrun_prints_once():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), *ARGS, "--gpus", "2"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _lines(r.stdout)
    assert len(lines) == 1
    _check(lines[0], 2)
