"""bench.py's reference arm on the CPU: `--impl reference` times the CPU
restatement of the reference solver and prints one JSON line with the
contract's keys; launched by torchrun with two ranks (gloo here), rank 0 alone
runs and prints, the other rank exits 0 without work."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _json_lines(text):
    return [json.loads(l) for l in text.splitlines() if l.startswith("{")]


def test_reference_arm_under_two_ranks():
    env = dict(os.environ, OMP_NUM_THREADS=os.environ.get("OMP_NUM_THREADS", "8"))
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           "bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3"]
    out = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = _json_lines(out.stdout)
    assert len(lines) == 1, out.stdout[-2000:]
    d = lines[0]
    assert d["impl"] == "reference" and d["metric"] == "DOF-stage updates/s" and d["unit"] == "DOF-stage/s"
    assert d["value"] > 0 and d["higher_is_better"] is True and d["n_gpus"] == 2
    # the requested steps were timed (after the requested untimed ones) and their time is reported
    assert d["steps"] == 1 and d["warmup"] == 3 and d["ms_per_step"] > 0
    assert "1 LSERK4 steps" in d["cpu_baseline"]["sample"]
    # the same workload as the GPU arm: the full 192,000-tet model, not a smaller sample
    assert d["config"]["workload"] == "twolayer_anelastic_npml_192k_tets_N4_lserk4" and d["config"]["tets"] == 192000
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and "192000 tets" in cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
