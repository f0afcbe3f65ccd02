"""Two-rank runs of the replica path on CPU (gloo): bench.py's per-rank streams
and max-over-ranks timing, and its reference arm launched like the multi-GPU
bench (rank 0 reports, the other ranks exit without work)."""
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


def _torchrun(args, timeout):
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port())] + args
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", OMP_NUM_THREADS="1")
    return subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=timeout)


def test_replicas_max_over_ranks_and_own_streams(tmp_path):
    p = _torchrun([os.path.join(ROOT, "tests", "_multirank_worker.py"), str(tmp_path)], timeout=300)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in (0, 1)]
    assert sorted(d["rank"] for d in lines) == [0, 1]
    for d in lines:
        assert d["world"] == 2
        assert d["max_ms"] == 20.0          # the slower rank sets the time
        assert d["streams"][0] != d["streams"][1]   # each replica serves its own requests


def test_reference_arm_two_ranks_reports_once():
    p = _torchrun(["bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0",
                   "--nreq", "24", "--cpu-sample", "3", "--cpu-reps", "1"], timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [json.loads(ln) for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
