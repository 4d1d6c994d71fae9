"""bench.py's multi-rank path on the CPU: two gloo ranks (world size 2).

Rank 0 writes the deck while the other waits at the barrier; the step time is
the maximum over ranks; the whole-job rate counts every rank's elements; the
reference arm runs on rank 0 only and the other rank exits 0 silently."""
import json
import socket
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_bench_two_gloo_ranks(built, tmp_path):
    port = free_port()
    worker = ROOT / "tests" / "bench_ranks_worker.py"
    procs = [subprocess.Popen([sys.executable, str(worker), str(r), "2", str(port), str(tmp_path / "decks"),
                               str(tmp_path / f"rank{r}.json")]) for r in range(2)]
    for p in procs:
        assert p.wait(timeout=300) == 0
    res = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(2)]
    assert res[0]["deck"] == res[1]["deck"] and res[0]["complete"] and res[1]["complete"]
    assert res[0]["slowest"] == res[1]["slowest"] == 20.0
    assert res[0]["rc"] == res[1]["rc"] == 0
    assert res[1]["stdout"] == ""
    line = json.loads(res[0]["stdout"].strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0
    # the config-3 and ensemble decks: written once by rank 0, read by both
    assert res[0]["config3_ne"] == res[1]["config3_ne"] == 2 * 4 * 8
    assert res[0]["ensemble_ne"] == res[1]["ensemble_ne"] and len(res[0]["ensemble_ne"]) == 3


def test_whole_job_rate_counts_every_rank():
    import bench
    one = bench.whole_job_rate(1, 1000, 2, 10, 5.0)
    assert bench.whole_job_rate(2, 1000, 2, 10, 5.0) == 2 * one
    assert one == bench.DOFS_PER_ELEMENT * 1000 * 2 * 10 / 5e-3
    assert bench.max_over_ranks(3.5, 1) == 3.5
