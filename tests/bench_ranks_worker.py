"""One rank of the world-size-2 gloo check of bench.py's multi-rank logic
(launched by test_bench_ranks.py; CPU only)."""
import contextlib
import io
import json
import os
import sys
from datetime import timedelta
from pathlib import Path
from types import SimpleNamespace

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def main(rank: int, world: int, port: int, workdir: str, out: str) -> int:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench
    path = bench.ensure_deck(Path(workdir), 6, 3, rank, world, dist)
    slowest = bench.max_over_ranks(10.0 * (rank + 1), world, dist, "cpu")
    # decks of the config-3 and ensemble arms: rank 0 writes, the others open
    from dgswem_b200 import Deck, decks
    from dgswem_b200.ensemble import make_members
    c3 = bench.rank0_first(rank, world, dist, lambda: bench.config3_deck(workdir, 4, 8))
    d3 = Deck(c3)
    c3_ne = d3.s.ne
    d3.close()
    specs = decks.ensemble_specs(3, seed=4, ne_min=100, ne_max=300)
    ens, _ = bench.rank0_first(rank, world, dist, lambda: make_members(Path(workdir) / "ens", specs, nsteps=2))
    ens_ne = [d.s.ne for d in ens]
    args = SimpleNamespace(workdir=workdir, nx=6, ny=3, steps=2, warmup=1, ref_max_steps=2, gpus=world)
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        rc = bench.run_reference(args)
    dist.barrier()
    dist.destroy_process_group()
    Path(out).write_text(json.dumps({"rank": rank, "deck": str(path), "complete": (path / ".complete").exists(),
                                     "slowest": slowest, "rc": rc, "stdout": buf.getvalue(),
                                     "config3_ne": c3_ne, "ensemble_ne": ens_ne}))
    return 0


if __name__ == "__main__":
    sys.exit(main(int(sys.argv[1]), int(sys.argv[2]), int(sys.argv[3]), sys.argv[4], sys.argv[5]))
