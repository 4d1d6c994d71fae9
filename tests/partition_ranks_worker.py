"""One rank of the world-size-2 gloo check of the partition halo lists
(launched by test_partition_plan.py; CPU only)."""
import json
import os
import sys
from datetime import timedelta
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))


def main(rank: int, world: int, port: int, deck_dir: str, out: str) -> int:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    from dgswem_b200 import Deck
    from test_partition_plan import halo_ids
    deck = Deck(deck_dir)
    peer = 1 - rank
    mine = {k: [a.tolist() for a in halo_ids(deck, rank, world, peer, k)] for k in (0, 1)}
    got = [None] * world
    dist.all_gather_object(got, mine)
    theirs = got[peer]
    agree = all(mine[k][0] == theirs[k][1] and mine[k][1] == theirs[k][0] for k in (0, 1))
    dist.barrier()
    dist.destroy_process_group()
    Path(out).write_text(json.dumps({"rank": rank, "agree": agree, "nsend": len(mine[1][0])}))
    return 0


if __name__ == "__main__":
    sys.exit(main(int(sys.argv[1]), int(sys.argv[2]), int(sys.argv[3]), sys.argv[4], sys.argv[5]))
