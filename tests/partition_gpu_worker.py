"""One rank of the world-size-2 partitioned run on one GPU (launched by
test_partition_ranks_gpu.py): the rank steps its partition with
DistributedPartition, halos staged through pinned host buffers and moved
over gloo (the next stage's ghost-free tiles launched while the host moves
them, unless overlap is 0), and saves its owned rows."""
import os
import sys
from datetime import timedelta
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def main(rank: int, world: int, port: int, deck_dir: str, nsteps: int, strict: int, out: str,
         overlap: int = 1) -> int:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    torch.cuda.set_device(0)
    from dgswem_b200 import Deck, DistributedPartition
    deck = Deck(deck_dir)
    with DistributedPartition(deck, strict=bool(strict), transport="host", overlap=bool(overlap)) as dp:
        info = dp.hs.part_info()
        dp.run(1, nsteps)
        dp.hs.synchronize()
        ze, qx, qy, wd = dp.owned_state()
    dist.barrier()
    dist.destroy_process_group()
    np.savez(out, ze=ze, qx=qx, qy=qy, wd=wd, owned=info["owned"], local=info["local"])
    return 0


if __name__ == "__main__":
    sys.exit(main(int(sys.argv[1]), int(sys.argv[2]), int(sys.argv[3]), sys.argv[4], int(sys.argv[5]),
                  int(sys.argv[6]), sys.argv[7], int(sys.argv[8]) if len(sys.argv) > 8 else 1))
