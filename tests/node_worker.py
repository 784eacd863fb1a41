"""One node of a partitioned oracle run, exchanging its halo with the other
ranks through closures_b200.exchange_distributed over gloo.  Launched by
tests/test_partition.py as one process per node (RANK, WORLD_SIZE,
MASTER_ADDR, MASTER_PORT in the environment):

    python node_worker.py <deck> <steps> <out.npz>

Writes the node's final moments and alpha (all cells, ghosts included)."""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "closures-2d_b200"))
sys.path.insert(0, os.path.join(REPO, "oracle"))

import numpy as np  # noqa: E402
import torch  # noqa: E402
import torch.distributed as dist  # noqa: E402

import closures_b200 as cb  # noqa: E402
import pyoracle  # noqa: E402


def main():
    deck, steps, out = sys.argv[1], int(sys.argv[2]), sys.argv[3]
    rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
    dist.init_process_group("gloo", rank=rank, world_size=world)
    g = pyoracle.GridSolver(deck, node=rank, num_nodes=world)
    info = g.node_info()
    periodic = int(cb.deck_value(deck, "INIT_COND")) == 2
    plan = cb.HaloPlan(rank, info["nodes_x"], info["nodes_y"], periodic)
    counts = g.halo_counts()
    recv = [torch.zeros(c, dtype=torch.float64) for c in counts]
    for _ in range(steps):
        g.save_old()
        for _stage in (1, 2):
            send = [torch.from_numpy(g.halo_pack(k)) for k in cb.SIDES]
            cb.exchange_distributed(plan, send, recv)
            for k in cb.SIDES:
                if plan.peer[k] is not None:
                    g.halo_unpack(k, recv[k].numpy())
            g.stage_exchanged(g.max_dt)
        g.average()
    m, a = g.state()
    np.savez(out, moments=m, alpha=a)
    dist.barrier()
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
