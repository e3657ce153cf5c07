"""Shot-parallel gradient reduction (efwi.dist) with world_size 2 over gloo
on the CPU: the shards cover the shot list once, in order, by the
reference's linspace rule (Torch_Fwi.cpp:53-54), and after the all-reduce
every rank holds the sum over all shots."""
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import FWI_ops_3d as F
from efwi import dist as edist


def test_shards_cover_in_order_and_match_dropin_rule():
    for n in (1, 2, 5, 7, 16, 33):
        for world in range(1, min(n, 6) + 1):
            parts = [edist.shard(list(range(n)), r, world) for r in range(world)]
            assert sum(parts, []) == list(range(n))
            assert parts == F._shards(list(range(n)), world)


class FakeProp:
    """Per-shot images that depend on the shot id only."""

    shape = (3, 4, 5)

    def gradient(self, ids, obs, mode="reference"):
        gl = torch.zeros(self.shape)
        gm = torch.zeros(self.shape)
        gr = torch.zeros(self.shape)
        J = 0.0
        for i in ids:
            gl += i + 1.0
            gm += torch.arange(60, dtype=torch.float32).reshape(self.shape) * i
            gr -= 0.5 * i
            J += float(i * i)
        return J, gl, gm, gr


def _worker(rank, world, store_path, ids, q):
    from datetime import timedelta
    # file rendezvous: no TCP port to collide with other processes
    dist.init_process_group("gloo", init_method=f"file://{store_path}", rank=rank,
                            world_size=world, timeout=timedelta(seconds=60))
    try:
        sp = edist.ShotParallel(FakeProp())
        mine = sp.local_ids(ids)
        J, gl, gm, gr = sp.gradient(mine, None)
        q.put((rank, mine, J, gl, gm, gr))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("ids", [list(range(5)), [7, 3, 9, 1]])
def test_allreduce_sums_every_shot_once(ids, tmp_path):
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    store = str(tmp_path / "rendezvous")
    procs = [ctx.Process(target=_worker, args=(r, world, store, ids, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    J0, gl0, gm0, gr0 = FakeProp().gradient(ids, None)
    seen = []
    for rank, mine, J, gl, gm, gr in sorted(out, key=lambda r: r[0]):
        seen += mine
        assert J == J0
        assert torch.equal(gl, gl0) and torch.equal(gm, gm0) and torch.equal(gr, gr0)
    assert seen == ids
