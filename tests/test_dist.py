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


class FakeGridProp(FakeProp):
    """FakeProp with the engine's `out=` interface: images written into one
    stacked caller buffer."""

    class grid:
        ncell = 60

    device = torch.device("cpu")

    def gradient(self, ids, obs, mode="reference", out=None):
        J, gl, gm, gr = super().gradient(ids, obs, mode)
        if out is None:
            return J, gl, gm, gr
        n = self.grid.ncell
        views = [out[k * n:(k + 1) * n].view(self.shape) for k in range(3)]
        for v, t in zip(views, (gl, gm, gr)):
            v.copy_(t)
        return (J, *views)


def _worker(rank, world, store_path, ids, q, prop_cls="FakeProp"):
    from datetime import timedelta
    # file rendezvous: no TCP port to collide with other processes
    dist.init_process_group("gloo", init_method=f"file://{store_path}", rank=rank,
                            world_size=world, timeout=timedelta(seconds=60))
    try:
        sp = edist.ShotParallel(globals()[prop_cls]())
        mine = sp.local_ids(ids)
        J, gl, gm, gr = sp.gradient(mine, None)
        q.put((rank, mine, J, gl, gm, gr))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("prop_cls", ["FakeProp", "FakeGridProp"])
@pytest.mark.parametrize("ids", [list(range(5)), [7, 3, 9, 1]])
def test_allreduce_sums_every_shot_once(ids, prop_cls, tmp_path):
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    store = str(tmp_path / "rendezvous")
    procs = [ctx.Process(target=_worker, args=(r, world, store, ids, q, prop_cls))
             for r in range(world)]
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


def test_allreduce_matches_dropin_shard_sum(tmp_path):
    """The ranks' one stacked all-reduce gives the drop-in's own sum of the
    same per-shard results (FWI_ops_3d._shards, FWI_ops_3d._reduce_shards),
    images to float32 rounding and the misfit to float32 precision."""
    ids = [4, 0, 11, 6, 2, 9, 13]
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    store = str(tmp_path / "rendezvous")
    procs = [ctx.Process(target=_worker, args=(r, world, store, ids, q, "FakeGridProp"))
             for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    shards = F._shards(ids, world)
    results = [FakeProp().gradient(s, None) for s in shards]
    J0, gl0, gm0, gr0 = F._reduce_shards(results, torch.device("cpu"))
    for rank, mine, J, gl, gm, gr in out:
        assert mine == shards[rank]
        assert abs(J - J0) <= 1e-6 * abs(J0)
        for a, b in ((gl, gl0), (gm, gm0), (gr, gr0)):
            assert torch.allclose(a, b, rtol=1e-6, atol=0)


def test_misfit_packing_keeps_double_precision():
    buf = torch.zeros(8)
    J = 1.0 / 3.0 + 1e9
    edist.pack_misfit(buf, J)
    assert abs(edist.unpack_misfit(buf) - J) <= 1e-9 * J
