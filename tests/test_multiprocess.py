"""Multi-rank host logic on CPU with the gloo backend (world size 2): the point
sharding and all-gather used for internal points on several GPUs, and the bench's
max-over-ranks timing.  The per-rank compute is the oracle, so no GPU is needed."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    for p in (ROOT, os.path.join(ROOT, "oracle")):
        if p not in sys.path:
            sys.path.insert(0, p)
    from datetime import timedelta

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import bench
        import oracle as O
        from bem3d_elastostatic_b200.mesh import cube_grid_points, uniaxial_cube
        from bem3d_elastostatic_b200.shard import shard_range, sharded_points

        # max over ranks (the bench's step time)
        t = bench.allreduce_max(1.5 + rank, world)
        bench.barrier(world)

        mesh = uniaxial_cube(2, young=1.0, nu=0.3, points=cube_grid_points([0.2, 0.4, 0.6, 0.8]))
        orc = O.Oracle(mesh)
        ref = orc.run()
        seen = []

        def fn(p0, p1):
            seen.append((p0, p1))
            return orc.internal_points(ref["u"], ref["t"], p0, p1)

        u, s, pr, vm = sharded_points(fn, mesh.l)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), t=t, u=u, s=s, pr=pr, vm=vm,
                 block=np.array(seen[0]), expect=np.array(shard_range(mesh.l, rank, world)))
    finally:
        dist.destroy_process_group()


def test_shard_range_covers_once():
    from bem3d_elastostatic_b200.shard import shard_range

    for count in (0, 1, 5, 64, 1000):
        for world in (1, 2, 3, 8):
            blocks = [shard_range(count, r, world) for r in range(world)]
            assert blocks[0][0] == 0 and blocks[-1][1] == count
            assert all(a[1] == b[0] for a, b in zip(blocks, blocks[1:]))
            sizes = [p1 - p0 for p0, p1 in blocks]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def test_gloo_two_ranks_internal_points(tmp_path):
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from bem3d_elastostatic_b200.mesh import cube_grid_points, uniaxial_cube

    mesh = uniaxial_cube(2, young=1.0, nu=0.3, points=cube_grid_points([0.2, 0.4, 0.6, 0.8]))
    ref = O.Oracle(mesh).run()
    for r in range(world):
        d = np.load(tmp_path / f"rank{r}.npz")
        assert float(d["t"]) == 2.5
        assert tuple(d["block"]) == tuple(d["expect"])
        # every rank holds the full arrays, bitwise those of a single-process run
        np.testing.assert_array_equal(d["u"], ref["u_int"])
        np.testing.assert_array_equal(d["s"], ref["sigma"])
        np.testing.assert_array_equal(d["pr"], ref["prin"])
        np.testing.assert_array_equal(d["vm"], ref["vm"])
