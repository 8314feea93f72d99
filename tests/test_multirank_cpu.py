"""Multi-rank logic of the row/facet sharding (obit_b200.shard) on CPU: two
gloo ranks on 127.0.0.1 replicate the component table from rank 0, each
applies the model to its own rows, and the union is bit-identical to one
process applying it to every row.  The per-rank apply step is the FP64 oracle
here, standing in for the device call (which needs a GPU)."""
import socket

import numpy as np
import pytest

from obit_b200 import shard


def test_row_shard_partitions_exactly():
    for nrows in (0, 1, 7, 100, 100801):
        for world in (1, 2, 3, 8):
            spans = [shard.row_shard(nrows, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == nrows
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [hi - lo for lo, hi in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard.row_shard(10, 2, 2)


def test_facet_assignment_is_balanced_and_complete():
    rng = np.random.default_rng(5)
    work = np.exp(rng.uniform(np.log(1e9), np.log(1e13), 96))
    for world in (1, 2, 4, 8):
        a = shard.facet_assignment(work, world)
        flat = sorted(i for r in a for i in r)
        assert flat == list(range(96))
        loads = [sum(work[i] for i in r) for r in a]
        # LPT bound: makespan <= 4/3 of the optimum >= max(mean, largest)
        assert max(loads) <= 4.0 / 3.0 * max(sum(work) / world, max(work)) + 1.0
        assert a == shard.facet_assignment(list(work), world)  # deterministic


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port):
    import sys
    from pathlib import Path

    root = Path(__file__).resolve().parent.parent
    for p in (root, root / "oracle", root / "tests"):
        sys.path.insert(0, str(p))
    import datetime

    import torch
    import torch.distributed as dist

    import oracle
    from helpers import small
    from obit_b200 import shard as S
    from obit_b200 import uvdata as U

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        uv, sky = small(U.MOD_GAUSS_SPEC, nrow=53, nchan=12, nif=2, nstok=2, ncomp=40, seed=31)
        comps = torch.from_numpy(sky.comps.copy())
        if rank != 0:
            comps.zero_()  # only rank 0 holds the model
        S.broadcast_model(comps)
        assert np.array_equal(comps.numpy(), sky.comps)
        sky.comps = comps.numpy()
        lo, hi = S.row_shard(uv.nvis, rank, world)
        mine = oracle.apply_fp64(uv.rows(lo, hi), sky, nthreads=1) if hi > lo else \
            np.zeros((0, uv.lrec), np.float32)
        parts = [None] * world
        dist.all_gather_object(parts, (lo, hi, mine))
        got = np.concatenate([p[2] for p in sorted(parts, key=lambda p: p[0])])
        want = oracle.apply_fp64(uv, sky, nthreads=1)
        assert np.array_equal(got, want)
        assert S.max_over_ranks(rank + 1.5) == world + 0.5
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_subtract_equals_single_process(world):
    mp = pytest.importorskip("torch.multiprocessing")
    mp.spawn(_worker, args=(world, _free_port()), nprocs=world, join=True)


def _facet_worker(rank, world, port):
    import sys
    from pathlib import Path

    root = Path(__file__).resolve().parent.parent
    for p in (root, root / "oracle", root / "tests"):
        sys.path.insert(0, str(p))
    import datetime

    import torch.distributed as dist

    import oracle
    from helpers import small
    from obit_b200 import shard as S
    from obit_b200 import uvdata as U

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # uneven facets: different rows, channels, IFs and components
        specs = [(U.MOD_POINT_SPEC, 30 + 17 * i, 8 + 4 * (i % 3), 1 + i % 2, 20 + 13 * i, 70 + i)
                 for i in range(7)]
        facets = [small(mt, nrow=nr, nchan=nc, nif=ni, nstok=2, ncomp=ncp, seed=sd)
                  for mt, nr, nc, ni, ncp, sd in specs]
        work = [uv.nvis * uv.nchan * uv.nif * sky.ncomp for uv, sky in facets]
        mine = S.facet_assignment(work, world)[rank]  # no communication
        done = {i: oracle.apply_fp64(facets[i][0], facets[i][1], nthreads=1) for i in mine}
        parts = [None] * world
        dist.all_gather_object(parts, done)
        got = {}
        for d in parts:
            assert not set(d) & set(got)  # each facet on exactly one rank
            got.update(d)
        assert sorted(got) == list(range(len(facets)))
        for i, (uv, sky) in enumerate(facets):
            assert np.array_equal(got[i], oracle.apply_fp64(uv, sky, nthreads=1))
        loads = [sum(work[i] for i in S.facet_assignment(work, world)[r]) for r in range(world)]
        assert max(loads) - min(loads) <= max(work)  # greedy LPT balance
        assert S.max_over_ranks(float(len(mine))) == max(len(a) for a in S.facet_assignment(work, world))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_facet_sharded_subtract_equals_single_process(world):
    """Whole facets per rank (bench.py --workload config5 under torchrun): the
    union of the ranks' facets is every facet once, each applied as a single
    process applies it."""
    mp = pytest.importorskip("torch.multiprocessing")
    mp.spawn(_facet_worker, args=(world, _free_port()), nprocs=world, join=True)
