"""Host logic of a multi-rank solve (one process per GPU): the shot split and
the one exchange of a gradient, run as gloo ranks on the CPU."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _local_sums(rank, n=(37, 29)):
    g = torch.Generator().manual_seed(100 + rank)
    # unnormalised imaging sums of the rank's shots (float32, as
    # adjoint_reference(..., normalize=False) returns them)
    ge = torch.randn(n, generator=g, dtype=torch.float32) * (10.0 ** rank)
    gs = torch.randn(n, generator=g, dtype=torch.float32) * 1e-3
    return ge, gs


def _rank_main(rank, world, port, out_dir, normalize):
    import importlib
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    fg = importlib.import_module("fast-gpr-fwi_b200")
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        first, count = fg.shots.shot_range(64 * world, rank, world)
        ge, gs = _local_sums(rank)
        fg.shots.combine_gradients(ge, gs, normalize=normalize)
        np.savez(os.path.join(out_dir, "rank%d.npz" % rank), ge=ge.numpy(), gs=gs.numpy(),
                 shots=np.array([first, count]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("normalize", [True, False])
def test_combine_gradients_two_ranks(tmp_path, normalize):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path), normalize), nprocs=world,
                       join=True, start_method="spawn")
    res = [np.load(tmp_path / ("rank%d.npz" % r)) for r in range(world)]
    sums = [_local_sums(r) for r in range(world)]
    for k, name in enumerate(("ge", "gs")):
        tot = sum(s[k].double() for s in sums)
        want = (tot / torch.linalg.vector_norm(tot) if normalize else tot).float().numpy()
        for r in range(world):
            # every rank holds the same bits, equal to the single-process total
            assert np.array_equal(res[r][name], want), (name, r)
    assert [tuple(r["shots"]) for r in res] == [(0, 64), (64, 64)]


def test_combine_gradients_single_process(fg):
    ge, gs = _local_sums(0)
    want = (ge.double() / torch.linalg.vector_norm(ge.double())).float()
    fg.shots.combine_gradients(ge, None)
    assert torch.equal(ge, want)


@pytest.mark.parametrize("shots,world", [(64, 1), (64, 8), (37, 4), (3, 8), (0, 2)])
def test_shot_range_partitions(fg, shots, world):
    got = [fg.shots.shot_range(shots, r, world) for r in range(world)]
    counts = [c for _, c in got]
    assert sum(counts) == shots
    assert max(counts) - min(counts) <= 1
    nxt = 0
    for first, count in got:
        assert first == nxt
        nxt += count


def test_shot_range_rejects_bad_rank(fg):
    with pytest.raises(ValueError):
        fg.shots.shot_range(10, 2, 2)
    with pytest.raises(ValueError):
        fg.shots.shot_range(-1, 0, 1)
