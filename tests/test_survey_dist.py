"""Shot-parallel survey migration on CPU ranks (gloo, world size 2): the shot partition and the
join of the per-rank stacks (rtmb.survey).

Each rank runs rtmb.survey.migrate_survey with a stand-in per-shot image (a seeded array that depends
on the shot index), so the test exercises the partition (shotNumber = sh0 + processRank,
RTMAcousticController.cpp:193-199) and the join (joinDistributedOutputImage,
RTMController.cpp:202-319) without a GPU.  Rank 0's joined stack must equal the reference's sequence
-- each rank adds its shots' images in shot order, rank 0 then adds the ranks' stacks in rank order --
bit for bit in the exact mode, and to FP32 rounding with the collective reduce."""
import os
import socket

import numpy as np
import pytest

from rtmb import survey

P = dict(nx=20, ny=18, nz=16, source_count_x=3, source_count_y=4, source_distance_x=5, source_distance_y=4,
         source_start_x=2, source_start_y=1, source_depth_z=2)
SHAPE = (6, 5, 7)


def fake_image(k: int) -> np.ndarray:
    return np.random.default_rng(100 + k).standard_normal(SHAPE).astype(np.float32)


def expected(world: int) -> np.ndarray:
    shots = survey.shot_positions(P)
    stacks = []
    for r in range(world):
        s = np.zeros(SHAPE, np.float32)
        for k in survey.rank_shots(len(shots), r, world):
            s = s + fake_image(k)
        stacks.append(s)
    out = stacks[0].copy()
    for r in range(1, world):
        out = stacks[r] + out
    return out


def test_shot_list_and_partition():
    shots = survey.shot_positions(P)
    assert len(shots) == 12
    assert shots[0] == (2, 1, 2) and shots[1] == (2, 5, 2) and shots[4] == (7, 1, 2)  # x outer, y inner
    for world in (1, 2, 3, 5, 16):
        parts = [survey.rank_shots(len(shots), r, world) for r in range(world)]
        assert sorted(k for part in parts for k in part) == list(range(len(shots)))
        for r, part in enumerate(parts):
            assert all(k % world == r for k in part)
    with pytest.raises(ValueError):
        survey.shot_positions(dict(P, source_count_x=5))  # 2 + 4 * 5 = 22 >= nx


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, exact: bool, out_path: str):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        got = survey.migrate_survey(P, migrate=lambda k, pos: torch.from_numpy(fake_image(k)), exact_join=exact)
        if rank == 0:
            np.save(out_path, got.numpy())
        else:
            assert got is None
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("exact", [True, False], ids=["exact_join", "reduce"])
def test_two_ranks_join_the_stack(tmp_path, exact):
    import torch.multiprocessing as mp
    world = 2
    out = str(tmp_path / "joined.npy")
    mp.start_processes(_rank_main, args=(world, _free_port(), exact, out), nprocs=world, start_method="spawn",
                       join=True)
    got = np.load(out)
    want = expected(world)
    if exact:
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    else:
        np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-5)


def test_single_process_is_the_shot_sum():
    import torch
    got = survey.migrate_survey(P, migrate=lambda k, pos: torch.from_numpy(fake_image(k)))
    assert np.array_equal(got.numpy().view(np.uint32), expected(1).view(np.uint32))
