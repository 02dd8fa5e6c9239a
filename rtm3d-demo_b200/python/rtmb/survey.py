"""Shot-parallel migration of a survey over ranks: one process per GPU, shots dealt round-robin,
one join of the stacked images at the end.

This is the reference's distributed shot loop (rtmDistShotMigration,
src/controller/RTMAcousticController.cpp:172-269): the shot list is the source grid
(src/controller/RTMController.cpp:125-166, x outer, y inner), rank r takes shots r, r + N, r + 2N, ...
(shotNumber = sh0 + processRank, :193-199), migrates each on its own device and adds its image to a
per-rank stack (stackRegion, :223-225); rank 0 then joins the stacks (stackDistributedOutputImage ->
joinDistributedOutputImage, src/controller/RTMController.cpp:202-319), filters the image and strips
the border.  Here the ranks are torch.distributed processes (NCCL between GPUs, gloo on CPU) instead
of MPI, and the per-shot work is this library's migration driver.

The join has two modes:
  * exact (the reference's order): rank 0 gathers every rank's stack and adds them in rank order,
    out = remote + out for ranks 1 .. N-1, in FP32 as the reference does, so the result is the
    reference's image bit for bit for the same per-shot images;
  * reduce: one collective sum (dist.reduce), whose summation order is the backend's; with NCCL it
    crosses NVLink once per byte.  FP32 rounding may differ from the exact mode.
No shot is ever split across ranks (no halo exchange: the whole volume of a shot is on one GPU).
"""
from __future__ import annotations

from typing import Callable, Iterable, Sequence


def shot_positions(p: dict) -> list[tuple[int, int, int]]:
    """The reference's shot list (RTMController.cpp:139-165): for ix over source_count_x (outer) and
    iy over source_count_y (inner), (start_x + ix dist_x, start_y + iy dist_y, depth_z); a position
    outside the model raises, as the reference does ("Invalid Source Position")."""
    out = []
    for ix in range(int(p["source_count_x"])):
        for iy in range(int(p["source_count_y"])):
            sx = ix * int(p["source_distance_x"]) + int(p["source_start_x"])
            sy = iy * int(p["source_distance_y"]) + int(p["source_start_y"])
            sz = int(p["source_depth_z"])
            if sx >= p["nx"] or sy >= p["ny"] or sz >= p["nz"]:
                raise ValueError(f"Invalid Source Position: ({sx},{sy},{sz})")
            out.append((sx, sy, sz))
    return out


def rank_shots(nshots: int, rank: int, world: int) -> list[int]:
    """Shot indices of one rank: shotNumber = sh0 + rank for sh0 = 0, world, 2 world, ...
    (RTMAcousticController.cpp:193-199)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of world {world}")
    return list(range(rank, nshots, world))


def join_stacks(stack, group=None, exact: bool = True):
    """Joins the per-rank stacks into rank 0's: returns the joined stack on rank 0 and None on the
    other ranks.  exact: gather to rank 0 and add in rank order (the reference's sequence); else one
    dist.reduce (SUM).  Every rank must call it, with stacks of the same shape and dtype."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return stack
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    if world == 1:
        return stack
    if not exact:
        dist.reduce(stack, dst=0, group=group)
        return stack if rank == 0 else None
    parts = [torch.empty_like(stack) for _ in range(world)] if rank == 0 else None
    dist.gather(stack, parts, dst=0, group=group)
    if rank != 0:
        return None
    out = parts[0].clone()
    for pk in range(1, world):  # joinDistributedOutputImage: out = remote + out, ranks in order
        out = parts[pk] + out
    return out


def migrate_survey(p: dict, shots: Sequence[tuple[int, int, int]] | None = None,
                   migrate: Callable[[int, tuple[int, int, int]], object] | None = None,
                   stack=None, group=None, exact_join: bool = True,
                   context=None, load_record: Callable[[int, tuple[int, int, int]], object] | None = None,
                   finalize: bool = True):
    """Migrates the shots of this rank and joins the stacks on rank 0.

    p:        input.json parameters (the source grid keys give the shot list when shots is None).
    migrate:  per-shot image producer (shot index, position) -> padded image tensor; when None, the
              library runs: context (an rtmb.Context with v2dt2 loaded) migrates the record that
              load_record(index, position) returns into a padded FP32 image.
    stack:    this rank's padded FP32 stack (zeroed here); allocated like the first image when None.
    Returns (on rank 0) the joined padded stack, or with finalize and a context the final
    nx x ny x nz image (order-2 filter and border removal, RTMAcousticController.cpp:244-249);
    None on the other ranks."""
    import torch
    import torch.distributed as dist
    shots = list(shot_positions(p) if shots is None else shots)
    dist_on = dist.is_available() and dist.is_initialized()
    rank = dist.get_rank(group) if dist_on else 0
    world = dist.get_world_size(group) if dist_on else 1
    mine = rank_shots(len(shots), rank, world)
    if migrate is None:
        if context is None or load_record is None:
            raise ValueError("migrate_survey needs migrate, or a context and load_record")
        img = None

        def migrate(k, pos):
            nonlocal img
            if img is None:
                img = torch.empty(context.padded_shape, dtype=torch.float32, device=_device(context))
            context.migrate_shot(pos[0], pos[1], pos[2], load_record(k, pos), img)
            return img
    for k in mine:
        im = migrate(k, shots[k])
        if stack is None:
            stack = torch.zeros_like(im)
        if context is not None:
            context.image_stack(stack, im)  # RTMCube::stackRegion over the whole cube
        else:
            stack += im
    if stack is None:  # a rank without shots still takes part in the join
        if context is None:
            raise ValueError("a rank without shots needs a stack or a context to size it")
        stack = torch.zeros(context.padded_shape, dtype=torch.float32, device=_device(context))
    if context is not None:
        context.sync()
    joined = join_stacks(stack, group, exact_join)
    if joined is None or not finalize or context is None:
        return joined
    out = torch.empty((p["nx"], p["ny"], p["nz"]), dtype=torch.float32, device=joined.device)
    context.image_finalize(joined.contiguous(), out)
    context.sync()
    return out


def _device(context):
    import torch
    d = context.params.device
    return torch.device("cuda", d if d >= 0 else torch.cuda.current_device())


def iter_rank_positions(shots: Iterable[tuple[int, int, int]], rank: int, world: int):
    """(index, position) of this rank's shots, in the order the rank runs them."""
    shots = list(shots)
    for k in rank_shots(len(shots), rank, world):
        yield k, shots[k]
