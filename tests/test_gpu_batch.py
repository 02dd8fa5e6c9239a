"""Batched multi-shot migration (rtmb_migrate_batch): shots on uneven aperture sub-volumes of a survey
advance together, one launch per time step for all of them, and their images are stacked in FP64.
Each shot's contribution must equal the single-shot driver's on the same aperture bit for bit (the
batched launch runs the same kernel body), stacked at the aperture's origin."""
import numpy as np
import pytest

import rtmb

pytestmark = pytest.mark.gpu

BLEN = 12
VOLUME = (64, 56, 40)  # nz + 2*blen = 64
APERTURES = [  # (ox, oy, nx, ny), full depth; uneven sizes
    (0, 0, 40, 36),
    (20, 10, 44, 46),
    (8, 4, 32, 40),
]
NT, NTSTEP = 60, 30


def survey_model():
    nx, ny, nz = VOLUME
    rng = np.random.default_rng(5)
    v = np.full(VOLUME, 1800.0, np.float32)
    v[:, :, nz // 2:] = 2600.0
    v += (rng.random(VOLUME) * 40).astype(np.float32)
    return v


def params(nx, ny, nz, rcx, rcy):
    return dict(nx=nx, ny=ny, nz=nz, blen=BLEN, nt=NT, ntstep=NTSTEP, stencil_order=8, dx=10.0, dy=10.0, dz=10.0,
                dt=0.001, fpeak=20.0, taper_factor=0.2, receiver_start_x=0, receiver_start_y=0, receiver_depth_z=2,
                receiver_distance_x=2, receiver_distance_y=2, receiver_count_x=rcx, receiver_count_y=rcy,
                boundary_condition="rbc")


def build_shots(cuda):
    import torch
    v = survey_model()
    rng = np.random.default_rng(9)
    shots, keep = [], []
    for k, (ox, oy, nx, ny) in enumerate(APERTURES):
        nz = VOLUME[2]
        ve = rtmb.prepare_velocity(v[ox:ox + nx, oy:oy + ny, :], BLEN, "rbc", seed=11 + k)
        v2 = torch.from_numpy(rtmb.v2dt2(ve, 0.001)).to(cuda)
        rcx, rcy = nx // 2, ny // 2
        rec = torch.from_numpy((rng.standard_normal((NT // NTSTEP, rcx, rcy, NTSTEP)) * 1e-3).astype(np.float32)).to(cuda)
        s = rtmb.Shot(nx=nx, ny=ny, nz=nz, ox=ox, oy=oy, oz=0, sx=nx // 2, sy=ny // 2, sz=1,
                      receiver_start_x=0, receiver_start_y=0, receiver_depth_z=2, receiver_distance_x=2,
                      receiver_distance_y=2, receiver_count_x=rcx, receiver_count_y=rcy,
                      v2dt2=v2.data_ptr(), rec=rec.data_ptr())
        shots.append(s)
        keep += [v2, rec]
    return shots, keep


def one_by_one(shots, flags, cuda):
    """The single-shot drivers on each aperture, stacked at the origins in FP64."""
    import torch
    stack = np.zeros(VOLUME, np.float64)
    for s in shots:
        p = rtmb.Params.from_input(params(s.nx, s.ny, s.nz, s.receiver_count_x, s.receiver_count_y), flags=flags,
                                   device=0)
        ctx = rtmb.Context(p)
        n = ctx.padded_shape
        ctx.load_v2dt2(s.v2dt2, from_host=False)
        rec = s.rec
        if flags & (rtmb.FLAG_STORE_F16 | rtmb.FLAG_STORE_BF16):
            acc = torch.zeros(n, dtype=torch.float64, device=cuda)
            ctx.migrate_shot_acc64(s.sx, s.sy, s.sz, rec, acc)
            ctx.sync()
            img = acc.cpu().numpy()
        else:
            im = torch.zeros(n, dtype=torch.float32, device=cuda)
            ctx.migrate_shot(s.sx, s.sy, s.sz, rec, im)
            ctx.sync()
            img = im.cpu().numpy().astype(np.float64)
        stack[s.ox:s.ox + s.nx, s.oy:s.oy + s.ny, :] += img[BLEN:-BLEN, BLEN:-BLEN, BLEN:-BLEN]
    return stack


@pytest.mark.parametrize("flags", [0, rtmb.FLAG_FAST_FMA, rtmb.FLAG_STORE_F16,
                                   rtmb.FLAG_FAST_FMA | rtmb.FLAG_USE_GRAPH],
                         ids=["exact", "fma", "f16", "fma-graph"])
def test_batch_matches_single_shots(cuda, flags):
    import torch
    shots, keep = build_shots(cuda)
    nx, ny, nz = VOLUME
    ctx = rtmb.Context(rtmb.Params.from_input(params(nx, ny, nz, 1, 1), flags=flags, device=0))
    stack = torch.zeros(VOLUME, dtype=torch.float64, device=cuda)
    ctx.migrate_batch(shots, stack)
    ctx.sync()
    got = stack.cpu().numpy()
    ref = one_by_one(shots, flags & ~rtmb.FLAG_USE_GRAPH, cuda)
    assert np.abs(ref).max() > 0
    assert np.array_equal(got, ref), np.abs(got - ref).max()
    launches = ctx.launches
    assert launches <= 3 * NT + 2 * len(shots), launches  # one launch per batch step, not per shot


# more shots than one launch group, apertures clipped at every survey edge (origin 0 and far edge)
EDGE_APERTURES = APERTURES + [
    (24, 20, 40, 36),  # reaches the far x and y edges (24 + 40 = 64, 20 + 36 = 56)
    (0, 24, 28, 32),   # x from 0, y to the far edge
    (36, 0, 28, 24),   # x to the far edge, y from 0
    (12, 12, 36, 36),
]


def build_edge_shots(cuda):
    global APERTURES
    saved = APERTURES
    APERTURES = EDGE_APERTURES
    try:
        return build_shots(cuda)
    finally:
        APERTURES = saved


@pytest.mark.parametrize("group", [1, 3, 12])
def test_batch_groups_match_single_shots(cuda, group):
    """Seven shots on apertures clipped at the survey's edges, run in launch groups of 1, 3 (3 + 3 + 1)
    and 12 shots: the stack equals the single-shot drivers' bit for bit whatever the grouping."""
    import torch
    shots, keep = build_edge_shots(cuda)
    nx, ny, nz = VOLUME
    ctx = rtmb.Context(rtmb.Params.from_input(params(nx, ny, nz, 1, 1), flags=rtmb.FLAG_FAST_FMA | rtmb.FLAG_USE_GRAPH,
                                              device=0))
    ctx.set_batch_group(group)
    stack = torch.zeros(VOLUME, dtype=torch.float64, device=cuda)
    ctx.migrate_batch(shots, stack)
    ctx.sync()
    ref = one_by_one(shots, rtmb.FLAG_FAST_FMA, cuda)
    assert np.array_equal(stack.cpu().numpy(), ref)


def test_autotune_batch_picks_a_group_and_keeps_results(cuda):
    import torch
    shots, keep = build_edge_shots(cuda)
    nx, ny, nz = VOLUME
    ctx = rtmb.Context(rtmb.Params.from_input(params(nx, ny, nz, 1, 1), flags=rtmb.FLAG_FAST_FMA, device=0))
    g, rate = ctx.autotune_batch(shots)
    assert g in (1, 2, 3, 4, 6) and rate > 0
    stack = torch.zeros(VOLUME, dtype=torch.float64, device=cuda)
    ctx.migrate_batch(shots, stack)
    ctx.sync()
    assert np.array_equal(stack.cpu().numpy(), one_by_one(shots, rtmb.FLAG_FAST_FMA, cuda))
    with pytest.raises(rtmb.RtmbError):
        ctx.set_batch_group(25)
