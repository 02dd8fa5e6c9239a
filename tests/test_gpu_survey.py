"""rtmb.survey.migrate_survey with the library on one GPU: the survey's shots migrated through the
C ABI, stacked and finalised, equal the same shots migrated one by one and stacked with
rtmb_image_stack, then filtered with rtmb_image_finalize, bit for bit (the exact form)."""
import numpy as np
import pytest

import rtmb
from rtm_cases import CASES, layered_model, lib_input
from rtmb import survey

pytestmark = pytest.mark.gpu


def test_survey_equals_shot_by_shot(cuda, oracle):
    import torch
    case = CASES["golden"]
    p = dict(lib_input(case, "rbc"), source_count_x=2, source_count_y=2, source_distance_x=7,
             source_distance_y=6, source_start_x=5, source_start_y=4, source_depth_z=2)
    ve = oracle.extend_init_borders(layered_model(case), case["blen"], "rbc", seed=7)
    v2 = oracle.v2dt2(ve, case["dt"])
    ctx = rtmb.Context(rtmb.Params.from_input(p, device=0))
    ctx.load_v2dt2(v2, from_host=True)
    shape = (case["nt"] // case["ntstep"], case["rcx"], case["rcy"], case["ntstep"])
    recs = [torch.from_numpy(np.random.default_rng(k).standard_normal(shape).astype(np.float32) * 1e-2).to(cuda)
            for k in range(4)]
    got = survey.migrate_survey(p, context=ctx, load_record=lambda k, pos: recs[k])
    stack = torch.zeros(ctx.padded_shape, device=cuda)
    img = torch.empty(ctx.padded_shape, device=cuda)
    for k, pos in enumerate(survey.shot_positions(p)):
        ctx.migrate_shot(*pos, recs[k], img)
        ctx.image_stack(stack, img)
    want = torch.empty((case["nx"], case["ny"], case["nz"]), device=cuda)
    ctx.image_finalize(stack, want)
    ctx.sync()
    assert np.array_equal(got.cpu().numpy().view(np.uint32), want.cpu().numpy().view(np.uint32))
