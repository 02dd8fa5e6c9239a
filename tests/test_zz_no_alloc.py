"""rtmb_model_shot_noalloc: modeling for callers that cannot allocate device memory.

Some callers cannot call cudaMalloc -- a host framework whose allocator owns the GPU's memory, or a
latency-sensitive loop that cannot take cudaMalloc's implicit synchronisation.  The no-allocation
entry point keeps its scratch in a fixed 64 MiB array inside the library.  These tests call it
through the C ABI twice in a row (the scratch keeps the first call's contents, so the second call
checks that everything which must start at zero is cleared) and compare each record with the
context-based rtmb_model_shot, bit for bit (the exact stencil form reproduces the reference's
arithmetic, so the two entry points must agree exactly).  They also check that a call leaves the
device's free memory unchanged, and that what the entry point cannot serve (the learned boundary,
host pointers, blen above 1024, grids beyond the scratch) is rejected before any launch.  The file
is named to be collected last.
"""
import numpy as np
import pytest

import rtmb
from rtm_cases import CASES, bitexact, layered_model, lib_input

pytestmark = pytest.mark.gpu


def _record_with_context(case, v2, cuda):
    import torch
    ctx = rtmb.Context(rtmb.Params.from_input(lib_input(case), device=0))
    ctx.load_v2dt2(v2, from_host=True)
    rec = torch.zeros((case["nt"] // case["ntstep"], case["rcx"], case["rcy"], case["ntstep"]), device=cuda)
    ctx.model_shot(case["sx"], case["sy"], case["sz"], rec)
    ctx.sync()
    return rec.cpu().numpy()


@pytest.mark.parametrize("cname", ["golden", "mid"])
def test_noalloc_matches_context_entry_point_twice(cuda, cname):
    import torch
    case = CASES[cname]
    v2 = rtmb.v2dt2(rtmb.prepare_velocity(layered_model(case), case["blen"], "abc"), case["dt"])
    want = _record_with_context(case, v2, cuda)
    params = rtmb.Params.from_input(lib_input(case), device=0)
    dv2 = torch.from_numpy(v2).to(cuda)
    shape = (case["nt"] // case["ntstep"], case["rcx"], case["rcy"], case["ntstep"])
    for call in range(2):
        rec = torch.full(shape, float("nan"), device=cuda)  # every sample must be written
        rtmb.model_shot_noalloc(params, dv2, case["sx"], case["sy"], case["sz"], rec)
        torch.cuda.synchronize()
        got = rec.cpu().numpy()
        assert bitexact(got, want), f"call {call + 1} differs from rtmb_model_shot"


def test_noalloc_allocates_no_device_memory(cuda):
    """The entry point's contract: a warmed-up call leaves the device's free memory unchanged (the
    caller's stream carries no other work meanwhile)."""
    import torch
    case = CASES["mid"]
    v2 = rtmb.v2dt2(rtmb.prepare_velocity(layered_model(case), case["blen"], "abc"), case["dt"])
    params = rtmb.Params.from_input(lib_input(case), device=0)
    dv2 = torch.from_numpy(v2).to(cuda)
    rec = torch.zeros((case["nt"] // case["ntstep"], case["rcx"], case["rcy"], case["ntstep"]), device=cuda)
    rtmb.model_shot_noalloc(params, dv2, case["sx"], case["sy"], case["sz"], rec)  # warm-up: scratch lookup
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    rtmb.model_shot_noalloc(params, dv2, case["sx"], case["sy"], case["sz"], rec)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes during the call"


def test_noalloc_rejects_what_needs_a_context_or_host_memory(cuda):
    import torch
    case = CASES["golden"]
    shape = (case["nt"] // case["ntstep"], case["rcx"], case["rcy"], case["ntstep"])
    v2 = rtmb.v2dt2(rtmb.prepare_velocity(layered_model(case), case["blen"], "abc"), case["dt"])
    dv2 = torch.from_numpy(v2).to(cuda)
    rec = torch.zeros(shape, device=cuda)
    learned = rtmb.Params.from_input(lib_input(case), device=0)
    learned.boundary = rtmb.BC_LEARNED
    with pytest.raises(rtmb.RtmbError) as e:
        rtmb.model_shot_noalloc(learned, dv2, case["sx"], case["sy"], case["sz"], rec)
    assert e.value.code == rtmb.RTMB_EINVAL and "LEARNED" in str(e.value)
    params = rtmb.Params.from_input(lib_input(case), device=0)
    host_rec = np.zeros(shape, np.float32)  # pageable host memory: rejected before any launch
    with pytest.raises(rtmb.RtmbError) as e:
        rtmb.model_shot_noalloc(params, dv2, case["sx"], case["sy"], case["sz"], host_rec)
    assert e.value.code == rtmb.RTMB_EINVAL and "device memory" in str(e.value)
    wide = rtmb.Params.from_input(dict(lib_input(case), blen=1025), device=0)
    with pytest.raises(rtmb.RtmbError) as e:
        rtmb.model_shot_noalloc(wide, dv2, case["sx"], case["sy"], case["sz"], rec)
    assert e.value.code == rtmb.RTMB_EINVAL and "1024" in str(e.value)


def test_noalloc_rejects_grids_beyond_its_scratch(cuda):
    import torch
    big = dict(CASES["mid"], nx=256, ny=256, nz=256, blen=16, rcx=8, rcy=8)  # 288^3: 2 fields > 64 MiB
    params = rtmb.Params.from_input(lib_input(big), device=0)
    dummy = torch.zeros(16, device=cuda)
    with pytest.raises(rtmb.RtmbError) as e:
        rtmb.model_shot_noalloc(params, dummy, big["sx"], big["sy"], big["sz"], dummy)
    assert e.value.code == rtmb.RTMB_EINVAL
    assert "64 MiB" in str(e.value)
