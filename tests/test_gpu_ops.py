"""GPU parity of the per-step operators (RTMPlatform mirror) against the CPU oracle.

The exact form is compared BIT-EXACT; the FMA form within a stated tolerance."""
import numpy as np
import pytest

import rtmb
from rtm_cases import CASES, bitexact, lib_input, rel_l2

pytestmark = pytest.mark.gpu


def make_ctx(case, flags=0, bc="hbc"):
    return rtmb.Context(rtmb.Params.from_input(lib_input(case, bc), flags=flags, device=0))


def dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


def host(t):
    return t.detach().cpu().numpy()


def rand_fields(shape, seed):
    rng = np.random.default_rng(seed)
    P = rng.standard_normal(shape).astype(np.float32)
    PP = rng.standard_normal(shape).astype(np.float32)
    V = (rng.random(shape) * 0.1).astype(np.float32)
    return P, PP, V


@pytest.mark.parametrize("flags", [0, rtmb.FLAG_NO_TMA], ids=["tma", "plain"])
@pytest.mark.parametrize("order", [2, 4, 6, 8, 10, 12, 14, 16])
@pytest.mark.parametrize("cname", ["golden", "odd"])
def test_step_bitexact(cuda, oracle, cname, order, flags):
    case = dict(CASES[cname], order=order)
    ctx = make_ctx(case, flags=flags)
    P, PP, V = rand_fields(ctx.padded_shape, order)
    dP, dPP, dV = dev(P, cuda), dev(PP, cuda), dev(V, cuda)
    ctx.step(dP, dPP, dV)
    ctx.sync()
    c = oracle.stencil_coefs(order, case["dx"], case["dy"], case["dz"])
    ref, _ = oracle.step(order, c, P, PP, V)
    assert bitexact(host(dPP), ref)
    assert bitexact(host(dP), P)  # P is read-only


@pytest.mark.parametrize("flags", [0, rtmb.FLAG_NO_TMA], ids=["tma", "plain"])
def test_step_bitexact_large(cuda, oracle, flags):
    """Several CTAs along every axis, several x chunks, aligned rows; both kernel forms."""
    case = CASES["mid"]
    ctx = make_ctx(case, flags=flags)
    P, PP, V = rand_fields(ctx.padded_shape, 1)
    dPP = dev(PP, cuda)
    ctx.step(dev(P, cuda), dPP, dev(V, cuda))
    ctx.sync()
    ref, _ = oracle.step(8, oracle.stencil_coefs(8, 10.0, 10.0, 10.0), P, PP, V)
    assert bitexact(host(dPP), ref)


@pytest.mark.parametrize("cname", ["golden", "odd", "mid"])
def test_step_fma_tolerance(cuda, oracle, cname):
    case = CASES[cname]
    ctx = make_ctx(case, flags=rtmb.FLAG_FAST_FMA)
    P, PP, V = rand_fields(ctx.padded_shape, 2)
    dPP = dev(PP, cuda)
    ctx.step(dev(P, cuda), dPP, dev(V, cuda))
    ctx.sync()
    ref, _ = oracle.step(case["order"], oracle.stencil_coefs(case["order"], case["dx"], case["dy"], case["dz"]),
                         P, PP, V)
    assert rel_l2(host(dPP), ref) < 1e-6  # single step, FMA contraction only


@pytest.mark.parametrize("cname", ["golden", "odd"])
@pytest.mark.parametrize("upper", [False, True])
def test_taper_bitexact(cuda, oracle, cname, upper):
    case = CASES[cname]
    ctx = make_ctx(case)
    P, _, _ = rand_fields(ctx.padded_shape, 3)
    d = dev(P, cuda)
    (ctx.taper_upper if upper else ctx.taper_all)(d)
    ctx.sync()
    t = oracle.taper_vector(case["blen"], case["taper_factor"])
    assert bitexact(host(d), oracle.taper(P, case["blen"], t, upper))


def test_source_receivers_upb_image(cuda, oracle):
    from oracle import OrcParams, fptr  # noqa: F401
    case = CASES["odd"]
    b, h = case["blen"], case["order"] // 2
    ctx = make_ctx(case)
    shp = ctx.padded_shape
    P, PP, V = rand_fields(shp, 4)
    # source
    d = dev(PP, cuda)
    ctx.apply_source(d, case["sx"], case["sy"], case["sz"], 17)
    ctx.sync()
    exp = PP.copy()
    w = oracle.ricker(case["nt"], case["dt"], case["fpeak"])
    exp[case["sx"] + b, case["sy"] + b, case["sz"] + b] += w[17]
    assert bitexact(host(d), exp)
    # receivers: save then restore (overwrite)
    nts = case["ntstep"]
    rec = np.zeros((case["rcx"], case["rcy"], nts), np.float32)
    drec = dev(rec, cuda)
    ctx.save_receivers(dev(PP, cuda), drec, 5)
    ctx.sync()
    idx_x = case["rsx"] + b + case["rdx"] * np.arange(case["rcx"])
    idx_y = case["rsy"] + b + case["rdy"] * np.arange(case["rcy"])
    rz = case["rdz"] + b
    exp_rec = rec.copy()
    exp_rec[:, :, 5] = PP[np.ix_(idx_x, idx_y, [rz])][:, :, 0]
    assert bitexact(host(drec), exp_rec)
    rng = np.random.default_rng(9)
    rec2 = rng.standard_normal(rec.shape).astype(np.float32)
    dP = dev(P, cuda)
    ctx.restore_receivers(dP, dev(rec2, cuda), 7)
    ctx.sync()
    exp = P.copy()
    exp[np.ix_(idx_x, idx_y, [rz])] = rec2[:, :, 7:8]
    assert bitexact(host(dP), exp)
    # upper border save / restore, 64-bit offsets in the [ntstep][nxe][nye][h] layout
    upb = np.zeros((nts, shp[0], shp[1], h), np.float32)
    dupb = dev(upb, cuda)
    ctx.save_upb(dev(P, cuda), dupb, 3)
    ctx.sync()
    exp_upb = upb.copy()
    exp_upb[3] = P[:, :, b - h:b]
    assert bitexact(host(dupb), exp_upb)
    dPP = dev(PP, cuda)
    ctx.restore_upb(dPP, dupb, 3)
    ctx.sync()
    exp = PP.copy()
    exp[:, :, b - h:b] = P[:, :, b - h:b]
    assert bitexact(host(dPP), exp)
    # image condition (CPU z range)
    img = rng.standard_normal(shp).astype(np.float32)
    di = dev(img, cuda)
    ctx.image(di, dev(P, cuda), dev(PP, cuda))
    ctx.sync()
    assert bitexact(host(di), oracle.image(img, P, PP, b))
    # finalize: order-2 filter + border removal; stack
    out = dev(np.zeros((case["nx"], case["ny"], case["nz"]), np.float32), cuda)
    ctx.image_finalize(di, out)
    acc = dev(P, cuda)
    ctx.image_stack(acc, dev(PP, cuda))
    ctx.sync()
    assert bitexact(host(out), oracle.filter_remove(host(di), b, case["dx"], case["dy"], case["dz"]))
    assert bitexact(host(acc), P + PP)


def test_step_reports_nan(cuda):
    case = CASES["golden"]
    ctx = make_ctx(case)
    shp = ctx.padded_shape
    P = np.zeros(shp, np.float32)
    P[20, 18, 22] = np.nan
    ctx.step(dev(P, cuda), dev(np.zeros(shp, np.float32), cuda), dev(np.ones(shp, np.float32), cuda))
    with pytest.raises(rtmb.RtmbError) as e:
        ctx.sync()
    assert e.value.code == rtmb.RTMB_ENAN
    ctx.sync()  # the flag is cleared after it is reported
