"""The rtm3d_b200 command-line host end to end on the GPU: input.json in, the reference's files out.

* Modeling writes the .seism chunks the reference writes, bit-identical to the reference program's
  own output (tests/golden/model_abc.npz).
* HBC migration of those chunks with the reference's extended velocity (load_vpe_from_file) writes
  the reference's RTMIMG file, bit-identical to its output (tests/golden/mig_hbc.npz).
* Frequency-domain migration ("fmig": true) writes the reference program's RTMIMG file
  (tests/golden/mig_fmig.npz).
* Several shots: the records are written, and read back, by a background task while the next shot
  runs; the files and the stacked image equal the library calls shot by shot."""
import glob
import json
import os
import subprocess

import numpy as np
import pytest

import rtmb
from rtm_cases import CASES, bitexact, input_json, layered_model

pytestmark = pytest.mark.gpu

BIN = os.path.join(os.path.dirname(__file__), "..", "rtm3d-demo_b200", "bin", "rtm3d_b200")


def run_cli(d, tmp):
    p = os.path.join(tmp, "in.json")
    with open(p, "w") as f:
        json.dump(d, f)
    r = subprocess.run([BIN, p], cwd=tmp, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return r


def read_record(d, sx, sy, sz):
    n = d["nt"] // d["ntstep"]
    out = []
    for c in range(n):
        f = os.path.join(d["datdir"], f"RTMSEISMOGRAM_S{sx}x{sy}x{sz}_NXNY_{d['receiver_count_x']}x"
                                      f"{d['receiver_count_y']}_NTSTART{c * d['ntstep']}_NTSTEP{d['ntstep']}.seism")
        out.append(np.fromfile(f, np.float32))
    return np.concatenate(out).reshape(n, d["receiver_count_x"], d["receiver_count_y"], d["ntstep"])


def test_cli_model_and_hbc_migration_match_reference_files(cuda, golden, tmp_path):
    case = CASES["golden"]
    tmp = str(tmp_path)
    vp = os.path.join(tmp, "vel.bin")
    layered_model(case).tofile(vp)
    d = input_json(case, vpfile=vp, workdir=tmp)
    d.update(modeling=True, migration=False)
    run_cli(d, tmp)
    rec = read_record(d, case["sx"], case["sy"], case["sz"])
    assert bitexact(rec, golden["model_abc"]["rec"])
    g = golden["mig_hbc"]
    g["vpe"].astype(np.float32).tofile(d["vpefile"])
    d.update(modeling=False, migration=True, boundary_condition="hbc", load_vpe_from_file=True)
    run_cli(d, tmp)
    files = glob.glob(os.path.join(d["outdir"], "RTMIMG_*"))
    assert len(files) == 1 and files[0].endswith(f"_NXNYNZ_{case['nx']}x{case['ny']}x{case['nz']}_NT{case['nt']}.bin.NP1")
    img = np.fromfile(files[0], np.float32).reshape(case["nx"], case["ny"], case["nz"])
    assert bitexact(img, g["img"])


def test_cli_fmig_matches_reference_file(cuda, golden, tmp_path):
    """"fmig": true runs the frequency-domain migration: the RTMIMG file equals the reference
    program's (tests/golden/mig_fmig.npz, the same band, all frequencies in one pass)."""
    case = CASES["golden"]
    tmp = str(tmp_path)
    vp = os.path.join(tmp, "vel.bin")
    layered_model(case).tofile(vp)
    d = input_json(case, vpfile=vp, workdir=tmp)
    d.update(modeling=True, migration=False)
    run_cli(d, tmp)
    g = golden["mig_fmig"]
    g["vpe"].astype(np.float32).tofile(d["vpefile"])
    d.update(modeling=False, migration=True, boundary_condition="hbc", load_vpe_from_file=True, fmig=True,
             fmig_min_freq=float(g["fmin"]), fmig_max_freq=float(g["fmax"]), fmig_nwstep=0)
    run_cli(d, tmp)
    files = glob.glob(os.path.join(d["outdir"], "RTMIMG_*"))
    assert len(files) == 1
    img = np.fromfile(files[0], np.float32).reshape(case["nx"], case["ny"], case["nz"])
    assert bitexact(img, g["img"])


def test_cli_twod_matches_reference_files(cuda, golden, tmp_path):
    """A 2D model (nx = 1) through the CLI: the .seism chunks and the HBC RTMIMG file equal the
    reference program's (tests/golden/twod.npz)."""
    case = dict(CASES["golden"], nx=1, sx=0, rsx=0, rcx=1, rdx=1)
    tmp = str(tmp_path)
    vp = os.path.join(tmp, "vel.bin")
    layered_model(case).tofile(vp)
    d = input_json(case, vpfile=vp, workdir=tmp)
    d.update(modeling=True, migration=False)
    run_cli(d, tmp)
    g = golden["twod"]
    assert bitexact(read_record(d, case["sx"], case["sy"], case["sz"]), g["rec"])
    g["vpe_hbc"].astype(np.float32).tofile(d["vpefile"])
    d.update(modeling=False, migration=True, boundary_condition="hbc", load_vpe_from_file=True)
    run_cli(d, tmp)
    img = np.fromfile(glob.glob(os.path.join(d["outdir"], "RTMIMG_*"))[0], np.float32).reshape(1, case["ny"], case["nz"])
    assert bitexact(img, g["img_hbc"])


def test_cli_several_shots_overlapped_io_matches_library(cuda, oracle, tmp_path):
    import torch
    case = CASES["golden"]
    tmp = str(tmp_path)
    vp = os.path.join(tmp, "vel.bin")
    v = layered_model(case)
    v.tofile(vp)
    d = input_json(case, vpfile=vp, workdir=tmp)
    d.update(modeling=True, migration=False, source_count_x=2, source_count_y=2, source_distance_x=5,
             source_distance_y=4, source_start_x=6, source_start_y=5, source_total=4, b200_rbc_seed=11)
    run_cli(d, tmp)
    shots = [(6 + 5 * i, 5 + 4 * j, case["sz"]) for i in range(2) for j in range(2)]
    # the library, shot by shot
    pm = rtmb.Params.from_input(dict(d, boundary_condition="hbc"), device=0)
    ctx = rtmb.Context(pm)
    ctx.load_v2dt2(rtmb.v2dt2(rtmb.prepare_velocity(v, case["blen"], "abc"), case["dt"]), from_host=True)
    recs = []
    for s in shots:
        r = torch.zeros((case["nt"] // case["ntstep"], case["rcx"], case["rcy"], case["ntstep"]), device=cuda)
        ctx.model_shot(*s, r)
        ctx.sync()
        recs.append(r.cpu().numpy())
        assert bitexact(read_record(d, *s), recs[-1])
    d.update(modeling=False, migration=True, boundary_condition="rbc")
    run_cli(d, tmp)
    img = np.fromfile(glob.glob(os.path.join(d["outdir"], "RTMIMG_*NS4_*"))[0], np.float32)
    mctx = rtmb.Context(rtmb.Params.from_input(dict(d, boundary_condition="rbc"), device=0))
    ve = rtmb.prepare_velocity(v, case["blen"], "rbc", seed=11)
    mctx.load_v2dt2(rtmb.v2dt2(ve, case["dt"]), from_host=True)
    stack = torch.zeros(mctx.padded_shape, device=cuda)
    one = torch.zeros_like(stack)
    for s, r in zip(shots, recs):
        mctx.migrate_shot(*s, torch.from_numpy(r).to(cuda), one)
        mctx.image_stack(stack, one)
    out = torch.zeros((case["nx"], case["ny"], case["nz"]), device=cuda)
    mctx.image_finalize(stack, out)
    mctx.sync()
    assert bitexact(img.reshape(out.shape), out.cpu().numpy())
