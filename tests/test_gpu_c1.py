"""The CPU-runnable modeling configuration at full size, on the GPU, against the reference program.

128^3 three-layer model at 10 m (1500 / 2500 / 3500 m/s from depths 0, 40 and 80 cells), a 32-cell
border (ABC velocity, every face tapered: RTMController.cpp:51-56, RTMFiniteDifferencesKernel.cpp:
169-216), 1000 steps of 1 ms, a 15 Hz Ricker at (64, 64, 4) and 64 x 64 receivers every 2 cells at
depth 4, stencil order 8, the record in four 250-step chunks.  tests/golden/c1_model.npz holds the
SHA-256 of the record the reference program (RTM3D.bin) wrote for this input and the traces of every
8th receiver; tests/golden/make_golden.py made it.

* The exact form, through the C ABI and through the rtm3d_b200 command-line host, must reproduce the
  reference's record bit for bit over the whole run (same digest).
* The FMA form must stay within the record tolerance (rel-L2 <= 1e-5) on the golden traces.
"""
import json
import os
import subprocess

import numpy as np
import pytest

import rtmb
from rtm_cases import C1, c1_model, input_json, lib_input, record_digest, rel_l2

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "c1_model.npz")
BIN = os.path.join(os.path.dirname(__file__), "..", "rtm3d-demo_b200", "bin", "rtm3d_b200")


@pytest.fixture(scope="module")
def c1_golden():
    return dict(np.load(GOLD))


def _model(cuda, flags):
    import torch
    v2 = rtmb.v2dt2(rtmb.prepare_velocity(c1_model(), C1["blen"], "abc"), C1["dt"])
    ctx = rtmb.Context(rtmb.Params.from_input(lib_input(C1), flags=flags, device=0))
    ctx.load_v2dt2(v2, from_host=True)
    rec = torch.full((C1["nt"] // C1["ntstep"], C1["rcx"], C1["rcy"], C1["ntstep"]), float("nan"), device=cuda)
    ctx.model_shot(C1["sx"], C1["sy"], C1["sz"], rec)
    ctx.sync()
    ctx.close()
    return rec.cpu().numpy()


def test_c1_exact_record_equals_reference_program(cuda, c1_golden):
    rec = _model(cuda, 0)
    assert tuple(rec.shape) == tuple(c1_golden["shape"])
    assert np.array_equal(rec[:, ::8, ::8, :].view(np.uint32), c1_golden["traces"].view(np.uint32))
    assert record_digest(rec) == str(c1_golden["sha256"]), "the 1000-step record differs from RTM3D.bin's"


def test_c1_fma_record_within_tolerance(cuda, c1_golden):
    rec = _model(cuda, rtmb.FLAG_FAST_FMA)
    err = rel_l2(rec[:, ::8, ::8, :], c1_golden["traces"])
    assert err <= 1e-5, err


def test_c1_cli_writes_the_reference_files(cuda, c1_golden, tmp_path):
    tmp = str(tmp_path)
    vp = os.path.join(tmp, "vel.bin")
    c1_model().tofile(vp)
    d = input_json(C1, vpfile=vp, workdir=tmp)
    d.update(modeling=True, migration=False, mname="c1")
    p = os.path.join(tmp, "in.json")
    with open(p, "w") as f:
        json.dump(d, f)
    r = subprocess.run([BIN, p], cwd=tmp, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    chunks = []
    for c in range(C1["nt"] // C1["ntstep"]):
        f = os.path.join(d["datdir"], f"RTMSEISMOGRAM_S{C1['sx']}x{C1['sy']}x{C1['sz']}_NXNY_{C1['rcx']}x{C1['rcy']}"
                                      f"_NTSTART{c * C1['ntstep']}_NTSTEP{C1['ntstep']}.seism")
        chunks.append(np.fromfile(f, np.float32))
    rec = np.concatenate(chunks).reshape(tuple(c1_golden["shape"]))
    assert record_digest(rec) == str(c1_golden["sha256"])
