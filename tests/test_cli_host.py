"""CPU tests of the rtm3d_b200 command-line host: it reads the reference's input.json and rejects bad
files with the reference's messages before any device work (RTMParam::validateParameters,
src/param/RTMParam.cpp:59-96; Main.cpp:11-20)."""
import json
import os
import subprocess

import pytest

from rtm_cases import CASES, input_json

BIN = os.path.join(os.path.dirname(__file__), "..", "rtm3d-demo_b200", "bin", "rtm3d_b200")


def run(args, cwd):
    return subprocess.run([BIN] + args, cwd=cwd, capture_output=True, text=True, timeout=60)


@pytest.fixture
def base(tmp_path):
    d = input_json(CASES["golden"], vpfile=str(tmp_path / "vel.bin"), workdir=str(tmp_path))
    return d, tmp_path


def write(d, tmp_path):
    p = tmp_path / "in.json"
    p.write_text(json.dumps(d))
    return str(p)


def test_binary_exists():
    assert os.access(BIN, os.X_OK), "build the CLI first (make -C rtm3d-demo_b200)"


def test_no_argument_is_an_error(tmp_path):
    r = run([], tmp_path)
    assert r.returncode != 0 and "forgot the input.json" in r.stdout


def test_missing_file(tmp_path):
    r = run([str(tmp_path / "nope.json")], tmp_path)
    assert r.returncode == 1 and "doesn't exists" in r.stdout


@pytest.mark.parametrize("key,value,expect", [
    ("nx", "24", "'nx' has wrong type"),            # a string where an unsigned is required
    ("dt", True, "'dt' has wrong type"),
    ("modeling", 1, "'modeling' has wrong type"),
])
def test_wrong_types(base, key, value, expect):
    d, tmp = base
    d[key] = value
    r = run([write(d, tmp)], tmp)
    assert r.returncode == 1 and expect in r.stdout, r.stdout


def test_missing_key(base):
    d, tmp = base
    del d["receiver_count_y"]
    r = run([write(d, tmp)], tmp)
    assert r.returncode == 1 and "'receiver_count_y' has wrong type" in r.stdout


@pytest.mark.parametrize("patch,expect", [
    (dict(nt=30, ntstep=40), "NT smaller than NTSTEP"),
    (dict(nt=100, ntstep=40), "multiple of ntstep"),
    (dict(fmig=True, fmig_min_freq=30.0, fmig_max_freq=20.0), "fmig_max_freq must be greater"),
    (dict(fmig=True, fmig_distributed_imaging=True), "fmig_distributed_imaging"),
    (dict(distributed_grid=True), "distributed_grid"),
])
def test_rejected_modes(base, patch, expect):
    d, tmp = base
    d.update(patch)
    r = run([write(d, tmp)], tmp)
    assert r.returncode == 1 and expect in r.stdout, r.stdout
