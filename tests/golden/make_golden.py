"""Generate the golden fixtures of tests/golden/ by running the REFERENCE itself.

The reference CPU program (oracle/_ref/RTM3D.bin, built from the reference's sources by
``make -C oracle ref``) is driven through its own input.json on small seeded synthetic models:

  * model_abc.npz  -- modeling shot record (ABC velocity + all-face taper), reference .seism files
  * mig_hbc.npz    -- HBC migration image (RTMIMG file) with the extended velocity it used (vpe)
  * mig_rbc.npz    -- RBC migration image with its extended velocity
  * mig_fmig.npz   -- frequency-domain RTM image (fmig = true) with its extended velocity
  * twod.npz       -- 2D model (nx = 1): record, HBC / RBC / fmig images and a 2D step vector
  * ops.npz        -- per-operator vectors from the reference CPU platform (oracle/_ref/librtmref.so)
  * c1_model.npz   -- the full-size modeling configuration (128^3 + 32-cell border, 1000 steps): the
                      SHA-256 of the reference's whole record and every 8th receiver's traces

Run:  python tests/golden/make_golden.py [names...]   (needs oracle/_ref, i.e. the reference sources;
      names: model mig ops fmig twod c1, default all)
"""
from __future__ import annotations

import glob
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from oracle import REF_BIN, Reference  # noqa: E402
from rtm_cases import C1, c1_model, input_json, layered_model, record_digest, CASES  # noqa: E402


FMIG = dict(fmig_min_freq=5.0, fmig_max_freq=40.0, fmig_nwstep=2)


def run_reference(case: dict, mode: str, workdir: str, vpe_path: str | None = None, extra: dict | None = None,
                  v: np.ndarray | None = None):
    """Run RTM3D.bin for one case. mode: 'model' | 'hbc' | 'rbc'. Returns output arrays."""
    v = layered_model(case) if v is None else v
    vp = os.path.join(workdir, "vel.bin")
    v.tofile(vp)
    d = input_json(case, vpfile=vp, workdir=workdir)
    if mode == "model":
        d.update(modeling=True, migration=False)
    else:
        d.update(modeling=False, migration=True, boundary_condition=mode,
                 save_vpe_file=True, vpefile=vpe_path or os.path.join(workdir, f"vpe_{mode}.bin"))
    d.update(extra or {})
    jp = os.path.join(workdir, f"{mode}.json")
    with open(jp, "w") as f:
        json.dump(d, f)
    subprocess.run([REF_BIN, jp], check=True, capture_output=True, cwd=workdir)
    return d


def read_record(d: dict):
    files = glob.glob(os.path.join(d["datdir"], "RTMSEISMOGRAM_*.seism"))
    files.sort(key=lambda f: int(f.split("NTSTART")[1].split("_")[0]))
    n = d["nt"] // d["ntstep"]
    assert len(files) == n, files
    return np.concatenate([np.fromfile(f, np.float32) for f in files]).reshape(
        n, d["receiver_count_x"], d["receiver_count_y"], d["ntstep"])


def fmig_fixture(case: dict, rec: np.ndarray, wd: str):
    """Frequency-domain RTM of the modeled shot (HBC-extended velocity; the CPU build runs every
    frequency in one pass whatever fmig_nwstep says)."""
    for f in glob.glob(os.path.join(wd, "out", "RTMIMG_*")):
        os.remove(f)
    dm = run_reference(case, "hbc", wd, vpe_path=os.path.join(wd, "vpe_fmig.bin"), extra=dict(fmig=True, **FMIG))
    img = np.fromfile(glob.glob(os.path.join(wd, "out", "RTMIMG_*"))[0], np.float32)
    img = img.reshape(case["nx"], case["ny"], case["nz"])
    vpe = np.fromfile(dm["vpefile"], np.float32).reshape(
        case["nx"] + 2 * case["blen"], case["ny"] + 2 * case["blen"], case["nz"] + 2 * case["blen"])
    np.savez_compressed(os.path.join(HERE, "mig_fmig.npz"), img=img, vpe=vpe, rec=rec,
                        fmin=FMIG["fmig_min_freq"], fmax=FMIG["fmig_max_freq"])


def twod_fixture(wd_root: str):
    """2D models (nx = 1; the reference's rtmStep2D): modeling record, HBC / RBC / fmig images with
    the extended velocities they used, and a per-operator 2D step vector."""
    case = dict(CASES["golden"], nx=1, sx=0, rsx=0, rcx=1, rdx=1)
    out = {}
    with tempfile.TemporaryDirectory(dir=wd_root) as wd:
        rec = read_record(run_reference(case, "model", wd))
        out["rec"] = rec
        for name, bc, extra in (("hbc", "hbc", None), ("rbc", "rbc", None),
                                ("fmig", "hbc", dict(fmig=True, **FMIG))):
            for f in glob.glob(os.path.join(wd, "out", "RTMIMG_*")):
                os.remove(f)
            dm = run_reference(case, bc, wd, vpe_path=os.path.join(wd, f"vpe2d_{name}.bin"), extra=extra)
            out[f"img_{name}"] = np.fromfile(glob.glob(os.path.join(wd, "out", "RTMIMG_*"))[0], np.float32).reshape(
                1, case["ny"], case["nz"])
            out[f"vpe_{name}"] = np.fromfile(dm["vpefile"], np.float32).reshape(
                1 + 2 * case["blen"], case["ny"] + 2 * case["blen"], case["nz"] + 2 * case["blen"])
    R = Reference()
    rng = np.random.default_rng(17)
    ny, nz, b = 12, 9, 6
    shp = (1 + 2 * b, ny + 2 * b, nz + 2 * b)
    P = rng.standard_normal(shp).astype(np.float32)
    PP = rng.standard_normal(shp).astype(np.float32)
    V = (rng.random(shp) * 0.1).astype(np.float32)
    out.update(P=P, PP=PP, V=V)
    for order in (4, 8):
        out[f"step{order}"], _ = R.step(1, ny, nz, b, order, 10.0, 12.5, 7.5, P, PP, V)
    out.update(fmin=FMIG["fmig_min_freq"], fmax=FMIG["fmig_max_freq"])
    np.savez_compressed(os.path.join(HERE, "twod.npz"), **out)


def c1_fixture():
    """The full-size modeling configuration: the reference's record (64 x 64 receivers x 1000
    steps, 16 MB) is kept as its SHA-256 and the traces of every 8th receiver in x and y."""
    with tempfile.TemporaryDirectory() as wd:
        d = run_reference(C1, "model", wd, v=c1_model())
        rec = read_record(d)
    np.savez_compressed(os.path.join(HERE, "c1_model.npz"), sha256=np.array(record_digest(rec)),
                        shape=np.array(rec.shape), traces=rec[:, ::8, ::8, :].copy(),
                        rms=np.array(float(np.sqrt(np.mean(rec.astype(np.float64) ** 2)))))


def main(names=("model", "mig", "ops", "fmig", "twod", "c1")):
    if not os.path.exists(REF_BIN):
        raise SystemExit("oracle/_ref/RTM3D.bin missing: run `make -C oracle ref` first")
    if "c1" in names:
        c1_fixture()
        if set(names) == {"c1"}:
            print("golden fixtures written to", HERE)
            return
    rng = np.random.default_rng(7)
    case = CASES["golden"]
    with tempfile.TemporaryDirectory() as wd:
        d = run_reference(case, "model", wd)
        rec = read_record(d)
        if "model" in names:
            np.savez_compressed(os.path.join(HERE, "model_abc.npz"), rec=rec)
        if "fmig" in names:
            fmig_fixture(case, rec, wd)
        if "twod" in names:
            twod_fixture(wd)
        for bc in ("hbc", "rbc") if "mig" in names else ():
            for f in glob.glob(os.path.join(wd, "out", "RTMIMG_*")):
                os.remove(f)
            dm = run_reference(case, bc, wd)
            img = np.fromfile(glob.glob(os.path.join(wd, "out", "RTMIMG_*"))[0], np.float32)
            img = img.reshape(case["nx"], case["ny"], case["nz"])
            vpe = np.fromfile(dm["vpefile"], np.float32).reshape(
                case["nx"] + 2 * case["blen"], case["ny"] + 2 * case["blen"], case["nz"] + 2 * case["blen"])
            np.savez_compressed(os.path.join(HERE, f"mig_{bc}.npz"), img=img, vpe=vpe, rec=rec)

    if "ops" not in names:
        print("golden fixtures written to", HERE)
        return
    # per-operator vectors from the reference CPU platform
    R = Reference()
    nx, ny, nz, b = 10, 12, 9, 6
    shp = (nx + 2 * b, ny + 2 * b, nz + 2 * b)
    P = rng.standard_normal(shp).astype(np.float32)
    PP = rng.standard_normal(shp).astype(np.float32)
    V = (rng.random(shp) * 0.1).astype(np.float32)
    out = dict(P=P, PP=PP, V=V)
    for order in (2, 4, 8, 12):
        out[f"coefs{order}"] = R.stencil_coefs(order, 10.0, 12.5, 7.5)
        out[f"step{order}"], _ = R.step(nx, ny, nz, b, order, 10.0, 12.5, 7.5, P, PP, V)
    out["taper"] = R.taper_vector(b, 0.2)
    out["taper_all"] = R.taper(P, nx, ny, nz, b, 0.2, upper=False)
    out["taper_upper"] = R.taper(P, nx, ny, nz, b, 0.2, upper=True)
    out["image"] = R.image(P, PP, V, nx, ny, nz, b)
    out["filter"] = R.filter_remove(P, b, 10.0, 12.5, 7.5)
    out["ricker"] = R.ricker(500, 0.001, 15.0)
    vel = (1500 + 3000 * rng.random((nx, ny, nz))).astype(np.float32)
    out["vel"] = vel
    for bc in ("abc", "rbc", "hbc"):
        out[f"borders_{bc}"] = R.extend_init_borders(vel, b, bc, seed=1234)
    np.savez_compressed(os.path.join(HERE, "ops.npz"), **out)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main(tuple(sys.argv[1:]) or ("model", "mig", "ops", "fmig", "twod", "c1"))
