#!/usr/bin/env python3
"""Benchmark: single-shot reverse-time migration (RTM) on B200 through librtm3d_b200.

Workload (the reference's RTM path on a synthetic model): 512^3 grid at 10 m, seeded background
v(z) = 1500 + 0.6 z_m m/s clipped at 4500, a 4500 m/s salt ellipsoid (semi-axes 120 x 100 x 60 cells
centred at (256, 256, 300)), a Gaussian-smoothed (sigma = 8 cells) +-3% random perturbation, random
boundary (RBC) border of 40 cells, 12 Hz Ricker source at the surface centre, receivers every 2
cells over the whole surface, dt = 1 ms, 3000 steps, stencil order 8.  The shot record comes from
this library's own modeling pass on the same model (ABC border, tapered faces).

One bench "step" = one migrated shot: forward pass, backward pass with source-wavefield
reconstruction, receiver back-propagation and cross-correlation imaging.  value = G point-updates/s
(padded grid points x (3 nt - 2) sweeps per shot / device time).  e2e = the same metric through the
host-buffer C-ABI call (record copied in, padded image copied out, inside the timed region).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

--impl reference times the reference's own CPU program (oracle/_ref/RTM3D.bin, built from its
sources) on a truncated-nt sample of the same workload on this host's cores.

The line's "forms" object compares, on the same grid and shot with nt cut to --forms-nt steps, the
plain FP32 form (bit-exact with the reference CPU path), the FMA form and the 16-bit storage forms:
device time per sweep, the seconds per shot that gives at the full nt, and the image rel-L2 against
the FP64 GPU oracle run on the same grid and record.  "chosen" is the fastest form whose image
stays within rel-L2 1e-3 of the FP64 oracle.
"""
from __future__ import annotations

import argparse
import csv
import io
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "rtm3d-demo_b200", "python"))

HBM_FALLBACK_GBS = 6650.0
L2_BYTES = 126 * 2**20


# ------------------------------------------------------------------------------------------ workload
METRIC = "G point-updates/s per migrated RTM shot (512^3 RBC, nt=3000)"


def workload(n: int, nt: int, ny: int | None = None, nz: int | None = None) -> dict:
    """input.json parameters of the benchmark shot on an n x ny x nz model (default cubic; the
    workload is 512^3): 40-cell RBC border, 12 Hz Ricker at the surface centre, receivers every 2
    cells over the whole surface."""
    ny = n if ny is None else ny
    nz = n if nz is None else nz
    return dict(nx=n, ny=ny, nz=nz, blen=40, nt=nt, ntstep=nt, stencil_order=8, dx=10.0, dy=10.0, dz=10.0,
                dt=0.001, fpeak=12.0, taper_factor=0.2, receiver_start_x=0, receiver_start_y=0,
                receiver_depth_z=0, receiver_distance_x=2, receiver_distance_y=2,
                receiver_count_x=n // 2, receiver_count_y=ny // 2, boundary_condition="rbc",
                sx=n // 2, sy=ny // 2, sz=0)


def salt_model(nx: int, ny: int | None = None, nz: int | None = None, seed: int = 1234) -> np.ndarray:
    """Seeded synthetic velocity (x slowest, z fastest), float32 m/s, on an nx x ny x nz grid at 10 m:
    the 512^3 salt model scaled per axis to the grid (ellipsoid semi-axes 120 x 100 x 60 cells and
    centre (256, 256, 300) at 512^3; the background depends on depth in metres only)."""
    from scipy import ndimage
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    fx, fy, fz = nx / 512.0, ny / 512.0, nz / 512.0
    z = np.arange(nz, dtype=np.float32) * 10.0
    v = np.broadcast_to(np.minimum(1500.0 + 0.6 * z, 4500.0), (nx, ny, nz)).astype(np.float32)
    ex = ((np.arange(nx, dtype=np.float32) - 256 * fx) / (120 * fx)) ** 2
    ey = ((np.arange(ny, dtype=np.float32) - 256 * fy) / (100 * fy)) ** 2
    ez = ((np.arange(nz, dtype=np.float32) - 300 * fz) / (60 * fz)) ** 2
    salt = (ex[:, None, None] + ey[None, :, None] + ez[None, None, :]) <= 1.0
    v[salt] = 4500.0
    # +-3% perturbation: white noise on a grid 8x coarser, Gaussian-smoothed (sigma 1 coarse cell
    # = 8 cells) and interpolated trilinearly to the model grid
    rng = np.random.default_rng(seed)
    nc = [max(4, k // 8) for k in (nx, ny, nz)]
    pert = ndimage.gaussian_filter(rng.standard_normal(nc).astype(np.float32), 1.0, mode="wrap")
    pert = ndimage.zoom(pert, (nx / nc[0], ny / nc[1], nz / nc[2]), order=1, mode="nearest")[:nx, :ny, :nz]
    pert *= 0.03 / max(float(np.abs(pert).max()), 1e-12)
    v = v * (1.0 + pert)
    # keep the order-8 leapfrog inside its CFL bound (v dt / dx <= 0.453 at 10 m, 1 ms)
    return np.clip(v, 1500.0, 4500.0).astype(np.float32)


def n_points(p: dict) -> int:
    b = p["blen"]
    return (p["nx"] + 2 * b) * (p["ny"] + 2 * b) * (p["nz"] + 2 * b)


def updates_per_shot(p: dict) -> int:
    """Point updates of one migrated shot: nt forward steps, nt-2 source-reconstruction steps and
    nt receiver steps over the padded grid."""
    return n_points(p) * (3 * p["nt"] - 2)


# ------------------------------------------------------------------------------------------ helpers
def measured_hbm_gbs() -> tuple[float, str]:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


def dual_kernel_name(tuning) -> str:
    """Kernel of the dual backward step: variants 4-7 are the merged form (every thread steps both
    wavefields), 0-3 the split form; 5 is the default."""
    dv = 5 if not tuning else int(tuning.get("dual_variant", 5))
    return "dual_merged_kernel" if dv >= 4 else "dual_step_kernel"


def dual_bytes_per_point(tuning, nt: int) -> float:
    """Algorithmic bytes per grid point of a dual backward step, averaged over a shot's nt - 2 dual
    launches: 36 (read S, S_prev, R, R_prev, v2dt2 and IMG, write S_new, R_new and IMG); the merged
    form pairs its launches on the image, so the first of a pair moves 28 (no image) and the second
    36, an odd last launch 36."""
    n = max(nt - 2, 1)
    if dual_kernel_name(tuning) != "dual_merged_kernel":
        return 36.0
    skip = n // 2 if n % 2 == 0 else (n - 1) // 2
    return (28.0 * skip + 36.0 * (n - skip)) / n


def ncu_traffic_per_point(kind: str):
    """DRAM bytes per grid point of one launch, from the committed ncu summary (profiles/)."""
    path = os.path.join(ROOT, "profiles", "step_kernels_ncu.md")
    try:
        for line in open(path):
            if line.startswith(f"dram_bytes_per_point[{kind}]"):
                return float(line.split("=")[1].split()[0])
    except Exception:
        pass
    return None


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.out = None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            self.out = tempfile.TemporaryFile(mode="w+")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        if not self.out:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.out.seek(0)
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for row in csv.reader(io.StringIO(self.out.read())):
            if len(row) < 9:
                continue
            try:
                sm.append(float(row[1]))
                smax.append(float(row[2]))
            except ValueError:
                continue
            for name, val in zip(names, row[5:9]):
                if val.strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------------------------------ reference CPU
def ref_input(p: dict, workdir: str, vp: str, nts: int, threads: int, migration: bool) -> dict:
    """input.json of the reference program for the workload p with nt cut to nts."""
    sx, sy, sz = p["sx"], p["sy"], p["sz"]
    return dict(mname="bench", vpfile=vp, vpefile=os.path.join(workdir, "vpe.bin"), save_vpe_file=False,
                outdir=os.path.join(workdir, "out"), tmpdir=os.path.join(workdir, "tmp"),
                datdir=os.path.join(workdir, "dat"), nx=p["nx"], ny=p["ny"], nz=p["nz"], blen=p["blen"],
                width_m=0, height_m=0, depth_m=0, nt=nts, dz=p["dz"], dy=p["dy"], dx=p["dx"], dt=p["dt"],
                fpeak=p["fpeak"], fmax=30.0, taper_factor=p["taper_factor"], stencil_order=p["stencil_order"],
                modeling=not migration, migration=migration, rtm_type="rtm",
                boundary_condition=p["boundary_condition"], source_total=1, source_start_x=sx, source_start_y=sy,
                source_depth_z=sz, source_distance_x=1, source_distance_y=1, source_count_x=1, source_count_y=1,
                receiver_total=p["receiver_count_x"] * p["receiver_count_y"],
                receiver_start_x=p["receiver_start_x"], receiver_start_y=p["receiver_start_y"],
                receiver_depth_z=p["receiver_depth_z"], receiver_distance_x=p["receiver_distance_x"],
                receiver_distance_y=p["receiver_distance_y"], receiver_count_x=p["receiver_count_x"],
                receiver_count_y=p["receiver_count_y"], ntstep=nts, nthreads=threads, load_vpe_from_file=False,
                save_snapshots=False, distributed_grid=False, snapshot_step=10, fmig=False, fmig_max_freq=30.0,
                fmig_min_freq=1.0, fmig_nwstep=1, fmig_distributed_imaging=False, fpga_xclbin="",
                fpga_fwd_kernel="", fpga_bwd_kernel="", verbose=True)


def run_reference_program(binary: str, p: dict, v: np.ndarray, rec: np.ndarray | None, nts: int, workdir: str,
                          migration: bool = True):
    """Run one of the reference's own programs (RTM3D.bin, or its GPU build RTM3D_GPU.bin) on the
    workload p with nt cut to nts: an RBC migration of the given record (the program builds its own
    random border), or a modeling shot.  Returns (seconds of the program's own migration or modeling
    timer, point updates, threads, the record it wrote when modeling)."""
    if not os.path.exists(binary):
        raise FileNotFoundError(f"{os.path.relpath(binary, ROOT)} is not built")
    for sub in ("out", "tmp", "dat"):
        os.makedirs(os.path.join(workdir, sub), exist_ok=True)
    vp = os.path.join(workdir, "vel.bin")
    if not os.path.exists(vp):
        v.tofile(vp)
    sx, sy, sz = p["sx"], p["sy"], p["sz"]
    seism = os.path.join(workdir, "dat", f"RTMSEISMOGRAM_S{sx}x{sy}x{sz}_NXNY_{p['receiver_count_x']}x"
                                         f"{p['receiver_count_y']}_NTSTART0_NTSTEP{nts}.seism")
    if migration:  # the record chunk [rcx][rcy][nts] under the reference's file name (RTMBase.hpp:131-138)
        np.ascontiguousarray(rec[..., :nts]).tofile(seism)
    elif os.path.exists(seism):
        os.remove(seism)
    threads = os.cpu_count() or 1
    d = ref_input(p, workdir, vp, nts, threads, migration)
    jp = os.path.join(workdir, "run.json")
    with open(jp, "w") as f:
        json.dump(d, f)
    r = subprocess.run([binary, jp], capture_output=True, text=True, cwd=workdir, timeout=1200)
    if r.returncode != 0:
        raise RuntimeError(f"{os.path.basename(binary)} failed: {r.stdout[-400:]} {r.stderr[-400:]}")
    key = '"migration_time"' if migration else '"modeling_time"'
    t = None
    for line in r.stdout.splitlines():
        if key in line:
            t = float(line.split(":")[1].strip().rstrip(","))
    if not t:
        raise RuntimeError(f"no {key} in the report of {os.path.basename(binary)}")
    pts = n_points(p)
    upd = pts * (3 * nts - 2) if migration else pts * nts
    out_rec = None if migration else np.fromfile(seism, np.float32)
    return t, upd, threads, out_rec


def workload_config(args, p: dict, world: int) -> dict:
    """The workload description shared by both arms of the benchmark."""
    b = p["blen"]
    return {"workload": f"rtm_rbc_{args.size}^3_nt{args.nt}",
            "grid": [p["nx"] + 2 * b, p["ny"] + 2 * b, p["nz"] + 2 * b], "nt": p["nt"], "stencil_order": 8,
            "boundary": "rbc", "shots_per_step_per_gpu": 1,
            "l2": "inputs larger than L2 (%.0f MB per wavefield)" % (n_points(p) * 4 / 1e6),
            "parallelism": f"shot-parallel x{world}"}


def ref_gpu_bin() -> str:
    return os.path.join(ROOT, "oracle", "_ref", "RTM3D_GPU.bin")


def ref_cpu_bin() -> str:
    return os.path.join(ROOT, "oracle", "_ref", "RTM3D.bin")


# ------------------------------------------------------------------------------------------ arms
def build_inputs(p: dict, with_abc: bool):
    import rtmb
    v = salt_model(p["nx"], p["ny"], p["nz"])
    vpe = rtmb.prepare_velocity(v, p["blen"], "rbc", seed=1234)
    v2 = rtmb.v2dt2(vpe, p["dt"])
    v2m = rtmb.v2dt2(rtmb.prepare_velocity(v, p["blen"], "abc"), p["dt"]) if with_abc else None
    return v, vpe, v2, v2m


FORMS = ("fp32_exact", "fp32_fma", "fp16", "bf16", "fp16_diff", "bf16_diff")
C3_FORMS = ("fp32_exact", "fp32_fma", "fp16", "bf16", "fp16_diff")
ALL_FORMS = FORMS + ("fp16_img64", "bf16_img64", "fp16_diff_img64", "bf16_diff_img64")


def form_flags(rtmb, form: str) -> int:
    """Flags of a form: fp32_exact (bit-exact with the reference CPU path), fp32_fma, 16-bit storage
    of the two levels (fp16, bf16), of the level and its increment (*_diff), FP64 image (*_img64)."""
    f = {"fp32_exact": 0, "fp32_fma": rtmb.FLAG_FAST_FMA}.get(form)
    if f is not None:
        return f
    f = rtmb.FLAG_STORE_F16 if form.startswith("fp16") else rtmb.FLAG_STORE_BF16
    if "_diff" in form:
        f |= rtmb.FLAG_STORE_DIFF
    if form.endswith("_img64"):
        f |= rtmb.FLAG_IMG_F64
    return f


def rel_l2_dev(a, ref, ref_norm: float) -> float:
    import torch
    return float(torch.linalg.vector_norm(a.double() - ref)) / (ref_norm if ref_norm > 0 else 1.0)


def time_ctx(ctxs, fn) -> float:
    """Device milliseconds of the work fn() enqueues on the contexts ctxs: the contexts run on one
    torch stream for the call and the two CUDA events are recorded on that stream (a context's own
    stream is non-blocking, so events on torch's default stream would not bracket its work)."""
    import torch
    ctxs = ctxs if isinstance(ctxs, (list, tuple)) else [ctxs]
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    for c in ctxs:
        c.set_stream(s.cuda_stream)
    try:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        fn()
        e1.record(s)
        s.synchronize()
    finally:
        for c in ctxs:
            c.set_stream(None)
    return e0.elapsed_time(e1)


def compare_forms(p: dict, v2: np.ndarray, v2m: np.ndarray | None, rec_full, dev, nt_cmp: int,
                  forms=FORMS, autotune: bool = True) -> dict:
    """Per-form device time and error against the FP64 GPU oracle on the same grid, over nt_cmp
    steps (the full nt by default): the migrated image of the given record (image rel-L2) and, when
    v2m (the modeling velocity) is given, the modeled shot record (record rel-L2)."""
    import torch
    import rtmb
    q = dict(p, nt=nt_cmp, ntstep=nt_cmp)
    rec = rec_full[..., :nt_cmp].contiguous()
    sx, sy, sz = q["sx"], q["sy"], q["sz"]
    d = dev.index or 0
    ctx = rtmb.Context(rtmb.Params.from_input(q, device=d))
    ctx.load_v2dt2(v2, from_host=True)
    shape = ctx.padded_shape
    ref = torch.zeros(shape, dtype=torch.float64, device=dev)
    t0 = time.time()
    ctx.migrate_shot_f64(sx, sy, sz, rec, ref)
    ctx.sync()
    f64_s = time.time() - t0
    ctx.close()
    ref_norm = float(torch.linalg.vector_norm(ref))
    rec_ref = None
    if v2m is not None:
        mc = rtmb.Context(rtmb.Params.from_input(dict(q, boundary_condition="hbc"), device=d))
        mc.load_v2dt2(v2m, from_host=True)
        rec_ref = torch.zeros(rec.shape, dtype=torch.float64, device=dev)
        mc.model_shot_f64(sx, sy, sz, rec_ref)
        mc.sync()
        mc.close()
        rec_ref_norm = float(torch.linalg.vector_norm(rec_ref))
    sweeps_cmp = 3 * nt_cmp - 2
    sweeps_full = 3 * p["nt"] - 2
    out = {}
    img = torch.zeros(shape, dtype=torch.float32, device=dev)
    for name in forms:
        fl = form_flags(rtmb, name)
        c = rtmb.Context(rtmb.Params.from_input(q, flags=fl, device=d))
        c.load_v2dt2(v2, from_host=True)
        if autotune:
            c.autotune_full()
        # one full shot, timed (buffers are allocated on first use)
        ms = time_ctx(c, lambda: c.migrate_shot(sx, sy, sz, rec, img))
        c.close()
        per_sweep = ms / sweeps_cmp
        r = {"ms_per_sweep": round(per_sweep, 4), "s_per_shot": round(per_sweep * sweeps_full / 1e3, 3),
             "gpt_s": round(n_points(p) / (per_sweep * 1e-3) / 1e9, 2),
             "image_rel_l2_vs_fp64": float("%.3e" % rel_l2_dev(img, ref, ref_norm))}
        if rec_ref is not None and "_diff" in name:
            r["record_rel_l2_vs_fp64"] = None  # the increment form runs RBC migration only, no modeling
        elif rec_ref is not None:
            mc = rtmb.Context(rtmb.Params.from_input(dict(q, boundary_condition="hbc"), flags=fl, device=d))
            mc.load_v2dt2(v2m, from_host=True)
            got = torch.zeros(rec.shape, dtype=torch.float32, device=dev)
            mc.model_shot(sx, sy, sz, got)
            mc.sync()
            mc.close()
            r["record_rel_l2_vs_fp64"] = float("%.3e" % rel_l2_dev(got, rec_ref, rec_ref_norm))
        out[name] = r
    ok = {k: v for k, v in out.items() if v["image_rel_l2_vs_fp64"] <= 1e-3}
    chosen = min(ok, key=lambda k: ok[k]["ms_per_sweep"]) if ok else "fp32_exact"
    note = (f"every form run over the full nt={nt_cmp}" if nt_cmp == p["nt"] else
            f"s_per_shot scaled to nt={p['nt']} from the nt={nt_cmp} run")
    res = {"nt": nt_cmp, "grid": list(shape), "note": f"{note}; FP64 oracle migration took {f64_s:.1f} s",
           "forms": out, "chosen": chosen}
    if "fp32_exact" in out:
        res["chosen_vs_plain"] = round(out["fp32_exact"]["ms_per_sweep"] / out[chosen]["ms_per_sweep"], 3)
    return res


def run_precision(args, forms=FORMS) -> dict:
    """The precision configuration: 896 x 896 x 512 at 10 m (the salt model scaled to the grid),
    40-cell RBC border (976 x 976 x 592 padded), 12 Hz, receivers every 2 cells over the surface,
    the full nt; each storage form's shot record and image against the FP64 GPU oracle on the same
    grid, and its device time.  The record comes from this library's FP32 modeling pass."""
    import torch
    import rtmb
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    nx, ny, nz = args.c3_grid
    p = workload(nx, args.nt, ny=ny, nz=nz)
    v = salt_model(nx, ny, nz)
    v2 = rtmb.v2dt2(rtmb.prepare_velocity(v, p["blen"], "rbc", seed=1234), p["dt"])
    v2m = rtmb.v2dt2(rtmb.prepare_velocity(v, p["blen"], "abc"), p["dt"])
    mctx = rtmb.Context(rtmb.Params.from_input(dict(p, boundary_condition="hbc"), flags=rtmb.FLAG_FAST_FMA,
                                               device=0))
    rec = torch.zeros((1, p["receiver_count_x"], p["receiver_count_y"], p["nt"]), dtype=torch.float32, device=dev)
    mctx.load_v2dt2(v2m, from_host=True)
    mctx.model_shot(p["sx"], p["sy"], p["sz"], rec)
    mctx.sync()
    mctx.close()
    res = compare_forms(p, v2, v2m, rec, dev, p["nt"], forms)
    res["workload"] = f"precision_{nx}x{ny}x{nz}_nt{p['nt']}"
    return res


def reference_gpu_bar(args, p: dict, v: np.ndarray, rec, value: float) -> dict:
    """The reference's own GPU program (oracle/_ref/RTM3D_GPU.bin: its CUDA back-end built for
    sm_100a from its sources) on this GPU: the modeling configuration in full (128^3 + 32-cell
    border, 1000 steps), and the RBC migration of the benchmark shot with nt cut to --ref-gpu-nt,
    each timed by the program's own timer; beside them this library on the same work."""
    import torch
    import rtmb
    out = {"program": "oracle/_ref/RTM3D_GPU.bin (the reference's kernel/gpu/rtmgpu_finitediff.cu, sm_100a)"}
    binary = ref_gpu_bin()
    with tempfile.TemporaryDirectory() as wd:
        nts = args.ref_gpu_nt
        sec, upd, _, _ = run_reference_program(binary, p, v, rec.cpu().numpy(), nts, wd)
        out["rtm_rbc"] = {"nt_sample": nts, "gpt_s": round(upd / sec / 1e9, 3),
                          "s_per_shot_extrapolated": round(sec * (3 * p["nt"] - 2) / (3 * nts - 2), 2),
                          "this_library_gpt_s": round(value, 3), "speedup": round(value / (upd / sec / 1e9), 2)}
    mp, vm = c1_workload()
    with tempfile.TemporaryDirectory() as wd:
        sec, upd, _, ref_rec = run_reference_program(binary, mp, vm, None, mp["nt"], wd, migration=False)
    dev = torch.device("cuda", 0)
    v2 = rtmb.v2dt2(rtmb.prepare_velocity(vm, mp["blen"], "abc"), mp["dt"])
    ctx = rtmb.Context(rtmb.Params.from_input(mp, flags=rtmb.FLAG_FAST_FMA | rtmb.FLAG_USE_GRAPH, device=0))
    ctx.load_v2dt2(v2, from_host=True)
    got = torch.zeros((1, 64, 64, mp["nt"]), device=dev)
    ctx.model_shot(mp["sx"], mp["sy"], mp["sz"], got)  # warm-up: graph capture
    ctx.sync()
    ms = time_ctx(ctx, lambda: ctx.model_shot(mp["sx"], mp["sy"], mp["sz"], got))
    ctx.close()
    g = got.cpu().numpy().reshape(-1).astype(np.float64)
    r = ref_rec.astype(np.float64)
    out["model_c1"] = {"nt": mp["nt"], "s_per_shot": round(sec, 4), "gpt_s": round(upd / sec / 1e9, 3),
                       "this_library_s_per_shot": round(ms / 1e3, 4), "speedup": round(sec / (ms / 1e3), 2),
                       "record_rel_l2_vs_this_library": float("%.3e" % (np.linalg.norm(g - r) / np.linalg.norm(g)))}
    return out


def c1_workload():
    """The CPU-runnable modeling configuration (128^3 three-layer model, 32-cell border, 1000 steps)."""
    n, blen = 128, 32
    v = np.full((n, n, n), 3500.0, np.float32)
    v[:, :, :40] = 1500.0
    v[:, :, 40:80] = 2500.0
    p = dict(nx=n, ny=n, nz=n, blen=blen, nt=1000, ntstep=1000, stencil_order=8, dx=10.0, dy=10.0, dz=10.0,
             dt=0.001, fpeak=15.0, taper_factor=0.2, receiver_start_x=0, receiver_start_y=0, receiver_depth_z=4,
             receiver_distance_x=2, receiver_distance_y=2, receiver_count_x=64, receiver_count_y=64,
             boundary_condition="hbc", sx=64, sy=64, sz=4)
    return p, v


def run_b200(args, rank: int, world: int, local_rank: int) -> dict | None:
    import torch
    import rtmb
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    p = workload(args.size, args.nt)
    flags = form_flags(rtmb, args.form)
    params = rtmb.Params.from_input(p, flags=flags, device=local_rank)
    v, vpe, v2, v2m = build_inputs(p, with_abc=True)
    stream = torch.cuda.Stream(device=dev)
    # shot-parallel ranks (rtmb.survey): one shot position per rank on a line through the surface
    # centre, 8 cells apart, dealt as the reference deals its shot list (shotNumber = sh0 + rank)
    from rtmb import survey
    line = dict(p, source_count_x=world, source_count_y=1, source_distance_x=8, source_distance_y=1,
                source_start_x=p["sx"] - 4 * (world - 1), source_start_y=p["sy"], source_depth_z=p["sz"])
    shots = survey.shot_positions(line)
    (k_mine,) = survey.rank_shots(len(shots), rank, world)
    sx, sy, sz = shots[k_mine]
    rec_shape = (1, p["receiver_count_x"], p["receiver_count_y"], p["nt"])

    # the shot record: this library's modeling pass (FP32, FMA form) on the ABC-bordered model
    mctx = rtmb.Context(rtmb.Params.from_input(dict(p, boundary_condition="hbc"), flags=rtmb.FLAG_FAST_FMA,
                                               device=local_rank))
    mctx.set_stream(stream.cuda_stream)
    with torch.cuda.stream(stream):
        rec = torch.zeros(rec_shape, dtype=torch.float32, device=dev)
    mctx.load_v2dt2(v2m, from_host=True)
    mctx.model_shot(sx, sy, sz, rec)
    mctx.close()
    v2m_keep = v2m  # the modeling velocity, for the per-form record errors

    ctx = rtmb.Context(params)
    ctx.set_stream(stream.cuda_stream)
    ctx.load_v2dt2(v2, from_host=True)
    # the launch shape measured on this context (rtmb_autotune_full), before the warm-up
    tuning = ctx.autotune_full() if not args.no_autotune else None
    shape = ctx.padded_shape
    with torch.cuda.stream(stream):
        img = torch.zeros(shape, dtype=torch.float32, device=dev)
        stack = torch.zeros(shape, dtype=torch.float32, device=dev)

    for _ in range(args.warmup):
        ctx.migrate_shot(sx, sy, sz, rec, img)

    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    stream.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = ctx.launches
    ctx.profile(True)
    with ClockSampler(local_rank) as clocks:
        e0.record(stream)
        for _ in range(args.steps):
            ctx.migrate_shot(sx, sy, sz, rec, img)
            ctx.image_stack(stack, img)           # the shot image stack (RTMAcousticController.cpp:223-225)
        if world > 1:
            with torch.cuda.stream(stream):
                survey.join_stacks(stack, exact=False)  # the ranks' stacks summed on rank 0 (NCCL)
        e1.record(stream)
        stream.synchronize()
    ms = e0.elapsed_time(e1)
    prof = ctx.profile_read()
    ctx.profile(False)
    launches = ctx.launches - launches0
    clk = clocks.summary()

    # e2e: the host-buffer C-ABI call, record in and image out through pinned host memory
    rec_h = rec.cpu().pin_memory()
    img_h = torch.empty(shape, dtype=torch.float32).pin_memory()
    stream.synchronize()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(args.steps):
        ctx.migrate_shot_host(sx, sy, sz, rec_h, img_h)
    e3.record(stream)
    stream.synchronize()
    ms_e2e = e2.elapsed_time(e3)

    # max over ranks
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([ms, ms_e2e], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, ms_e2e = float(t[0]), float(t[1])
    upd = updates_per_shot(p)
    total_upd = upd * args.steps * world
    value = total_upd / (ms * 1e-3) / 1e9
    e2e_value = total_upd / (ms_e2e * 1e-3) / 1e9

    # roofline of the dominant kernel (largest summed device time)
    peak, peak_kind = measured_hbm_gbs()
    cat = max(("forward", "backward_source", "backward_receiver", "backward_dual"), key=lambda k: prof[k]["ms"])
    bpp = {"forward": 16, "backward_source": 16, "backward_receiver": 28, "backward_dual": dual_bytes_per_point(
        tuning, p["nt"])}[cat]
    per_launch_ms = prof[cat]["ms"] / max(prof[cat]["launches"], 1)
    bytes_launch = bpp * n_points(p)
    achieved = bytes_launch / (per_launch_ms * 1e-3) / 1e9
    tpp = ncu_traffic_per_point(cat)
    if rank != 0:
        return None
    out = {
        "metric": METRIC,
        "value": round(value, 3),
        "unit": "Gpt/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms / args.steps, 3),
        "s_per_shot": round(ms / args.steps / 1e3, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": {"fp32_exact": "f32", "fp32_fma": "f32-fma"}.get(args.form, args.form + "-storage/f32-math"),
        "data": "synthetic (seeded salt model; record from this library's modeling pass)",
        "config": workload_config(args, p, world),
        "form": args.form,
        "tuning": tuning,
        "e2e": {"value": round(e2e_value, 3), "unit": "Gpt/s",
                "h2d_bytes_per_step": int(np.prod(rec_shape) * 4), "d2h_bytes_per_step": int(np.prod(shape) * 4)},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": (dual_kernel_name(tuning) if cat == "backward_dual" else "tma_step_kernel") +
                     f" ({cat})", "achieved": round(achieved, 1),
                     "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "traffic": (round(tpp * n_points(p)) if tpp else None),
                     "bytes_per_launch": bytes_launch, "launch_ms": round(per_launch_ms, 4)},
        "kernels": {k: {"ms_total": round(v_["ms"], 2), "launches": v_["launches"]} for k, v_ in prof.items()
                    if v_["launches"]},
        "clocks": clk,
    }
    if world == 1 and args.forms_nt >= 0:
        try:
            nt_cmp = p["nt"] if args.forms_nt == 0 else min(args.forms_nt, p["nt"])
            out["forms"] = compare_forms(p, v2, v2m_keep, rec, dev, nt_cmp)
        except Exception as exc:  # report, do not fail the headline measurement
            out["forms"] = {"failed": f"{exc}"[:300]}
    if world == 1 and not args.no_cpu_baseline:
        try:
            with tempfile.TemporaryDirectory() as wd:
                nts = args.ref_nt
                sec, upd_s, thr, _ = run_reference_program(ref_cpu_bin(), p, v, rec.cpu().numpy(), nts, wd)
            out["cpu_baseline"] = {"value": round(upd_s / sec / 1e9, 4), "unit": "Gpt/s", "cores": thr,
                                   "kind": "reference",
                                   "sample": f"reference RTM3D.bin RBC migration of the same shot, nt={nts} "
                                             f"({3 * nts - 2} sweeps of {n_points(p)} points), its own "
                                             f"migration timer"}
        except Exception as exc:  # report, do not fail the GPU measurement
            out["cpu_baseline"] = {"value": None, "unit": "Gpt/s", "cores": os.cpu_count(), "kind": "reference",
                                   "sample": f"failed: {exc}"[:300]}
    if world == 1 and not args.no_reference_gpu:
        try:
            out["reference_gpu"] = reference_gpu_bar(args, p, v, rec, value)
        except Exception as exc:  # report, do not fail the GPU measurement
            out["reference_gpu"] = {"failed": f"{exc}"[:300]}
    if world == 1 and args.c3:
        try:
            out["precision_c3"] = run_precision(args, forms=C3_FORMS)
        except Exception as exc:  # report, do not fail the headline measurement
            out["precision_c3"] = {"failed": f"{exc}"[:300]}
    return out


# ------------------------------------------------------------------------------------------ batch
def survey_model(nx: int, ny: int, nz: int, dz: float, seed: int = 1234) -> np.ndarray:
    """Seeded survey velocity: v(z) = 1500 + 0.6 z_m clipped at 4500 and a 4500 m/s salt ellipsoid
    (semi-axes nx/8, ny/10, nz/8 cells) centred at 60% depth."""
    z = np.arange(nz, dtype=np.float32) * dz
    v = np.broadcast_to(np.minimum(1500.0 + 0.6 * z, 4500.0), (nx, ny, nz)).astype(np.float32)
    cx, cy, cz = np.arange(nx) - nx / 2, np.arange(ny) - ny / 2, np.arange(nz) - 0.6 * nz
    salt = ((cx / (nx / 8))[:, None, None] ** 2 + (cy / (ny / 10))[None, :, None] ** 2 +
            (cz / (nz / 8))[None, None, :] ** 2) <= 1.0
    v[salt] = 4500.0
    rng = np.random.default_rng(seed)
    v *= (1.0 + 0.01 * rng.standard_normal(v.shape)).astype(np.float32)
    return np.clip(v, 1500.0, 4500.0).astype(np.float32)


def run_batch(args) -> dict:
    """Shots on uneven aperture sub-volumes of a survey, batched (rtmb_migrate_batch: the shots of a
    launch group advance together, one launch per step for the group, graph-captured time loop, the
    group size picked by rtmb_autotune_batch) against the single-shot driver one by one.

    --batch-config c4 (the batched configuration): a 1024 x 1024 x 512 survey at 12.5 m, 64 shots on
    an 8 x 8 surface grid, apertures +-256 cells around the source clipped at the survey's edges
    (320 to 512 cells wide), 40-cell RBC border, 10 Hz Ricker, 2500 steps, 16-bit storage; the
    one-by-one comparison runs the 8 shots of the grid's diagonal (one per aperture width).
    --batch-config small: a 512 x 512 x 256 survey, 12 shots on a 4 x 3 grid, apertures +-128, nt 500."""
    import torch
    import rtmb
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    c4 = args.batch_config == "c4"
    if c4:
        snx, sny, snz, half, nt, gx, gy = 1024, 1024, 512, 256, 2500, 8, 8
        form = args.form if args.form != "fp32_fma" else "fp16"
    else:
        snx, sny, snz, half, nt, gx, gy = 2 * args.batch_size, 2 * args.batch_size, args.batch_size, \
            args.batch_size // 2, args.batch_nt, 4, 3
        form = args.form
    blen, dx = 40, 12.5
    t_prep = time.time()
    v = survey_model(snx, sny, snz, dx)
    grid = [(int(snx * (i + 0.5) / gx), int(sny * (j + 0.5) / gy)) for i in range(gx) for j in range(gy)]
    flags = form_flags(rtmb, form) | rtmb.FLAG_USE_GRAPH
    keep, shots = [], []
    for k, (sx_, sy_) in enumerate(grid):
        x0, x1 = max(0, sx_ - half), min(snx, sx_ + half)
        y0, y1 = max(0, sy_ - half), min(sny, sy_ + half)
        nx, ny = x1 - x0, y1 - y0
        ve = rtmb.prepare_velocity(np.ascontiguousarray(v[x0:x1, y0:y1, :]), blen, "rbc", seed=100 + k)
        v2 = torch.from_numpy(rtmb.v2dt2(ve, 0.001)).to(dev)
        del ve
        rcx, rcy = nx // 2, ny // 2
        gen = torch.Generator(device=dev).manual_seed(7 + k)
        rec = torch.randn((1, rcx, rcy, nt), generator=gen, device=dev) * 1e-3
        keep += [v2, rec]
        shots.append(rtmb.Shot(nx=nx, ny=ny, nz=snz, ox=x0, oy=y0, oz=0, sx=sx_ - x0, sy=sy_ - y0, sz=0,
                               receiver_start_x=0, receiver_start_y=0, receiver_depth_z=0, receiver_distance_x=2,
                               receiver_distance_y=2, receiver_count_x=rcx, receiver_count_y=rcy,
                               v2dt2=v2.data_ptr(), rec=rec.data_ptr()))
    del v
    t_prep = time.time() - t_prep
    base = dict(nx=snx, ny=sny, nz=snz, blen=blen, nt=nt, ntstep=nt, stencil_order=8, dx=dx, dy=dx, dz=dx, dt=0.001,
                fpeak=10.0, taper_factor=0.2, receiver_start_x=0, receiver_start_y=0, receiver_depth_z=0,
                receiver_distance_x=2, receiver_distance_y=2, receiver_count_x=1, receiver_count_y=1,
                boundary_condition="rbc")
    ctx = rtmb.Context(rtmb.Params.from_input(base, flags=flags, device=0))
    group, rate = ctx.autotune_batch(shots)
    stack = torch.zeros((snx, sny, snz), dtype=torch.float64, device=dev)
    if not c4:
        ctx.migrate_batch(shots, stack)  # warm-up: graph capture and instantiation
        ctx.sync()
    l0 = ctx.launches
    ms_batch = time_ctx(ctx, lambda: ctx.migrate_batch(shots, stack))
    launches_batch = ctx.launches - l0
    pts_all = sum((s.nx + 2 * blen) * (s.ny + 2 * blen) * (snz + 2 * blen) for s in shots)
    # one by one: the single-shot driver per aperture, images stacked in FP64 (the grid's diagonal
    # for c4: one shot per aperture width)
    subset = [shots[i * gy + i] for i in range(min(gx, gy))] if c4 else shots
    ms_single = 0.0
    pts = 0
    for s in subset:
        q = dict(base, nx=s.nx, ny=s.ny, receiver_count_x=s.receiver_count_x, receiver_count_y=s.receiver_count_y)
        c = rtmb.Context(rtmb.Params.from_input(q, flags=form_flags(rtmb, form), device=0))
        c.load_v2dt2(s.v2dt2, from_host=False)
        acc = torch.zeros(c.padded_shape, dtype=torch.float64, device=dev)
        if not c4:
            c.migrate_shot_acc64(s.sx, s.sy, s.sz, s.rec, acc)
            c.sync()
        ms_single += time_ctx(c, lambda: c.migrate_shot_acc64(s.sx, s.sy, s.sz, s.rec, acc))
        pts += int(np.prod(c.padded_shape))
        c.close()
        del acc
    upd_single = pts * (3 * nt - 2)
    upd_batch = pts_all * (3 * nt - 2)
    sizes = sorted({(s.nx, s.ny) for s in shots})
    gpt_b, gpt_1 = upd_batch / ms_batch / 1e6, upd_single / ms_single / 1e6
    return {"metric": "s per migrated shot, batched aperture shots", "workload": f"batch_{args.batch_config}",
            "config": {"survey": [snx, sny, snz], "dx_m": dx, "shots": len(shots), "apertures_xy": sizes,
                       "blen": blen, "nt": nt, "form": form, "fpeak_hz": 10.0, "graph": True,
                       "shots_per_launch": group, "autotune_rate_gpt_s": round(rate, 2),
                       "host_preparation_s": round(t_prep, 1)},
            "batched": {"s_per_shot": round(ms_batch / 1e3 / len(shots), 4), "gpt_s": round(gpt_b, 2),
                        "launches": launches_batch, "s_total": round(ms_batch / 1e3, 2)},
            "one_by_one": {"shots": len(subset), "s_per_shot": round(ms_single / 1e3 / len(subset), 4),
                           "gpt_s": round(gpt_1, 2)},
            "speedup_per_point_update": round(gpt_b / gpt_1, 3)}


# ------------------------------------------------------------------------------------------ model
def run_model(args) -> dict:
    """The CPU-runnable modeling configuration in full: a 128^3 three-layer model (1500, 2500 and
    3500 m/s from depths 0, 40 and 80 cells), a 32-cell border tapered on every face but the free
    surface's velocity, 1000 steps of 1 ms, a 15 Hz Ricker at (64, 64, 4), 64 x 64 receivers every
    2 cells at depth 4.  GPU: s per modeled shot in the exact and FMA forms.  With the reference
    program built: its own modeling of the same shot truncated to a bounded number of steps (the
    cpu_baseline), and the GPU's exact-form record of that run compared with the reference's .seism
    file bit for bit."""
    import tempfile
    import torch
    import rtmb
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    n, blen, nt = 128, 32, args.model_nt
    v = np.full((n, n, n), 3500.0, np.float32)
    v[:, :, :40] = 1500.0
    v[:, :, 40:80] = 2500.0
    p = dict(nx=n, ny=n, nz=n, blen=blen, nt=nt, ntstep=nt, stencil_order=8, dx=10.0, dy=10.0, dz=10.0, dt=0.001,
             fpeak=15.0, taper_factor=0.2, receiver_start_x=0, receiver_start_y=0, receiver_depth_z=4,
             receiver_distance_x=2, receiver_distance_y=2, receiver_count_x=64, receiver_count_y=64,
             boundary_condition="hbc", sx=64, sy=64, sz=4)
    v2 = rtmb.v2dt2(rtmb.prepare_velocity(v, blen, "abc"), p["dt"])
    out = {"metric": "s per modeled shot (128^3, 32-cell border, nt=1000)", "workload": "model",
           "config": {"grid": [n + 2 * blen] * 3, "model": "3-layer 1500/2500/3500 m/s", "nt": nt, "fpeak_hz": 15.0,
                      "receivers": [64, 64]}, "forms": {}}
    npad = (n + 2 * blen) ** 3

    def shot(flags, ntr):
        q = dict(p, nt=ntr, ntstep=ntr)
        ctx = rtmb.Context(rtmb.Params.from_input(q, flags=flags | rtmb.FLAG_USE_GRAPH, device=0))
        ctx.load_v2dt2(v2, from_host=True)
        rec = torch.zeros((1, 64, 64, ntr), device=dev)
        ctx.model_shot(p["sx"], p["sy"], p["sz"], rec)  # warm-up: graph capture
        ctx.sync()
        ms = time_ctx(ctx, lambda: ctx.model_shot(p["sx"], p["sy"], p["sz"], rec))
        ctx.close()
        return ms, rec.cpu().numpy()

    for form, flags in (("fp32_exact", 0), ("fp32_fma", rtmb.FLAG_FAST_FMA)):
        ms, _ = shot(flags, nt)
        out["forms"][form] = {"s_per_shot": round(ms / 1e3, 4), "gpt_s": round(npad * nt / ms / 1e6, 2)}
    out["value"] = out["forms"]["fp32_fma"]["gpt_s"]
    out["unit"] = "Gpt/s"
    if not args.no_cpu_baseline and os.path.exists(ref_cpu_bin()):
        nts = args.model_ref_nt
        with tempfile.TemporaryDirectory() as wd:
            t, upd_r, threads, ref_rec = run_reference_program(ref_cpu_bin(), dict(p, ntstep=nts), v, None, nts, wd,
                                                               migration=False)
        out["cpu_baseline"] = {"value": round(upd_r / t / 1e9, 4), "unit": "Gpt/s", "cores": threads,
                               "kind": "reference",
                               "sample": f"RTM3D.bin modeling of the same shot, nt={nts}, its own modeling timer"}
        _, got = shot(0, nts)
        out["record_vs_reference"] = {"nt": nts, "bitexact": bool(np.array_equal(
            got.reshape(-1).view(np.uint32), ref_rec.view(np.uint32)))}
    return out


# ------------------------------------------------------------------------------------------ fmig
def run_fmig(args) -> dict:
    """Frequency-domain RTM of one shot (rtmb_migrate_shot_fmig): the salt model, HBC border, both
    wavefields stepped forward in time and the running DFT of nw frequencies imaged every step.
    Reported: s per shot, wavefield point-updates/s, and the roofline of the DFT/image kernel (HBM:
    16 B per interior point for ps, pr and the image, plus 32 B per frequency for the four
    frequency grids).  cpu_baseline: the oracle restatement of the same migration (OpenMP) on the
    same grid and the same number of frequencies, for a few time steps."""
    import torch
    import rtmb
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    n, nt, blen, dt = args.fmig_size, args.fmig_nt, 32, 0.001
    fmin, fmax = args.fmig_band
    p = dict(workload(n, nt), blen=blen, boundary_condition="hbc", receiver_depth_z=2)
    nw = rtmb.fmig_nw(dt, nt, fmin, fmax)
    flags = form_flags(rtmb, args.form if args.form in ("fp32_exact", "fp32_fma") else "fp32_fma")
    ctx = rtmb.Context(rtmb.Params.from_input(p, flags=flags | rtmb.FLAG_USE_GRAPH, device=0))
    ve = rtmb.prepare_velocity(salt_model(n), blen, "hbc", seed=5)
    ctx.load_v2dt2(rtmb.v2dt2(ve, dt), from_host=True)
    rng = np.random.default_rng(3)
    rec = torch.from_numpy((rng.standard_normal((1, n // 2, n // 2, nt)) * 1e-3).astype(np.float32)).to(dev)
    img = torch.zeros(ctx.padded_shape, dtype=torch.float32, device=dev)
    shot = (p["sx"], p["sy"], p["sz"])
    for _ in range(max(1, args.warmup - 2)):
        ctx.migrate_shot_fmig(*shot, rec, img, fmin, fmax, args.fmig_nwstep)
    ctx.sync()
    ms = time_ctx(ctx, lambda: ctx.migrate_shot_fmig(*shot, rec, img, fmin, fmax, args.fmig_nwstep))
    # per-kernel split (a separate run: events around every launch)
    pctx = rtmb.Context(rtmb.Params.from_input(p, flags=flags, device=0))
    pctx.load_v2dt2(rtmb.v2dt2(ve, dt), from_host=True)
    pctx.profile(True)
    pctx.migrate_shot_fmig(*shot, rec, img, fmin, fmax, args.fmig_nwstep)
    prof = pctx.profile_read()
    pctx.close()
    nws = nw if args.fmig_nwstep in (0,) or args.fmig_nwstep > nw else args.fmig_nwstep
    groups = -(-nw // nws)
    npad = int(np.prod(ctx.padded_shape))
    ni = n * n * n
    upd = 2 * nt * groups * npad
    fq = prof["fmig_freq"]
    f_ms = fq["ms"] / max(fq["launches"], 1)
    bytes_freq = ni * (16 + 32 * nws)  # the last group may be smaller; nw = nws x groups here
    peak, peak_kind = measured_hbm_gbs()
    achieved = bytes_freq / (f_ms * 1e-3) / 1e9
    out = {"metric": "s per migrated shot, frequency-domain RTM", "workload": "fmig",
           "config": {"grid": list(ctx.padded_shape), "model": f"salt {n}^3", "blen": blen, "nt": nt,
                      "band_hz": [fmin, fmax], "nw": nw, "nwstep": nws, "form": "fp32_exact" if flags == 0 else "fp32_fma"},
           "s_per_shot": round(ms / 1e3, 4), "gpt_s": round(upd / ms / 1e6, 2),
           "kernels": {k: {"ms_total": round(v["ms"], 2), "launches": v["launches"]} for k, v in prof.items()
                       if v["launches"]},
           "roofline": {"bound": "hbm", "kernel": "fmig_freq_kernel", "achieved": round(achieved, 1),
                        "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                        "bytes_per_launch": bytes_freq, "launch_ms": round(f_ms, 4)}}
    if not args.no_cpu_baseline:
        from oracle import Oracle
        O = Oracle()
        nts = 6
        p_or = {k: p[k] for k in ("nx", "ny", "nz", "blen", "nt", "ntstep", "dx", "dy", "dz", "dt", "fpeak",
                                  "taper_factor", "sx", "sy", "sz")}
        p_or.update(order=8, nt=nts, ntstep=nts, rsx=0, rsy=0, rdz=2, rdx=2, rdy=2, rcx=n // 2, rcy=n // 2)
        fmax_s = fmin + (nw + 0.5) / (nts * dt)  # the same number of frequencies over nts steps
        v2 = rtmb.v2dt2(ve, dt)
        rs = rec[..., :nts].cpu().numpy()
        t0 = time.time()
        O.migrate_fmig(p_or, v2, rs, fmin, fmax_s, 0)
        cpu_s = time.time() - t0
        cpu_upd = 2 * nts * npad
        out["cpu_baseline"] = {"value": round(cpu_upd / cpu_s / 1e9, 4), "unit": "Gpt/s", "cores": os.cpu_count(),
                               "kind": "port", "sample": f"oracle fmig on the same grid, nw={O.L.orc_fmig_nw(nts, dt, fmin, fmax_s)}, "
                                                        f"{nts} time steps"}
    return out


# ------------------------------------------------------------------------------------------ closure
def run_closure(args) -> dict:
    """The learned 8-cell boundary closure against the tapered borders of 8 and 32 cells: reflected
    energy = shot-record rel-L2 against the same shot on a domain padded so widely that no boundary
    reflection returns within nt; wall time of a modeling shot on each grid."""
    import torch
    import rtmb
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    n, nt, wide = args.closure_size, args.closure_nt, args.closure_wide
    v = salt_model(n)

    def prm(blen, bc="hbc"):
        return dict(nx=n, ny=n, nz=n, blen=blen, nt=nt, ntstep=nt, stencil_order=8, dx=10.0, dy=10.0, dz=10.0,
                    dt=0.001, fpeak=15.0, taper_factor=0.2, receiver_start_x=0, receiver_start_y=0,
                    receiver_depth_z=2, receiver_distance_x=2, receiver_distance_y=2, receiver_count_x=n // 2,
                    receiver_count_y=n // 2, boundary_condition=bc)

    def model(blen, shot, closure=None, min_scale=0.0, damp=0.0):
        par = rtmb.Params.from_input(prm(blen), flags=rtmb.FLAG_FAST_FMA, device=0)
        if closure is not None:
            par.boundary = rtmb.BC_LEARNED
        c = rtmb.Context(par)
        c.load_v2dt2(rtmb.v2dt2(rtmb.prepare_velocity(v, blen, "abc"), 0.001), from_host=True)
        if closure is not None:
            c.closure_set(closure, min_scale, damp)
        rec = torch.zeros((1, n // 2, n // 2, nt), device=dev)
        c.model_shot(*shot, rec)  # warm-up
        c.sync()
        ms = time_ctx(c, lambda: c.model_shot(*shot, rec))
        c.close()
        return rec, ms

    rng = np.random.default_rng(2024)
    pos = lambda: (int(rng.integers(n // 6, n - n // 6)), int(rng.integers(n // 6, n - n // 6)), int(rng.integers(1, n // 8)))
    train = [pos() for _ in range(args.closure_train_shots)]
    held = [pos() for _ in range(args.closure_eval_shots)]
    val = pos()  # model selection among the trained candidates (not an evaluation shot)
    t0 = time.time()
    pilot, _ = model(wide, train[0])
    min_scale = 1e-4 * float(pilot.abs().max())
    per_step, ts0, tstride = args.closure_rows_per_step, nt // 6, 2
    cap = len(train) * per_step * ((nt - ts0) // tstride + 1)
    X = torch.zeros((cap, rtmb.CLOSURE_NIN), dtype=torch.bfloat16, device=dev)
    R = torch.zeros(cap, dtype=torch.float32, device=dev)
    rows = 0
    for k, sh in enumerate(train):
        c = rtmb.Context(rtmb.Params.from_input(prm(wide), flags=rtmb.FLAG_FAST_FMA, device=0))
        c.load_v2dt2(rtmb.v2dt2(rtmb.prepare_velocity(v, wide, "abc"), 0.001), from_host=True)
        rows += c.closure_collect(*sh, ts0, tstride, per_step, 1000 + k, min_scale, X[rows:], R[rows:])
        c.close()
    t_collect = time.time() - t0
    t1 = time.time()
    vref, _ = model(wide, val)
    cands = []
    for seed in range(23, 23 + args.closure_candidates):
        p_ = torch.from_numpy(rtmb.closure_init(17)).to(dev)
        l_ = rtmb.closure_train(p_, X, R, rows, args.closure_steps, 8192, 2e-3, seed, noise=0.05)
        r_, _ = model(8, val, p_, min_scale, 0.3)
        cands.append((float(torch.linalg.vector_norm((r_ - vref).double()) / torch.linalg.vector_norm(vref.double())),
                      seed, p_, l_))
    val_err, seed, params, losses = min(cands, key=lambda c: c[0])
    torch.cuda.synchronize()
    t_train = time.time() - t1
    res = {"learned_8": [], "taper_8": [], "taper_32": []}
    ms = {k: [] for k in res}
    for sh in held:
        ref, _ = model(wide, sh)
        for key, blen, cl in (("learned_8", 8, params), ("taper_8", 8, None), ("taper_32", 32, None)):
            r, t = model(blen, sh, cl, min_scale, 0.3) if cl is not None else model(blen, sh)
            res[key].append(float(torch.linalg.vector_norm((r - ref).double()) / torch.linalg.vector_norm(ref.double())))
            ms[key].append(t)
    mean = {k: float(np.mean(x)) for k, x in res.items()}
    # the in-driver judge on the validation shot (rtmb_closure_judge) and the judged modeling call
    # on each held-out shot (rtmb_model_shot_judged): the boundary that ran
    def ctx_of(blen, closure=None):
        par = rtmb.Params.from_input(prm(blen), flags=rtmb.FLAG_FAST_FMA, device=0)
        if closure is not None:
            par.boundary = rtmb.BC_LEARNED
        c = rtmb.Context(par)
        c.load_v2dt2(rtmb.v2dt2(rtmb.prepare_velocity(v, blen, "abc"), 0.001), from_host=True)
        if closure is not None:
            c.closure_set(closure, min_scale, 0.3)
        return c
    lc, hc, wc = ctx_of(8, params), ctx_of(32), ctx_of(wide)
    j_l, j_h, passed = lc.closure_judge(hc, wc, *val)
    ran = []
    for sh in held:
        r = torch.zeros((1, n // 2, n // 2, nt), device=dev)
        ran.append("learned_8" if lc.model_shot_judged(hc, *sh, r) == rtmb.BC_LEARNED else "taper_32")
    lc.sync()
    for c in (lc, hc, wc):
        c.close()
    return {"metric": "reflected energy (record rel-L2 vs wide-padded run) and modeling time", "workload": "closure",
            "judge": {"shot": list(val), "reflection_learned_8": round(j_l, 4), "reflection_taper_32": round(j_h, 4),
                      "passed": passed, "ran_on_held_out_shots": ran},
            "config": {"model": [n, n, n], "nt": nt, "wide_border": wide, "fpeak_hz": 15.0,
                       "train_shots": len(train), "eval_shots": len(held), "rows": rows,
                       "train_steps": args.closure_steps, "batch": 8192, "candidates": args.closure_candidates,
                       "selected_seed": seed, "validation_reflection": round(val_err, 4)},
            "reflected_energy": {k: round(x, 4) for k, x in mean.items()},
            "modeling_ms": {k: round(float(np.mean(x)), 2) for k, x in ms.items()},
            "grid": {"learned_8": (n + 16) ** 3, "taper_8": (n + 16) ** 3, "taper_32": (n + 64) ** 3},
            "falls_back_to_hbc": rtmb.closure_falls_back(mean["learned_8"], mean["taper_32"]),
            "loss": {"first": float(losses[:10].mean()), "last": float(losses[-50:].mean())},
            "seconds": {"collect": round(t_collect, 1), "train": round(t_train, 1)}}


def run_reference_arm(args, rank: int) -> dict | None:
    """The reference's own CPU program (oracle/_ref/RTM3D.bin, built from its sources) on the same
    workload: an RBC migration of the same shot geometry with nt cut to --ref-nt steps per bench
    step, every host thread, timed by the program's own migration timer.  Nothing of this
    repository's library is loaded: the program builds its own random border, and the record is a
    seeded random array of the record's shape (the CPU program's cost does not depend on its values)."""
    if rank != 0:
        return None
    p = workload(args.size, args.nt)
    binary = ref_cpu_bin()
    if not os.path.exists(binary):
        return {"impl": "reference", "unavailable": "oracle/_ref/RTM3D.bin was not built from the reference sources"}
    v = salt_model(p["nx"], p["ny"], p["nz"])
    nts = args.ref_nt
    rng = np.random.default_rng(5)
    rec = (rng.standard_normal((1, p["receiver_count_x"], p["receiver_count_y"], nts)) * 1e-3).astype(np.float32)
    secs, upds, thr = [], 0, 1
    with tempfile.TemporaryDirectory() as wd:
        for _ in range(args.warmup):
            run_reference_program(binary, p, v, rec, nts, wd)
        for _ in range(args.steps):
            s_, u_, thr, _ = run_reference_program(binary, p, v, rec, nts, wd)
            secs.append(s_)
            upds += u_
    value = upds / sum(secs) / 1e9
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": round(value, 4), "unit": "Gpt/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * sum(secs) / len(secs), 1), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded salt model, seeded random record)",
        "config": workload_config(args, p, 1),
        "sample": {"nt": nts, "sweeps": 3 * nts - 2, "note": "each step is one run of the reference program on the "
                                                              "workload with nt cut to the sample"},
        "cpu_baseline": {"value": round(value, 4), "unit": "Gpt/s", "cores": thr, "kind": "reference",
                         "sample": f"RTM3D.bin RBC migration, nt={nts} ({3 * nts - 2} sweeps of {n_points(p)} "
                                   f"points) per step, its own migration timer"},
        "e2e": {"value": round(value, 4), "unit": "Gpt/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("b200", "reference"), default="b200")
    ap.add_argument("--size", type=int, default=512, help="model edge in cells (workload: 512)")
    ap.add_argument("--nt", type=int, default=3000)
    ap.add_argument("--form", choices=ALL_FORMS, default="fp32_fma", help="arithmetic/storage form of the timed shots")
    ap.add_argument("--exact", action="store_true", help="same as --form fp32_exact")
    ap.add_argument("--workload", choices=("rtm", "batch", "closure", "fmig", "model", "precision"), default="rtm",
                    help="rtm: the single-shot RTM line (default); batch: batched aperture shots against "
                         "one-by-one; closure: the learned boundary closure against the tapered borders; "
                         "fmig: frequency-domain RTM of one shot; model: the 128^3 modeling configuration; "
                         "precision: the 896 x 896 x 512 storage-form comparison against the FP64 oracle")
    ap.add_argument("--model-nt", type=int, default=1000)
    ap.add_argument("--model-ref-nt", type=int, default=200, help="steps of the reference program's timed sample")
    ap.add_argument("--fmig-size", type=int, default=192)
    ap.add_argument("--fmig-nt", type=int, default=400)
    ap.add_argument("--fmig-band", type=float, nargs=2, default=(4.0, 20.0))
    ap.add_argument("--fmig-nwstep", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-config", choices=("small", "c4"), default="small",
                    help="batch workload: c4 = 64 shots on a 1024 x 1024 x 512 survey, nt 2500; small = 12 shots")
    ap.add_argument("--batch-size", type=int, default=256, help="batch workload (small): survey 2s x 2s x s cells")
    ap.add_argument("--batch-nt", type=int, default=500)
    ap.add_argument("--closure-config", choices=("small", "c5"), default="small",
                    help="closure workload: c5 = 384^3 at 10 m, nt 2000, training on a 200-cell-padded run, 64 "
                         "training and 16 held-out shots; small = the sizes given by the --closure-* options")
    ap.add_argument("--closure-size", type=int, default=96)
    ap.add_argument("--closure-nt", type=int, default=600)
    ap.add_argument("--closure-wide", type=int, default=120)
    ap.add_argument("--closure-train-shots", type=int, default=8)
    ap.add_argument("--closure-eval-shots", type=int, default=4)
    ap.add_argument("--closure-steps", type=int, default=8000)
    ap.add_argument("--closure-rows-per-step", type=int, default=4096,
                    help="training pairs sampled per collected time step of each training shot")
    ap.add_argument("--closure-candidates", type=int, default=3,
                    help="networks trained with different seeds; the one reflecting least on a validation shot is kept")
    ap.add_argument("--forms-nt", type=int, default=0,
                    help="nt of the storage-form comparison against the FP64 oracle (0: the full nt; -1: skip)")
    ap.add_argument("--ref-nt", type=int, default=8,
                    help="steps of the reference CPU program's RBC migration sample (reference arm, cpu_baseline)")
    ap.add_argument("--ref-gpu-nt", type=int, default=100,
                    help="steps of the reference GPU program's RBC migration sample")
    ap.add_argument("--no-reference-gpu", action="store_true", help="skip the reference GPU program bar")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default launch shape instead of measuring it (rtmb_autotune_full) per context")
    ap.add_argument("--c3", dest="c3", action="store_true", default=True,
                    help="add the precision configuration (896 x 896 x 512) to the default line (default)")
    ap.add_argument("--no-c3", dest="c3", action="store_false")
    ap.add_argument("--c3-grid", type=int, nargs=3, default=(896, 896, 512))
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.closure_config == "c5":
        args.closure_size, args.closure_nt, args.closure_wide = 384, 2000, 200
        args.closure_train_shots, args.closure_eval_shots, args.closure_rows_per_step = 64, 16, 2048
    if args.exact:
        args.form = "fp32_exact"

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    sys.path.insert(0, ROOT)

    if args.impl == "reference":
        out = run_reference_arm(args, rank)
    elif args.workload != "rtm":
        runner = {"batch": run_batch, "closure": run_closure, "fmig": run_fmig, "model": run_model,
                  "precision": run_precision}[args.workload]
        out = runner(args) if rank == 0 else None
    else:
        if world > 1:
            import datetime
            import torch
            import torch.distributed as dist
            torch.cuda.set_device(local_rank)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        try:
            out = run_b200(args, rank, world, local_rank)
        finally:
            if world > 1:
                import torch.distributed as dist
                dist.destroy_process_group()
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
