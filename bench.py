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
def workload(n: int, nt: int) -> dict:
    """input.json parameters of the benchmark shot (configs scale with n, reference value 512)."""
    return dict(nx=n, ny=n, nz=n, blen=40, nt=nt, ntstep=nt, stencil_order=8, dx=10.0, dy=10.0, dz=10.0,
                dt=0.001, fpeak=12.0, taper_factor=0.2, receiver_start_x=0, receiver_start_y=0,
                receiver_depth_z=0, receiver_distance_x=2, receiver_distance_y=2,
                receiver_count_x=n // 2, receiver_count_y=n // 2, boundary_condition="rbc",
                sx=n // 2, sy=n // 2, sz=0)


def salt_model(n: int, seed: int = 1234) -> np.ndarray:
    """Seeded synthetic velocity (x slowest, z fastest), float32 m/s."""
    from scipy import ndimage
    f = n / 512.0
    z = np.arange(n, dtype=np.float32) * 10.0
    v = np.broadcast_to(np.minimum(1500.0 + 0.6 * z, 4500.0), (n, n, n)).astype(np.float32)
    c = np.arange(n, dtype=np.float32)
    ex = ((c - 256 * f) / (120 * f)) ** 2
    ey = ((c - 256 * f) / (100 * f)) ** 2
    ez = ((c - 300 * f) / (60 * f)) ** 2
    salt = (ex[:, None, None] + ey[None, :, None] + ez[None, None, :]) <= 1.0
    v[salt] = 4500.0
    # +-3% perturbation: white noise on a grid 8x coarser, Gaussian-smoothed (sigma 1 coarse cell
    # = 8 cells) and interpolated trilinearly to the model grid
    rng = np.random.default_rng(seed)
    nc = max(4, n // 8)
    pert = ndimage.gaussian_filter(rng.standard_normal((nc, nc, nc)).astype(np.float32), 1.0, mode="wrap")
    pert = ndimage.zoom(pert, n / nc, order=1, mode="nearest")[:n, :n, :n]
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
def run_reference_sample(p: dict, v: np.ndarray, vpe: np.ndarray, rec: np.ndarray, nts: int, workdir: str):
    """Run the reference's own CPU program (RTM3D.bin) for an RBC migration of the same shot with
    nt truncated to nts.  Returns (seconds of its migration timer, point updates, threads)."""
    from oracle import REF_BIN
    if not os.path.exists(REF_BIN):
        raise FileNotFoundError("oracle/_ref/RTM3D.bin is not built")
    for sub in ("out", "tmp", "dat"):
        os.makedirs(os.path.join(workdir, sub), exist_ok=True)
    vp = os.path.join(workdir, "vel.bin")
    vpe_path = os.path.join(workdir, "vpe.bin")
    if not os.path.exists(vp):
        v.tofile(vp)
        vpe.tofile(vpe_path)
    # the record chunk [rcx][rcy][nts] under the reference's file name (RTMBase.hpp:131-138)
    sx, sy, sz = p["sx"], p["sy"], p["sz"]
    seism = os.path.join(workdir, "dat", f"RTMSEISMOGRAM_S{sx}x{sy}x{sz}_NXNY_{p['receiver_count_x']}x"
                                         f"{p['receiver_count_y']}_NTSTART0_NTSTEP{nts}.seism")
    np.ascontiguousarray(rec[..., :nts]).tofile(seism)
    threads = os.cpu_count() or 1
    d = dict(mname="bench", vpfile=vp, vpefile=vpe_path, save_vpe_file=False, outdir=os.path.join(workdir, "out"),
             tmpdir=os.path.join(workdir, "tmp"), datdir=os.path.join(workdir, "dat"), nx=p["nx"], ny=p["ny"],
             nz=p["nz"], blen=p["blen"], width_m=0, height_m=0, depth_m=0, nt=nts, dz=p["dz"], dy=p["dy"],
             dx=p["dx"], dt=p["dt"], fpeak=p["fpeak"], fmax=30.0, taper_factor=p["taper_factor"],
             stencil_order=p["stencil_order"], modeling=False, migration=True, rtm_type="rtm",
             boundary_condition="rbc", source_total=1, source_start_x=sx, source_start_y=sy, source_depth_z=sz,
             source_distance_x=1, source_distance_y=1, source_count_x=1, source_count_y=1,
             receiver_total=p["receiver_count_x"] * p["receiver_count_y"],
             receiver_start_x=p["receiver_start_x"], receiver_start_y=p["receiver_start_y"],
             receiver_depth_z=p["receiver_depth_z"], receiver_distance_x=p["receiver_distance_x"],
             receiver_distance_y=p["receiver_distance_y"], receiver_count_x=p["receiver_count_x"],
             receiver_count_y=p["receiver_count_y"], ntstep=nts, nthreads=threads, load_vpe_from_file=True,
             save_snapshots=False, distributed_grid=False, snapshot_step=10, fmig=False, fmig_max_freq=30.0,
             fmig_min_freq=1.0, fmig_nwstep=1, fmig_distributed_imaging=False, fpga_xclbin="",
             fpga_fwd_kernel="", fpga_bwd_kernel="", verbose=True)
    jp = os.path.join(workdir, "mig.json")
    with open(jp, "w") as f:
        json.dump(d, f)
    r = subprocess.run([REF_BIN, jp], capture_output=True, text=True, cwd=workdir, timeout=900)
    if r.returncode != 0:
        raise RuntimeError(f"RTM3D.bin failed: {r.stdout[-500:]} {r.stderr[-500:]}")
    mig = None
    for line in r.stdout.splitlines():
        if '"migration_time"' in line:
            mig = float(line.split(":")[1].strip().rstrip(","))
    if not mig:
        raise RuntimeError("no migration_time in the reference report")
    pts = n_points(p)
    return mig, pts * (3 * nts - 2), threads


def reference_sample_steps(p: dict) -> int:
    return 8


# ------------------------------------------------------------------------------------------ arms
def build_inputs(p: dict, with_abc: bool):
    import rtmb
    v = salt_model(p["nx"])
    vpe = rtmb.prepare_velocity(v, p["blen"], "rbc", seed=1234)
    v2 = rtmb.v2dt2(vpe, p["dt"])
    v2m = rtmb.v2dt2(rtmb.prepare_velocity(v, p["blen"], "abc"), p["dt"]) if with_abc else None
    return v, vpe, v2, v2m


def run_b200(args, rank: int, world: int, local_rank: int) -> dict | None:
    import torch
    import rtmb
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    p = workload(args.size, args.nt)
    flags = 0 if args.exact else rtmb.FLAG_FAST_FMA
    params = rtmb.Params.from_input(p, flags=flags, device=local_rank)
    v, vpe, v2, v2m = build_inputs(p, with_abc=True)
    stream = torch.cuda.Stream(device=dev)
    sx, sy, sz = p["sx"], p["sy"], p["sz"]
    rec_shape = (1, p["receiver_count_x"], p["receiver_count_y"], p["nt"])

    # the shot record: this library's modeling pass on the ABC-bordered model
    mctx = rtmb.Context(rtmb.Params.from_input(dict(p, boundary_condition="hbc"), flags=flags, device=local_rank))
    mctx.set_stream(stream.cuda_stream)
    with torch.cuda.stream(stream):
        rec = torch.zeros(rec_shape, dtype=torch.float32, device=dev)
    mctx.load_v2dt2(v2m, from_host=True)
    mctx.model_shot(sx, sy, sz, rec)
    mctx.close()
    del v2m

    ctx = rtmb.Context(params)
    ctx.set_stream(stream.cuda_stream)
    ctx.load_v2dt2(v2, from_host=True)
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
            import torch.distributed as dist
            with torch.cuda.stream(stream):
                dist.all_reduce(stack)            # images summed across shot-parallel ranks
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
    cat = max(("forward", "backward_source", "backward_receiver"), key=lambda k: prof[k]["ms"])
    bpp = {"forward": 16, "backward_source": 16, "backward_receiver": 28}[cat]
    per_launch_ms = prof[cat]["ms"] / max(prof[cat]["launches"], 1)
    bytes_launch = bpp * n_points(p)
    achieved = bytes_launch / (per_launch_ms * 1e-3) / 1e9
    tpp = ncu_traffic_per_point(cat)
    if rank != 0:
        return None
    out = {
        "metric": "G point-updates/s per migrated RTM shot (512^3 RBC, nt=3000)",
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
        "dtype": "f32" + ("" if args.exact else "-fma"),
        "data": "synthetic (seeded salt model; record from this library's modeling pass)",
        "config": {"workload": f"rtm_rbc_{args.size}^3_nt{args.nt}", "grid": list(shape), "nt": p["nt"],
                   "stencil_order": 8, "boundary": "rbc", "shots_per_step_per_gpu": 1,
                   "form": "exact" if args.exact else "fma",
                   "l2": "inputs larger than L2 (%.0f MB per wavefield)" % (n_points(p) * 4 / 1e6),
                   "parallelism": f"shot-parallel x{world}"},
        "e2e": {"value": round(e2e_value, 3), "unit": "Gpt/s",
                "h2d_bytes_per_step": int(np.prod(rec_shape) * 4), "d2h_bytes_per_step": int(np.prod(shape) * 4)},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": f"tma_step_kernel ({cat})", "achieved": round(achieved, 1),
                     "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "traffic": (round(tpp * n_points(p)) if tpp else None),
                     "bytes_per_launch": bytes_launch, "launch_ms": round(per_launch_ms, 4)},
        "kernels": {k: {"ms_total": round(v_["ms"], 2), "launches": v_["launches"]} for k, v_ in prof.items()
                    if v_["launches"]},
        "clocks": clk,
    }
    if world == 1 and not args.no_cpu_baseline:
        try:
            with tempfile.TemporaryDirectory() as wd:
                nts = reference_sample_steps(p)
                sec, upd_s, thr = run_reference_sample(p, v, vpe, rec.cpu().numpy(), nts, wd)
            out["cpu_baseline"] = {"value": round(upd_s / sec / 1e9, 4), "unit": "Gpt/s", "cores": thr,
                                   "kind": "reference",
                                   "sample": f"reference RTM3D.bin RBC migration of the same shot, nt={nts} "
                                             f"({3 * nts - 2} sweeps of {n_points(p)} points), its own "
                                             f"migration timer"}
        except Exception as exc:  # report, do not fail the GPU measurement
            out["cpu_baseline"] = {"value": None, "unit": "Gpt/s", "cores": os.cpu_count(), "kind": "reference",
                                   "sample": f"failed: {exc}"[:300]}
    return out


def run_reference_arm(args, rank: int) -> dict | None:
    if rank != 0:
        return None
    from oracle import REF_BIN
    p = workload(args.size, args.nt)
    if not os.path.exists(REF_BIN):
        return {"impl": "reference", "unavailable": "oracle/_ref/RTM3D.bin was not built from the reference sources"}
    import rtmb
    v = salt_model(p["nx"])
    vpe = rtmb.prepare_velocity(v, p["blen"], "rbc", seed=1234)
    nts = reference_sample_steps(p)
    # a record of the right shape; the reference's cost does not depend on its values
    rng = np.random.default_rng(5)
    rec = (rng.standard_normal((1, p["receiver_count_x"], p["receiver_count_y"], nts)) * 1e-3).astype(np.float32)
    secs, upds, thr = [], 0, 1
    with tempfile.TemporaryDirectory() as wd:
        for _ in range(args.warmup):
            run_reference_sample(p, v, vpe, rec, nts, wd)
        for _ in range(args.steps):
            s_, u_, thr = run_reference_sample(p, v, vpe, rec, nts, wd)
            secs.append(s_)
            upds += u_
    value = upds / sum(secs) / 1e9
    return {
        "impl": "reference",
        "metric": "G point-updates/s per migrated RTM shot (512^3 RBC, nt=3000)",
        "value": round(value, 4), "unit": "Gpt/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * sum(secs) / len(secs), 1), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded salt model)",
        "config": {"workload": f"rtm_rbc_{args.size}^3_nt{args.nt}", "nt_sample": nts, "boundary": "rbc",
                   "stencil_order": 8},
        "cpu_baseline": {"value": round(value, 4), "unit": "Gpt/s", "cores": thr, "kind": "reference",
                         "sample": f"RTM3D.bin RBC migration, nt={nts} per step, its own migration timer"},
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
    ap.add_argument("--exact", action="store_true", help="bit-exact stencil form instead of the FMA form")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    sys.path.insert(0, ROOT)

    if args.impl == "reference":
        out = run_reference_arm(args, rank)
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
