"""Shared test cases: small seeded synthetic models and the reference's input.json for them."""
from __future__ import annotations

import os

import numpy as np

# small cases the CPU oracle finishes in seconds
CASES = {
    # used for the committed golden fixtures (reference run)
    "golden": dict(nx=24, ny=20, nz=28, blen=8, nt=120, ntstep=40, order=8, dx=10.0, dy=10.0, dz=10.0,
                   dt=0.001, fpeak=20.0, taper_factor=0.2, sx=12, sy=10, sz=2,
                   rsx=1, rsy=0, rdz=3, rdx=2, rdy=3, rcx=11, rcy=7, seed=3),
    # odd sizes: nze = 37 is not a multiple of 4 (unaligned rows), order 4
    "odd": dict(nx=21, ny=17, nz=25, blen=6, nt=90, ntstep=30, order=4, dx=12.0, dy=9.0, dz=10.0,
                dt=0.0012, fpeak=18.0, taper_factor=0.3, sx=10, sy=7, sz=3,
                rsx=0, rsy=1, rdz=2, rdx=3, rdy=2, rcx=7, rcy=8, seed=5),
    # larger, several CTAs per axis and several x chunks
    "mid": dict(nx=80, ny=72, nz=96, blen=16, nt=200, ntstep=100, order=8, dx=10.0, dy=10.0, dz=10.0,
                dt=0.001, fpeak=15.0, taper_factor=0.2, sx=40, sy=36, sz=4,
                rsx=0, rsy=0, rdz=4, rdx=2, rdy=2, rcx=40, rcy=36, seed=11),
}

# The CPU-runnable modeling configuration at full size: 128^3 at 10 m, three layers (1500, 2500 and
# 3500 m/s from depths 0, 40 and 80 cells), 32-cell border, 1000 steps of 1 ms, 15 Hz Ricker at
# (64, 64, 4), 64 x 64 receivers every 2 cells at depth 4, order 8; the record in four 250-step chunks.
C1 = dict(nx=128, ny=128, nz=128, blen=32, nt=1000, ntstep=250, order=8, dx=10.0, dy=10.0, dz=10.0,
          dt=0.001, fpeak=15.0, taper_factor=0.2, sx=64, sy=64, sz=4,
          rsx=0, rsy=0, rdz=4, rdx=2, rdy=2, rcx=64, rcy=64)


def c1_model() -> np.ndarray:
    """The three-layer velocity of C1 (x slowest, z fastest)."""
    v = np.full((C1["nx"], C1["ny"], C1["nz"]), 3500.0, np.float32)
    v[:, :, :40] = 1500.0
    v[:, :, 40:80] = 2500.0
    return v


def record_digest(rec) -> str:
    """SHA-256 of a record's float32 bytes in file layout (chunk, rcx, rcy, ntstep)."""
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(rec, np.float32).tobytes()).hexdigest()


def layered_model(case: dict) -> np.ndarray:
    """Three layers plus a little seeded roughness, x slowest, z fastest."""
    nx, ny, nz = case["nx"], case["ny"], case["nz"]
    v = np.full((nx, ny, nz), 1800.0, np.float32)
    v[:, :, nz // 3:] = 2600.0
    v[:, :, 2 * nz // 3:] = 3200.0
    rng = np.random.default_rng(case.get("seed", 0))
    v += (rng.random(v.shape) * 50.0).astype(np.float32)
    return v


def input_json(case: dict, vpfile: str, workdir: str) -> dict:
    """All keys the reference requires (RTMParam.hpp:115-186, plus 'verbose')."""
    for sub in ("out", "tmp", "dat"):
        os.makedirs(os.path.join(workdir, sub), exist_ok=True)
    return dict(
        mname="golden", vpfile=vpfile, vpefile=os.path.join(workdir, "vpe.bin"), save_vpe_file=False,
        outdir=os.path.join(workdir, "out"), tmpdir=os.path.join(workdir, "tmp"),
        datdir=os.path.join(workdir, "dat"),
        nx=case["nx"], ny=case["ny"], nz=case["nz"], blen=case["blen"],
        width_m=0, height_m=0, depth_m=0, nt=case["nt"],
        dz=float(case["dz"]), dy=float(case["dy"]), dx=float(case["dx"]), dt=float(case["dt"]),
        fpeak=float(case["fpeak"]), fmax=30.0, taper_factor=float(case["taper_factor"]),
        stencil_order=case["order"], modeling=True, migration=False, rtm_type="rtm",
        boundary_condition="hbc", source_total=1,
        source_start_x=case["sx"], source_start_y=case["sy"], source_depth_z=case["sz"],
        source_distance_x=1, source_distance_y=1, source_count_x=1, source_count_y=1,
        receiver_total=case["rcx"] * case["rcy"],
        receiver_start_x=case["rsx"], receiver_start_y=case["rsy"], receiver_depth_z=case["rdz"],
        receiver_distance_x=case["rdx"], receiver_distance_y=case["rdy"],
        receiver_count_x=case["rcx"], receiver_count_y=case["rcy"],
        ntstep=case["ntstep"], nthreads=max(1, os.cpu_count() or 1), load_vpe_from_file=False,
        save_snapshots=False, distributed_grid=False, snapshot_step=10,
        fmig=False, fmig_max_freq=30.0, fmig_min_freq=1.0, fmig_nwstep=1, fmig_distributed_imaging=False,
        fpga_xclbin="", fpga_fwd_kernel="", fpga_bwd_kernel="", verbose=False,
    )


def oracle_params(case: dict) -> dict:
    return {k: case[k] for k in ("nx", "ny", "nz", "blen", "order", "nt", "ntstep", "dx", "dy", "dz", "dt",
                                 "fpeak", "taper_factor", "sx", "sy", "sz", "rsx", "rsy", "rdz", "rdx", "rdy",
                                 "rcx", "rcy")}


def lib_input(case: dict, bc: str = "hbc") -> dict:
    """The input.json subset rtmb.Params.from_input() reads."""
    return dict(nx=case["nx"], ny=case["ny"], nz=case["nz"], blen=case["blen"], nt=case["nt"],
                ntstep=case["ntstep"], stencil_order=case["order"], dx=case["dx"], dy=case["dy"],
                dz=case["dz"], dt=case["dt"], fpeak=case["fpeak"], taper_factor=case["taper_factor"],
                receiver_start_x=case["rsx"], receiver_start_y=case["rsy"], receiver_depth_z=case["rdz"],
                receiver_distance_x=case["rdx"], receiver_distance_y=case["rdy"],
                receiver_count_x=case["rcx"], receiver_count_y=case["rcy"], boundary_condition=bc)


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def bitexact(a, b) -> bool:
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))
