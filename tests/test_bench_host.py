"""Host-side arithmetic of bench.py (no GPU): the workload's size and update count, the algorithmic
bytes the roofline divides by, and the traffic figures it reads from the committed ncu summaries."""
import math
import os

import bench


def test_workload_size_and_updates():
    p = bench.workload(512, 3000)
    assert (p["nx"], p["ny"], p["nz"], p["blen"], p["nt"]) == (512, 512, 512, 40, 3000)
    assert bench.n_points(p) == 592 ** 3
    # nt forward, nt - 2 source-reconstruction and nt receiver steps over the padded grid
    assert bench.updates_per_shot(p) == 592 ** 3 * (3 * 3000 - 2)


def test_dual_step_bytes_per_point():
    # split form: every launch reads S, S_prev, R, R_prev, v2dt2 and IMG and writes S, R and IMG
    assert bench.dual_bytes_per_point({"dual_variant": 1}, 3000) == 36.0
    assert bench.dual_kernel_name({"dual_variant": 3}) == "dual_step_kernel"
    # merged form (the default, variants 4-7): launches pair up on the image, 28 + 36 bytes a pair
    assert bench.dual_kernel_name(None) == "dual_merged_kernel"
    assert bench.dual_bytes_per_point(None, 3000) == 32.0
    assert bench.dual_bytes_per_point({"dual_variant": 4}, 62) == 32.0
    # an odd number of dual launches (nt - 2 = 3): one pair and one unpaired launch
    assert math.isclose(bench.dual_bytes_per_point({"dual_variant": 5}, 5), (28 + 36 + 36) / 3)


def test_traffic_figures_come_from_the_profiles():
    for kind in ("forward", "backward_source", "backward_receiver", "backward_dual", "model"):
        v = bench.ncu_traffic_per_point(kind)
        assert v is not None and 8 < v < 40, (kind, v)
    # the measured traffic stays at or below the algorithmic bytes (no re-reads from DRAM)
    assert bench.ncu_traffic_per_point("forward") <= 16
    assert bench.ncu_traffic_per_point("backward_dual") <= bench.dual_bytes_per_point(None, 3000)
    assert bench.ncu_traffic_per_point("unknown") is None


def test_peak_falls_back_without_the_measured_file(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    gbs, kind = bench.measured_hbm_gbs()
    assert kind == "fallback" and gbs == bench.HBM_FALLBACK_GBS
    (tmp_path / "MEASURED_PEAKS.json").write_text('{"hbm_gbs": 6545.9}')
    gbs, kind = bench.measured_hbm_gbs()
    assert kind == "measured" and gbs == 6545.9
    assert os.path.exists(tmp_path / "MEASURED_PEAKS.json")
