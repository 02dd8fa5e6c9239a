"""Pin the CPU oracle: bit-exact against the reference's golden fixtures (always) and against the
reference build itself (when oracle/_ref is present)."""
import numpy as np
import pytest

from rtm_cases import CASES, bitexact, layered_model, oracle_params


def test_ops_vs_golden(oracle, golden):
    g = golden["ops"]
    P, PP, V = g["P"], g["PP"], g["V"]
    b = 6
    for order in (2, 4, 8, 12):
        c = oracle.stencil_coefs(order, 10.0, 12.5, 7.5)
        assert bitexact(c, g[f"coefs{order}"]), order
        out, nan = oracle.step(order, c, P, PP, V)
        assert nan == 0
        assert bitexact(out, g[f"step{order}"]), order
    t = oracle.taper_vector(b, 0.2)
    assert bitexact(t, g["taper"])
    assert bitexact(oracle.taper(P, b, t, upper=False), g["taper_all"])
    assert bitexact(oracle.taper(P, b, t, upper=True), g["taper_upper"])
    assert bitexact(oracle.image(P, PP, V, b), g["image"])
    assert bitexact(oracle.filter_remove(P, b, 10.0, 12.5, 7.5), g["filter"])
    assert bitexact(oracle.ricker(500, 0.001, 15.0), g["ricker"])
    for bc in ("abc", "rbc", "hbc"):
        assert bitexact(oracle.extend_init_borders(g["vel"], b, bc, seed=1234), g[f"borders_{bc}"]), bc


def _golden_case(oracle):
    case = CASES["golden"]
    return case, oracle_params(case)


def test_model_vs_golden(oracle, golden):
    case, p = _golden_case(oracle)
    ve = oracle.extend_init_borders(layered_model(case), case["blen"], "abc")
    rec, rc = oracle.model_shot(p, oracle.v2dt2(ve, case["dt"]))
    assert rc == 0
    assert bitexact(rec, golden["model_abc"]["rec"])


@pytest.mark.parametrize("bc", ["hbc", "rbc"])
def test_migration_vs_golden(oracle, golden, bc):
    case, p = _golden_case(oracle)
    g = golden[f"mig_{bc}"]
    img, rc = oracle.migrate(p, oracle.v2dt2(g["vpe"], case["dt"]), g["rec"], bc)
    assert rc == 0
    fin = oracle.filter_remove(img, case["blen"], case["dx"], case["dy"], case["dz"])
    assert bitexact(fin, g["img"])


def test_fmig_vs_golden(oracle, golden):
    """Frequency-domain RTM: the oracle's image equals the reference program's (fmig = true)."""
    case, p = _golden_case(oracle)
    g = golden["mig_fmig"]
    img, rc = oracle.migrate_fmig(p, oracle.v2dt2(g["vpe"], case["dt"]), g["rec"], float(g["fmin"]), float(g["fmax"]))
    assert rc == 0
    fin = oracle.filter_remove(img, case["blen"], case["dx"], case["dy"], case["dz"])
    assert np.abs(fin).max() > 0
    assert bitexact(fin, g["img"])


def test_fmig_tables_and_grouping(oracle):
    """nw = (fmax - fmin) / df with df = 1 / (nt dt); one pass over all frequencies (nwstep 0) and
    nwstep = nw are the same run; smaller groups change only the order of the image sums."""
    w2, kre, kim = oracle.fmig_tables(120, 0.001, 5.0, 40.0)
    assert len(w2) == 4 and kre.shape == (4, 120)
    assert kre[0, 0] == 1.0 and kim[0, 0] == 0.0
    case, p = _golden_case(oracle)
    ve = oracle.extend_init_borders(layered_model(case), case["blen"], "abc")
    v2 = oracle.v2dt2(ve, case["dt"])
    rec, _ = oracle.model_shot(p, v2)
    a, _ = oracle.migrate_fmig(p, v2, rec, 5.0, 40.0, 0)
    b, _ = oracle.migrate_fmig(p, v2, rec, 5.0, 40.0, 4)
    c, _ = oracle.migrate_fmig(p, v2, rec, 5.0, 40.0, 1)
    assert bitexact(a, b)
    assert np.linalg.norm(c - a) <= 1e-5 * np.linalg.norm(a)


def test_fmig_vs_reference_program(oracle):
    """A second case run through the reference program itself (order 4, rows of 37 floats)."""
    import glob
    import os
    import sys
    import tempfile
    from oracle import REF_BIN
    if not os.path.exists(REF_BIN):
        pytest.skip("reference program (oracle/_ref/RTM3D.bin) not present")
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    from make_golden import read_record, run_reference
    case = CASES["odd"]
    with tempfile.TemporaryDirectory() as wd:
        rec = read_record(run_reference(case, "model", wd))
        d = run_reference(case, "rbc", wd, extra=dict(fmig=True, fmig_min_freq=2.0, fmig_max_freq=30.0,
                                                      fmig_nwstep=1))
        want = np.fromfile(glob.glob(os.path.join(wd, "out", "RTMIMG_*"))[0], np.float32)
        b = case["blen"]
        vpe = np.fromfile(d["vpefile"], np.float32).reshape(case["nx"] + 2 * b, case["ny"] + 2 * b,
                                                            case["nz"] + 2 * b)
    p = oracle_params(case)
    img, rc = oracle.migrate_fmig(p, oracle.v2dt2(vpe, case["dt"]), rec, 2.0, 30.0)
    assert rc == 0
    fin = oracle.filter_remove(img, b, case["dx"], case["dy"], case["dz"])
    assert np.abs(want).max() > 0
    assert bitexact(fin, want.reshape(fin.shape))


def twod_case():
    """The golden case as a 2D model (nx = 1): the reference runs rtmStep2D on the plane x = blen."""
    return dict(CASES["golden"], nx=1, sx=0, rsx=0, rcx=1, rdx=1)


def test_twod_vs_golden(oracle, golden):
    g = golden["twod"]
    for order in (4, 8):
        c = oracle.stencil_coefs(order, 10.0, 12.5, 7.5)
        out, nan = oracle.step2d(order, c, g["P"], g["PP"], g["V"], 6)
        assert nan == 0
        assert bitexact(out, g[f"step{order}"]), order
    case = twod_case()
    p = oracle_params(case)
    ve = oracle.extend_init_borders(layered_model(case), case["blen"], "abc")
    rec, rc = oracle.model_shot(p, oracle.v2dt2(ve, case["dt"]))
    assert rc == 0 and bitexact(rec, g["rec"])
    for name in ("hbc", "rbc", "fmig"):
        v2 = oracle.v2dt2(g[f"vpe_{name}"], case["dt"])
        if name == "fmig":
            img, rc = oracle.migrate_fmig(p, v2, g["rec"], float(g["fmin"]), float(g["fmax"]))
        else:
            img, rc = oracle.migrate(p, v2, g["rec"], name)
        assert rc == 0
        fin = oracle.filter_remove(img, case["blen"], case["dx"], case["dy"], case["dz"])
        assert np.abs(fin).max() > 0
        assert bitexact(fin, g[f"img_{name}"]), name


def test_twod_vs_reference_program(oracle):
    """A second 2D case through the reference program itself (order 4, unequal spacing): record,
    HBC image and fmig image."""
    import glob
    import os
    import sys
    import tempfile
    from oracle import REF_BIN
    if not os.path.exists(REF_BIN):
        pytest.skip("reference program (oracle/_ref/RTM3D.bin) not present")
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    from make_golden import read_record, run_reference
    case = dict(CASES["odd"], nx=1, sx=0, rsx=0, rcx=1, rdx=1)
    b = case["blen"]
    shp = (1 + 2 * b, case["ny"] + 2 * b, case["nz"] + 2 * b)
    p = oracle_params(case)
    with tempfile.TemporaryDirectory() as wd:
        rec = read_record(run_reference(case, "model", wd))
        ve = oracle.extend_init_borders(layered_model(case), b, "abc")
        got, rc = oracle.model_shot(p, oracle.v2dt2(ve, case["dt"]))
        assert rc == 0 and np.abs(rec).max() > 0 and bitexact(got, rec)
        for name, extra in (("hbc", None), ("fmig", dict(fmig=True, fmig_min_freq=2.0, fmig_max_freq=30.0,
                                                            fmig_nwstep=1))):
            for f in glob.glob(os.path.join(wd, "out", "RTMIMG_*")):
                os.remove(f)
            d = run_reference(case, "hbc", wd, vpe_path=os.path.join(wd, f"vpe_{name}.bin"), extra=extra)
            want = np.fromfile(glob.glob(os.path.join(wd, "out", "RTMIMG_*"))[0], np.float32)
            v2 = oracle.v2dt2(np.fromfile(d["vpefile"], np.float32).reshape(shp), case["dt"])
            if name == "fmig":
                img, rc = oracle.migrate_fmig(p, v2, rec, 2.0, 30.0)
            else:
                img, rc = oracle.migrate(p, v2, rec, "hbc")
            assert rc == 0
            fin = oracle.filter_remove(img, b, case["dx"], case["dy"], case["dz"])
            assert np.abs(want).max() > 0
            assert bitexact(fin, want.reshape(fin.shape)), name


def test_step2d_vs_reference_build(oracle, reference):
    rng = np.random.default_rng(5)
    for (ny, nz, b, order) in ((11, 17, 5, 6), (16, 10, 8, 12)):
        shp = (1 + 2 * b, ny + 2 * b, nz + 2 * b)
        P = rng.standard_normal(shp).astype(np.float32)
        PP = rng.standard_normal(shp).astype(np.float32)
        V = (rng.random(shp) * 0.1).astype(np.float32)
        c = oracle.stencil_coefs(order, 9.0, 11.0, 13.0)
        ref, rc = reference.step(1, ny, nz, b, order, 9.0, 11.0, 13.0, P, PP, V)
        got, nan = oracle.step2d(order, c, P, PP, V, b)
        assert rc == 0 and nan == 0
        assert bitexact(got, ref)


def test_ops_vs_reference_build(oracle, reference):
    rng = np.random.default_rng(123)
    for (nx, ny, nz, b, order) in ((13, 11, 17, 5, 6), (9, 16, 10, 8, 16)):
        shp = (nx + 2 * b, ny + 2 * b, nz + 2 * b)
        P = rng.standard_normal(shp).astype(np.float32)
        PP = rng.standard_normal(shp).astype(np.float32)
        V = (rng.random(shp) * 0.1).astype(np.float32)
        c = oracle.stencil_coefs(order, 9.0, 11.0, 13.0)
        assert bitexact(c, reference.stencil_coefs(order, 9.0, 11.0, 13.0))
        a, _ = oracle.step(order, c, P, PP, V)
        r, _ = reference.step(nx, ny, nz, b, order, 9.0, 11.0, 13.0, P, PP, V)
        assert bitexact(a, r)
        t = oracle.taper_vector(b, 0.35)
        assert bitexact(t, reference.taper_vector(b, 0.35))
        for up in (False, True):
            assert bitexact(oracle.taper(P, b, t, up), reference.taper(P, nx, ny, nz, b, 0.35, up))
        vel = (1500 + 3000 * rng.random((nx, ny, nz))).astype(np.float32)
        for bc in ("abc", "rbc", "hbc"):
            assert bitexact(oracle.extend_init_borders(vel, b, bc, seed=99),
                            reference.extend_init_borders(vel, b, bc, seed=99)), bc
    for nt, dt, fp in ((3000, 0.001, 12.0), (2500, 0.00125, 10.0)):
        assert bitexact(oracle.ricker(nt, dt, fp), reference.ricker(nt, dt, fp))


def test_oracle_reports_nan(oracle):
    """The reference throws "Numerical Dispersion" on NaN (RTMCPUPlatform.cpp:374-391)."""
    shp = (12, 12, 12)
    P = np.zeros(shp, np.float32)
    P[6, 6, 6] = np.nan
    c = oracle.stencil_coefs(8, 10.0, 10.0, 10.0)
    _, nan = oracle.step(8, c, P, np.zeros(shp, np.float32), np.ones(shp, np.float32))
    assert nan == 1
