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
