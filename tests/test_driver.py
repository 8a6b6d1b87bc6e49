"""The operator-split caller's formats: mass fractions <-> number densities
and t_stop ladders (tests/rober.f90, tests/orego.f90, tests/primordial.f90
of the reference).

CPU tests check the reference drivers' schedules, the oracle's conversion
against its formula and conservation along oracle ladders; GPU tests check
the device conversion and the device ladder (eager and replayed as CUDA
graphs) bit for bit against the oracle's ladder."""
import numpy as np
import pytest

from odevec_b200 import driver as D
from odevec_b200.networks import PRIMORDIAL_IMASSES, PRIMORDIAL_MASSES


def test_reference_schedules():
    r = D.rober_schedule(64)
    assert len(r.t_stops) == 21 and r.t_stops[0] == 1e-10 and r.t_stops[-1] < np.float32(1e11)
    assert r.rtol == 1e-8 and r.atol == 1e-6 * 1e-8 and r.dt_reset == 1e-10 and r.group == 32
    o = D.orego_schedule(64, t_end=2.0)
    assert o.t_stops[0] == 1.0 and o.t_stops[1] == 1.0 + float(np.float32(0.01))
    assert all(t <= np.float32(2.0) for t in o.t_stops) and len(o.t_stops) in (100, 101)
    p = D.primordial_schedule(64)
    assert len(p.t_stops) == 100 and p.t_stops[-1] == 1e10 and p.rho is not None
    assert np.allclose(p.y0[:12].sum(axis=0), 1.0, rtol=1e-15) and np.all(p.y0[14] == 1000.0)


def test_oracle_conversion_is_the_reference_formula(oracle):
    rng = np.random.default_rng(4)
    x = rng.uniform(0, 1, (16, 50))
    x[14] = rng.uniform(10, 1e4, 50)  # temperature row passes through
    rho = 10.0 ** rng.uniform(-25, -5, 50)
    m, im = np.array(PRIMORDIAL_MASSES), np.array(PRIMORDIAL_IMASSES)
    n = oracle.convert("PRIMORDIAL_CSC_FF", x, rho, 0)
    want = np.where(m[:, None] != 0, rho[None, :] * x * im[:, None], x)
    assert np.array_equal(n, want)
    back = oracle.convert("PRIMORDIAL_CSC_FF", n, rho, 1)
    assert np.array_equal(back, np.where(m[:, None] != 0, n * m[:, None] / rho[None, :], n))
    # KROME's inverse masses are rounded to 12 digits
    assert np.allclose(back, x, rtol=1e-10, atol=0)
    with pytest.raises(ValueError):
        oracle.convert("ROBER_DENSE_NONE", x[:3], rho, 0)


def test_oracle_ladders_conserve(oracle):
    p = D.primordial_schedule(32)
    p.t_stops = p.t_stops[:20]
    x, t, d, st = oracle.ladder(p.network, p.y0, p.time, p.dt, p.t_stops, p.rtol, p.atol, p.dt_min,
                                rho=p.rho, dt_reset=p.dt_reset)
    assert np.all(st == 0) and np.all(t == p.t_stops[-1])
    # mass fractions: every reaction conserves mass (KROME's masses add up)
    assert np.max(np.abs(x[:12].sum(axis=0) - 1.0)) < 1e-8
    r = D.rober_schedule(64)
    y, t, d, st = oracle.ladder(r.network, r.y0, r.time, r.dt, r.t_stops, r.rtol, r.atol, r.dt_min,
                                dt_reset=r.dt_reset, group=32)
    assert np.all(st == 0) and np.max(np.abs(y.sum(axis=0) - 1.0)) < 1e-12


# ------------------------------------------------------------------- GPU
@pytest.mark.gpu
def test_gpu_conversion_matches_oracle(gpu_lib, oracle):
    import torch
    rng = np.random.default_rng(5)
    x = rng.uniform(0, 1, (16, 1000))
    rho = 10.0 ** rng.uniform(-25, -5, 1000)
    xt, rt = torch.tensor(x, device="cuda"), torch.tensor(rho, device="cuda")
    n = D.x2n("PRIMORDIAL_CSC_FF", xt, rt)
    assert np.array_equal(n.cpu().numpy(), oracle.convert("PRIMORDIAL_CSC_FF", x, rho, 0))
    D.n2x("PRIMORDIAL_CSC_FF", n, rt, out=n)  # in place
    assert np.array_equal(n.cpu().numpy(), oracle.convert("PRIMORDIAL_CSC_FF", oracle.convert(
        "PRIMORDIAL_CSC_FF", x, rho, 0), rho, 1))


def _schedules():
    p = D.primordial_schedule(128)
    o = D.orego_schedule(128, t_end=1.5)
    return [("rober", D.rober_schedule(256)), ("primordial", p), ("orego", o)]


@pytest.mark.gpu
@pytest.mark.parametrize("graph", [False, True])
@pytest.mark.parametrize("name,sch", _schedules())
def test_gpu_ladder_bit_exact_vs_oracle(gpu_lib, oracle, name, sch, graph):
    ref = oracle.ladder(sch.network, sch.y0, sch.time, sch.dt, sch.t_stops, sch.rtol, sch.atol, sch.dt_min,
                        rho=sch.rho, dt_reset=sch.dt_reset, group=sch.group)
    got = D.run_schedule(sch, "fp64", graph=graph, chunk=16)
    for what, a, b in zip(("y", "time", "dt", "status"), got, ref):
        assert np.array_equal(a, b), "%s %s graph=%s" % (name, what, graph)


@pytest.mark.gpu
def test_gpu_ladder_graph_equals_eager_fp32(gpu_lib):
    sch = D.primordial_schedule(256)
    a = D.run_schedule(sch, "fp32_lu", graph=False)
    b = D.run_schedule(sch, "fp32_lu", graph=True, chunk=32)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


@pytest.mark.gpu
def test_gpu_ladder_graph_with_visit_order(gpu_lib):
    """A ladder of more than 32,768 cells: every call sorts its cells
    longest span first on the stream, inside the captured graphs too; the
    replayed graphs give the eager ladder's bits."""
    sch = D.primordial_schedule(40000)
    sch.t_stops = sch.t_stops[:6]
    a = D.run_schedule(sch, "fp32_lu", graph=False)
    b = D.run_schedule(sch, "fp32_lu", graph=True, chunk=3)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
