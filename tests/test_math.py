"""The shared elementary functions (odevec_b200/csrc/ov_common.h) against the
C library, through the oracle build (same source as the device code)."""
import numpy as np
import pytest


def ulps(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) / np.spacing(np.abs(b))


@pytest.fixture(scope="module")
def lib(oracle):
    return oracle.lib()


def test_exp(lib):
    rng = np.random.default_rng(0)
    xs = np.concatenate([rng.uniform(-745, 709.7, 20000), rng.uniform(-1, 1, 20000),
                         [0.0, -0.0, 1.0, -1.0, 700.0, -700.0, -740.0]])
    got = np.array([lib.ov_oracle_exp(float(x)) for x in xs])
    ref = np.exp(xs)
    normal = ref > 2.3e-308
    assert np.max(ulps(got[normal], ref[normal])) <= 2.0
    sub = (ref > 0) & ~normal
    assert np.all(np.abs(got[sub] - ref[sub]) <= 2 * 4.9e-324 * 4)
    assert lib.ov_oracle_exp(1000.0) == np.inf and lib.ov_oracle_exp(-1000.0) == 0.0
    assert np.isnan(lib.ov_oracle_exp(float("nan")))


def test_log(lib):
    rng = np.random.default_rng(1)
    xs = np.concatenate([10.0 ** rng.uniform(-300, 300, 20000), rng.uniform(0.5, 2.0, 20000),
                         [1.0, 2.0, 0.5, 1e-310, 5e-324, 1.7e308]])
    got = np.array([lib.ov_oracle_log(float(x)) for x in xs])
    ref = np.log(xs)
    nz = ref != 0
    assert np.max(ulps(got[nz], ref[nz])) <= 2.0
    assert lib.ov_oracle_log(1.0) == 0.0
    assert lib.ov_oracle_log(0.0) == -np.inf and np.isnan(lib.ov_oracle_log(-1.0))


def test_pow(lib):
    rng = np.random.default_rng(2)
    x = 10.0 ** rng.uniform(-10, 10, 20000)
    y = rng.uniform(-3, 3, 20000)
    got = np.array([lib.ov_oracle_pow(float(a), float(b)) for a, b in zip(x, y)])
    ref = np.power(x, y)
    # exp(y log x): relative error grows with |y log x| (<= 70 here)
    rel = np.abs(got - ref) / ref
    assert np.max(rel / (1.0 + np.abs(y * np.log(x)))) < 4e-16
    assert lib.ov_oracle_pow(0.0, 0.5) == 0.0 and lib.ov_oracle_pow(7.0, 0.0) == 1.0
    assert abs(lib.ov_oracle_pow(-2.0, 3.0) + 8.0) < 1e-14 and np.isnan(lib.ov_oracle_pow(-2.0, 0.5))


def _bits(v):
    return np.float64(v).view(np.int64)


def _same(a, b):
    return _bits(a) == _bits(b) or (np.isnan(a) and np.isnan(b))


SPECIAL = [0.0, -0.0, 1.0, -1.0, 2.0, -2.0, 0.5, -0.5, 3.0, -3.0, np.inf, -np.inf, np.nan, 5e-324, -5e-324,
           1e-310, 2.2250738585072014e-308, 1.7976931348623157e308, 709.782712893384, 709.7827128933841,
           -745.1332191019412, -745.1332191019413, 700.0, -740.0, 1e-300, 1e300]


def test_branch_free_functions_are_bit_identical(lib):
    # the step-size selection evaluates its three powers with the branch-free
    # forms; every result must be the branching function's, bit for bit
    rng = np.random.default_rng(5)
    xs = np.concatenate([rng.uniform(-800, 800, 4000), 10.0 ** rng.uniform(-320, 308, 4000),
                         -(10.0 ** rng.uniform(-320, 308, 1000)), SPECIAL])
    for x in xs:
        assert _same(lib.ov_oracle_exp_sel(float(x)), lib.ov_oracle_exp(float(x))), x
        assert _same(lib.ov_oracle_log_sel(float(x)), lib.ov_oracle_log(float(x))), x
    px = np.concatenate([10.0 ** rng.uniform(-30, 30, 3000), -(10.0 ** rng.uniform(-5, 5, 500)), SPECIAL])
    py = np.concatenate([rng.uniform(-4, 4, 3000), rng.integers(-5, 6, 500).astype(float), SPECIAL])
    ys = np.concatenate([py, [1.0 / k for k in range(1, 8)], SPECIAL])
    for x in px:
        for y in rng.choice(ys, 8):
            assert _same(lib.ov_oracle_pow_sel(float(x), float(y)), lib.ov_oracle_pow(float(x), float(y))), (x, y)
    for x in SPECIAL:
        for y in SPECIAL + [1.0 / k for k in range(1, 8)]:
            assert _same(lib.ov_oracle_pow_sel(float(x), float(y)), lib.ov_oracle_pow(float(x), float(y))), (x, y)


def _rate_floor_reference(y):
    # src/odevec_commons.F90:127-130: running maximum from y_1, clamped to 1
    nmax = y[0]
    for v in y[1:]:
        nmax = v if v > nmax else nmax
    nmax = nmax if nmax > 1.0 else 1.0
    return 1e-40 / (nmax * nmax * nmax)


def test_rate_floor_tree_maximum_matches_running_maximum(lib):
    import ctypes
    rng = np.random.default_rng(9)
    r = np.zeros(38)
    k = np.zeros(38)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    for trial in range(3000):
        y = 10.0 ** rng.uniform(-30, 8, 16)
        y *= rng.choice([1.0, -1.0], 16, p=[0.8, 0.2])
        for _ in range(rng.integers(0, 4)):
            y[rng.integers(0, 16)] = rng.choice([np.nan, 0.0, -0.0, 1.0, np.inf, -np.inf, 0.5, 2.0])
        if trial % 7 == 0:
            y[0] = np.nan
        y = np.ascontiguousarray(y)
        lib.ov_oracle_rates_k(P(y), 16, P(r), P(k))
        want = _rate_floor_reference(list(y))
        assert _same(k[0], want), (y, k[0], want)
