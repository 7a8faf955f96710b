"""CPU checks of the arithmetic the vertex-move delta-MDL uses for g(a) - g(b), g(x) = x log x, of
integer counts (dxlogx_int in sbp_device.cuh), restated in numpy float64 and compared with a
long-double evaluation of the same quantity:

  g(a) - g(b) = (a - b) log a + b log(a / b),
  log x from a table of (hi, lo) doubles (hi = log x rounded, lo = the rest),
  log(a / b) = 2 atanh(z), z = (a - b) / (a + b), by 2 (z + z^3/3 + z^5/5 + z^7/7) when
  128 |a - b| <= b (b > 0), else (hi_a - hi_b) + (lo_a - lo_b).

The form the kernels used before it, (a - b) log a + b log1p((a - b) / b), is checked beside it."""
import numpy as np
import pytest

TABLE = 1 << 20


@pytest.fixture(scope="module")
def log_table():
    x = np.arange(TABLE, dtype=np.longdouble)
    x[0] = 1
    full = np.log(x)
    hi = full.astype(np.float64)
    lo = (full - hi.astype(np.longdouble)).astype(np.float64)
    return hi, lo


def table_form(hi, lo, a, b):
    a = np.asarray(a, np.int64)
    b = np.asarray(b, np.int64)
    sa, sb = np.maximum(a, 1), np.maximum(b, 1)
    d = a - b
    close = (b > 0) & (128 * np.abs(d) <= b)
    with np.errstate(divide="ignore", invalid="ignore"):
        z = d.astype(np.float64) / (a.astype(np.float64) + b.astype(np.float64))
    w = z * z
    series = 2.0 * z + 2.0 * z * w * (1.0 / 3.0 + w * (1.0 / 5.0 + w * (1.0 / 7.0)))
    diff = (hi[sa] - hi[sb]) + (lo[sa] - lo[sb])
    lab = np.where(close, series, diff)
    return d.astype(np.float64) * (hi[sa] + lo[sa]) + b.astype(np.float64) * lab


def log1p_form(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    sa, sb = np.where(a > 0, a, 1.0), np.where(b > 0, b, 1.0)
    return (a - b) * np.log(sa) + b * np.log1p((sa - sb) / sb)


def reference(a, b):
    a = np.asarray(a, np.longdouble)
    b = np.asarray(b, np.longdouble)
    sa, sb = np.where(a > 0, a, 1), np.where(b > 0, b, 1)
    return (a - b) * np.log(sa) + b * np.log1p((sa - sb) / sb)


def pairs(seed, n):
    rng = np.random.default_rng(seed)
    a = np.concatenate([rng.integers(0, 100, n), rng.integers(0, 5000, n), rng.integers(0, 1_000_000, n)])
    d = np.concatenate([rng.integers(-100, 101, 2 * n), rng.integers(-3000, 3001, n)])
    b = a + d
    ok = (b >= 0) & (b < TABLE) & (a < TABLE) & (d != 0)
    return a[ok], b[ok]


def test_table_form_matches_long_double(log_table):
    hi, lo = log_table
    a, b = pairs(1, 200_000)
    ref = reference(a, b)
    got = table_form(hi, lo, a, b).astype(np.longdouble)
    rel = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300)
    assert float(rel.max()) < 1e-15
    # no worse than the log + log1p form it replaced
    old = log1p_form(a, b).astype(np.longdouble)
    rel_old = np.abs(old - ref) / np.maximum(np.abs(ref), 1e-300)
    assert float(rel.max()) <= float(rel_old.max())


def test_zero_sides_and_equal_counts(log_table):
    hi, lo = log_table
    for a, b in [(0, 7), (7, 0), (1, 0), (0, 1), (5, 5), (1000, 1000), (0, 0)]:
        ref = float(reference(np.array([a]), np.array([b]))[0])
        got = float(table_form(hi, lo, np.array([a]), np.array([b]))[0])
        assert got == pytest.approx(ref, rel=1e-15, abs=1e-15)
    # g(a) - g(a) is exactly zero
    assert float(table_form(hi, lo, np.array([12345]), np.array([12345]))[0]) == 0.0


def test_delta_is_antisymmetric(log_table):
    hi, lo = log_table
    a, b = pairs(2, 50_000)
    s = table_form(hi, lo, a, b) + table_form(hi, lo, b, a)
    scale = np.abs(table_form(hi, lo, a, b)) + 1.0
    assert float(np.max(np.abs(s) / scale)) < 1e-14
