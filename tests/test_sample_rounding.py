"""The history sample of FP32 state is taken as the float product x * 1e6f.  The reference
stores Float32(x * 1e6) of a double (cutting.js:288-292), and the FP64 kernels round the
double product to float.  The two agree because the double product of a float and 1e6
is exact (24 + 14 significant bits), so both are the correctly rounded float product.
This checks the claim with IEEE arithmetic on the host."""
from __future__ import annotations

import numpy as np


def _both(x: np.ndarray):
    x = x.astype(np.float32)
    with np.errstate(over="ignore", invalid="ignore", under="ignore"):
        via_double = (x.astype(np.float64) * 1e6).astype(np.float32)
        in_float = x * np.float32(1e6)
    return via_double, in_float


def test_float_product_equals_rounded_double_product_random():
    rng = np.random.default_rng(20241204)
    # tool positions of a stable or chattering cut span ~1e-9..1e-3 m; cover far beyond
    mant = rng.uniform(1.0, 2.0, 2_000_000)
    expo = rng.integers(-149, 128, 2_000_000)
    sign = rng.choice([-1.0, 1.0], 2_000_000)
    x = (sign * np.ldexp(mant, expo)).astype(np.float32)
    a, b = _both(x)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_float_product_equals_rounded_double_product_edges():
    f = np.finfo(np.float32)
    x = np.array([0.0, -0.0, f.tiny, -f.tiny, f.smallest_subnormal, 3e-45, 1e-40,
                  f.max, -f.max, 3.4e32, 3.41e32, 1e-3, 2e-6, 1.0, np.inf, -np.inf],
                 dtype=np.float32)
    with np.errstate(over="ignore"):  # the neighbours of +-max are +-inf
        x = np.concatenate([x, np.nextafter(x, np.float32(np.inf)),
                            np.nextafter(x, np.float32(-np.inf))])
    a, b = _both(x)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    # a NaN stays a NaN either way (the run-away decision reads isfinite only)
    a, b = _both(np.array([np.nan], dtype=np.float32))
    assert np.isnan(a).all() and np.isnan(b).all()
