"""The identity behind the step kernels' CFL reduction, checked on the CPU.

Pass 1 needs min over cells of dt_c = 1 / (iv_c * lam_c).  The kernels keep the largest
x_c = iv_c * lam_c instead and form one reciprocal per block: a correctly rounded reciprocal
does not grow as its argument grows, so min_c fl(1 / x_c) == fl(1 / max_c x_c) bit for bit.
numpy's division is IEEE (correctly rounded), so it stands in for the device's FP64 division.
"""
import numpy as np
import pytest


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_min_of_reciprocals_is_reciprocal_of_max(dtype):
    rng = np.random.default_rng(11)
    for scale in (1e-300 if dtype == np.float64 else 1e-30, 1e-8, 1.0, 1e8):
        for _ in range(200):
            n = int(rng.integers(1, 300))
            x = (rng.random(n) * scale * rng.choice([1.0, 10.0, 1e3], n)).astype(dtype)
            x = x[x > 0]
            if x.size == 0:
                continue
            one = dtype(1)
            a = np.min(one / x)
            b = one / np.max(x)
            assert a.tobytes() == b.tobytes(), (scale, a, b)


def test_neighbouring_arguments_keep_the_order():
    # runs of arguments one ulp apart, in several binades: the reciprocals never cross
    for base in (1e-200, 0.75, 1.0, 3.0, 1e150):
        x = np.empty(4000)
        x[0] = base
        for i in range(1, x.size):
            x[i] = np.nextafter(x[i - 1], np.inf)
        r = 1.0 / x
        assert np.all(np.diff(r) <= 0)
