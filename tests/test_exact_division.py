"""The tracer's division by a known divisor (``div_known`` in ``csrc/common.cuh``).

The kernel divides by the mesh spacing with its reciprocal rounded once and two remainder
corrections by fused multiply-adds; Markstein's theorem makes that the correctly rounded
quotient.  The same steps in C with the C library's ``fma`` (a correctly rounded fused
multiply-add, as the GPU's) must give ``a / b`` bit for bit on spacings and coordinates of
the tracer's ranges, on multiples of the spacing (cell boundaries) and on random bit
patterns.  The device code itself is checked by the bit-exact trace parity tests.
"""

from __future__ import annotations

import ctypes
import shutil
import subprocess

import numpy as np
import pytest

SOURCE = r"""
#include <math.h>
#include <stdint.h>
#include <string.h>

static double div_known(double a, double b, double rb) {
    const double m = fabs(a);
    if (rb == 0.0 || !(m >= 0x1p-900 && m <= 0x1p900)) return a / b;
    double q = a * rb;
    double r = fma(-q, b, a);
    q = fma(r, rb, q);
    r = fma(-q, b, a);
    return fma(r, rb, q);
}

static double known_reciprocal(double b) {
    return (b >= 0x1p-60 && b <= 0x1p60) ? 1.0 / b : 0.0;
}

/* the number of a[i] / b[j] (all pairs) that differ from the IEEE quotient in any bit */
long mismatches(const double *a, long na, const double *b, long nb) {
    long bad = 0;
    for (long j = 0; j < nb; ++j) {
        const double rb = known_reciprocal(b[j]);
        for (long i = 0; i < na; ++i) {
            const double q = div_known(a[i], b[j], rb), e = a[i] / b[j];
            if (memcmp(&q, &e, sizeof q) != 0 && !(q != q && e != e)) ++bad;
        }
    }
    return bad;
}
"""


@pytest.fixture(scope="module")
def division(tmp_path_factory):
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    d = tmp_path_factory.mktemp("div")
    (d / "div.c").write_text(SOURCE)
    so = d / "div.so"
    subprocess.run([gcc, "-O2", "-ffp-contract=off", "-shared", "-fPIC", str(d / "div.c"),
                    "-o", str(so), "-lm"], check=True)  # fmt: skip
    lib = ctypes.CDLL(str(so))
    lib.mismatches.restype = ctypes.c_long
    lib.mismatches.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p, ctypes.c_long]

    def count(a: np.ndarray, b: np.ndarray) -> int:
        a = np.ascontiguousarray(a, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        return lib.mismatches(a.ctypes.data, a.size, b.ctypes.data, b.size)

    return count


def _random_bits(rng, n, lo_exp, hi_exp):
    mantissa = rng.integers(0, 1 << 52, n, dtype=np.uint64)
    exponent = rng.integers(lo_exp + 1023, hi_exp + 1023, n).astype(np.uint64)
    sign = rng.integers(0, 2, n).astype(np.uint64)
    return ((sign << np.uint64(63)) | (exponent << np.uint64(52)) | mantissa).view(np.float64)


def test_spacings_and_coordinates(division):
    rng = np.random.default_rng(11)
    spacings = np.concatenate([
        1e-4 * (0.5 + rng.random(200)),                    # mesh spacings of 50-150 um
        0.08 / (rng.integers(64, 4096, 200) - 1.0),        # 80 mm over n - 1 cells
        np.abs(_random_bits(rng, 200, -20, 4)),            # any spacing of 1 um to 16 m
        [6.0, 1e-4, 2.5e-4, 0.1, 1.0 / 3.0],
    ])  # fmt: skip
    coordinates = np.concatenate([
        (rng.random(2000) - 0.3) * 0.2,                    # positions less an origin
        _random_bits(rng, 2000, -40, 6),                   # differences of any size
        rng.random(2000) * 1e-9,                           # step sizes
    ])  # fmt: skip
    assert division(coordinates, spacings) == 0


def test_cell_boundaries(division):
    """Exact multiples of the spacing, and their neighbours, divide to integers exactly."""
    rng = np.random.default_rng(12)
    spacings = np.concatenate([1e-4 * (0.5 + rng.random(50)), 0.08 / (np.arange(60, 110) - 1)])
    for b in spacings:
        k = np.arange(-50, 4100, dtype=np.float64)
        a = k * b
        a = np.concatenate([a, np.nextafter(a, np.inf), np.nextafter(a, -np.inf)])
        assert division(a, np.array([b])) == 0


def test_edge_values_take_the_ieee_division(division):
    specials = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 5e-324, -5e-324, 2.2e-308, 1e300,
                         -1e300, 1.7e308, 2.0**-900, 2.0**900])  # fmt: skip
    assert division(specials, np.array([1e-4, 6.0, 1e-30, 1e30, 0.0, -1e-4, np.inf])) == 0
