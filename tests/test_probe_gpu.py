"""The FP64 issue-rate probe (subfv_probe_fp64_fma) runs through the C-ABI, rejects a
bad iteration count, and returns a rate that scales with the work (same TFLOP/s for
twice the iterations, about twice the time)."""
import ctypes as C

import pytest

pytestmark = pytest.mark.gpu


def test_fp64_probe(native, cuda_ok):
    tf, ms = C.c_double(), C.c_double()
    assert native.subfv_probe_fp64_fma(0, C.byref(tf), C.byref(ms)) == -2
    assert native.subfv_probe_fp64_fma(2048, C.byref(tf), C.byref(ms)) == 0
    t1, m1 = tf.value, ms.value
    assert native.subfv_probe_fp64_fma(4096, C.byref(tf), C.byref(ms)) == 0
    t2, m2 = tf.value, ms.value
    assert 1.0 < t1 < 500.0 and 1.0 < t2 < 500.0
    assert 1.5 < m2 / m1 < 2.5


def test_exact_division_by_3_and_6(native, cuda_ok):
    """div3 / div6 (the geometry kernels' reciprocal multiply with one FMA remainder
    correction) agree bit for bit with CUDA's division: on random doubles over the whole
    exponent range (every inexact x/3 sits exactly ulp/6 from a rounding midpoint, the
    closest any quotient by 3 can get, so random significands exercise the hard case),
    around powers of two and multiples of 3, and on zeros, subnormals, infinities, NaN."""
    import numpy as np
    rng = np.random.default_rng(7)
    bits = rng.integers(0, 1 << 63, size=1 << 24, dtype=np.int64, endpoint=False)
    x = bits.view(np.float64).copy()
    x[::2] *= -1.0
    # geometry-sized values: coordinates, areas and volumes of small cells
    y = rng.uniform(-1.0, 1.0, 1 << 22) * np.exp2(rng.integers(-60, 4, 1 << 22))
    near = []
    for k in range(-1070, 1024, 7):
        for base in (1.0, 3.0, 6.0, 1.5):
            v = np.ldexp(base, k)
            if np.isfinite(v) and v != 0.0:
                near.extend([np.nextafter(v, -np.inf), v, np.nextafter(v, np.inf)])
    special = [0.0, -0.0, 5e-324, -5e-324, 2.2250738585072014e-308, np.inf, -np.inf, np.nan,
               1.7976931348623157e308, -1.7976931348623157e308, 2.0 ** -960, 2.0 ** 960, 3.0, 6.0, -3.0]
    allx = np.ascontiguousarray(np.concatenate([x, y, np.array(near), np.array(special)]))
    bad = C.c_int64(-1)
    rc = native.subfv_probe_div_const(allx.ctypes.data_as(C.POINTER(C.c_double)), allx.size, C.byref(bad))
    assert rc == 0
    assert bad.value == 0, bad.value
