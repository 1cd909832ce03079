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
