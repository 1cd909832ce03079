"""The serving request stream (host logic, no GPU)."""
import numpy as np


def test_request_stream_is_seeded():
    from subfv_b200 import serve
    a = serve.make_requests(50, rate=5.0, seed=3)
    b = serve.make_requests(50, rate=5.0, seed=3)
    assert a == b
    gaps = np.diff([0.0] + [r.arrival for r in a])
    assert np.all(gaps > 0)
    cells = np.array([r.n_cells for r in a])
    assert cells.min() >= 4096 * 0.9 and cells.max() <= (1 << 20) * 1.1
    assert all(r.tri for r in a if r.kind == "sedov")
    assert {r.tri for r in a if r.kind == "gresho"} == {True, False}
    for r in a:
        nominal = serve.GRESHO_T_NOMINAL if r.kind == "gresho" else serve.SEDOV_T_NOMINAL
        assert 0.1 * nominal <= r.t_end <= nominal
