"""Serving: requests arriving while others run are admitted as memory frees up, their
work shares launches with the in-flight solves, and each result is the same, bit for
bit, as the same request solved alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [0, 1])
def test_served_results_equal_solo(native, cuda_ok, precision):
    from subfv_b200 import serve
    reqs = serve.make_requests(10, rate=40.0, seed=7, cells_min=600, cells_max=6000, time_scale=0.03)
    assert {r.kind for r in reqs} == {"gresho", "sedov"}
    # a budget that holds only some of the requests at once, so admission waits for frees
    sizes = []
    for r in reqs[:4]:
        m, _, _ = serve.build(r)
        sizes.append(m.device_bytes)
        m.close()
    srv = serve.Server(budget_bytes=int(3 * max(sizes) * 2.5), capacity=16, precision=precision, chunk=8,
                       build_threads=2)
    results, makespan = srv.run(reqs)
    srv.close()
    assert sorted(r.rid for r in results) == list(range(len(reqs)))
    assert makespan > 0
    by_id = {r.rid: r for r in results}
    for req in reqs:
        got = by_id[req.rid]
        steps, t, st, sol = serve.solve_alone(req, precision=precision)
        assert got.status == st == 0
        assert got.steps == steps and got.t == t, (req, got.steps, steps, got.t, t)
        assert t >= req.t_end
        np.testing.assert_array_equal(got.sol, sol)
    stats = serve.latency_stats(results)
    assert 0 < stats["p50_s"] <= stats["p99_s"]
