"""The request loop (fluxos_cpp_b200.serve): requests that arrive while
others run are admitted as memory frees up, share the batch launches, retire
at their horizon, and each result is bit-identical to the same scenario run
alone to its horizon."""
import numpy as np
import pytest

import fluxos_cpp_b200 as fx
from fluxos_cpp_b200 import scenarios as S
from fluxos_cpp_b200 import serve

pytestmark = pytest.mark.gpu


def _requests(precision):
    reqs = serve.poisson_requests(rate=20.0, duration=0.4, seed=4, n_min=40, n_max=160,
                                  horizon_h=(0.01, 0.03), nchem=(1, 3), precision=precision)
    assert len(reqs) >= 4
    return reqs


def _alone(r):
    sc = r.make()
    d = S.make_domain(sc, precision=r.precision, steps_in_flight=r.steps_in_flight)
    while True:
        st = d.step(512)
        if st["print_pending"]:
            d.print_done()
        if st["finished"]:
            break
    out = {k: d.download(k) for k in ("h", "qx", "conc")}
    out["steps"] = st["steps"]
    d.close()
    return out


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_serving_results_match_alone(precision):
    reqs = _requests(precision)
    # room for about two of the largest at a time: later arrivals wait
    cap = 2.2 * max(serve.Server.footprint(r) for r in reqs)
    srv = serve.Server(cap_bytes=cap, chunk_steps=16, keep=("h", "qx", "conc"))
    stats = srv.run(reqs)
    srv.close()
    assert stats["peak_device_bytes"] <= cap
    assert stats["peak_members"] >= 2
    assert all(r.done is not None and r.status["finished"] for r in reqs)
    assert stats["p99_s"] >= stats["p50_s"] > 0
    for r in reqs:
        ref = _alone(r)
        assert r.steps == ref["steps"], r.rid
        for k in ("h", "qx", "conc"):
            assert np.array_equal(r.state[k], ref[k]), (r.rid, k)
