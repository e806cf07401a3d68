"""Continuous-batching serving loop: requests arriving while others run are batched onto free
slots and overlap on the device; every result equals the one computed alone (batched call)."""
import numpy as np
import pytest
import torch

import dpcrypto_b200 as d
from dpcrypto_b200.serving import RequestPool, Server, poisson_arrivals

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("form", [d.FORM_TC, d.FORM_DP4A])
def test_serving_results_equal_alone(engine, form, oracle_check_items):
    pool = RequestPool(engine, 700, seed=3)
    srv = Server(slots=3, max_batch=128, form=form, hbm_budget=256 << 20)
    try:
        res = srv.run(pool, poisson_arrivals(pool.n, rate=20000.0, seed=1))
    finally:
        srv.close()
    torch.cuda.synchronize()
    assert pool.check()
    assert oracle_check_items(pool.items(), stride=11) >= 60
    assert res["batches"] > 1 and np.isfinite(res["latency_ms"]).all() and (res["latency_ms"] > 0).all()


def test_serving_split_classes(engine, oracle_check_items):
    """Frodo and Saber requests on separate slots: results unchanged, Saber requests no
    longer wait for Frodo batches."""
    from dpcrypto_b200.serving import FRODO_CLASS, SABER_CLASS

    pool = RequestPool(engine, 600, seed=4)
    srv = Server(slots=4, max_batch=128, form=d.FORM_TC, hbm_budget=256 << 20,
                 classes=[FRODO_CLASS, FRODO_CLASS, SABER_CLASS, SABER_CLASS])
    try:
        res = srv.run(pool, poisson_arrivals(pool.n, rate=20000.0, seed=2))
    finally:
        srv.close()
    torch.cuda.synchronize()
    assert pool.check()
    assert oracle_check_items(pool.items(), stride=13, offset=5) >= 40
    assert np.isfinite(res["latency_ms"]).all()
    assert res["saber_p50_ms"] < res["frodo_p50_ms"]


@pytest.mark.parametrize("form", [d.FORM_TC, d.FORM_DP4A])
def test_service_server_results_equal_alone(engine, form, oracle_check_items):
    """Admission inside the running kernel (dpkem_service_*): requests submitted one arrival
    at a time, results equal the batched calls' and a stride sample the oracle's."""
    from dpcrypto_b200.serving import ServiceServer

    pool = RequestPool(engine, 700, seed=5)
    srv = ServiceServer(form=form, saber_ctas=16)
    try:
        res = srv.run(pool, poisson_arrivals(pool.n, rate=20000.0, seed=3))
        pool.clear()
        res2 = srv.run(pool, np.zeros(pool.n))  # everything at once, on the same running service
    finally:
        srv.close()
    torch.cuda.synchronize()
    assert pool.check()
    assert oracle_check_items(pool.items(), stride=11, offset=3) >= 60
    for r in (res, res2):
        assert np.isfinite(r["latency_ms"]).all() and (r["latency_ms"] > 0).all()
    assert res["submits"] > 10
