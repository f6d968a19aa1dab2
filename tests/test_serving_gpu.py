"""Serving form: requests of different sizes arrive while others are being
stepped; each request's final state in the mix equals its state when solved
alone (bitwise), and the loop reports latency percentiles and throughput."""
import numpy as np
import pytest
import torch

from kineticeq_b200.serving import Request, Server, poisson_stream, solve_alone

pytestmark = pytest.mark.gpu
SP = dict(picard_iter=64, picard_tol=1e-10, abs_tol=1e-16)


def _stream(n=12, seed=4):
    reqs = poisson_stream(n, rate=1e9, seed=seed, steps_range=(3, 12))
    for k, r in enumerate(reqs):
        r.desc.nx = min(r.desc.nx, 400)
        r.arrival = 0.0
    return reqs


def test_results_in_the_mix_equal_alone():
    reqs = _stream()
    # realtime=False with admit_every=2 and max_live=5: later requests are
    # admitted while earlier ones are mid-flight, and slots retire at
    # different steps
    srv = Server(params=SP, admit_every=2, max_live=5)
    out = srv.run(reqs, realtime=False)
    assert out["requests"] == len(reqs)
    assert out["rebuilds"] >= 2
    for r in reqs:
        got = out["results"][r.rid]["state"]
        ref = solve_alone(r, SP)
        assert torch.equal(got, ref), r.rid


def test_latency_and_throughput_reported():
    reqs = poisson_stream(6, rate=200.0, seed=1, steps_range=(5, 20))
    for r in reqs:
        r.desc.nx = min(r.desc.nx, 300)
    out = Server(params=SP).run(reqs)
    assert out["requests"] == 6
    assert 0.0 < out["p50_latency_s"] <= out["p99_latency_s"]
    assert out["updates_per_s"] > 0
