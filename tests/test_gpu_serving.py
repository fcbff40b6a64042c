"""The serving loop: requests that arrive while others run are admitted by
footprint and batched, and each result is the same as the request run alone."""
import numpy as np
import pytest

import lbm3_b200 as L
from lbm3_b200 import serving as S
from helpers import rel_l2

pytestmark = pytest.mark.gpu


def requests():
    rng = np.random.default_rng(7)
    edges, steps, arrivals = [16, 16, 24, 16, 24], [60, 120, 90, 150, 60], [0.0, 0.0, 0.02, 0.05, 0.3]
    return [S.channel_request(q, e, rng, n, arrival=a) for q, (e, n, a) in enumerate(zip(edges, steps, arrivals))]


def test_results_in_the_mix_equal_results_alone():
    reqs = requests()
    # budget for about two domains at a time, at most three slots
    budget = int(2.5 * max(L.Plan(r.case).info().grid_memory_bytes for r in reqs))
    server = S.Server(hbm_budget=budget, max_slots=3, chunk_steps=40, keep_fields=True)
    results = {r.rid: r for r in server.run(reqs)}
    assert sorted(results) == [r.rid for r in reqs]
    for req in requests():
        # the request served alone: bit-identical fields; per-cell forces are
        # identical and their FP64 total is summed with atomics, so only its
        # last bits may depend on ordering
        alone, = S.Server(hbm_budget=budget, max_slots=1, chunk_steps=40, keep_fields=True).run([req])
        np.testing.assert_array_equal(alone.macro, results[req.rid].macro)
        fa, fb = alone.force, results[req.rid].force
        np.testing.assert_allclose(fa, fb, rtol=1e-12, atol=1e-12 * np.abs(fa).max())
        # and the plain stepping path, to the FP16 storage's rounding
        with L.build_grids(req.case) as g:
            g.update_all_grids(req.steps)
            m = g.macro()
            assert rel_l2(m[1:4].reshape(-1), results[req.rid].macro[1:4].reshape(-1)) < 1e-3
            fr = g.wall_force(0)
            assert np.abs(fr - fb).max() <= 1e-3 * np.abs(fr).max()
    # requests wait for memory, not only for slots
    admitted = sorted((r.admitted, r.finished) for r in results.values())
    overlap = max(sum(1 for a, f in admitted if a <= t < f) for t, _ in admitted)
    assert 2 <= overlap <= 3
    summary = S.summarize(list(results.values()), max(r.finished for r in results.values()))
    assert summary["requests"] == 5 and summary["p99_s"] >= summary["p50_s"] > 0


def test_energy_result_and_builds_off_the_stepping_thread():
    """A request with wall_id -1 returns its kinetic energy, equal to the
    request run alone; grids are built on builder threads."""
    rng = np.random.default_rng(3)
    reqs = [S.channel_request(q, 16, rng, 50 + 10 * q, arrival=0.01 * q) for q in range(4)]
    for r in reqs:
        r.wall_id = -1
    server = S.Server(hbm_budget=1 << 34, max_slots=4, chunk_steps=25, builders=2)
    results = {r.rid: r for r in server.run(reqs)}
    for req in reqs:
        alone, = S.Server(hbm_budget=1 << 34, max_slots=1, chunk_steps=25).run([req])
        assert results[req.rid].force is None
        # FP64 block partials are summed with atomics: equal up to ordering
        assert results[req.rid].energy == pytest.approx(alone.energy, rel=1e-12)
        with L.build_grids(req.case) as g:
            g.update_all_grids(req.steps)
            assert results[req.rid].energy == pytest.approx(g.kinetic_energy(*req.energy_ref), rel=1e-4)


def test_request_larger_than_the_budget_is_rejected():
    req = requests()[2]
    server = S.Server(hbm_budget=1000, max_slots=2)
    with pytest.raises(ValueError):
        server.run([req])
