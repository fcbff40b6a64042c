"""CUDA-graph replay of the step schedule gives the same state as launching
every kernel: fields, open-boundary reference values and tracked sums, wall
forces, for even and odd step counts, single domains and batches."""
import numpy as np
import pytest

import lbm3_b200 as L
from lbm3_b200 import geometry as G

pytestmark = pytest.mark.gpu


def channel():
    c = L.open_channel(48, 24, 24, u_in=0.04, nu_lattice=0.02)
    G.set_bodies(c, [G.icosphere(3, 4.0, (16.0, 12.0, 12.0))])
    c.track_wall_force = 1
    c.track_open_boundaries = 1
    return c


def run(graphs: bool, steps_list):
    with L.build_grids(channel()) as g:
        g.set_graphs(graphs)
        for n in steps_list:
            g.update_all_grids(n)
        g.synchronize()
        info = g.info()
        return (g.macro(), g.open_reference(), g.open_cumulative(), g.wall_force(0), info.iterations_finished,
                info.esotwist_flipper)


@pytest.mark.parametrize("steps_list", [[10], [7, 4, 1]])
def test_graph_replay_equals_direct_launches(steps_list):
    a, b = run(True, steps_list), run(False, steps_list)
    for x, y in zip(a[:3], b[:3]):
        np.testing.assert_array_equal(x, y)
    # FP64 totals of per-cell forces are summed with atomics
    np.testing.assert_allclose(a[3], b[3], rtol=1e-12, atol=1e-12 * np.abs(b[3]).max())
    assert a[4:] == b[4:]


def test_graph_timing_runs_whole_steps():
    with L.build_grids(channel()) as g:
        g.update_all_grids(2)
        ms = g.time_steps_graph(20)
        assert ms > 0
        assert g.info().iterations_finished == 22


def test_batch_with_graphs_equals_domains_alone():
    cases = [channel() for _ in range(3)]
    grids = [L.build_grids(c) for c in cases]
    import torch
    streams = [torch.cuda.Stream() for _ in grids]
    for g, s in zip(grids, streams):
        g.set_stream(s.cuda_stream)
    L.update_batch(grids, 9)
    for g in grids:
        g.synchronize()
    ref = run(False, [9])
    for g in grids:
        np.testing.assert_array_equal(g.macro(), ref[0])
        g.close()
