"""Multilevel time step on the GPU against the oracle: the recursive
substep schedule (updateAllGrids, include/updateGrid.h:388-396) with the
fine-to-coarse, coarse-to-fine and leftover interface updates
(include/updateInterface.h:155-891) after every fine pair, on grids the
oracle builds itself; and the reference's stored kinetic-energy history of
its refined Taylor-Green run."""
import numpy as np
import pytest

import lbm3_b200 as L
import oracle as O
from lbm3_b200 import geometry as G
from helpers import FIELD_REL_L2, density_velocity_errors, field_errors, load_golden

from test_multilevel import slab_channel_refined

pytestmark = pytest.mark.gpu


def compare_levels(g, d, near_rest=False):
    """Max field error over the levels (fluid cells only)."""
    worst = 0.0
    for l in range(d.level_count):
        o = d.level(l)
        fl = o.int_array("wallMap") != -3
        gm, om = g.macro(l)[:, fl], o.macro()[:, fl]
        if near_rest:
            e_rho, e_u, d_rho = density_velocity_errors(gm, om)
            assert d_rho < 1e-6, (l, d_rho)
        else:
            e_rho, e_u = field_errors(gm, om)
        assert e_rho < FIELD_REL_L2 and e_u < FIELD_REL_L2, (l, e_rho, e_u)
        worst = max(worst, e_rho, e_u)
    return worst


def test_refined_taylor_green_matches_oracle():
    s = L.taylor_green_refined(32)
    d = O.OracleDomain(s.case)
    with L.build_grids(s.case) as g:
        assert g.level_count() == 2
        for _ in range(4):
            g.update_all_grids(10)
            d.step(10)
        compare_levels(g, d)
        eg = g.kinetic_energy(s.u_initial_phys, s.domain_length)
        eo = d.kinetic_energy(s.u_initial_phys, s.domain_length)
        assert abs(eg - eo) / eo < 2 * FIELD_REL_L2, (eg, eo)
        assert g.info(1).iterations_finished == 80
    d.close()


def test_three_levels_match_oracle():
    """Taylor-Green initial field on three levels from a refinement hook."""
    s = L.taylor_green(32)
    c = s.case
    c.grid_level_count = 3
    q = float(s.domain_length)

    def refine(i, j, k, mark, info):
        x, y, z = i * info.res + info.ox, j * info.res + info.oy, k * info.res + info.oz
        h = 0.27 * q if info.grid_id == 0 else 0.13 * q
        return mark or (abs(x + 0.05 * q) < h and abs(y) < h and abs(z - 0.03 * q) < h)
    L.set_hooks(c, refinement=refine)
    d = O.OracleDomain(c)
    with L.build_grids(c) as g:
        assert g.level_count() == 3
        g.update_all_grids(12)
        d.step(12)
        compare_levels(g, d)
    d.close()


def test_refined_slab_channel_with_leftovers_matches_oracle():
    """Body-force channel whose refined block ends across the walls:
    leftover fine cells with the wall-side quadratic velocity."""
    c = slab_channel_refined()
    d = O.OracleDomain(c)
    with L.build_grids(c) as g:
        assert g.info(0).leftover_count > 0
        g.update_all_grids(60)
        d.step(60)
        compare_levels(g, d, near_rest=True)
    d.close()


def test_refined_sphere_channel_matches_oracle():
    """Open channel with a sphere refined by its walls and a refinement box:
    open boundaries on level 0, the body on level 1; fields and the drag
    force.  AllOne collision (limiter 0), as the reference's wall drivers
    use: at this resolution (D = 8 fine cells) K17 with a limiter makes the
    flow unstable within 20 steps on the GPU and in the oracle alike, and
    the two then diverge as any two roundings of an unstable run do."""
    c = L.open_channel(48, 24, 24, u_in=0.04, nu_lattice=0.02, collision_limiter=0.0)
    G.set_bodies(c, [G.icosphere(2, 4.0, (16.0, 12.0, 12.0))])
    L.set_refine_box(c, 0, (8.0, 4.0, 4.0), (26.0, 20.0, 20.0))
    c.grid_level_count = 2
    c.wall_refinement_count = 2
    c.track_wall_force = 1
    d = O.OracleDomain(c)
    steps = 40
    with L.build_grids(c) as g:
        g.update_all_grids(steps)
        d.step(steps)
        compare_levels(g, d, near_rest=True)
        info = g.info(1)
        dx = info.res / 1000.0
        to_si = c.rho_phys * dx ** 4 / info.dt_phys ** 2
        drag_gpu = g.wall_force(0)[0]
        drag_oracle = d.level(1).wall_force(0)[0] / (2 * steps) * to_si
        assert drag_gpu == pytest.approx(drag_oracle, rel=1e-4), (drag_gpu, drag_oracle)
    d.close()


def test_multilevel_sphere_configuration_matches_oracle():
    """The multilevel sphere configuration at its size (base 128x64x64, three
    levels, D = 48 finest cells, Re 300; AllOne on level 0 and K17 with
    limiter 0.1 on the finer levels, as the reference's sphere driver):
    10 coarse steps (40 finest substeps), fields on every level and the drag."""
    from lbm3_b200.cases import multilevel_sphere
    s = multilevel_sphere()
    c = s.case
    d = O.OracleDomain(c)
    steps = 10
    with L.build_grids(c) as g:
        assert g.level_count() == 3
        g.update_all_grids(steps)
        d.step(steps)
        compare_levels(g, d, near_rest=True)
        drag_gpu = g.wall_force(0)[0]
        drag_oracle = 0.0
        for l in range(3):
            info = g.info(l)
            dx = info.res / 1000.0
            to_si = c.rho_phys * dx ** 4 / info.dt_phys ** 2
            drag_oracle += d.level(l).wall_force(0)[0] / (steps << l) * to_si
        assert drag_gpu == pytest.approx(drag_oracle, rel=1e-4), (drag_gpu, drag_oracle)
    d.close()


def test_graph_replay_of_the_substep_schedule_is_identical():
    """Step pairs replayed from a captured CUDA graph of the whole substep
    schedule give the same populations as launching every kernel."""
    s = L.taylor_green_refined(32)
    with L.build_grids(s.case) as a, L.build_grids(s.case) as b:
        b.set_graphs(False)
        a.update_all_grids(20)
        b.update_all_grids(20)
        for l in range(2):
            np.testing.assert_array_equal(a.populations(l), b.populations(l))


def test_refined_taylor_green_reproduces_the_reference_curve():
    """Re 1600, Ma 0.1, 128^3 with the central cube refined (the reference's
    QUADRATIC run, 7057 coarse steps): the GPU's kinetic-energy history
    against the reference's stored one."""
    s = L.taylor_green_refined(128)
    gold = load_golden("tgv_re1600_128_refined_energy.txt")
    with L.build_grids(s.case) as g:
        energies = [g.kinetic_energy(s.u_initial_phys, s.domain_length)]
        done = 0
        while done < s.iteration_count:
            step = min(10, s.iteration_count - done)
            g.update_all_grids(step)
            done += step
            energies.append(g.kinetic_energy(s.u_initial_phys, s.domain_length))
    e = np.array(energies)
    assert len(e) == len(gold)
    rel = np.abs(e - gold[:, 1]) / gold[:, 1]
    print(f"refined TGV: max rel {rel.max():.3e} (first 50: {rel[:50].max():.3e}), at t*={gold[rel.argmax(), 0]:.2f}")
    assert rel[:50].max() < 1e-4, rel[:50].max()
    assert rel.max() < 5e-3, rel.max()
