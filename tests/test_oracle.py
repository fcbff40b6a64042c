"""CPU oracle: pinned against the reference's own stored results, and its invariants."""
import numpy as np
import pytest

import lbm3_b200 as L
import oracle as O
from helpers import load_golden


def test_oracle_tgv_matches_reference_energy_curve():
    """Re 1600 / Ma 0.1 / 128^3: the first three samples of the reference's
    stored energy history (every 10 steps) agree to ~1e-7 relative."""
    s = L.taylor_green(128)
    gold = load_golden("tgv_re1600_128_energy.txt")
    g = O.OracleGrid(s.case)
    got = [g.kinetic_energy(s.u_initial_phys, s.domain_length)]
    for _ in range(2):
        g.step(10)
        got.append(g.kinetic_energy(s.u_initial_phys, s.domain_length))
    g.close()
    for k, e in enumerate(got):
        t_star = s.time_star(10 * k)
        assert abs(t_star - gold[k, 0]) < 1e-6
        assert abs(e - gold[k, 1]) / gold[k, 1] < 5e-7, (k, e, gold[k, 1])


def _near_eq_populations(rng, n, amp=0.02):
    dRho = rng.uniform(-0.02, 0.02, n).astype(np.float32)
    u = rng.uniform(-0.08, 0.08, (3, n)).astype(np.float32)
    f = np.stack([O.feq(dRho[c], u[0, c], u[1, c], u[2, c]) for c in range(n)], axis=1)
    f = f + (amp * rng.standard_normal(f.shape) * np.abs(f).max(axis=0, keepdims=True) * 0.05)
    return f.astype(np.float32)


@pytest.mark.parametrize("limiter", [0.05, 0.0])
def test_collision_conserves_mass_and_momentum(limiter):
    rng = np.random.default_rng(1)
    f = _near_eq_populations(rng, 64)
    post = O.apply_collision_batch(f, nu=0.01, limiter=limiter)
    for c in range(f.shape[1]):
        a = O.drho_u(f[:, c])
        b = O.drho_u(post[:, c])
        assert abs(a[0] - b[0]) < 2e-7
        # the second half of the (zero) force flips nothing: momentum is kept
        assert np.allclose(a[1:] * (1 + a[0]), b[1:] * (1 + b[0]), atol=2e-7)


def test_equilibrium_is_a_fixed_point():
    rng = np.random.default_rng(2)
    for _ in range(20):
        dRho, ux, uy, uz = rng.uniform(-0.01, 0.01), *rng.uniform(-0.05, 0.05, 3)
        feq = O.feq(dRho, ux, uy, uz)
        for lim in (0.05, 0.0):
            post = O.apply_collision(feq, nu=0.02, limiter=lim)
            assert np.max(np.abs(post - feq)) < 2e-7


def test_collision_relaxes_shear_stress_at_rate_omega1():
    """A pure shear perturbation of the second-order moment decays by
    (1 - omega1) in one collision (AllOne, small amplitude)."""
    nu = 0.05
    omega1 = 1.0 / (3.0 * nu + 0.5)
    f = O.feq(0.0, 0.0, 0.0, 0.0).astype(np.float64)
    cx = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, 0, 0, -1, 1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1])
    cy = np.array([0, 0, 0, 0, 0, -1, 1, 0, 0, 0, 0, -1, 1, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1, -1, 1])
    w = np.array([8 / 27] + [2 / 27] * 6 + [1 / 54] * 12 + [1 / 216] * 8)
    eps = 1e-4
    f = (f + eps * w * cx * cy * 4.5).astype(np.float32)  # adds m_xy = eps
    mxy0 = float(np.sum(f.astype(np.float64) * cx * cy))
    post = O.apply_collision(f, nu=nu, limiter=0.0)
    mxy1 = float(np.sum(post.astype(np.float64) * cx * cy))
    assert abs(mxy1 - (1 - omega1) * mxy0) < 1e-7


def test_oracle_uniform_flow_stays_uniform():
    c = L.periodic_box(8, 6, 4, nu_lattice=0.02, ux=0.03, uy=-0.01, uz=0.02)
    g = O.OracleGrid(c)
    m0 = g.macro()
    g.step(5)
    m1 = g.macro()
    assert np.max(np.abs(m1 - m0)) < 1e-6
    g.close()


def test_section_image_of_one_level_equals_the_layer_sums():
    """On one level the section image holds exactly the cut layer's cells, so
    its sums equal the direct layer sums (crop included)."""
    import lbm3_b200 as L
    from lbm3_b200 import _abi as A
    c = L.open_channel(24, 12, 10, u_in=0.04, nu_lattice=0.02)
    d = O.OracleDomain(c)
    o = O.OracleGrid(c)
    d.step(3)
    o.step(3)
    p = L.Plan(c)
    info = p.info()
    bounds = (0.3, 2.8, 1.8, 23.7, 9.2, 7.2)
    for plane, cut in ((A.PLANE_ZY, 8.5), (A.PLANE_XY, 4.5), (A.PLANE_ZX, 6.5)):
        t, level = d.flow_image(plane, cut, bounds)
        assert level == 0
        axis = {A.PLANE_XY: 2, A.PLANE_ZY: 0, A.PLANE_ZX: 1}[plane]
        o_ = (info.ox, info.oy, info.oz)
        n = (info.cell_count_x, info.cell_count_y, info.cell_count_z)
        layer = int(np.float32((cut - o_[axis]) / info.res + 0.5))
        lo, hi = [], []
        for a in range(3):
            t_min = np.float32(o_[a] - 0.5 * info.res)
            t_max = np.float32(o_[a] + info.res * (n[a] - 0.5))
            lo.append(max(0, int(np.ceil(np.float32((bounds[a] - t_min) / info.res)))))
            hi.append(min(n[a], n[a] - int(np.ceil(np.float32((t_max - bounds[a + 3]) / info.res)))))
        ha, va = (0 if plane == A.PLANE_XY else 2), (0 if plane == A.PLANE_ZX else 1)
        ref = o.flow_sums(plane, layer, lo[ha], hi[ha], lo[va], hi[va])
        np.testing.assert_allclose(t, ref, rtol=1e-12, atol=1e-12)
    o.close()
