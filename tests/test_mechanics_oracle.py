"""The thermoelastic restatement (oracle/mechanics_oracle.py) checked for
what the elasticity operator must satisfy: symmetry, rigid-body modes in the
kernel of the unconstrained matrix, the patch test (a uniform strain field
leaves only boundary rows nonzero), and the exact thermal-expansion solution:
for a uniform temperature rise the field u = alpha dT (x - x0) satisfies
K u = rhs in every row (sigma = (3 lambda + 2 mu) alpha dT I), which ties the
operator and the right-hand side together; gravity's total force is
-rho g V."""
import numpy as np
import pytest

from mechanics_oracle import Elasticity, cells_with_displacement


def box(degree, nc=(3, 2, 2), extent=(6.0, 4.0, 3.0), clamped=0, lam=2.0, mu=3.0, alpha=1e-5, rho=7.9e3):
    C = int(np.prod(nc))
    return Elasticity(nc, extent, degree, range(C), np.zeros(C, int), [lam] * 4, [mu] * 4, [alpha] * 4,
                      [rho] * 4, clamped)


def coords(e):
    g = np.arange(e.n_nodes)
    i, j, k = e.node_ijk(g)
    return np.stack([i * e.h[0] / e.p, j * e.h[1] / e.p, k * e.h[2] / e.p], axis=1)


@pytest.mark.parametrize("degree", [1, 2])
def test_symmetric_with_rigid_body_kernel(degree):
    e = box(degree)
    K = e.matrix()
    assert np.abs(K - K.T).max() <= 1e-12 * np.abs(K).max()
    x = coords(e)
    n = e.n_nodes
    modes = []
    for c in range(3):
        t = np.zeros(3 * n)
        t[c * n:(c + 1) * n] = 1.0
        modes.append(t)
    for a, b in ((0, 1), (1, 2), (0, 2)):  # rotation in the (a, b) plane
        r = np.zeros(3 * n)
        r[a * n:(a + 1) * n] = -x[:, b]
        r[b * n:(b + 1) * n] = x[:, a]
        modes.append(r)
    for m in modes:
        assert np.abs(K @ m).max() <= 1e-11 * np.abs(K).max() * np.abs(m).max()


@pytest.mark.parametrize("degree", [1, 2])
def test_patch_test_interior_rows_vanish(degree):
    e = box(degree, nc=(3, 3, 3), extent=(3.0, 3.0, 3.0))
    x = coords(e)
    n = e.n_nodes
    E = np.array([[1.0, 0.3, -0.2], [0.1, -0.5, 0.4], [0.2, 0.0, 0.7]])
    u = (x @ E.T).T.reshape(-1)  # u_c = sum_d E[c, d] x_d
    r = e.matrix() @ u
    i, j, k = e.node_ijk(np.arange(n))
    interior = (i > 0) & (j > 0) & (k > 0) & (i < e.nn[0] - 1) & (j < e.nn[1] - 1) & (k < e.nn[2] - 1)
    for c in range(3):
        assert np.abs(r[c * n:(c + 1) * n][interior]).max() <= 1e-11 * np.abs(r).max()


@pytest.mark.parametrize("degree", [1, 2])
def test_uniform_heating_gives_free_thermal_expansion(degree):
    e = box(degree, alpha=1.2e-5)
    x = coords(e)
    dT, T0 = 150.0, 300.0
    u = (1.2e-5 * dT * x).T.reshape(-1)
    K = e.matrix()
    f = e.rhs(T=np.full(e.n_nodes, T0 + dT), initial_temperature=T0, gravity=False)
    assert np.abs(K @ u - f).max() <= 1e-10 * np.abs(f).max()


def test_gravity_total_force_and_melted_reference():
    e = box(2, rho=8000.0)
    f = e.rhs(T=None, thermoelastic=False, gravity=True)
    n = e.n_nodes
    assert abs(f[2 * n:].sum() + 8000.0 * 9.80665 * 6.0 * 4.0 * 3.0) <= 1e-9 * 8000 * 9.81 * 72
    assert np.abs(f[:2 * n]).max() == 0.0
    # melted cells expand from the material's reference temperature
    melted = np.zeros(12, np.uint8)
    melted[:6] = 1
    T = np.full(n, 500.0)
    a = e.rhs(T=T, melted=melted, reference_temperatures=[500.0] * 4, initial_temperature=300.0, gravity=False)
    b = Elasticity(e.nc, (6.0, 4.0, 3.0), 2, range(6, 12), np.zeros(12, int), [2.0] * 4, [3.0] * 4,
                   [1e-5] * 4).rhs(T=T, initial_temperature=300.0, gravity=False)
    assert np.allclose(a, b, rtol=0, atol=1e-12 * np.abs(b).max())


def test_cell_selection():
    assert cells_with_displacement([1, 1, 0, 1], [1.0, 0.5, 1.0, 0.995]) == [0, 3]


def test_j2_isotropic_return_lands_on_the_yield_surface():
    """Purely isotropic hardening (h = 1, no back stress): after a plastic
    step the deviatoric stress norm equals the updated plastic internal
    variable, kappa_new = kappa + H dgamma = |dev sigma|, at every point."""
    from mechanics_oracle import Elasticity, J2Points

    e = Elasticity((2, 1, 1), (2.0, 1.0, 1.0), 1, [0, 1], np.zeros(2, int), [2.0] * 4, [3.0] * 4)
    j = J2Points(e, 1.5, 1.0, 0.1)
    rng = np.random.default_rng(5)
    plastic = 0
    for _ in range(3):
        k0 = j.kappa.copy()
        j.update(rng.normal(size=3 * e.n_nodes) * 0.02)
        for c in range(2):
            for q in range(8):
                s = j._tensor(j.stress[:, c, q])
                dev = s - np.trace(s) / 3.0 * np.eye(3)
                nrm = np.sqrt(np.sum(dev * dev))
                assert (j.back[:, c, q] == 0.0).all()
                if j.kappa[c, q] > k0[c, q]:  # yielded in this step
                    plastic += 1
                    assert abs(nrm - j.kappa[c, q]) <= 1e-14 * j.kappa[c, q]
                else:  # elastic: inside the surface
                    assert nrm < j.kappa[c, q]
    assert plastic > 0


def test_j2_elastic_steps_add_up():
    """Below the elastic limit the stress is C : (sum of the strain
    increments): two increments give the stress of their sum."""
    from mechanics_oracle import Elasticity, J2Points

    e = Elasticity((1, 1, 2), (1.0, 1.0, 2.0), 2, [0, 1], np.zeros(2, int), [2.0] * 4, [3.0] * 4)
    a, b = J2Points(e, 1.5, 0.5, np.inf), J2Points(e, 1.5, 0.5, np.inf)
    rng = np.random.default_rng(6)
    d1, d2 = rng.normal(size=3 * e.n_nodes), rng.normal(size=3 * e.n_nodes)
    a.update(d1)
    a.update(d2)
    b.update(d1 + d2)
    assert np.abs(a.stress - b.stress).max() <= 1e-12 * np.abs(b.stress).max()
    assert np.isinf(a.kappa).all() and (a.back == 0.0).all()


def test_old_displacement_transfer_keeps_nodes_of_the_last_old_cell():
    """setup_dofs's write-back in cell order: a node shared by a cell that
    carried displacement and a later one that did not restarts from 0."""
    from mechanics_oracle import Elasticity, transfer_old_displacement

    e = Elasticity((3, 1, 1), (3.0, 1.0, 1.0), 1, [0, 1, 2], np.zeros(3, int), [2.0] * 4, [3.0] * 4)
    u = np.arange(3 * e.n_nodes, dtype=float) + 1.0
    prev = np.array([1, 0, 0], np.uint8)  # cell 0 carried displacement
    now = np.array([1, 1, 0], np.uint8)   # cell 1 starts carrying it
    out = transfer_old_displacement(e, prev, now, u)
    n = e.n_nodes
    for g in range(n):
        i = g % e.nn[0]
        want = 0.0 if i >= 1 else 1.0  # x = 1 is also cell 1's (written last): 0
        for comp in range(3):
            assert out[comp * n + g] == (u[comp * n + g] if want else 0.0), (g, comp)


@pytest.mark.parametrize("degree", [1, 2])
def test_j2_monotone_shear_matches_the_closed_form(degree):
    """Simple shear u_x = gamma y applied in increments, linear isotropic
    hardening (h = 1): the stress stays pure shear and, past the elastic
    limit kappa_0, |dev sigma| = kappa_0 + H (sqrt(2) mu gamma - kappa_0) /
    (2 mu + H), the closed form of the radial return under proportional
    loading (Simo and Hughes, Computational Inelasticity, sec. 3.3), for
    any split of the path into increments."""
    from mechanics_oracle import Elasticity, J2Points

    lam, mu, H, k0 = 2.0, 3.0, 1.5, 0.1
    e = Elasticity((1, 1, 1), (1.0, 1.0, 1.0), degree, [0], np.zeros(1, int), [lam] * 4, [mu] * 4)
    y = coords(e)[:, 1]
    n = e.n_nodes
    gamma_yield = k0 / (np.sqrt(2.0) * mu)
    for steps in (1, 3, 10):
        j = J2Points(e, H, 1.0, k0)
        gamma = 0.0
        for g in np.linspace(0.0, 5.0 * gamma_yield, steps + 1)[1:]:
            du = np.zeros(3 * n)
            du[:n] = (g - gamma) * y
            j.update(du)
            gamma = g
        expect = k0 + H * (np.sqrt(2.0) * mu * gamma - k0) / (2.0 * mu + H)
        for q in range(len(e.jxw)):
            s = j._tensor(j.stress[:, 0, q])
            assert abs(np.trace(s)) <= 1e-13 * expect
            assert abs(s[0, 1] * np.sqrt(2.0) - expect) <= 1e-12 * expect  # |dev sigma| = sqrt(2) sigma_xy
            assert abs(j.kappa[0, q] - expect) <= 1e-12 * expect
            assert abs(s[0, 0]) + abs(s[1, 1]) + abs(s[2, 2]) + abs(s[0, 2]) + abs(s[1, 2]) <= 1e-13 * expect
