"""Thermoelastic displacement on the GPU (through the C ABI) against the dense
restatement (oracle/mechanics_oracle.py): the elasticity operator of the
reference's own operator test (3 x 3 x 3 FE_Q(2)^3 cells of a 6 m cube,
lambda = 2, mu = 3, boundary id 0 clamped: tests/test_mechanical_operator.cc
:49-256) on free rows and the identity on clamped rows; the thermoelastic
right-hand side from a GPU temperature field with melted and liquid cells
(the liquid ones carry no displacement, melted ones expand from the
material's reference temperature); and the CG displacement against the
dense solve."""
import numpy as np
import pytest
import torch

from amr_cases import amr_test_config
from mechanics_oracle import Elasticity, cells_with_displacement

from adamantine_b200.config import Boundary, Geometry, ThermalConfig
from adamantine_b200.mechanics import MechanicalPhysics
from adamantine_b200.thermal import ThermalPhysics

pytestmark = pytest.mark.gpu


def plain(phys, v):
    """(3 m) device displacement -> (3 n_nodes) plain-grid numpy vector."""
    nx, ny, nz = phys.nodes
    a = v.detach().cpu().numpy().reshape(3, nz, ny, phys.pitch)[:, :, :, :nx]
    return np.ascontiguousarray(a).reshape(-1)


def padded(phys, u):
    nx, ny, nz = phys.nodes
    full = np.zeros((3, nz, ny, phys.pitch))
    full[:, :, :, :nx] = np.asarray(u).reshape(3, nz, ny, nx)
    return torch.tensor(full.reshape(-1), device=phys.device)


def reference_cube(degree):
    cfg = amr_test_config(degree=degree, n_cells=(3, 3, 3), n_states=1)
    cfg.geometry = Geometry(dim=3, n_cells=(3, 3, 3), extent=(6.0, 6.0, 6.0))
    cfg.sources = []
    return cfg


@pytest.mark.parametrize("degree", [1, 2])
def test_elastostatic_operator_matches_textbook_assembly(degree):
    cfg = reference_cube(degree)
    phys = ThermalPhysics(cfg)
    mech = MechanicalPhysics(phys, 2.0, 3.0, density=1.0, thermoelastic=False, gravity=True, clamped=("x-",))
    mech.setup_dofs()
    C = 27
    e = Elasticity((3, 3, 3), (6.0, 6.0, 6.0), degree, range(C), np.zeros(C, int), [2.0] * 4, [3.0] * 4,
                   density=[1.0] * 4, clamped_faces=1)
    assert (mech.node_mask() .reshape(phys.nodes[2], phys.nodes[1], phys.pitch)[:, :, :phys.nodes[0]]
            .reshape(-1) == e.mask).all()
    assert mech.n_dofs == 3 * e.n_nodes and mech.n_cells == C
    K = e.matrix()
    fr = e.free()
    cl = np.concatenate([c * e.n_nodes + np.nonzero(e.mask == 2)[0] for c in range(3)])
    rng = np.random.default_rng(4)
    for _ in range(3):
        x = rng.normal(size=3 * e.n_nodes)
        dst = mech.new_vector()
        mech.vmult(dst, padded(phys, x))
        y = plain(phys, dst)
        xf = np.zeros_like(x)
        xf[fr] = x[fr]
        ref = K @ xf
        assert np.abs(y[fr] - ref[fr]).max() <= 1e-12 * np.abs(ref[fr]).max()
        assert (y[cl] == x[cl]).all()
    f = plain(phys, mech.rhs())
    fo = e.rhs(thermoelastic=False, gravity=True)
    fo[cl] = 0.0
    assert np.abs(f - fo).max() <= 1e-12 * np.abs(fo).max()
    u = mech.solve()
    uo = e.solve(K, e.rhs(thermoelastic=False, gravity=True))
    assert np.abs(plain(phys, u) - uo).max() <= 1e-8 * np.abs(uo).max()
    assert mech.residual <= 1e-12 * np.linalg.norm(fo) * 1.0001


def test_thermoelastic_after_a_melting_beam():
    cfg = amr_test_config(degree=2, n_cells=(6, 6, 2), boundary="adiabatic", max_power=40000.0)
    phys = ThermalPhysics(cfg)
    T = phys.from_grid(np.full(tuple(reversed(cfg.geometry.node_shape(2))), 300.0))
    t = 0.0
    for _ in range(40):
        t = phys.evolve_one_time_step(t, 2e-6, T)
    # flag the cells heated along the path (the flag compares the cell
    # average, far below the peak on these 0.8 mm cells), so that solid
    # cells expand from the material's reference temperature
    melted = phys.mark_has_melted(320.0, T)
    phys.set_state_to_material_properties()
    st = phys.get_cell_state()
    active = cfg.geometry.active_cells()
    cells = cells_with_displacement(active, st[0])
    assert 0 < len(cells) < phys.n_cells  # liquid cells are left out
    assert melted[cells].any() and not melted[cells].all()
    lam, mu, alpha, rho = 1.1e11, 7.9e10, 1.6e-5, 7904.0
    mech = MechanicalPhysics(phys, lam, mu, alpha, rho, reference_temperatures=[1673.0], initial_temperature=300.0,
                             clamped=("z-",))
    mech.setup_dofs(T)
    e = Elasticity(cfg.geometry.n_cells, cfg.geometry.extent, 2, cells, np.zeros(phys.n_cells, int), [lam] * 4,
                   [mu] * 4, [alpha] * 4, [rho] * 4, clamped_faces=1 << 4)
    Tg = phys.to_grid(T).reshape(-1)
    f = e.rhs(T=Tg, melted=melted, reference_temperatures=[1673.0] * 4, initial_temperature=300.0)
    fr = e.free()
    fg = plain(phys, mech.rhs())
    assert np.abs(fg[fr] - f[fr]).max() <= 1e-11 * np.abs(f[fr]).max()
    K = e.matrix()
    u = mech.solve()
    uo = e.solve(K, f)
    assert np.abs(plain(phys, u) - uo).max() <= 1e-7 * np.abs(uo).max()
    assert mech.iterations > 0 and np.abs(uo).max() > 0.0


def test_eshelby_inclusion_matches_reference_values():
    """The reference's thermoelastic_eshelby case (test_mechanical_physics.cc
    :343-557): a 40 um cube clamped on boundary 4 (z-), K = 160 GPa,
    G = 79 GPa, alpha = 0.01, the temperature 3 inside a 1 um sphere at the
    centre and 2 (the reference temperature) outside, FE_Q(1); the
    displacement at two points against the reference's expected values
    (the analytic inclusion solution) with its 16 % tolerance. The reference
    refines the mesh around the inclusion to 0.31 um cells; here the whole
    cube is 128^3 cells of that size."""
    n, L, a = 128, 4.0e-5, 1.0e-6
    cfg = amr_test_config(degree=1, n_cells=(n, n, n), n_states=1)
    cfg.geometry = Geometry(dim=3, n_cells=(n, n, n), extent=(L, L, L))
    cfg.sources = []
    phys = ThermalPhysics(cfg)
    x = np.linspace(0.0, L, n + 1)
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    dist = np.sqrt((X - 2e-5) ** 2 + (Y - 2e-5) ** 2 + (Z - 2e-5) ** 2)
    T = phys.from_grid(np.where(dist < a, 3.0, 2.0))
    K, G = 160.0e9, 79.0e9
    mech = MechanicalPhysics(phys, K - 2.0 / 3.0 * G, G, 0.01, reference_temperatures=[2.0],
                             initial_temperature=2.0, gravity=False, clamped=("z-",), rel_tol=1e-10)
    mech.setup_dofs(T)
    u = plain(phys, mech.solve()).reshape(3, n + 1, n + 1, n + 1)
    h = L / n

    def point_value(p):
        idx = [min(int(p[d] / h), n - 1) for d in range(3)]
        t = [p[d] / h - idx[d] for d in range(3)]
        out = np.zeros(3)
        for c in range(8):
            o = (c & 1, (c >> 1) & 1, c >> 2)
            w = np.prod([t[d] if o[d] else 1.0 - t[d] for d in range(3)])
            out += w * u[:, idx[2] + o[2], idx[1] + o[1], idx[0] + o[0]]
        return out

    for p, ref in (((2.08e-5, 2.0e-5, 2.0e-5), (4.8241206e-09, 0.0, 0.0)),
                   ((2.3e-5, 2.2e-5, 1.9e-5), (3.45348338e-10, 2.30232226e-10, -1.15116113e-10))):
        v = point_value(p)
        print("eshelby", p, v, "relative deviation", [abs(v[i] - ref[i]) / abs(ref[i]) for i in range(3) if ref[i]])
        for i in range(3):
            if ref[i] == 0.0:
                assert abs(v[i]) <= 0.16 * abs(ref[0] if ref[0] else 1e-9)
            else:
                assert abs(v[i] - ref[i]) <= 0.16 * abs(ref[i]), (p, i, v[i], ref[i])


def test_elastostatic_physics_case():
    """The reference's MechanicalPhysics elastostatic case
    (test_mechanical_physics.cc:196-264): 6 x 3 x 3 FE_Q(1)^3 cells over
    12 x 6 x 6 m, density 1, lambda = 2, mu = 3, boundary 4 (z-) clamped,
    gravity; its check is against a textbook CG solve with 2e-9 absolute
    tolerance, here against the dense solve of the restatement."""
    cfg = amr_test_config(degree=1, n_cells=(6, 3, 3), n_states=1)
    cfg.geometry = Geometry(dim=3, n_cells=(6, 3, 3), extent=(12.0, 6.0, 6.0))
    cfg.sources = []
    phys = ThermalPhysics(cfg)
    mech = MechanicalPhysics(phys, 2.0, 3.0, density=1.0, thermoelastic=False, gravity=True, clamped=("z-",))
    mech.setup_dofs()
    e = Elasticity((6, 3, 3), (12.0, 6.0, 6.0), 1, range(54), np.zeros(54, int), [2.0] * 4, [3.0] * 4,
                   density=[1.0] * 4, clamped_faces=1 << 4)
    uo = e.solve(e.matrix(), e.rhs(thermoelastic=False, gravity=True))
    u = plain(phys, mech.solve())
    assert np.abs(u - uo).max() <= 2e-9
    assert np.abs(uo).max() > 1.0  # O(1) and larger displacements, as the reference notes


def test_handles_of_different_degrees_coexist():
    """A FE_Q(1) and a FE_Q(2) handle alive on one device, their operator
    applications and solves interleaved, give the results each gives alone
    (the reference-element tables belong to the handle)."""
    def make(degree):
        phys = ThermalPhysics(reference_cube(degree))
        mech = MechanicalPhysics(phys, 2.0, 3.0, density=1.0, thermoelastic=False, gravity=True,
                                 clamped=("x-",))
        mech.setup_dofs()
        return phys, mech

    rng = np.random.default_rng(11)
    alone = {}
    for degree in (1, 2):
        phys, mech = make(degree)
        x = torch.tensor(rng.uniform(-1, 1, 3 * phys.m()), device=phys.device)
        dst = mech.new_vector()
        mech.vmult(dst, x)
        alone[degree] = (x, dst.clone(), mech.solve().clone())
        del mech, phys
    p1, m1 = make(1)
    p2, m2 = make(2)
    d1, d2 = m1.new_vector(), m2.new_vector()

    def close(a, b, tol):
        return float((a - b).abs().max() / b.abs().max()) <= tol

    # the operator adds with atomics (rounding order varies): 1e-13; the
    # CG solve: 1e-10 (a swapped table would be off by O(1))
    for _ in range(2):
        d1.zero_()
        d2.zero_()
        m1.vmult(d1, alone[1][0])
        m2.vmult(d2, alone[2][0])
        assert close(d1, alone[1][1], 1e-13) and close(d2, alone[2][1], 1e-13)
        u2 = m2.solve()
        u1 = m1.solve()
        assert close(u1, alone[1][2], 1e-10) and close(u2, alone[2][2], 1e-10)


def elastoplastic_box(degree, material_height=1e9):
    """The reference's elastoplastic case (tests/test_mechanical_physics.cc
    :559-617): a 12 x 6 x 6 box of 6 x 3 x 3 cells, one solid material."""
    cfg = amr_test_config(degree=degree, n_cells=(6, 3, 3), n_states=1)
    cfg.geometry = Geometry(dim=3, n_cells=(6, 3, 3), extent=(12.0, 6.0, 6.0), material_height=material_height)
    cfg.sources = []
    return cfg


J2_PARAMS = dict(plastic_modulus=1.5, isotropic_hardening=0.5, elastic_limit=0.1)


def assert_state_matches(mech, j):
    from mechanics_oracle import J2Points  # noqa: F401  (the oracle's state j)

    s, b, k = (x.cpu().numpy() for x in mech.stress_state())
    for got, ref in ((s, j.stress), (b, j.back)):
        scale = max(np.abs(ref).max(), 1e-300)
        assert np.abs(got - ref).max() <= 1e-11 * scale
    fin = np.isfinite(j.kappa)
    assert (np.isfinite(k) == fin).all()
    assert np.abs(k[fin] - j.kappa[fin]).max() <= 1e-11 * np.abs(j.kappa[fin]).max()


@pytest.mark.parametrize("degree", [1, 2])
def test_elastoplastic_stress_matches_the_j2_restatement(degree):
    """Gravity on the clamped box (lambda = 2, mu = 3, rho = 1, plastic
    modulus 1.5, isotropic hardening 0.5, elastic limit 0.1): after the CG
    solve the stress, back stress and plastic internal variable at every
    Gauss point equal the restatement's update from the same displacement
    (plastic almost everywhere), and a second identical solve (increment 0)
    updates both the same way."""
    from mechanics_oracle import Elasticity, J2Points

    cfg = elastoplastic_box(degree)
    phys = ThermalPhysics(cfg)
    mech = MechanicalPhysics(phys, 2.0, 3.0, density=1.0, thermoelastic=False, gravity=True, clamped=("z-",),
                             **J2_PARAMS)
    C = phys.n_cells
    e = Elasticity((6, 3, 3), (12.0, 6.0, 6.0), degree, range(C), np.zeros(C, int), [2.0] * 4, [3.0] * 4,
                   density=[1.0] * 4, clamped_faces=1 << 4)
    j = J2Points(e, **J2_PARAMS)
    u_prev = np.zeros(3 * e.n_nodes)
    for _ in range(2):
        mech.setup_dofs()
        u = plain(phys, mech.solve())
        j.update(u - u_prev)
        u_prev = u
        assert_state_matches(mech, j)
    assert (j.kappa > 0.1).mean() > 0.5  # the plastic branch is exercised


def test_cells_that_start_carrying_displacement():
    """The box with its top layer inactive, solved; the layer added, solved
    again: the new cells start from the elastic limit and zero stresses, and
    the displacement increment uses the previous displacement as setup_dofs
    carries it over (the nodes the new layer shares with the old one restart
    from 0, the new cells coming later in cell order)."""
    from mechanics_oracle import Elasticity, J2Points, transfer_old_displacement

    cfg = elastoplastic_box(1, material_height=4.0)
    phys = ThermalPhysics(cfg)
    T = phys.initialize_dof_vector(300.0)
    mech = MechanicalPhysics(phys, 2.0, 3.0, density=1.0, thermoelastic=False, gravity=True, clamped=("z-",),
                             **J2_PARAMS)
    C = phys.n_cells
    active1 = phys.active_cells().astype(bool)
    assert 0 < active1.sum() < C

    def elasticity(active):
        return Elasticity((6, 3, 3), (12.0, 6.0, 6.0), 1, np.nonzero(active)[0], np.zeros(C, int), [2.0] * 4,
                          [3.0] * 4, density=[1.0] * 4, clamped_faces=1 << 4)

    e1 = elasticity(active1)
    j = J2Points(e1, **J2_PARAMS)
    mech.setup_dofs()
    u1 = plain(phys, mech.solve())
    j.update(u1)
    assert_state_matches(mech, j)
    new = np.nonzero(~active1)[0]
    phys.add_material(new, 300.0, T)
    active2 = phys.active_cells().astype(bool)
    assert active2.all()
    mech.setup_dofs()
    u2 = plain(phys, mech.solve())
    e2 = elasticity(active2)
    u_old = transfer_old_displacement(e2, active1.astype(np.uint8), active2.astype(np.uint8), u1)
    assert (u_old != u1).any()  # the shared nodes restarted from 0
    j.e = e2
    j.start(new)
    j.update(u2 - u_old)
    assert_state_matches(mech, j)


@pytest.mark.parametrize("degree,n_cells", [(1, (32, 32, 8)), (2, (16, 16, 4))])
def test_multigrid_and_jacobi_preconditioners_give_the_same_displacement(degree, n_cells):
    """The multigrid-preconditioned CG (the default) against the
    Jacobi-preconditioned one on a thermoelastic problem whose liquid cells
    carry no displacement: the same displacement to the solver tolerance,
    in a fraction of the iterations, over a hierarchy of several levels."""
    cfg = amr_test_config(degree=degree, n_cells=n_cells, boundary="adiabatic", max_power=40000.0)
    phys = ThermalPhysics(cfg)
    T = phys.from_grid(np.full(tuple(reversed(cfg.geometry.node_shape(degree))), 300.0))
    t = 0.0
    for _ in range(40):
        t = phys.evolve_one_time_step(t, 2e-6, T)
    phys.mark_has_melted(320.0, T)
    mech = MechanicalPhysics(phys, 1.1e11, 7.9e10, 1.6e-5, 7904.0, reference_temperatures=[1673.0],
                             initial_temperature=300.0, clamped=("z-",))
    mech.setup_dofs(T)
    assert 0 < mech.n_cells < phys.n_cells
    u_mg = plain(phys, mech.solve())
    it_mg, res_mg = mech.iterations, mech.residual
    levels, coarse = mech.multigrid_levels()
    mech.set_preconditioner("jacobi")
    u_j = plain(phys, mech.solve())
    it_j = mech.iterations
    f = np.linalg.norm(plain(phys, mech.rhs()))
    assert res_mg <= 1e-12 * f * 1.0001
    assert levels >= 3 and 0 < coarse <= 640
    assert it_mg * 4 <= it_j, (it_mg, it_j)
    assert np.abs(u_mg - u_j).max() <= 1e-9 * np.abs(u_j).max()
