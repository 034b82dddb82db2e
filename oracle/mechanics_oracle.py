"""Thermoelastic restatement -- TEST INFRASTRUCTURE ONLY (tests/ import it as
the checker; nothing in the package uses it).

Dense assembly, on a box mesh, of the isotropic elasticity matrix exactly as
the reference's own test states it (tests/test_mechanical_operator.cc:170-
205: per cell, K(i, j) += (d_ci phi_i d_cj phi_j lambda + d_cj phi_i d_ci
phi_j mu + [ci == cj] grad phi_i . grad phi_j mu) JxW over QGauss(p + 1)),
of the right-hand side of MechanicalOperator::assemble_rhs
(source/MechanicalOperator.cc:354-476: (3 lambda + 2 mu) alpha (T - T_ref)
div phi_i + f . phi_i, f = (0, 0, -rho g)), the cell selection of
MechanicalPhysics::setup_dofs (solid ratio > 0.99 among the thermally
active cells) and the zero displacement on clamped box faces, solved by a
dense direct solve; and the J2 stress update after a solve with the state
carried over when the cells change (J2Points, transfer_old_displacement).
Small meshes only.

The elastic part is pinned to the reference's operator and Eshelby tests.
The J2 part has no reference pin (parity unpinned against the reference):
its own elastoplastic test (tests/test_mechanical_physics.cc:559-617)
computes the stress but checks nothing. The restatement follows
compute_stress line by line; its isotropic case is checked against the
closed form of monotone simple shear with linear isotropic hardening and
the yield-surface consistency of the return (the kinematic update as the
reference writes it has no closed form to check against).

Vectors are component-major over the plain node grid: index c * n_nodes +
node, node = i + nn0 (j + nn1 k).
"""
from __future__ import annotations

import numpy as np

G = 9.80665


def basis_1d(p: int):
    """Gauss points / weights on [0, 1] and the Lagrange basis on the
    equidistant nodes (values and derivatives at the points), from the
    monomial coefficients of each basis function."""
    xg, wg = np.polynomial.legendre.leggauss(p + 1)
    x, w = 0.5 * (xg + 1.0), 0.5 * wg
    nodes = np.linspace(0.0, 1.0, p + 1)
    V = np.vander(nodes, p + 1, increasing=True)
    coef = np.linalg.solve(V, np.eye(p + 1))  # column a: coefficients of phi_a
    P = np.vander(x, p + 1, increasing=True)
    dP = np.zeros_like(P)
    for k in range(1, p + 1):
        dP[:, k] = k * x ** (k - 1)
    return x, w, P @ coef, dP @ coef  # val[q, a], der[q, a]


class Elasticity:
    def __init__(self, n_cells, extent, degree, cells, matid, lame_first, lame_second, thermal_expansion=None,
                 density=None, clamped_faces=0):
        self.nc = tuple(int(n) for n in n_cells)
        self.p = int(degree)
        self.h = [extent[d] / self.nc[d] for d in range(3)]
        self.nn = [self.p * n + 1 for n in self.nc]
        self.n_nodes = int(np.prod(self.nn))
        self.cells = [int(c) for c in cells]
        self.matid = np.asarray(matid, np.int64)
        self.lam = np.asarray(lame_first, float)
        self.mu = np.asarray(lame_second, float)
        self.alpha = np.zeros(4) if thermal_expansion is None else np.asarray(thermal_expansion, float)
        self.rho = np.zeros(4) if density is None else np.asarray(density, float)
        x, w, v1, d1 = basis_1d(self.p)
        np1 = self.p + 1
        # 3-D tables: val[q, n], grad[q, n, d] (physical), JxW[q]
        Q = N = np1 ** 3
        self.val = np.zeros((Q, N))
        self.grad = np.zeros((Q, N, 3))
        self.jxw = np.zeros(Q)
        vol = self.h[0] * self.h[1] * self.h[2]
        for q in range(Q):
            qi, qj, qk = q % np1, (q // np1) % np1, q // (np1 * np1)
            self.jxw[q] = w[qi] * w[qj] * w[qk] * vol
            for n in range(N):
                a, b, c = n % np1, (n // np1) % np1, n // (np1 * np1)
                self.val[q, n] = v1[qi, a] * v1[qj, b] * v1[qk, c]
                self.grad[q, n] = (d1[qi, a] * v1[qj, b] * v1[qk, c] / self.h[0],
                                   v1[qi, a] * d1[qj, b] * v1[qk, c] / self.h[1],
                                   v1[qi, a] * v1[qj, b] * d1[qk, c] / self.h[2])
        # node mask: 1 free, 2 clamped
        self.mask = np.zeros(self.n_nodes, np.uint8)
        for c in self.cells:
            for g in self.cell_nodes(c):
                ijk = self.node_ijk(g)
                cl = any(((clamped_faces >> f) & 1) and ijk[f // 2] == ((self.nn[f // 2] - 1) if f & 1 else 0)
                         for f in range(6))
                self.mask[g] = 2 if cl else max(self.mask[g], 1)

    def node_ijk(self, g):
        return (g % self.nn[0], (g // self.nn[0]) % self.nn[1], g // (self.nn[0] * self.nn[1]))

    def cell_nodes(self, c):
        np1 = self.p + 1
        cx, cy, cz = c % self.nc[0], (c // self.nc[0]) % self.nc[1], c // (self.nc[0] * self.nc[1])
        out = []
        for n in range(np1 ** 3):
            a, b, d = n % np1, (n // np1) % np1, n // (np1 * np1)
            out.append((self.p * cx + a) + self.nn[0] * ((self.p * cy + b) + self.nn[1] * (self.p * cz + d)))
        return out

    def matrix(self):
        """The assembled 3 n_nodes x 3 n_nodes matrix (no constraints)."""
        n = self.n_nodes
        K = np.zeros((3 * n, 3 * n))
        for c in self.cells:
            m = self.matid[c]
            lam, mu = self.lam[m], self.mu[m]
            nodes = self.cell_nodes(c)
            gr, jw = self.grad, self.jxw
            for ci in range(3):
                for cj in range(3):
                    # Ke[a, b] for components (ci, cj)
                    Ke = (np.einsum("q,qa,qb->ab", jw, gr[:, :, ci], gr[:, :, cj]) * lam +
                          np.einsum("q,qa,qb->ab", jw, gr[:, :, cj], gr[:, :, ci]) * mu)
                    if ci == cj:
                        Ke = Ke + mu * np.einsum("q,qad,qbd->ab", jw, gr, gr)
                    rows = [ci * n + g for g in nodes]
                    cols = [cj * n + g for g in nodes]
                    K[np.ix_(rows, cols)] += Ke
        return K

    def rhs(self, T=None, melted=None, reference_temperatures=None, initial_temperature=0.0, thermoelastic=True,
            gravity=True):
        """T: nodal temperature on the plain grid (or None)."""
        n = self.n_nodes
        f = np.zeros(3 * n)
        for c in self.cells:
            m = self.matid[c]
            lam, mu = self.lam[m], self.mu[m]
            nodes = self.cell_nodes(c)
            tref = (reference_temperatures[m] if (melted is not None and melted[c]) else initial_temperature)
            B = np.zeros(len(self.jxw))
            if thermoelastic:
                Tq = self.val @ np.asarray(T)[nodes]
                B = (3.0 * lam + 2.0 * mu) * self.alpha[m] * (Tq - tref)
            for comp in range(3):
                fe = np.einsum("q,qa->a", self.jxw * B, self.grad[:, :, comp])
                if comp == 2 and gravity:
                    fe = fe + np.einsum("q,qa->a", self.jxw * (-self.rho[m] * G), self.val)
                f[[comp * n + g for g in nodes]] += fe
        return f

    def free(self):
        idx = np.nonzero(self.mask == 1)[0]
        return np.concatenate([comp * self.n_nodes + idx for comp in range(3)])

    def solve(self, K, f):
        """Displacement with the clamped and absent entries 0."""
        fr = self.free()
        u = np.zeros(3 * self.n_nodes)
        u[fr] = np.linalg.solve(K[np.ix_(fr, fr)], f[fr])
        return u


def cells_with_displacement(active, solid_ratio):
    """MechanicalPhysics::setup_dofs: thermally active and solid > 0.99."""
    return [int(c) for c in np.nonzero((np.asarray(active) != 0) & (np.asarray(solid_ratio) > 0.99))[0]]


class J2Points:
    """The stress state at the Gauss points and its update after a solve,
    restating MechanicalPhysics::compute_stress (source/MechanicalPhysics.cc
    :542-634, combined isotropic-kinematic J2 plasticity after Borja,
    Plasticity, ch. 3) and the state of cells that start carrying
    displacement (setup_dofs, :366-378; constructor :76-98).

    Arrays over every cell of the mesh: kappa[C, nq] (plastic internal
    variable), stress[6, C, nq] and back[6, C, nq] with components xx, yy,
    zz, xy, xz, yz; nq Gauss points per cell, x fastest."""

    def __init__(self, e: Elasticity, plastic_modulus, isotropic_hardening, elastic_limit):
        self.e = e
        C = int(np.prod(e.nc))
        nq = len(e.jxw)
        self.H = np.broadcast_to(np.asarray(plastic_modulus, float), (4,)).copy()
        self.h = np.broadcast_to(np.asarray(isotropic_hardening, float), (4,)).copy()
        self.limit = np.broadcast_to(np.asarray(elastic_limit, float), (4,)).copy()
        self.kappa = np.repeat(self.limit[e.matid][:, None], nq, axis=1)
        self.stress = np.zeros((6, C, nq))
        self.back = np.zeros((6, C, nq))

    def start(self, cells):
        """Cells that start carrying displacement: the elastic limit and zero
        stresses."""
        for c in cells:
            self.kappa[c, :] = self.limit[self.e.matid[c]]
            self.stress[:, c, :] = 0.0
            self.back[:, c, :] = 0.0

    def update(self, du):
        """The stress update from the displacement increment du (3 n_nodes,
        component-major plain grid) at the points of the cells that carry
        displacement."""
        e = self.e
        n = e.n_nodes
        for c in e.cells:
            m = e.matid[c]
            lam, mu, H, h = e.lam[m], e.mu[m], self.H[m], self.h[m]
            nodes = e.cell_nodes(c)
            U = np.stack([np.asarray(du)[comp * n + np.asarray(nodes)] for comp in range(3)])  # [comp, node]
            for q in range(len(e.jxw)):
                G = U @ e.grad[q]  # [comp, d] = d u_comp / d x_d
                eps = 0.5 * (G + G.T)
                sig = self._tensor(self.stress[:, c, q]) + lam * np.trace(eps) * np.eye(3) + 2.0 * mu * eps
                dev = sig - np.trace(sig) / 3.0 * np.eye(3)
                eta = dev - self._tensor(self.back[:, c, q])
                nrm = np.sqrt(np.sum(eta * eta))
                kap = self.kappa[c, q]
                if nrm < kap:
                    self.stress[:, c, q] = self._voigt(sig)
                    continue
                dg = (nrm - kap) / (2.0 * mu + H)
                nflow = eta / nrm
                self.stress[:, c, q] = self._voigt(sig - 2.0 * mu * dg * nflow)
                self.kappa[c, q] = kap + h * H * dg
                # the reference's back-stress update as written (:626-630)
                self.back[:, c, q] = self._voigt(self._tensor(self.back[:, c, q]) + (1.0 - h) * H * H * nflow)

    @staticmethod
    def _tensor(v):
        xx, yy, zz, xy, xz, yz = v
        return np.array([[xx, xy, xz], [xy, yy, yz], [xz, yz, zz]])

    @staticmethod
    def _voigt(t):
        return np.array([t[0, 0], t[1, 1], t[2, 2], t[0, 1], t[0, 2], t[1, 2]])


def transfer_old_displacement(e: Elasticity, carry_prev, carry_now, u_old):
    """The previous displacement after the cells that carry displacement
    changed, as MechanicalPhysics::setup_dofs writes it
    (source/MechanicalPhysics.cc:310-337, :418-437): each cell saves its
    nodes' old values if it carried displacement, zeros if not; the vector is
    cleared and every cell that carries displacement now writes its saved
    values back, in cell order."""
    n = e.n_nodes
    saved = {}
    for c in range(int(np.prod(e.nc))):
        nodes = e.cell_nodes(c)
        saved[c] = (np.stack([np.asarray(u_old)[comp * n + np.asarray(nodes)] for comp in range(3)])
                    if carry_prev[c] else np.zeros((3, len(nodes))))
    out = np.zeros(3 * n)
    for c in range(int(np.prod(e.nc))):
        if carry_now[c]:
            nodes = np.asarray(e.cell_nodes(c))
            for comp in range(3):
                out[comp * n + nodes] = saved[c][comp]
    return out
