"""Independent dense FE assembly on a structured box -- test infrastructure.

The reference pins its matrix-free operator against matrices assembled by
deal.II (tests/test_thermal_operator.cc: MatrixCreator::create_laplace_matrix,
FEValues/FEFaceValues loops).  This module restates those assemblies with
plain numpy loops over cells, quadrature points and local DoFs (no sum
factorization), using the full-grid lexicographic node numbering of the
oracle and the product.
"""
from __future__ import annotations

import itertools

import numpy as np


def gl_nodes(degree):
    """FE_Q support points (Gauss-Lobatto) on [0,1] for degree 1..4: the end
    points and the roots of P'_degree."""
    if degree == 1:
        return np.array([0.0, 1.0])
    inner = np.polynomial.legendre.Legendre.basis(degree).deriv().roots()
    return np.concatenate([[0.0], np.sort((inner + 1.0) / 2.0), [1.0]])


def gauss(n):
    x, w = np.polynomial.legendre.leggauss(n)
    return (x + 1.0) / 2.0, w / 2.0


def lagrange(nodes, x):
    """Values and derivatives of the 1D Lagrange basis at points x."""
    n = len(nodes)
    x = np.atleast_1d(x)
    V = np.ones((len(x), n))
    D = np.zeros((len(x), n))
    for i in range(n):
        for j in range(n):
            if j == i:
                continue
            den = nodes[i] - nodes[j]
            D[:, i] = D[:, i] * (x - nodes[j]) / den + V[:, i] / den
            V[:, i] = V[:, i] * (x - nodes[j]) / den
    return V, D


class BoxFE:
    def __init__(self, dim, n_cells, extent, degree, origin=(0.0, 0.0, 0.0)):
        self.dim, self.deg = dim, degree
        self.nc = list(n_cells[:dim])
        self.h = [extent[d] / n_cells[d] for d in range(dim)]
        self.origin = list(origin[:dim])
        self.nn = [degree * n + 1 for n in self.nc]
        self.n_nodes = int(np.prod(self.nn))
        self.np1 = degree + 1
        self.nodes1 = gl_nodes(degree)
        self.qx, self.qw = gauss(degree + 1)
        self.V, self.D = lagrange(self.nodes1, self.qx)

    def node_id(self, idx):
        out, mul = 0, 1
        for d in range(self.dim):
            out += idx[d] * mul
            mul *= self.nn[d]
        return out

    def cells(self):
        return itertools.product(*[range(n) for n in reversed(self.nc)])

    def cell_dofs(self, cell_rev):
        cc = list(reversed(cell_rev))
        ids = []
        for loc_rev in itertools.product(range(self.np1), repeat=self.dim):
            loc = list(reversed(loc_rev))
            ids.append(self.node_id([self.deg * cc[d] + loc[d] for d in range(self.dim)]))
        return cc, ids

    def local_tables(self):
        """phi[q, i] and grad[q, i, d] (real coordinates) and JxW[q]."""
        np1, dim = self.np1, self.dim
        qidx = list(itertools.product(range(np1), repeat=dim))
        nq = len(qidx)
        phi = np.zeros((nq, np1 ** dim))
        grad = np.zeros((nq, np1 ** dim, dim))
        jxw = np.zeros(nq)
        for qq, qrev in enumerate(qidx):
            q = list(reversed(qrev))
            jxw[qq] = np.prod([self.qw[q[d]] * self.h[d] for d in range(dim)])
            for ii, irev in enumerate(itertools.product(range(np1), repeat=dim)):
                i = list(reversed(irev))
                phi[qq, ii] = np.prod([self.V[q[d], i[d]] for d in range(dim)])
                for e in range(dim):
                    g = 1.0
                    for d in range(dim):
                        g *= (self.D[q[d], i[d]] / self.h[d]) if d == e else self.V[q[d], i[d]]
                    grad[qq, ii, e] = g
        return phi, grad, jxw

    def stiffness(self, coef):
        """Global K[i,j] = sum_cells int (coef grad phi_j) . grad phi_i."""
        phi, grad, jxw = self.local_tables()
        K = np.zeros((self.n_nodes, self.n_nodes))
        ke = np.einsum("qie,ef,qjf,q->ij", grad, coef, grad, jxw)
        for c in self.cells():
            _, ids = self.cell_dofs(c)
            K[np.ix_(ids, ids)] += ke
        return K

    def boundary_faces(self):
        """(cell dofs, face id, tangential dims) of every outer face."""
        for c in self.cells():
            cc, ids = self.cell_dofs(c)
            for f in range(2 * self.dim):
                d, side = divmod(f, 2)
                if (side == 0 and cc[d] == 0) or (side == 1 and cc[d] == self.nc[d] - 1):
                    yield cc, ids, f

    def face_tables(self, f):
        """phi[fq, i] of the cell basis on face f, and face JxW[fq]."""
        dim, np1 = self.dim, self.np1
        d, side = divmod(f, 2)
        tdirs = [e for e in range(dim) if e != d]
        fidx = list(itertools.product(range(np1), repeat=dim - 1))
        phi = np.zeros((len(fidx), np1 ** dim))
        jxw = np.zeros(len(fidx))
        xface = 1.0 if side else 0.0
        Vf, _ = lagrange(self.nodes1, np.array([xface]))
        for qq, qrev in enumerate(fidx):
            q = list(reversed(qrev))
            jxw[qq] = np.prod([self.qw[q[k]] * self.h[tdirs[k]] for k in range(dim - 1)])
            for ii, irev in enumerate(itertools.product(range(np1), repeat=dim)):
                i = list(reversed(irev))
                v = Vf[0, i[d]]
                for k, e in enumerate(tdirs):
                    v *= self.V[q[k], i[e]]
                phi[qq, ii] = v
        return phi, jxw
