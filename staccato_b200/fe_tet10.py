"""Sparse Tet10 stiffness and mass of a clamped steel block: the projection workload's FOM.

Geometry: an nx x ny x nz block of cubes of side h (default 10 x 10 x 40, h = 0.01 m); every
cube is split into 6 tetrahedra along its main diagonal (Kuhn / Freudenthal split, conforming
between neighbours); edge midpoints of all tetrahedra fall on the half-grid, so the Tet10
nodes are the (2nx+1)(2ny+1)(2nz+1) half-grid points, 3 DOFs each, numbered node-major
(node = i + (2nx+1)(j + (2ny+1) k), dof = 3 node + component).  Default N = 21*21*81*3 = 107,163.

Element matrices restate the reference's isoparametric Tet10 element
(src/FEPart/FeTetrahedron10NodeElement.cpp:35-227): corner nodes 1-4, mid-side nodes
5 (1-2), 6 (2-3), 7 (3-1), 8 (1-4), 9 (2-4), 10 (3-4); Jacobian and shape-function
derivatives scaled by det J; stiffness with the 4-point Gauss rule (weight 1/4 each) as
w/(6 det J) B^T E B, mass with the 15-point rule as rho w det J / 6 N^T N; Gauss tables of
src/tools/MathLibrary.h:1419-1459; isotropic elasticity matrix of the same file (:44-52).
Dirichlet: the z = 0 face is clamped by skipping its DOFs in the assembly
(src/analysis/KrylovROMSubstructure.cpp:327-338 with HMesh::killDirichletDOF,
src/datastructure/HMesh.cpp:164-203); the matrix keeps all N DOFs (FOM_DOF is the raw DOF
count, KrylovROMSubstructure.cpp:824), so clamped DOFs have empty rows and columns.
The reference assembles the upper triangle into a symmetric CSR; this generator returns the
full pattern (both triangles), 0-based, sorted columns, K and M sharing one pattern.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class FeModel:
    indptr: np.ndarray  # int64, N+1
    indices: np.ndarray  # int32, nnz
    K: np.ndarray  # float64, nnz (shares the pattern)
    M: np.ndarray  # float64, nnz
    n_dof: int
    clamped: np.ndarray  # bool per DOF
    meta: dict


def _gauss4():
    a = (5 + 3 * math.sqrt(5.0)) / 20.0
    b = (5 - math.sqrt(5.0)) / 20.0
    pts = np.array([[a, b, b, b], [b, a, b, b], [b, b, a, b], [b, b, b, a]])
    return pts, np.full(4, 0.25)


def _gauss15():
    g1a = (7.0 - math.sqrt(15.0)) / 34.0
    g1b = 1.0 - 3.0 * g1a
    g2a = 7.0 / 17.0 - g1a
    g2b = 1.0 - 3.0 * g2a
    g3a = (10.0 - 2.0 * math.sqrt(15.0)) / 40.0
    g3b = 0.5 - g3a
    g4 = 0.25
    w1 = (2665.0 + 14.0 * math.sqrt(15.0)) / 37800.0
    w2 = (2665.0 - 14.0 * math.sqrt(15.0)) / 37800.0
    w3 = 10.0 / 189.0
    w4 = 16.0 / 135.0
    pts = np.array([
        [g1b, g1a, g1a, g1a], [g1a, g1b, g1a, g1a], [g1a, g1a, g1b, g1a], [g1a, g1a, g1a, g1b],
        [g2b, g2a, g2a, g2a], [g2a, g2b, g2a, g2a], [g2a, g2a, g2b, g2a], [g2a, g2a, g2a, g2b],
        [g3b, g3b, g3a, g3a], [g3b, g3a, g3b, g3a], [g3b, g3a, g3a, g3b],
        [g3a, g3b, g3b, g3a], [g3a, g3b, g3a, g3b], [g3a, g3a, g3b, g3b],
        [g4, g4, g4, g4]])
    w = np.array([w1] * 4 + [w2] * 4 + [w3] * 6 + [w4])
    return pts, w


def _shape(coords, xi):
    """Felippa's Tet10 formulas for a batch of elements at one Gauss point.

    coords: (E, 10, 3).  Returns N (10,), dN (E, 3, 10) scaled by det J, det J (E,)."""
    x1, x2, x3, x4 = xi
    c = coords
    q = 0.25

    def J(comp):
        X = c[:, :, comp]
        j1 = 4 * (X[:, 0] * (x1 - q) + X[:, 4] * x2 + X[:, 6] * x3 + X[:, 7] * x4)
        j2 = 4 * (X[:, 4] * x1 + X[:, 1] * (x2 - q) + X[:, 5] * x3 + X[:, 8] * x4)
        j3 = 4 * (X[:, 6] * x1 + X[:, 5] * x2 + X[:, 2] * (x3 - q) + X[:, 9] * x4)
        j4 = 4 * (X[:, 7] * x1 + X[:, 8] * x2 + X[:, 9] * x3 + X[:, 3] * (x4 - q))
        return j1, j2, j3, j4

    Jx1, Jx2, Jx3, Jx4 = J(0)
    Jy1, Jy2, Jy3, Jy4 = J(1)
    Jz1, Jz2, Jz3, Jz4 = J(2)
    Jx12, Jx13, Jx14, Jx23, Jx24, Jx34 = Jx1 - Jx2, Jx1 - Jx3, Jx1 - Jx4, Jx2 - Jx3, Jx2 - Jx4, Jx3 - Jx4
    Jy12, Jy13, Jy14, Jy23, Jy24, Jy34 = Jy1 - Jy2, Jy1 - Jy3, Jy1 - Jy4, Jy2 - Jy3, Jy2 - Jy4, Jy3 - Jy4
    Jz12, Jz13, Jz14, Jz23, Jz24, Jz34 = Jz1 - Jz2, Jz1 - Jz3, Jz1 - Jz4, Jz2 - Jz3, Jz2 - Jz4, Jz3 - Jz4
    Jx21, Jx31, Jx32, Jx42, Jx43 = -Jx12, -Jx13, -Jx23, -Jx24, -Jx34
    Jy21, Jy31, Jy32, Jy42, Jy43 = -Jy12, -Jy13, -Jy23, -Jy24, -Jy34
    Jz21, Jz31, Jz32, Jz42, Jz43 = -Jz12, -Jz13, -Jz23, -Jz24, -Jz34
    det = Jx21 * (Jy23 * Jz34 - Jy34 * Jz23) + Jx32 * (Jy34 * Jz12 - Jy12 * Jz34) + Jx43 * (Jy12 * Jz23 - Jy23 * Jz12)
    a1 = Jy42 * Jz32 - Jy32 * Jz42
    a2 = Jy31 * Jz43 - Jy34 * Jz13
    a3 = Jy24 * Jz14 - Jy14 * Jz24
    a4 = Jy13 * Jz21 - Jy12 * Jz31
    b1 = Jx32 * Jz42 - Jx42 * Jz32
    b2 = Jx43 * Jz31 - Jx13 * Jz34
    b3 = Jx14 * Jz24 - Jx24 * Jz14
    b4 = Jx21 * Jz13 - Jx31 * Jz12
    c1 = Jx42 * Jy32 - Jx32 * Jy42
    c2 = Jx31 * Jy43 - Jx34 * Jy13
    c3 = Jx24 * Jy14 - Jx14 * Jy24
    c4 = Jx13 * Jy21 - Jx12 * Jy31
    N = np.array([x1 * (2 * x1 - 1), x2 * (2 * x2 - 1), x3 * (2 * x3 - 1), x4 * (2 * x4 - 1),
                  4 * x1 * x2, 4 * x2 * x3, 4 * x3 * x1, 4 * x1 * x4, 4 * x2 * x4, 4 * x3 * x4])

    def d(a1, a2, a3, a4):
        return np.stack([(4 * x1 - 1) * a1, (4 * x2 - 1) * a2, (4 * x3 - 1) * a3, (4 * x4 - 1) * a4,
                         4 * (x1 * a2 + x2 * a1), 4 * (x2 * a3 + x3 * a2), 4 * (x3 * a1 + x1 * a3),
                         4 * (x1 * a4 + x4 * a1), 4 * (x2 * a4 + x4 * a2), 4 * (x3 * a4 + x4 * a3)], axis=1)

    dN = np.stack([d(a1, a2, a3, a4), d(b1, b2, b3, b4), d(c1, c2, c3, c4)], axis=1)
    return N, dN, det


def element_matrices(coords, E=210e9, nu=0.3, rho=7850.0):
    """Ke, Me (E, 30, 30) for Tet10 elements with node coordinates coords (E, 10, 3)."""
    tmp = E / ((1 + nu) * (1 - 2 * nu))
    Em = np.zeros((6, 6))
    Em[:3, :3] = tmp * nu
    for i in range(3):
        Em[i, i] = tmp * (1 - nu)
        Em[3 + i, 3 + i] = tmp * (0.5 - nu)
    ne = coords.shape[0]
    Ke = np.zeros((ne, 30, 30))
    Me = np.zeros((ne, 30, 30))
    p4, w4 = _gauss4()
    for k in range(4):
        _, dN, det = _shape(coords, p4[k])
        B = np.zeros((ne, 6, 30))
        dx, dy, dz = dN[:, 0], dN[:, 1], dN[:, 2]
        B[:, 0, 0::3] = dx
        B[:, 1, 1::3] = dy
        B[:, 2, 2::3] = dz
        B[:, 3, 0::3] = dy
        B[:, 3, 1::3] = dx
        B[:, 4, 1::3] = dz
        B[:, 4, 2::3] = dy
        B[:, 5, 0::3] = dz
        B[:, 5, 2::3] = dx
        Ke += np.einsum("eki,kl,elj->eij", B, Em, B) * (w4[k] / (6.0 * det))[:, None, None]
    p15, w15 = _gauss15()
    for k in range(15):
        N, _, det = _shape(coords, p15[k])
        Nm = np.zeros((3, 30))
        for c in range(3):
            Nm[c, c::3] = N
        Me += (Nm.T @ Nm)[None] * (det * rho * w15[k] / 6.0)[:, None, None]
    return Ke, Me


# Kuhn split of the unit cube along the main diagonal (0,0,0)-(1,1,1): one tetrahedron per
# permutation of the axes.
_PERMS = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]


def block_mesh(nx=10, ny=10, nz=40, h=0.01):
    """Tet10 connectivity (E, 10) of half-grid node ids, and node coordinates."""
    gx, gy, gz = 2 * nx + 1, 2 * ny + 1, 2 * nz + 1
    nid = lambda i, j, k: i + gx * (j + gy * k)
    conn = []
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                base = np.array([2 * i, 2 * j, 2 * k])
                for perm in _PERMS:
                    v = [base.copy()]
                    cur = base.copy()
                    for ax in perm:
                        cur = cur.copy()
                        cur[ax] += 2
                        v.append(cur)
                    corners = v
                    # orientation: positive volume
                    e1, e2, e3 = corners[1] - corners[0], corners[2] - corners[0], corners[3] - corners[0]
                    if np.dot(e1, np.cross(e2, e3)) < 0:
                        corners = [corners[0], corners[2], corners[1], corners[3]]
                    c1, c2, c3, c4 = corners
                    mid = lambda a, b: (a + b) // 2
                    nodes = [c1, c2, c3, c4, mid(c1, c2), mid(c2, c3), mid(c3, c1), mid(c1, c4),
                             mid(c2, c4), mid(c3, c4)]
                    conn.append([nid(*p) for p in nodes])
    conn = np.array(conn, dtype=np.int64)
    ii, jj, kk = np.meshgrid(np.arange(gx), np.arange(gy), np.arange(gz), indexing="ij")
    coords = np.zeros((gx * gy * gz, 3))
    ids = (ii + gx * (jj + gy * kk)).ravel()
    coords[ids, 0] = ii.ravel() * h / 2
    coords[ids, 1] = jj.ravel() * h / 2
    coords[ids, 2] = kk.ravel() * h / 2
    return conn, coords


def clamped_block(nx=10, ny=10, nz=40, h=0.01, E=210e9, nu=0.3, rho=7850.0) -> FeModel:
    """Assembled full-pattern CSR K and M of the block, z = 0 face clamped."""
    import scipy.sparse as sp

    conn, coords = block_mesh(nx, ny, nz, h)
    Ke, Me = element_matrices(coords[conn], E, nu, rho)
    n_nodes = coords.shape[0]
    n_dof = 3 * n_nodes
    dofs = (3 * conn[:, :, None] + np.arange(3)[None, None, :]).reshape(conn.shape[0], 30)
    clamped_node = coords[:, 2] == 0.0
    clamped = np.repeat(clamped_node, 3)
    keep = ~clamped[dofs]  # (E, 30)
    mask = keep[:, :, None] & keep[:, None, :]
    rows = np.broadcast_to(dofs[:, :, None], Ke.shape)[mask]
    cols = np.broadcast_to(dofs[:, None, :], Ke.shape)[mask]
    K = sp.coo_matrix((Ke[mask], (rows, cols)), shape=(n_dof, n_dof)).tocsr()
    M = sp.coo_matrix((Me[mask], (rows, cols)), shape=(n_dof, n_dof)).tocsr()
    K.sort_indices()
    M.sort_indices()
    assert np.array_equal(K.indptr, M.indptr) and np.array_equal(K.indices, M.indices)
    return FeModel(indptr=K.indptr.astype(np.int64), indices=K.indices.astype(np.int32),
                   K=K.data.astype(np.float64), M=M.data.astype(np.float64), n_dof=n_dof,
                   clamped=clamped,
                   meta={"elements": int(conn.shape[0]), "nodes": int(n_nodes), "nnz": int(K.nnz),
                         "clamped_dofs": int(clamped.sum()), "h": h, "E": E, "nu": nu, "rho": rho})


def basis(n_dof: int, k: int = 96, seed: int = 1) -> np.ndarray:
    """Seeded N(0,1) basis (n_dof x k, column-major) before orthonormalisation."""
    rng = np.random.default_rng(seed)
    return np.asfortranarray(rng.standard_normal((n_dof, k)))
