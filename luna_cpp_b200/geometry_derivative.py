"""The derivatives of a periodic 2D Voronoi mesh's geometry in its generator positions at fixed topology, the
``GeometryDerivative`` the moving step's tangent and adjoint read (luna-cpp's src/hydro/mesh_derivative.hpp:10-29; the
mesh library is to provide them, and until it does luna-cpp's tests build their own, src/test/reference_geometry_2d.hpp).

    G = Geometry2D(mesh)                   # a luna_cpp_b200.mesh.Mesh (dim 2)
    dV, dc, dA, dxf = G.tangent(dx)        # dx [N, 2] -> volumes [N], centroids [N, 2], areas [F, 2], face centroids [F, 2]
    xbar = G.adjoint(Vbar, cbar, Abar, xfbar)   # the transpose, [N, 2]

The quantities are those the hydro reads: V_i, c_i (relative to the generator), A_f (owner to neighbour), x_f (relative
to the owner). Each Voronoi vertex is the circumcentre of its Delaunay triangle, x_o + C(a, b) with a, b the nearest-image
offsets of the triangle's other two generators; a face's two vertices v+ and v- give e = v+ - v-, A = (e_y, -e_x),
x_f = (v+ + v-) / 2 - x_o; a cell's faces give p_f = A_f . d_f (d_f from the owner to the neighbour), V = sum p_f / 4,
c = (2/3) sum p_f x_f,i / sum p_f with x_f,i the face centroid relative to the cell. Each vertex's triangle is found
from the mesh: the third generator is the common neighbour of the face's two cells whose circumcentre is that vertex
(where four generators are cocircular, as on an exact lattice, a neighbour of either cell: one triangulation's).
The Jacobian is assembled once per mesh as a sparse matrix (rows V, c, A, x_f; columns x), so the tangent and the
adjoint are exact transposes. Host code (numpy, scipy): test and driver infrastructure beside the library, as in the
reference.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def _circle(a, b):
    """The circumcentre of the origin, a and b (rows), relative to the origin."""
    la, lb = np.sum(a * a, -1), np.sum(b * b, -1)
    det = a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]
    return np.stack([(la * b[:, 1] - lb * a[:, 1]) / (2 * det), (lb * a[:, 0] - la * b[:, 0]) / (2 * det)], -1)


def _circle_jacobians(a, b):
    """d C / d a and d C / d b, [n, 2, 2] each (row: the component of C, column: of a or b), from the derivative of the
    formula above (C = (l_a b_perp - l_b a_perp) / (2 det))."""
    la, lb = np.sum(a * a, -1), np.sum(b * b, -1)
    det = a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]
    c = _circle(a, b)
    Ja = np.empty(a.shape[:1] + (2, 2))
    Jb = np.empty(a.shape[:1] + (2, 2))
    for q in range(2):  # seed da = e_q, then db = e_q
        da = np.zeros_like(a)
        da[:, q] = 1.0
        zero = np.zeros_like(a)
        for which, J in ((0, Ja), (1, Jb)):
            dA, dB = (da, zero) if which == 0 else (zero, da)
            dla, dlb = 2 * np.sum(a * dA, -1), 2 * np.sum(b * dB, -1)
            ddet = dA[:, 0] * b[:, 1] + a[:, 0] * dB[:, 1] - dA[:, 1] * b[:, 0] - a[:, 1] * dB[:, 0]
            J[:, 0, q] = (dla * b[:, 1] + la * dB[:, 1] - dlb * a[:, 1] - lb * dA[:, 1]) / (2 * det) - c[:, 0] * ddet / det
            J[:, 1, q] = (dlb * a[:, 0] + lb * dA[:, 0] - dla * b[:, 0] - la * dB[:, 0]) / (2 * det) - c[:, 1] * ddet / det
    return Ja, Jb


class Geometry2D:
    """The geometry Jacobian of a 2D periodic Voronoi mesh (see the module docstring)."""

    def __init__(self, mesh, tolerance: float = 1e-7):
        if mesh.dim != 2:
            raise ValueError("Geometry2D: a 2D mesh")
        self.n, self.f = mesh.n_cells, mesh.n_faces
        x = np.asarray(mesh.positions, dtype=np.float64)
        box = np.asarray(mesh.box[:2], dtype=np.float64)
        own, nbr = np.asarray(mesh.owner), np.asarray(mesh.neighbour)
        area, fcen = np.asarray(mesh.area), np.asarray(mesh.face_centroid)

        def wrap(d):
            return d - box * np.round(d / box)

        # each cell's neighbours (for the common neighbours of a face's two cells)
        start, lst = np.asarray(mesh.cell_face_start), np.asarray(mesh.cell_face)
        face_of = np.where(lst >= 0, lst, ~lst)
        cell_of = np.repeat(np.arange(self.n), np.diff(start))
        other = np.where(own[face_of] == cell_of, nbr[face_of], own[face_of])
        neighbours = [set(other[start[i]:start[i + 1]].tolist()) for i in range(self.n)]

        d = wrap(x[nbr] - x[own])  # owner -> neighbour
        mag = np.sqrt(np.sum(area * area, -1))
        t = np.stack([-area[:, 1], area[:, 0]], -1)  # |A| times the edge direction: v+ - v- = (-A_y, A_x)
        ends = [fcen + 0.5 * t, fcen - 0.5 * t]  # v+, v- relative to the owner's generator
        third = np.full((2, self.f), -1, dtype=np.int64)
        offset = np.zeros((2, self.f, 2))  # the third generator's nearest image relative to the owner
        scale = np.sqrt(np.prod(box) / self.n)
        for f in range(self.f):
            o, j = int(own[f]), int(nbr[f])
            common = sorted(neighbours[o] & neighbours[j])
            # A vertex where four or more generators are cocircular (an exact lattice) has no face between the diagonal
            # pairs, so its third generator need not be a common neighbour: then any neighbour of either cell whose
            # circumcentre with the face's two is the vertex (the derivative there is that of one triangulation).
            either = sorted((neighbours[o] | neighbours[j]) - {o, j})
            for s in range(2):
                for cands in (common, either):
                    if not cands:
                        continue
                    b = wrap(x[cands] - x[o])
                    with np.errstate(divide="ignore", invalid="ignore"):  # a candidate in line with the face's two
                        cc = _circle(np.repeat(d[f:f + 1], len(cands), 0), b)
                    err = np.sqrt(np.sum((cc - ends[s][f]) ** 2, -1))
                    err = np.where(np.isfinite(err), err, np.inf)
                    k = int(np.argmin(err))
                    if err[k] <= tolerance * scale:
                        break
                else:
                    raise ValueError(f"Geometry2D: face {f}'s vertex {s} is no circumcentre of its cells' neighbours")
                third[s, f] = cands[k]
                offset[s, f] = b[k]
        self.own, self.nbr, self.d = own.astype(np.int64), nbr.astype(np.int64), d
        # vertices: C(d, b) relative to the owner; derivative blocks d v / d x_o, x_j, x_k
        rows, cols, vals = [], [], []
        N, F = self.n, self.f
        rV, rc, rA, rxf = 0, N, 3 * N, 3 * N + 2 * F  # row blocks: V [N], c [N][2], A [F][2], x_f [F][2]
        V_of = np.zeros(N)
        dvert = []  # per end: (Jo, Jj, Jk) [F, 2, 2]
        vert = []
        for s in range(2):
            Ja, Jb = _circle_jacobians(d, offset[s])
            vert.append(_circle(d, offset[s]))
            dvert.append((np.eye(2)[None] - Ja - Jb, Ja, Jb))
        # A = (e_y, -e_x), e = v+ - v-; x_f = (v+ + v-) / 2 - x_o (relative to the owner: d x_o drops out of v - x_o's
        # own term, handled by the blocks below, which are d (v relative to x_o) = Ja da + Jb db with da = dx_j - dx_o)
        rot = np.array([[0.0, 1.0], [-1.0, 0.0]])  # A = rot e
        cells = [self.own, self.nbr, third[0], third[1]]

        def add(row0, comp_rows, col_cells, block):
            # block [F, 2(rows), 2(cols)] for the columns of the cells col_cells [F]
            for p in range(comp_rows):
                for q in range(2):
                    rows.append(row0 + p)
                    cols.append(2 * col_cells + q)
                    vals.append(block[:, p, q])

        fidx = np.arange(F)
        for s, sign in ((0, 1.0), (1, -1.0)):
            Jo_rel = -(dvert[s][1] + dvert[s][2])  # d (v - x_o) / d x_o
            Ja, Jb = dvert[s][1], dvert[s][2]
            for J, cell in ((Jo_rel, self.own), (Ja, self.nbr), (Jb, third[s])):
                # A rows: rot (sign J)
                add(rA + 2 * fidx, 2, cell, np.einsum("pr,frq->fpq", rot, sign * J))
                # x_f rows: J / 2 (v - x_o relative, the x_o of x_f's definition cancels with v's)
                add(rxf + 2 * fidx, 2, cell, 0.5 * J)
        JA_x = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                             shape=(3 * N + 4 * F, 2 * N)).tocsr()
        # the face rows as functions of x, then the cells' V and c from them and from the separations
        A_val = np.einsum("pr,fr->fp", rot, vert[0] - vert[1])
        xf_val = 0.5 * (vert[0] + vert[1])
        self.area_check = float(np.max(np.abs(A_val - area)) / np.max(np.abs(area)))
        self.centroid_check = float(np.max(np.abs(xf_val - fcen)) / scale)
        p = np.sum(A_val * d, -1)  # A . d > 0
        P = np.zeros(N)
        np.add.at(P, self.own, p)
        np.add.at(P, self.nbr, p)
        V_of = P / 4
        xfi = [xf_val, xf_val - d]  # the face centroid relative to the owner, to the neighbour
        S = np.zeros((N, 2))
        np.add.at(S, self.own, p[:, None] * xfi[0])
        np.add.at(S, self.nbr, p[:, None] * xfi[1])
        c_val = (2.0 / 3.0) * S / P[:, None]
        self.volume_check = float(np.max(np.abs(V_of - np.asarray(mesh.volume))) / np.max(np.asarray(mesh.volume)))
        self.cell_centroid_check = float(np.max(np.abs(c_val - np.asarray(mesh.centroid))) / scale)
        # dp = dA . d + A . (dx_j - dx_o); dV_i = sum dp / 4; dS_i = sum (dp x_fi + p dx_fi); dc = (2/3)(dS / P - S dP / P^2)
        # assembled as sparse products: p_x = JA_p + d_x parts
        A_rows = JA_x[rA:rA + 2 * F]
        xf_rows = JA_x[rxf:rxf + 2 * F]
        Dsel = sp.csr_matrix((np.concatenate([np.ones(2 * F), -np.ones(2 * F)]),
                              (np.concatenate([np.arange(2 * F), np.arange(2 * F)]),
                               np.concatenate([2 * np.repeat(self.nbr, 2) + np.tile([0, 1], F),
                                               2 * np.repeat(self.own, 2) + np.tile([0, 1], F)]))), shape=(2 * F, 2 * N))
        dot_d = sp.csr_matrix((d.reshape(-1), (np.repeat(np.arange(F), 2), np.arange(2 * F))), shape=(F, 2 * F))
        dot_A = sp.csr_matrix((A_val.reshape(-1), (np.repeat(np.arange(F), 2), np.arange(2 * F))), shape=(F, 2 * F))
        Jp = dot_d @ A_rows + dot_A @ Dsel  # [F, 2N]
        to_own = sp.csr_matrix((np.ones(F), (self.own, np.arange(F))), shape=(N, F))
        to_nbr = sp.csr_matrix((np.ones(F), (self.nbr, np.arange(F))), shape=(N, F))
        JP = (to_own + to_nbr) @ Jp
        JV = 0.25 * JP
        # dS: owner rows sum dp x_f + p dx_f; neighbour rows dp (x_f - d) + p (dx_f - dd)
        blocks = []
        for comp in range(2):
            xo = sp.diags(xfi[0][:, comp]) @ Jp
            xn = sp.diags(xfi[1][:, comp]) @ Jp
            sel = sp.csr_matrix((np.ones(F), (np.arange(F), 2 * np.arange(F) + comp)), shape=(F, 2 * F))
            dxf_c = sel @ xf_rows
            dd_c = sel @ Dsel
            JS = to_own @ (xo + sp.diags(p) @ dxf_c) + to_nbr @ (xn + sp.diags(p) @ (dxf_c - dd_c))
            Jc = (2.0 / 3.0) * (sp.diags(1.0 / P) @ JS - sp.diags(S[:, comp] / (P * P)) @ JP)
            blocks.append(Jc)
        Jc_rows = sp.vstack([blocks[0], blocks[1]]).tocsr()
        # interleave c's components: rows 2 i + comp
        perm = np.empty(2 * N, dtype=np.int64)
        perm[0::2] = np.arange(N)
        perm[1::2] = N + np.arange(N)
        Jc_rows = Jc_rows[perm]
        self.J = sp.vstack([JV, Jc_rows, A_rows, xf_rows]).tocsr()
        self.blocks = (N, F)

    def tangent(self, dx):
        """dx [N, 2] -> dV [N], dc [N, 2], dA [F, 2], dx_f [F, 2]."""
        N, F = self.blocks
        y = self.J @ np.asarray(dx, dtype=np.float64).reshape(-1)
        return y[:N], y[N:3 * N].reshape(N, 2), y[3 * N:3 * N + 2 * F].reshape(F, 2), y[3 * N + 2 * F:].reshape(F, 2)

    def adjoint(self, Vbar, cbar, Abar, xfbar):
        """The transpose: the bars of V [N], c [N, 2], A [F, 2], x_f [F, 2] -> x's bar [N, 2]."""
        N, F = self.blocks
        b = np.concatenate([np.asarray(Vbar, np.float64).reshape(-1), np.asarray(cbar, np.float64).reshape(-1),
                            np.asarray(Abar, np.float64).reshape(-1), np.asarray(xfbar, np.float64).reshape(-1)])
        return (self.J.T @ b).reshape(N, 2)


class NullGeometry:
    """A geometry derivative that is zero: the mesh's V, c, A and x_f held fixed as the generators move (the reference's
    cost test stands one in for the mesh library's, hydro_derivatives_test.cpp:1853-1857). Any dimension. The moving
    step's derivatives then hold every term but the geometry's own (the separations, the face velocity and the drift
    still take dx)."""

    def __init__(self, mesh):
        self.n, self.f, self.dim = int(mesh.n_cells), int(mesh.n_faces), int(mesh.dim)

    def tangent(self, dx):
        D = self.dim
        return np.zeros(self.n), np.zeros((self.n, D)), np.zeros((self.f, D)), np.zeros((self.f, D))

    def adjoint(self, Vbar, cbar, Abar, xfbar):
        return np.zeros((self.n, self.dim))
