"""The plate workload restated in Python and numpy, for the CPU side of the benchmark.

TEST INFRASTRUCTURE ONLY. The reference arm of bench.py builds its matrix here, so that the timed reference process
never loads the CUDA library of the package. The product's own generator (o_o_solver_b200/csrc/host/model.cpp:
Model::plate, Model::assemble, Model::toCsc, Model::loads) stays the source of the workload. This file repeats its
arithmetic operation for operation, so the two agree bit for bit. tests/test_plate_model.py checks that on the
100 x 100 and 20 x 20 plates.

The model is a flat plate of nx x ny rectangular shells on lx x ly, clamped along x = 0, with 6 DOFs per free node.
The element is the package's own flat shell (bilinear membrane, MITC4 bending, drilling spring). Every element of
the plate is the same rectangle, so one element matrix serves all of them.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

SHELL_DOFS = 24
GAUSS = 0.57735026918962576451
NODE_XI = (-1.0, 1.0, 1.0, -1.0)
NODE_ETA = (-1.0, -1.0, 1.0, 1.0)
MASK64 = (1 << 64) - 1


def _shape(xi, eta, a, b):
    n, dx, dy = [0.0] * 4, [0.0] * 4, [0.0] * 4
    for i in range(4):
        n[i] = 0.25 * (1.0 + xi * NODE_XI[i]) * (1.0 + eta * NODE_ETA[i])
        dx[i] = 0.25 * NODE_XI[i] * (1.0 + eta * NODE_ETA[i]) * (2.0 / a)
        dy[i] = 0.25 * NODE_ETA[i] * (1.0 + xi * NODE_XI[i]) * (2.0 / b)
    return n, dx, dy


def _shear_rows(xi, eta, a, b):
    n, dx, dy = _shape(xi, eta, a, b)
    gxz, gyz = [0.0] * SHELL_DOFS, [0.0] * SHELL_DOFS
    for i in range(4):
        gxz[6 * i + 2] = dx[i]
        gxz[6 * i + 4] = n[i]
        gyz[6 * i + 2] = dy[i]
        gyz[6 * i + 3] = -n[i]
    return gxz, gyz


def _add_bt_d_b(k, n, b, rows, d):
    """k += B^T D B, the sums in the order of the package's element code (B rows x n, D rows x rows, row-major)."""
    db = [0.0] * (rows * n)
    for r in range(rows):
        for c in range(n):
            s = 0.0
            for q in range(rows):
                s += d[r * rows + q] * b[q * n + c]
            db[r * n + c] = s
    for i in range(n):
        for j in range(n):
            s = 0.0
            for r in range(rows):
                s += b[r * n + i] * db[r * n + j]
            k[i * n + j] += s


def shell_stiffness(a, b, t, young, poisson):
    """The 24 x 24 element stiffness (row-major list) of an a x b flat shell."""
    k = [0.0] * (SHELL_DOFS * SHELL_DOFS)
    membrane = young * t / (1.0 - poisson * poisson)
    bending = young * t * t * t / (12.0 * (1.0 - poisson * poisson))
    shear = (5.0 / 6.0) * young / (2.0 * (1.0 + poisson)) * t
    dm = [membrane, membrane * poisson, 0.0, membrane * poisson, membrane, 0.0, 0.0, 0.0,
          membrane * (1.0 - poisson) / 2.0]
    dbend = [bending, bending * poisson, 0.0, bending * poisson, bending, 0.0, 0.0, 0.0,
             bending * (1.0 - poisson) / 2.0]
    ds = [shear, 0.0, 0.0, shear]
    det_j = a * b / 4.0
    gxz_a, _ = _shear_rows(0.0, 1.0, a, b)
    gxz_c, _ = _shear_rows(0.0, -1.0, a, b)
    _, gyz_d = _shear_rows(1.0, 0.0, a, b)
    _, gyz_b = _shear_rows(-1.0, 0.0, a, b)
    for gx in range(2):
        for gy in range(2):
            xi = -GAUSS if gx == 0 else GAUSS
            eta = -GAUSS if gy == 0 else GAUSS
            _, dx, dy = _shape(xi, eta, a, b)
            bm = [0.0] * (3 * SHELL_DOFS)
            bb = [0.0] * (3 * SHELL_DOFS)
            bs = [0.0] * (2 * SHELL_DOFS)
            for i in range(4):
                bm[0 * SHELL_DOFS + 6 * i + 0] = dx[i]
                bm[1 * SHELL_DOFS + 6 * i + 1] = dy[i]
                bm[2 * SHELL_DOFS + 6 * i + 0] = dy[i]
                bm[2 * SHELL_DOFS + 6 * i + 1] = dx[i]
                bb[0 * SHELL_DOFS + 6 * i + 4] = dx[i]
                bb[1 * SHELL_DOFS + 6 * i + 3] = -dy[i]
                bb[2 * SHELL_DOFS + 6 * i + 4] = dy[i]
                bb[2 * SHELL_DOFS + 6 * i + 3] = -dx[i]
            for c in range(SHELL_DOFS):
                bs[c] = 0.5 * (1.0 + eta) * gxz_a[c] + 0.5 * (1.0 - eta) * gxz_c[c]
                bs[SHELL_DOFS + c] = 0.5 * (1.0 + xi) * gyz_d[c] + 0.5 * (1.0 - xi) * gyz_b[c]
            _add_bt_d_b(k, SHELL_DOFS, bm, 3, [v * det_j for v in dm])
            _add_bt_d_b(k, SHELL_DOFS, bb, 3, [v * det_j for v in dbend])
            _add_bt_d_b(k, SHELL_DOFS, bs, 2, [v * det_j for v in ds])
    drilling = 1.0e-3 * shear * a * b / 4.0
    for i in range(4):
        k[(6 * i + 5) * SHELL_DOFS + 6 * i + 5] += drilling
    return np.array(k).reshape(SHELL_DOFS, SHELL_DOFS)


def splitmix64(state):
    """One draw of splitmix64 (Steele, Lea and Flood, OOPSLA 2014): (new state, value)."""
    state = (state + 0x9E3779B97F4A7C15) & MASK64
    z = state
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
    return state, z ^ (z >> 31)


@dataclass
class Csc:
    """Lower triangle of a symmetric matrix, compressed columns (int64 offsets, int32 rows, float64 values)."""

    offsets: np.ndarray
    rows: np.ndarray
    values: np.ndarray

    @property
    def dimension(self) -> int:
        return len(self.offsets) - 1


class Plate:
    """The plate: node graph, stiffness node blocks, pressure load."""

    def __init__(self, nx, ny, lx=1.0, ly=1.0, thickness=0.002, young=70.0e9, poisson=0.33, pressure=1000.0):
        self.nx, self.ny = nx, ny
        grid_x, grid_y = nx + 1, ny + 1
        ix, iy = np.meshgrid(np.arange(grid_x), np.arange(grid_y))
        free_of = np.full(grid_x * grid_y, -1, dtype=np.int64)
        free = (ix > 0).ravel()
        free_of[free] = np.arange(int(free.sum()))
        self.node_count = int(free.sum())
        self.node_dofs = 6
        # elements in the generator's order (ey outer, ex inner), nodes counter-clockwise from (ex, ey)
        ex, ey = np.meshgrid(np.arange(nx), np.arange(ny))
        ex, ey = ex.ravel(), ey.ravel()
        corners = [(ex, ey), (ex + 1, ey), (ex + 1, ey + 1), (ex, ey + 1)]
        self.elements = np.stack([free_of[y * grid_x + x] for x, y in corners], axis=1)  # (elements, 4)
        self._graph()
        self._assemble(shell_stiffness(lx / nx, ly / ny, thickness, young, poisson))
        a, b = lx / nx, ly / ny
        self.pressure_load = np.zeros(self.node_count * 6)
        counts = np.bincount(self.elements[self.elements >= 0], minlength=self.node_count)
        # the same value added once per element of the node, in sequence
        share = pressure * a * b / 4.0
        for k in range(1, int(counts.max()) + 1):
            self.pressure_load[np.flatnonzero(counts >= k) * 6 + 2] += share

    def _graph(self):
        pairs = []
        for i in range(4):
            for j in range(4):
                if i != j:
                    pairs.append(self.elements[:, [i, j]])
        pairs = np.concatenate(pairs)
        pairs = pairs[(pairs >= 0).all(axis=1)]
        key = np.unique(pairs[:, 0] * self.node_count + pairs[:, 1])
        a, b = key // self.node_count, key % self.node_count
        self.offsets = np.zeros(self.node_count + 1, dtype=np.int64)
        np.cumsum(np.bincount(a, minlength=self.node_count), out=self.offsets[1:])
        self.neighbours = b.astype(np.int32)
        self.weights = np.full(self.node_count, 6, dtype=np.int32)

    def _slot(self, a, b):
        """The CSR position of neighbour b in node a's sorted neighbour list."""
        owner = np.repeat(np.arange(self.node_count), np.diff(self.offsets))
        flat = owner.astype(np.int64) * self.node_count + self.neighbours
        return np.searchsorted(flat, a.astype(np.int64) * self.node_count + b)

    def _assemble(self, ke):
        """Node blocks: for node a, its diagonal block and one block per neighbour, each 6 x 6 with rows the DOFs of
        a; each block's element terms added in increasing element order, starting from zero."""
        w = 6
        self.diagonal_blocks = np.zeros((self.node_count, w, w))
        self.off_blocks = np.zeros((len(self.neighbours), w, w))
        element_ids = np.arange(len(self.elements))
        blocks = np.stack([ke[i * w:(i + 1) * w, j * w:(j + 1) * w] for i in range(4) for j in range(4)])
        terms = {"diagonal": ([], [], []), "off": ([], [], [])}  # target block, element, local pair (i, j)
        for i in range(4):
            for j in range(4):
                a, b = self.elements[:, i], self.elements[:, j]
                keep = (a >= 0) & (b >= 0)
                kind = "diagonal" if i == j else "off"
                target = a[keep] if i == j else self._slot(a[keep], b[keep])
                terms[kind][0].append(target)
                terms[kind][1].append(element_ids[keep])
                terms[kind][2].append(np.full(int(keep.sum()), 4 * i + j))
        for kind, store in (("diagonal", self.diagonal_blocks), ("off", self.off_blocks)):
            target, element, pair = (np.concatenate(part) for part in terms[kind])
            order = np.lexsort((element, target))
            target, pair = target[order], pair[order]
            first = np.r_[True, target[1:] != target[:-1]]
            rank = np.arange(len(target)) - np.maximum.accumulate(np.where(first, np.arange(len(target)), 0))
            for r in range(int(rank.max()) + 1 if len(rank) else 0):
                chosen = rank == r  # each target at most once per pass: the terms of a block in element order
                store[target[chosen]] += blocks[pair[chosen]]

    def csc(self, node_at_position) -> Csc:
        """The stiffness in the equation order of a node order (a node's DOFs consecutive), lower triangle: per
        column its diagonal block's part from the diagonal down, then the full rows of every neighbour at a later
        position, by position."""
        w = 6
        order = np.asarray(node_at_position, dtype=np.int64)
        position = np.empty(self.node_count, dtype=np.int64)
        position[order] = np.arange(self.node_count)
        owner = np.repeat(np.arange(self.node_count), np.diff(self.offsets))
        p_of_pair = position[owner]
        q_of_pair = position[self.neighbours]
        later = q_of_pair > p_of_pair
        pair_p, pair_q, pair_k = p_of_pair[later], q_of_pair[later], np.flatnonzero(later)
        sort = np.lexsort((pair_q, pair_p))
        pair_p, pair_q, pair_k = pair_p[sort], pair_q[sort], pair_k[sort]
        later_count = np.bincount(pair_p, minlength=self.node_count)
        pair_rank = np.arange(len(pair_p)) - np.repeat(np.cumsum(later_count) - later_count, later_count)
        c = np.arange(w)
        per_column = ((w - c)[None, :] + later_count[:, None] * w).ravel()  # (position, c) in column order
        offsets = np.zeros(self.node_count * w + 1, dtype=np.int64)
        np.cumsum(per_column, out=offsets[1:])
        rows = np.empty(offsets[-1], dtype=np.int32)
        values = np.empty(offsets[-1])
        # diagonal blocks: rows r >= c
        rr, cc = np.tril_indices(w)  # r >= c
        p = np.arange(self.node_count)
        at = offsets[(p[:, None] * w + cc[None, :])] + (rr - cc)[None, :]
        rows[at] = (p[:, None] * w + rr[None, :]).astype(np.int32)
        values[at] = self.diagonal_blocks[order][:, rr, cc]
        # neighbour blocks: K(neighbour r, node c) = block(node -> neighbour)[c, r]
        cgrid, rgrid = np.meshgrid(c, c, indexing="ij")  # (c, r)
        at = (offsets[pair_p[:, None, None] * w + cgrid[None]] + (w - cgrid)[None] + pair_rank[:, None, None] * w
              + rgrid[None])
        rows[at] = (pair_q[:, None, None] * w + rgrid[None]).astype(np.int32)
        values[at] = self.off_blocks[pair_k][:, cgrid, rgrid]
        return Csc(offsets, rows, values)

    def loads(self, node_at_position, columns, seed_base=0xB200, points=10, sigma=100.0):
        """Column 0 the pressure; column j >= 1 `points` seeded nodes with N(0, sigma) forces on their out-of-plane
        translation (splitmix64 seeded seed_base + j, Box-Muller). Fortran-ordered (n, columns)."""
        w = 6
        order = np.asarray(node_at_position, dtype=np.int64)
        position = np.empty(self.node_count, dtype=np.int64)
        position[order] = np.arange(self.node_count)
        rhs = np.zeros((self.node_count * w, columns), order="F")
        for j in range(columns):
            if j == 0:
                rhs[(position[:, None] * w + np.arange(w)).ravel(), 0] = self.pressure_load
                continue
            state = (seed_base + j) & MASK64
            for _ in range(points):
                state, draw = splitmix64(state)
                node = draw % self.node_count
                state, draw = splitmix64(state)
                u1 = 1.0 - (draw >> 11) * 2.0 ** -53
                state, draw = splitmix64(state)
                u2 = (draw >> 11) * 2.0 ** -53
                normal = math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * 3.14159265358979323846 * u2)
                rhs[position[node] * w + 2, j] += sigma * normal
        return rhs


def lower_multiply(csc: Csc, x):
    """y = A x for the symmetric matrix whose lower triangle `csc` holds (a residual check on the host)."""
    import scipy.sparse as sp

    n = csc.dimension
    lower = sp.csc_matrix((csc.values, csc.rows, csc.offsets), shape=(n, n))
    diag = lower.diagonal()
    return lower @ x + lower.T @ x - (diag[:, None] * x if x.ndim == 2 else diag * x)


def accuracy(csc: Csc, x, b):
    """(largest relative residual ||b - Ax||_2/||b||_2, largest normwise backward error
    ||b - Ax||_inf / (||A||_inf ||x||_inf + ||b||_inf)) over the columns."""
    r = b - lower_multiply(csc, x)
    norm_a = lower_multiply(Csc(csc.offsets, csc.rows, np.abs(csc.values)), np.ones((csc.dimension, 1)))[:, 0].max()
    residual = np.linalg.norm(r, axis=0) / np.linalg.norm(b, axis=0)
    backward = np.abs(r).max(axis=0) / (norm_a * np.abs(x).max(axis=0) + np.abs(b).max(axis=0))
    return float(residual.max()), float(backward.max())
