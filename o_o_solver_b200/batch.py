"""Many independent models factorised and solved together (the batched form; no counterpart in the reference, which
factorises one model per call).

The models are joined into one block-diagonal system: their supernode forests side by side (each model's supernodes,
columns and rows shifted past the models before it), their matrices as the diagonal blocks of one CSC, their
right-hand sides stacked. The factorisation's level schedule then batches the fronts of every model that sit at the
same height of their trees into the same launches: the many small fronts of all models per launch, the larger fronts
of the larger models in the later levels, each front exactly the one a single-model factorisation would have. Nothing
couples two models: every supernode's rows stay inside its own model, so each model's factor, inertia and solution are
those of its own factorisation.

Each model keeps the reference's symbolic stage (its node order and supernode partition); the join only renumbers.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .linalg import SymbolicFactor, SymmetricCsc


@dataclass
class Part:
    """One model of a batch: its symbolic structure as the arrays of a SymbolicFactor (first column of each supernode
    with the total at the end, parents, row starts with the total at the end, rows) and its lower CSC in that
    symbolic factor's equation order."""

    first_column: np.ndarray
    parent: np.ndarray
    row_start: np.ndarray
    rows: np.ndarray
    matrix: SymmetricCsc

    @property
    def dof_count(self) -> int:
        return int(self.first_column[-1])


def part_of(model, fixture, symbolic: SymbolicFactor | None = None, matrix: SymmetricCsc | None = None) -> Part:
    """The Part of a workloads.Model in the reference's order and partition (`fixture`: node_order, first_position,
    parent); `symbolic` may be given when several models share the topology."""
    order = np.asarray(fixture["node_order"], dtype=np.int32)
    first_position = np.asarray(fixture["first_position"], dtype=np.int64)
    if symbolic is None:
        symbolic = SymbolicFactor.from_partition(model.offsets, model.neighbours, model.weights, order,
                                                 fixture["first_position"], fixture["parent"])
    column_of_position = np.concatenate([[0], np.cumsum(np.asarray(model.weights, dtype=np.int64)[order])])
    row_start, rows = symbolic.row_structure()
    return Part(column_of_position[first_position].astype(np.int32), np.asarray(fixture["parent"], dtype=np.int32),
                row_start, rows, matrix if matrix is not None else model.csc(order, 0))


@dataclass
class Batch:
    """A block-diagonal join of parts: the joined symbolic factor and matrix, and each part's first equation."""

    symbolic: SymbolicFactor
    matrix: SymmetricCsc
    dof_offsets: np.ndarray  # part i owns equations [dof_offsets[i], dof_offsets[i + 1])

    @property
    def dimension(self) -> int:
        return int(self.dof_offsets[-1])

    def stack(self, blocks) -> np.ndarray:
        """The parts' right-hand-side blocks (each dof_count x k) stacked into one Fortran-ordered block."""
        k = blocks[0].shape[1]
        out = np.zeros((self.dimension, k), order="F")
        for i, b in enumerate(blocks):
            out[self.dof_offsets[i]:self.dof_offsets[i + 1]] = b
        return out

    def split(self, x) -> list:
        """The joined solution split back into the parts' blocks."""
        return [x[self.dof_offsets[i]:self.dof_offsets[i + 1]] for i in range(len(self.dof_offsets) - 1)]


def join(parts) -> Batch:
    """The block-diagonal join of `parts` (children before parents in each part, so in the join too)."""
    first_columns, parents, row_starts, rows = [], [], [], []
    offsets, csc_rows, values = [np.zeros(1, dtype=np.int64)], [], []
    dof = supernode = row = term = 0
    dof_offsets = [0]
    for p in parts:
        count = len(p.parent)
        first_columns.append(p.first_column[:-1].astype(np.int64) + dof)
        parents.append(np.where(p.parent >= 0, p.parent.astype(np.int64) + supernode, -1))
        row_starts.append(p.row_start[:-1].astype(np.int64) + row)
        rows.append(p.rows.astype(np.int64) + dof)
        offsets.append(p.matrix.offsets[1:].astype(np.int64) + term)
        csc_rows.append(p.matrix.rows.astype(np.int64) + dof)
        values.append(p.matrix.values)
        dof += p.dof_count
        supernode += count
        row += int(p.row_start[-1])
        term += int(p.matrix.offsets[-1])
        dof_offsets.append(dof)
    if dof > np.iinfo(np.int32).max or row > np.iinfo(np.int32).max:
        raise ValueError("batch: more than 2^31 equations or row entries")
    first_column = np.concatenate(first_columns + [np.array([dof])]).astype(np.int32)
    parent = np.concatenate(parents).astype(np.int32)
    row_start = np.concatenate(row_starts + [np.array([row])]).astype(np.int64)
    symbolic = SymbolicFactor.from_arrays(dof, first_column, parent, row_start,
                                          np.concatenate(rows).astype(np.int32))
    matrix = SymmetricCsc(np.concatenate(offsets), np.concatenate(csc_rows).astype(np.int32),
                          np.concatenate(values))
    return Batch(symbolic, matrix, np.array(dof_offsets, dtype=np.int64))


PANEL_SIZES = (18, 22, 26, 30, 34, 38, 42, 46, 50, 55, 60, 65, 70, 75, 78, 81)


@dataclass
class PanelCase:
    """One seeded stiffened panel of a batch: its mesh size, blade count and skin thickness."""

    n: int
    stringers: int
    thickness: float


def panel_cases(count: int, seed: int = 0xB200):
    """`count` seeded stiffened panels: mesh n x n with n drawn from PANEL_SIZES (2,052 to 39,852 equations), 4 to 12
    blades, skin thickness U[1, 4] mm (numpy's PCG64 seeded seed + i for panel i)."""
    cases = []
    for i in range(count):
        rng = np.random.default_rng(seed + i)
        cases.append(PanelCase(int(PANEL_SIZES[rng.integers(len(PANEL_SIZES))]), int(rng.integers(4, 13)),
                               float(rng.uniform(0.001, 0.004))))
    return cases


def panel_batch(cases, fixture_of, columns: int = 8, seed: int = 0xB200):
    """The batch of `cases` (panel_cases) and its stacked right-hand sides: per panel the pressure and columns - 1
    seeded patterns of 10 point loads N(0, 100 N) (seed base seed + 1000 i). fixture_of(n): the reference's ordering
    of the n x n skin (node_order, first_position, parent). Returns (batch, rhs, parts)."""
    from . import workloads

    symbolic_of = {}
    parts, loads = [], []
    for i, case in enumerate(cases):
        fixture = fixture_of(case.n)
        model = workloads.Model(workloads.PanelSpec(n=case.n, stringers=case.stringers, thickness=case.thickness))
        if case.n not in symbolic_of:
            symbolic_of[case.n] = SymbolicFactor.from_partition(model.offsets, model.neighbours, model.weights,
                                                                fixture["node_order"], fixture["first_position"],
                                                                fixture["parent"])
        parts.append(part_of(model, fixture, symbolic_of[case.n]))
        loads.append(model.loads(fixture["node_order"], columns, seed_base=seed + 1000 * i))
        model.close()
    joined = join(parts)
    return joined, joined.stack(loads), parts


def deal(work, ranks: int):
    """Longest processing time first: the items (by index) dealt to `ranks` workers, each item to the worker with the
    least work so far (ties to the lowest rank), the heaviest items first; returns each worker's item indices in
    increasing order. The same on every rank (no exchange needed)."""
    work = np.asarray(work, dtype=np.float64)
    order = sorted(range(len(work)), key=lambda i: (-work[i], i))
    loads = [0.0] * ranks
    share = [[] for _ in range(ranks)]
    for i in order:
        r = min(range(ranks), key=lambda k: (loads[k], k))
        loads[r] += work[i]
        share[r].append(i)
    return [sorted(s) for s in share]
