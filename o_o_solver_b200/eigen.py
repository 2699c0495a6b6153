"""The reference's eigenvalue interface over the GPU library (jcdulas/O_o_Solver, include/oos/linalg/eigen): an
EigenRequest, the LanczosOptions, and BlockLanczos(options).solve(pencil, request) -> EigenSolution, with a
SparsePencil (o_o_solver_b200.linalg) as the pencil. The Lanczos basis, the blocks and the eigenvectors stay in
device memory; the projected problem and the Sturm walk are host logic of the library (C++).

Every call runs the CUDA library (include/oos_gpu.h); nothing here computes on the CPU.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import numpy as np

from . import _native as nat
from .linalg import SparsePencil, _check

PURPOSES = ["lowest_bound", "lower_bound", "upper_bound", "advance", "fill_gap"]


@dataclass
class EigenRequest:
    """EigenRequest (EigenRequest.hpp:21-35): every root of [lower_bound, upper_bound] (mode_count 0), or the lowest
    mode_count roots above lower_bound (below upper_bound when finite). lower_bound <= 0 starts from the lowest root."""

    lower_bound: float = -math.inf
    upper_bound: float = math.inf
    mode_count: int = 0


def _defaults():
    options = nat.LanczosOptions()
    nat.load().oosgpu_lanczos_defaults(ctypes.byref(options))
    return options


@dataclass
class LanczosOptions:
    """LanczosOptions (BlockLanczos.hpp:21-64); None takes the reference's default."""

    block_size: int | None = None
    modes_per_shift: int | None = None
    convergence_tolerance: float | None = None
    maximum_shifts: int | None = None
    maximum_restarts: int | None = None
    seed: int | None = None

    def native(self):
        options = _defaults()
        for name in ("block_size", "modes_per_shift", "convergence_tolerance", "maximum_shifts", "maximum_restarts",
                     "seed"):
            value = getattr(self, name)
            if value is not None:
                setattr(options, name, value)
        return options


@dataclass
class ShiftRecord:
    """ShiftRecord (BlockLanczos.hpp:68-78)."""

    shift: float
    purpose: str
    sturm_count: int
    has_lanczos_run: bool
    block_steps: int
    restarts: int
    converged_count: int


@dataclass
class EigenSolution:
    """EigenSolution (BlockLanczos.hpp:81-100): eigenvalues increasing, M-orthonormal eigenvectors (host copy, n x k),
    the residual bounds, the shifts, and the solve's wall seconds and its factorisations' device seconds; phases: wall
    seconds by phase; slow_paths: blocks orthonormalised column by column on the host and the one-column operator
    applications that replaced dependent columns."""

    eigenvalues: np.ndarray
    eigenvectors: np.ndarray | None
    residual_bounds: np.ndarray
    shifts: list = field(default_factory=list)
    factorisation_count: int = 0
    verified_count: int = 0
    is_complete: bool = False
    block_steps: int = 0
    seconds: float = 0.0
    factor_seconds: float = 0.0
    phases: dict = field(default_factory=dict)
    slow_paths: dict = field(default_factory=dict)


class BlockLanczos:
    """BlockLanczos (BlockLanczos.hpp:102-161) on the GPU."""

    def __init__(self, options: LanczosOptions | None = None):
        self.options = options or LanczosOptions()

    def solve(self, pencil: SparsePencil, request: EigenRequest, vectors: bool = True,
              start_block=None) -> EigenSolution:
        """BlockLanczos::solve. start_block: a device tensor of the first run's start vectors (block size x dimension,
        contiguous: each row a vector in the pencil's equation order) in place of the random start block."""
        lib = nat.load()
        native_request = nat.EigenRequest(float(request.lower_bound), float(request.upper_bound),
                                          int(request.mode_count))
        options = self.options.native()
        handle = nat.vp()
        if start_block is None:
            _check(lib.oosgpu_modes_solve(pencil._handle, ctypes.byref(native_request), ctypes.byref(options),
                                          ctypes.byref(handle)))
        else:
            if start_block.dim() != 2 or not start_block.is_contiguous() or start_block.shape[1] != pencil.dimension:
                raise ValueError("BlockLanczos.solve: expected a contiguous (block size, dimension) start block")
            _check(lib.oosgpu_modes_solve_start(pencil._handle, ctypes.byref(native_request), ctypes.byref(options),
                                                start_block.data_ptr(), pencil.dimension, start_block.shape[0],
                                                ctypes.byref(handle)))
        try:
            counts = np.zeros(6, dtype=np.int64)
            seconds = np.zeros(6)
            _check(lib.oosgpu_modes_summary(handle, nat.ptr(counts, nat.i64p), nat.ptr(seconds, nat.f64p)))
            k = int(counts[0])
            values = np.zeros(max(k, 1))
            bounds = np.zeros(max(k, 1))
            _check(lib.oosgpu_modes_values(handle, nat.ptr(values, nat.f64p), nat.ptr(bounds, nat.f64p)))
            phi = None
            if vectors:
                phi = np.zeros((pencil.dimension, k), order="F")
                if k > 0:
                    _check(lib.oosgpu_modes_vectors(handle, nat.ptr(phi, nat.f64p), pencil.dimension))
            records = np.zeros((max(int(counts[2]), 1), 7))
            _check(lib.oosgpu_modes_shifts(handle, nat.ptr(records, nat.f64p)))
            shifts = [ShiftRecord(float(r[0]), PURPOSES[int(r[1])], int(r[2]), bool(r[3]), int(r[4]), int(r[5]),
                                  int(r[6])) for r in records[: int(counts[2])]]
            phases = {"factorisation": float(seconds[2]), "operator": float(seconds[3]),
                      "orthogonalisation": float(seconds[4]), "projected": float(seconds[5])}
            work = np.zeros(2, dtype=np.int64)
            parts = np.zeros(7)
            _check(lib.oosgpu_modes_work(handle, nat.ptr(work, nat.i64p), nat.ptr(parts, nat.f64p)))
            slow = {"host_blocks": int(work[0]), "replacement_solves": int(work[1])}
            phases.update({"orthogonalisation_start": float(parts[0]), "orthogonalisation_steps": float(parts[1]),
                           "orthogonalisation_restarts": float(parts[2]), "orthogonalisation_harvest": float(parts[3]),
                           "setup": float(parts[4]), "answer": float(parts[5]), "release": float(parts[6])})
            return EigenSolution(values[:k], phi, bounds[:k], shifts, int(counts[1]), int(counts[3]),
                                 bool(counts[4]), int(counts[5]), float(seconds[0]), float(seconds[1]), phases, slow)
        finally:
            lib.oosgpu_modes_destroy(handle)


@dataclass
class SturmVerification:
    """SturmVerification (SturmCheck.hpp:14-70): the eigenvalues below `verified_up_to` that the Sturm counts confirm,
    and the first interval whose count disagrees with the eigenvalues found (expected, found)."""

    verified_up_to: float
    verified_count: int
    has_mismatch: bool = False
    mismatch_lower: float = 0.0
    mismatch_upper: float = 0.0
    mismatch_expected: int = 0
    mismatch_found: int = 0

    def _packed(self):
        return np.array([self.verified_up_to, self.verified_count, float(self.has_mismatch), self.mismatch_lower,
                         self.mismatch_upper, self.mismatch_expected * 1e6 + self.mismatch_found])


def symmetric_eigen(a):
    """SmallEigenSolver::decompose (src/linalg/dense/SmallEigenSolver.cpp:261-297) of the lower triangle of `a`:
    (eigenvalues increasing, eigenvectors as columns signed by their first largest component). The projected problem
    of each Lanczos step uses this routine."""
    a = np.asfortranarray(a, dtype=np.float64)
    p = a.shape[0]
    values = np.zeros(max(p, 1))
    vectors = np.zeros((p, p), order="F")
    _check(nat.load().oosgpu_symmetric_eigen(nat.ptr(a, nat.f64p), p, max(p, 1), nat.ptr(values, nat.f64p),
                                             nat.ptr(vectors, nat.f64p)))
    return values[:p], vectors


def sturm_verify(points, sorted_values) -> SturmVerification:
    """SturmCheck::addPoint for each (shift, count below it), then verify against the eigenvalues found
    (src/linalg/eigen/SturmCheck.cpp)."""
    shifts = np.array([float(s) for s, _ in points])
    counts = np.array([int(c) for _, c in points], dtype=np.int64)
    values = np.ascontiguousarray(sorted_values, dtype=np.float64)
    r = np.zeros(6)
    _check(nat.load().oosgpu_sturm_verify(len(shifts), nat.ptr(shifts, nat.f64p), nat.ptr(counts, nat.i64p),
                                          len(values), nat.ptr(values, nat.f64p), nat.ptr(r, nat.f64p)))
    expected, found = divmod(int(round(r[5])), 1000000)
    return SturmVerification(float(r[0]), int(r[1]), bool(r[2]), float(r[3]), float(r[4]), expected, found)


def next_shift(request: EigenRequest, scale: float, verification: SturmVerification, sorted_values, ritz_estimates,
               lanczos_shifts):
    """ShiftStrategy(request, scale).nextShift (src/linalg/eigen/ShiftStrategy.cpp:121-193): (shift, purpose)."""
    values = np.ascontiguousarray(sorted_values, dtype=np.float64)
    ritz = np.ascontiguousarray(ritz_estimates, dtype=np.float64)
    shifts = np.ascontiguousarray(lanczos_shifts, dtype=np.float64)
    packed = verification._packed()
    shift = np.zeros(1)
    purpose = np.zeros(1, dtype=np.int32)
    _check(nat.load().oosgpu_shift_next(float(request.lower_bound), float(request.upper_bound),
                                        int(request.mode_count), float(scale), nat.ptr(packed, nat.f64p),
                                        len(values), nat.ptr(values, nat.f64p), len(ritz), nat.ptr(ritz, nat.f64p),
                                        len(shifts), nat.ptr(shifts, nat.f64p), nat.ptr(shift, nat.f64p),
                                        nat.ptr(purpose, nat.i32p)))
    return float(shift[0]), PURPOSES[int(purpose[0])]
