"""The reference's factorisation interface over the GPU library, with the same names, argument meanings and errors
(jcdulas/O_o_Solver, include/oos/linalg): SymbolicFactor (the structure a factorisation is given), SupernodalFactor
.factorise, FactorSolve.solve, the FactorOptions / PivotPolicy fields, and the exceptions the C ABI's status codes map
(SingularityError, MemoryBudgetError, ...).

Every call runs the CUDA library (include/oos_gpu.h); nothing here computes on the CPU.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _native as nat

# ---- errors: one per status code (include/oos_gpu.h), named after the reference's exceptions ----------------------


class SolverError(RuntimeError):
    """base::SolverError."""


class SingularityError(SolverError):
    """base::SingularityError: a zero pivot, or pivots flagged by the ratio test with SingularityBailOut >= 0."""


class MemoryBudgetError(MemoryError):
    """base::MemoryBudgetError (device memory)."""


class OperationCancelledError(RuntimeError):
    """base::OperationCancelledError."""


class CudaError(RuntimeError):
    """A CUDA runtime error (no counterpart in the CPU reference)."""


class InternalError(RuntimeError):
    """base::InternalError."""


_ERRORS = {
    1: ValueError,  # std::invalid_argument
    2: MemoryBudgetError,
    3: SingularityError,
    4: OperationCancelledError,
    5: CudaError,
    6: InternalError,
    7: RuntimeError,  # std::logic_error: solve before factorise
    8: SolverError,
}


def _check(status: int):
    if status != 0:
        raise _ERRORS.get(status, RuntimeError)(nat.load().oosgpu_last_error().decode())


def device_count() -> int:
    return int(nat.load().oosgpu_device_count())


def release_cached_buffers(device: int = -1) -> int:
    """Frees the idle device buffers the eigenvalue solves keep for reuse (of `device`, or of every device); returns
    the bytes freed."""
    return int(nat.load().oosgpu_release_cached_buffers(int(device)))


# ---- symbolic structure ----------------------------------------------------------------------------------------------


class SymbolicFactor:
    """The symbolic structure of a factorisation (include/oos/linalg/symbolic/SymbolicFactor.hpp:37-126): supernode s
    owns the DOF columns [first_column[s], first_column[s + 1]), its rows below them are rows(s), ascending, and
    parent[s] is -1 for a root."""

    def __init__(self, handle):
        self._handle = handle
        sizes = np.zeros(8, dtype=np.int64)
        flops = ctypes.c_double()
        _check(nat.load().oosgpu_symbolic_sizes(handle, nat.ptr(sizes, nat.i64p), ctypes.byref(flops)))
        (self.dof_count, self.supernode_count, self.row_entry_count, self.panel_value_count,
         self.factor_entry_count, self.level_count, self.update_value_count) = (int(v) for v in sizes[:7])
        self.flop_count = float(flops.value)

    @classmethod
    def from_arrays(cls, dof_count, first_column, parent, row_start, rows):
        first_column = np.ascontiguousarray(first_column, dtype=np.int32)
        parent = np.ascontiguousarray(parent, dtype=np.int32)
        row_start = np.ascontiguousarray(row_start, dtype=np.int64)
        rows = np.ascontiguousarray(rows, dtype=np.int32)
        handle = nat.vp()
        _check(nat.load().oosgpu_symbolic_create(int(dof_count), len(parent), nat.ptr(first_column, nat.i32p),
                                                 nat.ptr(parent, nat.i32p), nat.ptr(row_start, nat.i64p),
                                                 nat.ptr(rows, nat.i32p), ctypes.byref(handle)))
        return cls(handle)

    @classmethod
    def from_partition(cls, offsets, neighbours, weights, node_at_position, first_position, parent):
        """The row structures of a supernode partition of the final node order (SymbolicFactor::analyse's last
        step)."""
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        neighbours = np.ascontiguousarray(neighbours, dtype=np.int32)
        weights = np.ascontiguousarray(weights, dtype=np.int32)
        order = np.ascontiguousarray(node_at_position, dtype=np.int32)
        first_position = np.ascontiguousarray(first_position, dtype=np.int32)
        parent = np.ascontiguousarray(parent, dtype=np.int32)
        handle = nat.vp()
        _check(nat.load().oosgpu_symbolic_from_partition(len(weights), nat.ptr(offsets, nat.i64p),
                                                         nat.ptr(neighbours, nat.i32p), nat.ptr(weights, nat.i32p),
                                                         nat.ptr(order, nat.i32p), len(parent),
                                                         nat.ptr(first_position, nat.i32p), nat.ptr(parent, nat.i32p),
                                                         ctypes.byref(handle)))
        return cls(handle)

    def solve_chains(self):
        """The solves' chain launches of this structure's plan, built on the host: launches, tasks, ready flags and the
        tasks of the largest launch (building the plan checks the tasks' order)."""
        counts = np.zeros(4, dtype=np.int64)
        _check(nat.load().oosgpu_symbolic_solve_chains(self._handle, nat.ptr(counts, nat.i64p)))
        return {"launches": int(counts[0]), "tasks": int(counts[1]), "flags": int(counts[2]),
                "largest_launch": int(counts[3])}

    def row_structure(self):
        row_start = np.zeros(self.supernode_count + 1, dtype=np.int64)
        rows = np.zeros(max(self.row_entry_count, 1), dtype=np.int32)
        _check(nat.load().oosgpu_symbolic_rows(self._handle, nat.ptr(row_start, nat.i64p), nat.ptr(rows, nat.i32p)))
        return row_start, rows[: self.row_entry_count]

    def close(self):
        if self._handle:
            nat.load().oosgpu_symbolic_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- factorisation ---------------------------------------------------------------------------------------------------


@dataclass
class PivotPolicy:
    """PivotPolicy (include/oos/linalg/supernodal/PivotDiagnostics.hpp:34-44)."""

    max_ratio: float = 1.0e7
    bailout: int = 0


@dataclass
class FactorOptions:
    """FactorOptions (SupernodalFactor.hpp:63-97). pivoting: "positive_definite" (PivotingMode::PositiveDefinite:
    no pivoting, the ratio test, a zero pivot refused) or "indefinite" (PivotingMode::Indefinite: Bunch-Kaufman 1x1 /
    2x2 pivots within each front, zero pivots counted in the inertia)."""

    pivot_policy: PivotPolicy = field(default_factory=PivotPolicy)
    reference_diagonal: np.ndarray | None = None
    pivoting: str = "positive_definite"
    # "fp64", or "mixed": the update matrices by 3xTF32 products on the tcgen05 tensor cores (about FP32 accuracy;
    # solve_refined recovers FP64 accuracy). Not in the reference.
    precision: str = "fp64"


@dataclass
class Inertia:
    positive: int = 0
    negative: int = 0
    zero: int = 0


@dataclass
class PivotDiagnostics:
    issue_count: int = 0
    largest_ratio: float = 0.0
    equation_of_largest_ratio: int = -1
    issues: list = field(default_factory=list)


class SymmetricCsc:
    """A lower-triangle CSC in the factor's equation order (SymmetricCsc.hpp:40-103): int64 column offsets, int32 rows
    ascending from the diagonal, float64 values. Host arrays, or device tensors (torch) for the device entry points."""

    def __init__(self, offsets, rows, values):
        self.offsets = offsets
        self.rows = rows
        self.values = values

    @property
    def dimension(self) -> int:
        return len(self.offsets) - 1


class SupernodalFactor:
    """The numeric LDL^T of a sparse symmetric matrix on the GPU (SupernodalFactor.hpp:171-292), positive definite
    mode. factorise() allocates the panels and update matrices on the device on its first call; later calls on the same
    structure reuse them (the reference's FactorOptions::storage)."""

    def __init__(self, symbolic: SymbolicFactor, device: int = 0):
        self.symbolic = symbolic
        self._handle = nat.vp()
        _check(nat.load().oosgpu_factor_create(symbolic._handle, device, ctypes.byref(self._handle)))
        self.inertia = Inertia()
        self.pivot_diagnostics = PivotDiagnostics()
        self.device_seconds = 0.0
        self.zero_pivots = []

    @classmethod
    def factorise(cls, symbolic: SymbolicFactor, matrix: SymmetricCsc, options: FactorOptions | None = None,
                  device: int = 0) -> "SupernodalFactor":
        factor = cls(symbolic, device)
        factor.refactorise(matrix, options)
        return factor

    def _options(self, options):
        options = options or FactorOptions()
        native = nat.FactorOptions()
        native.max_ratio = options.pivot_policy.max_ratio
        native.bailout = options.pivot_policy.bailout
        if options.pivoting not in ("positive_definite", "indefinite"):
            raise ValueError(f"FactorOptions.pivoting: expected positive_definite or indefinite, found {options.pivoting}")
        native.pivoting = 1 if options.pivoting == "indefinite" else 0
        if options.precision not in ("fp64", "mixed"):
            raise ValueError(f"FactorOptions.precision: expected fp64 or mixed, found {options.precision}")
        native.precision = 1 if options.precision == "mixed" else 0
        self._reference = None
        if options.reference_diagonal is not None:
            self._reference = np.ascontiguousarray(options.reference_diagonal, dtype=np.float64)
            native.reference_diagonal = nat.ptr(self._reference, nat.f64p)
        return native

    def refactorise(self, matrix: SymmetricCsc, options: FactorOptions | None = None):
        """A new factorisation of a matrix of the same structure (host or device arrays)."""
        native = self._options(options)
        info = nat.FactorInfo()
        lib = nat.load()
        if isinstance(matrix.offsets, np.ndarray):
            offsets = np.ascontiguousarray(matrix.offsets, dtype=np.int64)
            rows = np.ascontiguousarray(matrix.rows, dtype=np.int32)
            values = np.ascontiguousarray(matrix.values, dtype=np.float64)
            status = lib.oosgpu_factorise(self._handle, len(offsets) - 1, nat.ptr(offsets, nat.i64p),
                                          nat.ptr(rows, nat.i32p), nat.ptr(values, nat.f64p), ctypes.byref(native),
                                          ctypes.byref(info))
        else:
            status = lib.oosgpu_factorise_device(self._handle, matrix.offsets.numel() - 1, matrix.rows.numel(),
                                                 matrix.offsets.data_ptr(), matrix.rows.data_ptr(),
                                                 matrix.values.data_ptr(), ctypes.byref(native), ctypes.byref(info))
        self._record(info)
        _check(status)
        return self

    def _record(self, info):
        self.inertia = Inertia(int(info.positive), int(info.negative), int(info.zero))
        self.pivot_diagnostics = PivotDiagnostics(int(info.issue_count), float(info.largest_ratio),
                                                  int(info.equation_of_largest),
                                                  list(info.issues[: min(16, int(info.issue_count))]))
        self.zero_pivots = list(info.zero_pivots[: min(16, int(info.zero_pivot_count))])
        self.delayed_pivot_count = int(info.delayed)
        self.two_by_two_pivot_count = int(info.two_by_two)
        self.is_singular = self.inertia.zero > 0
        self.device_seconds = float(info.device_seconds)

    @property
    def stream(self) -> int:
        return int(nat.load().oosgpu_factor_stream(self._handle) or 0)

    KERNEL_KINDS = ["small_fronts", "assemble_fronts", "diagonal_blocks", "panel_rows", "panel_update",
                    "update_matrix"]

    def profile(self, enable: bool = True):
        """Brackets every launch of the following factorisations and solves with CUDA events (kernel_stats(),
        launch_profile())."""
        _check(nat.load().oosgpu_factor_profile(self._handle, 1 if enable else 0))

    def kernel_stats(self) -> dict:
        """Per kernel kind of the last profiled factorisation: device seconds, launches, algorithmic flops, bytes."""
        kinds = len(self.KERNEL_KINDS)
        seconds = np.zeros(kinds)
        launches = np.zeros(kinds, dtype=np.int64)
        flops = np.zeros(kinds)
        bytes_ = np.zeros(kinds)
        _check(nat.load().oosgpu_factor_kernel_stats(self._handle, kinds, nat.ptr(seconds, nat.f64p),
                                                     nat.ptr(launches, nat.i64p), nat.ptr(flops, nat.f64p),
                                                     nat.ptr(bytes_, nat.f64p)))
        return {name: {"seconds": float(seconds[k]), "launches": int(launches[k]), "flops": float(flops[k]),
                       "bytes": float(bytes_[k])} for k, name in enumerate(self.KERNEL_KINDS)}

    SIZE_CLASSES = ["1 block", "up to 8", "up to 148", "up to 592", "more"]

    def set_tuning(self, mode="tune"):
        """The kernel choice of the launch kinds with two kernels: "tune" (the default: on the next positive definite
        FP64 factorisation each is timed and each size class of launch keeps the faster), "default" (the plan's own
        kernels) or "alternative" (the other kernel everywhere)."""
        code = {"default": 0, "tune": 1, "alternative": 2}[mode]
        _check(nat.load().oosgpu_factor_set_tuning(self._handle, code))

    def tuning(self) -> list:
        """The autotuner's choices: per (launch kind, size class) the launches, the seconds of each kernel in the timing
        factorisations and the kernel chosen (0 or 1); empty before the tuning factorisation."""
        lib = nat.load()
        total = ctypes.c_int64()
        _check(lib.oosgpu_factor_tuning_report(self._handle, 0, None, None, None, None, None, None, ctypes.byref(total)))
        count = int(total.value)
        kinds, classes, launches, chosen = (np.zeros(max(count, 1), dtype=np.int32) for _ in range(4))
        seconds0, seconds1 = np.zeros(max(count, 1)), np.zeros(max(count, 1))
        _check(lib.oosgpu_factor_tuning_report(self._handle, count, nat.ptr(kinds, nat.i32p), nat.ptr(classes, nat.i32p),
                                               nat.ptr(launches, nat.i32p), nat.ptr(seconds0, nat.f64p),
                                               nat.ptr(seconds1, nat.f64p), nat.ptr(chosen, nat.i32p),
                                               ctypes.byref(total)))
        return [{"kind": self.LAUNCH_KINDS[kinds[k]], "size_class": self.SIZE_CLASSES[classes[k]],
                 "launches": int(launches[k]), "seconds": [float(seconds0[k]), float(seconds1[k])],
                 "chosen": int(chosen[k])} for k in range(count)]

    LAUNCH_KINDS = ["small_fronts", "assemble_fronts", "diagonal_blocks", "panel_rows", "panel_update",
                    "update_matrix", "forward_small", "forward_gather", "forward_chain", "backward_small",
                    "backward_rows", "backward_chain", "small_fronts_pivoted", "pivoted_diagonal",
                    "permute_earlier_rows", "panel_rows_pivoted", "update_pivoted", "level_end", "invert_diagonal",
                    "update_matrix_mixed", "backward_rows_reduce", "diagonal_sweep"]

    def launch_profile(self, which: str = "factor"):
        """The launches of the last profiled factorisation ("factor") or solve ("solve"), in order: a list of
        (kind, blocks, first column of the step, device seconds)."""
        code = {"factor": 0, "solve": 1}[which]
        total = ctypes.c_int64()
        lib = nat.load()
        _check(lib.oosgpu_factor_launch_profile(self._handle, code, 0, None, None, None, None, ctypes.byref(total)))
        count = int(total.value)
        kinds = np.zeros(max(count, 1), dtype=np.int32)
        blocks = np.zeros(max(count, 1), dtype=np.int32)
        k0 = np.zeros(max(count, 1), dtype=np.int32)
        seconds = np.zeros(max(count, 1))
        _check(lib.oosgpu_factor_launch_profile(self._handle, code, count, nat.ptr(kinds, nat.i32p),
                                                nat.ptr(blocks, nat.i32p), nat.ptr(k0, nat.i32p),
                                                nat.ptr(seconds, nat.f64p), ctypes.byref(total)))
        return [(self.LAUNCH_KINDS[kinds[i]], int(blocks[i]), int(k0[i]), float(seconds[i])) for i in range(count)]

    def launch_counts(self, columns: int):
        """(kernels of one factorisation, kernels of one solve of `columns` right-hand sides)."""
        counts = np.zeros(2, dtype=np.int64)
        _check(nat.load().oosgpu_factor_launch_counts(self._handle, columns, nat.ptr(counts, nat.i64p)))
        return int(counts[0]), int(counts[1])

    def prefetch(self, b: np.ndarray, deferred: bool = True):
        """Copies host right-hand sides (n x k, column-major) to the device ahead of their solve, overlapping what the
        factor does meanwhile: with `deferred`, from the moment the next refactorisation has queued its matrix's
        upload (the matrix first on the host link, then the loads while it is factorised). The next host-array solve
        of the same array uses the copy; the array must stay unchanged until then."""
        if b.ndim != 2 or not b.flags.f_contiguous or b.dtype != np.float64:
            raise ValueError("prefetch: expected a column-major float64 matrix")
        _check(nat.load().oosgpu_solve_prefetch(self._handle, nat.ptr(b, nat.f64p), b.shape[0], b.shape[1],
                                                1 if deferred else 0))

    def panel(self, s: int):
        """(values rows x eliminated, row equations, subdiagonal) of supernode s (SupernodalFactor::panel)."""
        lib = nat.load()
        e = ctypes.c_int64()
        r = ctypes.c_int64()
        _check(lib.oosgpu_factor_panel(self._handle, s, ctypes.byref(e), ctypes.byref(r), None, None, None))
        values = np.zeros((e.value, r.value))
        rows = np.zeros(r.value, dtype=np.int32)
        sub = np.zeros(max(e.value, 1))
        _check(lib.oosgpu_factor_panel(self._handle, s, ctypes.byref(e), ctypes.byref(r), nat.ptr(values, nat.f64p),
                                       nat.ptr(rows, nat.i32p), nat.ptr(sub, nat.f64p)))
        return values.T.copy(), rows, sub[: e.value]

    def close(self):
        if self._handle:
            nat.load().oosgpu_factor_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PartialFactor:
    """PartialFactor (include/oos/linalg/supernodal/PartialFactor.hpp:48-112): the interior of a unit factorised on
    the GPU, its boundary (the symbolic factor's trailing set, ordered last: its last supernode) left as the Schur
    complement K* = K_bb - K_bi K_ii^-1 K_ib; condensed loads f* = f_b - K_bi K_ii^-1 f_i and the recovery of the
    interior u_i = K_ii^-1 (f_i - K_ib u_b) from boundary values. Positive definite FP64 only, as the reference."""

    def __init__(self, symbolic: SymbolicFactor, trailing: int, device: int = 0):
        self._factor = SupernodalFactor(symbolic, device)
        self.dimension = symbolic.dof_count
        self.trailing = int(trailing)
        self.schur_complement = None

    @classmethod
    def factorise(cls, symbolic: SymbolicFactor, matrix: SymmetricCsc, trailing: int,
                  options: FactorOptions | None = None, device: int = 0) -> "PartialFactor":
        partial = cls(symbolic, trailing, device)
        partial.refactorise(matrix, options)
        return partial

    def refactorise(self, matrix: SymmetricCsc, options: FactorOptions | None = None):
        native = self._factor._options(options)
        info = nat.FactorInfo()
        offsets = np.ascontiguousarray(matrix.offsets, dtype=np.int64)
        rows = np.ascontiguousarray(matrix.rows, dtype=np.int32)
        values = np.ascontiguousarray(matrix.values, dtype=np.float64)
        schur = np.zeros((self.trailing, self.trailing), order="F")
        status = nat.load().oosgpu_factorise_partial(
            self._factor._handle, len(offsets) - 1, nat.ptr(offsets, nat.i64p), nat.ptr(rows, nat.i32p),
            nat.ptr(values, nat.f64p), self.trailing, ctypes.byref(native), nat.ptr(schur, nat.f64p),
            ctypes.byref(info))
        self._factor._record(info)
        _check(status)
        self.schur_complement = schur
        return self

    @property
    def inertia(self) -> Inertia:
        return self._factor.inertia

    def condense_loads(self, loads) -> np.ndarray:
        """f* = f_b - K_bi K_ii^-1 f_i (trailing x columns) of loads (dimension x columns)."""
        x = np.asfortranarray(np.asarray(loads, dtype=np.float64).reshape(self.dimension, -1))
        out = np.zeros((self.trailing, x.shape[1]), order="F")
        _check(nat.load().oosgpu_partial_condense(self._factor._handle, nat.ptr(x, nat.f64p), self.dimension,
                                                   x.shape[1], nat.ptr(out, nat.f64p), self.trailing))
        return out

    def recover(self, loads, trailing_values) -> np.ndarray:
        """The solution of the unit (dimension x columns) from its loads and its boundary values u_b."""
        x = np.array(np.asarray(loads, dtype=np.float64).reshape(self.dimension, -1), order="F", copy=True)
        t = np.asfortranarray(np.asarray(trailing_values, dtype=np.float64).reshape(self.trailing, -1))
        _check(nat.load().oosgpu_partial_recover(self._factor._handle, nat.ptr(x, nat.f64p), self.dimension,
                                                  x.shape[1], nat.ptr(t, nat.f64p), self.trailing))
        return x

    def close(self):
        self._factor.close()


class FactorSolve:
    """Solves with a supernodal factor (FactorSolve.hpp:59-100): B <- A^-1 B for many right-hand sides."""

    def __init__(self, factor: SupernodalFactor):
        self.factor = factor
        self.device_seconds = 0.0

    def solve(self, b):
        """In place on a float64 array (n,) or (n, k) (host: Fortran order or a column; device: a torch tensor whose
        columns are contiguous, i.e. the transpose of a contiguous (k, n) tensor, or a 1-D tensor)."""
        lib = nat.load()
        if isinstance(b, np.ndarray):
            if b.dtype != np.float64:
                raise ValueError("FactorSolve.solve: expected float64 right-hand sides")
            if b.ndim == 1:
                if not b.flags.c_contiguous:
                    raise ValueError("FactorSolve.solve: expected a contiguous vector")
                n, k, ld = b.shape[0], 1, b.shape[0]
            else:
                if not b.flags.f_contiguous:
                    raise ValueError("FactorSolve.solve: expected a column-major (Fortran-order) block")
                n, k = b.shape
                ld = n
            _check(lib.oosgpu_solve(self.factor._handle, nat.ptr(b, nat.f64p), ld, k))
        else:
            if b.dim() == 1:
                n, k, ld = b.shape[0], 1, b.shape[0]
            else:
                n, k = b.shape
                if b.stride(0) != 1:
                    raise ValueError("FactorSolve.solve: expected a device block with contiguous columns")
                ld = b.stride(1) if k > 1 else n
            _check(lib.oosgpu_solve_device(self.factor._handle, b.data_ptr(), ld, k))
        self.device_seconds = float(lib.oosgpu_last_solve_seconds(self.factor._handle))
        return b


def _block_layout(a):
    """(rows, columns, leading dimension) of a column-major host array or a device tensor with contiguous columns."""
    if isinstance(a, np.ndarray):
        if a.ndim == 1:
            return a.shape[0], 1, a.shape[0]
        if not a.flags.f_contiguous:
            raise ValueError("expected a column-major (Fortran-order) block")
        return a.shape[0], a.shape[1], a.shape[0]
    if a.dim() == 1:
        return a.shape[0], 1, a.shape[0]
    if a.stride(0) != 1:
        raise ValueError("expected a device block with contiguous columns")
    return a.shape[0], a.shape[1], (a.stride(1) if a.shape[1] > 1 else a.shape[0])


@dataclass
class RefinementInfo:
    steps: int
    residual: float
    device_seconds: float
    backward_error: float


def solve_refined(factor: SupernodalFactor, b, x, tolerance: float = 1.0e-10, max_steps: int = 10,
                  krylov: int = 0) -> RefinementInfo:
    """X = A^-1 B refined in FP64 on the device until every column's normwise backward error is at most `tolerance`
    (oosgpu_solve_refined): B and X float64, both host (column-major) or both device tensors. krylov > 0: each
    correction by GMRES with at most that many Krylov vectors, the factor's solve as preconditioner (GMRES-IR)."""
    lib = nat.load()
    n, k, ldb = _block_layout(b)
    nx, kx, ldx = _block_layout(x)
    if (n, k) != (nx, kx):
        raise ValueError("solve_refined: B and X differ in shape")
    options = nat.RefineOptions(tolerance, max_steps, krylov)
    info = nat.RefineInfo()
    if isinstance(b, np.ndarray):
        if b.dtype != np.float64 or x.dtype != np.float64:
            raise ValueError("solve_refined: expected float64 blocks")
        _check(lib.oosgpu_solve_refined(factor._handle, nat.ptr(b, nat.f64p), ldb, nat.ptr(x, nat.f64p), ldx, k,
                                        ctypes.byref(options), ctypes.byref(info)))
    else:
        _check(lib.oosgpu_solve_refined_device(factor._handle, b.data_ptr(), ldb, x.data_ptr(), ldx, k,
                                               ctypes.byref(options), ctypes.byref(info)))
    return RefinementInfo(int(info.steps), float(info.residual), float(info.device_seconds),
                          float(info.backward_error))


# ---- the shifted pencil of an eigenvalue analysis --------------------------------------------------------------------


@dataclass
class ShiftFactorisation:
    """ShiftFactorisation (include/oos/linalg/eigen/ShiftedPencil.hpp:34-42): the inertia of K - shift M, whose
    negative count is the Sturm count of the shift."""

    shift: float
    inertia: Inertia
    two_by_two: int = 0
    delayed: int = 0

    @property
    def sturm_count(self) -> int:
        return self.inertia.negative

    @property
    def is_singular(self) -> bool:
        return self.inertia.zero > 0


class SparsePencil:
    """SparsePencil (include/oos/linalg/eigen/SparsePencil.hpp:29-85) on the GPU: the pencil (K, M) of two lower CSC
    matrices of one structure. factorise(shift) factorises S (K - shift M) S in indefinite mode (S the powers of two of
    PencilScaling); solve() applies (K - shift M)^-1 and multiply_mass() M to device blocks with contiguous columns
    (torch tensors) or to column-major host arrays (copied through the device)."""

    _CREATE = "oosgpu_pencil_create"
    _NAME = "SparsePencil"

    def __init__(self, symbolic: SymbolicFactor, stiffness: SymmetricCsc, mass: SymmetricCsc, device: int = 0):
        offsets = np.ascontiguousarray(stiffness.offsets, dtype=np.int64)
        rows = np.ascontiguousarray(stiffness.rows, dtype=np.int32)
        if not (np.array_equal(offsets, np.asarray(mass.offsets)) and np.array_equal(rows, np.asarray(mass.rows))):
            raise ValueError(f"{self._NAME}: the two matrices differ in structure")
        k = np.ascontiguousarray(stiffness.values, dtype=np.float64)
        m = np.ascontiguousarray(mass.values, dtype=np.float64)
        self.symbolic = symbolic
        self.device = device
        self._handle = nat.vp()
        _check(getattr(nat.load(), self._CREATE)(symbolic._handle, device, len(offsets) - 1, nat.ptr(offsets, nat.i64p),
                                                 nat.ptr(rows, nat.i32p), nat.ptr(k, nat.f64p), nat.ptr(m, nat.f64p),
                                                 ctypes.byref(self._handle)))
        self._dimension = len(offsets) - 1

    @property
    def dimension(self) -> int:
        return self._dimension

    @property
    def stream(self) -> int:
        return int(nat.load().oosgpu_pencil_stream(self._handle) or 0)

    def _properties(self):
        bound = ctypes.c_double()
        lumped = ctypes.c_int32()
        count = ctypes.c_int64()
        _check(nat.load().oosgpu_pencil_properties(self._handle, ctypes.byref(bound), ctypes.byref(lumped),
                                                   ctypes.byref(count)))
        return bound.value, bool(lumped.value), int(count.value)

    @property
    def diagonal_rayleigh_bound(self) -> float:
        return self._properties()[0]

    @property
    def has_diagonal_mass(self) -> bool:
        return self._properties()[1]

    @property
    def factorisation_count(self) -> int:
        return self._properties()[2]

    def factorise(self, shift: float) -> ShiftFactorisation:
        info = nat.FactorInfo()
        _check(nat.load().oosgpu_pencil_factorise(self._handle, float(shift), ctypes.byref(info)))
        return ShiftFactorisation(float(shift), Inertia(int(info.positive), int(info.negative), int(info.zero)),
                                  int(info.two_by_two), int(info.delayed))

    def _device_call(self, fn, *blocks):
        """Runs fn on device blocks; host blocks are copied to the device and the last one back."""
        if all(not isinstance(b, np.ndarray) for b in blocks):
            fn(*blocks)
            return blocks[-1]
        import torch

        staged = []
        for b in blocks:
            n, k, _ = _block_layout(b)
            t = torch.empty((k, n), dtype=torch.float64, device=f"cuda:{self.device}").t()
            t.copy_(torch.from_numpy(np.asarray(b).reshape(n, k, order="F")))
            staged.append(t)
        fn(*staged)
        torch.cuda.synchronize(self.device)
        out = blocks[-1]
        out.reshape(out.shape[0], -1, order="F")[...] = staged[-1].cpu().numpy()
        return out

    def solve(self, block):
        """X <- (K - shift M)^-1 X with the last factor, in place."""
        def run(x):
            n, k, ld = _block_layout(x)
            _check(nat.load().oosgpu_pencil_solve_device(self._handle, x.data_ptr(), ld, k))
        return self._device_call(run, block)

    def multiply_mass(self, x, y):
        """Y <- M X (distinct storage)."""
        def run(a, b):
            n, k, ldx = _block_layout(a)
            _, _, ldy = _block_layout(b)
            _check(nat.load().oosgpu_pencil_multiply_mass_device(self._handle, a.data_ptr(), ldx, b.data_ptr(), ldy, k))
        return self._device_call(run, x, y)

    def close(self):
        if self._handle:
            nat.load().oosgpu_pencil_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BucklingPencil(SparsePencil):
    """BucklingPencil (include/oos/linalg/eigen/BucklingPencil.hpp:29-72) on the GPU: K phi = lambda B phi with B = -K_d,
    K the stiffness and K_d the differential stiffness of a preload, two lower CSC matrices of one structure.
    factorise(shift) factorises S (K + shift K_d) S in indefinite mode (S the powers of two of K's diagonal);
    multiply_mass() applies B = -K_d. BlockLanczos.solve on it finds the load factors nearest 0 of either sign
    (BlockLanczos::solveBuckling)."""

    _CREATE = "oosgpu_pencil_create_buckling"
    _NAME = "BucklingPencil"

    def __init__(self, symbolic: SymbolicFactor, stiffness: SymmetricCsc, differential: SymmetricCsc, device: int = 0):
        super().__init__(symbolic, stiffness, differential, device)
