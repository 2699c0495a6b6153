"""ctypes access to the oracle: the reference's own linear algebra (oracle/_ref/liboos_ref.so, built from the
reference's sources by oracle/Makefile) and the C restatement of its factorisation (oracle/_ref/libldlt_port.so,
oracle/ldlt_port.c).

TEST INFRASTRUCTURE ONLY: the checker of the GPU path (tests, smoke) and the timed CPU baseline of the benchmark. The
product (o_o_solver_b200) never imports this module.
"""

from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "liboos_ref.so")
PORT_LIB = os.path.join(HERE, "_ref", "libldlt_port.so")

_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_f64p = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p

_ref = None
_port = None


def _ptr(array, kind):
    if array is None:
        return None
    return array.ctypes.data_as(kind)


def reference_available() -> bool:
    return os.path.exists(REF_LIB)


def ref_lib():
    """The reference library (oracle/_ref/liboos_ref.so); raises when it was not built."""
    global _ref
    if _ref is not None:
        return _ref
    if not os.path.exists(REF_LIB):
        raise RuntimeError(f"the reference oracle is not built: {REF_LIB} (make -C oracle)")
    lib = ctypes.CDLL(REF_LIB)
    lib.ref_last_error.restype = ctypes.c_char_p
    lib.ref_analyse.restype = _vp
    lib.ref_analyse.argtypes = [ctypes.c_int32, _i64p, _i32p, _i32p, _f64p, ctypes.c_int, _i32p, ctypes.c_int,
                                ctypes.c_int]
    lib.ref_analyse_trailing.restype = _vp
    lib.ref_analyse_trailing.argtypes = [ctypes.c_int32, _i64p, _i32p, _i32p, _f64p, ctypes.c_int, _i32p, ctypes.c_int,
                                         ctypes.c_int, _i32p, ctypes.c_int32]
    lib.ref_partial_factorise.restype = _vp
    lib.ref_partial_factorise.argtypes = [_vp, ctypes.c_int32, _i64p, _i32p, _f64p, ctypes.c_int, _f64p]
    lib.ref_partial_free.argtypes = [_vp]
    lib.ref_partial_condense.argtypes = [_vp, _f64p, ctypes.c_int64, _f64p]
    lib.ref_partial_recover.argtypes = [_vp, _f64p, ctypes.c_int64, _f64p]
    lib.ref_symbolic_free.argtypes = [_vp]
    lib.ref_sym_sizes.argtypes = [_vp, _i64p]
    lib.ref_sym_flops.restype = ctypes.c_double
    lib.ref_sym_flops.argtypes = [_vp]
    lib.ref_sym_times.argtypes = [_vp, _f64p]
    lib.ref_sym_node_order.argtypes = [_vp, _i32p]
    lib.ref_sym_first_columns.argtypes = [_vp, _i32p]
    lib.ref_sym_supernodes.argtypes = [_vp, _i32p, _i32p]
    lib.ref_sym_rows.argtypes = [_vp, _i64p, _i32p]
    lib.ref_factorise.restype = _vp
    lib.ref_factorise.argtypes = [_vp, ctypes.c_int32, _i64p, _i32p, _f64p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_double, ctypes.c_int, _f64p]
    lib.ref_factor_free.argtypes = [_vp]
    lib.ref_factor_info.argtypes = [_vp, _i64p, _f64p]
    lib.ref_factor_panel.argtypes = [_vp, ctypes.c_int32, _i64p, _i64p, _f64p, _i32p, _f64p]
    lib.ref_solve.argtypes = [_vp, _f64p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int, _f64p]
    lib.ref_modes.argtypes = [_vp, ctypes.c_int32, _i64p, _i32p, _f64p, _f64p, ctypes.c_double, ctypes.c_double,
                              ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int, ctypes.c_int, _f64p,
                              ctypes.c_int64, _f64p, _f64p, ctypes.c_int64, _i64p, _f64p]
    lib.ref_buckling.argtypes = lib.ref_modes.argtypes
    lib.ref_pencil_scale.argtypes = [ctypes.c_int32, _i64p, _i32p, _f64p, _f64p]
    lib.ref_symmetric_eigen.argtypes = [_f64p, ctypes.c_int64, ctypes.c_int64, _f64p, _f64p]
    lib.ref_sturm_verify.argtypes = [ctypes.c_int64, _f64p, _i64p, ctypes.c_int64, _f64p, _f64p]
    lib.ref_shift_next.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int64, ctypes.c_double, _f64p,
                                   ctypes.c_int64, _f64p, ctypes.c_int64, _f64p, ctypes.c_int64, _f64p, _f64p,
                                   ctypes.POINTER(ctypes.c_int32)]
    _ref = lib
    return lib


def _check(status):
    if status != 0:
        raise RuntimeError("reference: " + ref_lib().ref_last_error().decode())


@dataclass
class RefSymbolic:
    """The reference's SymbolicFactor of a node graph, with its arrays copied out."""

    handle: int
    node_count: int
    dof_count: int
    supernode_count: int
    node_order: np.ndarray  # node at each position
    first_column_of_position: np.ndarray
    first_position: np.ndarray
    parent: np.ndarray
    row_start: np.ndarray
    rows: np.ndarray
    flops: float
    panel_values: int
    factor_entries: int
    ordering_seconds: float
    analyse_seconds: float
    trailing_dofs: int = 0

    @property
    def first_column(self) -> np.ndarray:
        return self.first_column_of_position[self.first_position]

    def close(self):
        if self.handle:
            ref_lib().ref_symbolic_free(self.handle)
            self.handle = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def analyse(offsets, neighbours, weights, coords=None, method=0, given_order=None, amalgamate=True, threads=1,
            trailing_nodes=None):
    """ConstrainedOrdering + SymbolicFactor::analyse of the reference on a node graph (method 0 automatic, 1 AMD,
    2 nested dissection, 3 natural, 4 given order); trailing_nodes: a trailing set, ordered last (the boundary of a
    unit: the last supernode)."""
    lib = ref_lib()
    trailing = None if trailing_nodes is None else np.ascontiguousarray(trailing_nodes, dtype=np.int32)
    offsets = np.ascontiguousarray(offsets, dtype=np.int64)
    neighbours = np.ascontiguousarray(neighbours, dtype=np.int32)
    weights = np.ascontiguousarray(weights, dtype=np.int32)
    n = len(weights)
    coords = None if coords is None else np.ascontiguousarray(coords, dtype=np.float64)
    order = None if given_order is None else np.ascontiguousarray(given_order, dtype=np.int32)
    handle = lib.ref_analyse_trailing(n, _ptr(offsets, _i64p), _ptr(neighbours, _i32p), _ptr(weights, _i32p),
                                      _ptr(coords, _f64p), method if order is None else 4, _ptr(order, _i32p),
                                      1 if amalgamate else 0, threads, _ptr(trailing, _i32p),
                                      0 if trailing is None else len(trailing))
    if not handle:
        raise RuntimeError("reference analyse: " + lib.ref_last_error().decode())
    sizes = np.zeros(10, dtype=np.int64)
    lib.ref_sym_sizes(handle, _ptr(sizes, _i64p))
    nodes, dofs, count, row_entries = (int(v) for v in sizes[:4])
    node_order = np.zeros(nodes, dtype=np.int32)
    lib.ref_sym_node_order(handle, _ptr(node_order, _i32p))
    fcp = np.zeros(nodes + 1, dtype=np.int32)
    lib.ref_sym_first_columns(handle, _ptr(fcp, _i32p))
    first_position = np.zeros(count + 1, dtype=np.int32)
    parent = np.zeros(count, dtype=np.int32)
    lib.ref_sym_supernodes(handle, _ptr(first_position, _i32p), _ptr(parent, _i32p))
    row_start = np.zeros(count + 1, dtype=np.int64)
    rows = np.zeros(max(row_entries, 1), dtype=np.int32)
    lib.ref_sym_rows(handle, _ptr(row_start, _i64p), _ptr(rows, _i32p))
    times = np.zeros(2)
    lib.ref_sym_times(handle, _ptr(times, _f64p))
    return RefSymbolic(handle, nodes, dofs, count, node_order, fcp, first_position, parent, row_start,
                       rows[:row_entries], float(lib.ref_sym_flops(handle)), int(sizes[4]), int(sizes[5]),
                       float(times[0]), float(times[1]), int(sizes[8]))


@dataclass
class RefFactor:
    handle: int
    positive: int
    negative: int
    zero: int
    delayed: int
    two_by_two: int
    issue_count: int
    equation_of_largest: int
    largest_ratio: float
    kernel: int
    seconds: float

    def close(self):
        if self.handle:
            ref_lib().ref_factor_free(self.handle)
            self.handle = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def panel(self, s):
        lib = ref_lib()
        e = ctypes.c_int64()
        r = ctypes.c_int64()
        _check(lib.ref_factor_panel(self.handle, s, ctypes.byref(e), ctypes.byref(r), None, None, None))
        values = np.zeros((e.value, r.value), dtype=np.float64)  # column-major: [col][row]
        rows = np.zeros(r.value, dtype=np.int32)
        sub = np.zeros(max(e.value, 1), dtype=np.float64)
        _check(lib.ref_factor_panel(self.handle, s, ctypes.byref(e), ctypes.byref(r), _ptr(values, _f64p),
                                    _ptr(rows, _i32p), _ptr(sub, _f64p)))
        return values.T.copy(), rows, sub[:e.value]

    def solve(self, b, threads=1):
        """B <- A^-1 B for a (n,) or (n, k) array (returns a new array)."""
        lib = ref_lib()
        x = np.array(b, dtype=np.float64, order="F", copy=True)
        if x.ndim == 1:
            x = x.reshape(-1, 1, order="F")
        seconds = np.zeros(1)
        _check(lib.ref_solve(self.handle, _ptr(x, _f64p), x.shape[0], x.shape[1], threads, _ptr(seconds, _f64p)))
        self.solve_seconds = float(seconds[0])
        return x


def factorise(symbolic: RefSymbolic, offsets, rows, values, indefinite=False, family=-1, threads=1,
              max_ratio=1.0e7, bailout=0) -> RefFactor:
    lib = ref_lib()
    offsets = np.ascontiguousarray(offsets, dtype=np.int64)
    rows = np.ascontiguousarray(rows, dtype=np.int32)
    values = np.ascontiguousarray(values, dtype=np.float64)
    seconds = np.zeros(1)
    handle = lib.ref_factorise(symbolic.handle, symbolic.dof_count, _ptr(offsets, _i64p), _ptr(rows, _i32p),
                               _ptr(values, _f64p), 1 if indefinite else 0, family, threads, max_ratio, bailout,
                               _ptr(seconds, _f64p))
    if not handle:
        raise RuntimeError("reference factorise: " + lib.ref_last_error().decode())
    info = np.zeros(8, dtype=np.int64)
    ratio = ctypes.c_double()
    lib.ref_factor_info(handle, _ptr(info, _i64p), ctypes.byref(ratio))
    return RefFactor(handle, *(int(v) for v in info[:7]), float(ratio.value), int(info[7]), float(seconds[0]))


class RefPartial:
    """PartialFactor of the reference (src/linalg/supernodal/PartialFactor.cpp): the interior factorised, K* kept."""

    def __init__(self, symbolic, offsets, rows, values, family=-1):
        lib = ref_lib()
        self.dimension = symbolic.dof_count
        self.trailing = symbolic.trailing_dofs
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        rows = np.ascontiguousarray(rows, dtype=np.int32)
        values = np.ascontiguousarray(values, dtype=np.float64)
        schur = np.zeros((self.trailing, self.trailing), order="F")
        self.handle = lib.ref_partial_factorise(symbolic.handle, self.dimension, _ptr(offsets, _i64p),
                                                _ptr(rows, _i32p), _ptr(values, _f64p), family, _ptr(schur, _f64p))
        if not self.handle:
            raise RuntimeError("reference partial factorise: " + lib.ref_last_error().decode())
        self.schur_complement = schur

    def condense(self, loads):
        x = np.asfortranarray(np.asarray(loads, dtype=np.float64).reshape(self.dimension, -1))
        out = np.zeros((self.trailing, x.shape[1]), order="F")
        _check(ref_lib().ref_partial_condense(self.handle, _ptr(x, _f64p), x.shape[1], _ptr(out, _f64p)))
        return out

    def recover(self, loads, trailing_values):
        x = np.array(np.asarray(loads, dtype=np.float64).reshape(self.dimension, -1), order="F", copy=True)
        t = np.asfortranarray(np.asarray(trailing_values, dtype=np.float64).reshape(self.trailing, -1))
        _check(ref_lib().ref_partial_recover(self.handle, _ptr(x, _f64p), x.shape[1], _ptr(t, _f64p)))
        return x

    def close(self):
        if self.handle:
            ref_lib().ref_partial_free(self.handle)
            self.handle = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def modes(symbolic: RefSymbolic, offsets, rows, stiffness, mass, mode_count, block_size=8, family=-1, threads=1,
          vectors=True, lower=-np.inf, upper=np.inf, modes_per_shift=0, capacity=None, buckling=False):
    """SparsePencil + BlockLanczos::solve of the request (lower, upper, mode_count). shifts: one row per shift of
    (shift, purpose, sturm count, has run, block steps, restarts, converged). buckling: BucklingPencil instead, `mass`
    then being the differential stiffness K_d (BlockLanczos::solveBuckling, the load factors of K x = -lambda K_d x
    nearest 0)."""
    lib = ref_lib()
    solve = lib.ref_buckling if buckling else lib.ref_modes
    n = symbolic.dof_count
    offsets = np.ascontiguousarray(offsets, dtype=np.int64)
    rows = np.ascontiguousarray(rows, dtype=np.int32)
    stiffness = np.ascontiguousarray(stiffness, dtype=np.float64)
    mass = np.ascontiguousarray(mass, dtype=np.float64)
    capacity = capacity if capacity is not None else max(mode_count, 1)
    values = np.zeros(capacity)
    vecs = np.zeros((capacity, n)) if vectors else None
    shifts = np.zeros((64, 7))
    counts = np.zeros(5, dtype=np.int64)
    seconds = np.zeros(1)
    _check(solve(symbolic.handle, n, _ptr(offsets, _i64p), _ptr(rows, _i32p), _ptr(stiffness, _f64p),
                 _ptr(mass, _f64p), lower, upper, mode_count, block_size, modes_per_shift, family, threads,
                 _ptr(values, _f64p), capacity, _ptr(vecs, _f64p), _ptr(shifts, _f64p), 64,
                 _ptr(counts, _i64p), _ptr(seconds, _f64p)))
    found = int(counts[0])
    return {
        "eigenvalues": values[:found],
        "eigenvectors": None if vecs is None else vecs[:found].T.copy(),
        "shifts": shifts[: int(min(counts[2], 64))],
        "factorisations": int(counts[1]),
        "verified": int(counts[3]),
        "complete": bool(counts[4]),
        "seconds": float(seconds[0]),
    }


def pencil_scale(offsets, rows, values):
    lib = ref_lib()
    offsets = np.ascontiguousarray(offsets, dtype=np.int64)
    rows = np.ascontiguousarray(rows, dtype=np.int32)
    values = np.ascontiguousarray(values, dtype=np.float64)
    n = len(offsets) - 1
    scale = np.zeros(n)
    _check(lib.ref_pencil_scale(n, _ptr(offsets, _i64p), _ptr(rows, _i32p), _ptr(values, _f64p), _ptr(scale, _f64p)))
    return scale


def symmetric_eigen(a):
    """SmallEigenSolver::decompose (src/linalg/dense/SmallEigenSolver.cpp:261-297): (eigenvalues, eigenvectors)."""
    lib = ref_lib()
    a = np.asfortranarray(a, dtype=np.float64)
    p = a.shape[0]
    values = np.zeros(p)
    vectors = np.zeros((p, p), order="F")
    _check(lib.ref_symmetric_eigen(_ptr(a, _f64p), p, max(p, 1), _ptr(values, _f64p), _ptr(vectors, _f64p)))
    return values, vectors


def sturm_verify(points, sorted_values):
    """SturmCheck::addPoint then verify (src/linalg/eigen/SturmCheck.cpp) over (shift, count) points: the six
    values verified up to, verified count, has mismatch, mismatch lower, mismatch upper, expected * 1e6 + found."""
    lib = ref_lib()
    shifts = np.array([p[0] for p in points], dtype=np.float64)
    counts = np.array([p[1] for p in points], dtype=np.int64)
    values = np.ascontiguousarray(sorted_values, dtype=np.float64)
    result = np.zeros(6)
    _check(lib.ref_sturm_verify(len(points), _ptr(shifts, _f64p), _ptr(counts, _i64p), len(values),
                                _ptr(values, _f64p), _ptr(result, _f64p)))
    return result


def shift_next(lower, upper, mode_count, scale, verification, sorted_values, ritz, lanczos_shifts):
    """ShiftStrategy(request, scale).nextShift (src/linalg/eigen/ShiftStrategy.cpp:121-193): (shift, purpose)."""
    lib = ref_lib()
    verification = np.ascontiguousarray(verification, dtype=np.float64)
    values = np.ascontiguousarray(sorted_values, dtype=np.float64)
    ritz = np.ascontiguousarray(ritz, dtype=np.float64)
    shifts = np.ascontiguousarray(lanczos_shifts, dtype=np.float64)
    shift = np.zeros(1)
    purpose = ctypes.c_int32(0)
    _check(lib.ref_shift_next(lower, upper, mode_count, scale, _ptr(verification, _f64p), len(values),
                              _ptr(values, _f64p), len(ritz), _ptr(ritz, _f64p), len(shifts), _ptr(shifts, _f64p),
                              _ptr(shift, _f64p), ctypes.byref(purpose)))
    return float(shift[0]), int(purpose.value)


def port_lib():
    """The C restatement (oracle/_ref/libldlt_port.so)."""
    global _port
    if _port is not None:
        return _port
    if not os.path.exists(PORT_LIB):
        raise RuntimeError(f"the C restatement is not built: {PORT_LIB} (make -C oracle port)")
    lib = ctypes.CDLL(PORT_LIB)
    lib.port_factorise.argtypes = [ctypes.c_int32, ctypes.c_int32, _i32p, _i32p, _i64p, _i32p, _i64p, _i32p, _f64p,
                                   _f64p, _i64p, _i32p]
    lib.port_solve.argtypes = [ctypes.c_int32, ctypes.c_int32, _i32p, _i32p, _i64p, _i32p, _f64p, _f64p,
                               ctypes.c_int64, ctypes.c_int64]
    _port = lib
    return lib


class PortFactor:
    """The C restatement's factor of a symbolic structure (arrays as in oosgpu_symbolic_create)."""

    def __init__(self, dof_count, first_column, parent, row_start, rows, offsets, col_rows, values):
        lib = port_lib()
        self.n = int(dof_count)
        self.first_column = np.ascontiguousarray(first_column, dtype=np.int32)
        self.parent = np.ascontiguousarray(parent, dtype=np.int32)
        self.row_start = np.ascontiguousarray(row_start, dtype=np.int64)
        self.rows = np.ascontiguousarray(rows, dtype=np.int32)
        c = np.diff(self.first_column).astype(np.int64)
        r = np.diff(self.row_start)
        self.panel_offset = np.concatenate([[0], np.cumsum(c * (c + r))])
        self.panels = np.zeros(int(self.panel_offset[-1]))
        self.inertia = np.zeros(3, dtype=np.int64)
        zero = ctypes.c_int32()
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        col_rows = np.ascontiguousarray(col_rows, dtype=np.int32)
        values = np.ascontiguousarray(values, dtype=np.float64)
        self.status = lib.port_factorise(self.n, len(self.parent), _ptr(self.first_column, _i32p),
                                         _ptr(self.parent, _i32p), _ptr(self.row_start, _i64p),
                                         _ptr(self.rows, _i32p), _ptr(offsets, _i64p), _ptr(col_rows, _i32p),
                                         _ptr(values, _f64p), _ptr(self.panels, _f64p), _ptr(self.inertia, _i64p),
                                         ctypes.byref(zero))
        self.zero_pivot_equation = int(zero.value)

    def panel(self, s):
        c = int(self.first_column[s + 1] - self.first_column[s])
        r = int(self.row_start[s + 1] - self.row_start[s])
        values = self.panels[self.panel_offset[s]: self.panel_offset[s + 1]].reshape(c, c + r).T
        return values

    def solve(self, b):
        x = np.array(b, dtype=np.float64, order="F", copy=True)
        if x.ndim == 1:
            x = x.reshape(-1, 1, order="F")
        port_lib().port_solve(self.n, len(self.parent), _ptr(self.first_column, _i32p), _ptr(self.parent, _i32p),
                              _ptr(self.row_start, _i64p), _ptr(self.rows, _i32p), _ptr(self.panels, _f64p),
                              _ptr(x, _f64p), x.shape[0], x.shape[1])
        return x
