"""The host logic of the shift-invert Lanczos, on the CPU, against the reference's own classes (through the oracle's
shim): the dense symmetric eigensolver of the projected problems (SmallEigenSolver), the Sturm-count verification
(SturmCheck) and the choice of the next shift (ShiftStrategy), over seeded scenarios that reach their branches:
repeated roots, missing and surplus roots, contradicting counts, open and closed intervals, shifts already used.
SturmCheck and ShiftStrategy are pure arithmetic on the same doubles, so their results must agree bit for bit."""

import math

import numpy as np
import pytest

from o_o_solver_b200 import eigen
from o_o_solver_b200.linalg import SolverError


def symmetric_cases():
    rng = np.random.default_rng(11)
    yield "empty", np.zeros((0, 0))
    yield "one", np.array([[3.5]])
    yield "diagonal", np.diag([4.0, -1.0, 2.0, 2.0, 0.0])
    for p in (2, 3, 7, 16, 40, 96):
        a = rng.standard_normal((p, p))
        yield f"random{p}", a + a.T
    for p in (12, 35):
        q, _ = np.linalg.qr(rng.standard_normal((p, p)))
        d = np.repeat(rng.standard_normal(p // 3 + 1), 3)[:p]
        yield f"repeated{p}", (q * d) @ q.T
    t = np.diag(np.full(30, 2.0)) - np.diag(np.ones(29), 1) - np.diag(np.ones(29), -1)
    yield "tridiagonal30", t
    # graded, as the projected matrices of a shift-invert run are (1/(lambda - sigma) spans decades)
    q, _ = np.linalg.qr(rng.standard_normal((24, 24)))
    yield "graded24", (q * np.logspace(-10, 4, 24)) @ q.T


@pytest.mark.parametrize("name,a", list(symmetric_cases()), ids=lambda v: v if isinstance(v, str) else "")
def test_symmetric_eigen_matches_reference(name, a, lib, oracle_mod):
    values, vectors = eigen.symmetric_eigen(a)
    ref_values, ref_vectors = oracle_mod.symmetric_eigen(a)
    p = a.shape[0]
    if p == 0:
        assert values.size == 0
        return
    scale = max(np.abs(a).max(), 1e-300)
    assert np.all(np.diff(values) >= 0)
    np.testing.assert_allclose(values, ref_values, rtol=0, atol=1e-13 * p * scale)
    np.testing.assert_allclose(values, np.linalg.eigvalsh(a), rtol=0, atol=1e-13 * p * scale)
    # orthonormal eigenvectors with small residuals
    np.testing.assert_allclose(vectors.T @ vectors, np.eye(p), rtol=0, atol=1e-12 * p)
    assert np.abs(a @ vectors - vectors * values).max() <= 1e-12 * p * scale
    # the same sign rule as the reference: for every simple, well separated root the vectors agree; where two
    # components tie in magnitude (a symmetric vector of the tridiagonal case) rounding picks the sign, on both sides
    gaps = np.minimum(np.r_[np.inf, np.diff(values)], np.r_[np.diff(values), np.inf])
    for j in range(p):
        if gaps[j] > 1e-6 * scale:
            magnitudes = np.sort(np.abs(vectors[:, j]))[::-1]
            if p > 1 and magnitudes[1] > magnitudes[0] * (1 - 1e-9):
                sign = np.sign(vectors[:, j] @ ref_vectors[:, j])
                np.testing.assert_allclose(vectors[:, j], sign * ref_vectors[:, j], rtol=0, atol=1e-8)
                continue
            np.testing.assert_allclose(vectors[:, j], ref_vectors[:, j], rtol=0, atol=1e-8)
            assert vectors[int(np.argmax(np.abs(vectors[:, j]))), j] > 0


def test_symmetric_eigen_refuses_non_finite_terms(lib, oracle_mod):
    a = np.eye(4)
    a[2, 1] = math.nan
    with pytest.raises(SolverError):
        eigen.symmetric_eigen(a)
    with pytest.raises(RuntimeError):
        oracle_mod.symmetric_eigen(a)
    # only the lower triangle is read, as in the reference
    b = np.eye(4)
    b[1, 2] = math.nan
    values, _ = eigen.symmetric_eigen(b)
    np.testing.assert_array_equal(values, np.ones(4))


def spectrum(rng, count, repeated):
    values = np.sort(rng.uniform(-50.0, 400.0, count))
    if repeated:
        picks = rng.choice(count - 1, size=count // 5, replace=False)
        values[picks + 1] = values[picks]
        values.sort()
    return values


def sturm_scenarios():
    """(points, found eigenvalues) pairs: the counts are those of a true spectrum; the found set is the true one, or
    one with roots left out (a mismatch), or with a surplus root (more found than counted)."""
    rng = np.random.default_rng(2024)
    for case in range(120):
        true = spectrum(rng, int(rng.integers(4, 40)), repeated=case % 3 == 0)
        shifts = np.sort(rng.uniform(-80.0, 450.0, int(rng.integers(1, 6))))
        if case % 7 == 0:
            # a shift exactly on a root and one at the same place twice
            shifts = np.sort(np.r_[shifts, true[len(true) // 2], shifts[0]])
        points = [(float(s), int(np.searchsorted(true, s, side="left"))) for s in shifts]
        found = true.copy()
        kind = case % 4
        if kind == 1:
            drop = rng.choice(len(found), size=int(rng.integers(1, 4)), replace=False)
            found = np.delete(found, drop)
        elif kind == 2:
            found = np.sort(np.r_[found, rng.uniform(-50.0, 400.0)])
        elif kind == 3:
            found = found[: int(rng.integers(0, len(found)))]
        order = rng.permutation(len(points))
        yield case, [points[i] for i in order], found


@pytest.mark.parametrize("case,points,found", list(sturm_scenarios()), ids=lambda v: str(v) if isinstance(v, int)
                         else "")
def test_sturm_verification_is_the_reference_s(case, points, found, lib, oracle_mod):
    try:
        ref = oracle_mod.sturm_verify(points, found)
    except RuntimeError:
        with pytest.raises(SolverError):
            eigen.sturm_verify(points, found)
        return
    ours = eigen.sturm_verify(points, found)
    np.testing.assert_array_equal(ours._packed(), ref)


def test_contradicting_sturm_counts_are_refused(lib, oracle_mod):
    points = [(1.0, 5), (2.0, 3)]
    with pytest.raises(RuntimeError):
        oracle_mod.sturm_verify(points, [0.5])
    with pytest.raises(SolverError):
        eigen.sturm_verify(points, [0.5])


def test_sturm_without_points_is_refused(lib, oracle_mod):
    with pytest.raises(RuntimeError, match="no Sturm point"):
        oracle_mod.sturm_verify([], [1.0, 2.0])
    with pytest.raises(ValueError, match="no Sturm point"):
        eigen.sturm_verify([], [1.0, 2.0])


def shift_scenarios():
    rng = np.random.default_rng(77)
    requests = [(-math.inf, math.inf, 10), (0.0, math.inf, 25), (5.0, math.inf, 8), (10.0, 300.0, 0),
                (-math.inf, 120.0, 0), (50.0, 60.0, 0), (0.0, math.inf, 3)]
    for case in range(160):
        lower, upper, count = requests[case % len(requests)]
        scale = float(2.0 ** rng.integers(-3, 12))
        true = spectrum(rng, int(rng.integers(3, 30)), repeated=case % 4 == 0)
        shifts = np.sort(rng.uniform(-60.0, 420.0, int(rng.integers(1, 5))))
        points = [(float(s), int(np.searchsorted(true, s, side="left"))) for s in shifts]
        found = true.copy()
        if case % 3 == 1:
            found = np.delete(found, rng.choice(len(found), size=int(rng.integers(1, 3)), replace=False))
        elif case % 3 == 2:
            found = found[: int(rng.integers(0, len(found) + 1))]
        ritz = np.sort(np.r_[rng.uniform(-60.0, 420.0, int(rng.integers(0, 8))),
                             rng.choice(true, size=min(3, len(true)), replace=False)])
        lanczos = np.sort(rng.choice(np.r_[shifts, ritz], size=int(rng.integers(0, 4)), replace=True)) \
            if ritz.size else shifts[:1]
        yield case, (lower, upper, count, scale), points, found, ritz, lanczos


@pytest.mark.parametrize("case,request_,points,found,ritz,lanczos", list(shift_scenarios()),
                         ids=lambda v: str(v) if isinstance(v, int) else "")
def test_next_shift_is_the_reference_s(case, request_, points, found, ritz, lanczos, lib, oracle_mod):
    lower, upper, count, scale = request_
    try:
        packed = oracle_mod.sturm_verify(points, found)
    except RuntimeError:
        pytest.skip("contradicting counts: covered by the verification tests")
    verification = eigen.sturm_verify(points, found)
    np.testing.assert_array_equal(verification._packed(), packed)
    ref_shift, ref_purpose = oracle_mod.shift_next(lower, upper, count, scale, packed, found, ritz, lanczos)
    shift, purpose = eigen.next_shift(eigen.EigenRequest(lower, upper, count), scale, verification, found, ritz,
                                      lanczos)
    assert purpose == eigen.PURPOSES[ref_purpose]
    assert shift == ref_shift or (math.isnan(shift) and math.isnan(ref_shift)), (shift, ref_shift)


def test_next_shift_moves_off_used_shifts(lib, oracle_mod):
    """The shift the rules pick first was used already: the widest gap decides (ShiftStrategy.cpp:168-190)."""
    found = np.array([1.0, 2.0, 3.0])
    packed = oracle_mod.sturm_verify([(3.5, 3)], found)
    verification = eigen.sturm_verify([(3.5, 3)], found)
    first, _ = eigen.next_shift(eigen.EigenRequest(0.0, math.inf, 10), 1.0, verification, found, [], [])
    again, purpose = eigen.next_shift(eigen.EigenRequest(0.0, math.inf, 10), 1.0, verification, found, [], [first])
    ref = oracle_mod.shift_next(0.0, math.inf, 10, 1.0, packed, found, [], [first])
    assert again != first
    assert (again, purpose) == (ref[0], eigen.PURPOSES[ref[1]])
