"""The host side of the learned start block, on the CPU: the principal-angle diagnostic, the snapshot basis and the
projector targets the network is trained on (no device needed; the network's kernels are tested in
test_gpu_learned.py)."""

import numpy as np

from o_o_solver_b200.learned import SnapshotBasis, signed_modes, subspace_sines


def m_orthonormal(v, mass):
    values, vectors = np.linalg.eigh(v.T @ (mass[:, None] * v))
    return v @ (vectors / np.sqrt(values))


def test_subspace_sines_of_known_angles():
    rng = np.random.default_rng(3)
    n = 60
    mass = rng.uniform(0.5, 4.0, n)
    q = m_orthonormal(rng.standard_normal((n, 5)), mass)
    # the same subspace, mixed and scaled: every angle zero (to the resolution of sqrt(1 - cos^2), about 1e-7)
    same = q @ rng.standard_normal((5, 5))
    np.testing.assert_allclose(subspace_sines(q, same, mass), 0.0, atol=1e-6)
    # one direction rotated by a known angle out of the subspace, in the M inner product
    outside = rng.standard_normal(n)
    outside -= q @ (q.T @ (mass * outside))
    outside /= np.sqrt(outside @ (mass * outside))
    theta = 0.3
    tilted = q.copy()
    tilted[:, 2] = np.cos(theta) * q[:, 2] + np.sin(theta) * outside
    sines = subspace_sines(q, tilted, mass)
    assert np.all(np.diff(sines) >= 0)
    np.testing.assert_allclose(sines[-1], np.sin(theta), rtol=1e-10)
    np.testing.assert_allclose(sines[:-1], 0.0, atol=1e-6)
    # an orthogonal subspace: every sine one
    other = m_orthonormal(np.c_[outside, rng.standard_normal((n, 4))], mass)
    other -= q @ (q.T @ (mass[:, None] * other))
    np.testing.assert_allclose(subspace_sines(q, other, mass), 1.0, rtol=1e-10)


def test_basis_least_squares_and_projector_targets():
    rng = np.random.default_rng(7)
    n, modes, designs = 80, 4, 6
    mean_mass = rng.uniform(1.0, 2.0, n)
    hidden = rng.standard_normal((n, 10))  # every design's modes lie in this span
    masses = [mean_mass * rng.uniform(0.5, 2.0) for _ in range(designs)]
    snapshots = [m_orthonormal(hidden @ rng.standard_normal((10, modes)), m) for m in masses]
    probe = rng.standard_normal(n)
    signed = [signed_modes(s, m, probe) for s, m in zip(snapshots, masses)]
    for s, m in zip(signed, masses):
        assert np.all(probe @ (m[:, None] * s) >= 0)
    basis = SnapshotBasis.of(signed, mean_mass, 10)
    np.testing.assert_allclose(basis.phi.T @ (mean_mass[:, None] * basis.phi), np.eye(10), atol=1e-9)
    for s, m in zip(signed, masses):
        a = basis.least_squares(s, m)
        np.testing.assert_allclose(basis.phi @ a, s, atol=1e-9)  # the modes lie in the basis: recovered exactly
        q, _ = np.linalg.qr(a)
        projector = q @ q.T
        np.testing.assert_allclose(projector @ projector, projector, atol=1e-10)
        assert abs(np.trace(projector) - modes) < 1e-10
        # its leading eigenvectors span the modes again
        values, vectors = np.linalg.eigh(projector)
        predicted = basis.phi @ vectors[:, np.argsort(values)[::-1][:modes]]
        assert subspace_sines(s, predicted, m)[-1] < 1e-6
