"""The learned start block of the eigenvalue analysis (no counterpart in the reference): over a sweep of designs of one
structure, a small network maps a design's variables to its lowest modes, expressed on a basis of modes the solver
computed for earlier designs, and the predicted modes give the first Lanczos run its start block. The solver's answer
does not depend on the start (the Sturm counts decide what is found and verified); a good start only shortens the runs.

- Network: a multilayer perceptron (inputs -> hidden -> hidden -> outputs, ReLU) in FP32 on the GPU, trained by
  full-batch Adam on the mean squared error; inference and training run on this library's kernels (oosgpu_mlp_*).
- Snapshot basis: the principal directions of the training designs' modes in the inner product of their mean mass
  (each mode's sign fixed by a seeded probe vector so that a mode keeps one sign across designs), the first
  `basis_size` of them.
- Targets: the orthogonal projector onto a design's wanted modes in the basis's coordinates, P = Q Q^T, Q an
  orthonormal basis of the modes' least-squares coefficients A = (Phi^T M Phi)^-1 Phi^T M Psi in the design's own
  mass M (the thicknesses change the mass several-fold): the subspace of the wanted modes, indifferent to their
  signs and to the order of modes that cross between designs (which make the coefficients of "mode j" jump); its
  upper triangle is the network's output.
- Start block: Phi U W, U the leading `modes` eigenvectors of the predicted projector, mixed by a seeded Gaussian
  (modes x block size) matrix, so that the block and one application of the operator span the predicted subspace.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _native as nat
from .linalg import _check

_f32p = ctypes.POINTER(ctypes.c_float)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


class Network:
    """oosgpu_mlp: inputs -> hidden -> hidden -> outputs on CUDA device `device`."""

    def __init__(self, inputs: int, hidden: int, outputs: int, seed: int = 0x5EED, device: int = 0):
        self.shape = (inputs, hidden, outputs)
        handle = nat.vp()
        _check(nat.load().oosgpu_mlp_create(inputs, hidden, outputs, seed, device, ctypes.byref(handle)))
        self._handle = handle

    @property
    def parameter_count(self) -> int:
        return int(nat.load().oosgpu_mlp_parameter_count(self._handle))

    @property
    def parameters(self) -> np.ndarray:
        out = np.zeros(self.parameter_count, dtype=np.float32)
        _check(nat.load().oosgpu_mlp_get_parameters(self._handle, out.ctypes.data_as(_f32p)))
        return out

    @parameters.setter
    def parameters(self, values):
        values = _f32(values)
        if values.shape != (self.parameter_count,):
            raise ValueError("Network: expected the flat parameter vector")
        _check(nat.load().oosgpu_mlp_set_parameters(self._handle, values.ctypes.data_as(_f32p)))

    def predict(self, x) -> np.ndarray:
        x = _f32(x)
        out = np.zeros((x.shape[0], self.shape[2]), dtype=np.float32)
        _check(nat.load().oosgpu_mlp_predict(self._handle, x.ctypes.data_as(_f32p), x.shape[0],
                                             out.ctypes.data_as(_f32p)))
        return out

    def gradients(self, x, t):
        """(gradient of the mean squared error, flat like the parameters; the loss)."""
        x, t = _f32(x), _f32(t)
        grads = np.zeros(self.parameter_count, dtype=np.float32)
        loss = ctypes.c_float()
        _check(nat.load().oosgpu_mlp_gradients(self._handle, x.ctypes.data_as(_f32p), t.ctypes.data_as(_f32p),
                                               x.shape[0], grads.ctypes.data_as(_f32p), ctypes.byref(loss)))
        return grads, float(loss.value)

    def train(self, x, t, epochs: int, rate: float = 1.0e-3) -> np.ndarray:
        """Full-batch Adam; the loss before each step."""
        x, t = _f32(x), _f32(t)
        losses = np.zeros(max(epochs, 1), dtype=np.float32)
        _check(nat.load().oosgpu_mlp_train(self._handle, x.ctypes.data_as(_f32p), t.ctypes.data_as(_f32p), x.shape[0],
                                           epochs, rate, losses.ctypes.data_as(_f32p)))
        return losses[:epochs]

    def close(self):
        if self._handle:
            nat.load().oosgpu_mlp_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def signed_modes(modes: np.ndarray, mass: np.ndarray, probe: np.ndarray) -> np.ndarray:
    """The modes (n x k, M-orthonormal) each signed so that probe^T M psi_j >= 0."""
    signs = np.sign(probe @ (mass[:, None] * modes))
    signs[signs == 0] = 1.0
    return modes * signs


def subspace_sines(modes: np.ndarray, predicted: np.ndarray, mass: np.ndarray) -> np.ndarray:
    """The sines of the principal angles between span(modes) and span(predicted) in the M inner product, increasing:
    the last one is how far the worst-placed direction of the modes lies from the predicted subspace."""

    def orthonormal(v):
        values, vectors = np.linalg.eigh(v.T @ (mass[:, None] * v))
        keep = values > values.max() * 1e-12
        return v @ (vectors[:, keep] / np.sqrt(values[keep]))

    cosines = np.linalg.svd(orthonormal(modes).T @ (mass[:, None] * orthonormal(predicted)), compute_uv=False)
    return np.sort(np.sqrt(np.clip(1.0 - cosines ** 2, 0.0, None)))


@dataclass
class SnapshotBasis:
    """An M-orthonormal basis (n x size) of the training designs' modes."""

    phi: np.ndarray

    @classmethod
    def of(cls, modes_of_designs, mass: np.ndarray, size: int) -> "SnapshotBasis":
        snapshots = np.concatenate(modes_of_designs, axis=1)  # n x (designs * modes)
        gram = snapshots.T @ (mass[:, None] * snapshots)
        values, vectors = np.linalg.eigh(gram)
        order = np.argsort(values)[::-1][:size]
        phi = snapshots @ (vectors[:, order] / np.sqrt(np.maximum(values[order], 1e-300)))
        return cls(phi)

    def coefficients(self, modes: np.ndarray, mass: np.ndarray) -> np.ndarray:
        """Phi^T M psi_j (size x k)."""
        return self.phi.T @ (mass[:, None] * modes)

    def least_squares(self, modes: np.ndarray, mass: np.ndarray) -> np.ndarray:
        """The coefficients A (size x k) of the M-closest combinations Phi A of the basis to the modes."""
        return np.linalg.solve(self.phi.T @ (mass[:, None] * self.phi), self.coefficients(modes, mass))


@dataclass
class LearnedStart:
    """A trained start-block predictor for one structure: the basis, the network, the input scaling, the mixing."""

    basis: SnapshotBasis
    network: Network
    mean: np.ndarray
    scale: np.ndarray
    modes: int
    mixing: np.ndarray  # modes x block size

    @classmethod
    def train(cls, designs: np.ndarray, modes_of_designs, masses, basis_size: int, block_size: int,
              hidden: int = 256, epochs: int = 2000, rate: float = 1.0e-3, seed: int = 0x5EED):
        """designs: (count x variables); modes_of_designs: the solver's modes of each (n x modes, M-orthonormal);
        masses: each design's lumped mass diagonal (a list), or one diagonal shared by all."""
        if isinstance(masses, np.ndarray) and masses.ndim == 1:
            masses = [masses] * len(modes_of_designs)
        rng = np.random.default_rng(seed)
        mean_mass = np.mean(masses, axis=0)
        probe = rng.standard_normal(mean_mass.shape[0])
        signed = [signed_modes(m, mass, probe) for m, mass in zip(modes_of_designs, masses)]
        basis = SnapshotBasis.of(signed, mean_mass, basis_size)
        modes = signed[0].shape[1]
        upper = np.triu_indices(basis_size)
        targets = []
        for m, mass in zip(signed, masses):
            q, _ = np.linalg.qr(basis.least_squares(m, mass))
            targets.append((q @ q.T)[upper])
        targets = np.stack(targets)
        mean = designs.mean(axis=0)
        scale = designs.std(axis=0) + 1e-12
        network = Network(designs.shape[1], hidden, targets.shape[1], seed=seed)
        losses = network.train((designs - mean) / scale, targets, epochs, rate)
        mixing = rng.standard_normal((modes, block_size))
        learned = cls(basis, network, mean, scale, modes, mixing)
        learned.losses = losses
        learned.probe = probe
        return learned

    def predicted_modes(self, design: np.ndarray) -> np.ndarray:
        """An M-orthonormal basis (n x modes) of the predicted subspace of the wanted modes."""
        size = self.basis.phi.shape[1]
        out = self.network.predict(((design - self.mean) / self.scale)[None, :])[0].astype(np.float64)
        projector = np.zeros((size, size))
        projector[np.triu_indices(size)] = out
        projector = projector + np.triu(projector, 1).T
        values, vectors = np.linalg.eigh(projector)
        return self.basis.phi @ vectors[:, np.argsort(values)[::-1][:self.modes]]

    def start_block(self, design: np.ndarray) -> np.ndarray:
        """The start block (block size x n, rows the vectors) for a design."""
        return np.ascontiguousarray((self.predicted_modes(design) @ self.mixing).T)


class DesignSweep:
    """The eigenvalue analyses of the designs of one structure: model_of(design) builds the model (a workloads.Model)
    of a design vector; every design shares the node order and supernode partition of `fixture` (node_order,
    first_position, parent: the reference's symbolic stage of the structure), so one symbolic factor serves all."""

    def __init__(self, model_of, fixture, modes: int, block_size: int = 8, device: int = 0):
        from .eigen import BlockLanczos, EigenRequest, LanczosOptions
        from .linalg import SymbolicFactor

        self.model_of = model_of
        self.order = np.asarray(fixture["node_order"], dtype=np.int32)
        self._fixture = fixture
        self._symbolic = None
        self.device = device
        self.request = EigenRequest(mode_count=modes)
        self.solver = BlockLanczos(LanczosOptions(block_size=block_size))
        self._symbolic_type = SymbolicFactor

    def _symbolic_of(self, model):
        if self._symbolic is None:
            f = self._fixture
            self._symbolic = self._symbolic_type.from_partition(model.offsets, model.neighbours, model.weights,
                                                                f["node_order"], f["first_position"], f["parent"])
        return self._symbolic

    def solve(self, design, start=None, vectors: bool = True):
        """(EigenSolution, lumped mass diagonal) of a design; start: a start block (block size x n array, rows the
        vectors), or None for the random one."""
        from .linalg import SparsePencil

        model = self.model_of(design)
        k = model.csc(self.order, 0)
        m = model.csc(self.order, 1)
        mass = m.values[m.offsets[:-1]].copy()
        pencil = SparsePencil(self._symbolic_of(model), k, m, device=self.device)
        try:
            block = None
            if start is not None:
                import torch

                block = torch.from_numpy(np.ascontiguousarray(start, dtype=np.float64)).to(f"cuda:{self.device}")
            solution = self.solver.solve(pencil, self.request, vectors=vectors, start_block=block)
        finally:
            pencil.close()
            model.close()
        return solution, mass
