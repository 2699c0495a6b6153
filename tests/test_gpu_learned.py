"""The learned start block on the GPU. The network's kernels: its gradients are the CPU oracle's (oracle/mlp.py, FP64)
to FP32 rounding, and training lowers its loss. The learned start: trained on the modes the solver itself computed for
a sweep of designs of a small wing box, it gives the same eigenvalues and the same Sturm verification as the random
start on designs it has not seen, in fewer Lanczos block steps."""

import os

import numpy as np
import pytest

from conftest import has_gpu

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "orderings")


@pytest.fixture(scope="module")
def gpu():
    if not has_gpu():
        pytest.skip("no CUDA device")
    import torch

    torch.cuda.init()
    return torch


def test_network_gradients_match_the_oracle(lib, gpu):
    import mlp as oracle_mlp

    from o_o_solver_b200.learned import Network

    rng = np.random.default_rng(7)
    shape = (5, 40, 9)
    net = Network(*shape, seed=3)
    x = rng.standard_normal((13, shape[0])).astype(np.float32)
    t = rng.standard_normal((13, shape[2])).astype(np.float32)
    grads, loss = net.gradients(x, t)
    ref_loss, ref_grads = oracle_mlp.loss_and_gradients(net.parameters, x, t, shape)
    assert abs(loss - ref_loss) <= 1e-5 * ref_loss
    scale = np.abs(ref_grads).max()
    assert np.abs(grads - ref_grads).max() <= 1e-5 * scale
    _, _, y = oracle_mlp.forward(net.parameters, x.astype(np.float64), shape)
    np.testing.assert_allclose(net.predict(x), y, rtol=0, atol=1e-5 * np.abs(y).max())
    net.close()


def test_network_training_lowers_the_loss(lib, gpu):
    from o_o_solver_b200.learned import Network

    rng = np.random.default_rng(11)
    x = rng.standard_normal((64, 6)).astype(np.float32)
    a = rng.standard_normal((6, 4))
    t = (np.tanh(x @ a)).astype(np.float32)
    net = Network(6, 64, 4, seed=5)
    losses = net.train(x, t, epochs=400, rate=3e-3)
    assert losses[-1] < 0.05 * losses[0]
    net.close()


def small_wing_box(design):
    from o_o_solver_b200 import workloads

    return workloads.Model(workloads.WingBoxSpec(thicknesses=tuple(design), span=2.0, chord=0.6, height=0.15))


def test_learned_start_keeps_the_answer_in_fewer_steps(lib, gpu):
    from o_o_solver_b200.learned import DesignSweep, LearnedStart

    fixture = dict(np.load(os.path.join(GOLDEN, "wingbox_small.npz")))
    modes = 10
    sweep = DesignSweep(small_wing_box, fixture, modes=modes, block_size=8)
    rng = np.random.default_rng(2026)
    designs = rng.uniform(0.001, 0.004, (30, 24))
    train, test = designs[:24], designs[24:]
    solved = [sweep.solve(d) for d in train]
    mass = solved[0][1]
    learned = LearnedStart.train(train, [s.eigenvectors for s, _ in solved], mass, basis_size=48, block_size=8,
                                 hidden=128, epochs=1500, rate=1e-3)
    assert learned.losses[-1] < 0.1 * learned.losses[0]
    random_steps = learned_steps = 0
    for d in test:
        plain, _ = sweep.solve(d, vectors=False)
        guided, _ = sweep.solve(d, start=learned.start_block(d), vectors=False)
        assert plain.is_complete and guided.is_complete
        assert plain.verified_count == guided.verified_count
        np.testing.assert_allclose(guided.eigenvalues, plain.eigenvalues, rtol=1e-9)
        random_steps += plain.block_steps
        learned_steps += guided.block_steps
    assert learned_steps < random_steps, (learned_steps, random_steps)
    learned.network.close()
