"""CPU restatement of the learned start block's network (TEST INFRASTRUCTURE ONLY: the checker of the GPU kernels of
o_o_solver_b200/csrc/device/mlp_kernels.cu, never called by the product): the same multilayer perceptron
(inputs -> hidden -> hidden -> outputs, ReLU after each hidden layer, parameters flat as W1 (inputs x hidden,
row-major), b1, W2, b2, W3, b3), its mean squared error and its gradients by the chain rule, in FP64 with numpy.
The network has no counterpart in the reference: this is the oracle of its gradients."""

import numpy as np


def unpack(parameters, inputs, hidden, outputs):
    p = np.asarray(parameters, dtype=np.float64)
    sizes = [inputs * hidden, hidden, hidden * hidden, hidden, hidden * outputs, outputs]
    parts = np.split(p, np.cumsum(sizes)[:-1])
    return (parts[0].reshape(inputs, hidden), parts[1], parts[2].reshape(hidden, hidden), parts[3],
            parts[4].reshape(hidden, outputs), parts[5])


def forward(parameters, x, shape):
    w1, b1, w2, b2, w3, b3 = unpack(parameters, *shape)
    h1 = np.maximum(x @ w1 + b1, 0.0)
    h2 = np.maximum(h1 @ w2 + b2, 0.0)
    return h1, h2, h2 @ w3 + b3


def loss_and_gradients(parameters, x, t, shape):
    """(mean squared error over the batch and the outputs, its gradient flat like the parameters)."""
    x = np.asarray(x, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    w1, b1, w2, b2, w3, b3 = unpack(parameters, *shape)
    h1, h2, y = forward(parameters, x, shape)
    count = y.size
    dy = 2.0 * (y - t) / count
    dw3 = h2.T @ dy
    db3 = dy.sum(axis=0)
    dh2 = (dy @ w3.T) * (h2 > 0)
    dw2 = h1.T @ dh2
    db2 = dh2.sum(axis=0)
    dh1 = (dh2 @ w2.T) * (h1 > 0)
    dw1 = x.T @ dh1
    db1 = dh1.sum(axis=0)
    loss = float(((y - t) ** 2).mean())
    return loss, np.concatenate([dw1.ravel(), db1, dw2.ravel(), db2, dw3.ravel(), db3])
