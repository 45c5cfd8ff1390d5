"""ORACLE (test infrastructure only): NumPy forward/backward of the learned
preconditioner's MLP, for the gradient check of the CUDA kernels (csrc/mlp.cu).

h1 = relu(W1 x + b1), h2 = relu(W2 h1 + b2), y = W3 h2 + b3, weights given as
the BF16-rounded values the kernels read (passed here as float64 arrays).
"""
import numpy


def forward(X, W1, b1, W2, b2, W3, b3):
    h1 = numpy.maximum(X @ W1.T + b1, 0.0)
    h2 = numpy.maximum(h1 @ W2.T + b2, 0.0)
    return h2 @ W3.T + b3, h1, h2


def backward(X, W1, W2, W3, h1, h2, dY):
    g = {}
    g["W3"] = dY.T @ h2
    g["b3"] = dY.sum(0)
    g2 = (dY @ W3) * (h2 > 0)
    g["W2"] = g2.T @ h1
    g["b2"] = g2.sum(0)
    g1 = (g2 @ W2) * (h1 > 0)
    g["W1"] = g1.T @ X
    g["b1"] = g1.sum(0)
    return g
