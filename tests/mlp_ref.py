"""numpy restatement of the cost model's MLP (the CPU reference its device
kernels are checked against): y = relu(x W1 + b1) W2 + b2, loss = mean over
rows and outputs of (y - t)^2, and the loss gradient by hand-written
backpropagation.  Parameter layout: W1[in][hid], b1[hid], W2[hid][out],
b2[out], flattened in that order."""
import numpy as np


def unpack(p, n_in, n_hid, n_out):
    p = np.asarray(p, dtype=np.float64)
    k = 0
    W1 = p[k:k + n_in * n_hid].reshape(n_in, n_hid); k += n_in * n_hid
    b1 = p[k:k + n_hid]; k += n_hid
    W2 = p[k:k + n_hid * n_out].reshape(n_hid, n_out); k += n_hid * n_out
    b2 = p[k:k + n_out]
    return W1, b1, W2, b2


def forward(p, X, shape):
    W1, b1, W2, b2 = unpack(p, *shape)
    Z = np.asarray(X, np.float64) @ W1 + b1
    H = np.maximum(Z, 0.0)
    return H @ W2 + b2, Z, H


def loss_grad(p, X, T, shape):
    X = np.asarray(X, np.float64)
    T = np.asarray(T, np.float64)
    n, n_out = T.shape
    W1, b1, W2, b2 = unpack(p, *shape)
    Y, Z, H = forward(p, X, shape)
    E = Y - T
    loss = float((E ** 2).sum() / (n * n_out))
    dY = 2.0 * E / (n * n_out)
    gW2 = H.T @ dY
    gb2 = dY.sum(axis=0)
    dZ = (dY @ W2.T) * (Z > 0)
    gW1 = X.T @ dZ
    gb1 = dZ.sum(axis=0)
    return loss, np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2])
