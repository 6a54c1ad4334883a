"""CPU oracle of the warm-start MLP's forward and backward passes.

TEST INFRASTRUCTURE ONLY (imported by tests/): the checker for the device MLP's gradients.
There is no reference implementation to pin it to (snoo.py has no surrogate); its own
backward pass is pinned to central finite differences of its forward pass in float64
(tests/test_oracle.py), and with ``bf16=True`` it rounds to BF16 at the points the device
rounds: weights, the padded input, hidden activations and the output gradients fed to the
GEMMs.  Sums are float64.

Network: Z_l = H_{l-1} W_l^T + b_l; H_l = GELU(Z_l) (exact, 0.5 z (1 + erf(z / sqrt 2)))
for hidden layers; Y = Z_L; loss = mean((Y - T)^2).
"""

import math

import numpy as np

_erf = np.vectorize(math.erf)


def bf16(x):
    """Round float values to BF16 (nearest, ties to even) and return them as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32)).view(np.uint32).astype(np.uint64)
    r = ((a + 0x7FFF + ((a >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def forward(W, b, X, bf=False):
    """W, b: per-layer weights [out, in] and biases; X [B, in0].  Returns (Y, cache)."""
    r = bf16 if bf else (lambda v: np.asarray(v, dtype=np.float64))
    H = r(X)
    cache = [(None, H)]
    L = len(W)
    for l in range(L):
        Z = H @ r(W[l]).T + b[l]
        if l < L - 1:
            H = r(gelu(Z))
            cache.append((Z, H))
        else:
            cache.append((Z, None))
            H = Z
    return H, cache


def backward(W, b, X, T, bf=False):
    """Gradients of mean((Y - T)^2) w.r.t. every W_l, b_l, and the loss."""
    r = bf16 if bf else (lambda v: np.asarray(v, dtype=np.float64))
    Y, cache = forward(W, b, X, bf)
    dZ = 2.0 * (Y - T) / Y.size
    grads = [None] * len(W)
    for l in range(len(W) - 1, -1, -1):
        Hprev = cache[l][1]
        dZr = r(dZ)
        grads[l] = (dZr.T @ Hprev, dZ.sum(0))
        if l > 0:
            dH = dZr @ r(W[l])
            dZ = dH * gelu_grad(cache[l][0])
    return grads, float(np.mean((Y - T) ** 2))
