"""CPU check of the learned boundary closure's network (test infrastructure only).

The closure has no reference counterpart; this module restates, in float64 numpy, the network the
library's tensor-core kernels compute (rtm3d-demo_b200/csrc/closure.cu) so that the tests can check
the GPU forward pass, the gradients and the feature layout:

    z1 = bf16(W1) x + b1,  h1 = bf16(tanh z1),  z2 = bf16(W2) h1 + b2,  h2 = tanh z2,
    y  = w3 . h2 + b3,     loss = mean_i (y_i - r_i)^2

x is the row of 64 BF16 features.  Gradients treat the BF16 roundings as identity (straight-through),
as the library's backward kernels do.  The backward pass runs on the tensor cores, whose operands
are BF16: the pre-activation gradients dz2 and dz1 enter the products dz2 W2, dz1^T x, dz2^T h1 and
the bias sums rounded to BF16, as restated in grad() below.
"""
import numpy as np

NIN, NHID = 64, 32
OFF_W1, OFF_B1 = 0, NHID * NIN
OFF_W2 = OFF_B1 + NHID
OFF_B2 = OFF_W2 + NHID * NHID
OFF_W3 = OFF_B2 + NHID
OFF_B3 = OFF_W3 + NHID
NPARAM = OFF_B3 + 1


def bf16(a: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    a = np.asarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def unpack(p: np.ndarray):
    p = np.asarray(p, np.float64)
    return (p[OFF_W1:OFF_B1].reshape(NHID, NIN), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(NHID, NHID),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3], p[OFF_B3])


def forward(p: np.ndarray, X: np.ndarray):
    """X: [n, 64] float32 holding BF16 values.  Returns y, h1, h2 (float64)."""
    W1, b1, W2, b2, w3, b3 = unpack(p)
    W1b = bf16(W1.astype(np.float32)).astype(np.float64)
    W2b = bf16(W2.astype(np.float32)).astype(np.float64)
    x = np.asarray(X, np.float64)
    h1 = bf16(np.tanh(x @ W1b.T + b1).astype(np.float32)).astype(np.float64)
    h2 = np.tanh(h1 @ W2b.T + b2)
    y = h2 @ w3 + b3
    return y, h1, h2


def grad(p: np.ndarray, X: np.ndarray, R: np.ndarray):
    """Gradient of mean (y - r)^2 and the loss."""
    W1, b1, W2, b2, w3, b3 = unpack(p)
    W2b = bf16(W2.astype(np.float32)).astype(np.float64)
    y, h1, h2 = forward(p, X)
    n = len(y)
    e = y - np.asarray(R, np.float64)
    dy = 2.0 * e / n
    dz2 = bf16(((dy[:, None] * w3[None, :]) * (1.0 - h2 * h2)).astype(np.float32)).astype(np.float64)
    dz1 = bf16(((dz2 @ W2b) * (1.0 - h1 * h1)).astype(np.float32)).astype(np.float64)
    x = np.asarray(X, np.float64)
    g = np.zeros(NPARAM)
    g[OFF_W1:OFF_B1] = (dz1.T @ x).ravel()
    g[OFF_B1:OFF_W2] = dz1.sum(0)
    g[OFF_W2:OFF_B2] = (dz2.T @ h1).ravel()
    g[OFF_B2:OFF_W3] = dz2.sum(0)
    g[OFF_W3:OFF_B3] = dy @ h2
    g[OFF_B3] = dy.sum()
    return g, float(np.mean(e * e))
