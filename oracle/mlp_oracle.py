"""CPU restatement (numpy, FP64) of the surrogate network's forward and
backward passes, the checker of the tensor-core kernels (lcg_mlp_*) in the
GPU tests. Test infrastructure only: the library never calls it.

The network is lcurve_re_b200.mlp.MLP: an FP32 input layer, BF16 hidden and
output layers with FP32 accumulation, GELU, mean squared error. The oracle
rounds to BF16 exactly where the kernels store BF16 (weights of layers >= 1,
activations, pre-activations, gradients), and keeps every sum in FP64, so
the kernels differ from it only by FP32 accumulation order and the
occasional BF16 rounding tie.
"""
import numpy as np
from scipy.special import erf


def bf16(x):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32)).view(np.uint32)
    r = (a + np.uint32(0x7FFF) + ((a >> np.uint32(16)) & np.uint32(1))) & np.uint32(0xFFFF0000)
    return r.view(np.float32).astype(np.float64)


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def forward(W, b, x):
    """W, b: lists of layer weights [out x in] and biases (float arrays);
    x: [n x nin]. Returns the output and the saved activations."""
    depth = len(W) - 1
    x = np.asarray(x, dtype=np.float64)
    z = x @ np.asarray(W[0], np.float64).T + b[0]
    zs, ys = [bf16(z)], [bf16(gelu(z))]
    for l in range(1, depth):
        z = ys[-1] @ bf16(W[l]).T + b[l]
        zs.append(bf16(z))
        ys.append(bf16(gelu(z)))
    out = ys[-1] @ bf16(W[depth]).T + b[depth]
    return out, zs, ys


def backward(W, b, x, target):
    """Gradients of mean((out - target)^2) with the kernels' BF16 points."""
    depth = len(W) - 1
    out, zs, ys = forward(W, b, x)
    n, nout = out.shape
    g = bf16(2.0 * (out - target) / (n * nout))
    dW = [None] * (depth + 1)
    db = [None] * (depth + 1)
    dW[depth] = g.T @ ys[depth - 1]
    db[depth] = g.sum(axis=0)
    for l in range(depth, 0, -1):
        g = bf16((g @ bf16(W[l])) * gelu_grad(zs[l - 1]))
        if l - 1 > 0:
            dW[l - 1] = g.T @ ys[l - 2]
        else:
            dW[0] = g.T @ np.asarray(x, np.float64)
        db[l - 1] = g.sum(axis=0)
    loss = float(np.mean((out - target) ** 2))
    return loss, dW, db, out
