"""TEST INFRASTRUCTURE ONLY: an FP64 NumPy restatement of the learned
radiance cache's network (hydra_lotus_b200/csrc/radiance_cache.cu), the
checker of its tensor-core forward and backward passes. Only tests may use
it; the product never does.

The cache has no counterpart in hydra-lotus, so nothing here follows a
reference file: it restates the CUDA kernels' arithmetic in FP64 with the
same BF16 roundings where the kernels store BF16 operands (inputs, weights,
activations after the ReLU, loss gradients, masked layer gradients).
"""

import numpy as np

LAYERS = 6
WIDTH = 64
OUTPUTS = 16
WEIGHTS = 5 * 64 * 64 + 64 * 16


def bf16(x):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def layers(weights):
    """The six weight matrices W[in][out] from the flat FP32 array."""
    w = np.asarray(weights, dtype=np.float64)
    out = [w[l * 4096:(l + 1) * 4096].reshape(64, 64) for l in range(5)]
    out.append(w[5 * 4096:5 * 4096 + 64 * 16].reshape(64, 16))
    return out


def forward(weights, inputs, quantize=True):
    """Activations H_0..H_5 (BF16-rounded) and the outputs y (n x 16).
    quantize=False skips the roundings (plain FP64, for finite differences)."""
    q = bf16 if quantize else (lambda a: np.asarray(a, dtype=np.float64))
    W = [q(m) for m in layers(weights)]
    H = [q(inputs)]
    for l in range(5):
        H.append(q(np.maximum(H[-1] @ W[l], 0.0)))
    return H, H[5] @ W[5]


def infer(weights, inputs):
    return forward(weights, inputs)[1][:, :3]


def loss_value(weights, inputs, targets, quantize=False):
    """The relative L2 loss with its denominator evaluated, not held."""
    y = forward(weights, inputs, quantize)[1][:, :3]
    d = y - np.asarray(targets, dtype=np.float64)
    return float(np.sum(d * d / (y * y + 0.01)))


def gradients(weights, inputs, targets, quantize=True):
    """Weight gradients (flat, WEIGHTS), input gradients (n x 64) and the
    loss sum_s,c (y - t)^2 / (y^2 + 0.01), its denominator held constant."""
    q = bf16 if quantize else (lambda a: np.asarray(a, dtype=np.float64))
    W = [q(m) for m in layers(weights)]
    H, y = forward(weights, inputs, quantize)
    n = inputs.shape[0]
    t = np.asarray(targets, dtype=np.float64)
    d = y[:, :3] - t
    denom = y[:, :3] ** 2 + 0.01
    loss = float(np.sum(d * d / denom))
    dy = np.zeros((n, OUTPUTS))
    dy[:, :3] = 2.0 * d / denom
    cur = q(dy)
    grads = [None] * LAYERS
    dx = None
    for l in range(LAYERS - 1, -1, -1):
        grads[l] = H[l].T @ cur
        dh = cur @ W[l].T
        if l > 0:
            cur = q(np.where(H[l] > 0.0, dh, 0.0))
        else:
            dx = dh
    flat = np.concatenate([g.ravel() for g in grads])
    return flat, dx, loss


SH_C = [0.28209479177387814, 0.48860251190291987, 1.0925484305920792, 0.94617469575755997,
        0.31539156525251999, 0.54627421529603959, 0.59004358992664352, 2.8906114426405538,
        0.45704579946446572, 0.3731763325901154, 1.4453057213202769]


def sh_basis(d):
    """Real spherical harmonics of bands 0..3 (the kernel's order)."""
    x, y, z = d[:, 0], d[:, 1], d[:, 2]
    xx, yy, zz = x * x, y * y, z * z
    c = SH_C
    return np.stack([
        np.full_like(x, c[0]), -c[1] * y, c[1] * z, -c[1] * x,
        c[2] * x * y, -c[2] * y * z, c[3] * zz - c[4], -c[2] * x * z, c[5] * (xx - yy),
        c[6] * y * (-3.0 * xx + yy), c[7] * x * y * z, c[8] * y * (1.0 - 5.0 * zz),
        c[9] * z * (5.0 * zz - 3.0), c[8] * x * (1.0 - 5.0 * zz), c[10] * z * (xx - yy),
        c[6] * x * (-xx + 3.0 * yy)], axis=1)


def encode_direct(records):
    """Inputs 32..63 of raw records (n x 16): everything but the hash grid."""
    r = np.asarray(records, dtype=np.float64)
    n = r.shape[0]
    out = np.zeros((n, 32))
    out[:, 0:16] = sh_basis(r[:, 4:7])
    out[:, 16:19] = r[:, 8:11]
    out[:, 19] = r[:, 3]
    out[:, 20:23] = r[:, 12:15]
    out[:, 23] = 1.0
    return out
