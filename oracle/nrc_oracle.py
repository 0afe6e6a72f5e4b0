"""CPU restatement of the neural radiance cache (hdcodex_b200/csrc/nrc.cu).

TEST INFRASTRUCTURE ONLY: the GPU tests compare the tensor-core kernels with
this numpy version (same hash-grid encoding, same BF16 rounding of weights,
activations and output gradients, FP32 accumulation) and check its analytic
gradients against central differences in FP64.

Network: 64 inputs (16 levels x 2 hash-grid features of the position,
direction, normal, roughness, wavelength, zeros), four 64-wide ReLU layers and
a 16-wide output layer (output 0 = radiance), no biases; loss = mean over the
batch of (p - y)^2 / (p^2 + 0.01), p held constant in the denominator.
Hash grid (Mueller et al. 2022): level l has N_l cells per axis; corners are
indexed densely, x + (N+1)(y + (N+1) z), while (N+1)^3 fits the table, else by
x ^ 2654435761 y ^ 805459861 z (uint32), masked to the table size.
"""
from __future__ import annotations

import numpy as np

LEVELS = 16
WIDTH = 64
OUT = 16
LAYER_ROWS = [64, 64, 64, 64, 16]
LAYER_OFFSET = [0, 4096, 8192, 12288, 16384]
WEIGHT_COUNT = 17408


def bf16(x):
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(np.shape(x))


def weights(mlp):
    return [np.asarray(mlp[LAYER_OFFSET[l]:LAYER_OFFSET[l] + LAYER_ROWS[l] * WIDTH], np.float32).reshape(LAYER_ROWS[l], WIDTH)
            for l in range(5)]


def corners(positions, resolution, log2_table, level):
    """(indices (n, 8), weights (n, 8)) of one level, as levelCorners() in nrc.cu."""
    n = np.uint64(resolution)
    fn = np.float32(resolution)
    p = np.clip(positions.astype(np.float32), 0.0, 1.0)
    s = (p * fn).astype(np.float32)
    c = np.minimum(s.astype(np.uint64), n - 1)
    f = (s - c.astype(np.float32)).astype(np.float32)
    side = n + np.uint64(1)
    mask = np.uint64((1 << log2_table) - 1)
    dense = int(side) ** 3 <= (1 << log2_table)
    idx = np.zeros((len(p), 8), np.uint64)
    w = np.zeros((len(p), 8), np.float32)
    for k in range(8):
        x = c[:, 0] + np.uint64(k & 1)
        y = c[:, 1] + np.uint64((k >> 1) & 1)
        z = c[:, 2] + np.uint64((k >> 2) & 1)
        if dense:
            h = x + side * (y + side * z)
        else:
            h = (x ^ ((y * np.uint64(2654435761)) & np.uint64(0xFFFFFFFF)) ^ ((z * np.uint64(805459861)) & np.uint64(0xFFFFFFFF)))
        idx[:, k] = (np.uint64(level) << np.uint64(log2_table)) + (h & mask)
        wx = f[:, 0] if (k & 1) else np.float32(1.0) - f[:, 0]
        wy = f[:, 1] if (k >> 1) & 1 else np.float32(1.0) - f[:, 1]
        wz = f[:, 2] if (k >> 2) & 1 else np.float32(1.0) - f[:, 2]
        w[:, k] = (wx * wy * wz).astype(np.float32)
    return idx.astype(np.int64), w


def encode(queries, grid, resolutions, log2_table):
    """Network inputs (n, 64) in float32 from query records (n, 12) and the
    FP32 table (rounded to FP16 as the GPU stores it)."""
    q = np.asarray(queries, np.float32)
    table = np.asarray(grid, np.float32).astype(np.float16).astype(np.float32).reshape(-1, 2)
    x = np.zeros((len(q), WIDTH), np.float32)
    for level in range(LEVELS):
        idx, w = corners(q[:, :3], resolutions[level], log2_table, level)
        feats = table[idx]  # (n, 8, 2)
        x[:, 2 * level] = np.einsum("nk,nk->n", w.astype(np.float64), feats[:, :, 0].astype(np.float64))
        x[:, 2 * level + 1] = np.einsum("nk,nk->n", w.astype(np.float64), feats[:, :, 1].astype(np.float64))
    x[:, 32:41] = q[:, 3:12]
    return x


def forward(queries, mlp, grid, resolutions, log2_table):
    """(prediction (n,), activations X_0..X_4) with the GPU's BF16 roundings."""
    ws = [bf16(w) for w in weights(mlp)]
    xs = [bf16(encode(queries, grid, resolutions, log2_table))]
    for l in range(4):
        xs.append(bf16(np.maximum(xs[-1] @ ws[l].T, 0.0)))
    z = xs[-1] @ ws[4].T
    return z[:, 0].astype(np.float32), xs


def gradients(queries, targets, mlp, grid, resolutions, log2_table):
    """(mean loss, dL/dW as a flat array of WEIGHT_COUNT, dL/dgrid like `grid`)."""
    q = np.asarray(queries, np.float32)
    y = np.asarray(targets, np.float32)
    n = len(q)
    ws = [bf16(w) for w in weights(mlp)]
    pred, xs = forward(q, mlp, grid, resolutions, log2_table)
    den = pred * pred + np.float32(0.01)
    diff = pred - y
    loss = float(np.mean(diff * diff / den))
    g = np.zeros((n, OUT), np.float32)
    g[:, 0] = 2.0 * diff / den / np.float32(n)
    g = bf16(g)
    dmlp = np.zeros(WEIGHT_COUNT, np.float32)
    for l in range(4, -1, -1):
        dW = (g[:, :LAYER_ROWS[l]].T @ xs[l]).astype(np.float32)
        dmlp[LAYER_OFFSET[l]:LAYER_OFFSET[l] + LAYER_ROWS[l] * WIDTH] = dW.ravel()
        dA = g[:, :LAYER_ROWS[l]] @ ws[l]
        if l > 0:
            g = bf16(np.where(xs[l] > 0, dA, 0.0).astype(np.float32))
        else:
            dinput = dA.astype(np.float32)
    dgrid = np.zeros(len(grid), np.float64)
    for level in range(LEVELS):
        idx, w = corners(q[:, :3], resolutions[level], log2_table, level)
        for f in range(2):
            np.add.at(dgrid, (2 * idx + f).ravel(), (w * dinput[:, 2 * level + f][:, None]).ravel())
    return loss, dmlp, dgrid.astype(np.float32)


def resolutions(base=16, finest=2048):
    """Cells per axis of the 16 levels: floor(base * growth^l), growth =
    (finest / base)^(1/15), evaluated in binary64 as the GPU host code does."""
    import math
    growth = math.exp((math.log(finest) - math.log(base)) / (LEVELS - 1))
    return [int(math.floor(base * growth ** l)) for l in range(LEVELS)]


def loss64(queries, targets, mlp, grid, resolutions, log2_table, denominators=None):
    """The loss in FP64 without any rounding (for finite-difference checks);
    `denominators` fixes p^2 + 0.01 per query (the training loss holds it
    constant)."""
    q = np.asarray(queries, np.float64)
    ws = [w.astype(np.float64) for w in weights(np.asarray(mlp, np.float64))]
    x = np.zeros((len(q), WIDTH))
    table = np.asarray(grid, np.float64).reshape(-1, 2)
    for level in range(LEVELS):
        idx, w = corners(q[:, :3].astype(np.float32), resolutions[level], log2_table, level)
        x[:, 2 * level] = (w * table[idx][:, :, 0]).sum(1)
        x[:, 2 * level + 1] = (w * table[idx][:, :, 1]).sum(1)
    x[:, 32:41] = q[:, 3:12]
    for l in range(4):
        x = np.maximum(x @ ws[l].T, 0.0)
    p = (x @ ws[4].T)[:, 0]
    d = p - np.asarray(targets, np.float64)
    den = (p * p + 0.01) if denominators is None else denominators
    return float(np.mean(d * d / den))


def predictions64(queries, mlp, grid, resolutions, log2_table):
    q = np.asarray(queries, np.float64)
    ws = [w.astype(np.float64) for w in weights(np.asarray(mlp, np.float64))]
    x = np.zeros((len(q), WIDTH))
    table = np.asarray(grid, np.float64).reshape(-1, 2)
    for level in range(LEVELS):
        idx, w = corners(q[:, :3].astype(np.float32), resolutions[level], log2_table, level)
        x[:, 2 * level] = (w * table[idx][:, :, 0]).sum(1)
        x[:, 2 * level + 1] = (w * table[idx][:, :, 1]).sum(1)
    x[:, 32:41] = q[:, 3:12]
    for l in range(4):
        x = np.maximum(x @ ws[l].T, 0.0)
    return (x @ ws[4].T)[:, 0]


def gradients64(queries, targets, mlp, grid, resolutions, log2_table):
    """Analytic gradients of loss64 (FP64, no rounding, denominator constant)."""
    q = np.asarray(queries, np.float64)
    y = np.asarray(targets, np.float64)
    n = len(q)
    ws = [w.astype(np.float64) for w in weights(np.asarray(mlp, np.float64))]
    table = np.asarray(grid, np.float64).reshape(-1, 2)
    x = np.zeros((n, WIDTH))
    cache = []
    for level in range(LEVELS):
        idx, w = corners(q[:, :3].astype(np.float32), resolutions[level], log2_table, level)
        cache.append((idx, w))
        x[:, 2 * level] = (w * table[idx][:, :, 0]).sum(1)
        x[:, 2 * level + 1] = (w * table[idx][:, :, 1]).sum(1)
    x[:, 32:41] = q[:, 3:12]
    xs = [x]
    for l in range(4):
        xs.append(np.maximum(xs[-1] @ ws[l].T, 0.0))
    p = (xs[-1] @ ws[4].T)[:, 0]
    g = np.zeros((n, OUT))
    g[:, 0] = 2.0 * (p - y) / (p * p + 0.01) / n
    dmlp = np.zeros(WEIGHT_COUNT)
    for l in range(4, -1, -1):
        dmlp[LAYER_OFFSET[l]:LAYER_OFFSET[l] + LAYER_ROWS[l] * WIDTH] = (g[:, :LAYER_ROWS[l]].T @ xs[l]).ravel()
        dA = g[:, :LAYER_ROWS[l]] @ ws[l]
        g = np.where(xs[l] > 0, dA, 0.0) if l > 0 else dA
    dgrid = np.zeros(len(grid))
    for level, (idx, w) in enumerate(cache):
        for f in range(2):
            np.add.at(dgrid, (2 * idx + f).ravel(), (w * g[:, 2 * level + f][:, None]).ravel())
    return dmlp, dgrid
