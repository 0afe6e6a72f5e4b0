"""The CPU oracle of the radiance cache (oracle/nrc_oracle.py): its analytic
FP64 gradients against central differences, and its BF16-rounded gradients
(the arithmetic of the tensor-core kernels) against the FP64 ones."""
import numpy as np
import pytest

import nrc_oracle as N

LOG2 = 12


def problem(seed=0, n=96):
    rng = np.random.default_rng(seed)
    res = N.resolutions(4, 64)
    mlp = np.zeros(N.WEIGHT_COUNT)
    for l in range(5):
        rows = 1 if l == 4 else N.LAYER_ROWS[l]
        b = np.sqrt(6.0 / (N.WIDTH + N.LAYER_ROWS[l]))
        mlp[N.LAYER_OFFSET[l]:N.LAYER_OFFSET[l] + rows * N.WIDTH] = rng.uniform(-b, b, rows * N.WIDTH)
    grid = rng.uniform(-0.5, 0.5, N.LEVELS * (1 << LOG2) * 2)
    q = np.zeros((n, 12))
    q[:, :3] = rng.uniform(0, 1, (n, 3))
    d = rng.normal(size=(n, 3))
    q[:, 3:6] = d / np.linalg.norm(d, axis=1, keepdims=True)
    q[:, 6:9] = -q[:, 3:6]
    q[:, 9] = rng.uniform(0, 1, n)
    q[:, 10] = rng.uniform(0, 1, n)
    y = rng.uniform(0.1, 2.0, n)
    return q, y, mlp, grid, res


def test_resolutions_follow_the_geometric_series():
    r = N.resolutions(16, 2048)
    assert r[0] == 16 and r[-1] in (2047, 2048) and all(b > a for a, b in zip(r, r[1:]))


def test_fp64_gradients_match_central_differences():
    q, y, mlp, grid, res = problem()
    dmlp, dgrid = N.gradients64(q, y, mlp, grid, res, LOG2)
    p = N.predictions64(q, mlp, grid, res, LOG2)
    den = p * p + 0.01
    rng = np.random.default_rng(1)
    h = 1e-4  # small enough for the curvature, large enough for FP64 cancellation
    for kind, params, grad in (("mlp", mlp, dmlp), ("grid", grid, dgrid)):
        candidates = np.flatnonzero(np.abs(grad) > 1e-6 * np.abs(grad).max())
        for i in rng.choice(candidates, size=12, replace=False):
            plus, minus = params.copy(), params.copy()
            plus[i] += h
            minus[i] -= h
            args_p = (plus, grid) if kind == "mlp" else (mlp, plus)
            args_m = (minus, grid) if kind == "mlp" else (mlp, minus)
            fd = (N.loss64(q, y, *args_p, res, LOG2, den) - N.loss64(q, y, *args_m, res, LOG2, den)) / (2 * h)
            assert fd == pytest.approx(grad[i], rel=1e-3, abs=1e-8), (kind, i)


def test_bf16_gradients_track_fp64():
    q, y, mlp, grid, res = problem(seed=3, n=256)
    loss, dmlp, dgrid = N.gradients(q, y, mlp.astype(np.float32), grid.astype(np.float32), res, LOG2)
    dmlp64, dgrid64 = N.gradients64(q, y, mlp, grid, res, LOG2)
    for a, b in ((dmlp, dmlp64), (dgrid, dgrid64)):
        cos = float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b)))
        assert cos > 0.99
    assert np.isfinite(loss) and loss > 0
