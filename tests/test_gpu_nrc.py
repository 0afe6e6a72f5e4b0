"""The radiance cache's tensor-core kernels (hdcx_nrc_*) against the CPU
oracle (oracle/nrc_oracle.py): predictions, MLP weight gradients and hash-grid
gradients on the same parameters and queries, and online training that fits a
radiance field which the untrained cache does not."""
import numpy as np
import pytest

import nrc_oracle as N

pytestmark = pytest.mark.gpu

LOG2 = 14
# Both a small table and the config's 2^19 entries per level.
TABLE_SIZES = [14, 19]


def queries(n, seed):
    rng = np.random.default_rng(seed)
    q = np.zeros((n, 12), np.float32)
    q[:, :3] = rng.uniform(0, 1, (n, 3))
    d = rng.normal(size=(n, 3))
    q[:, 3:6] = d / np.linalg.norm(d, axis=1, keepdims=True)
    q[:, 6:9] = -q[:, 3:6]
    q[:, 9] = rng.uniform(0, 1, n)
    q[:, 10] = rng.uniform(0, 1, n)
    return q


def radiance_field(q):
    """A smooth synthetic radiance over position and wavelength."""
    x, y, z, lam = q[:, 0], q[:, 1], q[:, 2], q[:, 10]
    return (1.0 + 0.6 * np.sin(6 * x) * np.cos(4 * y) + 0.5 * z + 0.3 * lam).astype(np.float32)


@pytest.fixture(scope="module", params=TABLE_SIZES, ids=[f"2^{k}" for k in TABLE_SIZES])
def cache(request):
    from hdcodex_b200 import RadianceCache
    c = RadianceCache(0, log2_table_size=request.param, base_resolution=16, finest_resolution=512, seed=7)
    rng = np.random.default_rng(11)
    mlp, grid = c.parameters()
    for l in range(5):
        rows = N.LAYER_ROWS[l]
        b = np.sqrt(6.0 / (N.WIDTH + rows))
        mlp[N.LAYER_OFFSET[l]:N.LAYER_OFFSET[l] + rows * N.WIDTH] = rng.uniform(-b, b, rows * N.WIDTH)
    grid[:] = rng.uniform(-0.5, 0.5, grid.size)
    c.set_parameters(mlp, grid)
    yield c
    c.close()


def device(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_forward_matches_oracle(cache):
    import torch
    q = queries(1000, 1)  # 7 full tiles of 128 and a partial one
    mlp, grid = cache.parameters()
    dq = device(q)
    out = torch.zeros(len(q), dtype=torch.float32, device="cuda")
    cache.query(dq.data_ptr(), len(q), out.data_ptr())
    got = out.cpu().numpy()
    ref, _ = N.forward(q, mlp, grid, cache.resolutions(), cache.config.log2_table_size)
    assert np.isfinite(got).all()
    # The oracle rounds weights, activations and output gradients to BF16 as
    # the kernels do; what remains is the FP32 summation order (measured:
    # relative L2 4e-5, largest difference 1e-3 of the largest prediction).
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert err < 1e-3, err
    assert np.abs(got - ref).max() < 5e-3 * np.abs(ref).max()


@pytest.mark.parametrize("n", [1, 100, 129, 383, 120_001])
def test_forward_tile_counts(cache, n):
    """Query counts of a single partial tile (1, 100), a full tile and a
    partial one (129, 383), and more tiles than the grid holds at once, so
    that blocks step to further tiles (120,001 queries: 938 tiles over at
    most four blocks per SM)."""
    import torch
    q = queries(n, 100 + n % 97)
    mlp, grid = cache.parameters()
    out = torch.full((n,), float("nan"), dtype=torch.float32, device="cuda")
    cache.query(device(q).data_ptr(), n, out.data_ptr())
    got = out.cpu().numpy()
    ref, _ = N.forward(q, mlp, grid, cache.resolutions(), cache.config.log2_table_size)
    assert np.isfinite(got).all()
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-3
    assert np.abs(got - ref).max() < 5e-3 * np.abs(ref).max()


def test_gradients_match_oracle(cache):
    q = queries(640, 2)
    y = radiance_field(q)
    mlp, grid = cache.parameters()
    dq, dy = device(q), device(y)  # held: the cache reads them during the call
    g_mlp, g_grid = cache.gradients(dq.data_ptr(), dy.data_ptr(), len(q))
    _, r_mlp, r_grid = N.gradients(q, y, mlp, grid, cache.resolutions(), cache.config.log2_table_size)
    for l in range(5):
        a = g_mlp[N.LAYER_OFFSET[l]:N.LAYER_OFFSET[l] + N.LAYER_ROWS[l] * N.WIDTH]
        b = r_mlp[N.LAYER_OFFSET[l]:N.LAYER_OFFSET[l] + N.LAYER_ROWS[l] * N.WIDTH]
        if l == 4:  # only output 0 carries a loss; the padded outputs' gradients are zero
            assert not a[N.WIDTH:].any()
        cos = float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-30))
        assert cos > 0.9999, (l, cos)
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-4, l  # measured ~2e-7
    cos = float(g_grid @ r_grid / (np.linalg.norm(g_grid) * np.linalg.norm(r_grid)))
    assert cos > 0.9999, cos
    assert np.linalg.norm(g_grid - r_grid) / np.linalg.norm(r_grid) < 1e-4  # measured ~5e-8


def test_training_fits_a_radiance_field():
    import torch
    from hdcodex_b200 import RadianceCache
    with RadianceCache(0, log2_table_size=LOG2, base_resolution=16, finest_resolution=512, seed=3,
                       learning_rate=1e-2) as c:
        test = queries(4096, 99)
        truth = radiance_field(test)
        out = torch.zeros(len(test), dtype=torch.float32, device="cuda")
        dtest = device(test)

        def error():
            c.query(dtest.data_ptr(), len(test), out.data_ptr())
            p = out.cpu().numpy()
            return float(np.sqrt(np.mean((p - truth) ** 2)) / np.sqrt(np.mean(truth ** 2)))

        before = error()
        first = None
        for step in range(300):
            q = queries(1 << 14, 1000 + step)
            dq, dy = device(q), device(radiance_field(q))
            loss = c.train(dq.data_ptr(), dy.data_ptr(), len(q), 1)
            first = loss if first is None else first
        after = error()
        assert np.isfinite(loss) and loss < 0.1 * first, (first, loss)
        # The trained cache predicts the field; the untrained one does not.
        assert after < 0.1 and after < 0.2 * before, (before, after)


def test_bounded_wait_times_out_and_the_context_survives(cache):
    import torch
    # An mbarrier that nothing arrives at: the wait runs out instead of hanging.
    status, message = cache.check_wait_timeout(1 << 12)
    assert status == "HDCX_ERROR_TIMEOUT" and "timed out" in message
    q = queries(256, 5)
    dq = device(q)
    out = torch.zeros(len(q), dtype=torch.float32, device="cuda")
    cache.query(dq.data_ptr(), len(q), out.data_ptr())
    assert np.isfinite(out.cpu().numpy()).all()
