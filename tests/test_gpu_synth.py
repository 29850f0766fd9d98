"""The device data generator (disorder_synth_phantom / _coils / add_noise)
against the NumPy recipe it restates (disorder_b200.synth), from the same
seeds."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import disorder_b200 as db
    return db.Context(0)


def test_phantom_matches_the_numpy_recipe(ctx):
    from disorder_b200 import synth, synth_gpu
    N = (48, 40, 32)
    xg = synth_gpu.phantom(ctx, N, 12, np.random.default_rng(5)).numpy()
    xh = synth.phantom(N, 12, np.random.default_rng(5))
    xh = xh / np.linalg.norm(xh)
    assert abs(np.linalg.norm(xg) - 1.0) < 1e-5
    # voxels on an ellipsoid surface may fall either side in single precision
    bad = np.abs(xg - xh) > 1e-4 * np.abs(xh).max()
    assert bad.mean() < 2e-3
    assert np.linalg.norm((xg - xh)[~bad]) < 1e-4 * np.linalg.norm(xh)


def test_coil_maps_match_the_numpy_recipe(ctx):
    from disorder_b200 import synth, synth_gpu
    N = (40, 36, 24)
    Sg = synth_gpu.coil_maps(ctx, N, 8, np.random.default_rng(6)).numpy()
    Sh = synth.coil_maps(N, 8, np.random.default_rng(6))
    assert np.linalg.norm(Sg - Sh) < 1e-5 * np.linalg.norm(Sh)
    assert np.allclose(np.sum(np.abs(Sg) ** 2, axis=3), 1.0, atol=1e-5)


def test_noise_is_gaussian_and_reproducible(ctx):
    from disorder_b200 import synth_gpu
    n = 1 << 20
    a = ctx.upload(np.zeros(n, np.complex64))
    b = ctx.upload(np.zeros(n, np.complex64))
    synth_gpu.add_noise(ctx, a, 0.5, 1234)
    synth_gpu.add_noise(ctx, b, 0.5, 1234)
    va, vb = a.numpy(), b.numpy()
    assert np.array_equal(va, vb)
    for part in (va.real, va.imag):
        assert abs(part.mean()) < 5 * 0.5 / np.sqrt(n)
        assert abs(part.std() - 0.5) < 0.01 * 0.5
        assert abs(np.mean(((part / 0.5) ** 4)) - 3.0) < 0.05  # normal kurtosis
    synth_gpu.add_noise(ctx, b, 0.5, 1235)
    assert not np.array_equal(b.numpy(), 2 * va)
