"""The float64 oracle of the learned preconditioner's network checks itself: its hand-written backward pass against
central finite differences of its own loss, and its building blocks against their definitions (CPU only)."""
import numpy as np
import pytest

import unet_oracle as U


def sample(shape, seed):
    rng = np.random.default_rng(seed)
    r = rng.standard_normal(shape)
    occ = (rng.random(shape) < 0.15).astype(np.uint8)
    t = rng.standard_normal(shape)
    return r, occ, t


def test_parameter_count_matches_library():
    assert U.param_count() == 582257


@pytest.mark.parametrize("shape", [(5, 4, 3), (4, 6, 7)])
def test_backward_matches_finite_differences(shape):
    r, occ, t = sample(shape, 3)
    p = U.initial_like(1).astype(np.float64)
    loss, g = U.loss_and_gradient(p, r, occ, t)
    rng = np.random.default_rng(5)
    offsets = np.cumsum([0] + [27 * ci * co + co for ci, co, _ in U.LAYERS])
    picks = []
    for L in range(len(U.LAYERS)):  # weights and the bias of every layer
        picks += list(rng.integers(offsets[L], offsets[L + 1] - U.LAYERS[L][1], 4)) + [offsets[L + 1] - 1]
    h = 1e-6
    for i in picks:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (U.loss_and_gradient(pp, r, occ, t)[0] - U.loss_and_gradient(pm, r, occ, t)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(fd)) + 1e-7, (i, fd, g[i])


def test_adjoints():
    rng = np.random.default_rng(2)
    f = rng.standard_normal((5, 4, 7, 3))
    c = rng.standard_normal((3, 2, 4, 3))
    assert np.isclose(np.sum(U.pool(f) * c), np.sum(f * U.pool_adjoint(c, f.shape[:3])))
    assert np.isclose(np.sum(U.up(c, f.shape[:3]) * f), np.sum(c * U.up_adjoint(f, c.shape[:3])))
    w = rng.standard_normal((27, 3, 2))
    g = rng.standard_normal((5, 4, 7, 2))
    assert np.isclose(np.sum(U.conv(f, w) * g), np.sum(f * U.conv_data(g, w)))
    dw, db = U.conv_weight(f, g)
    assert np.isclose(np.sum(U.conv(f, w) * g), np.sum(dw * w))


def test_bf16_rounding():
    v = np.array([1.0, 1.00390625, 1.005859375, -3.0e-3, 65504.0], np.float32)
    r = U.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0  # halfway rounds to even
    assert r[2] == 1.0078125
    assert abs(r[3] - v[3]) <= abs(v[3]) * 2 ** -8


def test_network_is_positively_homogeneous():
    r, occ, t = sample((6, 5, 4), 9)
    p = U.initial_like(4)
    a = U.apply(p, r, occ)
    b = U.apply(p, 3.5 * r, occ)
    assert np.allclose(b, 3.5 * a, rtol=1e-5, atol=1e-6 * np.abs(a).max())  # the input scale s is FP32, as on the GPU
    assert not np.any(a[occ != 0])


def test_level1_training_pairs():
    """The network's training pairs on the multigrid level 1 (train_preconditioner.coarse_pair / coarse_mask): the
    input is the sum of a cell's 2 x 2 x 2 children (the solve's restriction of r - A V(r)), the target the mean of
    e - V(r) over its fluid children, the mask 1 where a cell has no fluid child; odd extents round up."""
    import torch

    import train_preconditioner as T

    rng = np.random.default_rng(3)
    nz, ny, nx = 5, 6, 7
    r = rng.standard_normal((nz, ny, nx)).astype(np.float32)
    t = rng.standard_normal((nz, ny, nx)).astype(np.float32)
    occ = (rng.random((nz, ny, nx)) < 0.4).astype(np.uint8)
    occ[0:2, 0:2, 0:2] = 1  # one level-1 cell without a fluid child
    got_r, got_t = T.coarse_pair(torch.from_numpy(r), torch.from_numpy(t), torch.from_numpy(occ))
    got_m = T.coarse_mask(torch.from_numpy(occ))
    assert got_r.shape == (3, 3, 4) and got_m.shape == (3, 3, 4)
    for Z in range(3):
        for Y in range(3):
            for X in range(4):
                sl = (slice(2 * Z, 2 * Z + 2), slice(2 * Y, 2 * Y + 2), slice(2 * X, 2 * X + 2))
                fluid = occ[sl] == 0
                assert np.isclose(got_r[Z, Y, X].item(), r[sl].sum(), atol=1e-5)
                assert got_m[Z, Y, X].item() == (0 if fluid.any() else 1)
                want = t[sl][fluid].mean() if fluid.any() else 0.0
                assert np.isclose(got_t[Z, Y, X].item(), want, atol=1e-5)
    assert got_m[0, 0, 0].item() == 1
