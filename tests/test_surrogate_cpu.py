"""CPU checks of the surrogate's FP64 restatement (the checker of the
tensor-core kernels): its gradient against finite differences, the feature
transform, BF16 rounding and the element matrix used by the projection."""
import numpy as np
import pytest

import mechanism
import mlp


def test_fp64_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    w = mlp.init_weights(seed=5)
    # non-zero biases so that their gradients are exercised
    blocks = mlp.unpack(w)
    blocks[0][:, 15] = rng.normal(0, 0.3, 128)
    for b in (1, 2):
        blocks[b][:, 128] = rng.normal(0, 0.3, 128)
    blocks[3][:11, 128] = rng.normal(0, 0.3, 11)
    w = mlp.pack(blocks)
    X = rng.normal(size=(9, 12))
    T = rng.normal(size=(9, 11))
    loss, g = mlp.loss_and_grad(w, X, T)
    # real parameters only (padding has zero gradient by construction)
    idx = [0, 5, 11, 15, 16 * 127 + 15,                                     # W0 incl. bias column
           mlp.OFF[1] + 3, mlp.OFF[1] + 128, mlp.OFF[1] + 144 * 77 + 128,   # W1
           mlp.OFF[2] + 144 * 5 + 17, mlp.OFF[2] + 144 * 127 + 128,          # W2
           mlp.OFF[3] + 2, mlp.OFF[3] + 144 * 10 + 128, mlp.OFF[3] + 144 * 10 + 127]
    for i in idx:
        h = 1e-6
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd = (mlp.loss_and_grad(wp, X, T)[0] - mlp.loss_and_grad(wm, X, T)[0]) / (2 * h)
        assert g[i] == pytest.approx(fd, rel=1e-6, abs=1e-10), f"parameter {i}"
    mask = [np.zeros(s, bool) for s in mlp.SHAPES]
    mask[0][:, 12:15] = True
    mask[1][:, 129:] = True
    mask[2][:, 129:] = True
    mask[3][11:, :] = True
    mask[3][:, 129:] = True
    assert np.all(g[mlp.pack(mask).astype(bool)] == 0)


def test_boxcox_round_trip_and_range():
    y = np.array([0.0, 1e-30, 1e-12, 1e-6, 3e-3, 0.2, 0.75, 1.0])
    b = mlp.boxcox(y)
    assert np.all(np.diff(b) >= 0)
    back = mlp.boxcox_inv(b)
    assert np.allclose(back, y, rtol=1e-10, atol=1e-19)
    assert mlp.boxcox_inv(np.array([-20.0]))[0] == 0.0


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 1e-20, 3.14159])
    r = mlp.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == 1.0 + 2 ** -7        # tie rounds up to even mantissa
    assert r[3] == -2.5
    assert abs(r[5] - 3.140625) < 1e-12
    assert np.all(np.abs(r - x) <= np.abs(x) * 2 ** -8)


def test_element_mass_fractions_conserve_mass():
    for name in ("li2004", "premix_h2_ar"):
        m = mechanism.load(name)
        mu = m.element_mass_fractions()
        assert mu.shape == (3, 9)
        assert np.allclose(mu.sum(axis=0), 1.0, atol=1e-14)
        # water: two H and one O by mass
        k = m.index("H2O")
        assert mu[0, k] == pytest.approx(2 * 1.008 / m.mw[k])


def test_raw_features_layout():
    Y = np.zeros((2, 9))
    Y[:, 0] = 0.03
    Y[:, 2] = 0.2
    Y[:, 8] = 0.77
    f = mlp.raw_features([1200.0, 1300.0], 2e5, Y, 1e-7)
    assert f.shape == (2, 12)
    assert f[0, 0] == 1200.0 and f[1, 1] == pytest.approx(np.log(2e5))
    assert f[0, 2] == pytest.approx(mlp.boxcox(0.03)) and f[0, 11] == pytest.approx(np.log(1e-7))
    assert f[0, 3] == pytest.approx(mlp.boxcox(0.0))
