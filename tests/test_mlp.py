"""The learned switch's network: device forward / gradient / SGD kernels
against the CPU reference (oracle/mlp.py), a finite-difference check of the
reference itself, and feature construction. Tolerances are stated per test:
the device works in FP32, the reference in FP64."""
import numpy as np
import pytest

from oracle import mlp as ref


def random_weights(seed=0):
    from xbfs_b200 import learned
    rng = np.random.default_rng(seed)
    feats = rng.normal(0, 3, size=(64, 8)).astype(np.float32)
    return learned.init_weights(feats, seed), feats


def test_reference_gradient_matches_finite_differences():
    w, feats = random_weights(1)
    w = w.astype(np.float64)
    labels = np.random.default_rng(2).integers(0, 3, size=len(feats))
    loss, g = ref.loss_and_grad(w, feats, labels)
    rng = np.random.default_rng(3)
    for i in rng.choice(len(g), 40, replace=False):
        h = 1e-6
        wp, wm = w.copy(), w.copy()
        wp[16 + i] += h
        wm[16 + i] -= h
        fd = (ref.loss_and_grad(wp, feats, labels)[0] - ref.loss_and_grad(wm, feats, labels)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_packed_size():
    from xbfs_b200._lib import lib
    assert lib.xbfs_mlp_num_params() == 16 + 1443


def test_features_follow_kernel_formulas():
    from xbfs_b200.learned import features_from_trace
    tr = [{"level": 0, "strategy_id": 0, "n_f": 1, "m_f": 18, "n_u": 100, "m_u": 900},
          {"level": 1, "strategy_id": 2, "n_f": 18, "m_f": 500, "n_u": 80, "m_u": 800}]
    f = features_from_trace(tr)
    assert f.dtype == np.float32 and f.shape == (2, 8)
    assert f[0, 5] == 0 and f[1, 5] == 0          # previous strategy (level 0 has none: TD_QUEUE)
    assert np.isclose(f[1, 6], np.log(19) - np.log(2))
    assert np.isclose(f[1, 7], np.log1p(500 / 18))
    assert np.isclose(f[0, 4], 0.0) and np.isclose(f[1, 4], np.log(2))


@pytest.mark.gpu
def test_device_logits_match_cpu():
    from xbfs_b200 import learned
    w, feats = random_weights(4)
    dev = learned.logits(w, feats)
    cpu = ref.forward(w, feats)[-1]
    np.testing.assert_allclose(dev, cpu, rtol=1e-4, atol=1e-4)


@pytest.mark.gpu
def test_device_gradient_matches_cpu():
    import ctypes as C

    from xbfs_b200._lib import check, lib
    w, feats = random_weights(5)
    labels = np.random.default_rng(6).integers(0, 3, size=len(feats)).astype(np.int32)
    grad = np.zeros(1443, dtype=np.float32)
    loss = np.zeros(1, dtype=np.float32)
    check(lib.xbfs_mlp_grad(0, w.ctypes.data, feats.ctypes.data, labels.ctypes.data, len(labels),
                            grad.ctypes.data, loss.ctypes.data))
    rl, rg = ref.loss_and_grad(w, feats, labels)
    assert abs(loss[0] - rl) < 1e-4 * max(1, abs(rl))
    np.testing.assert_allclose(grad, rg, rtol=2e-3, atol=2e-5)


@pytest.mark.gpu
def test_device_training_reduces_loss_and_fits_a_separable_rule():
    from xbfs_b200 import learned
    rng = np.random.default_rng(7)
    feats = rng.normal(0, 1, size=(600, 8)).astype(np.float32)
    labels = np.where(feats[:, 1] > 0.5, 2, np.where(feats[:, 0] > 0, 1, 0)).astype(np.int32)
    ds = learned.Dataset(feats, labels, np.zeros((600, 3), dtype=np.float32))
    w, losses = learned.train(ds, epochs=1500, lr=0.1)
    assert losses[-1] < 0.5 * losses[0]
    acc = (np.argmax(learned.logits(w, feats), axis=1) == labels).mean()
    assert acc > 0.9
