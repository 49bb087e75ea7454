"""The fp32 oracle of the band proposal network (oracle_bandnet_loss_grad): its
analytic gradient against central finite differences of its loss."""
import ctypes as C

import numpy as np

from chiaro_b200.bandnet import INPUTS, init_params

F = C.POINTER(C.c_float)


def _loss_grad(lib, params, features, targets, mask, images, h, w):
    grads = np.zeros_like(params)
    loss = C.c_float()
    lib.oracle_bandnet_loss_grad(params.ctypes.data_as(F), features.ctypes.data_as(F), targets.ctypes.data_as(F),
                                 mask.ctypes.data_as(C.POINTER(C.c_uint8)), images, h, w, grads.ctypes.data_as(F),
                                 C.byref(loss), None)
    return float(loss.value), grads


def test_oracle_gradient_matches_finite_differences(oracle_lib):
    rng = np.random.default_rng(0)
    images, h, w = 2, 5, 6
    params = init_params(1)
    params += rng.normal(0, 0.02, params.size).astype(np.float32)  # move off the initial zeros
    features = rng.uniform(0, 1, (images, h, w, 32)).astype(np.float32)
    features[..., INPUTS:] = 0.0
    targets = rng.uniform(0, 1, images * h * w).astype(np.float32)
    mask = (rng.random(images * h * w) < 0.8).astype(np.uint8)
    loss, grads = _loss_grad(oracle_lib, params, features, targets, mask, images, h, w)
    assert loss > 0
    big = np.argsort(-np.abs(grads))[:40]  # the largest entries: well above the finite-difference noise
    checked = passed = 0
    for i in big:
        eps = 1e-3
        p = params.copy()
        p[i] += eps
        lp, _ = _loss_grad(oracle_lib, p, features, targets, mask, images, h, w)
        p[i] -= 2 * eps
        lm, _ = _loss_grad(oracle_lib, p, features, targets, mask, images, h, w)
        fd = (lp - lm) / (2 * eps)
        checked += 1
        passed += abs(fd - grads[i]) <= 0.05 * abs(grads[i]) + 1e-5
    assert passed >= 0.9 * checked, (passed, checked)


def test_oracle_features_of_a_node(oracle_lib):
    """The 16 sampled labels spread over 1..D-1 (first and last included); the features
    read them from a full row or from the pre-pass's compact row, with the same result."""
    labels = 49
    sampled = np.zeros(16, np.int32)
    oracle_lib.oracle_net_sample_labels(labels, sampled.ctypes.data_as(C.POINTER(C.c_int)))
    assert sampled[0] == 1 and sampled[-1] == labels - 1 and np.all(np.diff(sampled) > 0)
    assert list(sampled) == [1 + (b * (labels - 2) + 7) // 15 for b in range(16)]
    costs = np.full(labels, 1.5, np.float32)
    costs[0] = 0.0  # label 0 is not a depth label and stays out of the summary
    costs[sampled[[2, 6, 9]]] = [0.4, 0.2, 0.2]
    costs[sampled[4] + 1] = 0.05  # not a sampled label: invisible to the features
    guidance = np.array([4.0], np.float32)
    compact = np.concatenate([[costs[0]], costs[sampled]]).astype(np.float32)
    expected = np.full(16, 1.3, np.float32)
    expected[2], expected[6], expected[9] = 0.2, 0.0, 0.0  # minus the lowest sampled cost 0.2
    for row, stride in ((costs, labels), (compact, 17)):
        f = np.zeros(32, np.float32)
        oracle_lib.oracle_bandnet_features(row.ctypes.data_as(F), guidance.ctypes.data_as(F), 1, labels, stride,
                                           f.ctypes.data_as(F))
        assert f[0] == np.float32(0.5)
        assert np.allclose(f[1:17], expected)
        assert f[17] == np.float32((sampled[6] - 1) / (labels - 2))  # the first sampled label at the minimum
        assert f[18] == np.float32(0.2)
        assert not f[INPUTS:].any()
