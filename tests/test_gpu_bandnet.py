"""The band proposal network on the GPU (bf16 tensor-core kernels, fp32
accumulation) against the fp32 oracle (oracle_bandnet_loss_grad) on the same
bf16-rounded features and weights, and its training and proposals."""
import ctypes as C

import numpy as np
import pytest

from chiaro_b200 import runtime
from chiaro_b200.bandnet import BandNet, Sample

pytestmark = pytest.mark.gpu

F = C.POINTER(C.c_float)


def bf16_round(x: np.ndarray) -> np.ndarray:
    b = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) >> 16 << 16
    return b.astype(np.uint32).view(np.float32)


def _samples(images, rows, columns, labels, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(images):
        n = rows * columns
        costs = rng.uniform(0, 2.25, n * labels).astype(np.float32)
        guidance = rng.uniform(0, 7, n).astype(np.float32)
        winners = rng.integers(1, labels, n).astype(np.int32)
        mask = (rng.random(n) < 0.85).astype(np.uint8)
        out.append(Sample(costs, guidance, winners, mask, columns, rows, labels))
    return out


def test_gpu_gradient_matches_fp32_oracle(gpu_ctx):
    from oracle import oracle
    lib = oracle.lib()
    net = BandNet(gpu_ctx, seed=3)
    rng = np.random.default_rng(4)
    params = net.params.cpu().numpy() + rng.normal(0, 0.01, net.params.numel()).astype(np.float32)
    net.params.copy_(net.torch.from_numpy(params))
    samples = _samples(2, 9, 20, 49, 5)
    grads_gpu, loss_gpu = net.gradient(samples)
    # the oracle on what the GPU computes from: bf16 features and weights, fp32 biases
    n = 9 * 20
    features = np.zeros((2 * n, 32), np.float32)
    for i, s in enumerate(samples):
        lib.oracle_bandnet_features(s.costs.ctypes.data_as(F), s.guidance.ctypes.data_as(F), n, s.labels, s.labels,
                                    features[i * n:].ctypes.data_as(F))
    features = bf16_round(features)
    p = params.copy().reshape(6, -1)
    p[:, :9 * 32 * 32] = bf16_round(p[:, :9 * 32 * 32])
    p = np.ascontiguousarray(p.reshape(-1))
    targets = np.concatenate([(s.winners - 1) / (s.labels - 2) for s in samples]).astype(np.float32)
    mask = np.concatenate([s.mask for s in samples])
    grads = np.zeros_like(p)
    loss = C.c_float()
    # the oracle stores every activation and pre-activation gradient in bf16, as the GPU does;
    # what remains is the accumulation order (fp32 tensor-core sums against f64 loops)
    lib.oracle_bandnet_loss_grad_mode(p.ctypes.data_as(F), features.ctypes.data_as(F), targets.ctypes.data_as(F),
                                      mask.ctypes.data_as(C.POINTER(C.c_uint8)), 2, 9, 20, grads.ctypes.data_as(F),
                                      C.byref(loss), None, 1)
    # stated tolerance: loss within 1e-3 relative, gradient within 1e-2 relative L2
    assert abs(loss_gpu - loss.value) <= 1e-3 * loss.value, (loss_gpu, loss.value)
    rel = float(np.linalg.norm(grads_gpu - grads) / np.linalg.norm(grads))
    assert rel < 1e-2, rel


def test_training_lowers_the_loss(gpu_ctx):
    net = BandNet(gpu_ctx, seed=7)
    samples = _samples(3, 12, 33, 65, 8)
    for s in samples:  # a learnable target: the label of each node's cheapest cost
        s.winners = (1 + np.argmin(s.costs.reshape(-1, s.labels)[:, 1:], axis=1)).astype(np.int32)
    losses = net.train(samples, 60, 3e-3)
    assert np.all(np.isfinite(losses)) and losses[-1] < 0.7 * losses[0]


def test_proposals_are_valid_band_offsets(gpu_ctx):
    import torch
    net = BandNet(gpu_ctx, seed=1)
    s = _samples(1, 30, 41, 193, 9)[0]
    dev = torch.device("cuda", 0)
    costs, guidance = torch.from_numpy(s.costs).to(dev), torch.from_numpy(s.guidance).to(dev)
    a = net.propose(costs, guidance, 41, 30, 193, 4, 24).cpu().numpy()
    b = net.propose(costs, guidance, 41, 30, 193, 4, 24).cpu().numpy()
    assert a.shape == (11 * 8,) and np.array_equal(a, b)
    assert a.min() >= 1 and a.max() <= 193 - 24


def test_trained_network_against_the_naive_band(gpu_ctx):
    """What training buys: the band network trained on the GPU (tile-median targets from
    the exact plain search's winners, inputs from the pre-pass's 16 sampled labels)
    against the naive band (each tile's median lowest sampled label) on held-out
    1040x780 scenes with 192 planes: the learned-band coarse search scored against the
    plain search over tested nodes."""
    from chiaro_b200 import bandnet
    from chiaro_b200.depth import DeviceStage
    rendered = bandnet.render_scenes("band", list(range(300, 316)) + list(range(900, 906)))
    stages = [DeviceStage(s.inputs(), 0, s.alignments(), s.options, context=gpu_ctx) for s in rendered]
    samples = [bandnet.samples_from_prepass(st) for st in stages[:16]]
    net = BandNet(gpu_ctx, seed=0)
    targets = [bandnet.tile_targets(s, 4, "median") for s in samples]
    losses = np.concatenate([net.train(targets, 400, 2e-3), net.train(targets, 200, 5e-4)])
    scores = bandnet.evaluate_search(stages[16:], {"learned": net}, 4, 24, 8, 1.0)
    print(scores)
    assert losses[-1] < 0.2 * losses[0]
    learned, naive = scores["learned"], scores["naive"]
    assert learned["within_one_plane"] > naive["within_one_plane"]
