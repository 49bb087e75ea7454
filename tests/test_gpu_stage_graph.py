"""The device-buffer stage (chiaro_b200.depth.DeviceStage over
chiaro_refine_multiview_depth_device) and its whole-stage CUDA graph: the same bits as the
host-buffer API; launched, then captured, then replayed, each call bit-identical to the
stage without the graph; a replay reads new planes written into the same buffers, and a
new key or a reallocated buffer starts over."""
import dataclasses

import numpy as np
import pytest
import torch

from chiaro_b200 import scenes
from chiaro_b200.depth import DeviceStage, refine_multiview_depth

pytestmark = pytest.mark.gpu


def _stage(ctx, name, seed):
    sc = scenes.workload(name, seed=seed)
    return DeviceStage(sc.inputs(), sc.reference_index, sc.alignments(), sc.options, context=ctx)


def _run(stage, options=None):
    for t in stage.targets:
        stage.points[t].fill_(float("nan"))
    stage.depth.fill_(-1.0)
    assert stage(options)
    outputs = [stage.depth.cpu().numpy().view(np.uint64), stage.confidence.cpu().numpy().view(np.uint32),
               stage.provenance.cpu().numpy()]
    for t in stage.targets:
        outputs += [stage.points[t].cpu().numpy().reshape(-1).view(np.uint32),
                    stage.point_confidence[t].cpu().numpy().view(np.uint32)]
    return outputs, [bytes(r) for r in stage.reports], stage.graph_state


def _same(a, b):
    assert len(a[0]) == len(b[0]) and all(np.array_equal(x, y) for x, y in zip(a[0], b[0]))
    assert a[1] == b[1]


def test_device_stage_matches_the_host_api(gpu_ctx):
    sc = scenes.workload("small", seed=2)
    stage = DeviceStage(sc.inputs(), sc.reference_index, sc.alignments(), sc.options, context=gpu_ctx)
    outputs, _, _ = _run(stage)
    alignments = sc.alignments()
    dmap = refine_multiview_depth(sc.inputs(), sc.reference_index, alignments, sc.options, context=gpu_ctx)
    assert np.array_equal(outputs[0], dmap.depth.view(np.uint64))
    assert np.array_equal(outputs[1], dmap.confidence.view(np.uint32))
    assert np.array_equal(outputs[2], dmap.provenance)
    for k, t in enumerate(stage.targets):
        assert np.array_equal(outputs[3 + 2 * k], alignments[t].warp.points.reshape(-1).view(np.uint32))
        assert np.array_equal(outputs[4 + 2 * k], alignments[t].warp.confidence.view(np.uint32))
        assert stage.report(t) == alignments[t].report.depth
    assert stage.report(sc.reference_index) is None


def test_setting_the_same_graph_state_keeps_the_graph(gpu_ctx):
    stage = _stage(gpu_ctx, "tiny", 1)
    stage.graph = True
    try:
        states = []
        for _ in range(3):
            stage.graph = True  # every call sets it again
            states.append(_run(stage)[2])
        assert states == [0, 1, 2]
    finally:
        stage.graph = False


def test_stage_graph_captures_replays_and_starts_over(gpu_ctx):
    lib, h = gpu_ctx.lib, gpu_ctx.handle
    stage = _stage(gpu_ctx, "small", 3)
    plain = _run(stage)
    assert plain[2] == 0
    stage.graph = True
    try:
        states = []
        for _ in range(4):
            r = _run(stage)
            _same(r, plain)
            states.append(r[2])
        assert states == [0, 1, 2, 2]
        # new data in the same buffers: a replay reads it
        other = scenes.workload("small", seed=4)
        for plane, lum in zip(stage.planes, other.luminance):
            plane.copy_(torch.from_numpy(lum.data.reshape(-1).copy()))
        replayed = _run(stage)
        assert replayed[2] == 2
        stage.graph = False
        fresh = _run(stage)
        _same(replayed, fresh)
        assert not all(np.array_equal(x, y) for x, y in zip(replayed[0], plain[0]))
        stage.graph = True
        # other options: a new key
        stage.options = dataclasses.replace(stage.options, minimum_score=stage.options.minimum_score + 0.05)
        assert [_run(stage)[2] for _ in range(3)] == [0, 1, 2]
        # a buffer the graph uses reallocated by another entry point voids it
        big = torch.rand(600 * 500 * 129, device="cuda")
        guide = torch.rand(600 * 500, device="cuda")
        out = torch.empty_like(big)
        gpu_ctx.check(lib.chiaro_sgm_aggregate_device(h, big.data_ptr(), guide.data_ptr(), 600, 500, 129,
                                                      out.data_ptr()))
        after = _run(stage)
        assert after[2] == 0
        stage.graph = False
        _same(after, _run(stage))
    finally:
        stage.graph = False
