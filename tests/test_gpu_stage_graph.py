"""The whole-stage CUDA graph of chiaro_refine_multiview_depth_device: launched, then
captured, then replayed, each call bit-identical to the stage without it; a replay
reads new data from the same buffers, and a new key or a reallocated buffer starts
over."""
import ctypes as C
import dataclasses

import numpy as np
import pytest
import torch

from chiaro_b200 import scenes
from chiaro_b200.abi import DepthMapC, DepthReportC, WarpC
from chiaro_b200.depth import output_shape, pack_views

pytestmark = pytest.mark.gpu


class DeviceStage:
    """A scene's inputs and the stage's outputs in device memory, called through the ABI."""

    def __init__(self, ctx, scene, options=None):
        self.ctx, self.scene = ctx, scene
        self.options = options or scene.options
        self.views, keep = pack_views(scene.inputs(), scene.alignments())
        self.keep = keep
        self.planes = []
        for i, (lum, w) in enumerate(zip(scene.luminance, scene.warps)):
            tl = torch.from_numpy(lum.data.reshape(-1).copy()).cuda()
            tp = torch.from_numpy(w.points.reshape(-1).copy()).cuda()
            tc = torch.from_numpy(w.confidence.reshape(-1).copy()).cuda()
            self.planes.append(tl)
            self.keep += [tp, tc]
            self.views[i].luminance = C.cast(C.c_void_p(tl.data_ptr()), C.POINTER(C.c_float))
            self.views[i].warp.points = C.cast(C.c_void_p(tp.data_ptr()), C.POINTER(C.c_float))
            self.views[i].warp.confidence = C.cast(C.c_void_p(tc.data_ptr()), C.POINTER(C.c_float))
        (cols, rows, _), _ = output_shape(scene.width, scene.height, self.options)
        self.M = M = cols * rows
        self.n = n = len(scene.cameras)
        self.depth = torch.empty(M, dtype=torch.float64, device="cuda")
        self.conf = torch.empty(M, dtype=torch.float32, device="cuda")
        self.prov = torch.empty(M, dtype=torch.uint8, device="cuda")
        self.dmap = DepthMapC(capacity=M, depth=C.cast(C.c_void_p(self.depth.data_ptr()), C.POINTER(C.c_double)),
                              confidence=C.cast(C.c_void_p(self.conf.data_ptr()), C.POINTER(C.c_float)),
                              provenance=C.cast(C.c_void_p(self.prov.data_ptr()), C.POINTER(C.c_uint8)))
        self.refined = (WarpC * n)()
        self.warps = []
        for t in range(n):
            pts = torch.empty(2 * M, dtype=torch.float32, device="cuda")
            cf = torch.empty(M, dtype=torch.float32, device="cuda")
            self.warps += [pts, cf]
            self.refined[t].points = C.cast(C.c_void_p(pts.data_ptr()), C.POINTER(C.c_float))
            self.refined[t].confidence = C.cast(C.c_void_p(cf.data_ptr()), C.POINTER(C.c_float))
            self.refined[t].capacity = M
        self.reports = (DepthReportC * n)()

    def run(self):
        opt = self.options.to_c()
        for w in self.warps:
            w.fill_(float("nan"))
        self.depth.fill_(-1.0)
        self.ctx.check(self.ctx.lib.chiaro_refine_multiview_depth_device(
            self.ctx.handle, self.views, self.n, self.scene.reference_index, C.byref(opt), self.refined,
            self.reports, C.byref(self.dmap)))
        outputs = [self.depth.cpu().numpy().view(np.uint64), self.conf.cpu().numpy().view(np.uint32),
                   self.prov.cpu().numpy()] + [w.cpu().numpy().view(np.uint32) for w in self.warps]
        reports = [bytes(r) for r in self.reports]
        return outputs, reports, self.ctx.lib.chiaro_depth_stage_graph_state(self.ctx.handle)


def _same(a, b):
    assert len(a[0]) == len(b[0]) and all(np.array_equal(x, y) for x, y in zip(a[0], b[0]))
    assert a[1] == b[1]


def test_stage_graph_captures_replays_and_starts_over(gpu_ctx):
    lib, h = gpu_ctx.lib, gpu_ctx.handle
    stage = DeviceStage(gpu_ctx, scenes.workload("small", seed=3))
    gpu_ctx.check(lib.chiaro_depth_set_stage_graph(h, 0))
    plain = stage.run()
    assert plain[2] == 0
    gpu_ctx.check(lib.chiaro_depth_set_stage_graph(h, 1))
    try:
        states = []
        for _ in range(4):
            r = stage.run()
            _same(r, plain)
            states.append(r[2])
        assert states == [0, 1, 2, 2]
        # new data in the same buffers: a replay reads it
        other = scenes.workload("small", seed=4)
        for tl, lum in zip(stage.planes, other.luminance):
            tl.copy_(torch.from_numpy(lum.data.reshape(-1).copy()))
        replayed = stage.run()
        assert replayed[2] == 2
        gpu_ctx.check(lib.chiaro_depth_set_stage_graph(h, 0))
        fresh = stage.run()
        _same(replayed, fresh)
        assert not all(np.array_equal(x, y) for x, y in zip(replayed[0], plain[0]))
        gpu_ctx.check(lib.chiaro_depth_set_stage_graph(h, 1))
        # other options: a new key
        stage.options = dataclasses.replace(stage.options, minimum_score=stage.options.minimum_score + 0.05)
        assert [stage.run()[2] for _ in range(3)] == [0, 1, 2]
        # a buffer the graph uses reallocated by another entry point voids it
        big = torch.rand(600 * 500 * 129, device="cuda")
        guide = torch.rand(600 * 500, device="cuda")
        out = torch.empty_like(big)
        gpu_ctx.check(lib.chiaro_sgm_aggregate_device(h, big.data_ptr(), guide.data_ptr(), 600, 500, 129,
                                                      out.data_ptr()))
        after = stage.run()
        assert after[2] == 0
        gpu_ctx.check(lib.chiaro_depth_set_stage_graph(h, 0))
        _same(after, stage.run())
    finally:
        gpu_ctx.check(lib.chiaro_depth_set_stage_graph(h, 0))
