"""The frame pipeline (chiaro_b200.depth.DepthPipeline): a stream of frames of one rig whose
uploads and read-backs overlap the stages on the GPU. Every frame's outputs must be the bits a
DeviceStage call of its own gives for that frame. Frames are pinned tensors, numpy arrays,
frames with and without new warps, and the outputs are read after later frames were queued."""
import numpy as np
import pytest
import torch

from chiaro_b200 import scenes
from chiaro_b200.depth import DepthPipeline, DeviceStage

pytestmark = pytest.mark.gpu


def _frames(sc, count):
    """Frame k: the scene's planes scaled by 1 + k / 50 (every other frame as numpy), and on
    odd frames the warps shifted by a quarter pixel."""
    inputs, aligns = sc.inputs(), sc.alignments()
    frames = []
    for k in range(count):
        planes = [np.ascontiguousarray(i.luminance.data, dtype=np.float32) * np.float32(1 + k / 50) for i in inputs]
        points = conf = None
        if k % 2:
            points = [np.ascontiguousarray(a.warp.points, dtype=np.float32) + np.float32(0.25) for a in aligns]
            conf = [np.ascontiguousarray(a.warp.confidence, dtype=np.float32) for a in aligns]
        if k % 2 == 0:
            planes = [torch.from_numpy(p.reshape(-1)).pin_memory() for p in planes]
        frames.append((planes, points, conf))
    return frames


def _alone(ctx, sc, frame):
    """The frame through a DeviceStage of its own."""
    st = DeviceStage(sc.inputs(), sc.reference_index, sc.alignments(), sc.options, context=ctx)
    planes, points, conf = frame
    for dst, src in zip(st.planes, planes):
        dst.copy_(torch.as_tensor(np.asarray(src)).reshape(dst.shape))
    if points is not None:
        for dst, src in zip(st.warp_points, points):
            dst.copy_(torch.from_numpy(src.reshape(-1)))
        for dst, src in zip(st.warp_confidence, conf):
            dst.copy_(torch.from_numpy(src.reshape(-1)))
    torch.cuda.synchronize()
    ok = st()
    out = {"depth": st.depth.cpu().numpy(), "confidence": st.confidence.cpu().numpy(),
           "provenance": st.provenance.cpu().numpy(),
           "points": {t: st.points[t].cpu().numpy() for t in st.targets},
           "point_confidence": {t: st.point_confidence[t].cpu().numpy() for t in st.targets}}
    return ok, out


def _bits(a):
    a = np.ascontiguousarray(a)
    return a.view({8: np.uint64, 4: np.uint32, 1: np.uint8, 2: np.uint16}[a.dtype.itemsize])


@pytest.mark.parametrize("name,seed,count", [("small", 31, 5), ("small", 32, 1)])
def test_pipeline_frames_match_separate_calls(gpu_ctx, name, seed, count):
    sc = scenes.workload(name, seed=seed)
    frames = _frames(sc, count)
    expected = [_alone(gpu_ctx, sc, f) for f in frames]
    pipe = DepthPipeline(sc.inputs(), sc.reference_index, sc.alignments(), sc.options, context=gpu_ctx)
    got = []
    for ok, out in pipe.run(frames):
        got.append((ok, {k: ({t: v.copy() for t, v in out[k].items()} if isinstance(out[k], dict) else out[k].copy())
                         for k in out}))
    assert len(got) == count
    for (ok, out), (eok, eout) in zip(got, expected):
        assert ok == eok
        for key in ("depth", "confidence", "provenance"):
            assert np.array_equal(_bits(out[key]), _bits(eout[key])), key
        for key in ("points", "point_confidence"):
            assert out[key].keys() == eout[key].keys()
            for t in out[key]:
                assert np.array_equal(_bits(out[key][t]), _bits(eout[key][t])), (key, t)
    assert len(pipe.bytes_up) == count and len(pipe.bytes_down) == count
    assert pipe.bytes_up[0] == sum(p.numel() * 4 for p in pipe.stages[0].planes)


def test_pipeline_frames_differ_as_their_inputs_do(gpu_ctx):
    """The stream is not stuck on one frame: frames with other planes give other depths."""
    sc = scenes.workload("small", seed=31)
    pipe = DepthPipeline(sc.inputs(), sc.reference_index, sc.alignments(), sc.options, context=gpu_ctx)
    seen = [(out["depth"].copy(), out["confidence"].copy()) for _, out in pipe.run(_frames(sc, 3))]
    assert any(not np.array_equal(_bits(a), _bits(b)) for a, b in zip(seen[0], seen[1]))
