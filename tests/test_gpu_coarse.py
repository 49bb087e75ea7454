"""The coarse depth search operator, plain and learned-band, against the oracle (GPU).

Every expectation comes from the oracle's full cost volume and SGM
(crates/chiaro-fusion/src/depth.rs:1187-1383) on the same scene:
* plain: each node's winner is the first minimum over labels 1..D-1 of the oracle's
  regularised costs, and the tested flags are the oracle's;
* the pre-pass rows are the full volume's label 0 and 16 sampled labels, bit for bit;
* the banded search's winners and fallback flags equal the oracle's banded SGM with
  windowed full-range fallback (oracle_sgm_banded) run on the full volume with the
  same tile bands: a label's cost does not depend on which other labels a node scores;
* the naive bands are the tile medians of the pre-pass's lowest sampled labels;
* the cross-view flags follow from the volume's scores at the banded winners.
"""
import ctypes as C

import numpy as np
import pytest

from chiaro_b200 import scenes
from chiaro_b200.band import centred_offsets, tiles_of
from chiaro_b200.coarse import BandOptions, band_prepass, coarse_depth, sample_labels
from chiaro_b200.depth import DeviceStage, DepthOptions, output_shape

pytestmark = pytest.mark.gpu

F = C.POINTER(C.c_float)
I32 = C.POINTER(C.c_int)
U8 = C.POINTER(C.c_uint8)


def _case(name, seed, planes, **kw):
    sc = scenes.workload(name, seed=seed, options=dict(planes=planes), **kw)
    from oracle import oracle
    (columns, rows, _), (cc, cr, _) = output_shape(sc.width, sc.height, sc.options)
    d = sc.options.planes + 1
    dbg = oracle.debug_buffers(len(sc.cameras), cc * cr, d, columns * rows)
    oracle.refine_multiview_depth(sc.inputs(), 0, sc.alignments(), sc.options, threads=8, debug=dbg)
    return sc, dbg, cc, cr, d


@pytest.fixture(scope="module")
def small():
    return _case("small", 21, 40)


@pytest.fixture(scope="module")
def mirrored():
    return _case("small", 22, 48, mirrors={1: True, 2: False})


def _stage(sc, ctx):
    return DeviceStage(sc.inputs(), 0, sc.alignments(), sc.options, context=ctx)


def _oracle_banded(dbg, cc, cr, d, offsets, tile, band, margin):
    from oracle import oracle
    winner = np.zeros(cc * cr, np.int32)
    tx, ty = tiles_of(cc, cr, tile)
    fallback = np.zeros(tx * ty, np.uint8)
    costs = np.ascontiguousarray(dbg["coarse_costs"])
    guidance = np.ascontiguousarray(dbg["coarse_guidance"])
    offs = np.ascontiguousarray(offsets, np.int32)
    st = oracle.lib().oracle_sgm_banded(costs.ctypes.data_as(F), guidance.ctypes.data_as(F), cc, cr, d,
                                        offs.ctypes.data_as(I32), tile, band, margin, winner.ctypes.data_as(I32),
                                        fallback.ctypes.data_as(U8))
    assert st == 0
    return winner, fallback


@pytest.mark.parametrize("case", ["small", "mirrored"])
def test_plain_search_equals_the_oracle(gpu_ctx, case, request):
    sc, dbg, cc, cr, d = request.getfixturevalue(case)
    r = coarse_depth(_stage(sc, gpu_ctx))
    reg = dbg["regularised"].reshape(cc * cr, d)
    expected = 1 + np.argmin(reg[:, 1:], axis=1)
    assert np.array_equal(r.winner.cpu().numpy(), expected)
    assert np.array_equal(r.tested.cpu().numpy(), dbg["coarse_tested"])


def test_prepass_rows_are_the_full_volume_columns(gpu_ctx, small):
    sc, dbg, cc, cr, d = small
    costs, guidance, tested = band_prepass(_stage(sc, gpu_ctx))
    cols = [0] + sample_labels(d)
    full = dbg["coarse_costs"].reshape(cc * cr, d)[:, cols]
    assert np.array_equal(costs.cpu().numpy().view(np.uint32), np.ascontiguousarray(full).view(np.uint32))
    assert np.array_equal(guidance.cpu().numpy().view(np.uint32), dbg["coarse_guidance"].view(np.uint32))
    scores = dbg["coarse_scores"].reshape(cc * cr, d)[:, cols]
    assert np.array_equal(tested.cpu().numpy(), np.isfinite(scores).any(axis=1).astype(np.uint8))


@pytest.mark.parametrize("case", ["small", "mirrored"])
@pytest.mark.parametrize("tile,band,margin", [(4, 12, 8), (2, 16, 4), (8, 24, 6)])
def test_naive_banded_search_equals_the_oracle(gpu_ctx, case, tile, band, margin, request):
    sc, dbg, cc, cr, d = request.getfixturevalue(case)
    r = coarse_depth(_stage(sc, gpu_ctx), BandOptions(None, tile, band, margin, 1.0))
    offsets = r.offsets.cpu().numpy()
    # the naive bands: per tile, the median of each node's first sampled label at its lowest sampled cost
    sampled = np.array(sample_labels(d))
    pre = dbg["coarse_costs"].reshape(cc * cr, d)[:, sampled]
    lowest = sampled[np.argmin(pre, axis=1)].reshape(cr, cc)
    tx, ty = tiles_of(cc, cr, tile)
    centres = np.array([np.median(lowest[y * tile:(y + 1) * tile, x * tile:(x + 1) * tile])
                        for y in range(ty) for x in range(tx)])
    assert np.array_equal(offsets, centred_offsets(centres, d, band))
    winner, fallback = _oracle_banded(dbg, cc, cr, d, offsets, tile, band, margin)
    assert np.array_equal(r.fallback.cpu().numpy(), fallback)
    assert np.array_equal(r.winner.cpu().numpy(), winner)
    rep = r.report
    assert rep["fallback_tiles"] == rep["edge_tiles"] == int(fallback.sum()) and rep["consistency_tiles"] == 0


def test_network_banded_search_equals_the_oracle(gpu_ctx, small):
    """The band from an (untrained) network: whatever it proposes, the search given those
    bands equals the oracle's banded SGM with them."""
    import torch
    from chiaro_b200.bandnet import init_params
    sc, dbg, cc, cr, d = small
    params = torch.from_numpy(init_params(5)).cuda()
    r = coarse_depth(_stage(sc, gpu_ctx), BandOptions(params, 4, 16, 8, 1.0))
    offsets = r.offsets.cpu().numpy()
    assert offsets.min() >= 1 and offsets.max() <= d - 16
    winner, fallback = _oracle_banded(dbg, cc, cr, d, offsets, 4, 16, 8)
    assert np.array_equal(r.fallback.cpu().numpy(), fallback)
    assert np.array_equal(r.winner.cpu().numpy(), winner)


def test_cross_view_fallback_flags(gpu_ctx, mirrored):
    """Tiles whose winners are contradicted (score at the winner more than 0.12 below the
    score under the global warp, depth.rs:458-485) on more than the fraction of their
    tested nodes fall back; the flags follow from the full volume's scores."""
    sc, dbg, cc, cr, d = mirrored
    tile, band, margin, fraction = 4, 12, 8, 0.1
    stage = _stage(sc, gpu_ctx)
    off = coarse_depth(stage, BandOptions(None, tile, band, margin, 1.0))
    on = coarse_depth(stage, BandOptions(None, tile, band, margin, fraction))
    offsets = off.offsets.cpu().numpy()
    assert np.array_equal(on.offsets.cpu().numpy(), offsets)
    edge = off.fallback.cpu().numpy().astype(bool)
    winners = off.winner.cpu().numpy()  # banded winners wherever the edge rule kept the band
    scores = dbg["coarse_scores"].reshape(cr, cc, d)
    tx, ty = tiles_of(cc, cr, tile)
    expected = np.zeros(tx * ty, bool)
    for t in range(tx * ty):
        x, y = t % tx, t // tx
        o = offsets[t]
        tested = contradicted = 0
        for r in range(y * tile, min(cr, (y + 1) * tile)):
            for c in range(x * tile, min(cc, (x + 1) * tile)):
                row = scores[r, c]
                if not (np.isfinite(row[0]) or np.isfinite(row[o:o + band]).any()):
                    continue
                tested += 1
                w = winners[r * cc + c]
                contradicted += bool(np.isfinite(row[w]) and np.isfinite(row[0])
                                     and np.float32(row[w] + np.float32(0.12)) < row[0])
        expected[t] = contradicted > np.float32(fraction) * np.float32(tested)
    got = on.fallback.cpu().numpy().astype(bool)
    assert on.report["consistency_tiles"] > 0
    assert np.array_equal(got[~edge], expected[~edge])
    assert np.all(got[edge])
    # the nodes of tiles that kept their band keep the banded winner
    keep = np.repeat(np.repeat((~got).reshape(ty, tx), tile, 0), tile, 1)[:cr, :cc].reshape(-1)
    assert np.array_equal(on.winner.cpu().numpy()[keep], winners[keep])


def test_refusals(gpu_ctx, small):
    sc, dbg, cc, cr, d = small
    stage = _stage(sc, gpu_ctx)
    for bad in (BandOptions(None, 0, 12, 8), BandOptions(None, 9, 12, 8), BandOptions(None, 4, 33, 8),
                BandOptions(None, 4, 41, 8), BandOptions(None, 4, 12, 8, float("nan"))):
        with pytest.raises(RuntimeError, match="error 5"):
            coarse_depth(stage, bad)
    assert coarse_depth(stage, BandOptions(None, 4, 12, 8)).winner.numel() == cc * cr
