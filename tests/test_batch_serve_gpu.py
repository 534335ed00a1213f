"""Batched and served forms give each volume the same result as the per-call
path: labels bit for bit, statistics bit for bit (same kernels, same order of
float64 accumulation is not guaranteed across calls, so rtol 1e-5)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cle():
    import pyclesperanto_prototype_b200 as m
    from pyclesperanto_prototype_b200 import _build
    _build.build()
    return m


def _tiles():
    from pyclesperanto_prototype_b200 import synthetic
    shapes = [(64, 64), (200, 130), (512, 512), (16, 96, 80), (33, 128, 100), (8, 256, 256),
              (96, 96), (40, 200, 160), (300, 70), (12, 64, 300), (24, 128, 128), (5, 33, 31)]
    return [synthetic.blob_tile(s, 5e-4 if len(s) == 3 else 2e-3, seed=100 + i) for i, s in enumerate(shapes)]


@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_matches_per_call(cle, use_graph):
    from pyclesperanto_prototype_b200.batch import VolBatch
    tiles = _tiles()
    b = VolBatch(tiles, spot_sigma=3.5, outline_sigma=1.0, lanes=4, use_graph=use_graph)
    b.run()
    b.run()                       # replay twice: buffers and status are reused
    torch.cuda.synchronize()
    b.check()
    for t, out in zip(tiles, b.outputs):
        ref = cle.voronoi_otsu_labeling(t, spot_sigma=3.5, outline_sigma=1.0)
        assert torch.equal(out, ref.tensor)
        assert int(ref.tensor.to(torch.int64).max()) > 0


def test_served_results_equal_alone_and_in_mix(cle):
    from pyclesperanto_prototype_b200 import synthetic
    from pyclesperanto_prototype_b200.serving import Request, SegmentationServer, per_call_loop
    shapes = [(256, 256), (24, 128, 128), (48, 160, 160), (256, 256), (24, 128, 128),
              (48, 160, 160), (300, 200), (24, 128, 128)]
    vols = [synthetic.blob_tile(s, 1e-3 if len(s) == 2 else 3e-4, seed=200 + i).to(torch.uint16).cpu().pin_memory()
            for i, s in enumerate(shapes)]
    mixed = [Request(i, v, arrival=0.0) for i, v in enumerate(vols)]
    SegmentationServer(budget_bytes=8e9, slots=3, spot_sigma=2.0, outline_sigma=1.0,
                       keep_labels=True).run(mixed, realtime=False)
    alone = per_call_loop([Request(i, v, arrival=0.0) for i, v in enumerate(vols)], 2.0, 1.0,
                          realtime=False, keep_labels=True)
    for a, m in zip(alone, mixed):
        assert torch.equal(a.labels, m.labels)
        assert a.num_labels == m.num_labels > 0
        sa, sm = a.statistics(), m.statistics()
        for k in sa:
            x, y = np.asarray(sa[k], np.float64), np.asarray(sm[k], np.float64)
            assert np.array_equal(np.isnan(x), np.isnan(y)), k
            ok = ~np.isnan(x)
            assert np.allclose(x[ok], y[ok], rtol=1e-5, atol=0), k


def test_served_budget_limits_concurrency(cle):
    from pyclesperanto_prototype_b200 import synthetic
    from pyclesperanto_prototype_b200.serving import Request, SegmentationServer, request_bytes
    vols = [synthetic.blob_tile((32, 192, 192), 3e-4, seed=300 + i).to(torch.uint16).cpu() for i in range(4)]
    one = request_bytes(tuple(vols[0].shape), vols[0].dtype)
    reqs = [Request(i, v, arrival=0.0) for i, v in enumerate(vols)]
    # a budget for one request at a time: each starts after the previous finished
    SegmentationServer(budget_bytes=1.5 * one, slots=4, spot_sigma=2.0, outline_sigma=1.0).run(reqs, realtime=False)
    order = sorted(reqs, key=lambda r: r.admitted)
    for a, b in zip(order, order[1:]):
        assert b.admitted >= a.done - 1e-3


def test_batch_plan_tuned_lanes_and_shape_check(cle):
    """lanes = 0 takes the lane count from the library's tuned table; a launch
    with tiles of other shapes than planned is refused before any work."""
    import ctypes
    from pyclesperanto_prototype_b200 import _lib
    from pyclesperanto_prototype_b200.batch import VolBatch
    tiles = _tiles()[:6]
    b = VolBatch(tiles, spot_sigma=3.5, outline_sigma=1.0, lanes=0, use_graph=False)
    assert 1 <= b.lanes <= len(tiles)
    b.run()
    b.check()
    for t, out in zip(tiles, b.outputs):
        assert torch.equal(out, cle.voronoi_otsu_labeling(t, spot_sigma=3.5, outline_sigma=1.0).tensor)
    lib = _lib.load()
    wrong = (_lib.CleTensor * len(tiles))(*[_lib.tensor_desc(t) for t in reversed(tiles)])
    st = lib.cle_vol_batch_launch(b._plan, wrong, b._out, b.ws.data_ptr(), b.ws.numel(), b.status.data_ptr(),
                                  torch.cuda.current_stream().cuda_stream)
    assert st == 2 and b"planned" in lib.cle_last_error_message()


def test_batch_graph_with_tma_staged_blur(cle):
    # a uint16 volume whose blur grid fills two waves takes the TMA-staged blur;
    # captured in the batch's CUDA graph it gives the per-call labels
    from pyclesperanto_prototype_b200 import synthetic
    from pyclesperanto_prototype_b200.batch import VolBatch
    vol = torch.from_numpy(synthetic.nuclei_volume((64, 704, 1000), 400, seed=9)).cuda()
    small = torch.from_numpy(synthetic.nuclei_volume((24, 96, 112), 40, seed=3)).cuda()
    b = VolBatch([vol, small], spot_sigma=2.0, outline_sigma=2.0, lanes=2, use_graph=True)
    b.run()
    b.run()
    torch.cuda.synchronize()
    b.check()
    for t, out in zip([vol, small], b.outputs):
        ref = cle.voronoi_otsu_labeling(cle.B200Array(t), spot_sigma=2.0, outline_sigma=2.0)
        assert torch.equal(out, ref.tensor)
        assert int(ref.tensor.to(torch.int64).max()) > 0
