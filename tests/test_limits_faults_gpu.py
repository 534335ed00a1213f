"""Device-loop limits, cancellation and failure isolation, without faulting
the GPU: every failure here is made on the host (a per-call step limit of one
step, a cancel word set before the loop's first step, a volume of a dtype the
library rejects), the device loop returns an error status, and the context
stays usable for the next call.

The reference runs its growth as unbounded host loops
(_tier5/_masked_voronoi_labeling.py:62-69, _tier4/_connected_components_labeling_box.py:50-58);
here the loop runs on the device with per-call limits (cle_call_options)."""
import ctypes
import threading
import time

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


def _vol(shape=(24, 96, 96), n=30, seed=7):
    from pyclesperanto_prototype_b200 import synthetic
    return synthetic.nuclei_volume(shape, n, seed=seed)


def test_step_limit_raises_and_context_stays_usable(cle, oracle):
    vol = _vol()
    with cle.call_options(max_loop_steps=1):
        with pytest.raises(RuntimeError, match="voronoi_otsu_labeling"):
            cle.voronoi_otsu_labeling(vol, spot_sigma=2, outline_sigma=1)
    # the same thread without options, and the GPU, are unaffected
    got = cle.pull(cle.voronoi_otsu_labeling(vol, spot_sigma=2, outline_sigma=1))
    assert np.array_equal(got, oracle.voronoi_otsu_labeling(vol.astype(np.float32), 2, 1))


def test_step_limit_other_growth_ops(cle):
    vol = _vol(seed=8)
    binary = cle.threshold_otsu(cle.gaussian_blur(vol, sigma_x=1, sigma_y=1, sigma_z=1))
    spots = cle.detect_maxima_box(cle.gaussian_blur(vol, sigma_x=2, sigma_y=2, sigma_z=2))
    seeds = cle.binary_and(spots, binary)
    with cle.call_options(max_loop_steps=1):
        with pytest.raises(RuntimeError):
            cle.masked_voronoi_labeling(seeds, binary)
        with pytest.raises(RuntimeError):
            cle.masked_voronoi_labeling_binary(seeds, binary)
        with pytest.raises(RuntimeError):
            cle.voronoi_labeling(seeds)
    # options are per thread: another thread's calls run without the limit
    res = {}

    def other():
        res["labels"] = cle.pull(cle.voronoi_labeling(seeds))
    with cle.call_options(max_loop_steps=1):
        t = threading.Thread(target=other)
        t.start()
        t.join()
    assert res["labels"].max() > 0


def test_cooperative_cap_per_call_same_result(cle):
    vol = _vol(seed=9)
    ref = cle.pull(cle.voronoi_otsu_labeling(vol, spot_sigma=2, outline_sigma=1))
    for ctas in (1, 3, 16):
        with cle.call_options(cooperative_ctas=ctas):
            got = cle.pull(cle.voronoi_otsu_labeling(vol, spot_sigma=2, outline_sigma=1))
        assert np.array_equal(got, ref), ctas


def test_cancel_word_stops_the_loop(cle):
    """Through the C ABI: a cancel word that is already set stops the growth
    at its first step with CLE_ERR_CANCELLED in the status word."""
    from pyclesperanto_prototype_b200 import _lib
    lib = _lib.load()
    src = cle.push_native(_vol(seed=10))
    dst = cle.create_labels_like(src)
    s, d = _lib.tensor_desc(src.tensor), _lib.tensor_desc(dst.tensor)
    ws = torch.empty(int(lib.cle_voronoi_otsu_labeling_workspace_bytes(_lib.ref(s))), dtype=torch.uint8,
                     device="cuda")
    word = torch.ones(1, dtype=torch.int32).pin_memory()
    opts = _lib.call_options(cancel_ptr=word.data_ptr())
    stream = _lib.stream_ptr()
    assert lib.cle_voronoi_otsu_labeling(_lib.ref(s), _lib.ref(d), 2.0, 1.0, _lib.ref(opts), ws.data_ptr(),
                                         ws.numel(), stream) == 0
    assert lib.cle_workspace_status(ws.data_ptr(), ws.numel(), stream) == _lib.CLE_ERR_CANCELLED
    word.zero_()
    assert lib.cle_voronoi_otsu_labeling(_lib.ref(s), _lib.ref(d), 2.0, 1.0, _lib.ref(opts), ws.data_ptr(),
                                         ws.numel(), stream) == 0
    assert lib.cle_workspace_status(ws.data_ptr(), ws.numel(), stream) == 0
    # a cancel word in pageable memory is refused before any launch
    pageable = (ctypes.c_int32 * 1)()
    bad = _lib.call_options(cancel_ptr=ctypes.addressof(pageable))
    assert lib.cle_voronoi_otsu_labeling(_lib.ref(s), _lib.ref(d), 2.0, 1.0, _lib.ref(bad), ws.data_ptr(),
                                         ws.numel(), stream) == 3


def test_batch_check_reports_step_limit(cle):
    from pyclesperanto_prototype_b200 import synthetic
    from pyclesperanto_prototype_b200.batch import VolBatch
    tiles = [synthetic.blob_tile(s, 2e-3, seed=400 + i) for i, s in enumerate([(128, 128), (16, 64, 64)])]
    b = VolBatch(tiles, spot_sigma=3.5, outline_sigma=1.0, lanes=2, use_graph=False, max_loop_steps=1)
    b.run()
    with pytest.raises(RuntimeError, match="status 5"):
        b.check()
    ok = VolBatch(tiles, spot_sigma=3.5, outline_sigma=1.0, lanes=2, use_graph=False)
    ok.run()
    ok.check()


def _server_vols(n, seed0):
    from pyclesperanto_prototype_b200 import synthetic
    shapes = [(256, 256), (24, 128, 128), (300, 200), (16, 96, 96)]
    return [synthetic.blob_tile(shapes[i % 4], 1e-3 if len(shapes[i % 4]) == 2 else 3e-4, seed=seed0 + i)
            .to(torch.uint16).cpu().pin_memory() for i in range(n)]


def _same(a, m):
    assert torch.equal(a.labels, m.labels)
    assert a.num_labels == m.num_labels > 0
    sa, sm = a.statistics(), m.statistics()
    for k in sa:
        x, y = np.asarray(sa[k], np.float64), np.asarray(sm[k], np.float64)
        assert np.array_equal(np.isnan(x), np.isnan(y)), k
        ok = ~np.isnan(x)
        assert np.allclose(x[ok], y[ok], rtol=1e-5, atol=0), k


def test_server_isolates_failed_requests(cle):
    """One request hits the step limit, one has a dtype the library rejects,
    one is cancelled while waiting; the loop goes on and every other request
    equals the per-call result."""
    from pyclesperanto_prototype_b200.serving import Request, SegmentationServer, per_call_loop
    vols = _server_vols(6, 500)
    reqs = [Request(i, v, arrival=0.0) for i, v in enumerate(vols)]
    reqs[1].max_loop_steps = 1
    reqs.append(Request(6, torch.zeros((8, 32, 32), dtype=torch.float64), arrival=0.0))
    reqs.append(Request(7, vols[0], arrival=0.0))
    server = SegmentationServer(budget_bytes=8e9, slots=2, spot_sigma=2.0, outline_sigma=1.0, keep_labels=True)
    server.cancel(7)
    server.run(reqs, realtime=False)
    assert reqs[1].status == 5 and "status 5" in reqs[1].error and reqs[1].num_labels == 0
    assert reqs[6].status == 1 and "KeyError" in reqs[6].error
    assert reqs[7].cancelled and reqs[7].num_labels == 0
    good = [r for r in reqs if r.ok]
    assert [r.rid for r in good] == [0, 2, 3, 4, 5]
    alone = per_call_loop([Request(r.rid, vols[r.rid], arrival=0.0) for r in good], 2.0, 1.0,
                          realtime=False, keep_labels=True)
    for a, m in zip(alone, good):
        _same(a, m)
    # the same server serves a later batch normally
    again = [Request(10 + i, v, arrival=0.0) for i, v in enumerate(vols[:2])]
    server.run(again, realtime=False)
    assert all(r.ok for r in again)
    assert torch.equal(again[0].labels, good[0].labels)


def test_server_cancels_admitted_request(cle):
    """cancel() of a request already on the GPU: the request ends cancelled
    (stopped by its cancel word or discarded), the others finish."""
    from pyclesperanto_prototype_b200.serving import Request, SegmentationServer
    vols = _server_vols(4, 600)
    reqs = [Request(i, v, arrival=0.0) for i, v in enumerate(vols)]
    server = SegmentationServer(budget_bytes=8e9, slots=4, spot_sigma=2.0, outline_sigma=1.0)
    t = threading.Thread(target=server.run, args=(reqs,), kwargs={"realtime": False})
    t.start()
    t_end = time.time() + 30
    while reqs[2].admitted < 0 and reqs[2].done < 0 and time.time() < t_end:
        time.sleep(1e-4)
    server.cancel(2)
    t.join(60)
    assert not t.is_alive()
    # cancelled unless it had finished before cancel() was called
    assert reqs[2].cancelled or reqs[2].ok
    assert all(r.ok for r in reqs if r.rid != 2)


def test_two_servers_on_two_threads(cle):
    """Two servers in one process, each on its own host thread with its own
    streams and per-call CTA caps, give the per-call results."""
    from pyclesperanto_prototype_b200.serving import Request, SegmentationServer, per_call_loop
    vols = _server_vols(8, 700)
    out = {}

    def serve(name, vs, base):
        torch.cuda.set_device(0)
        reqs = [Request(base + i, v, arrival=0.0) for i, v in enumerate(vs)]
        SegmentationServer(budget_bytes=6e9, slots=3, spot_sigma=2.0, outline_sigma=1.0, keep_labels=True,
                           compute_streams=2, express_voxels=1 << 16).run(reqs, realtime=False)
        out[name] = reqs
    ts = [threading.Thread(target=serve, args=("a", vols[:4], 0)),
          threading.Thread(target=serve, args=("b", vols[4:], 4))]
    for t in ts:
        t.start()
    for t in ts:
        t.join(120)
    torch.cuda.synchronize()
    served = out["a"] + out["b"]
    assert all(r.ok for r in served)
    alone = per_call_loop([Request(i, v, arrival=0.0) for i, v in enumerate(vols)], 2.0, 1.0,
                          realtime=False, keep_labels=True)
    for a, m in zip(alone, served):
        _same(a, m)


def test_server_returns_labels_to_host(cle):
    from pyclesperanto_prototype_b200.serving import Request, SegmentationServer, per_call_loop
    vols = _server_vols(4, 800)
    outs = [torch.empty(tuple(v.shape), dtype=torch.uint32).pin_memory() for v in vols]
    reqs = [Request(i, v, arrival=0.0, labels_out=o) for i, (v, o) in enumerate(zip(vols, outs))]
    SegmentationServer(budget_bytes=8e9, slots=2, spot_sigma=2.0, outline_sigma=1.0).run(reqs, realtime=False)
    alone = per_call_loop([Request(i, v, arrival=0.0) for i, v in enumerate(vols)], 2.0, 1.0,
                          realtime=False, keep_labels=True)
    for a, o in zip(alone, outs):
        assert torch.equal(a.labels.cpu(), o)
