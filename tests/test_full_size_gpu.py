"""Parity at the benchmark sizes: the nuclei volume (uint16 128x512x512) and
the light-sheet volume (uint16 512x1024x1024) through voronoi_otsu_labeling and
statistics_of_labelled_pixels, against the oracle run on the host cores
(labels bit for bit, statistics within rtol 1e-5), plus properties that hold at
any size (sequential labels, labels exactly on the thresholded mask, repeated
runs identical).  The dense path (gauss_otsu_labeling) is compared on a
128-plane slab of the light-sheet volume (the oracle's union-find is
single-threaded)."""
import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

RTOL = 1e-5


@pytest.fixture(scope="module")
def cle():
    import pyclesperanto_prototype_b200 as m
    from pyclesperanto_prototype_b200 import _build
    _build.build()
    return m


def _stats_equal(got, ref):
    for k in ref:
        g, r = np.asarray(got[k], np.float64), np.asarray(ref[k], np.float64)
        assert g.shape == r.shape, k
        assert np.array_equal(np.isnan(g), np.isnan(r)), k
        m = ~np.isnan(r)
        assert np.allclose(g[m], r[m], rtol=RTOL, atol=0), k


def _check(cle, oracle, vol, spot, outline):
    import torch
    src = cle.push_native(vol)
    lab = cle.voronoi_otsu_labeling(src, spot_sigma=spot, outline_sigma=outline)
    got = cle.pull(lab)
    again = cle.pull(cle.voronoi_otsu_labeling(src, spot_sigma=spot, outline_sigma=outline))
    assert np.array_equal(got, again)                          # deterministic
    f = vol.astype(np.float32)
    ref, dbg = oracle.voronoi_otsu_labeling(f, spot, outline, debug=True)
    assert np.array_equal(got, ref)
    n = int(ref.max())
    assert n > 100
    assert np.array_equal(np.unique(got), np.arange(n + 1))    # sequential labels
    assert np.array_equal(got != 0, dbg["segmentation"] != 0)  # labels exactly on the mask
    _stats_equal(cle.statistics_of_labelled_pixels(src, lab), oracle.statistics_of_labelled_pixels(f, ref))
    del src, lab
    torch.cuda.empty_cache()


def test_nuclei_volume_128x512x512(cle, oracle):
    from pyclesperanto_prototype_b200 import synthetic
    vol = synthetic.cached("c2_nuclei_128x512x512_s1", synthetic.nuclei_volume)
    _check(cle, oracle, vol, 2.0, 1.0)


@pytest.fixture(scope="module")
def lightsheet():
    from pyclesperanto_prototype_b200 import synthetic
    return synthetic.lightsheet_volume((512, 1024, 1024), 30000, seed=2, device="cuda").cpu().numpy()


def test_lightsheet_volume_512x1024x1024(cle, oracle, lightsheet):
    _check(cle, oracle, lightsheet, 2.0, 2.0)


def test_lightsheet_dense_slab(cle, oracle, lightsheet):
    slab = np.ascontiguousarray(lightsheet[:128])
    got = cle.pull(cle.gauss_otsu_labeling(slab, outline_sigma=2))
    ref = oracle.gauss_otsu_labeling(slab.astype(np.float32), 2.0)
    assert ref.max() > 100
    assert np.array_equal(got, ref)
