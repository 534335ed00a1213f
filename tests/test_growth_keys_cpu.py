"""The arrival-key formulation of the Voronoi growth (the rule the key growth
kernel relaxes, voronoi_bricks.cu) against the oracle's step-by-step masked
Voronoi (_tier5/_masked_voronoi_labeling.py:44-76), on the CPU.

A voxel labelled at step A gets the key K = s << 24 | (0xFFFFFF - label) with
s = A + 1 (seeds s = 0); a voxel's key is the minimum over its neighbours u of
K(u) + 2^24 (face neighbours) or (K(u) + 2^24) | 2^24 (edge / corner
neighbours: box steps only), each neighbour mapped before the minimum, and it
is recomputed from the neighbours (never min-accumulated with its own key).
Any order of re-evaluation reaches the fixpoint; the reference's stop at the
first step that labels nothing keeps the voxels of s below the smallest
unused s >= 1.  The test relaxes with random partial updates (a different
evaluation order in every case) and requires the oracle's labels exactly.
"""
import itertools

import numpy as np
import pytest

INF = (1 << 32) - 1
S1 = 1 << 24


def _neighbour_offsets(ndim):
    offs = []
    for d in itertools.product((-1, 0, 1), repeat=3):
        if d == (0, 0, 0) or (ndim == 2 and d[0] != 0):
            continue
        offs.append((d, abs(d[0]) + abs(d[1]) + abs(d[2]) == 1))
    return offs


def key_growth(seeds_lab, mask, rng, ndim):
    """Labels of the masked growth from seed labels (0 = none) by arrival keys."""
    D, H, W = mask.shape
    is_seed = seeds_lab > 0
    k = np.full(mask.shape, INF, np.int64)
    k[is_seed] = 0xFFFFFF - seeds_lab[is_seed]
    offs = _neighbour_offsets(ndim)
    face = lambda x: np.where(x >= INF, INF, x + S1)
    diag = lambda x: np.where(x >= INF, INF, (x + S1) | S1)
    while True:
        p = np.pad(k, 1, constant_values=INF)
        pd = diag(p)
        fm = np.full(k.shape, INF, np.int64)
        bm = np.full(k.shape, INF, np.int64)
        for (dz, dy, dx), is_face in offs:
            sl = (slice(1 + dz, 1 + dz + D), slice(1 + dy, 1 + dy + H), slice(1 + dx, 1 + dx + W))
            bm = np.minimum(bm, pd[sl])
            if is_face:
                fm = np.minimum(fm, p[sl])
        new = np.where(mask & ~is_seed, np.minimum(face(fm), bm), k)
        if np.array_equal(new, k):
            break
        upd = rng.random(k.shape) < 0.6          # chaotic order: a random subset per sweep
        k = np.where(upd, new, k)
    s = np.where(k >= INF, -1, k >> 24)
    used = set(np.unique(s[s >= 1]).tolist())
    stop = 1
    while stop in used:
        stop += 1
    keep = (k < INF) & (s < stop)
    return np.where(mask & keep, 0xFFFFFF - (k & 0xFFFFFF), 0).astype(np.uint32)


@pytest.mark.parametrize("ndim", [2, 3])
def test_arrival_keys_equal_the_reference_steps(oracle, ndim):
    rng = np.random.default_rng(7 + ndim)
    for trial in range(120):
        D = 1 if ndim == 2 else int(rng.integers(2, 6))
        H, W = int(rng.integers(3, 14)), int(rng.integers(3, 14))
        mask = rng.random((D, H, W)) < rng.uniform(0.3, 0.95)
        seeds = (rng.random((D, H, W)) < 0.04) & mask
        if not seeds.any():
            continue
        shape = (H, W) if ndim == 2 else (D, H, W)
        ref = oracle.masked_voronoi_labeling(seeds.reshape(shape).astype(np.uint8),
                                             mask.reshape(shape).astype(np.uint8))
        # the oracle's seed labels: connected components of the seeds
        lab0 = oracle.connected_components_labeling_box(seeds.reshape(shape).astype(np.uint8))
        got = key_growth(lab0.reshape(D, H, W).astype(np.int64), mask, rng, ndim)
        assert np.array_equal(got.reshape(shape), ref), (trial, shape)


def test_arrival_keys_keep_the_diagonal_stop(oracle):
    # a diagonal-only path: a face step changes nothing before the next box
    # step would, so the reference stops there and so must the cut
    n = 20
    mask = np.zeros((1, n, n), bool)
    for i in range(n):
        mask[0, i, i] = True
    mask[0, 0, 1] = True
    seeds = np.zeros_like(mask)
    seeds[0, 0, 0] = True
    ref = oracle.masked_voronoi_labeling(seeds[0].astype(np.uint8), mask[0].astype(np.uint8))
    got = key_growth(seeds.astype(np.int64), mask, np.random.default_rng(3), 2)
    assert np.array_equal(got[0], ref)
    assert (ref > 0).sum() < mask.sum()
