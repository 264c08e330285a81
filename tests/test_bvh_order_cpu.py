"""The level-parallel form of the reference's BVH build that the GPU locator uses
(otmap_b200/csrc/locate.cu, build_bvh_order), replayed on the CPU with the kernels'
own index arithmetic, against the oracle's sequential restatement of the reference
build (bvh2d.cpp:29-64, 167-242): same final face array and the same leaf box per face.

Meshes include the undeformed grid, whose centroids fall exactly on split values for
odd n -- the case where split()'s return value depends on the element left at the
partition boundary and on how its loop exits.
"""

import numpy as np
import pytest

LEAF, DEPTH = 4, 24
EPS = np.finfo(np.float64).eps


def face_corners(xy, n):
    f = np.arange(n * n)
    i, j = f // n, f % n
    vid = np.stack([j + i * (n + 1), j + (i + 1) * (n + 1), (j + 1) + (i + 1) * (n + 1), (j + 1) + i * (n + 1)], 1)
    return xy[vid]  # (N, 4, 2)


def replay(xy, n):
    """The kernels of build_bvh_order, one level at a time (vectorised over positions)."""
    N = n * n
    P = face_corners(xy, n)
    cen = np.zeros((N, 2))
    for k in range(4):
        cen = cen + P[:, k, :]
    cen = cen / 4
    fbox = np.concatenate([P.min(axis=1), P.max(axis=1)], axis=1)
    fac = np.arange(N)
    node_of = np.zeros(N, dtype=np.int64)
    nodes = [dict(start=0, end=N)]
    rank = np.full(N, -1)
    lbox = np.zeros((N, 4))
    pos = np.arange(N)
    for level in range(DEPTH + 1):
        nxt = []
        act = node_of >= 0
        # k_bvh_bbox + k_bvh_decide
        for k, nd in enumerate(nodes):
            sel = node_of == k
            mn, mx = fbox[sel, :2].min(axis=0), fbox[sel, 2:].max(axis=0)
            diag = mx - mn
            en = diag * (2.0 * EPS) + EPS
            nd["box"] = np.concatenate([mn - en, mx + en])
            nd["leaf"] = (nd["end"] - nd["start"] <= LEAF) or level >= DEPTH
            if not nd["leaf"]:
                nd["dim"] = 1 if diag[1] > diag[0] else 0
                nd["sv"] = float(np.float32(0.5 * (nd["box"][2 + nd["dim"]] + nd["box"][nd["dim"]])))
        # k_bvh_classify
        small = np.zeros(N, dtype=np.int64)
        for k, nd in enumerate(nodes):
            if nd["leaf"]:
                continue
            sel = node_of == k
            small[sel] = (cen[sel, nd["dim"]] < nd["sv"]).astype(np.int64)
        spre = np.concatenate([[0], np.cumsum(small)])
        # k_bvh_slots
        slot_big = np.full(N, -1)
        slot_small = np.full(N, -1)
        for p in np.nonzero(act)[0]:
            nd = nodes[node_of[p]]
            if nd["leaf"]:
                continue
            s, e = nd["start"], nd["end"]
            S = spre[e] - spre[s]
            if not small[p] and p < s + S:
                slot_big[s + (p - s) - (spre[p] - spre[s])] = p
            elif small[p] and p >= s + S:
                slot_small[s + spre[e] - spre[p + 1]] = p
        # k_bvh_swap
        for p in np.nonzero(act)[0]:
            nd = nodes[node_of[p]]
            if nd["leaf"] or small[p]:
                continue
            s, e = nd["start"], nd["end"]
            S = spre[e] - spre[s]
            if p >= s + S:
                continue
            r = slot_small[s + (p - s) - (spre[p] - spre[s])]
            assert r >= 0
            fac[[p, r]] = fac[[r, p]]
            cen[[p, r]] = cen[[r, p]]
            fbox[[p, r]] = fbox[[r, p]]
        # k_bvh_children
        for nd in nodes:
            if nd["leaf"]:
                continue
            s, e = nd["start"], nd["end"]
            S = spre[e] - spre[s]
            if S == e - s:
                mid = e
            else:
                q = s + S
                m = S - (spre[q] - spre[s])
                eq = 1 if cen[q, nd["dim"]] == nd["sv"] else 0
                if eq and m >= 1 and slot_big[s + m - 1] == q - 2 and slot_small[s + m - 1] == q:
                    eq = 0
                mid = q + eq
            nd["mid"] = mid
            if mid == s or mid == e:
                nd["leaf"] = True
                continue
            nd["lo"], nd["hi"] = len(nxt), len(nxt) + 1
            nxt += [dict(start=s, end=mid), dict(start=mid, end=e)]
        # k_bvh_assign
        for p in np.nonzero(act)[0]:
            nd = nodes[node_of[p]]
            if nd["leaf"]:
                rank[fac[p]] = p
                lbox[fac[p]] = nd["box"]
                node_of[p] = -1
            else:
                node_of[p] = nd["lo"] if p < nd["mid"] else nd["hi"]
        nodes = nxt
        if not nodes:
            break
    assert (rank >= 0).all()
    return rank, lbox


def grid_xy(n):
    t = np.arange(n + 1, dtype=np.float64) / n
    return np.stack([np.repeat(t, n + 1), np.tile(t, n + 1)], axis=1)


def meshes(oracle_port):
    from otmap_b200 import workloads as W

    out = []
    for n in (1, 2, 3, 5, 8, 9, 17, 31, 33):
        out.append((f"grid{n}", n, grid_xy(n)))
    for n, seed in ((16, 0), (32, 1), (37, 2)):
        o = oracle_port.solve(W.to_cells(W.gaussian_mixture(n, seed)), n)
        out.append((f"solve{n}", n, o.fwd))
    o = oracle_port.solve(W.to_cells(W.blurred_shapes(48, 4, sigma_px=1.0)), 48)
    out.append(("shapes48", 48, o.fwd))
    rng = np.random.default_rng(3)
    n = 24
    xy = grid_xy(n)
    inner = (xy[:, 0] > 0) & (xy[:, 0] < 1) & (xy[:, 1] > 0) & (xy[:, 1] < 1)
    xy[inner] += rng.uniform(-0.3, 0.3, size=(inner.sum(), 2)) / n
    # some interior vertices snapped to multiples of 1/8, so centroids meet split values
    snap = inner & (rng.uniform(size=len(xy)) < 0.3)
    xy[snap] = np.round(xy[snap] * 8) / 8
    out.append(("jitter24", n, xy))
    return out


def test_level_parallel_build_matches_sequential(oracle_port):
    for name, n, xy in meshes(oracle_port):
        faces_ref, box_ref = oracle_port.bvh_order(xy, n)
        rank_ref = np.empty(n * n, dtype=np.int64)
        rank_ref[faces_ref] = np.arange(n * n)
        rank, lbox = replay(xy, n)
        assert np.array_equal(rank, rank_ref), name
        assert np.array_equal(lbox, box_ref), name


def test_replay_covers_the_equal_to_split_case():
    """On odd undeformed grids some centroid equals a split value at a node boundary."""
    n = 9
    xy = grid_xy(n)
    P = face_corners(xy, n)
    cen = P.sum(axis=1) / 4
    assert (cen[:, 0] == 0.5).any()
