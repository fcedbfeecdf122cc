"""Host collapse of the binary BVH into the 8-wide quantised layout the
trace kernels read (crt_bvh8_collapse), on the CPU: a binary tree in the
library's 64 B two-child layout is built here by a median split, collapsed
through the C ABI, and checked for

* structure: every binary leaf appears exactly once among the wide links,
  interior links point at wide nodes, and the depth matches;
* conservative boxes: every child box decoded the way the kernels decode it
  (fmaf(2^23 + q, 2^(e-127), p') with one rounding) contains the float
  bounds of every triangle below that child, so no hit can be pruned."""
import numpy as np
import pytest

from cudaraytracer_b200 import scenes
from cudaraytracer_b200.tracer import bvh8_collapse


def leaf_link(first, count):
    return ~((first << 4) | count)


def build_binary(tris, leaf_max=4):
    """Median-split binary BVH in the library's node layout. Returns
    (nodes (n,16) f32, leaf-ordered triangle indices, depth)."""
    t = tris.reshape(-1, 3, 3)
    cen = t.mean(1)
    lo_all, hi_all = t.min(1), t.max(1)
    nodes = []
    order = []

    def box(idx):
        return lo_all[idx].min(0), hi_all[idx].max(0)

    def rec(idx, depth):
        # returns link of this subtree
        if len(idx) <= leaf_max:
            first = len(order)
            order.extend(idx.tolist())
            return leaf_link(first, len(idx)), depth
        me = len(nodes)
        nodes.append(None)
        lo, hi = box(idx)
        ax = int(np.argmax(hi - lo))
        srt = idx[np.argsort(cen[idx, ax], kind="stable")]
        half = len(srt) // 2
        kids = (srt[:half], srt[half:])
        links, boxes, dmax = [], [], depth
        for k in kids:
            l, d = rec(k, depth + 1)
            links.append(l)
            boxes.append(box(k))
            dmax = max(dmax, d)
        (l0, h0), (l1, h1) = boxes
        n = np.zeros(16, np.float32)
        n[0:4] = [l0[0], h0[0], l0[1], h0[1]]
        n[4:8] = [l1[0], h1[0], l1[1], h1[1]]
        n[8:12] = [l0[2], h0[2], l1[2], h1[2]]
        n[12:14] = np.array(links, np.int32).view(np.float32)
        nodes[me] = n
        return me, dmax

    rec(np.arange(len(t)), 0)
    return np.stack(nodes).astype(np.float32), np.array(order), None


def decode(words, s, pp):
    """Decoded bounds (8,) of one axis for all slots: fmaf(2^23 + q, s, pp)
    as float32 (the product is exact, the float64 sum is exact for these
    magnitudes, so rounding it once to float32 is the fma's single rounding)."""
    q = np.frombuffer(np.asarray(words, np.uint32).tobytes(), np.uint8).astype(np.float64)
    return ((8388608.0 + q) * np.float64(s) + np.float64(pp)).astype(np.float32)


def wide_leaves(links):
    return sorted(int(l) for l in links.ravel() if l < 0)


@pytest.mark.parametrize("which", ["cornell", "icospheres", "soup"])
def test_collapse_structure_and_conservative_boxes(which):
    if which == "cornell":
        tris = scenes.cornell_box().triangles()
    elif which == "icospheres":
        tris = scenes.icosphere_field(n_spheres=6, level=2, with_env=False).triangles()
    else:
        rng = np.random.default_rng(3)
        c = rng.uniform(-50, 50, (3000, 1, 3))
        tris = (c + rng.normal(0, 0.02, (3000, 3, 3))).astype(np.float32).reshape(-1, 9)
    tris = np.asarray(tris, np.float32).reshape(-1, 9)
    bnodes, order, _ = build_binary(tris)
    wn, wl, depth = bvh8_collapse(bnodes)
    assert wn.shape[0] >= 1 and wl.shape == (wn.shape[0], 8)
    # structure: binary leaves appear once each among the wide links
    bin_leaves = sorted(int(x) for x in bnodes[:, 12:14].view(np.int32).ravel() if x < 0)
    w = wn.view(np.uint32)
    valid = (w[:, 3] >> 24) & 0xFF
    used = []
    for i in range(wn.shape[0]):
        for s in range(8):
            if valid[i] >> s & 1:
                used.append(int(wl[i, s]))
            else:
                assert wl[i, s] == 0
    assert sorted(l for l in used if l < 0) == bin_leaves
    inner = [l for l in used if l >= 0]
    assert sorted(inner) == list(range(1, wn.shape[0]))  # every wide node but the root is linked once
    # conservative boxes: decode every slot and check it contains its triangles
    t = tris.reshape(-1, 3, 3)

    def tri_bounds_of(link):
        if link < 0:
            code = ~link
            first, count = code >> 4, code & 15
            idx = order[first:first + count]
            return t[idx].min((0, 1)), t[idx].max((0, 1))
        los, his = [], []
        for s in range(8):
            if valid[link] >> s & 1:
                lo, hi = tri_bounds_of(int(wl[link, s]))
                los.append(lo)
                his.append(hi)
        return np.min(los, 0), np.max(his, 0)

    max_depth = [0]

    def check(node, level):
        max_depth[0] = max(max_depth[0], level + 1)
        hdr = w[node]
        s = [np.uint32(((hdr[3] >> (8 * k)) & 0xFF) << 23).view(np.float32) for k in range(3)]
        pp = wn[node, 0:3]
        qw = w[node, 4:16]
        dec_lo = [decode(qw[2 * k:2 * k + 2], s[k], pp[k]) for k in range(3)]
        dec_hi = [decode(qw[6 + 2 * k:6 + 2 * k + 2], s[k], pp[k]) for k in range(3)]
        for slot in range(8):
            if not (valid[node] >> slot & 1):
                continue
            lo, hi = tri_bounds_of(int(wl[node, slot]))
            for k in range(3):
                assert dec_lo[k][slot] <= lo[k], (node, slot, k, dec_lo[k][slot], lo[k])
                assert dec_hi[k][slot] >= hi[k], (node, slot, k, dec_hi[k][slot], hi[k])
            if wl[node, slot] >= 0:
                check(int(wl[node, slot]), level + 1)

    check(0, 0)
    assert depth == max_depth[0]


def test_collapse_single_leaf_tree():
    """The device builder's tree for a tiny soup: the root holds all
    triangles in child 0 and an empty leaf in child 1."""
    n = np.zeros((1, 16), np.float32)
    n[0, 0:4] = [0, 1, 0, 1]
    n[0, 4:8] = [0, 1, 0, 1]
    n[0, 8:12] = [0, 1, 0, 1]
    n[0, 12:14] = np.array([leaf_link(0, 3), leaf_link(0, 0)], np.int32).view(np.float32)
    wn, wl, depth = bvh8_collapse(n)
    assert wn.shape[0] == 1 and depth == 1
    valid = (wn.view(np.uint32)[0, 3] >> 24) & 0xFF
    assert bin(int(valid)).count("1") == 1
    assert sorted(int(x) for x in wl[0] if x < 0) == [leaf_link(0, 3)]
