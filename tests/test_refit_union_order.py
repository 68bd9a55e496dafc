"""The refit's union order, on the CPU: the closed form the CUDA build uses for it (k_eorder in csrc/lbvh.cu)
against an explicit walk of the oracle's tree, and a fold of leaf boxes in that order against the oracle's
bottom-up refit, bit for bit, on boxes whose extremes tie at +0 and -0.

The reference unions each node's children in its child layout's order (lbvh.cpp:702-754; a right child that
is a leaf comes first, lbvh.cpp:561-592), with `a < b ? a : b`, which keeps the later of equal values.  A
node's box is therefore the fold of its leaves' boxes in the tree's in-order sequence taken in layout order,
and the GPU refit computes every inner box from its range of positions in that sequence."""
import numpy as np

from oracle import oracle as O


def _zero_tie_edges(g=40, seed=3):
    rng = np.random.default_rng(seed)
    ii, jj = np.meshgrid(np.arange(g), np.arange(g), indexing="ij")
    x = np.zeros((g * g, 4), np.float32)
    x[:, 0] = np.where(rng.random(g * g) < 0.5, np.float32(0.0), np.float32(-0.0))
    x[:, 1] = (ii.ravel() * 0.01).astype(np.float32)
    x[:, 2] = np.where(rng.random(g * g) < 0.5, np.float32(0.0), np.float32(-0.0))
    idx = ii * g + jj
    edges = np.concatenate([np.stack([idx[:, :-1].ravel(), idx[:, 1:].ravel()], 1),
                            np.stack([idx[:-1, :].ravel(), idx[1:, :].ravel()], 1)]).astype(np.uint32)
    return x, edges


def _union_order(t, n):
    """k_eorder's closed form: (position of each sorted leaf, first position of each inner node)."""
    ni = n - 1
    ch = np.asarray(t.children, np.int64).reshape(-1, 2)
    par = np.asarray(t.parent, np.int64)
    lo = np.zeros(2 * n - 1, np.int64)
    hi = np.zeros(2 * n - 1, np.int64)
    lo[ni:] = np.arange(n)
    hi[ni:] = np.arange(n)
    order, stack = [], [0]
    while stack:
        u = stack.pop()
        order.append(u)
        stack.extend(int(c) for c in ch[u] if c < ni)
    for u in reversed(order):
        a, b = ch[u]
        lo[u], hi[u] = min(lo[a], lo[b]), max(hi[a], hi[b])
    # a node whose right child is the leaf b has that leaf as its first child: +1 over its left range [a, b - 1]
    swapped = np.array([ch[i][0] >= ni and ch[i][0] - ni == hi[i] for i in range(ni)])
    diff = np.zeros(n + 1, np.int64)
    for i in np.nonzero(swapped)[0]:
        diff[lo[i]] += 1
        diff[hi[i]] -= 1
    cov = np.cumsum(diff)[:n]
    pos = np.array([lo[par[ni + p]] + cov[p] if (swapped[par[ni + p]] and hi[par[ni + p]] == p) else p + cov[p]
                    for p in range(n)])
    first = lo[:ni] + cov[hi[:ni]]
    return pos, first, lo, hi, ch


def test_union_order_closed_form_and_fold_match_the_walk():
    x, edges = _zero_tie_edges()
    n = edges.shape[0]
    ni = n - 1
    t = O.lbvh_build(O.TREE_EDGE, x, edges, x.shape[0])
    O.lbvh_refit(t, x, x.copy(), edges, np.zeros(x.shape[0], np.float32))
    pos, first, lo, hi, ch = _union_order(t, n)

    # the in-order sequence with children in layout order
    seq, stack = [], [0]
    while stack:
        u = stack.pop()
        if u >= ni:
            seq.append(u - ni)
            continue
        stack.extend([int(ch[u][1]), int(ch[u][0])])
    walk = np.empty(n, np.int64)
    walk[np.array(seq)] = np.arange(n)
    np.testing.assert_array_equal(pos, walk)
    leftmost = np.empty(ni, np.int64)
    for i in range(ni):
        u = i
        while u < ni:
            u = int(ch[u][0])
        leftmost[i] = walk[u - ni]
    np.testing.assert_array_equal(first, leftmost)

    # each inner box as the fold of its leaves in union order, `a < b ? a : b` with the earlier piece first
    boxes = np.asarray(t.node_aabb, np.float32).reshape(-1, 8)
    leaf = boxes[ni:][np.argsort(pos)]
    got = np.empty((ni, 6), np.float32)
    for i in range(ni):
        mn = [np.float32(np.inf)] * 3
        mx = [np.float32(-np.inf)] * 3
        for k in range(first[i], first[i] + hi[i] - lo[i] + 1):
            for c in range(3):
                mn[c] = mn[c] if mn[c] < leaf[k][c] else leaf[k][c]
                mx[c] = mx[c] if mx[c] > leaf[k][4 + c] else leaf[k][4 + c]
        got[i] = mn + mx
    want = np.concatenate([boxes[:ni, 0:3], boxes[:ni, 4:7]], axis=1)
    assert np.signbit(want[:, 0:3]).any() and (~np.signbit(want[:, 0:3])).any()
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))
    # a fold in sorted order instead is not the walk's result on these ties
    sorted_fold = np.empty((ni, 3), np.float32)
    for i in range(ni):
        mn = [np.float32(np.inf)] * 3
        for k in range(lo[i], hi[i] + 1):
            for c in range(3):
                mn[c] = mn[c] if mn[c] < boxes[ni + k][c] else boxes[ni + k][c]
        sorted_fold[i] = mn
    assert (sorted_fold.view(np.uint32) != want[:, 0:3].view(np.uint32)).any()
