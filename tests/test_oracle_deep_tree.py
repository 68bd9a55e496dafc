"""The oracle's traversal on a tree deeper than the reference's 32-entry stack (CPU): the tree really is that
deep, and the reference's early exit really removes pairs there, so the GPU test on it pins the exit."""
import collections

import numpy as np

from oracle import oracle as O
from tests import scenarios as SC


def _max_inner_depth(t):
    ni = t.n - 1
    depth, todo, deepest = {0: 0}, collections.deque([0]), 0
    while todo:
        u = todo.popleft()
        for c in t.children[u]:
            c = int(c)
            depth[c] = depth[u] + 1
            if c < ni:
                todo.append(c)
                deepest = max(deepest, depth[c])
    return deepest


def test_deep_tree_is_deeper_than_the_reference_stack_and_its_queries_end_early():
    for kind_name, kind in (("face", O.TREE_FACE), ("edge", O.TREE_EDGE)):
        x, el = SC.deep_tree_elements(kind_name)
        V = x.shape[0]
        t = O.lbvh_build(kind, x, el, V)
        assert t.healthy and _max_inner_depth(t) >= 32
        z = np.zeros(V, np.float32)
        O.lbvh_refit(t, x, x, el, z)
        small, big = np.full(V, 300.0, np.float32), np.full(V, 600.0, np.float32)
        q = O.lbvh_query_ee if kind_name == "edge" else O.lbvh_query_vf
        args = (el,) if kind_name == "edge" else ()
        _, n_small = q(t, x, x, *args, small, z)
        _, n_big = q(t, x, x, *args, big, z)
        # a larger query box can only find more pairs -- unless the walk ends early, as it does here
        assert n_small > 0 and n_big < n_small
