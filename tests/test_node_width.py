"""Node width (imbart_set_node_width): 4-wide trees in the 80-byte record, host side.

A 4-wide conversion fills slots 0..3 of each node in x/y-quadrant order and leaves slots
4..7 empty (no child, no primitives, an empty box). The restated walk over it finds the
same closest hits and occlusion answers as over the 8-wide tree and as the two-wide
reference layout.
"""
import numpy as np
import pytest

from imbatracer_b200 import native as N
from oracle import oracle as O
from tests import helpers as H


def test_width_setting_round_trip():
    lib = N.load()
    prev = lib.imbart_get_node_width()
    assert prev in (4, 8)
    try:
        assert lib.imbart_set_node_width(4) == 0 and lib.imbart_get_node_width() == 4
        assert lib.imbart_set_node_width(8) == 0 and lib.imbart_get_node_width() == 8
        for bad in (0, 2, 6, 16, -1):
            assert lib.imbart_set_node_width(bad) == 1   # IMBART_ERR_INVALID_ARGUMENT
            assert lib.imbart_get_node_width() == 8
        lib.imbart_clear_error()
    finally:
        lib.imbart_set_node_width(prev)


@pytest.mark.parametrize("name", ["tiny", "config1"])
def test_four_wide_layout_uses_four_slots(name):
    td = H.traversal_data(name)
    wn8, wt8, _, _ = H.wide_arrays(td, node_width=8)
    wn4, wt4, _, _ = H.wide_arrays(td, node_width=4)
    # Slots 4..7 are empty in every node: not internal, no primitive run, an empty box.
    assert (wn4["imask"] & 0xF0 == 0).all()
    assert (wn4["meta"][:, 4:] == 0).all()
    for a in "xyz":
        assert (wn4[f"qlo_{a}"][:, 4:] > wn4[f"qhi_{a}"][:, 4:]).all()
    # Every internal child and primitive run fits in four slots; the tree has more nodes.
    kids = np.array([bin(int(m)).count("1") for m in wn4["imask"]]) + (wn4["meta"][:, :4] != 0).sum(1)
    assert (kids >= 1).all() and (kids <= 4).all()
    if name != "tiny":
        assert len(wn4) > len(wn8)
    # The same triangle records (leaf order may differ).
    assert len(wt4) == len(wt8)
    assert sorted(wt4["id"].tolist()) == sorted(wt8["id"].tolist())


@pytest.mark.parametrize("name,n", [("tiny", 3000), ("config1", 20000)])
def test_four_wide_walk_equals_reference_layout(name, n):
    td = H.traversal_data(name)
    rays = H.ray_set(name, n, seed=11)
    ref = O.trace_node2(td, rays)
    refa = O.trace_node2(td, rays, any_hit=True)
    wn, wt, wi, root = H.wide_arrays(td, node_width=4)
    hits, _, counts = O.wide_walk(wn, wt, wi, root, rays)
    assert H.hits_equal(ref, hits).all()
    hitsa, _, _ = O.wide_walk(wn, wt, wi, root, rays, any_hit=True)
    assert np.array_equal(refa["tri_id"] >= 0, hitsa["tri_id"] >= 0)
    assert counts[0] > 0 and counts[1] > 0
