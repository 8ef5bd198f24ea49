"""CPU tests of the traversal boundary: the oracle against brute force, the restated 8-wide
walk against the oracle (which checks libimbart's layout conversion on the host), the
library's exported symbols, and the builder's reference-layout output."""
import ctypes as C
import re
import os

import numpy as np
import pytest

from imbatracer_b200 import native as N
from imbatracer_b200 import scene as S
from oracle import oracle as O
from tests import helpers as H

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if not f.endswith(".h"):
            continue
        text = open(os.path.join(inc, f)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b([a-z_][a-z0-9_]*)\s*\(", text, flags=re.M):
            name = m.group(1)
            if name not in ("if", "while", "for", "return", "sizeof", "defined"):
                names.add(name)
    return sorted(names)


def test_library_loads_and_exports_every_header_symbol():
    lib = N.load()
    declared = [n for n in header_functions() if n.startswith(("imbart_", "intersect_", "occluded_"))]
    assert "intersect_gpu_masked_instanced" in declared
    missing = [n for n in declared if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"
    unbound = [n for n in declared if n not in N.exported_symbols()]
    assert not unbound, f"declared but not bound in native.py: {unbound}"
    assert lib.imbart_version().startswith(b"imbart")


def header_arities():
    """Parameter count of every function the headers declare."""
    out = {}
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if not f.endswith(".h"):
            continue
        text = re.sub(r"/\*.*?\*/", "", open(os.path.join(inc, f)).read(), flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b((?:imbart|intersect|occluded)_[a-z0-9_]*)\s*\(", text, flags=re.M):
            depth, i, params = 1, m.end(), ""
            while depth:
                c = text[i]
                depth += (c == "(") - (c == ")")
                params += c if depth else ""
                i += 1
            params = params.strip()
            out[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_bindings_take_the_declared_number_of_arguments():
    """native.py's ctypes signatures match the C declarations in include/*.h, argument for
    argument (a missing or extra argument would pass garbage through the C ABI)."""
    lib = N.load()
    arity = header_arities()
    wrong = {}
    for name in N.exported_symbols():
        if name in arity:
            got = len(getattr(lib, name).argtypes or [])
            if got != arity[name]:
                wrong[name] = (arity[name], got)
    assert len(arity) > 50
    assert not wrong, f"declared vs bound argument counts: {wrong}"


def test_error_reporting_without_gpu():
    lib = N.load()
    lib.imbart_clear_error()
    rc = lib.imbart_trace(None, None, None, 10, 0, None)
    assert rc == 1
    code, msg = N.last_error()
    assert code == 1 and "imbart_trace" in msg
    lib.imbart_clear_error()
    assert N.last_error()[0] == 0


@pytest.mark.parametrize("name", ["tiny", "config1", "config2"])
def test_oracle_bvh_walk_matches_brute_force(name):
    d = H.scene_desc(name)
    td = H.traversal_data(name)
    n = 3000 if name != "config2" else 600
    rays = H.ray_set(name, n, seed=1)
    for any_hit in (False, True):
        hb, vb = O.trace_brute(d.meshes, d.instances, td.tri_layout, rays, any_hit=any_hit, with_v=True)
        h2, v2 = O.trace_node2(td, rays, any_hit=any_hit, with_v=True)
        if any_hit:
            # Any hit: occlusion must agree; the reported triangle may differ.
            assert np.array_equal(hb["tri_id"] >= 0, h2["tri_id"] >= 0)
        else:
            assert H.hits_equal(hb, h2).all()
            assert np.array_equal(vb.view(np.int32), v2.view(np.int32))


@pytest.mark.parametrize("name", ["config1", "config2"])
def test_object_split_bvh_walk_matches_brute_force(name):
    """Bottom levels built with object splits only (no duplicated references)."""
    d = H.scene_desc(name)
    td = S.build_traversal_data(d.meshes, d.instances, split_budget=0.0)
    rays = H.ray_set(name, 1500 if name != "config2" else 600, seed=5)
    hb, vb = O.trace_brute(d.meshes, d.instances, td.tri_layout, rays, with_v=True)
    h2, v2 = O.trace_node2(td, rays, with_v=True)
    assert H.hits_equal(hb, h2).all()
    assert np.array_equal(vb.view(np.int32), v2.view(np.int32))


def test_spatial_split_budget_bounds_references():
    """The reference count never exceeds the budget or the output capacity; a capacity too
    small for the triangles themselves is an error, not an overrun."""
    lib = N.load()
    m = H.scene_desc("config2").meshes[0]
    n = m.triangle_count
    for budget in (0.05, 0.5):
        nodes = np.zeros(4 * n, N.NODE2_DTYPE)
        tris = np.zeros((12 * n, 4), np.float32)
        nn, nt = C.c_int(0), C.c_int(0)
        rc = lib.imbart_build_mesh_node2_ex(N.ptr(m.vertices), len(m.vertices), 3, N.ptr(m.indices), n, 0, 2,
                                            C.c_float(budget), N.ptr(nodes), len(nodes), C.byref(nn), N.ptr(tris),
                                            len(tris), C.byref(nt))
        assert rc == 0
        assert n <= nt.value // 3 <= int(n * (1.0 + budget))
    cap = 3 * n + 30
    tris = np.zeros((cap, 4), np.float32)
    nn, nt = C.c_int(0), C.c_int(0)
    rc = lib.imbart_build_mesh_node2_ex(N.ptr(m.vertices), len(m.vertices), 3, N.ptr(m.indices), n, 0, 2,
                                        C.c_float(2.0), N.ptr(nodes), len(nodes), C.byref(nn), N.ptr(tris),
                                        cap, C.byref(nt))
    assert rc == 0 and n <= nt.value // 3 <= n + 10
    rc = lib.imbart_build_mesh_node2_ex(N.ptr(m.vertices), len(m.vertices), 3, N.ptr(m.indices), n, 0, 2,
                                        C.c_float(2.0), N.ptr(nodes), len(nodes), C.byref(nn), N.ptr(tris),
                                        3 * n - 3, C.byref(nt))
    assert rc != 0
    lib.imbart_clear_error()


@pytest.mark.parametrize("name", ["tiny", "config1", "config2"])
def test_wide_layout_walk_matches_oracle(name):
    """The restated GPU walk over libimbart's converted 8-wide layout finds bit-identical
    closest hits: the conversion (collapse + conservative 8-bit quantization) loses nothing."""
    td = H.traversal_data(name)
    wn, wt, wi, root = H.wide_arrays(td)
    rays = H.ray_set(name, 20000, seed=2)
    h2 = O.trace_node2(td, rays)
    hw, nbytes, counts = O.wide_walk(wn, wt, wi, root, rays)
    assert H.hits_equal(h2, hw).all()
    h2a = O.trace_node2(td, rays, any_hit=True)
    hwa, _, _ = O.wide_walk(wn, wt, wi, root, rays, any_hit=True)
    assert np.array_equal(h2a["tri_id"] >= 0, hwa["tri_id"] >= 0)
    assert (nbytes >= 48).all()
    assert counts[0] > 0 and counts[1] > 0


def test_wide_layout_invariants():
    td = H.traversal_data("config2")
    wn, wt, wi, root = H.wide_arrays(td)
    # every internal child index is in range, leaf ranges stay in the triangle/instance arrays
    for n in wn[:2000]:
        k = bin(int(n["imask"])).count("1")
        assert n["child_base"] + k <= len(wn)
        for s in range(8):
            meta = int(n["meta"][s])
            if not (int(n["imask"]) >> s) & 1 and meta:
                assert (meta >> 5) <= 3
    assert set(np.unique(wt["id"])) <= set(range(sum(m.triangle_count for m in H.scene_desc("config2").meshes)))
    assert len(wi) == len(H.scene_desc("config2").instances)
    assert 0 <= root < len(wn)


@pytest.mark.parametrize("split_budget", [0.0, 2.0])
def test_builder_writes_reference_layout(split_budget):
    """Leaves end with the 0x80000000 sentinel in the last v2.w, ids sit in v1.w
    (gpu_adapter.cpp:129-141), every triangle appears (exactly once without spatial splits,
    at most 1 + split_budget references per triangle on average with them), node links are
    in range."""
    d = H.scene_desc("config1")
    td = S.build_traversal_data(d.meshes, d.instances, split_budget=split_budget)
    tris = td.tris
    ids = tris[1::3, 3].view(np.int32)
    n = d.meshes[0].triangle_count
    if split_budget == 0.0:
        assert sorted(ids.tolist()) == list(range(n))
    else:
        assert np.array_equal(np.unique(ids), np.arange(n))
        assert n < len(ids) <= int(n * (1.0 + split_budget))
    sent = tris[2::3, 3].view(np.int32)
    assert (sent == np.int32(-2 ** 31)).sum() > 0
    nodes = td.nodes
    for k in ("left", "right"):
        c = nodes[k]
        inner = c[(c >= 0) & (c != 0x76543210)]
        assert (inner < len(nodes)).all()
        leaf = ~c[c < 0]
        assert (leaf < len(tris)).all() and (leaf % 3 == 0).all()
    assert td.root == td.layout[-1] + 0 or td.root >= td.layout[-1]


def test_single_triangle_mesh_root_wrapper():
    td = H.traversal_data("tiny")
    mesh1_root = td.layout[1]
    assert td.nodes[mesh1_root]["right"] == 0x76543210


def test_node_layout_guards():
    """Malformed input is rejected with an error, not a crash."""
    lib = N.load()
    td = H.traversal_data("tiny")
    cnt = np.zeros(4, np.int32)
    bad = td.nodes.copy()
    bad["left"][0] = 10 ** 6
    rc = lib.imbart_wide_from_node2(td.root, N.ptr(bad), len(bad), N.ptr(td.instances), len(td.instances),
                                    N.ptr(td.tris), len(td.tris), None, 0, None, 0, None, 0, N.ptr(cnt))
    assert rc == 4
    assert "out of bounds" in N.last_error()[1]
