"""The hash-grid build that allocates nothing, checked through the C ABI against the regular
build (imbart_hashgrid_build) on the same photons, for two calls in a row.

Some callers cannot allocate device memory: a server that admits requests against a fixed
HBM budget (and must not let cudaMalloc/cudaFree synchronize the device under other
requests' streams), or a host that only hands out buffers from its own arena. For them
imbart_hashgrid_build_noalloc keeps its scratch in a static device array and writes to
outputs the caller allocated. Its results must equal the regular build's: identical grid
parameters and bucket ends, and the same photons in every bucket (the order inside a bucket
comes from atomic cursors in both builds, so buckets are compared as sets).
"""
import ctypes as C

import numpy as np
import pytest

from imbatracer_b200 import native as N

pytestmark = pytest.mark.gpu


class _DeviceView:
    """A device array the library owns, exposed to torch without a copy."""

    def __init__(self, ptr, shape, typestr):
        self.__cuda_array_interface__ = {"data": (ptr, False), "shape": shape, "typestr": typestr, "version": 3}


def regular_build(torch, pos_d, radius, cell_factor, table):
    from imbatracer_b200.hashgrid import HashGrid
    g = HashGrid(0)
    g.build(pos_d, radius, cell_factor, table)
    torch.cuda.synchronize()
    prm = g.params()
    sp, ep = C.c_void_p(), C.c_void_p()
    N.check(N.load().imbart_hashgrid_get_arrays(g.handle, C.byref(sp), C.byref(ep)), "arrays")
    n, t = prm["n"], prm["table_size"]
    sorted_h = torch.as_tensor(_DeviceView(sp.value, (n, 4), "<f4"), device="cuda").cpu().numpy()
    ends_h = torch.as_tensor(_DeviceView(ep.value, (t,), "<i4"), device="cuda").cpu().numpy()
    params = np.concatenate([prm["lo"], prm["hi"], [prm["radius"], prm["radius_sqr"], prm["cell_size"],
                                                    prm["inv_cell_size"]]]).astype(np.float32)
    g.close()
    return params, ends_h, sorted_h


def noalloc_build(torch, pos_d, radius, cell_factor, table):
    n = pos_d.shape[0]
    t = table if table > 0 else max(2 * n, 1)
    sorted_d = torch.full((max(n, 1), 4), -1.0, dtype=torch.float32, device="cuda")
    ends_d = torch.full((t,), -7, dtype=torch.int32, device="cuda")
    params_d = torch.zeros(10, dtype=torch.float32, device="cuda")
    rc = N.load().imbart_hashgrid_build_noalloc(N.ptr(pos_d), pos_d.shape[1], n, float(radius), float(cell_factor),
                                                int(table), N.ptr(sorted_d), N.ptr(ends_d), N.ptr(params_d), None)
    N.check(rc, "imbart_hashgrid_build_noalloc")
    torch.cuda.synchronize()
    return params_d.cpu().numpy(), ends_d.cpu().numpy(), sorted_d.cpu().numpy()[:n]


def bucket_sets(ends, sorted_rows):
    ids = sorted_rows[:, 3].copy().view(np.int32)
    out, start = {}, 0
    for b, e in enumerate(ends):
        if e > start:
            out[b] = sorted(ids[start:e].tolist())
        start = e
    return out


def test_noalloc_build_matches_regular_build_twice(cuda):
    import torch
    rng = np.random.default_rng(77)
    cases = [
        (rng.uniform(-5, 5, size=(200000, 3)).astype(np.float32), 0.05, 2.0, 0),       # reference parameters
        (rng.normal(size=(60000, 3)).astype(np.float32) * 3.0, 0.1, 1.0, 1 << 20),    # larger table, cell = r
    ]
    for pos, radius, cf, table in cases:            # two calls in a row, different inputs
        pos_d = torch.from_numpy(pos).cuda()
        p_ref, e_ref, s_ref = regular_build(torch, pos_d, radius, cf, table)
        p_new, e_new, s_new = noalloc_build(torch, pos_d, radius, cf, table)
        assert np.array_equal(p_ref.view(np.int32), p_new.view(np.int32))
        assert np.array_equal(e_ref, e_new)
        assert bucket_sets(e_ref, s_ref) == bucket_sets(e_new, s_new)
        # every photon lands exactly once, with its exact position
        ids = s_new[:, 3].copy().view(np.int32)
        assert np.array_equal(np.sort(ids), np.arange(len(pos)))
        assert np.array_equal(s_new[np.argsort(ids), :3].view(np.int32), pos.view(np.int32))


def test_noalloc_build_rejects_oversize(cuda):
    import torch
    lib = N.load()
    dummy = torch.zeros((4, 4), dtype=torch.float32, device="cuda")
    ends = torch.zeros(8, dtype=torch.int32, device="cuda")
    prm = torch.zeros(10, dtype=torch.float32, device="cuda")
    rc = lib.imbart_hashgrid_build_noalloc(N.ptr(dummy), 3, (1 << 20) + 1, 1.0, 2.0, 0, N.ptr(dummy), N.ptr(ends),
                                           N.ptr(prm), None)
    assert rc == 6 and "1048576 photons" in N.last_error()[1]
    rc = lib.imbart_hashgrid_build_noalloc(N.ptr(dummy), 3, 4, 1.0, 2.0, (1 << 21) + 1, N.ptr(dummy), N.ptr(ends),
                                           N.ptr(prm), None)
    assert rc == 6
