"""Regenerates the golden vectors in this folder from the reference's own code (oracle/_ref,
built from the reference sources where the reference tree exists). Run from the repo root:

    python tests/golden/make_golden.py

Files: rng_seeding.npz (MWC64X sequences of random.h and the PixelRayGen seed scrambling of
ray_gen.h:49-72), hashgrid.npz (HashGrid::build/query of rangesearch.h), ref_layout_tiny.npz
(the reference adapters' GPU layout of a small scene and the hits the oracle finds on it).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from oracle import refwrap as R  # noqa: E402


def main():
    seeds = np.array([0, 1, 987654321, (-7) & (2 ** 64 - 1), 2 ** 63 + 5], np.uint64)
    floats = np.stack([R.rng_floats(int(s), 256) for s in seeds])
    _, _, _, st = R.camera_rays(8, 4, 3, [0, 0, -5], [0, 0, 1], [0, 1, 0], 60.0, 987654321)
    np.savez_compressed(os.path.join(HERE, "rng_seeding.npz"), seeds=seeds, floats=floats, seed_base=987654321,
                        spp=3, cam_states_after=st)

    from tests.test_hashgrid import photon_cloud, queries_near
    pos = photon_cloud(4000, 41)
    q = queries_near(pos, 600, 42, 0.4)
    ids, cnt = R.hashgrid_query(pos, 0.4, q, 10)
    np.savez_compressed(os.path.join(HERE, "hashgrid.npz"), pos=pos, queries=q, radius=np.float32(0.4), k=10,
                        ids=ids, counts=cnt)

    from tests import helpers as H
    desc = H.scene_desc("tiny")
    rs = R.RefScene(desc)
    root, nodes, insts, tris = rs.gpu_layout()
    nodes = nodes[: root + 8]   # the tiny scene's nodes all lie below root + 8
    from imbatracer_b200 import scene as S
    td = S.TraversalData(root, nodes, insts, tris, None, None, None, None, None, None)
    rays = H.ray_set("tiny", 600, seed=43)
    hits = O.trace_node2(td, rays)
    brute = O.trace_brute(desc.meshes, desc.instances, S.build_traversal_data(desc.meshes, desc.instances).tri_layout,
                          rays)
    assert (hits.view(np.int32) == brute.view(np.int32)).all()
    np.savez_compressed(os.path.join(HERE, "ref_layout_tiny.npz"), root=root, nodes=nodes.view(np.uint8),
                        insts=insts.view(np.uint8), tris=tris, rays=rays.view(np.uint8), hits=hits.view(np.uint8))
    print("golden vectors written")


if __name__ == "__main__":
    main()
