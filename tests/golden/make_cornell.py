"""Regenerates the Cornell-box fixtures in this folder from the reference's own code and
assets (oracle/_ref built from the reference sources, the reference's test scenes under
test/scenes/cornell, loaded from a temporary copy). Run from the repo root where the
reference tree exists:

    python tests/golden/make_cornell.py

For each scene, cornell_<name>.npz holds:
  * the scene as the asset loader reads it (imbatracer_b200.assets.load_scene_file; the CPU
    tests check that these arrays equal the reference frontend's), flattened by
    scene_to_arrays below;
  * ref_pt: the reference's PathTracer (its TileScheduler, oracle CPU traversal) on the
    scene as the reference's frontend built it: 64x64, 16 spp, max_path_len 10, seed 2024;
  * golden / golden_valid (scenes with a converged reference image in test/references):
    that image (1024x1024, 8-bit, gamma 0.5, written by store_png.h) decoded, linearized
    ((v / 255)^2) and averaged over 16x16 blocks to 64x64, and the blocks without clipped
    (255) texels.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from imbatracer_b200 import assets as A  # noqa: E402
from oracle import refwrap as R  # noqa: E402

SCENES = {"org": "ref_cornell_org.png", "indirect": "ref_cornell_indirect.png", "specular": "ref_cornell_specular.png",
          "specular_front": "ref_cornell_specular_front.png"}
W = H = 64
SPP, MAX_LEN, SEED = 16, 10, 2024


def scene_to_arrays(desc) -> dict:
    out = {"n_meshes": len(desc.meshes)}
    for k, m in enumerate(desc.meshes):
        for a in ("vertices", "indices", "normals", "texcoords", "geom_normals"):
            out[f"mesh{k}_{a}"] = getattr(m, a)
    out["inst_mesh"] = np.array([i.mesh_id for i in desc.instances], np.int32)
    out["inst_mats"] = np.stack([i.mat for i in desc.instances]).astype(np.float32)
    out["mat_kind"] = np.array([m.kind for m in desc.materials], np.int32)
    out["mat_params"] = np.array([list(m.color) + list(m.specular) + [m.exponent, m.eta, m.kappa] +
                                  list(m.emission) + [m.texture, m.bump] for m in desc.materials], np.float32)
    out["lights"] = np.array([np.concatenate([a, b, c, e]) for a, b, c, e in desc.lights], np.float32).reshape(-1, 12)
    c = desc.camera
    out["camera"] = np.array(list(c.pos) + list(c.dir) + list(c.up) + [c.fov], np.float32)
    return out


def main():
    import tempfile
    ref = R.reference_root()
    if ref is None:
        raise SystemExit("the reference tree is needed (build oracle/_ref first, or set IMBART_REFERENCE)")
    # The scenes are loaded from a copy: their `accel` lines make the reference write .bvh
    # cache files beside the meshes.
    tmp = tempfile.TemporaryDirectory()
    cornell = R.copy_reference_scenes(tmp.name)
    for name, golden in SCENES.items():
        path = os.path.join(cornell, f"cornell_{name}.scene")
        desc = A.load_scene_file(path, width=W, height=H)
        arrays = scene_to_arrays(desc)
        rs = R.RefScene.from_file(path, W, H)
        arrays["ref_pt"] = rs.render_pt(W, H, SPP, MAX_LEN, SEED)
        arrays["ref_settings"] = np.array([W, H, SPP, MAX_LEN, SEED], np.int64)
        gpath = os.path.join(ref, "test", "references", golden)
        if os.path.exists(gpath):
            img = A.load_png(gpath)[..., :3]
            lin = (img.astype(np.float64)) ** 2
            k = img.shape[0] // H
            arrays["golden"] = lin.reshape(H, k, W, k, 3).mean((1, 3)).astype(np.float32)
            arrays["golden_valid"] = ~(img >= 1.0).reshape(H, k, W, k, 3).any((1, 3, 4))
        np.savez_compressed(os.path.join(HERE, f"cornell_{name}.npz"), **arrays)
        print("wrote", f"cornell_{name}.npz", file=sys.stderr)


if __name__ == "__main__":
    main()
