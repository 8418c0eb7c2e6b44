"""Generates the golden fixtures in this folder from the CPU oracle.

    python tests/golden/make_golden.py

Each .npz holds a scene's inputs (vertices, indices, cell values, camera,
ray jitter) and the oracle's outputs: the integer stages (tile counts,
rectangles, depth keys, sorted ids, ranges, n_contributors), the FP32
restatement's image / distortion and the FP64 integrator's image.  The
scenes follow the reference's renderer tests (tests/single_tet_test.py,
tests/multi_tet_test.py) and the gradient-check workload.  The fixtures pin
the oracle against drift (tests/test_oracle_golden.py) and give the GPU tests
committed expected values.
"""
import os
import sys
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle import oracle as O  # noqa: E402
from radiance_meshes_b200 import scenes  # noqa: E402
import scenarios  # noqa: E402

CAM_FIELDS = ["world_view", "K", "cam_pos", "min_t", "image_height", "image_width", "tile_height",
              "tile_width", "grid_height", "grid_width"]


def cases():
    out = {}
    for i, view in enumerate(["center", "center", "face", "outside"]):
        out[f"single_tet_{view}_{i}"] = scenarios.single_tet(100 + i, view)
    out["multi_tet_center"] = scenarios.multi_tet(7, 20, 10.0, "center")
    out["multi_tet_random_point"] = scenarios.multi_tet(7, 20, 10.0, "random_point")
    out["multi_tet_outside"] = scenarios.multi_tet(8, 20, 100.0, "outside", 100.0)
    mesh, view = scenes.workload_gradient_check()
    out["ball2000"] = (mesh.vertices, mesh.indices, mesh.cell_values, view.tcam())
    return out


def run_case(verts, idx, cv, tcam, jitter):
    L = O.rasterize_lists(idx, verts, tcam)
    img, dist, nc = O.blend_fwd_f32(L, idx, verts, cv, jitter)
    img64, dist64, _, own, inv = O.blend_fwd_f64(L, idx, verts.astype(np.float64), cv.astype(np.float64),
                                                 jitter, cut=nc)
    return L, img, dist, nc, img64, dist64


def main():
    for name, (verts, idx, cv, tcam) in cases().items():
        H, W = int(tcam["image_height"]), int(tcam["image_width"])
        jitter = np.random.default_rng(zlib.crc32(name.encode())).uniform(0, 1, (H, W, 2)).astype(np.float32)
        if name.startswith("single"):
            jitter[:] = 0.5
        L, img, dist, nc, img64, dist64 = run_case(verts, idx, cv, tcam, jitter)
        cs = L["cam"]
        camd = {f"cam_{k}": np.array(getattr(cs, k) if not hasattr(getattr(cs, k), "__len__")
                                     else list(getattr(cs, k))) for k in CAM_FIELDS}
        np.savez_compressed(
            os.path.join(HERE, f"{name}.npz"), vertices=verts, indices=idx, cell_values=cv, jitter=jitter,
            tiles_touched=L["tiles_touched"], rect=L["rect"], vs=L["vs"], circumcenter=L["circumcenter"],
            offsets=L["offsets"], keys=L["keys"], values=L["values"], sorted_keys=L["sorted_keys"],
            sorted_ids=L["sorted_ids"], ranges=L["ranges"], img=img, dist=dist, n_contrib=nc,
            img64=img64.astype(np.float32), dist64=dist64.astype(np.float32), **camd)
        print(name, "T", len(idx), "P", len(L["sorted_ids"]), "sum nc", int(nc.sum()))


if __name__ == "__main__":
    main()
