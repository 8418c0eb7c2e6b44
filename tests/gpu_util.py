"""Helpers shared by the GPU parity tests."""
import numpy as np
import torch

from radiance_meshes_b200 import rasterizer as R
from radiance_meshes_b200.camera import tcam_to_struct


def to_dev(a, dev="cuda"):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def run_gpu_forward(verts, idx, cv, tcam, jitter, keep_debug=True, hit_masks=False):
    cam = tcam_to_struct(tcam)
    v, i, c, j = to_dev(verts), to_dev(idx), to_dev(cv), to_dev(jitter)
    tiles, rect, vs, cc = R.project_fwd(i, v, cam)
    lists = R.build_tile_lists(tiles, rect, vs, cam, keep_debug=keep_debug)
    img, dist, nc, recs = R.blend_fwd(lists.sorted_ids, lists.ranges, i, v, c, j, cam, tiles_touched=tiles,
                                      hit_masks=hit_masks)
    torch.cuda.synchronize()
    return dict(cam=cam, v=v, i=i, c=c, j=j, tiles=tiles, rect=rect, vs=vs, cc=cc, lists=lists, img=img,
                dist=dist, nc=nc, records=recs)


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32 if a.dtype == np.float32 else np.uint64)
