"""The per-tet feature producer that runs before the blend: a drop-in for
``activate_output`` (utils/model_util.py:93-105; offset_normalize :82-91,
eval_sh utils/eval_sh_py.py:138-200) computed by one fused sm_100a kernel per
direction (``rm_activate_features`` / ``rm_activate_features_bwd``).

``activate_output(camera_center, density, rgb, grd, sh, indices,
circumcenters, vertices, current_sh_deg, max_sh_deg)`` returns the [T, 7]
cell values (density, softplus(colour at v0 through the SH, beta 10), grd *
min(rgb) / |v0 - circumcenter|) with gradients for density, rgb, grd, sh,
circumcenters and vertices.
"""
from __future__ import annotations

import collections
import ctypes

import torch

from . import _capi as C
from . import rasterizer as R
from .camera import _key_of

__all__ = ["activate_output", "ActivateOutput"]


def _prep(t, dtype=torch.float32):
    """t detached, as a contiguous tensor of dtype (no copy when it is one)."""
    t = t.detach()
    return t if (t.dtype == dtype and t.is_contiguous()) else t.to(dtype).contiguous()


class ActivateOutput(torch.autograd.Function):
    @staticmethod
    def forward(ctx, camera_center, density, rgb, grd, sh, indices, circumcenters, vertices, sh_deg: int):
        for name, t in (("density", density), ("vertices", vertices), ("indices", indices)):
            if not t.is_cuda:
                raise RuntimeError(f"{name} must be a CUDA tensor (the producer has no CPU path)")
        T = indices.shape[0]
        dev = vertices.device
        idx = _prep(indices, torch.int32)
        v, cc = _prep(vertices), _prep(circumcenters)
        d, c, g = _prep(density).reshape(T), _prep(rgb).reshape(T, 3), _prep(grd).reshape(T, 3)
        shr = _prep(sh).reshape(T, -1, 3) if sh is not None and sh.numel() else torch.zeros((T, 0, 3), device=dev)
        cam = (ctypes_floats := _cam3(camera_center))
        feat = torch.empty((T, 7), dtype=torch.float32, device=dev)
        R._call("rm_activate_features", lambda: C.lib().rm_activate_features(
            C.ptr(idx), C.ptr(v), v.shape[0], C.ptr(cc), C.ptr(d), C.ptr(c), C.ptr(g), C.ptr(shr), shr.shape[1], int(sh_deg),
            ctypes_floats, T, C.ptr(feat), C.stream_handle()))
        ctx.save_for_backward(idx, v, cc, d, c, g, shr)
        ctx.cam = cam
        ctx.sh_deg = int(sh_deg)
        ctx.shapes = (density.shape, rgb.shape, grd.shape, None if sh is None else sh.shape, vertices.shape)
        return feat

    @staticmethod
    def backward(ctx, grad_feat):
        idx, v, cc, d, c, g, shr = ctx.saved_tensors
        T = idx.shape[0]
        gf = grad_feat.to(torch.float32).contiguous()
        gd = torch.empty(T, device=v.device)
        grgb = torch.empty((T, 3), device=v.device)
        ggrd = torch.empty((T, 3), device=v.device)
        gsh = torch.empty_like(shr)
        gv = torch.zeros_like(v)
        gcc = torch.empty_like(cc)
        R._call("rm_activate_features_bwd", lambda: C.lib().rm_activate_features_bwd(
            C.ptr(idx), C.ptr(v), v.shape[0], C.ptr(cc), C.ptr(d), C.ptr(c), C.ptr(g), C.ptr(shr), shr.shape[1], ctx.sh_deg,
            ctx.cam, T, C.ptr(gf), C.ptr(gd), C.ptr(grgb), C.ptr(ggrd), C.ptr(gsh), C.ptr(gv), C.ptr(gcc),
            C.stream_handle()))
        ds, rs, gs, ss, vs = ctx.shapes
        return (None, gd.reshape(ds), grgb.reshape(rs), ggrd.reshape(gs), None if ss is None else gsh.reshape(ss),
                None, gcc, gv.reshape(vs), None)


_CAM3: "collections.OrderedDict" = collections.OrderedDict()


def _cam3(camera_center):
    """The camera centre as three host floats.  Reading a device tensor waits
    on the stream, so the values are cached per tensor (identity, storage and
    in-place version, with the tensor held by the cache, as camera.tcam_to_struct
    does): a training loop that passes the same camera tensor every step reads
    it once."""
    key = _key_of(camera_center)
    hit = _CAM3.get(key)
    if hit is not None:
        _CAM3.move_to_end(key)
        return hit[1]
    vals = [float(x) for x in torch.as_tensor(camera_center).detach().reshape(-1)[:3].cpu()]
    out = (ctypes.c_float * 3)(*vals)
    _CAM3[key] = (camera_center, out)
    if len(_CAM3) > 64:
        _CAM3.popitem(last=False)
    return out


def activate_output(camera_center, density, rgb, grd, sh, indices, circumcenters, vertices, current_sh_deg: int,
                    max_sh_deg: int):
    """Same arguments and result as the reference's activate_output."""
    return ActivateOutput.apply(camera_center, density, rgb, grd, sh, indices, circumcenters, vertices,
                                int(current_sh_deg))
