"""Projection and tile binning: drop-in for
delaunay_rasterization/internal/tile_shader_slang.py (``vertex_and_tile_shader``,
``VertexShader``), running the sm_100a kernels of librm_b200.so.

Differences from the reference, none of them visible in the results:
  * the NaN check on vertices (reference line 78) is not a separate
    host-side assert, which would synchronise the stream: the projection
    kernel checks every tet's vertices (and that its indices lie in
    [0, n_verts)) and reports through the frame's device status word, which
    is read with the pair count; a NaN or infinite vertex or a bad index
    raises ``_capi.DeviceStatusError`` (a ``RuntimeError``) here, as the
    reference's assert raises;
  * the pair count is read back once instead of three times;
  * no cudaMalloc/cudaFree per call: scratch comes from a reusable pool.
"""
import torch

from ... import rasterizer as R
from ...camera import tcam_to_struct


def ceil_div(x, y):
    return (x + y - 1) // y


def vertex_and_tile_shader(indices, vertices, cam, render_grid):
    """Returns (sorted_tetra_idx [P] i32, tile_ranges [G,2] i32, vs_tetra [T,3],
    circumcenter [T,3], mask [T] bool, rect_tile_space [T,4] i32) exactly as
    the reference (tile_shader_slang.py:24-72).

    For tiles of 16x16 pixels or more, what it takes to cut the lists of the
    same frame on the grid of 8x8-pixel tiles (the tets' image footprints) is
    attached to the returned ``sorted_tetra_idx`` (attribute ``rm_fine``);
    ``AlphaBlendTiledRender`` cuts them for its ray jitter and blends over
    them when it is handed that tensor, which gives the same image with fewer
    ray/tet tests (see ``rasterizer.FineLists``).  The per-tet tile counts
    ride along the same way (attribute ``rm_frame``), so that the blend packs
    the records of visible tets only."""
    camst = tcam_to_struct(cam)
    fs = R.fine_shift_for(camst) if R.fine_lists_enabled() else 0
    pre = None
    if fs:
        with torch.no_grad():
            tiles, rect, vs, cc, footprint = R.project_fwd_fine(indices, vertices, camst)
        pre = (tiles, rect, vs, cc)
    tiles_touched, rect_tile_space, vs_tetra, circumcenter = VertexShader.apply(
        indices, vertices, cam, render_grid, "cuda", pre)
    with torch.no_grad():
        lists = R.build_tile_lists(tiles_touched, rect_tile_space, vs_tetra, camst)
        status = R.frame_status(indices.shape[0], vertices.device)
        R.attach_frame(lists.sorted_ids, tiles_touched, status)
        if fs:
            R.attach_fine_lists(lists.sorted_ids, lists.ranges, camst, fs, footprint, lists.sorted_keys, status)
    mask = tiles_touched > 0
    return lists.sorted_ids, lists.ranges, vs_tetra, circumcenter, mask, rect_tile_space


class VertexShader(torch.autograd.Function):
    @staticmethod
    def forward(ctx, indices, vertices, tcam, render_grid, device="cuda", precomputed=None):
        camst = tcam_to_struct(tcam)
        indices = indices.contiguous()
        vertices = vertices.contiguous()
        if precomputed is not None:  # outputs of project_fwd_fine for these inputs
            tiles_touched, rect_tile_space, vs_tetra, circumcenter = precomputed
        else:
            tiles_touched, rect_tile_space, vs_tetra, circumcenter = R.project_fwd(indices, vertices, camst)
        ctx.save_for_backward(indices, vertices, tiles_touched)
        ctx.camst = camst
        ctx.render_grid = render_grid
        ctx.mark_non_differentiable(tiles_touched, rect_tile_space)
        return tiles_touched, rect_tile_space, vs_tetra, circumcenter

    @staticmethod
    def backward(ctx, grad_tiles_touched, grad_rect_tile_space, grad_vs_tetra, grad_circumcenter):
        indices, vertices, tiles_touched = ctx.saved_tensors
        grad_vertices = R.project_bwd(indices, vertices, ctx.camst, tiles_touched, grad_vs_tetra,
                                      grad_circumcenter)
        return None, grad_vertices, None, None, None, None
