"""Tile blend: drop-in for delaunay_rasterization/internal/alphablend_tiled_slang_interp.py
(``AlphaBlendTiledRender``), running the sm_100a kernels of librm_b200.so.

Tile sizes of 16, 64, 256 or 1024 pixels (4x4, 8x8, 16x16, 32x32 and other
shapes with those pixel counts) are supported; the reference compiles 4x4 only
(slang_modules.py:20).  The packed per-tet records built by the forward pass
are kept for the backward pass instead of being re-gathered.

``forward`` takes the reference's arguments (alphablend_tiled_slang_interp.py:11-14)
and nothing else.  When ``sorted_tetra_idx`` is the tensor that
``vertex_and_tile_shader`` returned, the projection's per-tet tile counts
travel with it, and only the records of visible tets are packed; for any other
tensor every tet is packed, with the same results.
"""
import torch

from ... import rasterizer as R
from ...camera import tcam_to_struct


class AlphaBlendTiledRender(torch.autograd.Function):
    @staticmethod
    def forward(ctx, sorted_tetra_idx, tile_ranges, indices, vertices, tet_density, render_grid, tcam,
                ray_jitter, device="cuda"):
        camst = tcam_to_struct(tcam)
        if (render_grid.image_height, render_grid.image_width) != (camst.image_height, camst.image_width):
            raise ValueError("render_grid and tcam disagree on the image size")
        if (render_grid.tile_height, render_grid.tile_width) != (camst.tile_height, camst.tile_width):
            raise ValueError("render_grid and tcam disagree on the tile size")
        indices = indices.contiguous()
        vertices = vertices.contiguous()
        tet_density = tet_density.contiguous()
        ray_jitter = ray_jitter.contiguous()
        frame = R.frame_of(sorted_tetra_idx)
        tiles_touched = frame.tiles_touched if frame is not None else None
        # lists of the 8x8-pixel tiles cut from these ones for this jitter (same image, fewer tests)
        fine = R.fine_lists_of(sorted_tetra_idx, camst, ray_jitter)
        if fine is not None:
            sorted_tetra_idx, tile_ranges, camst = fine.sorted_ids, fine.ranges, fine.cam
        # hit masks let the backward skip the forward's misses
        status = frame.status if frame is not None else None
        output_img, distortion_img, n_contributors, records = R.blend_fwd(
            sorted_tetra_idx, tile_ranges, indices, vertices, tet_density, ray_jitter, camst,
            tiles_touched=tiles_touched, hit_masks=True, status=status)
        tet_alive = torch.zeros((indices.shape[0]), dtype=torch.bool, device=vertices.device)
        ctx.save_for_backward(sorted_tetra_idx, tile_ranges, indices, vertices, tet_density, output_img,
                              distortion_img, n_contributors, ray_jitter)
        ctx.records = records
        ctx.status = status
        ctx.camst = camst
        ctx.render_grid = render_grid
        ctx.mark_non_differentiable(tet_alive)
        return output_img, distortion_img, tet_alive

    @staticmethod
    def backward(ctx, grad_output_img, grad_distortion_img, grad_vert_alive):
        (sorted_tetra_idx, tile_ranges, indices, vertices, tet_density, output_img, distortion_img,
         n_contributors, ray_jitter) = ctx.saved_tensors
        vertices_grad, tet_density_grad = R.blend_bwd(
            sorted_tetra_idx, tile_ranges, indices, vertices, tet_density, ray_jitter, ctx.camst, output_img,
            distortion_img, n_contributors, grad_output_img, grad_distortion_img, ctx.records, reuse_records=True,
            hit_masks=True, status=ctx.status)
        return (None, None, None, vertices_grad, tet_density_grad, None, None, None, None)
