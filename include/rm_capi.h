/*
 * rm_capi.h - C ABI of the B200 tetrahedral tile rasterizer (sm_100a).
 *
 * Each entry point replaces one kernel launch (or one library call) of the
 * reference rasterizer in delaunay_rasterization/internal/.  Arguments are raw
 * device pointers, element counts, a POD camera and a cudaStream_t passed as
 * void*.  No torch types cross this boundary.  Every function returns an int
 * status (RM_OK on success) and never throws; the message of the last failure
 * on the calling thread is available from rm_last_error().
 *
 * Memory ownership: the caller allocates every buffer, including scratch
 * ("workspace") memory whose size is returned by the *_workspace_size queries
 * (two-phase, as with CUB).  The library itself never calls cudaMalloc on the
 * render path.  All launches are stream-ordered; apart from rm_read_status and
 * rm_scan_noalloc_read_status no call synchronises the host with the device.
 *
 * Errors found on the device (an index outside [0, n_verts), a non-finite
 * vertex, a pair count beyond int32, a full buffer, a bounded wait that gave
 * up) set RM_STATUS_* bits in a caller-visible status word instead of
 * faulting or stopping the stream; the work item concerned is skipped and
 * every store stays in bounds.  The reference asserts on the host instead
 * (delaunay_rasterization/internal/tile_shader_slang.py:78), which would
 * synchronise the stream.
 *
 * Tensor layouts follow the reference: indices [T,4] int32, vertices [V,3]
 * float32, cell_values [T,7] float32 (density, r, g, b, gx, gy, gz),
 * ray_jitter [H,W,2], output image [H,W,4] (r, g, b, log-transmittance),
 * distortion [H,W,5], n_contributors [H,W] int32, tile ranges [G,2] int32.
 */
#ifndef RM_CAPI_H
#define RM_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RM_ABI_VERSION 2

#if defined(__GNUC__)
#define RM_API __attribute__((visibility("default")))
#else
#define RM_API
#endif

/* Status codes. */
#define RM_OK 0
#define RM_EINVAL 1      /* bad argument (null pointer, size, unsupported camera)   */
#define RM_ECAPACITY 2   /* an output buffer is smaller than the pairs produced       */
#define RM_ECUDA 3       /* a CUDA runtime call failed                                */
#define RM_ETIMEOUT 4    /* a bounded device-side wait gave up (see rm_read_status)   */

/* Bits of a device status word (uint32, or-ed by the kernels, read and
 * cleared with rm_read_status). */
#define RM_STATUS_SCAN_TIMEOUT 0x1u   /* a scan look-back gave up (offsets invalid)          */
#define RM_STATUS_SORT_TIMEOUT 0x2u   /* a sort look-back gave up (order invalid)            */
#define RM_STATUS_CAPACITY 0x4u       /* more pairs than the buffers hold (retry larger)     */
#define RM_STATUS_QUEUE_TIMEOUT 0x8u
#define RM_STATUS_BAD_INDEX 0x10u     /* a tet index outside [0, n_verts): tet culled, unread */
#define RM_STATUS_NONFINITE 0x20u     /* a tet vertex is NaN or infinite: tet culled          */
#define RM_STATUS_OVERFLOW 0x40u      /* the pair count exceeds INT32_MAX (int32 offsets)     */

/*
 * Camera.  Mirrors the reference's TensorCamera/Camera
 * (delaunay_rasterization/internal/slang/camera.slang:13-76) as filled by
 * utils/train_util.py:31-38 and data/camera.py:72-91.
 * world_view is row-major world->camera (tcam['world_view_transform']),
 * K is row-major 3x3 intrinsics.  camera_type 0 (perspective) and 1
 * (fisheye) are supported, each with the radial/tangential distortion
 * (k1, k2, p1, p2); any other camera_type is rejected with RM_EINVAL.
 */
typedef struct rm_camera {
    float world_view[16];
    float K[9];
    float cam_pos[3];
    float min_t;
    float distortion[4];
    int32_t camera_type;
    int32_t image_height;
    int32_t image_width;
    int32_t tile_height;
    int32_t tile_width;
    int32_t grid_height;
    int32_t grid_width;
    int32_t reserved;
} rm_camera;

/* Message of the last failing call on this thread ("" if none). */
RM_API const char* rm_last_error(void);
RM_API int rm_abi_version(void);

/* Number of kernels this library has launched in the calling process. */
RM_API uint64_t rm_launch_count(void);

/*
 * Copies the device status word (RM_STATUS_* bits) held in a workspace to the
 * host and clears it.  This is the only call here that synchronises `stream`.
 */
RM_API int rm_read_status(const uint32_t* status_dev, uint32_t* status_host, void* stream);

/*
 * Iteration limit of every bounded device-side wait launched after this call
 * by any thread of the process (scan and sort look-backs); 0 restores the
 * default of 2^22 polls (about a second).  A wait that reaches the limit sets
 * its RM_STATUS_*_TIMEOUT bit and the kernel goes on with every store in
 * bounds.  Small values make waits give up on purpose (tests of the error
 * path); there is no other reason to change it.
 */
RM_API void rm_set_wait_limit(uint32_t polls);
RM_API uint32_t rm_wait_limit(void);

/* ---------------------------------------------------------------- stage (a) */
/*
 * Per-tet projection, cull, tile rectangle and depth key.
 * Replaces vertex_shader (delaunay_rasterization/internal/slang/vertex_shader.slang:23-89)
 * launched by VertexShader.forward (delaunay_rasterization/internal/tile_shader_slang.py:77-105).
 * Every output row is written (culled tets get zeros), so the caller need not
 * zero the outputs.  vs is [T,3] with only column 2 (the float depth key) set,
 * as in the reference.  A tet with an index outside [0, n_verts) is culled
 * before any vertex load and sets RM_STATUS_BAD_INDEX; a tet with a NaN or
 * infinite vertex is culled and sets RM_STATUS_NONFINITE (the reference
 * asserts on NaN vertices on the host, tile_shader_slang.py:78).  The bits are
 * or-ed into *status_dev (may be NULL).
 */
RM_API int rm_project_fwd(const int32_t* indices, const float* vertices, int64_t n_tets,
                   int64_t n_verts, const rm_camera* cam, int32_t* tiles_touched,
                   int32_t* rect, float* vs, float* circumcenter, uint32_t* status_dev,
                   void* stream);

/*
 * Adjoint of the projection: dL/dvertices from dL/dvs[:,2] and dL/dcircumcenter
 * through the FP64 circumsphere power.  Replaces vertex_shader.bwd
 * (delaunay_rasterization/internal/tile_shader_slang.py:128-150).
 * grad_vertices [V,3] is accumulated into (atomics); the caller zeroes it.
 * grad_vs or grad_circumcenter may be NULL (treated as zeros).
 */
RM_API int rm_project_bwd(const int32_t* indices, const float* vertices, int64_t n_tets,
                   int64_t n_verts, const rm_camera* cam, const int32_t* tiles_touched,
                   const float* grad_vs, const float* grad_circumcenter,
                   float* grad_vertices, void* stream);

/* ---------------------------------------------------------------- stage (b) */
RM_API size_t rm_scan_workspace_size(int64_t n_tets);

/*
 * Inclusive int32 prefix sum of tiles_touched; the total pair count P is
 * written to *total_dev (int64, device memory).  Replaces
 * torch.cumsum(tiles_touched) at delaunay_rasterization/internal/tile_shader_slang.py:36.
 * Single pass with decoupled look-back; a look-back that waits too long sets
 * RM_STATUS_SCAN_TIMEOUT in the workspace status word (first 4 bytes), and a
 * total above INT32_MAX (the offsets are int32, as the reference's cumsum)
 * sets RM_STATUS_OVERFLOW there.  The word keeps its bits across calls until
 * rm_read_status clears it; the rest of the workspace is reset by every call.
 */
RM_API int rm_scan_tiles(const int32_t* tiles_touched, int64_t n_tets, int32_t* offsets,
                  int64_t* total_dev, void* workspace, size_t workspace_bytes,
                  void* stream);

/*
 * rm_scan_tiles without a workspace argument: no counterpart in the reference.
 * For callers that cannot allocate device memory (for example a host runtime
 * that passes the library only its inputs and outputs and has no device
 * allocator of its own).  The look-back scratch is a fixed array inside the
 * library (about 128 KiB per GPU, held until the process exits), so at most
 * 2^26 tets are accepted; larger inputs return RM_EINVAL.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress) and caches
 * it; make that first call before any stream capture.  All calls share the one
 * array: calls whose kernels overlap on the GPU (different streams, or
 * different host threads without ordering between them) race and must not be
 * issued.  The call allocates nothing (no cudaMalloc, no allocating library
 * routine); it clears the part of the array that must start at zero itself.
 * The array's address is looked up once per CUDA context (a context created
 * after cudaDeviceReset, or another context made current by the driver API,
 * gets its own lookup).  Timeouts and overflow set their bits in the array's
 * status word, which rm_scan_noalloc_read_status reads.
 */
RM_API int rm_scan_tiles_noalloc(const int32_t* tiles_touched, int64_t n_tets, int32_t* offsets,
                                 int64_t* total_dev, void* stream);

/*
 * Reads and clears the status word (RM_STATUS_* bits) of the fixed scratch of
 * rm_scan_tiles_noalloc in the current context, after the work queued on
 * `stream`; synchronises `stream`.  Allocates nothing.  No counterpart in the
 * reference.
 */
RM_API int rm_scan_noalloc_read_status(uint32_t* status_host, void* stream);

/*
 * Tile/tet pair emission: key = (tile_id << 32) | sortable(depth), value = tet
 * id, rows in row-major rectangle order at the tet's exclusive offset.
 * Replaces generate_keys (delaunay_rasterization/internal/slang/tile_shader.slang:138-186)
 * launched at delaunay_rasterization/internal/tile_shader_slang.py:46-55.
 * Pairs at positions >= capacity are dropped; if total_dev is non-NULL and
 * *total_dev > capacity, RM_STATUS_CAPACITY is or-ed into *status_dev
 * (status_dev may be NULL).
 */
RM_API int rm_emit_pairs(const float* vs, const int32_t* rect, const int32_t* offsets,
                  int64_t n_tets, int32_t grid_width, int64_t capacity,
                  const int64_t* total_dev, int64_t* keys, int32_t* values,
                  uint32_t* status_dev, void* stream);

/* ---------------------------------------------------------------- stage (c) */
RM_API size_t rm_sort_workspace_size(int64_t n);

/*
 * Stable LSD radix sort (onesweep) of (key, value) pairs on key bits
 * [0, end_bit).  Replaces sort_by_keys
 * (delaunay_rasterization/internal/sort_by_keys/sort_by_keys.cu:10-53), which
 * calls cub::DeviceRadixSort::SortPairs with end_bit = 32 + highest_tile_id_msb
 * (delaunay_rasterization/internal/tile_shader_slang.py:57-59).
 * n is the buffer capacity; if n_dev is non-NULL the pair count is read from
 * device memory (<= n) so the call can be captured in a CUDA graph.
 * Inputs are not modified.  Look-back waits are bounded: one that gives up
 * sets RM_STATUS_SORT_TIMEOUT in *status_dev, or, when status_dev is NULL, in
 * the workspace's status word (its first 4 bytes).
 */
RM_API int rm_sort_pairs(const int64_t* keys_in, const int32_t* values_in, int64_t n,
                  const int64_t* n_dev, int end_bit, int64_t* keys_out,
                  int32_t* values_out, void* workspace, size_t workspace_bytes,
                  uint32_t* status_dev, void* stream);

/*
 * rm_sort_pairs on key bits [begin_bit, end_bit) only (cub::DeviceRadixSort::
 * SortPairs with a begin bit); stable, so equal keys keep their input order.
 */
RM_API int rm_sort_pairs_range(const int64_t* keys_in, const int32_t* values_in, int64_t n,
                               const int64_t* n_dev, int begin_bit, int end_bit, int64_t* keys_out,
                               int32_t* values_out, void* workspace, size_t workspace_bytes,
                               uint32_t* status_dev, void* stream);

/*
 * Depth-first list build, the same sorted lists in fewer sort passes (no
 * reference counterpart; the reference sorts the pairs once on 32 + msb
 * bits):
 *   1. rm_depth_order: the visible tets (tiles_touched > 0), in tet order,
 *      as (key = sortable depth key of vs[:,2], value = tet id) pairs;
 *      *n_visible_dev = their count.  Workspace rm_depth_order_workspace_size(T).
 *   2. rm_sort_pairs_range(..., 0, 32, ...) over them (stable: equal depths
 *      stay in tet order).
 *   3. rm_emit_pairs_ordered: the pairs of the tets in that order (keys and
 *      values as rm_emit_pairs); *total_dev = pair count; the tile counts are
 *      scanned in that order internally.  Workspace
 *      rm_emit_ordered_workspace_size(T).
 *   4. rm_sort_pairs_range(..., 32, 32 + msb, ...): a stable sort on the tile
 *      bits alone, which leaves each tile's pairs in (depth, tet id) order:
 *      keys and values equal rm_sort_pairs(..., 32 + msb, ...) of
 *      rm_emit_pairs' tet-order emission.
 */
RM_API size_t rm_depth_order_workspace_size(int64_t n_tets);
RM_API int rm_depth_order(const int32_t* tiles_touched, const float* vs, int64_t n_tets,
                          int64_t* keys, int32_t* values, int64_t* n_visible_dev,
                          void* workspace, size_t workspace_bytes, uint32_t* status_dev,
                          void* stream);
/*
 * The pair count of a frame before its lists are built: out[0] = the sum of
 * the positive tiles_touched (int64), the number the reference reads back
 * as the last inclusive offset (delaunay_rasterization/internal/tile_shader_slang.py:38-44)
 * and the count that steps 1-4 above emit and sort; out[1] = the status word
 * *status_dev (NULL: 0) as the work queued before this call left it, so one
 * read of out gives both.  Read on another stream, out tells the caller P
 * without waiting for the list build: it can size the pair buffers exactly
 * before it queues steps 3-4, or queue them on buffers sized from an
 * estimate and check the estimate against out[0] (steps 3-4 set
 * RM_STATUS_CAPACITY when it was too small).  The caller compares out[0]
 * with INT32_MAX (the lists' offsets are int32).
 */
RM_API int rm_count_pairs(const int32_t* tiles_touched, int64_t n_tets, const uint32_t* status_dev,
                          int64_t* out, void* stream);
RM_API size_t rm_emit_ordered_workspace_size(int64_t n_tets);
RM_API int rm_emit_pairs_ordered(const float* vs, const int32_t* rect, const int32_t* tiles_touched,
                                 const int32_t* order, int64_t n_tets, const int64_t* n_items_dev,
                                 int32_t grid_width, int64_t capacity, int64_t* total_dev,
                                 int64_t* keys, int32_t* values, void* workspace,
                                 size_t workspace_bytes, uint32_t* status_dev, void* stream);

/*
 * Per-tile [start, end) ranges of the sorted pair list; empty tiles get [0,0].
 * Replaces compute_tile_ranges (delaunay_rasterization/internal/slang/tile_shader.slang:188-214)
 * launched at delaunay_rasterization/internal/tile_shader_slang.py:61-69 (the
 * ranges buffer is zero-filled here, as the reference's torch.zeros does).
 */
RM_API int rm_tile_ranges(const int64_t* sorted_keys, int64_t n, const int64_t* n_dev,
                   int32_t* ranges, int64_t n_tiles, void* stream);

/* ---------------------------------------------------------------- stage (d) */
/*
 * Scratch of the blend passes: packed per-tet records (128 B per tet), the
 * heavy-first tile order of the work queue (4 B per tile) and queue tickets.
 */
RM_API size_t rm_blend_workspace_size(int64_t n_tets, int64_t n_tiles);
/* Extra workspace bytes for RM_BLEND_HIT_MASKS over n_pairs list entries in
 * n_tiles tiles of tile_pixels pixels (4 bytes per 32 entries per pixel). */
RM_API size_t rm_blend_hit_mask_bytes(int64_t n_pairs, int64_t n_tiles, int tile_pixels);
/* Byte offset, inside a workspace of rm_blend_workspace_size(n_tets, n_tiles)
 * bytes, of the status word a blend pass uses when given no status_dev. */
RM_API size_t rm_blend_status_offset(int64_t n_tets, int64_t n_tiles);

#define RM_BLEND_REUSE_RECORDS 0x1  /* workspace already holds this frame's records */
/* Hit masks: with this flag on rm_blend_fwd and rm_blend_bwd (same lists, same
 * workspace, 64-pixel work items) the forward stores, per list entry and work
 * item, which pixels it counted as hits, and the backward revisits only those,
 * skipping the ray/tet tests of the misses.  The workspace must extend
 * rm_blend_hit_mask_bytes(P, G, tile pixels) beyond rm_blend_workspace_size;
 * entries past that room are tested as without masks.  A forward without the
 * flag (or with 16-pixel items) marks the masks invalid, and the backward then
 * tests every entry. */
#define RM_BLEND_HIT_MASKS 0x2
/* Records of each shared-memory batch staged by bulk copies (cp.async.bulk
 * from this GPU's memory into the issuing CTA, completing on an mbarrier), two
 * batches in flight, instead of per-thread loads.  Backward, 64-pixel items. */
#define RM_BLEND_STAGE_TMA 0x4

/* flags bits 8..15: log2 of the pixels per work item strip (16 or 64; 0 = 64) */
#define RM_BLEND_STRIP_SHIFT 8
#define RM_BLEND_STRIP(log2_pixels) ((log2_pixels) << RM_BLEND_STRIP_SHIFT)
/* flags bits 16..19: heavy-tile threshold, in powers of two above the mean
 * list length (0 = default, 1 = every tile is heavy); bits 20..23: resident
 * CTAs per SM of the kernel that takes the heavy tiles (0 = default) */
#define RM_BLEND_HEAVY_SHIFT 16
#define RM_BLEND_PAIR_CTAS_SHIFT 20
/* flags bits 24..27: log2 of the tets staged per shared-memory batch by the
 * pass's main kernel (forward: the pair kernel, backward: the dense kernel);
 * 4, 5 or 6 (0 = default 32) */
#define RM_BLEND_BATCH_SHIFT 24

/*
 * Front-to-back tile blend.  A persistent kernel takes strips of pixels from
 * a work queue ordered heaviest tile first.  Replaces splat_tiled
 * (delaunay_rasterization/internal/slang/alphablend_shader_interp.slang:371-431,
 * alpha_blend at :194-271) launched by AlphaBlendTiledRender.forward
 * (delaunay_rasterization/internal/alphablend_tiled_slang_interp.py:165-202).
 * tiles_touched may be NULL; when given, records are packed only for visible
 * tets.  Writes every pixel of out_img [H,W,4], out_distortion [H,W,5] and
 * n_contrib [H,W].  A staging wait that gives up sets RM_STATUS_QUEUE_TIMEOUT
 * in *status_dev (NULL: in the workspace word at rm_blend_status_offset,
 * cleared by the call).
 */
RM_API int rm_blend_fwd(const int32_t* sorted_ids, const int32_t* ranges,
                 const int32_t* indices, const float* vertices,
                 const float* cell_values, int64_t n_tets, int64_t n_verts,
                 const int32_t* tiles_touched, const float* ray_jitter,
                 const rm_camera* cam, float* out_img, float* out_distortion,
                 int32_t* n_contrib, void* workspace, size_t workspace_bytes,
                 int flags, uint32_t* status_dev, void* stream);

/*
 * Back-to-front adjoint of the blend.  Replaces splat_tiled.bwd
 * (delaunay_rasterization/internal/alphablend_tiled_slang_interp.py:220-262),
 * i.e. bwd_alpha_blend (delaunay_rasterization/internal/slang/alphablend_shader_interp.slang:273-369).
 * grad_vertices [V,3] and grad_cell_values [T,7] are accumulated into; the
 * caller zeroes them.  grad_distortion may be NULL (zeros).  status_dev as
 * rm_blend_fwd.
 */
RM_API int rm_blend_bwd(const int32_t* sorted_ids, const int32_t* ranges,
                 const int32_t* indices, const float* vertices,
                 const float* cell_values, int64_t n_tets, int64_t n_verts,
                 const int32_t* tiles_touched, const float* ray_jitter,
                 const rm_camera* cam, const float* out_img,
                 const float* out_distortion, const int32_t* n_contrib,
                 const float* grad_img, const float* grad_distortion,
                 float* grad_vertices, float* grad_cell_values, void* workspace,
                 size_t workspace_bytes, int flags, uint32_t* status_dev, void* stream);

/*
 * rm_project_fwd plus each tet's image footprint, footprint [T,12] float:
 *   [0:4]  the image-space bounding box (min x, min y, max x, max y in pixels,
 *          from the same clipped and projected points as rect);
 *   [4:12] the four projected vertices (x0 y0 x1 y1 x2 y2 x3 y3) when all four
 *          lie in front of a pinhole camera without distortion (z > 1e-4, so
 *          nothing is clipped) and within 8192 pixels of the image origin,
 *          NaN otherwise;
 * rows of culled tets are not written.  The lists of smaller tiles are cut
 * from the coarse lists with it (rm_fine_lists).  Index and vertex checks and
 * status_dev as rm_project_fwd.  No reference counterpart.
 */
RM_API int rm_project_fwd_fine(const int32_t* indices, const float* vertices, int64_t n_tets,
                               int64_t n_verts, const rm_camera* cam,
                               int32_t* tiles_touched, int32_t* rect, float* vs,
                               float* circumcenter, float* footprint, uint32_t* status_dev,
                               void* stream);

/*
 * Bounds of the per-pixel ray jitter [n_pixels, 2]: bounds [4] on the device
 * = (min jx, min jy, max jx, max jy), NaNs ignored.  Two small launches, no
 * host synchronisation.  Workspace: rm_jitter_bounds_workspace_size() bytes,
 * 16-byte aligned.  No reference counterpart.
 */
RM_API size_t rm_jitter_bounds_workspace_size(void);
RM_API int rm_jitter_bounds(const float* ray_jitter, int64_t n_pixels, float* bounds,
                            void* workspace, size_t workspace_bytes, void* stream);

/*
 * Fine lists from the sorted coarse lists: splits each coarse tile's list
 * (sorted_ids, ranges [G,2]; sorted_keys are rm_sort_pairs' sorted keys,
 * whose high word is each entry's tile; n_pairs entries, or
 * min(*n_pairs_dev, n_pairs) when n_pairs_dev is given) in order into the
 * lists of its 2^fine_shift x
 * 2^fine_shift fine tiles (tile_width >> fine_shift by tile_height >>
 * fine_shift pixels, on a grid 2^fine_shift times larger).  An entry goes to
 * a fine tile when its tet's footprint (rm_project_fwd_fine) can meet the
 * image points that the fine tile's pixel rays pass through with any jitter
 * inside jitter_bounds (rm_jitter_bounds of the ray_jitter that the blend
 * will use): the box grown by 1/64 pixel meets them, and, when the projected
 * vertices are given, no edge of their convex hull has all of them more than
 * 1/16 pixel outside.  For a camera whose cam_pos is not the centre of its
 * world_view (rays and projection then see the scene from different points)
 * the image points are widened by 2 x focal length x offset / min_t pixels,
 * and without bound when the two cannot be reconciled (a projective last
 * row, a matrix that is not a rotation, an offset with min_t <= 0).  So the
 * fine list of a fine tile holds, in the coarse
 * list's order, every entry of the coarse list that can reach one of its
 * rays, and blending over the fine lists yields the image, log T and
 * distortion of blending over the coarse lists with fewer ray/tet tests
 * (n_contrib then counts fine-list entries).  The result equals emitting,
 * sorting and ranging the fine pairs: fine_ids (capacity entries;
 * 4^fine_shift * P always suffices) and fine_ranges [G * 4^fine_shift, 2] on
 * the fine grid, *total_dev = fine pair count.  fine_shift is 1, 2 or 3.
 * Workspace: rm_fine_lists_workspace_size(fine tiles, n_pairs, fine_shift),
 * 256-byte aligned.  The split's own scan look-back and a fine list longer
 * than capacity set RM_STATUS_SCAN_TIMEOUT / RM_STATUS_CAPACITY in
 * *status_dev (status_dev may be NULL: the bits then stay in the workspace).
 * Fine ranges are cut to capacity.  The sorted ids index the footprint
 * rows, so they must come from a list build whose status word was read
 * clean (rm_fine_lists_multi, which knows the tet count, skips ids outside
 * it).  No reference counterpart.
 */
RM_API size_t rm_fine_lists_workspace_size(int64_t n_fine_tiles, int64_t n_pairs, int fine_shift);
RM_API int rm_fine_lists(const int64_t* sorted_keys, const int32_t* sorted_ids, int64_t n_pairs,
                         const int64_t* n_pairs_dev, const int32_t* ranges,
                         const float* footprint, const float* jitter_bounds,
                         const rm_camera* cam, int fine_shift,
                         int64_t capacity, int32_t* fine_ids, int32_t* fine_ranges,
                         int64_t* total_dev, void* workspace, size_t workspace_bytes,
                         uint32_t* status_dev, void* stream);

/* ------------------------------------------------------- batched views -- */
/*
 * Batched entry points render up to RM_MAX_VIEWS cameras of one mesh in one
 * launch per stage.  They have no reference counterpart: the reference
 * renders one camera per call (utils/train_util.py:15-77), and a batch of
 * views through these calls yields, view by view, exactly what the
 * single-camera calls yield.  Conventions:
 *   - all cameras share one tile size;
 *   - tiles get one global, view-major numbering: view v owns the tile ids
 *     [tile_base(v), tile_base(v) + grid_w(v) * grid_h(v)), tile_base(v) being
 *     the sum of the earlier views' grid sizes;
 *   - per-view [T] arrays of the projection are stacked view-major ([n_views, T]);
 *   - per-pixel buffers (ray_jitter, images, n_contrib and their gradients)
 *     are the views' buffers concatenated in view order.
 * Pair emission, sort and tile ranges then run once over all views with the
 * single-camera calls (rm_scan_tiles over n_views * T counts, rm_sort_pairs
 * with end_bit = 32 + bit length of the total tile count, rm_tile_ranges
 * over the total tile count).
 */
#define RM_MAX_VIEWS 32

/*
 * Projection of every tet into every view; each tet's vertices are read once
 * for all views.  Per view the outputs equal rm_project_fwd's where
 * tiles_touched > 0: tiles_touched and rect [n_views, T] (rect rows of 4),
 * depth [n_views, T] (rm_project_fwd's vs[:, 2]).  tiles_any [T] (optional) receives the tet's tile count summed
 * over the views; circumcenter [T, 3] (optional) is view-independent.
 * footprint [n_views, T, 12] (optional) receives rm_project_fwd_fine's
 * footprints.  Only tiles_touched is written for a (view, tet) without
 * tiles: its rect, depth and footprint rows are left as they were (the
 * batched stages never read them).  Index and vertex checks and status_dev
 * as rm_project_fwd.
 */
RM_API int rm_project_fwd_multi(const int32_t* indices, const float* vertices,
                                int64_t n_tets, int64_t n_verts,
                                const rm_camera* cams, int n_views,
                                int32_t* tiles_touched, int32_t* rect,
                                float* depth, int32_t* tiles_any,
                                float* circumcenter, float* footprint,
                                uint32_t* status_dev, void* stream);

/*
 * rm_fine_lists for a view batch: the coarse lists of all views (global
 * view-major tiles) split into the lists of the finer tiles, numbered
 * view-major on the finer grids (view v's fine tiles start at
 * tile_base(v) * 4^fine_shift), using footprint [n_views, T, 12] of
 * rm_project_fwd_multi and the bounds of the batch's concatenated ray jitter.
 * Blending a batch of the fine cameras (tiles 2^fine_shift times smaller,
 * grids that much larger) over these lists gives the coarse batch's images
 * bit for bit.  footprint (and jitter_bounds) may be NULL when fine_shift is 1 and
 * the sorted values carry the packed 2x2 coverage bits of
 * rm_emit_pairs_multi; fine_ids then hold the plain tet ids.  status_dev as
 * rm_fine_lists.
 */
RM_API int rm_fine_lists_multi(const int64_t* sorted_keys, const int32_t* sorted_ids, int64_t n_pairs,
                               const int64_t* n_pairs_dev, const int32_t* ranges,
                               const float* footprint, const float* jitter_bounds, int64_t n_tets,
                               const rm_camera* cams, int n_views, int fine_shift,
                               int64_t capacity, int32_t* fine_ids, int32_t* fine_ranges,
                               int64_t* total_dev, void* workspace, size_t workspace_bytes,
                               uint32_t* status_dev, void* stream);

/*
 * Pair emission for the stacked projection: offsets is the inclusive scan of
 * tiles_touched [n_views * T].  Pair (view v, tet g, tile (x, y)) gets the key
 * ((tile_base(v) + y * grid_w(v) + x) << 32) | sortable(depth[v, g]) and the
 * value g.  Capacity handling as rm_emit_pairs.  footprint_2x (optional,
 * [n_views, T, 12], rm_project_fwd_multi's footprints) with jitter_bounds
 * (rm_jitter_bounds of the batch's ray jitter): the value then also carries,
 * in bits 28..31, which of the tile's 2x2 half-size tiles the tet can reach
 * (the test of rm_fine_lists; bit qy * 2 + qx; T < 2^28; even tile sizes),
 * for rm_fine_lists_multi to split the sorted lists without reading the
 * footprints again.  Such values are not plain tet ids.
 */
RM_API int rm_emit_pairs_multi(const float* depth, const int32_t* rect,
                               const int32_t* offsets, int64_t n_tets,
                               const rm_camera* cams, int n_views,
                               int64_t capacity, const int64_t* total_dev,
                               int64_t* keys, int32_t* values,
                               uint32_t* status_dev, const float* footprint_2x,
                               const float* jitter_bounds, void* stream);

/* Total tile count of a batch (the ranges length and the blend workspace's
 * n_tiles), or -1 on bad input. */
RM_API int64_t rm_views_tile_count(const rm_camera* cams, int n_views);

/*
 * Per-tet records of the blend kept outside the workspace, so that several
 * batches on one mesh (possibly in flight on different streams) read one
 * copy: rm_blend_records_size(T) bytes, filled by rm_blend_pack_records
 * (tiles_touched may be NULL: every tet is packed; a tet with an index outside
 * [0, n_verts) gets an all-zero record, which no ray hits).  No reference
 * counterpart (the reference reloads each tet from its index and vertex
 * arrays for every pixel batch, alphablend_shader_interp.slang:221-232).
 */
RM_API size_t rm_blend_records_size(int64_t n_tets);
RM_API int rm_blend_pack_records(const int32_t* indices, const float* vertices,
                                 const float* cell_values, int64_t n_tets, int64_t n_verts,
                                 const int32_t* tiles_touched, void* records, void* stream);

/*
 * Blend of all views in one persistent launch fed by one work queue over the
 * global tiles.  Arguments as rm_blend_fwd with the batched conventions above;
 * tiles_touched, when given, is a [T] visibility count (tiles_any).  records
 * may be NULL (records are packed into the workspace, sized by
 * rm_blend_workspace_size(T, n_tiles)) or hold rm_blend_pack_records' output
 * (then the workspace needs only rm_blend_workspace_size(0, n_tiles) bytes).
 */
RM_API int rm_blend_fwd_multi(const int32_t* sorted_ids, const int32_t* ranges,
                              const int32_t* indices, const float* vertices,
                              const float* cell_values, int64_t n_tets, int64_t n_verts,
                              const int32_t* tiles_touched, const float* ray_jitter,
                              const rm_camera* cams, int n_views, float* out_img,
                              float* out_distortion, int32_t* n_contrib,
                              const void* records, void* workspace,
                              size_t workspace_bytes, int flags, uint32_t* status_dev,
                              void* stream);

/* Adjoint of rm_blend_fwd_multi; gradients of all views are summed into
 * grad_vertices and grad_cell_values. */
RM_API int rm_blend_bwd_multi(const int32_t* sorted_ids, const int32_t* ranges,
                              const int32_t* indices, const float* vertices,
                              const float* cell_values, int64_t n_tets, int64_t n_verts,
                              const int32_t* tiles_touched, const float* ray_jitter,
                              const rm_camera* cams, int n_views, const float* out_img,
                              const float* out_distortion, const int32_t* n_contrib,
                              const float* grad_img, const float* grad_distortion,
                              float* grad_vertices, float* grad_cell_values,
                              const void* records, void* workspace,
                              size_t workspace_bytes, int flags, uint32_t* status_dev,
                              void* stream);

/* ------------------------------------------- densification statistics -- */
/*
 * Per-tet statistics of one view for densification.  Replaces calc_tet_err
 * (delaunay_rasterization/internal/slang/alphablend_shader_interp.slang:433-599)
 * launched by render_err (delaunay_rasterization/internal/render_err.py:138-150).
 * Walks the tile lists front to back from each pixel centre; for every hit
 * adds to tet_err [T,16] (float, accumulated) in columns 0, 1, 2, 5: T, T*e,
 * T*e^2, T*s (T = exp(log T) * density * dt, e = pixel_err [H,W], s = ssim_err
 * [H,W]), 6-8 / 9-11 / 13-15: T times the entry point / exit point / segment
 * midpoint, 12: T; and to tet_count [T,2] (int32, accumulated) the hit count
 * and the maximum of int(65535 * T).  Columns 3 and 4 are left untouched, as
 * in the reference, whose walk also starts from log T = 1 and stops once
 * log T < -5.5.  Workspace and flags as rm_blend_fwd (records are packed
 * unless RM_BLEND_REUSE_RECORDS).
 */
RM_API int rm_calc_tet_err(const int32_t* sorted_ids, const int32_t* ranges,
                           const int32_t* indices, const float* vertices,
                           const float* cell_values, int64_t n_tets, int64_t n_verts,
                           const int32_t* tiles_touched, const rm_camera* cam,
                           const float* pixel_err, const float* ssim_err,
                           float* tet_err, int32_t* tet_count, void* workspace,
                           size_t workspace_bytes, int flags, void* stream);

/* ------------------------------------------------- per-tet feature producer -- */
/*
 * The cell values the blend consumes, from the model's raw per-tet outputs:
 * activate_output (utils/model_util.py:93-105) with offset_normalize (:82-91)
 * and eval_sh (utils/eval_sh_py.py:138-200), fused, one thread per tet.
 * In: indices [T,4], vertices [V,3], circumcenters [T,3], density [T,1],
 * rgb [T,3], grd [T,3], sh_rest [T, n_rest, 3] (SH rows 1.. of degree
 * sh_degree <= 4; n_rest >= (sh_degree + 1)^2 - 1), camera_center (3 floats,
 * host memory).  Out: features [T,7] = (density, softplus_10(colour at v0
 * evaluated through the SH), grd * min(rgb) / |v0 - circumcenter|).  A tet
 * with an index outside [0, n_verts) gets zero features and no gradients.
 */
RM_API int rm_activate_features(const int32_t* indices, const float* vertices, int64_t n_verts,
                                const float* circumcenters, const float* density,
                                const float* rgb, const float* grd, const float* sh_rest,
                                int n_rest, int sh_degree, const float* camera_center,
                                int64_t n_tets, float* features, void* stream);

/* Adjoint of rm_activate_features: writes grad_density [T], grad_rgb [T,3],
 * grad_grd [T,3], grad_sh_rest [T,n_rest,3] and grad_circumcenters [T,3];
 * accumulates grad_vertices [V,3] (the mean and |v0 - circumcenter| carry
 * gradient; the vertex offsets inside the colour are detached, as in the
 * reference). */
RM_API int rm_activate_features_bwd(const int32_t* indices, const float* vertices, int64_t n_verts,
                                    const float* circumcenters, const float* density,
                                    const float* rgb, const float* grd, const float* sh_rest,
                                    int n_rest, int sh_degree, const float* camera_center,
                                    int64_t n_tets, const float* grad_features,
                                    float* grad_density, float* grad_rgb, float* grad_grd,
                                    float* grad_sh_rest, float* grad_vertices,
                                    float* grad_circumcenters, void* stream);

/* ------------------------------------------------------ Delaunay update -- */
/*
 * The steps of a Delaunay update after the tetrahedralisation itself
 * (update_triangulation, models/ingp_color.py:523-558; the tetrahedralisation,
 * gDel3D or scipy's Delaunay, is not part of this library).  Each output keeps
 * the input order.  Workspace: rm_tets_workspace_size(n_tets) bytes, 256-byte
 * aligned.
 *
 * rm_tets_orient: the rows of indices_in [n_tets,4] whose indices all lie in
 * [0, n_verts) (rows naming gDel3D's point at infinity are dropped, :533), with
 * vertices 0 and 1 swapped where the signed volume det(v1 - v0, v2 - v0,
 * v3 - v0) / 6 is negative (:538-542; evaluated in double, so the sign can
 * differ from the reference's float32 determinant only for tets whose volume
 * is at float32 rounding level).  indices_out has room for n_tets rows;
 * *n_out_dev receives the kept count.
 *
 * rm_tets_cull: tets with density > density_threshold or alpha >
 * alpha_threshold, alpha = 1 - exp(-density * shortest edge length)
 * (:548-554, calc_tet_alpha(mode="min"), models/base_model.py:82-105), go to
 * kept_out, the others to empty_out (may be NULL); *n_kept_dev receives the
 * kept count.  A row with an index outside [0, n_verts) is counted as empty,
 * never dereferenced, and sets RM_STATUS_BAD_INDEX in *status_dev.
 */
RM_API size_t rm_tets_workspace_size(int64_t n_tets);
RM_API int rm_tets_orient(const int32_t* indices_in, int64_t n_tets, const float* vertices,
                          int64_t n_verts, int32_t* indices_out, int64_t* n_out_dev,
                          void* workspace, size_t workspace_bytes, uint32_t* status_dev,
                          void* stream);
RM_API int rm_tets_cull(const int32_t* indices, int64_t n_tets, const float* vertices,
                        int64_t n_verts, const float* density, float density_threshold,
                        float alpha_threshold, int32_t* kept_out, int32_t* empty_out,
                        int64_t* n_kept_dev, void* workspace, size_t workspace_bytes,
                        uint32_t* status_dev, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* RM_CAPI_H */
