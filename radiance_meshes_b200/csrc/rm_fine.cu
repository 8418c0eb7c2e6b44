// rm_fine.cu - tile lists on a finer grid, derived from the sorted lists.
//
// Given the sorted lists of the caller's tiles and each tet's rectangle on a
// grid 2^fine_shift times finer (rm_project_fwd_fine), the list of a fine tile
// is the subsequence of its coarse tile's list whose fine rectangle covers it.
// Emitting fine pairs and sorting them again would reproduce exactly that
// order (depth key, then tet id), so instead each coarse list is split once,
// in order, into its 4 (or 16, 64) fine lists: a counting pass, a scan of the
// counts in fine-tile order, and a writing pass.  One CTA walks one coarse
// list in chunks of 1024 entries; the ranks inside a chunk come from warp
// ballots per fine tile.  No reference counterpart (the reference blends over
// the coarse lists directly).
#include "rm_internal.cuh"

namespace rm {
namespace {

constexpr int kFineThreads = 1024;
constexpr int kFineWarps = kFineThreads / 32;
constexpr int kMaxQuads = 64;  // fine tiles per coarse tile (fine_shift <= 3)

__device__ __forceinline__ bool covers(int4 fr, int fx, int fy) {
    return fr.x <= fx && fx < fr.z && fr.y <= fy && fy < fr.w;
}

// WRITE = false: counts[fine id] = entries of the coarse list covering the
// fine tile.  WRITE = true: write the fine lists at their scanned offsets and
// the fine ranges.
// Views: tile t of the coarse (global, view-major) numbering belongs to view
// v = views.find(t); its fine tiles are numbered view-major too, view v's
// starting at tiles[v] * f^2; rect_fine rows are stacked view-major ([v, T]).
template <bool WRITE, bool PACKED>
__global__ void __launch_bounds__(kFineThreads) fine_lists_kernel(
    const int32_t* __restrict__ ids, const int2* __restrict__ ranges, const int4* __restrict__ rect_fine,
    int64_t n_tets, const __grid_constant__ ViewSet views, int f, int32_t* __restrict__ counts,
    const int32_t* __restrict__ incl, int32_t* __restrict__ fine_ids, int64_t capacity,
    int2* __restrict__ fine_ranges, uint32_t* status) {
    __shared__ uint32_t wtot[kFineWarps][kMaxQuads];
    __shared__ uint32_t run[kMaxQuads];
    __shared__ int32_t start[kMaxQuads];
    const int t = blockIdx.x;
    const int v = views.find(t);
    const int local = t - views.tiles[v];
    const int grid_w = views.cams[v].grid_width;
    const int tx = local % grid_w, ty = local / grid_w;
    const int Q = f * f;
    const int fgw = grid_w * f;
    const int64_t fbase = (int64_t)views.tiles[v] * Q;
    const int4* __restrict__ rf_v = rect_fine + (int64_t)v * n_tets;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    if (threadIdx.x < Q) {
        run[threadIdx.x] = 0u;
        if (WRITE) {
            const int q = threadIdx.x;
            const int64_t fid = fbase + (ty * f + q / f) * fgw + tx * f + q % f;
            start[q] = __ldg(incl + fid) - __ldg(counts + fid);
        }
    }
    __syncthreads();
    const int2 r = __ldg(ranges + t);
    for (int base = r.x; base < r.y; base += kFineThreads) {
        const int e = base + (int)threadIdx.x;
        int4 fr = {0, 0, 0, 0};
        int32_t g = 0;
        uint32_t packed = 0;  // PACKED: the 2x2 coverage bits carried in the value's top bits
        if (e < r.y) {
            g = __ldg(ids + e);
            if (PACKED) {
                packed = (uint32_t)g >> 28;
                g &= 0x0fffffff;
            } else {
                fr = __ldg(rf_v + g);
            }
        }
        for (int q = 0; q < Q; ++q) {
            const bool in = PACKED ? ((packed >> q) & 1u) != 0 : covers(fr, tx * f + q % f, ty * f + q / f);
            const unsigned bal = __ballot_sync(0xffffffffu, in);
            if (lane == 0) wtot[warp][q] = __popc(bal);
        }
        __syncthreads();
        if (WRITE) {
            for (int q = 0; q < Q; ++q) {
                const bool in = PACKED ? ((packed >> q) & 1u) != 0 : covers(fr, tx * f + q % f, ty * f + q / f);
                const unsigned bal = __ballot_sync(0xffffffffu, in);
                if (in) {
                    uint32_t pos = run[q] + __popc(bal & lt);
                    for (int w = 0; w < warp; ++w) pos += wtot[w][q];
                    const int64_t o = (int64_t)start[q] + pos;
                    if (o < capacity) fine_ids[o] = g;
                    else if (status) atomicOr(status, RM_STATUS_CAPACITY);
                }
            }
        }
        __syncthreads();
        if (threadIdx.x < Q) {
            uint32_t s = 0;
            for (int w = 0; w < kFineWarps; ++w) s += wtot[w][threadIdx.x];
            run[threadIdx.x] += s;
        }
        __syncthreads();
    }
    if (threadIdx.x < Q) {
        const int q = threadIdx.x;
        const int64_t fid = fbase + (ty * f + q / f) * fgw + tx * f + q % f;
        if (WRITE) fine_ranges[fid] = make_int2(start[q], start[q] + (int)run[q]);
        else counts[fid] = (int32_t)run[q];
    }
}

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

}  // namespace
}  // namespace rm

extern "C" {

size_t rm_fine_lists_workspace_size(int64_t n_fine_tiles) {
    const int64_t n = n_fine_tiles > 0 ? n_fine_tiles : 1;
    return 2 * rm::align256((size_t)n * 4) + 256 + rm_scan_workspace_size(n);
}

}  // extern "C"

namespace {

int fine_lists_impl(const char* who, const int32_t* sorted_ids, const int32_t* ranges, const int32_t* rect_fine,
                    int64_t n_tets, const rm::ViewSet& views, int fine_shift, int64_t capacity, int32_t* fine_ids,
                    int32_t* fine_ranges, int64_t* total_dev, void* workspace, size_t workspace_bytes, void* stream) {
    if (fine_shift < 1 || fine_shift > 3) return rm_host::fail(RM_EINVAL, "%s: fine_shift %d", who, fine_shift);
    if (capacity < 0 || n_tets < 0) return rm_host::fail(RM_EINVAL, "%s: negative size", who);
    const int f = 1 << fine_shift;
    for (int v = 0; v < views.n; ++v)
        if (views.cams[v].tile_width % f || views.cams[v].tile_height % f)
            return rm_host::fail(RM_EINVAL, "%s: tile %dx%d not divisible by %d", who, views.cams[v].tile_width,
                                 views.cams[v].tile_height, f);
    const int64_t G = views.tiles[views.n];
    const int64_t Gf = G * f * f;
    if (Gf >= (int64_t)INT32_MAX) return rm_host::fail(RM_EINVAL, "%s: too many tiles", who);
    // no rect_fine: the 2x2 coverage bits come packed in bits 28..31 of the ids
    const bool packed = rect_fine == nullptr;
    if (packed && fine_shift != 1) return rm_host::fail(RM_EINVAL, "%s: packed masks need fine_shift 1", who);
    if (!ranges || !fine_ranges || !total_dev || !workspace || (capacity > 0 && (!sorted_ids || !fine_ids)))
        return rm_host::fail(RM_EINVAL, "%s: NULL pointer", who);
    if (((uintptr_t)rect_fine & 15) || ((uintptr_t)ranges & 7) || ((uintptr_t)fine_ranges & 7) ||
        ((uintptr_t)workspace & 255))
        return rm_host::fail(RM_EINVAL, "%s: misaligned rect_fine / ranges / workspace", who);
    if (workspace_bytes < rm_fine_lists_workspace_size(Gf))
        return rm_host::fail(RM_EINVAL, "%s: workspace %zu < %zu bytes", who, workspace_bytes,
                             rm_fine_lists_workspace_size(Gf));
    if (G == 0) return RM_OK;
    char* p = (char*)workspace;
    int32_t* counts = (int32_t*)p;
    int32_t* incl = (int32_t*)(p + rm::align256((size_t)Gf * 4));
    char* scan_ws = p + 2 * rm::align256((size_t)Gf * 4) + 256;
    uint32_t* status = (uint32_t*)scan_ws;  // the scan workspace's status word
    cudaStream_t s = (cudaStream_t)stream;
    auto count = packed ? rm::fine_lists_kernel<false, true> : rm::fine_lists_kernel<false, false>;
    auto write = packed ? rm::fine_lists_kernel<true, true> : rm::fine_lists_kernel<true, false>;
    count<<<(unsigned)G, rm::kFineThreads, 0, s>>>(sorted_ids, (const int2*)ranges, (const int4*)rect_fine, n_tets,
                                                   views, f, counts, nullptr, nullptr, 0, nullptr, nullptr);
    int rc = rm_host::check_launch("rm_fine_lists (count)");
    if (rc) return rc;
    if ((rc = rm_scan_tiles(counts, Gf, incl, total_dev, scan_ws, rm_scan_workspace_size(Gf), stream))) return rc;
    write<<<(unsigned)G, rm::kFineThreads, 0, s>>>(sorted_ids, (const int2*)ranges, (const int4*)rect_fine, n_tets,
                                                   views, f, counts, incl, fine_ids, capacity, (int2*)fine_ranges,
                                                   status);
    return rm_host::check_launch("rm_fine_lists (write)");
}

}  // namespace

extern "C" {

int rm_fine_lists(const int32_t* sorted_ids, const int32_t* ranges, const int32_t* rect_fine, const rm_camera* cam,
                  int fine_shift, int64_t capacity, int32_t* fine_ids, int32_t* fine_ranges, int64_t* total_dev,
                  void* workspace, size_t workspace_bytes, void* stream) {
    rm::ViewSet views;
    int rc = rm_host::make_views("rm_fine_lists", cam, 1, &views);
    if (rc) return rc;
    return fine_lists_impl("rm_fine_lists", sorted_ids, ranges, rect_fine, 0, views, fine_shift, capacity, fine_ids,
                           fine_ranges, total_dev, workspace, workspace_bytes, stream);
}

int rm_fine_lists_multi(const int32_t* sorted_ids, const int32_t* ranges, const int32_t* rect_fine, int64_t n_tets,
                        const rm_camera* cams, int n_views, int fine_shift, int64_t capacity, int32_t* fine_ids,
                        int32_t* fine_ranges, int64_t* total_dev, void* workspace, size_t workspace_bytes,
                        void* stream) {
    rm::ViewSet views;
    int rc = rm_host::make_views("rm_fine_lists_multi", cams, n_views, &views);
    if (rc) return rc;
    return fine_lists_impl("rm_fine_lists_multi", sorted_ids, ranges, rect_fine, n_tets, views, fine_shift, capacity,
                           fine_ids, fine_ranges, total_dev, workspace, workspace_bytes, stream);
}

}  // extern "C"
