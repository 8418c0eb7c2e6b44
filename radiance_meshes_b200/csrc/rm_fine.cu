// rm_fine.cu - tile lists on a finer grid, derived from the sorted lists.
//
// Given the sorted lists of the caller's tiles, each tet's image footprint
// (rm_project_fwd_fine: box and projected vertices) and the bounds of the
// per-pixel ray jitter (rm_jitter_bounds), the list of a fine tile
// (2^fine_shift times smaller) is the subsequence of its coarse tile's list of
// the tets that can reach one of its pixels' rays (footprint_bits).  Emitting
// fine pairs and sorting them again would reproduce exactly that order (depth
// key, then tet id), so instead each coarse list is split once, in order, into
// its 4 (or 16, 64) fine lists: a counting pass, a scan of the counts in
// fine-tile order, and a writing pass.  One CTA walks one coarse list in
// chunks of 1024 entries; the ranks inside a chunk come from warp ballots per
// fine tile.  No reference counterpart (the reference blends over the coarse
// lists directly).
#include <algorithm>

#include "rm_internal.cuh"

namespace rm {
namespace {

constexpr int kFineThreads = 1024;
constexpr int kFineWarps = kFineThreads / 32;

constexpr int kBoundsThreads = 256;
constexpr int kBoundsBlocks = 296;

// Jitter bounds, pass 1: per-CTA (min jx, min jy, max jx, max jy) over a
// grid-stride range of pixels; NaNs are ignored (a NaN ray reaches nothing).
__global__ void __launch_bounds__(kBoundsThreads) jitter_partial_kernel(const float2* __restrict__ jitter,
                                                                       int64_t n, float4* __restrict__ part) {
    float4 m = {INFINITY, INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = (int64_t)blockIdx.x * kBoundsThreads + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * kBoundsThreads) {
        const float2 j = __ldg(jitter + i);
        m = {fminf(m.x, j.x), fminf(m.y, j.y), fmaxf(m.z, j.x), fmaxf(m.w, j.y)};
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        m.x = fminf(m.x, __shfl_xor_sync(0xffffffffu, m.x, off));
        m.y = fminf(m.y, __shfl_xor_sync(0xffffffffu, m.y, off));
        m.z = fmaxf(m.z, __shfl_xor_sync(0xffffffffu, m.z, off));
        m.w = fmaxf(m.w, __shfl_xor_sync(0xffffffffu, m.w, off));
    }
    __shared__ float4 wm[kBoundsThreads / 32];
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kBoundsThreads / 32; ++w)
            m = {fminf(m.x, wm[w].x), fminf(m.y, wm[w].y), fmaxf(m.z, wm[w].z), fmaxf(m.w, wm[w].w)};
        part[blockIdx.x] = m;
    }
}

// Jitter bounds, pass 2: one warp folds the per-CTA partials.
__global__ void __launch_bounds__(32) jitter_final_kernel(const float4* __restrict__ part, int n_part,
                                                          float4* __restrict__ out) {
    float4 m = {INFINITY, INFINITY, -INFINITY, -INFINITY};
    for (int i = threadIdx.x; i < n_part; i += 32) {
        const float4 p = part[i];
        m = {fminf(m.x, p.x), fminf(m.y, p.y), fmaxf(m.z, p.z), fmaxf(m.w, p.w)};
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        m.x = fminf(m.x, __shfl_xor_sync(0xffffffffu, m.x, off));
        m.y = fminf(m.y, __shfl_xor_sync(0xffffffffu, m.y, off));
        m.z = fmaxf(m.z, __shfl_xor_sync(0xffffffffu, m.z, off));
        m.w = fmaxf(m.w, __shfl_xor_sync(0xffffffffu, m.w, off));
    }
    if (threadIdx.x == 0) *out = m;
}

// WRITE = false: counts[fine id] = entries of the coarse list reaching the
// fine tile.  WRITE = true: write the fine lists at their scanned offsets and
// the fine ranges.  FS = fine shift (2^FS x 2^FS fine tiles per tile).
// Views: tile t of the coarse (global, view-major) numbering belongs to view
// v = views.find(t); its fine tiles are numbered view-major too, view v's
// starting at tiles[v] * f^2; footprint rows are stacked view-major ([v, T]).
template <bool WRITE, bool PACKED, int FS>
__global__ void __launch_bounds__(kFineThreads, 2) fine_lists_kernel(
    const int32_t* __restrict__ ids, const int2* __restrict__ ranges, const float4* __restrict__ footprint,
    const float4* __restrict__ jitter_bounds, int64_t n_tets, const __grid_constant__ ViewSet views,
    int32_t* __restrict__ counts, const int32_t* __restrict__ incl, int32_t* __restrict__ fine_ids,
    int64_t capacity, int2* __restrict__ fine_ranges, uint32_t* status) {
    constexpr int f = 1 << FS, Q = f * f;
    __shared__ uint32_t wcnt[kFineWarps][Q];  // WRITE: this chunk's count per (warp, fine tile)
    __shared__ uint32_t wpre[kFineWarps][Q];  // WRITE: the warp's first position per fine tile
    __shared__ uint32_t run[Q];               // entries per fine tile so far
    __shared__ int32_t start[Q];
    const int t = blockIdx.x;
    const int v = views.find(t);
    const int local = t - views.tiles[v];
    const int grid_w = views.cams[v].grid_width;
    const int tx = local % grid_w, ty = local / grid_w;
    const int fgw = grid_w * f;
    const int64_t fbase = (int64_t)views.tiles[v] * Q;
    const float4* __restrict__ fp_v = footprint + (int64_t)v * n_tets * 3;
    const int ftw = views.cams[v].tile_width / f, fth = views.cams[v].tile_height / f;
    const int px0 = tx * views.cams[v].tile_width, py0 = ty * views.cams[v].tile_height;
    const float4 jb = PACKED ? make_float4(0.f, 0.f, 0.f, 0.f) : __ldg(jitter_bounds);
    const int2 r = __ldg(ranges + t);
    auto fine_id = [&](int q) { return fbase + (int64_t)(ty * f + q / f) * fgw + tx * f + q % f; };
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    if (threadIdx.x < Q) {
        run[threadIdx.x] = 0u;
        if (WRITE) start[threadIdx.x] = __ldg(incl + fine_id(threadIdx.x)) - __ldg(counts + fine_id(threadIdx.x));
    }
    __syncthreads();
    for (int base = r.x; base < r.y; base += kFineThreads) {
        const int e = base + (int)threadIdx.x;
        int32_t g = 0;
        uint64_t bits = 0;  // bit q: the entry reaches fine tile q
        if (e < r.y) {
            g = __ldg(ids + e);
            if (PACKED) {  // the 2x2 bits carried in the value's top bits
                bits = (uint32_t)g >> 28;
                g &= 0x0fffffff;
            } else {
                const Footprint fp = {__ldg(fp_v + 3 * (int64_t)g), __ldg(fp_v + 3 * (int64_t)g + 1),
                                      __ldg(fp_v + 3 * (int64_t)g + 2)};
                bits = footprint_bits<f>(fp, jb, px0, py0, ftw, fth);
            }
        }
        if constexpr (!WRITE) {
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const unsigned bal = __ballot_sync(0xffffffffu, (bits >> q) & 1u);
                if (lane == 0 && bal) atomicAdd(&run[q], (uint32_t)__popc(bal));
            }
        } else {
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const unsigned bal = __ballot_sync(0xffffffffu, (bits >> q) & 1u);
                if (lane == 0) wcnt[warp][q] = __popc(bal);
            }
            __syncthreads();
            if (warp == 0) {
                // per fine tile: exclusive prefix over the warps, offset by the
                // entries of the earlier chunks
                for (int q = 0; q < Q; ++q) {
                    const uint32_t x = wcnt[lane][q];
                    uint32_t inc = x;
#pragma unroll
                    for (int off = 1; off < 32; off <<= 1) {
                        const uint32_t y = __shfl_up_sync(0xffffffffu, inc, off);
                        if (lane >= off) inc += y;
                    }
                    const uint32_t r0 = run[q];
                    wpre[lane][q] = r0 + inc - x;
                    __syncwarp();
                    if (lane == 31) run[q] = r0 + inc;
                    __syncwarp();
                }
            }
            __syncthreads();
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const bool in = (bits >> q) & 1u;
                const unsigned bal = __ballot_sync(0xffffffffu, in);
                if (in) {
                    const int64_t o = (int64_t)start[q] + wpre[warp][q] + __popc(bal & lt);
                    if (o < capacity) fine_ids[o] = g;
                    else if (status) atomicOr(status, RM_STATUS_CAPACITY);
                }
            }
        }
    }
    __syncthreads();
    if (threadIdx.x < Q) {
        const int q = threadIdx.x;
        if (WRITE) fine_ranges[fine_id(q)] = make_int2(start[q], start[q] + (int)run[q]);
        else counts[fine_id(q)] = (int32_t)run[q];
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

size_t rm_jitter_bounds_workspace_size(void) { return sizeof(float4) * rm::kBoundsBlocks; }

int rm_jitter_bounds(const float* jitter, int64_t n_pixels, float* bounds, void* workspace, size_t workspace_bytes,
                     void* stream) {
    if (n_pixels < 0) return rm_host::fail(RM_EINVAL, "rm_jitter_bounds: negative size");
    if (!bounds || !workspace || (n_pixels > 0 && !jitter))
        return rm_host::fail(RM_EINVAL, "rm_jitter_bounds: NULL pointer");
    if (((uintptr_t)jitter & 7) || ((uintptr_t)bounds & 15) || ((uintptr_t)workspace & 15))
        return rm_host::fail(RM_EINVAL, "rm_jitter_bounds: misaligned jitter / bounds / workspace");
    if (workspace_bytes < rm_jitter_bounds_workspace_size())
        return rm_host::fail(RM_EINVAL, "rm_jitter_bounds: workspace %zu < %zu bytes", workspace_bytes,
                             rm_jitter_bounds_workspace_size());
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t want = (n_pixels + rm::kBoundsThreads - 1) / rm::kBoundsThreads;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(rm::kBoundsBlocks, want));
    float4* part = (float4*)workspace;
    rm::jitter_partial_kernel<<<blocks, rm::kBoundsThreads, 0, s>>>((const float2*)jitter, n_pixels, part);
    rm::jitter_final_kernel<<<1, 32, 0, s>>>(part, blocks, (float4*)bounds);
    return rm_host::check_launch("rm_jitter_bounds", 2);
}

}  // extern "C"

namespace {

int fine_lists_impl(const char* who, const int32_t* sorted_ids, const int32_t* ranges, const float* footprint,
                    const float* jitter_bounds, int64_t n_tets, const rm::ViewSet& views, int fine_shift,
                    int64_t capacity, int32_t* fine_ids, int32_t* fine_ranges, int64_t* total_dev, void* workspace,
                    size_t workspace_bytes, void* stream) {
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
    // no footprint: the 2x2 coverage bits come packed in bits 28..31 of the ids
    const bool packed = footprint == nullptr;
    if (packed && fine_shift != 1) return rm_host::fail(RM_EINVAL, "%s: packed masks need fine_shift 1", who);
    if (!packed && !jitter_bounds) return rm_host::fail(RM_EINVAL, "%s: footprint without jitter_bounds", who);
    if (!ranges || !fine_ranges || !total_dev || !workspace || (capacity > 0 && (!sorted_ids || !fine_ids)))
        return rm_host::fail(RM_EINVAL, "%s: NULL pointer", who);
    if (((uintptr_t)footprint & 15) || ((uintptr_t)jitter_bounds & 15) || ((uintptr_t)ranges & 7) ||
        ((uintptr_t)fine_ranges & 7) || ((uintptr_t)workspace & 255))
        return rm_host::fail(RM_EINVAL, "%s: misaligned footprint / jitter_bounds / ranges / workspace", who);
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
    using Kernel = void (*)(const int32_t*, const int2*, const float4*, const float4*, int64_t, const rm::ViewSet,
                            int32_t*, const int32_t*, int32_t*, int64_t, int2*, uint32_t*);
    Kernel count, write;
    if (packed) {
        count = rm::fine_lists_kernel<false, true, 1>;
        write = rm::fine_lists_kernel<true, true, 1>;
    } else if (fine_shift == 1) {
        count = rm::fine_lists_kernel<false, false, 1>;
        write = rm::fine_lists_kernel<true, false, 1>;
    } else if (fine_shift == 2) {
        count = rm::fine_lists_kernel<false, false, 2>;
        write = rm::fine_lists_kernel<true, false, 2>;
    } else {
        count = rm::fine_lists_kernel<false, false, 3>;
        write = rm::fine_lists_kernel<true, false, 3>;
    }
    count<<<(unsigned)G, rm::kFineThreads, 0, s>>>(sorted_ids, (const int2*)ranges, (const float4*)footprint,
                                                   (const float4*)jitter_bounds, n_tets, views, counts, nullptr,
                                                   nullptr, 0, nullptr, nullptr);
    int rc = rm_host::check_launch("rm_fine_lists (count)");
    if (rc) return rc;
    if ((rc = rm_scan_tiles(counts, Gf, incl, total_dev, scan_ws, rm_scan_workspace_size(Gf), stream))) return rc;
    write<<<(unsigned)G, rm::kFineThreads, 0, s>>>(sorted_ids, (const int2*)ranges, (const float4*)footprint,
                                                   (const float4*)jitter_bounds, n_tets, views, counts, incl,
                                                   fine_ids, capacity, (int2*)fine_ranges, status);
    return rm_host::check_launch("rm_fine_lists (write)");
}

}  // namespace

extern "C" {

int rm_fine_lists(const int32_t* sorted_ids, const int32_t* ranges, const float* footprint,
                  const float* jitter_bounds, const rm_camera* cam, int fine_shift, int64_t capacity,
                  int32_t* fine_ids, int32_t* fine_ranges, int64_t* total_dev, void* workspace,
                  size_t workspace_bytes, void* stream) {
    rm::ViewSet views;
    int rc = rm_host::make_views("rm_fine_lists", cam, 1, &views);
    if (rc) return rc;
    if (!footprint) return rm_host::fail(RM_EINVAL, "rm_fine_lists: NULL footprint");
    return fine_lists_impl("rm_fine_lists", sorted_ids, ranges, footprint, jitter_bounds, 0, views, fine_shift,
                           capacity, fine_ids, fine_ranges, total_dev, workspace, workspace_bytes, stream);
}

int rm_fine_lists_multi(const int32_t* sorted_ids, const int32_t* ranges, const float* footprint,
                        const float* jitter_bounds, int64_t n_tets, const rm_camera* cams, int n_views,
                        int fine_shift, int64_t capacity, int32_t* fine_ids, int32_t* fine_ranges,
                        int64_t* total_dev, void* workspace, size_t workspace_bytes, void* stream) {
    rm::ViewSet views;
    int rc = rm_host::make_views("rm_fine_lists_multi", cams, n_views, &views);
    if (rc) return rc;
    return fine_lists_impl("rm_fine_lists_multi", sorted_ids, ranges, footprint, jitter_bounds, n_tets, views, fine_shift,
                           capacity, fine_ids, fine_ranges, total_dev, workspace, workspace_bytes, stream);
}

}  // extern "C"
