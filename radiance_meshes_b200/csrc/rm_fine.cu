// rm_fine.cu - tile lists on a finer grid, derived from the sorted lists.
//
// Given the sorted lists of the caller's tiles, each tet's image footprint
// (rm_project_fwd_fine: box and projected vertices) and the bounds of the
// per-pixel ray jitter (rm_jitter_bounds), the list of a fine tile
// (2^fine_shift times smaller) is the subsequence of its coarse tile's list of
// the tets that can reach one of its pixels' rays (footprint_bits).  Emitting
// fine pairs and sorting them again would reproduce exactly that order (depth
// key, then tet id), so instead each coarse list is split once, in order, into
// its 4 (or 16, 64) fine lists: a flat pass over all entries that computes
// each entry's reach bits (the entry's tile is the high word of its sorted
// key) and counts them per fine tile, a scan of the counts in fine-tile
// order, and a writing pass in which one CTA walks one coarse list in chunks
// of 1024 entries, the ranks inside a chunk coming from warp ballots per fine
// tile.  No reference counterpart (the reference blends over the coarse lists
// directly).
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

// Storage of an entry's reach bits (one bit per fine tile of its tile).
template <int FS>
struct FineBits;
template <>
struct FineBits<1> {
    using type = uint8_t;
};
template <>
struct FineBits<2> {
    using type = uint16_t;
};
template <>
struct FineBits<3> {
    using type = uint64_t;
};

// Fine tile id of sub-tile q of coarse tile t: view v's fine tiles are
// numbered view-major from tiles[v] * f^2, row-major on its fine grid.
template <int FS>
__device__ __forceinline__ int64_t fine_tile_id(const ViewSet& views, int t, int q) {
    constexpr int f = 1 << FS;
    const int v = views.find(t);
    const int local = t - views.tiles[v];
    const int gw = views.cams[v].grid_width;
    const int tx = local % gw, ty = local / gw;
    return (int64_t)views.tiles[v] * (f * f) + (int64_t)(ty * f + q / f) * (gw * f) + tx * f + q % f;
}

// Pass 1, flat over the sorted coarse entries (their tile is the key's high
// word): each entry's reach bits -- footprint_bits against its tile's fine
// tiles, or the packed bits of the value -- stored for pass 3 (not when
// packed), and the entry counts per fine tile (warp-aggregated atomics over
// the lanes of one tile).  Footprint rows are stacked view-major ([v, T]).
template <bool PACKED, int FS>
__global__ void __launch_bounds__(256) fine_bits_kernel(
    const int64_t* __restrict__ keys, const int32_t* __restrict__ ids, int64_t cap, const int64_t* __restrict__ n_dev,
    const float4* __restrict__ footprint, const float4* __restrict__ jitter_bounds, int64_t n_tets,
    const __grid_constant__ ViewSet views, typename FineBits<FS>::type* __restrict__ bits_out,
    int32_t* __restrict__ counts) {
    constexpr int f = 1 << FS, Q = f * f;
    const int64_t n = n_dev ? min(*n_dev, cap) : cap;
    const float4 jb = PACKED ? make_float4(0.f, 0.f, 0.f, 0.f) : __ldg(jitter_bounds);
    const int lane = threadIdx.x & 31;
    for (int64_t base = (int64_t)blockIdx.x * 256; base < n; base += (int64_t)gridDim.x * 256) {
        const int64_t e = base + threadIdx.x;
        const bool in = e < n;
        int t = -1;
        uint64_t bits = 0;
        if (in) {
            t = (int)((uint64_t)__ldg((const unsigned long long*)keys + e) >> 32);
            int32_t g = __ldg(ids + e);
            // only lists left invalid by a sort that gave up hold a tile or
            // tet outside the frame: such an entry reaches no fine tile.  The
            // tet id is checked when the tet count is known (n_tets > 0:
            // stacked views); the single-view split runs on lists whose
            // frame status the caller has read.
            if (t < 0 || t >= views.tiles[views.n] || (!PACKED && (g < 0 || (n_tets > 0 && (int64_t)g >= n_tets))))
                t = -1;
            if (t < 0) {
                if (!PACKED) bits_out[e] = 0;  // the write pass reads it by the coarse ranges
            } else if (PACKED) {
                bits = (uint32_t)g >> 28;
            } else {
                const int v = views.find(t);
                const int local = t - views.tiles[v];
                const rm_camera& c = views.cams[v];
                const int tx = local % c.grid_width, ty = local / c.grid_width;
                const float4* fp_g = footprint + 3 * ((int64_t)v * n_tets + g);
                const Footprint fp = {__ldg(fp_g), __ldg(fp_g + 1), __ldg(fp_g + 2)};
                // the jitter range widened by the view's parallax allowance
                const float a = views.parallax[v];
                const float4 jbv = {jb.x - a, jb.y - a, jb.z + a, jb.w + a};
                bits = footprint_bits<f>(fp, jbv, tx * c.tile_width, ty * c.tile_height, c.tile_width / f,
                                         c.tile_height / f);
                bits_out[e] = (typename FineBits<FS>::type)bits;
            }
        }
        const unsigned peers = __match_any_sync(0xffffffffu, t);
        const bool leader = in && lane == __ffs(peers) - 1;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const unsigned bal = __ballot_sync(0xffffffffu, (bits >> q) & 1u) & peers;
            if (leader && bal) atomicAdd(counts + fine_tile_id<FS>(views, t, q), __popc(bal));
        }
    }
}

// Pass 3, one CTA per coarse tile: write the entries of its list into the
// lists of its fine tiles at their scanned offsets, in list order (ranks from
// warp ballots and a warp-0 scan of the per-warp counts per chunk of 1024
// entries), and the fine ranges.
template <bool PACKED, int FS>
__global__ void __launch_bounds__(kFineThreads, 2) fine_write_kernel(
    const int32_t* __restrict__ ids, const int2* __restrict__ ranges,
    const typename FineBits<FS>::type* __restrict__ bits_in, const __grid_constant__ ViewSet views,
    const int32_t* __restrict__ counts, const int32_t* __restrict__ incl, int32_t* __restrict__ fine_ids,
    int64_t capacity, int2* __restrict__ fine_ranges, uint32_t* status) {
    constexpr int Q = (1 << FS) * (1 << FS);
    __shared__ uint32_t wcnt[kFineWarps][Q];  // this chunk's count per (warp, fine tile)
    __shared__ uint32_t wpre[kFineWarps][Q];  // the warp's first position per fine tile
    __shared__ uint32_t run[Q];               // entries per fine tile so far
    __shared__ int32_t start[Q];
    const int t = blockIdx.x;
    const int2 r = __ldg(ranges + t);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    if (threadIdx.x < Q) {
        const int64_t fid = fine_tile_id<FS>(views, t, threadIdx.x);
        run[threadIdx.x] = 0u;
        start[threadIdx.x] = __ldg(incl + fid) - __ldg(counts + fid);
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
                bits = bits_in[e];
            }
        }
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const unsigned bal = __ballot_sync(0xffffffffu, (bits >> q) & 1u);
            if (lane == 0) wcnt[warp][q] = __popc(bal);
        }
        __syncthreads();
        // per fine tile (one warp each): exclusive prefix over the warps,
        // offset by the entries of the earlier chunks
        for (int q = warp; q < Q; q += kFineWarps) {
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
        __syncthreads();
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const bool hit = (bits >> q) & 1u;
            const unsigned bal = __ballot_sync(0xffffffffu, hit);
            if (hit) {
                const int64_t o = (int64_t)start[q] + wpre[warp][q] + __popc(bal & lt);
                if (o >= 0 && o < capacity) fine_ids[o] = g;  // o < 0 only after a scan that gave up
                else if (status) atomicOr(status, RM_STATUS_CAPACITY);
            }
        }
    }
    __syncthreads();
    if (threadIdx.x < Q) {
        const int q = threadIdx.x;
        // ranges past the capacity (RM_STATUS_CAPACITY) are cut to what was written
        const int64_t a = max((int64_t)0, min((int64_t)start[q], capacity));
        const int64_t b = max(a, min((int64_t)start[q] + run[q], capacity));
        fine_ranges[fine_tile_id<FS>(views, t, q)] = make_int2((int)a, (int)b);
    }
}

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

}  // namespace
}  // namespace rm

extern "C" {

size_t rm_fine_lists_workspace_size(int64_t n_fine_tiles, int64_t n_pairs, int fine_shift) {
    const int64_t n = n_fine_tiles > 0 ? n_fine_tiles : 1;
    const int64_t p = n_pairs > 0 ? n_pairs : 1;
    const size_t bits = fine_shift <= 1 ? 1 : (fine_shift == 2 ? 2 : 8);
    return 2 * rm::align256((size_t)n * 4) + 256 + rm::align256(rm_scan_workspace_size(n)) +
           rm::align256((size_t)p * bits);
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

template <bool PACKED, int FS>
int launch_split(const int64_t* keys, const int32_t* ids, int64_t n_pairs, const int64_t* n_pairs_dev,
                 const int32_t* ranges, const float* footprint, const float* jitter_bounds, int64_t n_tets,
                 const rm::ViewSet& views, int64_t G, int64_t Gf, int64_t capacity, int32_t* fine_ids,
                 int32_t* fine_ranges, int64_t* total_dev, char* ws, uint32_t* status_dev, cudaStream_t s) {
    using Bits = typename rm::FineBits<FS>::type;
    int32_t* counts = (int32_t*)ws;
    int32_t* incl = (int32_t*)(ws + rm::align256((size_t)Gf * 4));
    char* scan_ws = ws + 2 * rm::align256((size_t)Gf * 4) + 256;
    // the caller's status word, else the scan workspace's own
    uint32_t* status = status_dev ? status_dev : (uint32_t*)scan_ws;
    Bits* bits = (Bits*)(scan_ws + rm::align256(rm_scan_workspace_size(Gf)));
    if (cudaMemsetAsync(counts, 0, (size_t)Gf * 4, s) != cudaSuccess) return rm_host::check_launch("rm_fine_lists");
    if (n_pairs > 0) {
        const int64_t want = (n_pairs + 255) / 256;
        const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, 148 * 16));
        rm::fine_bits_kernel<PACKED, FS><<<blocks, 256, 0, s>>>(
            keys, ids, n_pairs, n_pairs_dev, (const float4*)footprint, (const float4*)jitter_bounds, n_tets, views,
            bits, counts);
        int rc = rm_host::check_launch("rm_fine_lists (bits)");
        if (rc) return rc;
    }
    int rc = rm_host::scan_tiles_status(counts, Gf, incl, total_dev, scan_ws, rm_scan_workspace_size(Gf), status, s);
    if (rc) return rc;
    rm::fine_write_kernel<PACKED, FS><<<(unsigned)G, rm::kFineThreads, 0, s>>>(
        ids, (const int2*)ranges, bits, views, counts, incl, fine_ids, capacity, (int2*)fine_ranges, status);
    return rm_host::check_launch("rm_fine_lists (write)");
}

int fine_lists_impl(const char* who, const int64_t* sorted_keys, const int32_t* sorted_ids, int64_t n_pairs,
                    const int64_t* n_pairs_dev, const int32_t* ranges, const float* footprint,
                    const float* jitter_bounds, int64_t n_tets, const rm::ViewSet& views, int fine_shift,
                    int64_t capacity, int32_t* fine_ids, int32_t* fine_ranges, int64_t* total_dev, void* workspace,
                    size_t workspace_bytes, uint32_t* status_dev, void* stream) {
    if (fine_shift < 1 || fine_shift > 3) return rm_host::fail(RM_EINVAL, "%s: fine_shift %d", who, fine_shift);
    if (capacity < 0 || n_tets < 0 || n_pairs < 0) return rm_host::fail(RM_EINVAL, "%s: negative size", who);
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
    if (!ranges || !fine_ranges || !total_dev || !workspace ||
        (n_pairs > 0 && (!sorted_keys || !sorted_ids)) || (capacity > 0 && !fine_ids))
        return rm_host::fail(RM_EINVAL, "%s: NULL pointer", who);
    if (((uintptr_t)footprint & 15) || ((uintptr_t)jitter_bounds & 15) || ((uintptr_t)ranges & 7) ||
        ((uintptr_t)sorted_keys & 7) || ((uintptr_t)fine_ranges & 7) || ((uintptr_t)workspace & 255))
        return rm_host::fail(RM_EINVAL, "%s: misaligned footprint / jitter_bounds / keys / ranges / workspace", who);
    const size_t need = rm_fine_lists_workspace_size(Gf, n_pairs, fine_shift);
    if (workspace_bytes < need)
        return rm_host::fail(RM_EINVAL, "%s: workspace %zu < %zu bytes", who, workspace_bytes, need);
    if (G == 0) return RM_OK;
    char* ws = (char*)workspace;
    cudaStream_t s = (cudaStream_t)stream;
    if (packed)
        return launch_split<true, 1>(sorted_keys, sorted_ids, n_pairs, n_pairs_dev, ranges, footprint, jitter_bounds,
                                     n_tets, views, G, Gf, capacity, fine_ids, fine_ranges, total_dev, ws, status_dev, s);
    if (fine_shift == 1)
        return launch_split<false, 1>(sorted_keys, sorted_ids, n_pairs, n_pairs_dev, ranges, footprint,
                                      jitter_bounds, n_tets, views, G, Gf, capacity, fine_ids, fine_ranges, total_dev,
                                      ws, status_dev, s);
    if (fine_shift == 2)
        return launch_split<false, 2>(sorted_keys, sorted_ids, n_pairs, n_pairs_dev, ranges, footprint,
                                      jitter_bounds, n_tets, views, G, Gf, capacity, fine_ids, fine_ranges, total_dev,
                                      ws, status_dev, s);
    return launch_split<false, 3>(sorted_keys, sorted_ids, n_pairs, n_pairs_dev, ranges, footprint, jitter_bounds,
                                  n_tets, views, G, Gf, capacity, fine_ids, fine_ranges, total_dev, ws, status_dev, s);
}

}  // namespace

extern "C" {

int rm_fine_lists(const int64_t* sorted_keys, const int32_t* sorted_ids, int64_t n_pairs,
                  const int64_t* n_pairs_dev, const int32_t* ranges, const float* footprint,
                  const float* jitter_bounds, const rm_camera* cam, int fine_shift, int64_t capacity,
                  int32_t* fine_ids, int32_t* fine_ranges, int64_t* total_dev, void* workspace,
                  size_t workspace_bytes, uint32_t* status_dev, void* stream) {
    rm::ViewSet views;
    int rc = rm_host::make_views("rm_fine_lists", cam, 1, &views);
    if (rc) return rc;
    if (!footprint) return rm_host::fail(RM_EINVAL, "rm_fine_lists: NULL footprint");
    return fine_lists_impl("rm_fine_lists", sorted_keys, sorted_ids, n_pairs, n_pairs_dev, ranges, footprint,
                           jitter_bounds, 0, views, fine_shift, capacity, fine_ids, fine_ranges, total_dev, workspace,
                           workspace_bytes, status_dev, stream);
}

int rm_fine_lists_multi(const int64_t* sorted_keys, const int32_t* sorted_ids, int64_t n_pairs,
                        const int64_t* n_pairs_dev, const int32_t* ranges, const float* footprint,
                        const float* jitter_bounds, int64_t n_tets, const rm_camera* cams, int n_views,
                        int fine_shift, int64_t capacity, int32_t* fine_ids, int32_t* fine_ranges,
                        int64_t* total_dev, void* workspace, size_t workspace_bytes, uint32_t* status_dev,
                        void* stream) {
    rm::ViewSet views;
    int rc = rm_host::make_views("rm_fine_lists_multi", cams, n_views, &views);
    if (rc) return rc;
    return fine_lists_impl("rm_fine_lists_multi", sorted_keys, sorted_ids, n_pairs, n_pairs_dev, ranges, footprint,
                           jitter_bounds, n_tets, views, fine_shift, capacity, fine_ids, fine_ranges, total_dev,
                           workspace, workspace_bytes, status_dev, stream);
}

}  // extern "C"
