// rm_scan.cu - stage (b): prefix sum of per-tet tile counts, tile/tet pair
// emission, and per-tile ranges of the sorted pair list.
//
//   rm_scan_tiles   torch.cumsum(tiles_touched) (tile_shader_slang.py:36), done
//                   as a single-pass block scan with decoupled look-back
//   rm_emit_pairs   generate_keys (tile_shader.slang:138-186)
//   rm_tile_ranges  compute_tile_ranges (tile_shader.slang:188-214)
#include <algorithm>
#include <mutex>

#include "rm_internal.cuh"

namespace rm {
namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;  // 4096 tets per CTA
constexpr uint64_t kFlagAgg = 1ull << 32;
constexpr uint64_t kFlagInc = 2ull << 32;
constexpr uint64_t kFlagOvf = 4ull << 32;  // an inclusive prefix up to this tile exceeds INT32_MAX

struct ScanWs {
    uint32_t status;
    uint32_t counter;
    uint32_t pad[2];
    // followed by uint64_t state[n_tiles]
};

// Look-back states: the flags and the sum share one 64-bit word and nothing
// else is published through it, so relaxed GPU-scope accesses suffice.
__device__ __forceinline__ void st_relaxed(uint64_t* p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint64_t ld_relaxed(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Tile states: bits 0..31 the tile's aggregate or inclusive prefix (uint32),
// bit 32 aggregate ready, bit 33 inclusive prefix ready, bit 34 overflow.
// Sums are formed in int64; a prefix above INT32_MAX (the offsets are int32,
// as the reference's cumsum) sets RM_STATUS_OVERFLOW.  The look-back polls a
// predecessor at most spin_limit times, then sets RM_STATUS_SCAN_TIMEOUT and
// goes on (the offsets are then invalid; every store stays in bounds).
// What the scan sums: the input values; 1 for each positive value (counts of
// the visible tets); or the values gathered through an order, in[order[i]],
// for i below *n_dev (counts in depth order).
enum ScanMode { kScanValues = 0, kScanPositive = 1, kScanGather = 2 };

template <int MODE>
__device__ __forceinline__ int32_t scan_item(const int32_t* __restrict__ in, const int32_t* __restrict__ order,
                                             int64_t i, int64_t n_eff, int64_t n) {
    if (i >= n_eff) return 0;
    if (MODE == kScanGather) {
        // an order left invalid by a sort that gave up may hold any value
        const int32_t g = __ldg(order + i);
        return (g >= 0 && (int64_t)g < n) ? __ldg(in + g) : 0;
    }
    const int32_t v = __ldg(in + i);
    return MODE == kScanPositive ? (v > 0 ? 1 : 0) : v;
}

template <int MODE>
__global__ void __launch_bounds__(kScanThreads) scan_kernel(const int32_t* __restrict__ in, int64_t n,
                                                            int32_t* __restrict__ out, int64_t* total_dev,
                                                            ScanWs* ws, uint32_t* status, uint32_t spin_limit,
                                                            const int32_t* __restrict__ order,
                                                            const int64_t* __restrict__ n_dev) {
    __shared__ uint32_t s_tile;
    __shared__ int64_t s_warp[kScanThreads / 32];
    __shared__ int64_t s_prefix;
    uint64_t* state = reinterpret_cast<uint64_t*>(ws + 1);
    if (threadIdx.x == 0) s_tile = atomicAdd(&ws->counter, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const int64_t base = (int64_t)tile * kScanTile + (int64_t)threadIdx.x * kScanItems;
    int32_t v[kScanItems];
    const int64_t n_eff = n_dev ? min(*n_dev, n) : n;
    if (MODE != kScanGather && base + kScanItems <= n_eff && ((((uintptr_t)(in + base)) & 15) == 0)) {
        const int4* p = reinterpret_cast<const int4*>(in + base);
#pragma unroll
        for (int k = 0; k < kScanItems / 4; ++k) {
            const int4 q = __ldg(p + k);
            v[4 * k] = q.x;
            v[4 * k + 1] = q.y;
            v[4 * k + 2] = q.z;
            v[4 * k + 3] = q.w;
        }
        if (MODE == kScanPositive)
#pragma unroll
            for (int k = 0; k < kScanItems; ++k) v[k] = v[k] > 0 ? 1 : 0;
    } else {
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) v[k] = scan_item<MODE>(in, order, base + k, n_eff, n);
    }
    int64_t sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) sum += v[k];
    // block-wide exclusive scan of the per-thread sums
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int64_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int64_t w = lane < kScanThreads / 32 ? s_warp[lane] : 0;
        int64_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += y;
        }
        if (lane < kScanThreads / 32) s_warp[lane] = wi - w;  // exclusive warp offsets
        const int64_t block_total = __shfl_sync(0xffffffffu, wi, kScanThreads / 32 - 1);
        if (lane == 0) {
            int64_t prefix = 0;
            bool ovf = block_total > (int64_t)INT32_MAX || block_total < 0;
            if (tile != 0) {
                st_relaxed(&state[tile], kFlagAgg | (ovf ? kFlagOvf : 0ull) | (uint32_t)block_total);
                int64_t t = (int64_t)tile - 1;
                uint32_t budget = spin_limit;
                while (t >= 0) {
                    const uint64_t s = ld_relaxed(&state[t]);
                    const uint64_t flag = s & (3ull << 32);
                    if (flag == 0) {
                        if (!spin_budget(budget)) {
                            atomicOr(status, RM_STATUS_SCAN_TIMEOUT);
                            break;
                        }
                        continue;
                    }
                    prefix += (int64_t)(uint32_t)s;
                    ovf |= (s & kFlagOvf) != 0;
                    if (flag == kFlagInc) break;
                    --t;
                }
            }
            const int64_t tile_incl = prefix + block_total;
            ovf |= tile_incl > (int64_t)INT32_MAX;
            if (ovf) atomicOr(status, RM_STATUS_OVERFLOW);
            st_relaxed(&state[tile], kFlagInc | (ovf ? kFlagOvf : 0ull) | (uint32_t)tile_incl);
            s_prefix = prefix;
            const int64_t last = (int64_t)tile * kScanTile + kScanTile;
            if (last >= n) *total_dev = tile_incl;
        }
    }
    __syncthreads();
    // int32 offsets (wrapped when RM_STATUS_OVERFLOW is set)
    int32_t run = (int32_t)(s_prefix + s_warp[warp] + incl - sum);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        run += v[k];
        v[k] = run;
    }
    if (base + kScanItems <= n && ((((uintptr_t)(out + base)) & 15) == 0)) {
        int4* p = reinterpret_cast<int4*>(out + base);
#pragma unroll
        for (int k = 0; k < kScanItems / 4; ++k) p[k] = make_int4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
    } else {
#pragma unroll
        for (int k = 0; k < kScanItems; ++k)
            if (base + k < n) out[base + k] = v[k];
    }
}

__device__ __forceinline__ uint32_t sortable_key(float f) {  // tile_shader.slang:107-136
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b ^ 0x80000000u);
}

// Flat emission: each CTA writes kEmitPerCta consecutive pairs, each thread
// kEmitItems of them.  Pair p belongs to the first tet g whose inclusive
// offset exceeds p; its rank k = p - (exclusive offset of g) walks g's rect
// row-major, exactly the order of generate_keys' nested loops
// (tile_shader.slang:51-97), so keys and values are those of the per-tet
// loop.  The offsets of the tets the CTA's pairs span are staged in shared
// memory when they fit (the search then runs there), else searched in
// global memory.  Work per thread is even however large a tet's rect is.
constexpr int kEmitThreads = 256;
constexpr int kEmitItems = 4;
constexpr int kEmitPerCta = kEmitThreads * kEmitItems;
constexpr int kEmitStage = 2048;

// First index in [lo, hi) with a[index] > p (hi when none).
__device__ __forceinline__ int64_t upper_bound_i32(const int32_t* a, int64_t lo, int64_t hi, int64_t p) {
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if ((int64_t)a[mid] > p) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

__global__ void __launch_bounds__(kEmitThreads) emit_kernel(const float* __restrict__ vs, const int4* __restrict__ rect,
                                                            const int32_t* __restrict__ offsets, int64_t n_tets,
                                                            int32_t grid_w, int64_t capacity,
                                                            const int64_t* __restrict__ total_dev,
                                                            int64_t* __restrict__ keys, int32_t* __restrict__ vals,
                                                            uint32_t* status) {
    __shared__ int32_t soff[kEmitStage];
    __shared__ int64_t sg[2];
    const int64_t n_pairs = min((int64_t)__ldg(offsets + n_tets - 1), capacity);
    if (blockIdx.x == 0 && threadIdx.x == 0 && total_dev && status && *total_dev > capacity)
        atomicOr(status, RM_STATUS_CAPACITY);
    const int64_t p0 = (int64_t)blockIdx.x * kEmitPerCta;
    if (p0 >= n_pairs) return;
    const int64_t p1 = min(p0 + kEmitPerCta, n_pairs);  // exclusive
    if (threadIdx.x < 2) sg[threadIdx.x] = upper_bound_i32(offsets, 0, n_tets, threadIdx.x ? p1 - 1 : p0);
    __syncthreads();
    const int64_t g0 = sg[0], g1 = sg[1];
    const bool staged = g1 - g0 + 1 <= kEmitStage;
    if (staged)
        for (int64_t i = threadIdx.x; i <= g1 - g0; i += kEmitThreads) soff[i] = __ldg(offsets + g0 + i);
    __syncthreads();
#pragma unroll
    for (int it = 0; it < kEmitItems; ++it) {
        const int64_t p = p0 + it * kEmitThreads + threadIdx.x;  // consecutive threads, consecutive pairs
        if (p >= p1) break;
        int64_t g;
        if (staged) g = g0 + upper_bound_i32(soff, 0, g1 - g0 + 1, p);
        else g = upper_bound_i32(offsets, g0, g1 + 1, p);
        const int64_t excl = g == 0 ? 0 : (int64_t)__ldg(offsets + g - 1);
        const int32_t k = (int32_t)(p - excl);
        const int4 r = __ldg(rect + g);
        const int32_t w = max(r.z - r.x, 1);  // >= 1 for every tet with pairs
        const int32_t y = r.y + k / w, x = r.x + k % w;
        const uint64_t fk = sortable_key(__ldg(vs + 3 * g + 2));
        keys[p] = (int64_t)(((uint64_t)(uint32_t)(y * grid_w + x) << 32) | fk);
        vals[p] = (int32_t)g;
    }
}

// Emission for the stacked projection of a view batch, flat like emit_kernel:
// the items are the (view, tet) pairs in view-major order (item i = view
// i / T, tet i % T), and tiles are numbered globally (tile_base + local id).
__global__ void __launch_bounds__(kEmitThreads) emit_multi_kernel(
    const float* __restrict__ depth, const int4* __restrict__ rect, const int32_t* __restrict__ offsets,
    int64_t n_tets, const __grid_constant__ ViewSet views, int64_t capacity, const int64_t* __restrict__ total_dev,
    int64_t* __restrict__ keys, int32_t* __restrict__ vals, uint32_t* status, const float4* __restrict__ footprint,
    const float4* __restrict__ jitter_bounds) {
    __shared__ int32_t soff[kEmitStage];
    __shared__ int64_t sg[2];
    const int64_t n_items = n_tets * views.n;
    const int64_t n_pairs = min((int64_t)__ldg(offsets + n_items - 1), capacity);
    if (blockIdx.x == 0 && threadIdx.x == 0 && total_dev && status && *total_dev > capacity)
        atomicOr(status, RM_STATUS_CAPACITY);
    const int64_t p0 = (int64_t)blockIdx.x * kEmitPerCta;
    if (p0 >= n_pairs) return;
    const int64_t p1 = min(p0 + kEmitPerCta, n_pairs);  // exclusive
    if (threadIdx.x < 2) sg[threadIdx.x] = upper_bound_i32(offsets, 0, n_items, threadIdx.x ? p1 - 1 : p0);
    __syncthreads();
    const int64_t i0 = sg[0], i1 = sg[1];
    const bool staged = i1 - i0 + 1 <= kEmitStage;
    if (staged)
        for (int64_t k = threadIdx.x; k <= i1 - i0; k += kEmitThreads) soff[k] = __ldg(offsets + i0 + k);
    __syncthreads();
    const float4 jb = footprint ? __ldg(jitter_bounds) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll 1
    for (int it = 0; it < kEmitItems; ++it) {
        const int64_t p = p0 + it * kEmitThreads + threadIdx.x;
        if (p >= p1) break;
        int64_t i;
        if (staged) i = i0 + upper_bound_i32(soff, 0, i1 - i0 + 1, p);
        else i = upper_bound_i32(offsets, i0, i1 + 1, p);
        const int64_t excl = i == 0 ? 0 : (int64_t)__ldg(offsets + i - 1);
        const int32_t k = (int32_t)(p - excl);
        const int v = (int)(i / n_tets);
        const int64_t g = i - (int64_t)v * n_tets;
        const rm_camera& c = views.cams[v];
        const int4 r = __ldg(rect + i);
        const int32_t w = max(r.z - r.x, 1);
        const int32_t y = r.y + k / w, x = r.x + k % w;
        const uint64_t fk = sortable_key(__ldg(depth + i));
        // with footprint: bits 28..31 of the value say which of the tile's 2x2
        // half-size tiles the tet can reach (bit qy * 2 + qx, footprint_bits)
        uint32_t q = 0;
        if (footprint) {
            const Footprint fp = {__ldg(footprint + 3 * i), __ldg(footprint + 3 * i + 1),
                                  __ldg(footprint + 3 * i + 2)};
            const float a = views.parallax[v];  // the view's parallax allowance
            const float4 jbv = {jb.x - a, jb.y - a, jb.z + a, jb.w + a};
            q = (uint32_t)footprint_bits<2>(fp, jbv, x * c.tile_width, y * c.tile_height, c.tile_width >> 1,
                                            c.tile_height >> 1);
        }
        keys[p] = (int64_t)(((uint64_t)((uint32_t)views.tiles[v] + (uint32_t)(y * c.grid_width + x)) << 32) | fk);
        vals[p] = (int32_t)((uint32_t)g | (q << 28));
    }
}

// Depth-first list build (rm_depth_order, rm_emit_pairs_ordered): the visible
// tets are compacted in tet order with their sortable depth keys, sorted by
// depth once (stable, so equal depths stay in tet order), and the pairs are
// emitted in that order; a stable sort on the tile bits alone then yields
// the reference's (tile, depth, emission order) sequence.
__global__ void __launch_bounds__(256) depth_scatter_kernel(const int32_t* __restrict__ tiles,
                                                            const float* __restrict__ vs, int64_t n_tets,
                                                            const int32_t* __restrict__ incl,
                                                            int64_t* __restrict__ keys, int32_t* __restrict__ vals) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_tets || __ldg(tiles + g) <= 0) return;
    const int64_t pos = (int64_t)__ldg(incl + g) - 1;
    if (pos < 0 || pos >= n_tets) return;  // only a count scan that gave up leaves such positions
    keys[pos] = (int64_t)sortable_key(__ldg(vs + 3 * g + 2));
    vals[pos] = (int32_t)g;
}

// emit_kernel over the tets in the given order (order[0 .. *n_items_dev)),
// with offsets the inclusive scan of their tile counts in that order.
__global__ void __launch_bounds__(kEmitThreads) emit_ordered_kernel(
    const float* __restrict__ vs, const int4* __restrict__ rect, const int32_t* __restrict__ order,
    const int32_t* __restrict__ offsets, const int64_t* __restrict__ n_items_dev, int64_t n_cap, int32_t grid_w,
    int64_t capacity, const int64_t* __restrict__ total_dev, int64_t* __restrict__ keys, int32_t* __restrict__ vals,
    uint32_t* status) {
    __shared__ int32_t soff[kEmitStage];
    __shared__ int64_t sg[2];
    const int64_t n_items = min(*n_items_dev, n_cap);
    if (n_items <= 0) return;
    const int64_t n_pairs = min((int64_t)__ldg(offsets + n_items - 1), capacity);
    if (blockIdx.x == 0 && threadIdx.x == 0 && total_dev && status && *total_dev > capacity)
        atomicOr(status, RM_STATUS_CAPACITY);
    const int64_t p0 = (int64_t)blockIdx.x * kEmitPerCta;
    if (p0 >= n_pairs) return;
    const int64_t p1 = min(p0 + kEmitPerCta, n_pairs);
    if (threadIdx.x < 2) sg[threadIdx.x] = upper_bound_i32(offsets, 0, n_items, threadIdx.x ? p1 - 1 : p0);
    __syncthreads();
    const int64_t s0 = sg[0], s1 = sg[1];
    const bool staged = s1 - s0 + 1 <= kEmitStage;
    if (staged)
        for (int64_t i = threadIdx.x; i <= s1 - s0; i += kEmitThreads) soff[i] = __ldg(offsets + s0 + i);
    __syncthreads();
#pragma unroll
    for (int it = 0; it < kEmitItems; ++it) {
        const int64_t p = p0 + it * kEmitThreads + threadIdx.x;
        if (p >= p1) break;
        int64_t si;
        if (staged) si = s0 + upper_bound_i32(soff, 0, s1 - s0 + 1, p);
        else si = upper_bound_i32(offsets, s0, s1 + 1, p);
        const int64_t excl = si == 0 ? 0 : (int64_t)__ldg(offsets + si - 1);
        const int32_t k = (int32_t)(p - excl);
        const int64_t g = __ldg(order + si);
        if (g < 0 || g >= n_cap) {  // an order left invalid by a sort that gave up: a key past every tile
            keys[p] = -1;
            vals[p] = 0;
            continue;
        }
        const int4 r = __ldg(rect + g);
        const int32_t w = max(r.z - r.x, 1);  // >= 1 for every tet with pairs
        const int32_t y = r.y + k / w, x = r.x + k % w;
        const uint64_t fk = sortable_key(__ldg(vs + 3 * g + 2));
        keys[p] = (int64_t)(((uint64_t)(uint32_t)(y * grid_w + x) << 32) | fk);
        vals[p] = (int32_t)g;
    }
}

__global__ void __launch_bounds__(256) ranges_kernel(const int64_t* __restrict__ keys, int64_t cap,
                                                     const int64_t* __restrict__ n_dev,
                                                     int32_t* __restrict__ ranges, int64_t n_tiles) {
    const int64_t n = n_dev ? min(*n_dev, cap) : cap;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t cur = (uint32_t)((uint64_t)keys[i] >> 32);
    if (cur >= n_tiles) return;
    if (i == 0) {
        ranges[2 * (int64_t)cur] = 0;
    } else {
        const uint32_t prev = (uint32_t)((uint64_t)keys[i - 1] >> 32);
        if (cur != prev) {
            if (prev < n_tiles) ranges[2 * (int64_t)prev + 1] = (int32_t)i;
            ranges[2 * (int64_t)cur] = (int32_t)i;
        }
    }
    if (i == n - 1) ranges[2 * (int64_t)cur + 1] = (int32_t)n;
}

// rm_count_pairs: grid-stride sums of the positive tile counts, one 64-bit
// atomic per block into out[0] (zeroed by the host call before the launch);
// block 0 also copies the status word into out[1].
constexpr int kCountThreads = 256;

__global__ void __launch_bounds__(kCountThreads) count_pairs_kernel(const int32_t* __restrict__ tiles, int64_t n,
                                                                    const uint32_t* __restrict__ status,
                                                                    int64_t* __restrict__ out) {
    __shared__ int64_t part[kCountThreads / 32];
    int64_t sum = 0;
    const int64_t stride = (int64_t)gridDim.x * kCountThreads;
    for (int64_t i = (int64_t)blockIdx.x * kCountThreads + threadIdx.x; i < n; i += stride)
        sum += max(__ldg(tiles + i), 0);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t b = 0;
#pragma unroll
        for (int w = 0; w < kCountThreads / 32; ++w) b += part[w];
        if (b) atomicAdd((unsigned long long*)out, (unsigned long long)b);
        if (blockIdx.x == 0) out[1] = status ? (int64_t)*status : 0;
    }
}

}  // namespace
}  // namespace rm

extern "C" {

size_t rm_scan_workspace_size(int64_t n_tets) {
    const int64_t tiles = (n_tets + rm::kScanTile - 1) / rm::kScanTile;
    return sizeof(rm::ScanWs) + sizeof(uint64_t) * (size_t)(tiles > 0 ? tiles : 1);
}

int rm_scan_tiles(const int32_t* tiles_touched, int64_t n_tets, int32_t* offsets, int64_t* total_dev,
                  void* workspace, size_t workspace_bytes, void* stream) {
    return rm_host::scan_tiles_status(tiles_touched, n_tets, offsets, total_dev, workspace, workspace_bytes, nullptr,
                                      stream);
}

}  // extern "C"

int rm_host::scan_tiles_status(const int32_t* tiles_touched, int64_t n_tets, int32_t* offsets, int64_t* total_dev,
                               void* workspace, size_t workspace_bytes, uint32_t* status, void* stream) {
    if (n_tets < 0) return rm_host::fail(RM_EINVAL, "rm_scan_tiles: negative size");
    if (!total_dev) return rm_host::fail(RM_EINVAL, "rm_scan_tiles: total_dev is NULL");
    cudaStream_t s = (cudaStream_t)stream;
    if (n_tets == 0) {
        cudaError_t e = cudaMemsetAsync(total_dev, 0, sizeof(int64_t), s);
        return e == cudaSuccess ? RM_OK : rm_host::fail(RM_ECUDA, "rm_scan_tiles: %s", cudaGetErrorString(e));
    }
    if (!tiles_touched || !offsets || !workspace) return rm_host::fail(RM_EINVAL, "rm_scan_tiles: NULL pointer");
    if (n_tets >= (int64_t)INT32_MAX) return rm_host::fail(RM_EINVAL, "rm_scan_tiles: too many tets");
    const size_t need = rm_scan_workspace_size(n_tets);
    if (workspace_bytes < need)
        return rm_host::fail(RM_EINVAL, "rm_scan_tiles: workspace %zu < %zu bytes", workspace_bytes, need);
    if ((uintptr_t)workspace & 15) return rm_host::fail(RM_EINVAL, "rm_scan_tiles: workspace must be 16-byte aligned");
    // status is preserved (it accumulates until rm_read_status); counter and tile states are reset
    cudaError_t e = cudaMemsetAsync((char*)workspace + 4, 0, need - 4, s);
    if (e != cudaSuccess) return rm_host::fail(RM_ECUDA, "rm_scan_tiles: %s", cudaGetErrorString(e));
    const int64_t blocks = (n_tets + rm::kScanTile - 1) / rm::kScanTile;
    rm::ScanWs* ws = (rm::ScanWs*)workspace;
    rm::scan_kernel<rm::kScanValues><<<(unsigned)blocks, rm::kScanThreads, 0, s>>>(
        tiles_touched, n_tets, offsets, total_dev, ws, status ? status : &ws->status, rm_host::wait_limit(), nullptr,
        nullptr);
    return rm_host::check_launch("rm_scan_tiles");
}

// The scans of the depth-first list build: counts of positive values, or
// values gathered through an order for the first *n_dev items.  Same
// workspace and checks as rm_scan_tiles.
int rm_host::scan_mode(int mode, const int32_t* in, const int32_t* order, int64_t n, const int64_t* n_dev,
                       int32_t* out, int64_t* total_dev, void* workspace, size_t workspace_bytes, uint32_t* status,
                       void* stream) {
    if (n < 0) return rm_host::fail(RM_EINVAL, "scan: negative size");
    cudaStream_t s = (cudaStream_t)stream;
    if (n == 0) {
        cudaError_t e = cudaMemsetAsync(total_dev, 0, sizeof(int64_t), s);
        return e == cudaSuccess ? RM_OK : rm_host::fail(RM_ECUDA, "scan: %s", cudaGetErrorString(e));
    }
    if (n >= (int64_t)INT32_MAX) return rm_host::fail(RM_EINVAL, "scan: too many items");
    const size_t need = rm_scan_workspace_size(n);
    if (workspace_bytes < need) return rm_host::fail(RM_EINVAL, "scan: workspace %zu < %zu bytes", workspace_bytes, need);
    cudaError_t e = cudaMemsetAsync((char*)workspace + 4, 0, need - 4, s);
    if (e != cudaSuccess) return rm_host::fail(RM_ECUDA, "scan: %s", cudaGetErrorString(e));
    const int64_t blocks = (n + rm::kScanTile - 1) / rm::kScanTile;
    rm::ScanWs* ws = (rm::ScanWs*)workspace;
    uint32_t* st = status ? status : &ws->status;
    if (mode == rm::kScanPositive)
        rm::scan_kernel<rm::kScanPositive><<<(unsigned)blocks, rm::kScanThreads, 0, s>>>(
            in, n, out, total_dev, ws, st, rm_host::wait_limit(), nullptr, n_dev);
    else
        rm::scan_kernel<rm::kScanGather><<<(unsigned)blocks, rm::kScanThreads, 0, s>>>(
            in, n, out, total_dev, ws, st, rm_host::wait_limit(), order, n_dev);
    return rm_host::check_launch("scan");
}

extern "C" {

int rm_emit_pairs(const float* vs, const int32_t* rect, const int32_t* offsets, int64_t n_tets, int32_t grid_width,
                  int64_t capacity, const int64_t* total_dev, int64_t* keys, int32_t* values, uint32_t* status_dev,
                  void* stream) {
    if (n_tets < 0 || capacity < 0) return rm_host::fail(RM_EINVAL, "rm_emit_pairs: negative size");
    if (n_tets == 0) return RM_OK;
    if (!vs || !rect || !offsets || (capacity > 0 && (!keys || !values)))
        return rm_host::fail(RM_EINVAL, "rm_emit_pairs: NULL pointer");
    if ((uintptr_t)rect & 15) return rm_host::fail(RM_EINVAL, "rm_emit_pairs: rect must be 16-byte aligned");
    if (capacity == 0) {
        // nothing to write; still flag an overflow of a zero capacity
        if (status_dev && total_dev)
            rm::emit_kernel<<<1, rm::kEmitThreads, 0, (cudaStream_t)stream>>>(
                vs, (const int4*)rect, offsets, n_tets, grid_width, capacity, total_dev, keys, values, status_dev);
        return rm_host::check_launch("rm_emit_pairs");
    }
    const int64_t blocks = (capacity + rm::kEmitPerCta - 1) / rm::kEmitPerCta;
    if (blocks > 0x7fffffff) return rm_host::fail(RM_EINVAL, "rm_emit_pairs: capacity too large");
    rm::emit_kernel<<<(unsigned)blocks, rm::kEmitThreads, 0, (cudaStream_t)stream>>>(
        vs, (const int4*)rect, offsets, n_tets, grid_width, capacity, total_dev, keys, values, status_dev);
    return rm_host::check_launch("rm_emit_pairs");
}

int rm_emit_pairs_multi(const float* depth, const int32_t* rect, const int32_t* offsets, int64_t n_tets,
                        const rm_camera* cams, int n_views, int64_t capacity, const int64_t* total_dev,
                        int64_t* keys, int32_t* values, uint32_t* status_dev, const float* footprint_2x,
                        const float* jitter_bounds, void* stream) {
    rm::ViewSet views;
    int rc = rm_host::make_views("rm_emit_pairs_multi", cams, n_views, &views);
    if (rc) return rc;
    if (n_tets < 0 || capacity < 0) return rm_host::fail(RM_EINVAL, "rm_emit_pairs_multi: negative size");
    if (n_tets == 0) return RM_OK;
    if (!depth || !rect || !offsets || (capacity > 0 && (!keys || !values)))
        return rm_host::fail(RM_EINVAL, "rm_emit_pairs_multi: NULL pointer");
    if (((uintptr_t)rect & 15) || ((uintptr_t)footprint_2x & 15) || ((uintptr_t)jitter_bounds & 15))
        return rm_host::fail(RM_EINVAL, "rm_emit_pairs_multi: rect, footprint, jitter_bounds not 16-byte aligned");
    if (footprint_2x && !jitter_bounds)
        return rm_host::fail(RM_EINVAL, "rm_emit_pairs_multi: footprint without jitter_bounds");
    if (footprint_2x && n_tets >= (1ll << 28))
        return rm_host::fail(RM_EINVAL, "rm_emit_pairs_multi: packed fine masks need fewer than 2^28 tets");
    if (footprint_2x)
        for (int v = 0; v < n_views; ++v)
            if ((cams[v].tile_width & 1) || (cams[v].tile_height & 1))
                return rm_host::fail(RM_EINVAL, "rm_emit_pairs_multi: packed fine masks need even tile sizes");
    const int64_t blocks = std::max<int64_t>(1, (capacity + rm::kEmitPerCta - 1) / rm::kEmitPerCta);
    if (blocks > 0x7fffffff) return rm_host::fail(RM_EINVAL, "rm_emit_pairs_multi: capacity too large");
    rm::emit_multi_kernel<<<(unsigned)blocks, rm::kEmitThreads, 0, (cudaStream_t)stream>>>(
        depth, (const int4*)rect, offsets, n_tets, views, capacity, total_dev, keys, values, status_dev,
        (const float4*)footprint_2x, (const float4*)jitter_bounds);
    return rm_host::check_launch("rm_emit_pairs_multi");
}

size_t rm_depth_order_workspace_size(int64_t n_tets) {
    const size_t a = ((sizeof(int32_t) * (size_t)(n_tets > 0 ? n_tets : 1)) + 255) / 256 * 256;
    return a + rm_scan_workspace_size(n_tets > 0 ? n_tets : 0);
}

int rm_depth_order(const int32_t* tiles_touched, const float* vs, int64_t n_tets, int64_t* keys, int32_t* values,
                   int64_t* n_visible_dev, void* workspace, size_t workspace_bytes, uint32_t* status_dev,
                   void* stream) {
    if (n_tets < 0) return rm_host::fail(RM_EINVAL, "rm_depth_order: negative size");
    if (!n_visible_dev) return rm_host::fail(RM_EINVAL, "rm_depth_order: NULL count");
    cudaStream_t s = (cudaStream_t)stream;
    if (n_tets == 0) {
        cudaError_t e = cudaMemsetAsync(n_visible_dev, 0, sizeof(int64_t), s);
        return e == cudaSuccess ? RM_OK : rm_host::fail(RM_ECUDA, "rm_depth_order: %s", cudaGetErrorString(e));
    }
    if (!tiles_touched || !vs || !keys || !values || !workspace)
        return rm_host::fail(RM_EINVAL, "rm_depth_order: NULL pointer");
    if (workspace_bytes < rm_depth_order_workspace_size(n_tets) || ((uintptr_t)workspace & 255))
        return rm_host::fail(RM_EINVAL, "rm_depth_order: workspace of %zu bytes, 256-byte aligned, needed",
                             rm_depth_order_workspace_size(n_tets));
    int32_t* incl = (int32_t*)workspace;
    char* scan_ws = (char*)workspace + (rm_depth_order_workspace_size(n_tets) - rm_scan_workspace_size(n_tets));
    int rc = rm_host::scan_mode(rm::kScanPositive, tiles_touched, nullptr, n_tets, nullptr, incl, n_visible_dev,
                                scan_ws, rm_scan_workspace_size(n_tets), status_dev, s);
    if (rc) return rc;
    const unsigned blocks = (unsigned)((n_tets + 255) / 256);
    rm::depth_scatter_kernel<<<blocks, 256, 0, s>>>(tiles_touched, vs, n_tets, incl, keys, values);
    return rm_host::check_launch("rm_depth_order");
}

int rm_count_pairs(const int32_t* tiles_touched, int64_t n_tets, const uint32_t* status_dev, int64_t* out,
                   void* stream) {
    if (n_tets < 0) return rm_host::fail(RM_EINVAL, "rm_count_pairs: negative size");
    if (!out || (n_tets > 0 && !tiles_touched)) return rm_host::fail(RM_EINVAL, "rm_count_pairs: NULL pointer");
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(int64_t), s);
    if (e != cudaSuccess) return rm_host::fail(RM_ECUDA, "rm_count_pairs: %s", cudaGetErrorString(e));
    const int64_t want = (n_tets + rm::kCountThreads * 8 - 1) / (rm::kCountThreads * 8);
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, 148 * 8));
    rm::count_pairs_kernel<<<blocks, rm::kCountThreads, 0, s>>>(tiles_touched, n_tets, status_dev, out);
    return rm_host::check_launch("rm_count_pairs");
}

size_t rm_emit_ordered_workspace_size(int64_t n_tets) { return rm_depth_order_workspace_size(n_tets); }

int rm_emit_pairs_ordered(const float* vs, const int32_t* rect, const int32_t* tiles_touched, const int32_t* order,
                          int64_t n_tets, const int64_t* n_items_dev, int32_t grid_width, int64_t capacity,
                          int64_t* total_dev, int64_t* keys, int32_t* values, void* workspace,
                          size_t workspace_bytes, uint32_t* status_dev, void* stream) {
    if (n_tets < 0 || capacity < 0) return rm_host::fail(RM_EINVAL, "rm_emit_pairs_ordered: negative size");
    if (!total_dev || !n_items_dev) return rm_host::fail(RM_EINVAL, "rm_emit_pairs_ordered: NULL count");
    cudaStream_t s = (cudaStream_t)stream;
    if (n_tets == 0) {
        cudaError_t e = cudaMemsetAsync(total_dev, 0, sizeof(int64_t), s);
        return e == cudaSuccess ? RM_OK : rm_host::fail(RM_ECUDA, "rm_emit_pairs_ordered: %s", cudaGetErrorString(e));
    }
    if (!vs || !rect || !tiles_touched || !order || !workspace || (capacity > 0 && (!keys || !values)))
        return rm_host::fail(RM_EINVAL, "rm_emit_pairs_ordered: NULL pointer");
    if ((uintptr_t)rect & 15) return rm_host::fail(RM_EINVAL, "rm_emit_pairs_ordered: rect must be 16-byte aligned");
    if (workspace_bytes < rm_emit_ordered_workspace_size(n_tets) || ((uintptr_t)workspace & 255))
        return rm_host::fail(RM_EINVAL, "rm_emit_pairs_ordered: workspace of %zu bytes, 256-byte aligned, needed",
                             rm_emit_ordered_workspace_size(n_tets));
    int32_t* offs = (int32_t*)workspace;
    char* scan_ws = (char*)workspace + (rm_emit_ordered_workspace_size(n_tets) - rm_scan_workspace_size(n_tets));
    int rc = rm_host::scan_mode(rm::kScanGather, tiles_touched, order, n_tets, n_items_dev, offs, total_dev, scan_ws,
                                rm_scan_workspace_size(n_tets), status_dev, s);
    if (rc) return rc;
    const int64_t blocks = std::max<int64_t>(1, (capacity + rm::kEmitPerCta - 1) / rm::kEmitPerCta);
    if (blocks > 0x7fffffff) return rm_host::fail(RM_EINVAL, "rm_emit_pairs_ordered: capacity too large");
    rm::emit_ordered_kernel<<<(unsigned)blocks, rm::kEmitThreads, 0, s>>>(
        vs, (const int4*)rect, order, offs, n_items_dev, n_tets, grid_width, capacity, total_dev, keys, values,
        status_dev);
    return rm_host::check_launch("rm_emit_pairs_ordered");
}

int64_t rm_views_tile_count(const rm_camera* cams, int n_views) {
    rm::ViewSet views;
    if (rm_host::make_views("rm_views_tile_count", cams, n_views, &views)) return -1;
    return views.tiles[n_views];
}

int rm_tile_ranges(const int64_t* sorted_keys, int64_t n, const int64_t* n_dev, int32_t* ranges, int64_t n_tiles,
                   void* stream) {
    if (n < 0 || n_tiles < 0) return rm_host::fail(RM_EINVAL, "rm_tile_ranges: negative size");
    if (n_tiles == 0) return RM_OK;
    if (!ranges) return rm_host::fail(RM_EINVAL, "rm_tile_ranges: NULL ranges");
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(ranges, 0, sizeof(int32_t) * 2 * (size_t)n_tiles, s);
    if (e != cudaSuccess) return rm_host::fail(RM_ECUDA, "rm_tile_ranges: %s", cudaGetErrorString(e));
    if (n == 0) return RM_OK;
    if (!sorted_keys) return rm_host::fail(RM_EINVAL, "rm_tile_ranges: NULL keys");
    const int threads = 256;
    const int64_t blocks = (n + threads - 1) / threads;
    rm::ranges_kernel<<<(unsigned)blocks, threads, 0, s>>>(sorted_keys, n, n_dev, ranges, n_tiles);
    return rm_host::check_launch("rm_tile_ranges");
}

}  // extern "C"

// ------------------------------------------------------------ no allocation --
// A variant of rm_scan_tiles for callers that cannot allocate device memory
// themselves, such as a host runtime that hands the library only its inputs
// and outputs (an FFI caller with no device allocator of its own, or a plugin
// inside an engine that owns every device allocation).  Its look-back scratch
// lives in the fixed array below instead of a caller-provided workspace.
namespace rm {
namespace {

// Largest tet count the fixed scratch covers: 2^26 tets (16,384 scan tiles).
constexpr int64_t kNoAllocMaxTets = int64_t(1) << 26;
constexpr size_t kNoAllocScratchBytes =
    sizeof(ScanWs) + sizeof(uint64_t) * (size_t)((kNoAllocMaxTets + kScanTile - 1) / kScanTile);

// 16 B header + 128 KiB of tile states.  Every GPU that loads this library
// holds one copy until the process exits.
static __device__ __align__(256) unsigned char g_noalloc_scan_scratch[kNoAllocScratchBytes];

// The array's device address, looked up once per CUDA context.  Each context
// loads the module on its own (a context created after cudaDeviceReset, or
// one made current through the driver API, sees the array at another
// address), so the cache is keyed by the context's unique id, never reused
// within a process, rather than by the device ordinal.
typedef int (*CtxGetCurrentFn)(void** ctx);
typedef int (*CtxGetIdFn)(void* ctx, unsigned long long* id);
struct NoAllocSlot {
    unsigned long long ctx_id;
    void* addr;
};
constexpr int kNoAllocSlots = 64;
std::mutex g_noalloc_mu;
NoAllocSlot g_noalloc_slots[kNoAllocSlots] = {};
int g_noalloc_next = 0;
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;

int current_context_id(unsigned long long* id) {
    if (!g_ctx_get_current || !g_ctx_get_id) {
        void* f0 = nullptr;
        void* f1 = nullptr;
        cudaDriverEntryPointQueryResult q0 = cudaDriverEntryPointSymbolNotFound, q1 = q0;
        cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f0, cudaEnableDefault, &q0);
        if (e == cudaSuccess) e = cudaGetDriverEntryPoint("cuCtxGetId", &f1, cudaEnableDefault, &q1);
        if (e != cudaSuccess || q0 != cudaDriverEntryPointSuccess || q1 != cudaDriverEntryPointSuccess || !f0 || !f1)
            return rm_host::fail(RM_ECUDA, "rm_scan_tiles_noalloc: driver context query unavailable (%s)",
                                 cudaGetErrorString(e));
        g_ctx_get_current = (CtxGetCurrentFn)f0;
        g_ctx_get_id = (CtxGetIdFn)f1;
    }
    void* ctx = nullptr;
    if (g_ctx_get_current(&ctx) != 0 || !ctx)
        return rm_host::fail(RM_ECUDA, "rm_scan_tiles_noalloc: no current CUDA context");
    if (g_ctx_get_id(ctx, id) != 0) return rm_host::fail(RM_ECUDA, "rm_scan_tiles_noalloc: cuCtxGetId failed");
    return RM_OK;
}

// Set-up: the device address of g_noalloc_scan_scratch in the current
// context.  In host code the array's name is only a host-side handle, so the
// address is looked up with cudaGetSymbolAddress (a host-side lookup that
// allocates nothing) and cached per context.
int noalloc_scratch(void** out) {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return rm_host::fail(RM_ECUDA, "rm_scan_tiles_noalloc: %s", cudaGetErrorString(e));
    unsigned long long id = 0;
    int rc = current_context_id(&id);
    if (rc) {
        // the runtime creates the device's primary context on its first call
        // that needs one; the symbol lookup is such a call
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scan_scratch);
        if (e != cudaSuccess) return rm_host::fail(RM_ECUDA, "rm_scan_tiles_noalloc: %s", cudaGetErrorString(e));
        if ((rc = current_context_id(&id))) return rc;
    }
    for (const NoAllocSlot& sl : g_noalloc_slots)
        if (sl.addr && sl.ctx_id == id) {
            *out = sl.addr;
            return RM_OK;
        }
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scan_scratch);
    if (e != cudaSuccess || !p)
        return rm_host::fail(RM_ECUDA, "rm_scan_tiles_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    g_noalloc_slots[g_noalloc_next] = {id, p};  // oldest context's entry is replaced when the table is full
    g_noalloc_next = (g_noalloc_next + 1) % kNoAllocSlots;
    *out = p;
    return RM_OK;
}

}  // namespace
}  // namespace rm

extern "C" {

int rm_scan_tiles_noalloc(const int32_t* tiles_touched, int64_t n_tets, int32_t* offsets, int64_t* total_dev,
                          void* stream) {
    using namespace rm;
    if (n_tets > kNoAllocMaxTets)
        return rm_host::fail(RM_EINVAL,
                             "rm_scan_tiles_noalloc: %lld tets exceed the fixed scratch limit of %lld tets; use "
                             "rm_scan_tiles with a caller-provided workspace",
                             (long long)n_tets, (long long)kNoAllocMaxTets);
    void* scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    // rm_scan_tiles clears the queue counter and the tile states before the
    // kernel runs, so the contents left by an earlier call do not matter
    return rm_scan_tiles(tiles_touched, n_tets, offsets, total_dev, scratch, kNoAllocScratchBytes, stream);
}

int rm_scan_noalloc_read_status(uint32_t* status_host, void* stream) {
    if (!status_host) return rm_host::fail(RM_EINVAL, "rm_scan_noalloc_read_status: NULL pointer");
    void* scratch = nullptr;
    int rc = rm::noalloc_scratch(&scratch);
    if (rc) return rc;
    return rm_read_status((const uint32_t*)scratch, status_host, stream);  // status is the array's first word
}

}  // extern "C"
