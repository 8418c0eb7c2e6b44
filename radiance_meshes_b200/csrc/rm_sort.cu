// rm_sort.cu - stage (c): stable onesweep LSD radix sort of (int64 key, int32
// value) pairs on key bits [0, end_bit).
//
// Replaces sort_by_keys (sort_by_keys/sort_by_keys.cu:10-53), i.e.
// cub::DeviceRadixSort::SortPairs(keys, values, n, 0, 32 + msb) with
// msb = bit_length(grid_w * grid_h) (tile_shader_slang.py:57-59).
//
// Design: one histogram kernel computes the digit histograms of every pass in
// a single read of the keys; then one kernel per 8-bit digit pass.  Each CTA of
// a pass takes the next 4096-pair tile (dynamic tile id, so predecessors are
// always running or done), ranks its keys per warp with match.any (warp-striped
// element order keeps the sort stable), publishes per-digit tile counts and
// obtains each digit's global offset by decoupled look-back over earlier tiles
// (bounded spin; a timeout sets RM_STATUS_SORT_TIMEOUT and the CTA proceeds),
// then scatters through shared memory so each digit run is written coalesced.
#include "rm_internal.cuh"

namespace rm {
namespace {

// Tile shape of a pass (threads x pairs per thread); a build may override it
// (threads >= 256: one thread per digit).
#ifndef RM_SORT_THREADS
#define RM_SORT_THREADS 512
#endif
#ifndef RM_SORT_ITEMS
#define RM_SORT_ITEMS 8
#endif
constexpr int kSortThreads = RM_SORT_THREADS;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = RM_SORT_ITEMS;
static_assert(kSortThreads >= 256, "one thread per 8-bit digit");
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096 pairs per CTA
constexpr int kRadix = 256;
constexpr int kMaxPasses = 8;
constexpr uint32_t kLbAgg = 1u << 30;
constexpr uint32_t kLbInc = 2u << 30;
constexpr uint32_t kLbMask = (1u << 30) - 1;

struct SortHeader {
    uint32_t status;
    uint32_t pad[3];
    uint32_t counters[kMaxPasses];
    uint32_t hist[kMaxPasses][kRadix];
};

__host__ __device__ __forceinline__ int64_t sort_tiles(int64_t n) { return (n + kSortTile - 1) / kSortTile; }

__host__ __forceinline__ size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

struct SortLayout {
    size_t lookback_off, alt_keys_off, alt_vals_off, total;
    size_t memset_bytes;  // header + lookback (zeroed every call, status excluded)
};

__host__ SortLayout sort_layout(int64_t n, int npasses) {
    SortLayout L;
    const int64_t tiles = sort_tiles(n) > 0 ? sort_tiles(n) : 1;
    L.lookback_off = align_up(sizeof(SortHeader), 256);
    const size_t lb = sizeof(uint32_t) * (size_t)npasses * (size_t)tiles * kRadix;
    L.alt_keys_off = align_up(L.lookback_off + lb, 256);
    L.alt_vals_off = align_up(L.alt_keys_off + sizeof(uint64_t) * (size_t)(n > 0 ? n : 1), 256);
    L.total = align_up(L.alt_vals_off + sizeof(uint32_t) * (size_t)(n > 0 ? n : 1), 256);
    L.memset_bytes = L.lookback_off + lb;
    return L;
}

// Look-back states: the flag and the count share one 32-bit word and nothing
// else is published through it, so relaxed GPU-scope accesses suffice (no
// release fence per store, no acquire per poll).
__device__ __forceinline__ void st_relaxed32(uint32_t* p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_relaxed32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Digit histograms of every pass in one read of the keys.  Each thread counts
// a contiguous run of kHistRun keys (16-byte vector loads when the run is
// whole and aligned; consecutive threads take consecutive runs) and adds to
// the block's shared histogram only where a pass's digit changes along the
// run, and once at its end: pairs emitted per tet or per tile repeat their
// digits, so most keys add nothing, and no warp vote is needed.
constexpr int kHistThreads = 256;
constexpr int kHistRun = 16;

__global__ void __launch_bounds__(kHistThreads) hist_kernel(const uint64_t* __restrict__ keys, int64_t cap,
                                                            const int64_t* __restrict__ n_dev, int npasses,
                                                            int begin_bit, int end_bit, SortHeader* hdr) {
    __shared__ uint32_t sh[kMaxPasses][kRadix];
    for (int j = threadIdx.x; j < kMaxPasses * kRadix; j += blockDim.x) (&sh[0][0])[j] = 0;
    __syncthreads();
    const int64_t n = n_dev ? min(*n_dev, cap) : cap;
    const uint64_t mask = end_bit >= 64 ? ~0ull : ((1ull << end_bit) - 1);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x * kHistRun;
    for (int64_t s0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * kHistRun; s0 < n; s0 += stride) {
        const int m = (int)min((int64_t)kHistRun, n - s0);  // >= 1
        uint64_t k[kHistRun];
        if (m == kHistRun && ((reinterpret_cast<uintptr_t>(keys + s0) & 15) == 0)) {
            const ulonglong2* v = reinterpret_cast<const ulonglong2*>(keys + s0);
#pragma unroll
            for (int i = 0; i < kHistRun / 2; ++i) {
                const ulonglong2 x = __ldg(v + i);
                k[2 * i] = x.x;
                k[2 * i + 1] = x.y;
            }
        } else {
#pragma unroll
            for (int i = 0; i < kHistRun; ++i) k[i] = i < m ? __ldg(keys + s0 + i) : 0ull;
        }
#pragma unroll
        for (int i = 0; i < kHistRun; ++i) k[i] = (k[i] & mask) >> begin_bit;
        for (int p = 0; p < npasses; ++p) {
            const int sh_p = 8 * p;
            uint32_t last = (uint32_t)(k[0] >> sh_p) & 255u, cnt = 1u;
#pragma unroll
            for (int i = 1; i < kHistRun; ++i) {
                const bool v = i < m;
                const uint32_t d = v ? ((uint32_t)(k[i] >> sh_p) & 255u) : last;
                if (d != last) {
                    atomicAdd(&sh[p][last], cnt);
                    last = d;
                    cnt = 0u;
                }
                cnt += v ? 1u : 0u;
            }
            atomicAdd(&sh[p][last], cnt);
        }
    }
    __syncthreads();
    for (int j = threadIdx.x; j < npasses * kRadix; j += blockDim.x) {
        const uint32_t c = (&sh[0][0])[j];
        if (c) atomicAdd(&(&hdr->hist[0][0])[j], c);
    }
}

// Turns each pass's digit histogram into exclusive global digit offsets.
__global__ void __launch_bounds__(kRadix) hist_scan_kernel(SortHeader* hdr) {
    __shared__ uint32_t s[kRadix / 32];
    const int p = blockIdx.x;
    const uint32_t v = hdr->hist[p][threadIdx.x];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) s[warp] = inc;
    __syncthreads();
    uint32_t wpre = 0;
    for (int w = 0; w < warp; ++w) wpre += s[w];
    hdr->hist[p][threadIdx.x] = wpre + inc - v;
}

struct PassSmem {
    uint32_t warp_hist[kSortWarps][kRadix];
    uint32_t tile_off[kRadix];
    uint32_t global_start[kRadix];
    uint32_t scan_tmp[kRadix / 32];
    uint32_t tile;
    uint64_t keys[kSortTile];
    uint32_t vals[kSortTile];
};

__global__ void __launch_bounds__(kSortThreads, 1024 / kSortThreads) onesweep_kernel(
    const uint64_t* __restrict__ kin, const uint32_t* __restrict__ vin, uint64_t* __restrict__ kout,
    uint32_t* __restrict__ vout, int64_t cap, const int64_t* __restrict__ n_dev, int pass, int shift,
    uint32_t dmask, SortHeader* hdr, uint32_t* __restrict__ lookback, uint32_t* status, uint32_t spin_limit) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    PassSmem& S = *reinterpret_cast<PassSmem*>(smem_raw);
    const int64_t n = n_dev ? min(*n_dev, cap) : cap;
    if (threadIdx.x == 0) S.tile = atomicAdd(&hdr->counters[pass], 1u);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int d = lane; d < kRadix; d += 32) S.warp_hist[warp][d] = 0;
    __syncthreads();
    const uint32_t tile = S.tile;
    const int64_t tile_base = (int64_t)tile * kSortTile;
    if (tile_base >= n) return;
    const int64_t valid_in_tile = min((int64_t)kSortTile, n - tile_base);
    const uint32_t invalid = (uint32_t)(kSortTile - valid_in_tile);

    uint64_t key[kSortItems];
    uint32_t val[kSortItems];
    uint32_t dig[kSortItems];
    uint32_t rank[kSortItems];
    const int64_t wbase = tile_base + (int64_t)warp * (kSortItems * 32);
#pragma unroll
    for (int i = 0; i < kSortItems; ++i) {
        const int64_t idx = wbase + i * 32 + lane;
        const bool valid = idx < n;
        key[i] = valid ? __ldg(kin + idx) : ~0ull;
        val[i] = valid ? __ldg(vin + idx) : 0u;
        dig[i] = valid ? ((uint32_t)(key[i] >> shift) & dmask) : 255u;
    }
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int i = 0; i < kSortItems; ++i) {
        const uint32_t peers = __match_any_sync(0xffffffffu, dig[i]);
        const uint32_t before = S.warp_hist[warp][dig[i]];
        __syncwarp();
        if ((peers & lt) == 0) S.warp_hist[warp][dig[i]] = before + __popc(peers);
        __syncwarp();
        rank[i] = before + __popc(peers & lt);
    }
    __syncthreads();
    // per digit: exclusive prefix over warps and the tile count, published at
    // once (the inclusive prefix for tile 0) so that successors can look back
    uint32_t count = 0, vcount = 0;
    if (threadIdx.x < kRadix) {
        const int d = threadIdx.x;
        uint32_t sum = 0;
        for (int w = 0; w < kSortWarps; ++w) {
            const uint32_t c = S.warp_hist[w][d];
            S.warp_hist[w][d] = sum;
            sum += c;
        }
        count = sum;
        vcount = (d == 255) ? sum - invalid : sum;
        uint32_t* lb = lookback + (size_t)tile * kRadix + d;
        if (tile == 0) {
            const uint32_t excl = hdr->hist[pass][d];
            st_relaxed32(lb, kLbInc | ((excl + vcount) & kLbMask));
            S.global_start[d] = excl;
        } else {
            st_relaxed32(lb, kLbAgg | (vcount & kLbMask));
        }
    }
    // exclusive scan of the tile's digit counts -> start of each digit run in smem
    if (threadIdx.x < kRadix) {
        uint32_t inc = count;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        if (lane == 31) S.scan_tmp[warp] = inc;
        S.tile_off[threadIdx.x] = inc - count;  // warp-local for now
    }
    __syncthreads();
    if (threadIdx.x < kRadix) {
        uint32_t wpre = 0;
        for (int w = 0; w < warp; ++w) wpre += S.scan_tmp[w];
        S.tile_off[threadIdx.x] += wpre;
    }
    __syncthreads();
    // the local scatter needs no global offsets: it runs before the look-back,
    // so the other warps' scatter overlaps the digit threads' polling
#pragma unroll
    for (int i = 0; i < kSortItems; ++i) {
        const uint32_t lpos = S.tile_off[dig[i]] + S.warp_hist[warp][dig[i]] + rank[i];
        S.keys[lpos] = key[i];
        S.vals[lpos] = val[i];
    }
    if (threadIdx.x < kRadix && tile != 0) {
        const int d = threadIdx.x;
        uint32_t excl = 0;
        int64_t t = (int64_t)tile - 1;
        uint32_t budget = spin_limit;
        while (t >= 0) {
            const uint32_t st = ld_relaxed32(lookback + (size_t)t * kRadix + d);
            const uint32_t flag = st & ~kLbMask;
            if (flag == 0) {
                if (!spin_budget(budget)) {
                    atomicOr(status, RM_STATUS_SORT_TIMEOUT);
                    break;
                }
                continue;
            }
            excl += st & kLbMask;
            if (flag == kLbInc) break;
            --t;
        }
        st_relaxed32(lookback + (size_t)tile * kRadix + d, kLbInc | ((excl + vcount) & kLbMask));
        S.global_start[d] = excl;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kSortItems; ++i) {
        const int pos = i * kSortThreads + threadIdx.x;
        if (pos < valid_in_tile) {
            const uint64_t k = S.keys[pos];
            const uint32_t d = (uint32_t)(k >> shift) & dmask;
            const uint64_t dst = (uint64_t)S.global_start[d] + (uint64_t)(pos - S.tile_off[d]);
            if (dst < (uint64_t)n) {  // only a timed-out look-back can produce dst >= n
                kout[dst] = k;
                vout[dst] = S.vals[pos];
            }
        }
    }
}

}  // namespace
}  // namespace rm

extern "C" {

size_t rm_sort_workspace_size(int64_t n) {
    if (n < 0) return 0;
    return rm::sort_layout(n, rm::kMaxPasses).total;
}

int rm_sort_pairs_range(const int64_t* keys_in, const int32_t* values_in, int64_t n, const int64_t* n_dev,
                        int begin_bit, int end_bit, int64_t* keys_out, int32_t* values_out, void* workspace,
                        size_t workspace_bytes, uint32_t* status_dev, void* stream) {
    using namespace rm;
    if (n < 0) return rm_host::fail(RM_EINVAL, "rm_sort_pairs: negative size");
    if (end_bit < 1 || end_bit > 64 || begin_bit < 0 || begin_bit >= end_bit)
        return rm_host::fail(RM_EINVAL, "rm_sort_pairs: key bits [%d, %d) out of range", begin_bit, end_bit);
    if (n >= (int64_t)kLbMask) return rm_host::fail(RM_EINVAL, "rm_sort_pairs: at most 2^30-1 pairs");
    if (n == 0) return RM_OK;
    if (!keys_in || !values_in || !keys_out || !values_out || !workspace)
        return rm_host::fail(RM_EINVAL, "rm_sort_pairs: NULL pointer");
    const int npasses = (end_bit - begin_bit + 7) / 8;
    const SortLayout L = sort_layout(n, npasses);
    if (workspace_bytes < L.total)
        return rm_host::fail(RM_EINVAL, "rm_sort_pairs: workspace %zu < %zu bytes", workspace_bytes, L.total);
    if ((uintptr_t)workspace & 255) return rm_host::fail(RM_EINVAL, "rm_sort_pairs: workspace must be 256-byte aligned");
    cudaStream_t s = (cudaStream_t)stream;
    char* ws = (char*)workspace;
    SortHeader* hdr = (SortHeader*)ws;
    uint32_t* lookback = (uint32_t*)(ws + L.lookback_off);
    uint64_t* alt_k = (uint64_t*)(ws + L.alt_keys_off);
    uint32_t* alt_v = (uint32_t*)(ws + L.alt_vals_off);
    cudaError_t e = cudaMemsetAsync(ws + 4, 0, L.memset_bytes - 4, s);
    if (e != cudaSuccess) return rm_host::fail(RM_ECUDA, "rm_sort_pairs: %s", cudaGetErrorString(e));
    e = cudaFuncSetAttribute(onesweep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(PassSmem));
    if (e != cudaSuccess) return rm_host::fail(RM_ECUDA, "rm_sort_pairs: %s", cudaGetErrorString(e));
    const int64_t tiles = sort_tiles(n);
    const int64_t runs = (n + kHistThreads * kHistRun - 1) / (kHistThreads * kHistRun);
    const int hist_blocks = (int)(runs < 148 * 4 ? runs : 148 * 4);
    hist_kernel<<<hist_blocks, kHistThreads, 0, s>>>((const uint64_t*)keys_in, n, n_dev, npasses, begin_bit, end_bit,
                                                     hdr);
    hist_scan_kernel<<<npasses, kRadix, 0, s>>>(hdr);
    const uint64_t* src_k = (const uint64_t*)keys_in;
    const uint32_t* src_v = (const uint32_t*)values_in;
    for (int p = 0; p < npasses; ++p) {
        // the last pass must land in the caller's output buffers
        const bool to_out = ((npasses - 1 - p) % 2) == 0;
        uint64_t* dk = to_out ? (uint64_t*)keys_out : alt_k;
        uint32_t* dv = to_out ? (uint32_t*)values_out : alt_v;
        const int shift = begin_bit + 8 * p;
        const int bits = (end_bit - shift) < 8 ? (end_bit - shift) : 8;
        const uint32_t dmask = (bits >= 8) ? 255u : ((1u << bits) - 1u);
        onesweep_kernel<<<(unsigned)tiles, kSortThreads, sizeof(PassSmem), s>>>(
            src_k, src_v, dk, dv, n, n_dev, p, shift, dmask, hdr, lookback + (size_t)p * tiles * kRadix,
            status_dev ? status_dev : &hdr->status, rm_host::wait_limit());
        src_k = dk;
        src_v = dv;
    }
    return rm_host::check_launch("rm_sort_pairs", 2 + npasses);
}

int rm_sort_pairs(const int64_t* keys_in, const int32_t* values_in, int64_t n, const int64_t* n_dev, int end_bit,
                  int64_t* keys_out, int32_t* values_out, void* workspace, size_t workspace_bytes,
                  uint32_t* status_dev, void* stream) {
    return rm_sort_pairs_range(keys_in, values_in, n, n_dev, 0, end_bit, keys_out, values_out, workspace,
                               workspace_bytes, status_dev, stream);
}

}  // extern "C"
