// rm_blend.cu - stage (d): front-to-back tile blend and its back-to-front
// adjoint.
//
// Forward: splat_tiled / alpha_blend (alphablend_shader_interp.slang:194-271,
// 371-431) with evaluate_tetra_interp and integrate_tetra_segment
// (interp_version.slang:21-98) and ray_tetrahedron_intersect_fused
// (intersect.slang:394-624).  Backward: bwd_alpha_blend
// (alphablend_shader_interp.slang:273-369), with the per-tet derivatives that
// the reference obtains from Slang autodiff written out by hand.
//
// Work decomposition.  Per-tile list lengths are heavy-tailed (a few tiles
// hold 10-30x the mean), and a pixel whose ray sees through a dense region
// crosses thousands of tets.  Each pass therefore runs two persistent kernels
// concurrently, fed by one heavy-first tile order computed on the device:
//   * the dense kernel walks the ordinary tiles, one thread per pixel, in
//     strips of 64 pixels (one CTA per strip);
//   * the pair kernel takes the heavy tiles (list length >= ~4x the mean) and
//     spreads each strip's (entry, pixel) pairs over 4 threads per pixel; the
//     strictly ordered part of the walk (log T, termination, distortion
//     moments in the forward; the undo chains in the backward) is a few adds
//     per entry done by one owner thread per pixel, in the same arithmetic as
//     the dense walk, so results do not depend on which kernel ran a tile.
// In both, per-tet records (128 B, packed once per frame by pack_kernel) are
// staged in shared memory per batch of list entries.  Backward gradients are
// summed per list entry across the pixels of a CTA (warp reduce-scatter, then
// shared-memory atomics) and converted to vertex gradients once per
// (CTA, entry) before the global atomics.
#include <mutex>

#include "rm_internal.cuh"

namespace rm {
namespace {

constexpr float kTermLogT = -5.5f;  // alphablend_shader_interp.slang:257
constexpr int kNGrad = 25;


// ------------------------------------------------------------------ packing --
// A tet with an index outside [0, n_verts) gets an all-zero record: zero
// normals and zero density, so no ray hits it, and its vertices are never read.
__global__ void __launch_bounds__(256) pack_kernel(const int4* __restrict__ indices, const float* __restrict__ verts,
                                                   int64_t n_verts, const float* __restrict__ cv, int64_t n_tets,
                                                   const int32_t* __restrict__ tiles, float4* __restrict__ recs) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_tets) return;
    if (tiles && __ldg(tiles + g) <= 0) return;
    const int4 id = __ldg(indices + g);
    if (!tet_indices_ok(id, n_verts)) {
        float4* r = recs + (int64_t)kRecFloat4 * g;
#pragma unroll
        for (int k = 0; k < kRecFloat4; ++k) r[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    const int ids[4] = {id.x, id.y, id.z, id.w};
    f3 v[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float* p = verts + 3 * (int64_t)ids[i];
        v[i] = {__ldg(p), __ldg(p + 1), __ldg(p + 2)};
    }
    // face normals of ray_tetrahedron_intersect_fused (intersect.slang:449-475)
    f3 n0 = cross3(v[1] - v[0], v[2] - v[0]);
    const bool f0 = dot3(n0, v[3] - v[0]) > 0.f;
    if (f0) n0 = neg3(n0);
    f3 n1 = cross3(v[1] - v[0], v[3] - v[0]);
    const bool f1 = dot3(n1, v[2] - v[0]) > 0.f;
    if (f1) n1 = neg3(n1);
    f3 n2 = cross3(v[2] - v[0], v[3] - v[0]);
    const bool f2 = dot3(n2, v[1] - v[0]) > 0.f;
    if (f2) n2 = neg3(n2);
    f3 n3 = cross3(v[2] - v[1], v[3] - v[1]);
    const bool f3b = dot3(n3, v[0] - v[1]) > 0.f;
    if (f3b) n3 = neg3(n3);
    const float* c = cv + 7 * g;
    const float density = fmaxf(__ldg(c), 0.f);
    const uint32_t flips = (f0 ? 1u : 0u) | (f1 ? 2u : 0u) | (f2 ? 4u : 0u) | (f3b ? 8u : 0u);
    float4* r = recs + (int64_t)kRecFloat4 * g;
    r[0] = make_float4(n0.x, n0.y, n0.z, density);
    r[1] = make_float4(n1.x, n1.y, n1.z, __ldg(c + 1));
    r[2] = make_float4(n2.x, n2.y, n2.z, __ldg(c + 2));
    r[3] = make_float4(n3.x, n3.y, n3.z, __ldg(c + 3));
    r[4] = make_float4(v[0].x, v[0].y, v[0].z, __ldg(c + 4));
    r[5] = make_float4(v[1].x, v[1].y, v[1].z, __ldg(c + 5));
    r[6] = make_float4(v[2].x, v[2].y, v[2].z, __ldg(c + 6));
    r[7] = make_float4(v[3].x, v[3].y, v[3].z, __uint_as_float(flips));
}

__device__ __forceinline__ f3 xyz(float4 q) { return {q.x, q.y, q.z}; }

// Ray / tet intersection (intersect.slang:394-624) on a staged record, with
// the clamps of evaluate_tetra_interp (interp_version.slang:88-89), written
// without branches: every plane is evaluated and the reference's sequential
// "if (tplane > t_enter)" / "if (tplane < t_exit)" updates become selects.
// The quotients are IEEE divisions, so t_enter / t_exit (and with them the
// hit decision, log T and n_contributors) are bit-identical to the reference
// rounding.  The backward also needs the selected planes and denominators.
struct Isect {
    float te, tx;        // raw entering / exiting distances
    float enter, exit;   // clamped
    float dene, denx;    // dot(n, d) of the selected planes
    int ie, ix;          // selected planes (-1: none)
    bool geo;            // geometric hit
};

template <bool PLANES>
__device__ __forceinline__ Isect intersect(const float4* __restrict__ q, f3 o, f3 d) {
    const f3 a0 = xyz(q[4]) - o;
    const f3 a1 = xyz(q[5]) - o;
    float te = -1e30f, tx = 1e30f, dene = 1.f, denx = 1.f;
    int ie = -1, ix = -1;
    bool miss = false;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const f3 n = xyz(q[i]);
        const float dist = -dot3(n, i == 3 ? a1 : a0);
        const float den = dot3(n, d);
        const bool par = fabsf(den) < 1e-10f;
        miss |= par && dist > 0.f;
        const float tp = -dist / den;
        const bool ue = !par && den < 0.f && tp > te;
        const bool ux = !par && !(den < 0.f) && tp < tx;
        te = ue ? tp : te;
        tx = ux ? tp : tx;
        if (PLANES) {
            ie = ue ? i : ie;
            dene = ue ? den : dene;
            ix = ux ? i : ix;
            denx = ux ? den : denx;
        }
    }
    Isect r;
    r.te = te;
    r.tx = tx;
    r.geo = !miss && !(te > tx) && !(tx <= 0.f);
    r.enter = fmaxf(te, 0.f);
    r.exit = fmaxf(tx, r.enter);
    r.dene = dene;
    r.denx = denx;
    r.ie = ie;
    r.ix = ix;
    return r;
}

// Weights of the closed-form segment integral (interp_version.slang:21-40)
// for optical depth x = density * dt >= 0:
//   alpha = exp(-x), phi = (1 - exp(-x)) / x, w0 = phi - alpha, w1 = 1 - phi.
// Below x = 0.25 w0 and w1 come from their Taylor series (8 terms, truncation
// < 4e-10 relative), which avoids the cancellation in phi - alpha and 1 - phi;
// above, phi = (1 - alpha) / x.  These feed only the colour channels, which
// are compared within a tolerance (log T uses x itself, never these weights).
struct Weights {
    float alpha, w0, w1;
};

__device__ __forceinline__ Weights seg_weights(float x) {
    Weights w;
    w.alpha = __expf(-x);
    if (x < 0.25f) {
        // w1 = x/2 - x^2/6 + x^3/24 - x^4/120 + x^5/720 - x^6/5040 + x^7/40320
        w.w1 = x * (0.5f + x * (-1.0f / 6.0f + x * (1.0f / 24.0f + x * (-1.0f / 120.0f + x * (1.0f / 720.0f +
                 x * (-1.0f / 5040.0f + x * (1.0f / 40320.0f)))))));
        // w0 = x/2 - x^2/3 + x^3/8 - x^4/30 + x^5/144 - x^6/840 + x^7/5760
        w.w0 = x * (0.5f + x * (-1.0f / 3.0f + x * (0.125f + x * (-1.0f / 30.0f + x * (1.0f / 144.0f +
                 x * (-1.0f / 840.0f + x * (1.0f / 5760.0f)))))));
    } else {
        const float phi = __fdividef(1.0f - w.alpha, x);
        w.w0 = phi - w.alpha;
        w.w1 = 1.0f - phi;
    }
    return w;
}

// d phi / dx = -(d w1 / dx): series below 0.25, (alpha - phi) / x = -w0 / x above.
__device__ __forceinline__ float dphi_f(float x, const Weights& w) {
    if (x < 0.25f)
        return -(0.5f + x * (-1.0f / 3.0f + x * (0.125f + x * (-1.0f / 30.0f + x * (1.0f / 144.0f +
                 x * (-1.0f / 840.0f))))));
    return -__fdividef(w.w0, x);
}

struct Segment {
    float dt, a, x;
    f3 ve, vx;
    float ce, cx;
    Weights w;
    float rgb[3];
};

// integrate_tetra_segment + compute_integral (interp_version.slang:30-69):
// rgb = w0 * c_exit + w1 * c_enter with c = base + dot(grd, p - v0).
// The colours at the entry and exit points, given those points relative to
// v0 (s.ve, s.vx).
__device__ __forceinline__ void integrate_rel(const float4* __restrict__ q, Segment& s) {
    const float density = q[0].w;
    const f3 grd = {q[4].w, q[5].w, q[6].w};
    s.ce = dot3(grd, s.ve);
    s.cx = dot3(grd, s.vx);
    s.x = s.dt * density;
    s.w = seg_weights(s.x);
    const float base[3] = {q[1].w, q[2].w, q[3].w};
#pragma unroll
    for (int k = 0; k < 3; ++k) s.rgb[k] = fmaf(s.w.w1, s.ce + base[k], s.w.w0 * (s.cx + base[k]));
}

__device__ __forceinline__ void integrate(const float4* __restrict__ q, f3 o, f3 d, float enter, float exit,
                                          Segment& s) {
    const f3 v0 = xyz(q[4]);
    s.ve = {fmaf(enter, d.x, o.x) - v0.x, fmaf(enter, d.y, o.y) - v0.y, fmaf(enter, d.z, o.z) - v0.z};
    s.vx = {fmaf(exit, d.x, o.x) - v0.x, fmaf(exit, d.y, o.y) - v0.y, fmaf(exit, d.z, o.z) - v0.z};
    integrate_rel(q, s);
}


// Pixel (lx, ly) inside the tile of thread t of work item `sub`, for items of
// NT pixels: square blocks of 8x8 (NT = 64) or 4x4 (NT = 16) pixels, row-major
// over the tile, so that the pixels of one item see similar lists; tiles whose
// sides are not multiples of the block fall back to runs of whole rows.
template <int NT>
__device__ __forceinline__ void strip_pixel(const rm_camera& cam, int sub, int t, int& lx, int& ly) {
    constexpr int bw = NT >= 64 ? 8 : 4;
    constexpr int bh = NT / bw;
    if (cam.tile_width % bw == 0 && cam.tile_height % bh == 0) {
        const int nbx = cam.tile_width / bw;
        lx = (sub % nbx) * bw + t % bw;
        ly = (sub / nbx) * bh + t / bw;
    } else {
        const int tp = sub * NT + t;
        lx = tp % cam.tile_width;
        ly = tp / cam.tile_width;
    }
}

struct PixelState {
    float c[3];
    float logT;
    float D[5];
};

// ------------------------------------------------------------------ forward --
template <int NT>
struct WarpShape {
    static constexpr unsigned kMask = NT >= 32 ? 0xffffffffu : ((1u << NT) - 1u);
    static constexpr int kTopOffset = NT >= 32 ? 16 : NT / 2;
    static constexpr int kWarps = NT >= 32 ? NT / 32 : 1;
};

// Work queue shared by the kernels of one pass.  order[] lists the tiles
// heaviest first; info[0] is the number of heavy tiles (the first entries of
// order[]), which go to the pair kernel, the rest to the dense kernel.
// Hit masks written by the forward and read by the backward
// (RM_BLEND_HIT_MASKS; 64-pixel work items only).  A tile's list is cut into
// blocks of 32 entries counted from its start; pixel p of work item `sub`
// keeps, for block k of global tile t whose list starts at position x, one
// word at mask_word(t, x, k, sub, subs, p) whose bit i says whether entry
// x + 32k + i was a hit for that pixel before its termination.  Block ids
// floor(x / 32) + k + t are distinct over all tiles, so the words never
// overlap; a pixel's words of consecutive blocks are 64 words apart, and the
// 64 pixels of an item are contiguous (coalesced stores and loads).  Words at
// or beyond cap do not exist: the entries they would describe are tested.
__device__ __forceinline__ int64_t mask_word(int gtile, int x, int k, int sub, int subs, int p) {
    return (((int64_t)(x >> 5) + k + gtile) * subs + sub) * 64 + p;
}

struct HitMasks {
    uint32_t* words;  // nullptr: no masks
    int64_t cap;      // words
    const uint32_t* header;  // kMaskValid: this pass's forward wrote masks with 64-pixel items
};

constexpr uint32_t kMaskValid = 0x6d61736bu;

// The masks a kernel may use: none unless the header says the forward wrote them.
__device__ __forceinline__ HitMasks live_masks(HitMasks hm) {
    if (hm.words && (!hm.header || __ldcg(hm.header) != kMaskValid)) hm.words = nullptr;
    return hm;
}

struct Queue {
    const int32_t* order;
    const int32_t* info;
    uint32_t* ticket;
    int G;
    int subs;  // strips per tile
    bool heavy;
    HitMasks hm;
    uint32_t* status;     // RM_STATUS_* bits of the pass (a staging copy whose wait gave up)
    uint32_t spin_limit;  // polls of a bounded wait
    int64_t n_recs;       // records (tets) the list ids may name
};

__device__ __forceinline__ int queue_items(const Queue& q) {
    const int nh = __ldg(q.info);
    return (q.heavy ? nh : q.G - nh) * q.subs;
}

__device__ __forceinline__ int queue_tile(const Queue& q, int item) {
    const int first = q.heavy ? 0 : __ldg(q.info);
    return __ldg(q.order + first + item / q.subs);
}

__device__ __forceinline__ int next_item(const Queue& q, int* s_item) {
    if (threadIdx.x == 0) *s_item = (int)atomicAdd(q.ticket, 1u);
    __syncthreads();
    const int item = *s_item;
    __syncthreads();
    return item;
}

// A list entry's tet id, or -1 when it names no record.  Only lists left
// invalid by a scan or sort that gave up (or a caller's corrupt lists) hold
// such ids; the entry is then staged as a zero record, which no ray hits, and
// RM_STATUS_BAD_INDEX is set.
__device__ __forceinline__ int32_t list_id(const int32_t* __restrict__ ids, int64_t e, const Queue& lq) {
    const int32_t g = __ldg(ids + e);
    if (g >= 0 && (int64_t)g < lq.n_recs) return g;
    if (lq.status) atomicOr(lq.status, RM_STATUS_BAD_INDEX);
    return -1;
}

__device__ __forceinline__ float4 record_part(const float4* __restrict__ recs, int32_t g, int c) {
    return g >= 0 ? __ldg(recs + (int64_t)kRecFloat4 * g + c) : make_float4(0.f, 0.f, 0.f, 0.f);
}

// Stores the hit bits of one batch (B a multiple of 32, starting 32-aligned
// relative to the list start) for pixel p: one word per 32 entries.
__device__ __forceinline__ void write_masks(const HitMasks& hm, uint64_t hb, int gtile, int x, int base, int n,
                                            int sub, int subs, int p) {
    const int k0 = (base - x) >> 5;
    for (int w = 0; w * 32 < n; ++w) {
        const int64_t i = mask_word(gtile, x, k0 + w, sub, subs, p);
        if (i < hm.cap) __stcg(hm.words + i, (uint32_t)(hb >> (32 * w)));
    }
}

// One hit folded into the pixel state (update_alpha_out,
// alphablend_shader_interp.slang:84-183): colour += rgb * T, log T -= a, and
// the five distortion moments with m0 = density, m1 = density * (a + b) / 2.
__device__ __forceinline__ void fold_hit(PixelState& st, float a, float m0, float m1, float d4, const float* rgb) {
    const float T = __expf(st.logT);
#pragma unroll
    for (int k = 0; k < 3; ++k) st.c[k] = fmaf(rgb[k], T, st.c[k]);
    st.logT = st.logT - a;
    const float D2 = st.D[2], D3 = st.D[3];
    st.D[0] = fmaf(2.0f * m1, D2, st.D[0]);
    st.D[1] = fmaf(2.0f * m0, D3, st.D[1]);
    st.D[2] = D2 + m0;
    st.D[3] = D3 + m1;
    st.D[4] = st.D[4] + d4;
}

// Result of testing one ray against one list entry, in the exact arithmetic of
// the dense path: a = density * dt (0 for a miss), m1, the D4 increment
// density^2 * dt / 3 and the segment colour.
struct EntryResult {
    float a, m1, d4;
    float rgb[3];
};

__device__ __forceinline__ EntryResult eval_entry(const float4* __restrict__ q, f3 o, f3 d) {
    EntryResult r;
    const Isect is = intersect<false>(q, o, d);
    Segment s;
    s.dt = fmaxf(is.exit - is.enter, 0.f);
    const float density = q[0].w;
    s.a = density * s.dt;
    r.a = 0.f;
    r.m1 = 0.f;
    r.d4 = 0.f;
    r.rgb[0] = r.rgb[1] = r.rgb[2] = 0.f;
    if (is.geo && s.a > 0.f) {
        integrate(q, o, d, is.enter, is.exit, s);
        r.a = s.a;
        r.m1 = density * (is.exit + is.enter) / 2.0f;
        r.d4 = density * density * s.dt / 3.0f;
#pragma unroll
        for (int k = 0; k < 3; ++k) r.rgb[k] = s.rgb[k];
    }
    return r;
}

// Dense forward item: a strip of NT pixels (NT / tile_width rows), one thread
// per pixel walking the tile's list in order.
template <int B>
struct FwdDenseSmem {
    float4 srec[B][kRecFloat4];
    int32_t sid[B];
};

template <int NT, int B>
__device__ __forceinline__ void fwd_dense_item(int tile, int sub, const int32_t* __restrict__ ids,
                                               const int2* __restrict__ ranges, const float4* __restrict__ recs,
                                               const float2* __restrict__ jitter, const rm_camera& cam,
                                               float4* __restrict__ out_img, float* __restrict__ out_dist,
                                               int32_t* __restrict__ out_nc, FwdDenseSmem<B>& S,
                                               const HitMasks& hm, int subs, int gtile, const Queue& lq) {
    constexpr bool kMasks = NT == 64 && B % 32 == 0;
    const int tx = tile % cam.grid_width, ty = tile / cam.grid_width;
    int lx, ly;
    strip_pixel<NT>(cam, sub, (int)threadIdx.x, lx, ly);
    const int px = tx * cam.tile_width + lx, py = ty * cam.tile_height + ly;
    const bool inside = px < cam.image_width && py < cam.image_height;
    const int64_t pix = (int64_t)py * cam.image_width + px;
    f3 o = {0.f, 0.f, 0.f}, d = {0.f, 0.f, 1.f};
    if (inside) {
        const float2 j = __ldg(jitter + pix);
        make_ray(cam, px, py, j.x, j.y, o, d);
    }
    const int2 rg = __ldg(ranges + tile);
    PixelState st = {{0.f, 0.f, 0.f}, 0.f, {0.f, 0.f, 0.f, 0.f, 0.f}};
    int32_t nc = 0;
    bool active = inside;
    if (__syncthreads_or(active)) {
        for (int base = rg.x; base < rg.y; base += B) {
            const int n = min(B, rg.y - base);
            for (int k = threadIdx.x; k < n; k += NT) S.sid[k] = list_id(ids, base + k, lq);
            __syncthreads();
            for (int k = threadIdx.x; k < n * kRecFloat4; k += NT) {
                const int j = k >> 3, c = k & 7;
                S.srec[j][c] = record_part(recs, S.sid[j], c);
            }
            __syncthreads();
            uint64_t hb = 0;  // bit j: entry j of the batch was a hit
            if (__any_sync(WarpShape<NT>::kMask, active)) {
                for (int j = 0; j < n; ++j) {
                    if (!active) break;
                    ++nc;
                    const EntryResult r = eval_entry(S.srec[j], o, d);
                    if (r.a > 0.f) {
                        hb |= 1ull << j;
                        fold_hit(st, r.a, S.srec[j][0].w, r.m1, r.d4, r.rgb);
                        if (st.logT < kTermLogT) active = false;
                    }
                }
            }
            if (kMasks && hm.words) write_masks(hm, hb, gtile, rg.x, base, n, sub, subs, (int)threadIdx.x);
            if (!__syncthreads_or(active)) break;
        }
    }
    if (inside) {
        out_img[pix] = make_float4(st.c[0], st.c[1], st.c[2], st.logT);
        float* dd = out_dist + 5 * pix;
#pragma unroll
        for (int k = 0; k < 5; ++k) dd[k] = st.D[k];
        out_nc[pix] = nc;
    }
}

// Pair forward item: a strip of PX pixels (PX / tile_width rows of one tile)
// handled by NT >= PX threads.  Threads 0..PX-1 own one pixel each.  Per batch
// of B list entries the records are staged in shared memory, the still-active
// pixels are compacted into slots, and all NT threads evaluate the
// (entry, slot) pairs -- a warp takes one entry at a time (its record is read
// as a broadcast) and its lanes take the slots -- writing each pair's a, m1,
// D4 increment and colour to shared memory.  Each owner then folds its
// pixel's results in list order: this sequential part is a handful of adds
// per entry, so a pixel whose ray crosses thousands of tets no longer runs
// the whole intersection/integration chain on one thread.  The fold uses
// exactly the arithmetic of the one-thread-per-pixel walk, so n_contributors,
// log T and the distortion moments are unchanged bit for bit.
template <int PX, int B>
struct FwdPairSmem {
    float4 srec[B][kRecFloat4];
    float dens[2][B];      // densities of the batch being folded and of the one being staged
    float ray[6][PX];      // o, d of each slot (structure of arrays)
    float res[6][B][PX];   // a (0: miss), m1, d4, r, g, b per (entry, slot)
    int32_t warp_base[(PX + 31) / 32];
    float pray[6][PX];     // each owner's own ray, by owner thread (kept out of registers)
};

template <int PX, int B>
__device__ __forceinline__ void store_result(FwdPairSmem<PX, B>& S, int j, int sl, const EntryResult& r) {
    S.res[0][j][sl] = r.a;
    S.res[1][j][sl] = r.m1;
    S.res[2][j][sl] = r.d4;
    S.res[3][j][sl] = r.rgb[0];
    S.res[4][j][sl] = r.rgb[1];
    S.res[5][j][sl] = r.rgb[2];
}

// Stages batch [base, base + n) into srec (and its densities into dens[buf])
// with threads t, t + nt, ...: one float4 of one record each, the thread
// loading the entry's id itself.
template <int PX, int B>
__device__ __forceinline__ void stage_pair_batch(FwdPairSmem<PX, B>& S, int buf, int base, int n,
                                                 const int32_t* __restrict__ ids, const float4* __restrict__ recs,
                                                 const Queue& lq, int t, int nt) {
    for (int k = t; k < n * kRecFloat4; k += nt) {
        const int j = k >> 3, c = k & 7;
        const float4 r = record_part(recs, list_id(ids, base + j, lq), c);
        S.srec[j][c] = r;
        if (c == 0) S.dens[buf][j] = r.w;
    }
}

template <int PX, int NT, int B>
__device__ __forceinline__ void fwd_pair_item(int tile, int sub, const int32_t* __restrict__ ids,
                                         const int2* __restrict__ ranges, const float4* __restrict__ recs,
                                         const float2* __restrict__ jitter, const rm_camera& cam,
                                         float4* __restrict__ out_img, float* __restrict__ out_dist,
                                         int32_t* __restrict__ out_nc, FwdPairSmem<PX, B>& S,
                                         const HitMasks& hm, int subs, int gtile, const Queue& lq) {
    static_assert(PX <= 64 && NT >= 64, "a lane evaluates at most two slots");
    constexpr bool kMasks = PX == 64 && B % 32 == 0;
    constexpr unsigned kOwnMask = WarpShape<PX>::kMask;
    constexpr int kWarps = NT / 32;
    constexpr int kOwnThreads = (PX + 31) / 32 * 32;  // the owners' warps; the rest stage during the fold
    static_assert(NT > kOwnThreads, "staging needs warps besides the owners'");
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const bool owner = tid < PX;
    const int tx = tile % cam.grid_width, ty = tile / cam.grid_width;
    int lx, ly;
    strip_pixel<PX>(cam, sub, tid, lx, ly);
    const int px = tx * cam.tile_width + lx, py = ty * cam.tile_height + ly;
    const bool inside = owner && px < cam.image_width && py < cam.image_height;
    const int64_t pix = (int64_t)py * cam.image_width + px;
    f3 o = {0.f, 0.f, 0.f}, d = {0.f, 0.f, 1.f};
    if (inside) {
        const float2 j = __ldg(jitter + pix);
        make_ray(cam, px, py, j.x, j.y, o, d);
    }
    if (owner) {
        S.pray[0][tid] = o.x; S.pray[1][tid] = o.y; S.pray[2][tid] = o.z;
        S.pray[3][tid] = d.x; S.pray[4][tid] = d.y; S.pray[5][tid] = d.z;
    }
    const int2 rg = __ldg(ranges + tile);
    PixelState st = {{0.f, 0.f, 0.f}, 0.f, {0.f, 0.f, 0.f, 0.f, 0.f}};
    int32_t nc = 0;
    bool active = inside;
    // The first batch is staged by all threads; each later one by the
    // non-owner warps while the owners fold the batch before it (srec is no
    // longer read by then: the fold reads the densities kept in dens[cur]).
    stage_pair_batch(S, 0, rg.x, min(B, rg.y - rg.x), ids, recs, lq, tid, NT);
    int rank = 0;  // the owner's rank among the active pixels of its warp
    if (owner) {
        const unsigned bal = __ballot_sync(kOwnMask, active);
        if (lane == 0) S.warp_base[warp] = __popc(bal);
        rank = __popc(bal & ((1u << lane) - 1u));
    }
    int n_active = __syncthreads_count(active);
    int cur = 0;
    for (int base = rg.x; base < rg.y && n_active > 0; base += B) {
        const int n = min(B, rg.y - base);
        int slot = rank;
        if (active) {
            for (int w = 0; w < warp; ++w) slot += S.warp_base[w];
#pragma unroll
            for (int k = 0; k < 6; ++k) S.ray[k][slot] = S.pray[k][tid];
        }
        __syncthreads();
        // Evaluate.  Rays stay in registers for the whole batch.  With more than
        // 32 active slots a lane takes slots lane and lane + 32 of each entry the
        // warp takes; with fewer, the warp splits into groups of `span` lanes
        // (the next power of two >= n_active, at least 4), each group taking
        // its own entry, so lanes do not idle when most pixels have terminated.
        if (n_active > 32) {
            const bool has1 = lane + 32 < n_active;
            const f3 o0 = {S.ray[0][lane], S.ray[1][lane], S.ray[2][lane]};
            const f3 d0 = {S.ray[3][lane], S.ray[4][lane], S.ray[5][lane]};
            f3 o1 = o0, d1 = d0;
            if (has1) {
                o1 = {S.ray[0][lane + 32], S.ray[1][lane + 32], S.ray[2][lane + 32]};
                d1 = {S.ray[3][lane + 32], S.ray[4][lane + 32], S.ray[5][lane + 32]};
            }
            for (int j = warp; j < n; j += kWarps) {
                store_result(S, j, lane, eval_entry(S.srec[j], o0, d0));
                if (has1) store_result(S, j, lane + 32, eval_entry(S.srec[j], o1, d1));
            }
        } else {
            const int span = n_active <= 4 ? 4 : n_active <= 8 ? 8 : n_active <= 16 ? 16 : 32;
            const int groups = 32 / span;
            const int sl = lane & (span - 1);
            const bool has = sl < n_active;
            f3 o = {0.f, 0.f, 0.f}, d = {0.f, 0.f, 1.f};
            if (has) {
                o = {S.ray[0][sl], S.ray[1][sl], S.ray[2][sl]};
                d = {S.ray[3][sl], S.ray[4][sl], S.ray[5][sl]};
            }
            for (int j = warp * groups + lane / span; j < n; j += kWarps * groups)
                if (has) store_result(S, j, sl, eval_entry(S.srec[j], o, d));
        }
        __syncthreads();
        if (tid >= kOwnThreads) {
            if (base + B < rg.y)
                stage_pair_batch(S, cur ^ 1, base + B, min(B, rg.y - base - B), ids, recs, lq, tid - kOwnThreads,
                                 NT - kOwnThreads);
        } else {
            // Fold in list order; the hit tests of four entries are read ahead.
            uint64_t hb = 0;  // bit j: entry j of the batch was a hit for this owner's pixel
            for (int j0 = 0; active && j0 < n; j0 += 4) {
                float a4[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) a4[u] = j0 + u < n ? S.res[0][j0 + u][slot] : 0.f;
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int j = j0 + u;
                    if (!active || j >= n) break;
                    ++nc;
                    if (a4[u] > 0.f) {
                        hb |= 1ull << j;
                        const float rgb[3] = {S.res[3][j][slot], S.res[4][j][slot], S.res[5][j][slot]};
                        fold_hit(st, a4[u], S.dens[cur][j], S.res[1][j][slot], S.res[2][j][slot], rgb);
                        if (st.logT < kTermLogT) active = false;
                    }
                }
            }
            if (kMasks && owner && hm.words) write_masks(hm, hb, gtile, rg.x, base, n, sub, subs, tid);
            // the next batch's slots: the pixels still active
            if (owner) {
                const unsigned bal = __ballot_sync(kOwnMask, active);
                if (lane == 0) S.warp_base[warp] = __popc(bal);
                rank = __popc(bal & ((1u << lane) - 1u));
            }
        }
        cur ^= 1;
        n_active = __syncthreads_count(active);
    }
    if (inside) {
        out_img[pix] = make_float4(st.c[0], st.c[1], st.c[2], st.logT);
        float* dd = out_dist + 5 * pix;
#pragma unroll
        for (int k = 0; k < 5; ++k) dd[k] = st.D[k];
        out_nc[pix] = nc;
    }
}

template <int NT, int B, class V>
__global__ void __launch_bounds__(NT, (NT >= 64 ? 1024 / NT : 32)) blend_fwd_dense_kernel(
    const int32_t* __restrict__ ids, const int2* __restrict__ ranges, const float4* __restrict__ recs,
    const float2* __restrict__ jitter, const __grid_constant__ V views, float4* __restrict__ out_img,
    float* __restrict__ out_dist, int32_t* __restrict__ out_nc, const Queue q) {
    __shared__ FwdDenseSmem<B> S;
    __shared__ int s_item;
    const int n_items = queue_items(q);
    const HitMasks hm = live_masks(q.hm);
    for (;;) {
        const int item = next_item(q, &s_item);
        if (item >= n_items) return;
        const int t = queue_tile(q, item), v = views.find(t);
        const int tb = views.tile_base(v);
        const int64_t pb = views.pixel_base(v);
        fwd_dense_item<NT, B>(t - tb, item % q.subs, ids, ranges + tb, recs, jitter + pb, views.camera(v),
                              out_img + pb, out_dist + 5 * pb, out_nc + pb, S, hm, q.subs, t, q);
    }
}

// MINB resident CTAs per SM: 1024 / NT caps registers at 64 (some spill),
// 768 / NT at 80 (none spill) for launches asking fewer CTAs per SM.
template <int PX, int NT, int B, int MINB, class V>
__global__ void __launch_bounds__(NT, MINB) blend_fwd_pair_kernel(
    const int32_t* __restrict__ ids, const int2* __restrict__ ranges, const float4* __restrict__ recs,
    const float2* __restrict__ jitter, const __grid_constant__ V views, float4* __restrict__ out_img,
    float* __restrict__ out_dist, int32_t* __restrict__ out_nc, const Queue q) {
    extern __shared__ __align__(16) unsigned char fwd_smem_raw[];
    FwdPairSmem<PX, B>& S = *reinterpret_cast<FwdPairSmem<PX, B>*>(fwd_smem_raw);
    __shared__ int s_item;
    const int n_items = queue_items(q);
    const HitMasks hm = live_masks(q.hm);
    for (;;) {
        const int item = next_item(q, &s_item);
        if (item >= n_items) return;
        const int t = queue_tile(q, item), v = views.find(t);
        const int tb = views.tile_base(v);
        const int64_t pb = views.pixel_base(v);
        fwd_pair_item<PX, NT, B>(t - tb, item % q.subs, ids, ranges + tb, recs, jitter + pb, views.camera(v),
                                 out_img + pb, out_dist + 5 * pb, out_nc + pb, S, hm, q.subs, t, q);
    }
}

// Orders the tiles heaviest first by floor(log2(list length)) (the order
// inside a bucket does not matter), marks as heavy the tiles whose bucket is
// at least heavy_shift above that of the mean non-empty list length and at
// least 2^10 entries (info[0] = their count), and resets the queue tickets.
__global__ void __launch_bounds__(1024) order_kernel(const int2* __restrict__ ranges, int G,
                                                     int32_t* __restrict__ order, int32_t* info,
                                                     uint32_t* tickets, int heavy_shift, uint32_t* mask_header,
                                                     uint32_t mask_state) {
    // Warp-aggregated counting: lanes that share a bucket elect one leader
    // (match_any) for the shared atomic, and the list-length sum and the
    // non-empty count are reduced per warp before one shared update each.
    __shared__ uint32_t cnt[33], base[33], cur[33];
    __shared__ unsigned long long wtotal[32];
    __shared__ uint32_t wnonempty[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x < 33) cnt[threadIdx.x] = 0, cur[threadIdx.x] = 0;
    __syncthreads();
    unsigned long long total = 0ull;
    uint32_t nonempty = 0u;
    const int G_pad = (G + 31) & ~31;  // whole warps iterate together
    for (int t = threadIdx.x; t < G_pad; t += blockDim.x) {
        uint32_t len = 0u;
        if (t < G) {
            const int2 r = __ldg(ranges + t);
            len = (uint32_t)max(r.y - r.x, 0);
        }
        total += len;
        nonempty += __popc(__ballot_sync(0xffffffffu, len != 0u));
        const int b = t < G ? 32 - __clz(len) : 33;
        const unsigned peers = __match_any_sync(0xffffffffu, b);
        if (b < 33 && lane == __ffs(peers) - 1) atomicAdd(&cnt[b], (uint32_t)__popc(peers));
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
    if (lane == 0) wtotal[warp] = total, wnonempty[warp] = nonempty;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long sum = 0ull;
        uint32_t ne = 0u;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) sum += wtotal[k], ne += wnonempty[k];
        uint32_t run = 0;
        for (int b = 32; b >= 0; --b) {
            base[b] = run;
            run += cnt[b];
        }
        const uint32_t mean = ne ? (uint32_t)(sum / ne) : 0u;
        // heavy_shift 1 sends every tile to the pair kernel
        const int b_thr = heavy_shift == 1 ? 0 : max(11, 32 - __clz(mean) + heavy_shift);
        int heavy = 0;
        for (int b = 32; b >= b_thr; --b) heavy += (int)cnt[b];
        info[0] = heavy;
        for (int k = 0; k < 4; ++k) tickets[k] = 0u;
        if (mask_header) *mask_header = mask_state;
    }
    __syncthreads();
    const unsigned lt = (1u << lane) - 1u;
    for (int t = threadIdx.x; t < G_pad; t += blockDim.x) {
        int b = 33;
        if (t < G) {
            const int2 r = __ldg(ranges + t);
            b = 32 - __clz((uint32_t)max(r.y - r.x, 0));
        }
        const unsigned peers = __match_any_sync(0xffffffffu, b);
        const int leader = __ffs(peers) - 1;
        uint32_t at = 0u;
        if (b < 33 && lane == leader) at = atomicAdd(&cur[b], (uint32_t)__popc(peers));
        at = __shfl_sync(0xffffffffu, at, leader);
        if (b < 33) order[base[b] + at + __popc(peers & lt)] = t;
    }
}

// --------------------------------------------------------------- backward --
// Warp reduce-scatter by recursive halving over lane offsets OFF, OFF/2, ..., 1:
// after run(), lane l holds in v[0..R) the warp sums of the original value
// indices [slot, slot + R) (indices >= M are padding).
template <int M, int OFF>
struct ReduceScatter {
    static constexpr int H = (M + 1) / 2;
    static constexpr int R = ReduceScatter<H, OFF / 2>::R;
    template <unsigned MASK>
    static __device__ __forceinline__ void run(float* v, int lane, int& slot) {
        const bool up = (lane & OFF) != 0;
#pragma unroll
        for (int i = 0; i < H; ++i) {
            const float lo = v[i];
            const float hi = (H + i < M) ? v[H + i] : 0.f;
            const float send = up ? lo : hi;
            const float keep = up ? hi : lo;
            v[i] = keep + __shfl_xor_sync(MASK, send, OFF);
        }
        if (up) slot += H;
        ReduceScatter<H, OFF / 2>::template run<MASK>(v, lane, slot);
    }
};
template <int M>
struct ReduceScatter<M, 0> {
    static constexpr int R = M;
    template <unsigned MASK>
    static __device__ __forceinline__ void run(float*, int, int&) {}
};

// Warp sum of the 25 per-lane partials of one entry, through shared memory,
// added to the entry's accumulator acc[0..25).  Each lane stores its row as
// seven float4 (row stride 28 floats: the eight lanes of each store phase
// hit distinct banks); then lane k < 25 adds column k over the 32 rows
// (consecutive lanes read consecutive words).  Fewer instructions than the
// 27-shuffle reduce-scatter for full warps.  red: 32 * kRedStride floats,
// 16-byte aligned, private to the warp.
constexpr int kRedStride = 28;

__device__ __forceinline__ void warp_sum_columns(const float* red, int lane, float* __restrict__ acc) {
    __syncwarp();
    if (lane < kNGrad) {
        float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
#pragma unroll
        for (int r = 0; r < 32; r += 4) {
            s0 += red[(r + 0) * kRedStride + lane];
            s1 += red[(r + 1) * kRedStride + lane];
            s2 += red[(r + 2) * kRedStride + lane];
            s3 += red[(r + 3) * kRedStride + lane];
        }
        const float sum = (s0 + s1) + (s2 + s3);
        if (sum != 0.f) atomicAdd(acc + lane, sum);
    }
    __syncwarp();
}

// Rows of hit_grads_planes' output: gl[12..25) and the two planes' normal
// gradients, stored at the planes' columns (ie, ix: -1 for none or a lane
// without a hit, whose gl[12..25) are zero).
// As warp_sum_columns for a warp that walked two entries at once: the rows
// of the lanes in bal_a go to acc_a, the others to acc_b.
__device__ __forceinline__ void warp_sum_columns_split(const float* red, int lane, uint32_t bal_a,
                                                       float* __restrict__ acc_a, float* __restrict__ acc_b) {
    __syncwarp();
    if (lane < kNGrad) {
        float a0 = 0.f, a1 = 0.f, b0 = 0.f, b1 = 0.f;
#pragma unroll
        for (int r = 0; r < 32; r += 2) {
            const float v0 = red[r * kRedStride + lane], v1 = red[(r + 1) * kRedStride + lane];
            const bool in0 = (bal_a >> r) & 1u, in1 = (bal_a >> (r + 1)) & 1u;
            a0 += in0 ? v0 : 0.f;
            b0 += in0 ? 0.f : v0;
            a1 += in1 ? v1 : 0.f;
            b1 += in1 ? 0.f : v1;
        }
        const float sa = a0 + a1, sb = b0 + b1;
        if (sa != 0.f) atomicAdd(acc_a + lane, sa);
        if (sb != 0.f) atomicAdd(acc_b + lane, sb);
    }
    __syncwarp();
}

// acc_b != nullptr: the rows of the lanes outside bal_a go to acc_b.
__device__ __forceinline__ void warp_sum_rows_planes(float* __restrict__ red, const float* gl, f3 dne, f3 dnx,
                                                     int ie, int ix, int lane, float* __restrict__ acc,
                                                     uint32_t bal_a = 0u, float* __restrict__ acc_b = nullptr) {
    float* rowf = red + lane * kRedStride;
    float4* row = reinterpret_cast<float4*>(rowf);
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    row[0] = z;
    row[1] = z;
    row[2] = z;
#pragma unroll
    for (int c = 3; c < 6; ++c) row[c] = make_float4(gl[4 * c], gl[4 * c + 1], gl[4 * c + 2], gl[4 * c + 3]);
    row[6] = make_float4(gl[24], 0.f, 0.f, 0.f);
    if (ie >= 0) {
        rowf[3 * ie] = dne.x;
        rowf[3 * ie + 1] = dne.y;
        rowf[3 * ie + 2] = dne.z;
    }
    if (ix >= 0) {
        rowf[3 * ix] = dnx.x;
        rowf[3 * ix + 1] = dnx.y;
        rowf[3 * ix + 2] = dnx.z;
    }
    if (acc_b)
        warp_sum_columns_split(red, lane, bal_a, acc, acc_b);
    else
        warp_sum_columns(red, lane, acc);
}

// Adjoint of one hit (the Slang autodiff of update_alpha_out,
// evaluate_tetra_interp and load_tet_alphablend_interp, written out by hand).
// Inputs: the entry's intersection and segment, T = exp(log T) and D2, D3 of
// the state before the hit, and dL/d(state after the hit) (dS_c, dS_logT,
// dS_D).  Outputs the 25 per-entry partials gl[] (face normals 0..11, direct
// v0 12..14, v1 15..17, density 18, rgb 19..21, grd 22..24) and returns
// dL/d(log T before the hit); nD2 / nD3 receive dL/d(D2, D3 before the hit).
// a0, a1: v0 - o and v1 - o (the reference vertices of the planes).
//
// hit_grads_planes leaves gl[0..12) alone and returns the gradients of the
// entering and exiting planes' normals (planes is.ie, is.ix) in dne, dnx
// (both zero for a plane index of -1); hit_grads_a scatters them into
// gl[0..12).
__device__ __forceinline__ float hit_grads_planes(const float4* __restrict__ q, f3 a0, f3 a1, f3 d,
                                                  const Isect& is, const Segment& s, float T, float D2_old,
                                                  float D3_old, const float* dS_c, float dS_logT, const float* dS_D,
                                                  float* gl, f3& dne, f3& dnx, float& nD2, float& nD3) {
    const float density = q[0].w;
    const float enter = is.enter, exit = is.exit;
    const float m1 = density * (exit + enter) / 2.0f;
    // update_distortion_state
    const float dm1 = dS_D[0] * 2.0f * D2_old + dS_D[3];
    const float dm0 = dS_D[1] * 2.0f * D3_old + dS_D[2];
    nD2 = dS_D[2] + dS_D[0] * 2.0f * m1;
    nD3 = dS_D[3] + dS_D[1] * 2.0f * density;
    float d_dens = dm0 + dm1 * (exit + enter) * 0.5f;
    float d_enter = dm1 * density * 0.5f;
    float d_exit = d_enter;
    float d_dt = dS_D[4] * density * density * (1.0f / 3.0f);
    d_dens += dS_D[4] * 2.0f * density * s.dt * (1.0f / 3.0f);
    // update_pixel_state
    float d_rgb[3], dT = 0.f, sum_drgb = 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        d_rgb[k] = dS_c[k] * T;
        dT = fmaf(dS_c[k], s.rgb[k], dT);
        sum_drgb += d_rgb[k];
    }
    const float d_a = -dS_logT;
    // compute_integral / integrate_tetra_segment
    const float base[3] = {q[1].w, q[2].w, q[3].w};
    float d_w0 = 0.f, d_w1 = 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        d_w0 = fmaf(d_rgb[k], s.cx + base[k], d_w0);
        d_w1 = fmaf(d_rgb[k], s.ce + base[k], d_w1);
        gl[19 + k] = d_rgb[k] * (s.w.w0 + s.w.w1);
    }
    const float d_sx = sum_drgb * s.w.w0, d_se = sum_drgb * s.w.w1;
    const float d_x = (d_w0 - d_w1) * dphi_f(s.x, s.w) + d_w0 * s.w.alpha;
    d_dt += (d_x + d_a) * density;
    d_dens += (d_x + d_a) * s.dt;
    const f3 grd = {q[4].w, q[5].w, q[6].w};
    gl[22] = d_se * s.ve.x + d_sx * s.vx.x;
    gl[23] = d_se * s.ve.y + d_sx * s.vx.y;
    gl[24] = d_se * s.ve.z + d_sx * s.vx.z;
    const float d_sum = d_se + d_sx;
    const float gd = dot3(grd, d);
    d_enter += d_se * gd;
    d_exit += d_sx * gd;
    gl[12] = -grd.x * d_sum;
    gl[13] = -grd.y * d_sum;
    gl[14] = -grd.z * d_sum;
    gl[15] = gl[16] = gl[17] = 0.f;
    if (exit - enter > 0.f) {
        d_exit += d_dt;
        d_enter -= d_dt;
    }
    gl[18] = density > 0.f ? d_dens : 0.f;
    float d_tx = 0.f;
    if (is.tx > enter) d_tx = d_exit; else d_enter += d_exit;
    const float d_te = is.te > 0.f ? d_enter : 0.f;
    // plane intersections t = dot(n, vref - o) / dot(n, d)
    // gradient factors only (the hit and its t values are exact above): the
    // approximate quotient (2 ulp) is far inside the gradients' tolerance
    const float ge = __fdividef(d_te, is.dene), gx = __fdividef(d_tx, is.denx);
    // a plane index of -1 (no entering / exiting plane) contributes nothing
    const float gek = is.ie >= 0 ? ge : 0.f, gxk = is.ix >= 0 ? gx : 0.f;
    const f3 ae = is.ie == 3 ? a1 : a0, ax = is.ix == 3 ? a1 : a0;
    dne = {gek * (ae.x - is.te * d.x), gek * (ae.y - is.te * d.y), gek * (ae.z - is.te * d.z)};
    dnx = {gxk * (ax.x - is.tx * d.x), gxk * (ax.y - is.tx * d.y), gxk * (ax.z - is.tx * d.z)};
    // the planes' reference vertices (v1 for plane 3, v0 for the others):
    // gradient +n * g; the normals are read from the staged record by index
    const f3 ne = xyz(q[is.ie < 0 ? 0 : is.ie]), nx = xyz(q[is.ix < 0 ? 0 : is.ix]);
    const float ge0 = is.ie == 3 ? 0.f : gek, ge1 = is.ie == 3 ? gek : 0.f;
    const float gx0 = is.ix == 3 ? 0.f : gxk, gx1 = is.ix == 3 ? gxk : 0.f;
    gl[12] += ne.x * ge0 + nx.x * gx0;
    gl[13] += ne.y * ge0 + nx.y * gx0;
    gl[14] += ne.z * ge0 + nx.z * gx0;
    gl[15] += ne.x * ge1 + nx.x * gx1;
    gl[16] += ne.y * ge1 + nx.y * gx1;
    gl[17] += ne.z * ge1 + nx.z * gx1;
    // safe_exp's clip at log(1e20) never binds: log T <= 0
    return dS_logT + dT * T;
}

__device__ __forceinline__ float hit_grads_a(const float4* __restrict__ q, f3 a0, f3 a1, f3 d, const Isect& is,
                                             const Segment& s, float T, float D2_old, float D3_old,
                                             const float* dS_c, float dS_logT, const float* dS_D, float* gl,
                                             float& nD2, float& nD3) {
    f3 dne, dnx;
    const float r = hit_grads_planes(q, a0, a1, d, is, s, T, D2_old, D3_old, dS_c, dS_logT, dS_D, gl, dne, dnx,
                                     nD2, nD3);
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        gl[3 * p + 0] = (is.ie == p ? dne.x : 0.f) + (is.ix == p ? dnx.x : 0.f);
        gl[3 * p + 1] = (is.ie == p ? dne.y : 0.f) + (is.ix == p ? dnx.y : 0.f);
        gl[3 * p + 2] = (is.ie == p ? dne.z : 0.f) + (is.ix == p ? dnx.z : 0.f);
    }
    return r;
}

__device__ __forceinline__ float hit_grads(const float4* __restrict__ q, f3 o, f3 d, const Isect& is,
                                           const Segment& s, float T, float D2_old, float D3_old,
                                           const float* dS_c, float dS_logT, const float* dS_D, float* gl,
                                           float& nD2, float& nD3) {
    return hit_grads_a(q, xyz(q[4]) - o, xyz(q[5]) - o, d, is, s, T, D2_old, D3_old, dS_c, dS_logT, dS_D, gl, nD2,
                       nD3);
}

// Converts the per-entry sums of the 25 partials into vertex and cell-value
// gradients and adds them to global memory (one thread per entry).
template <int NT, int B>
__device__ __forceinline__ void flush_entries(int n, const float4 (*srec)[kRecFloat4], const int32_t* sid,
                                              const float (*sacc)[kNGrad], const int4* __restrict__ indices,
                                              float* __restrict__ gverts, float* __restrict__ gcv) {
    for (int jj = threadIdx.x; jj < n; jj += NT) {
        float v[kNGrad];
        bool any = false;
#pragma unroll
        for (int k = 0; k < kNGrad; ++k) {
            v[k] = sacc[jj][k];
            any |= v[k] != 0.f;
        }
        const int g = sid[jj];
        if (!any || g < 0) continue;
        const float4* q = srec[jj];
        const f3 P[4] = {xyz(q[4]), xyz(q[5]), xyz(q[6]), xyz(q[7])};
        const uint32_t flips = __float_as_uint(q[7].w);
        f3 gv[4] = {{v[12], v[13], v[14]}, {v[15], v[16], v[17]}, {0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
        const int pp[4] = {1, 1, 2, 2}, pq[4] = {0, 0, 0, 1}, pr[4] = {2, 3, 3, 3};
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            f3 gc = {v[3 * p], v[3 * p + 1], v[3 * p + 2]};
            if (flips & (1u << p)) gc = neg3(gc);
            const f3 ea = P[pp[p]] - P[pq[p]], eb = P[pr[p]] - P[pq[p]];
            const f3 ga = cross3(eb, gc), gb = cross3(gc, ea);
            gv[pp[p]] = gv[pp[p]] + ga;
            gv[pr[p]] = gv[pr[p]] + gb;
            gv[pq[p]] = gv[pq[p]] - (ga + gb);
        }
        const int4 id = __ldg(indices + g);
        const int vid[4] = {id.x, id.y, id.z, id.w};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            float* dst = gverts + 3 * (int64_t)vid[i];
            if (gv[i].x != 0.f) atomicAdd(dst, gv[i].x);
            if (gv[i].y != 0.f) atomicAdd(dst + 1, gv[i].y);
            if (gv[i].z != 0.f) atomicAdd(dst + 2, gv[i].z);
        }
        float* dc = gcv + 7 * (int64_t)g;
#pragma unroll
        for (int k = 0; k < 7; ++k)
            if (v[18 + k] != 0.f) atomicAdd(dc + k, v[18 + k]);
    }
}

// Dense backward item: a strip of NT pixels, one thread per pixel walking its
// list back to front from the saved final state.
template <int NT, int B>
struct BwdDenseSmem {
    float4 srec[B][kRecFloat4];
    float4 red[NT >= 32 ? NT / 32 : 1][NT >= 32 ? 32 * kRedStride / 4 : 1];  // warp_sum_rows_planes rows, per warp
    int32_t sid[B];
    float sacc[B][kNGrad];
    int32_t smax[WarpShape<NT>::kWarps];
    uint32_t sor[WarpShape<NT>::kWarps][2];  // per warp: OR of its pixels' hit bits (two 32-entry blocks)
    uint8_t cidx[B];                          // batch positions of the entries some pixel hit
    int32_t n_keep;
};

template <int NT, int B>
__device__ __forceinline__ void bwd_dense_item(
    int tile, int sub, const int32_t* __restrict__ ids, const int2* __restrict__ ranges,
    const float4* __restrict__ recs, const int4* __restrict__ indices, const float2* __restrict__ jitter,
    const rm_camera& cam, const float4* __restrict__ img, const float* __restrict__ dist,
    const int32_t* __restrict__ ncs, const float4* __restrict__ gimg, const float* __restrict__ gdist,
    float* __restrict__ gverts, float* __restrict__ gcv, BwdDenseSmem<NT, B>& S, const HitMasks& hm, int subs, int gtile,
    const Queue& lq) {
    constexpr unsigned kMask = WarpShape<NT>::kMask;
    constexpr bool kMasks = NT == 64;
    const int tx = tile % cam.grid_width, ty = tile / cam.grid_width;
    int lx, ly;
    strip_pixel<NT>(cam, sub, (int)threadIdx.x, lx, ly);
    const int px = tx * cam.tile_width + lx, py = ty * cam.tile_height + ly;
    const bool inside = px < cam.image_width && py < cam.image_height;
    const int64_t pix = (int64_t)py * cam.image_width + px;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    f3 o = {0.f, 0.f, 0.f}, d = {0.f, 0.f, 1.f};
    float logT = 0.f, D2 = 0.f, D3 = 0.f;  // state along the reverse walk
    float dS_c[3] = {0.f, 0.f, 0.f}, dS_logT = 0.f, dS_D[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
    int32_t nc = 0;
    if (inside) {
        const float2 j = __ldg(jitter + pix);
        make_ray(cam, px, py, j.x, j.y, o, d);
        logT = __ldg(img + pix).w;
        D2 = __ldg(dist + 5 * pix + 2);
        D3 = __ldg(dist + 5 * pix + 3);
        const float4 g = __ldg(gimg + pix);
        dS_c[0] = g.x; dS_c[1] = g.y; dS_c[2] = g.z; dS_logT = g.w;
#pragma unroll
        for (int k = 0; k < 5; ++k) dS_D[k] = gdist ? __ldg(gdist + 5 * pix + k) : 0.f;
        nc = __ldg(ncs + pix);
    }
    int32_t m = nc;
#pragma unroll
    for (int off = WarpShape<NT>::kTopOffset; off > 0; off >>= 1) m = max(m, __shfl_xor_sync(kMask, m, off));
    if (lane == 0) S.smax[warp] = m;
    __syncthreads();
    int32_t tile_max = 0;
#pragma unroll
    for (int w = 0; w < WarpShape<NT>::kWarps; ++w) tile_max = max(tile_max, S.smax[w]);
    const int2 rg = __ldg(ranges + tile);
    const int end = min(rg.y, rg.x + tile_max);
    // batches aligned to multiples of B from the list start, so that one spans
    // at most two 32-entry mask blocks (B <= 64)
    for (int top = end, lo; top > rg.x; top = lo) {
        lo = rg.x + ((top - 1 - rg.x) / B) * B;
        const int n = top - lo;
        __syncthreads();
        // this pixel's hit bits of the (at most two) 32-entry blocks the batch spans
        const int kb0 = (lo - rg.x) >> 5, kb1 = (top - 1 - rg.x) >> 5;
        uint32_t hw0 = 0xffffffffu, hw1 = 0xffffffffu;
        if (kMasks && hm.words) {
            const int64_t i0 = mask_word(gtile, rg.x, kb0, sub, subs, (int)threadIdx.x);
            const int64_t i1 = mask_word(gtile, rg.x, kb1, sub, subs, (int)threadIdx.x);
            if (i0 < hm.cap) hw0 = __ldcg(hm.words + i0);
            if (i1 < hm.cap) hw1 = __ldcg(hm.words + i1);
        }
        // entries no pixel of the item hit are dropped from the batch before
        // staging (the masks of pixels past their n_contributors are zero)
        uint32_t o0 = hw0, o1 = hw1;
#pragma unroll
        for (int off = WarpShape<NT>::kTopOffset; off > 0; off >>= 1) {
            o0 |= __shfl_xor_sync(kMask, o0, off);
            o1 |= __shfl_xor_sync(kMask, o1, off);
        }
        if (lane == 0) {
            S.sor[warp][0] = o0;
            S.sor[warp][1] = o1;
        }
        __syncthreads();
        if (warp == 0) {
            uint32_t c0 = 0, c1 = 0;
#pragma unroll
            for (int w = 0; w < WarpShape<NT>::kWarps; ++w) {
                c0 |= S.sor[w][0];
                c1 |= S.sor[w][1];
            }
            int base_c = 0;
            constexpr int kLanes = NT >= 32 ? 32 : NT;
            for (int k0 = 0; k0 < n; k0 += kLanes) {
                const int k = k0 + lane;
                bool keep = false;
                if (k < n) {
                    const int off = lo + k - rg.x;
                    keep = ((((off >> 5) == kb0 ? c0 : c1) >> (off & 31)) & 1u) != 0u;
                }
                const unsigned bal = __ballot_sync(kMask, keep);
                if (keep) S.cidx[base_c + __popc(bal & ((1u << lane) - 1u))] = (uint8_t)k;
                base_c += __popc(bal);
            }
            if (lane == 0) S.n_keep = base_c;
        }
        __syncthreads();
        const int nk = S.n_keep;
        for (int k = threadIdx.x; k < nk; k += NT) S.sid[k] = list_id(ids, lo + S.cidx[k], lq);
        for (int k = threadIdx.x; k < nk * kNGrad; k += NT) (&S.sacc[0][0])[k] = 0.f;
        __syncthreads();
        for (int k = threadIdx.x; k < nk * kRecFloat4; k += NT) {
            const int j = k >> 3, c = k & 7;
            S.srec[j][c] = record_part(recs, S.sid[j], c);
        }
        __syncthreads();
        for (int jj = nk - 1; jj >= 0;) {
            const int off = lo + S.cidx[jj] - rg.x;
            // with the forward's masks, only its hits are revisited
            const uint32_t hw = (off >> 5) == kb0 ? hw0 : hw1;
            const bool act_a = inside && off < nc && ((hw >> (off & 31)) & 1u);
            const uint32_t bal_a = __ballot_sync(kMask, act_a);
            if (!bal_a) {
                --jj;
                continue;
            }
            // When no pixel of the warp walks both this entry and the one
            // before it, the warp takes both at once: each lane walks the one
            // it hits (its own order is unchanged), and the partials go to
            // the two entries' accumulators by lane.
            bool act_b = false;
            uint32_t bal_b = 0u;
            if constexpr (NT >= 32) {
                if (jj >= 1) {
                    const int off_b = lo + S.cidx[jj - 1] - rg.x;
                    const uint32_t hwb = (off_b >> 5) == kb0 ? hw0 : hw1;
                    act_b = inside && off_b < nc && ((hwb >> (off_b & 31)) & 1u);
                    bal_b = __ballot_sync(kMask, act_b);
                    if (bal_a & bal_b) {
                        act_b = false;
                        bal_b = 0u;
                    }
                }
            }
            const bool act = act_a || act_b;
            const int je = act_b ? jj - 1 : jj;
            const float4* q = S.srec[je];
            float gl[kNGrad];
#pragma unroll
            for (int k = 0; k < kNGrad; ++k) gl[k] = 0.f;
            const Isect is = intersect<true>(q, o, d);
            const float density = q[0].w;
            Segment s;
            s.dt = fmaxf(is.exit - is.enter, 0.f);
            s.a = density * s.dt;
            const bool hit = act && is.geo && s.a > 0.f;
            f3 dne = {0.f, 0.f, 0.f}, dnx = {0.f, 0.f, 0.f};
            if (hit) {
                integrate(q, o, d, is.enter, is.exit, s);
                // undo_alpha_out (alphablend_shader_interp.slang:128-192): only log T, D2
                // and D3 of the earlier state enter the adjoint
                const float m1 = density * (is.exit + is.enter) / 2.0f;
                const float logT_old = logT + s.a;
                const float T = __expf(logT_old);
                D2 = D2 - density;
                D3 = D3 - m1;
                logT = logT_old;
                float nD2, nD3;
                if constexpr (NT >= 32)
                    dS_logT = hit_grads_planes(q, xyz(q[4]) - o, xyz(q[5]) - o, d, is, s, T, D2, D3, dS_c, dS_logT,
                                               dS_D, gl, dne, dnx, nD2, nD3);
                else
                    dS_logT = hit_grads(q, o, d, is, s, T, D2, D3, dS_c, dS_logT, dS_D, gl, nD2, nD3);
                dS_D[2] = nD2;
                dS_D[3] = nD3;
            }
            if (__any_sync(kMask, hit)) {
                if constexpr (NT >= 32) {
                    warp_sum_rows_planes(reinterpret_cast<float*>(S.red[warp]), gl, dne, dnx, hit ? is.ie : -1,
                                         hit ? is.ix : -1, lane, S.sacc[jj], bal_a,
                                         bal_b ? S.sacc[jj - 1] : nullptr);
                } else {
                    using RS = ReduceScatter<kNGrad, WarpShape<NT>::kTopOffset>;
                    int slot = 0;
                    RS::template run<kMask>(gl, lane, slot);
#pragma unroll
                    for (int r = 0; r < RS::R; ++r)
                        if (slot + r < kNGrad && gl[r] != 0.f) atomicAdd(&S.sacc[jj][slot + r], gl[r]);
                }
            }
            jj -= bal_b ? 2 : 1;
        }
        __syncthreads();
        flush_entries<NT, B>(nk, S.srec, S.sid, S.sacc, indices, gverts, gcv);
    }
}

// Dense backward with the records staged by bulk copies (RM_BLEND_STAGE_TMA;
// 64-pixel items).  The walk and its arithmetic are bwd_dense_item's; what
// changes is the staging.  Each batch is planned one batch ahead: its hit
// masks are OR-ed over the item, the entries some pixel hit are listed, their
// tet ids loaded, and warp 0 starts one 128-byte cp.async.bulk per entry
// (global -> this CTA's shared memory, completing on the buffer's mbarrier).
// Two record buffers alternate, so batch k+1's copies are in flight while
// batch k is walked and flushed; each copy lands in the issuing CTA only.
template <int B>
struct BwdTmaSmem {
    float4 srec[2][B][kRecFloat4];
    float4 red[2][32 * kRedStride / 4];  // warp_sum_rows_planes rows, per warp
    float sacc[B][kNGrad];
    int32_t sid[2][B];
    uint8_t cidx[2][B];
    int32_t n_keep[2];
    uint32_t sor[2][2];  // per warp: OR of its pixels' hit bits (two 32-entry blocks)
    int32_t smax[2];
    uint64_t bar[2];
};

// Pipeline position carried across work items: the buffer the next plan
// fills and the parity of each buffer's next completion.
struct TmaPipe {
    uint32_t buf;
    uint32_t parity;  // bit b: parity to wait for on buffer b
};

template <int B>
__device__ __forceinline__ void bwd_tma_plan(BwdTmaSmem<B>& S, int b, int lo, int top, int rgx,
                                             const int32_t* __restrict__ ids, const float4* __restrict__ recs,
                                             const HitMasks& hm, int gtile, int sub, int subs, uint32_t& hw0,
                                             uint32_t& hw1, const Queue& lq) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int n = top - lo;
    const int kb0 = (lo - rgx) >> 5, kb1 = (top - 1 - rgx) >> 5;
    hw0 = 0xffffffffu;
    hw1 = 0xffffffffu;
    if (hm.words) {
        const int64_t i0 = mask_word(gtile, rgx, kb0, sub, subs, (int)threadIdx.x);
        const int64_t i1 = mask_word(gtile, rgx, kb1, sub, subs, (int)threadIdx.x);
        if (i0 < hm.cap) hw0 = __ldcg(hm.words + i0);
        if (i1 < hm.cap) hw1 = __ldcg(hm.words + i1);
    }
    uint32_t o0 = hw0, o1 = hw1;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        o0 |= __shfl_xor_sync(0xffffffffu, o0, off);
        o1 |= __shfl_xor_sync(0xffffffffu, o1, off);
    }
    if (lane == 0) {
        S.sor[warp][0] = o0;
        S.sor[warp][1] = o1;
    }
    __syncthreads();
    if (warp == 0) {
        const uint32_t c0 = S.sor[0][0] | S.sor[1][0], c1 = S.sor[0][1] | S.sor[1][1];
        int base_c = 0;
        for (int k0 = 0; k0 < n; k0 += 32) {
            const int k = k0 + lane;
            bool keep = false;
            if (k < n) {
                const int off = lo + k - rgx;
                keep = ((((off >> 5) == kb0 ? c0 : c1) >> (off & 31)) & 1u) != 0u;
            }
            const unsigned bal = __ballot_sync(0xffffffffu, keep);
            if (keep) S.cidx[b][base_c + __popc(bal & ((1u << lane) - 1u))] = (uint8_t)k;
            base_c += __popc(bal);
        }
        if (lane == 0) S.n_keep[b] = base_c;
    }
    __syncthreads();
    const int nk = S.n_keep[b];
    for (int k = threadIdx.x; k < nk; k += 64) S.sid[b][k] = list_id(ids, lo + S.cidx[b][k], lq);
    __syncthreads();
    if (warp == 0) {
        // every read of this buffer (the batch two back) is behind the barriers above
        int nv = 0;  // entries with a record to copy (the others are zero-filled)
        for (int k0 = 0; k0 < nk; k0 += 32)
            nv += __popc(__ballot_sync(0xffffffffu, k0 + lane < nk && S.sid[b][k0 + lane] >= 0));
        fence_proxy_async_smem();
        if (lane == 0) mbar_arrive_expect_tx(&S.bar[b], (uint32_t)nv * (uint32_t)(kRecFloat4 * sizeof(float4)));
        __syncwarp();
        for (int k = lane; k < nk; k += 32) {
            const int32_t g = S.sid[b][k];
            if (g >= 0)
                bulk_copy_g2s(&S.srec[b][k][0], recs + (int64_t)kRecFloat4 * g,
                              (uint32_t)(kRecFloat4 * sizeof(float4)), &S.bar[b]);
            else
                for (int c = 0; c < kRecFloat4; ++c) S.srec[b][k][c] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
    }
}

template <int B>
__device__ __forceinline__ void bwd_dense_item_tma(
    int tile, int sub, const int32_t* __restrict__ ids, const int2* __restrict__ ranges,
    const float4* __restrict__ recs, const int4* __restrict__ indices, const float2* __restrict__ jitter,
    const rm_camera& cam, const float4* __restrict__ img, const float* __restrict__ dist,
    const int32_t* __restrict__ ncs, const float4* __restrict__ gimg, const float* __restrict__ gdist,
    float* __restrict__ gverts, float* __restrict__ gcv, BwdTmaSmem<B>& S, const HitMasks& hm, int subs, int gtile,
    TmaPipe& pipe, const Queue& q) {
    constexpr int NT = 64;
    const int tx = tile % cam.grid_width, ty = tile / cam.grid_width;
    int lx, ly;
    strip_pixel<NT>(cam, sub, (int)threadIdx.x, lx, ly);
    const int px = tx * cam.tile_width + lx, py = ty * cam.tile_height + ly;
    const bool inside = px < cam.image_width && py < cam.image_height;
    const int64_t pix = (int64_t)py * cam.image_width + px;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    f3 o = {0.f, 0.f, 0.f}, d = {0.f, 0.f, 1.f};
    float logT = 0.f, D2 = 0.f, D3 = 0.f;
    float dS_c[3] = {0.f, 0.f, 0.f}, dS_logT = 0.f, dS_D[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
    int32_t nc = 0;
    if (inside) {
        const float2 j = __ldg(jitter + pix);
        make_ray(cam, px, py, j.x, j.y, o, d);
        logT = __ldg(img + pix).w;
        D2 = __ldg(dist + 5 * pix + 2);
        D3 = __ldg(dist + 5 * pix + 3);
        const float4 g = __ldg(gimg + pix);
        dS_c[0] = g.x; dS_c[1] = g.y; dS_c[2] = g.z; dS_logT = g.w;
#pragma unroll
        for (int k = 0; k < 5; ++k) dS_D[k] = gdist ? __ldg(gdist + 5 * pix + k) : 0.f;
        nc = __ldg(ncs + pix);
    }
    int32_t m = nc;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, off));
    if (lane == 0) S.smax[warp] = m;
    __syncthreads();
    const int32_t tile_max = max(S.smax[0], S.smax[1]);
    const int2 rg = __ldg(ranges + tile);
    const int end = min(rg.y, rg.x + tile_max);
    if (end <= rg.x) return;  // uniform over the CTA
    // batches aligned to multiples of B from the list start (at most two mask blocks each)
    int ctop = end, clo = rg.x + ((end - 1 - rg.x) / B) * B;
    uint32_t cw0, cw1;
    int cb = (int)pipe.buf;
    bwd_tma_plan<B>(S, cb, clo, ctop, rg.x, ids, recs, hm, gtile, sub, subs, cw0, cw1, q);
    pipe.buf ^= 1u;
    for (;;) {
        const int ntop = clo;
        const bool has_next = ntop > rg.x;
        int nlo = 0, nb = 0;
        uint32_t nw0 = 0u, nw1 = 0u;
        if (has_next) {  // the next batch's copies run while this one is walked
            nlo = rg.x + ((ntop - 1 - rg.x) / B) * B;
            nb = (int)pipe.buf;
            bwd_tma_plan<B>(S, nb, nlo, ntop, rg.x, ids, recs, hm, gtile, sub, subs, nw0, nw1, q);
            pipe.buf ^= 1u;
        }
        const int nk = S.n_keep[cb];
        for (int k = threadIdx.x; k < nk * kNGrad; k += NT) (&S.sacc[0][0])[k] = 0.f;
        if (!mbar_wait(&S.bar[cb], (pipe.parity >> cb) & 1u, q.spin_limit)) {
            if (threadIdx.x == 0 && q.status) atomicOr(q.status, RM_STATUS_QUEUE_TIMEOUT);
            mbar_wait(&S.bar[cb], (pipe.parity >> cb) & 1u, q.spin_limit);  // let the copies land before reuse
        }
        pipe.parity ^= 1u << cb;
        __syncthreads();
        const int kb0 = (clo - rg.x) >> 5;
        for (int jj = nk - 1; jj >= 0; --jj) {
            const int off = clo + S.cidx[cb][jj] - rg.x;
            // with the forward's masks, only its hits are revisited
            const uint32_t hw = (off >> 5) == kb0 ? cw0 : cw1;
            const bool act = inside && off < nc && ((hw >> (off & 31)) & 1u);
            if (!__any_sync(0xffffffffu, act)) continue;
            const float4* qr = S.srec[cb][jj];
            float gl[kNGrad];
#pragma unroll
            for (int k = 0; k < kNGrad; ++k) gl[k] = 0.f;
            const Isect is = intersect<true>(qr, o, d);
            const float density = qr[0].w;
            Segment sg;
            sg.dt = fmaxf(is.exit - is.enter, 0.f);
            sg.a = density * sg.dt;
            const bool hit = act && is.geo && sg.a > 0.f;
            f3 dne = {0.f, 0.f, 0.f}, dnx = {0.f, 0.f, 0.f};
            if (hit) {
                integrate(qr, o, d, is.enter, is.exit, sg);
                const float m1 = density * (is.exit + is.enter) / 2.0f;
                const float logT_old = logT + sg.a;
                const float T = __expf(logT_old);
                D2 = D2 - density;
                D3 = D3 - m1;
                logT = logT_old;
                float nD2, nD3;
                dS_logT = hit_grads_planes(qr, xyz(qr[4]) - o, xyz(qr[5]) - o, d, is, sg, T, D2, D3, dS_c, dS_logT,
                                           dS_D, gl, dne, dnx, nD2, nD3);
                dS_D[2] = nD2;
                dS_D[3] = nD3;
            }
            if (__any_sync(0xffffffffu, hit))
                warp_sum_rows_planes(reinterpret_cast<float*>(S.red[warp]), gl, dne, dnx, hit ? is.ie : -1,
                                     hit ? is.ix : -1, lane, S.sacc[jj]);
        }
        __syncthreads();
        flush_entries<NT, B>(nk, S.srec[cb], S.sid[cb], S.sacc, indices, gverts, gcv);
        __syncthreads();
        if (!has_next) break;
        cb = nb;
        clo = nlo;
        ctop = ntop;
        cw0 = nw0;
        cw1 = nw1;
    }
}

// Pair backward item: the same strip / thread split as the forward.  Per
// batch of B entries (walked back to front) the pixels that still have list
// offsets below their n_contributors are compacted into slots and
//   A. all warps test the (entry, slot) pairs: a (0: no hit), m1 and
//      dot(dL/dcolour, rgb);
//   B. each owner walks its pixel's entries back to front and records, per
//      hit, T and D2, D3 of the state before the hit and dL/d(log T, D2, D3)
//      after it (the only state the adjoint reads; colour and D0, D1, D4 need
//      no undo);
//   C. all warps compute the 25 per-entry partials of every hit pair (warp =
//      entry, lanes = slots), sum them over the warp with a reduce-scatter and
//      add them to the entry's shared accumulator.
template <int PX, int B>
struct BwdPairSmem {
    float4 srec[B][kRecFloat4];
    int32_t sid[B];
    float sacc[B][kNGrad];
    float ray[6][PX];
    float dc[6][PX];      // dL/dcolour (3), dL/dD0, dL/dD1, dL/dD4: constant along the walk
    int32_t nc[PX];
    float resA[3][B][PX];  // a (0: no hit), m1, dot(dL/dcolour, rgb)
    float resB[6][B][PX];  // T, D2, D3 before the hit; dL/d(log T, D2, D3) after it
    uint8_t hit_entry[PX][B];  // per slot: the batch entries it hits
    int32_t hit_pre[PX + 1];   // exclusive prefix of the per-slot hit counts
    int32_t warp_base[(PX + 31) / 32];
    int32_t smax[(PX + 31) / 32];
};

template <int PX, int NT, int B>
__device__ __forceinline__ void bwd_pair_item(
    int tile, int sub, const int32_t* __restrict__ ids, const int2* __restrict__ ranges,
    const float4* __restrict__ recs, const int4* __restrict__ indices, const float2* __restrict__ jitter,
    const rm_camera& cam, const float4* __restrict__ img, const float* __restrict__ dist,
    const int32_t* __restrict__ ncs, const float4* __restrict__ gimg, const float* __restrict__ gdist,
    float* __restrict__ gverts, float* __restrict__ gcv, BwdPairSmem<PX, B>& S, const Queue& lq) {
    constexpr unsigned kOwnMask = WarpShape<PX>::kMask;
    constexpr int kWarps = NT / 32;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const bool owner = tid < PX;
    const int tx = tile % cam.grid_width, ty = tile / cam.grid_width;
    int lx, ly;
    strip_pixel<PX>(cam, sub, tid, lx, ly);
    const int px = tx * cam.tile_width + lx, py = ty * cam.tile_height + ly;
    const bool inside = owner && px < cam.image_width && py < cam.image_height;
    const int64_t pix = (int64_t)py * cam.image_width + px;
    f3 o = {0.f, 0.f, 0.f}, d = {0.f, 0.f, 1.f};
    float logT = 0.f, D2 = 0.f, D3 = 0.f;  // state along the reverse walk
    float dS_c[3] = {0.f, 0.f, 0.f}, dS_logT = 0.f, dS_D[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
    int32_t nc = 0;
    if (inside) {
        const float2 j = __ldg(jitter + pix);
        make_ray(cam, px, py, j.x, j.y, o, d);
        logT = __ldg(img + pix).w;
        D2 = __ldg(dist + 5 * pix + 2);
        D3 = __ldg(dist + 5 * pix + 3);
        const float4 g = __ldg(gimg + pix);
        dS_c[0] = g.x; dS_c[1] = g.y; dS_c[2] = g.z; dS_logT = g.w;
#pragma unroll
        for (int k = 0; k < 5; ++k) dS_D[k] = gdist ? __ldg(gdist + 5 * pix + k) : 0.f;
        nc = __ldg(ncs + pix);
    }
    if (owner) {
        int32_t m = nc;
#pragma unroll
        for (int off = WarpShape<PX>::kTopOffset; off > 0; off >>= 1) m = max(m, __shfl_xor_sync(kOwnMask, m, off));
        if (lane == 0) S.smax[warp] = m;
    }
    __syncthreads();
    int32_t tile_max = 0;
#pragma unroll
    for (int w = 0; w < (PX + 31) / 32; ++w) tile_max = max(tile_max, S.smax[w]);
    const int2 rg = __ldg(ranges + tile);
    const int end = min(rg.y, rg.x + tile_max);
    for (int top = end; top > rg.x; top -= B) {
        const int lo = max(rg.x, top - B);
        const int n = top - lo;
        // pixels with list offsets below n_contributors in this batch
        const bool walking = inside && (lo - rg.x) < nc;
        __syncthreads();  // the previous batch's flush has read sid / srec / sacc
        for (int k = tid; k < n; k += NT) S.sid[k] = list_id(ids, lo + k, lq);
        for (int k = tid; k < n * kNGrad; k += NT) (&S.sacc[0][0])[k] = 0.f;
        int slot = 0;
        if (owner) {
            const unsigned bal = __ballot_sync(kOwnMask, walking);
            if (lane == 0) S.warp_base[warp] = __popc(bal);
            slot = __popc(bal & ((1u << lane) - 1u));
        }
        __syncthreads();
        for (int k = tid; k < n * kRecFloat4; k += NT) {
            const int j = k >> 3, c = k & 7;
            S.srec[j][c] = record_part(recs, S.sid[j], c);
        }
        int k_act = 0;
#pragma unroll
        for (int w = 0; w < (PX + 31) / 32; ++w) k_act += S.warp_base[w];
        if (walking) {
            for (int w = 0; w < warp; ++w) slot += S.warp_base[w];
            S.ray[0][slot] = o.x; S.ray[1][slot] = o.y; S.ray[2][slot] = o.z;
            S.ray[3][slot] = d.x; S.ray[4][slot] = d.y; S.ray[5][slot] = d.z;
            S.dc[0][slot] = dS_c[0]; S.dc[1][slot] = dS_c[1]; S.dc[2][slot] = dS_c[2];
            S.dc[3][slot] = dS_D[0]; S.dc[4][slot] = dS_D[1]; S.dc[5][slot] = dS_D[4];
            S.nc[slot] = nc;
        }
        __syncthreads();
        // A: hit test of every (entry, slot) pair
        for (int j = warp; j < n; j += kWarps) {
            const float4* q = S.srec[j];
            const float density = q[0].w;
            for (int sl = lane; sl < k_act; sl += 32) {
                float ra = 0.f, rm1 = 0.f, rdt = 0.f;
                if (lo + j - rg.x < S.nc[sl]) {
                    const f3 ro = {S.ray[0][sl], S.ray[1][sl], S.ray[2][sl]};
                    const f3 rd = {S.ray[3][sl], S.ray[4][sl], S.ray[5][sl]};
                    const Isect is = intersect<false>(q, ro, rd);
                    Segment s;
                    s.dt = fmaxf(is.exit - is.enter, 0.f);
                    s.a = density * s.dt;
                    if (is.geo && s.a > 0.f) {
                        integrate(q, ro, rd, is.enter, is.exit, s);
                        ra = s.a;
                        rm1 = density * (is.exit + is.enter) / 2.0f;
                        rdt = fmaf(S.dc[2][sl], s.rgb[2], fmaf(S.dc[1][sl], s.rgb[1], S.dc[0][sl] * s.rgb[0]));
                    }
                }
                S.resA[0][j][sl] = ra;
                S.resA[1][j][sl] = rm1;
                S.resA[2][j][sl] = rdt;
            }
        }
        __syncthreads();
        // B: each owner walks its chains back to front and lists its hits
        if (walking) {
            int cnt = 0;
            for (int j = n - 1; j >= 0; --j) {
                const float a = S.resA[0][j][slot];
                if (!(a > 0.f)) continue;
                S.hit_entry[slot][cnt++] = (uint8_t)j;
                const float density = S.srec[j][0].w;
                const float m1 = S.resA[1][j][slot];
                const float logT_old = logT + a;
                const float T = __expf(logT_old);
                D2 = D2 - density;
                D3 = D3 - m1;
                logT = logT_old;
                S.resB[0][j][slot] = T;
                S.resB[1][j][slot] = D2;
                S.resB[2][j][slot] = D3;
                S.resB[3][j][slot] = dS_logT;
                S.resB[4][j][slot] = dS_D[2];
                S.resB[5][j][slot] = dS_D[3];
                dS_logT = dS_logT + S.resA[2][j][slot] * T;
                dS_D[2] = dS_D[2] + dS_D[0] * 2.0f * m1;
                dS_D[3] = dS_D[3] + dS_D[1] * 2.0f * density;
            }
            S.hit_pre[slot + 1] = cnt;
        }
        __syncthreads();
        // exclusive prefix of the hit counts over the k_act slots
        if (warp == 0) {
            int carry = 0;
            for (int s0 = 0; s0 < k_act; s0 += 32) {
                const int v = (s0 + lane < k_act) ? S.hit_pre[s0 + lane + 1] : 0;
                int inc = v;
#pragma unroll
                for (int o2 = 1; o2 < 32; o2 <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, inc, o2);
                    if (lane >= o2) inc += y;
                }
                if (s0 + lane < k_act) S.hit_pre[s0 + lane + 1] = carry + inc;
                carry += __shfl_sync(0xffffffffu, inc, 31);
            }
            if (lane == 0) S.hit_pre[0] = 0;
        }
        __syncthreads();
        // C: adjoint of every hit, one hit per thread (the hits are packed, so
        // all lanes do useful work); consecutive hits belong to one slot and
        // hit different entries, so the per-entry shared accumulators see no
        // address conflicts inside a warp
        const int n_hits = S.hit_pre[k_act];
        for (int h = tid; h < n_hits; h += NT) {
            int lo_s = 0, hi_s = k_act - 1;
            while (lo_s < hi_s) {  // last slot with hit_pre[slot] <= h
                const int mid = (lo_s + hi_s + 1) >> 1;
                if (S.hit_pre[mid] <= h) lo_s = mid; else hi_s = mid - 1;
            }
            const int sl = lo_s;
            const int j = S.hit_entry[sl][h - S.hit_pre[sl]];
            const float4* q = S.srec[j];
            const f3 ro = {S.ray[0][sl], S.ray[1][sl], S.ray[2][sl]};
            const f3 rd = {S.ray[3][sl], S.ray[4][sl], S.ray[5][sl]};
            const Isect is = intersect<true>(q, ro, rd);
            Segment sg;
            sg.dt = fmaxf(is.exit - is.enter, 0.f);
            sg.a = q[0].w * sg.dt;
            integrate(q, ro, rd, is.enter, is.exit, sg);
            const float dsc[3] = {S.dc[0][sl], S.dc[1][sl], S.dc[2][sl]};
            const float dsd[5] = {S.dc[3][sl], S.dc[4][sl], S.resB[4][j][sl], S.resB[5][j][sl], S.dc[5][sl]};
            float gl[kNGrad];
            float nD2, nD3;
            hit_grads(q, ro, rd, is, sg, S.resB[0][j][sl], S.resB[1][j][sl], S.resB[2][j][sl], dsc, S.resB[3][j][sl],
                      dsd, gl, nD2, nD3);
#pragma unroll
            for (int k = 0; k < kNGrad; ++k)
                if (gl[k] != 0.f) atomicAdd(&S.sacc[j][k], gl[k]);
        }
        __syncthreads();
        flush_entries<NT, B>(n, S.srec, S.sid, S.sacc, indices, gverts, gcv);
    }
}

// Resident CTAs per SM (of 64 threads) the dense backward is compiled for.
#ifndef RM_BWD_DENSE_MINB
#define RM_BWD_DENSE_MINB 8
#endif

template <int NT, int B, class V>
__global__ void __launch_bounds__(NT, (NT >= 64 ? RM_BWD_DENSE_MINB * 64 / NT : 16)) blend_bwd_dense_kernel(
    const int32_t* __restrict__ ids, const int2* __restrict__ ranges, const float4* __restrict__ recs,
    const int4* __restrict__ indices, const float2* __restrict__ jitter, const __grid_constant__ V views,
    const float4* __restrict__ img, const float* __restrict__ dist, const int32_t* __restrict__ ncs,
    const float4* __restrict__ gimg, const float* __restrict__ gdist, float* __restrict__ gverts,
    float* __restrict__ gcv, const Queue q) {
    __shared__ BwdDenseSmem<NT, B> S;
    __shared__ int s_item;
    const int n_items = queue_items(q);
    const HitMasks hm = live_masks(q.hm);
    for (;;) {
        const int item = next_item(q, &s_item);
        if (item >= n_items) return;
        const int t = queue_tile(q, item), v = views.find(t);
        const int tb = views.tile_base(v);
        const int64_t pb = views.pixel_base(v);
        bwd_dense_item<NT, B>(t - tb, item % q.subs, ids, ranges + tb, recs, indices, jitter + pb, views.camera(v),
                              img + pb, dist + 5 * pb, ncs + pb, gimg + pb, gdist ? gdist + 5 * pb : nullptr,
                              gverts, gcv, S, hm, q.subs, t, q);
    }
}

template <int B, class V>
__global__ void __launch_bounds__(64, 8) blend_bwd_dense_tma_kernel(
    const int32_t* __restrict__ ids, const int2* __restrict__ ranges, const float4* __restrict__ recs,
    const int4* __restrict__ indices, const float2* __restrict__ jitter, const __grid_constant__ V views,
    const float4* __restrict__ img, const float* __restrict__ dist, const int32_t* __restrict__ ncs,
    const float4* __restrict__ gimg, const float* __restrict__ gdist, float* __restrict__ gverts,
    float* __restrict__ gcv, const Queue q) {
    __shared__ BwdTmaSmem<B> S;
    __shared__ int s_item;
    if (threadIdx.x == 0) {
        mbar_init(&S.bar[0], 1);
        mbar_init(&S.bar[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    const int n_items = queue_items(q);
    const HitMasks hm = live_masks(q.hm);
    TmaPipe pipe = {0u, 0u};
    for (;;) {
        const int item = next_item(q, &s_item);
        if (item >= n_items) return;
        const int t = queue_tile(q, item), v = views.find(t);
        const int tb = views.tile_base(v);
        const int64_t pb = views.pixel_base(v);
        bwd_dense_item_tma<B>(t - tb, item % q.subs, ids, ranges + tb, recs, indices, jitter + pb,
                              views.camera(v), img + pb, dist + 5 * pb, ncs + pb, gimg + pb,
                              gdist ? gdist + 5 * pb : nullptr, gverts, gcv, S, hm, q.subs, t, pipe, q);
    }
}

template <int PX, int NT, int B, class V>
__global__ void __launch_bounds__(NT, 512 / NT) blend_bwd_pair_kernel(
    const int32_t* __restrict__ ids, const int2* __restrict__ ranges, const float4* __restrict__ recs,
    const int4* __restrict__ indices, const float2* __restrict__ jitter, const __grid_constant__ V views,
    const float4* __restrict__ img, const float* __restrict__ dist, const int32_t* __restrict__ ncs,
    const float4* __restrict__ gimg, const float* __restrict__ gdist, float* __restrict__ gverts,
    float* __restrict__ gcv, const Queue q) {
    extern __shared__ __align__(16) unsigned char bwd_smem_raw[];
    BwdPairSmem<PX, B>& S = *reinterpret_cast<BwdPairSmem<PX, B>*>(bwd_smem_raw);
    __shared__ int s_item;
    const int n_items = queue_items(q);
    for (;;) {
        const int item = next_item(q, &s_item);
        if (item >= n_items) return;
        const int t = queue_tile(q, item), v = views.find(t);
        const int tb = views.tile_base(v);
        const int64_t pb = views.pixel_base(v);
        bwd_pair_item<PX, NT, B>(t - tb, item % q.subs, ids, ranges + tb, recs, indices, jitter + pb,
                                 views.camera(v), img + pb, dist + 5 * pb, ncs + pb, gimg + pb,
                                 gdist ? gdist + 5 * pb : nullptr, gverts, gcv, S, q);
    }
}

// ------------------------------------------------------ per-tet statistics --
// calc_tet_err / kern_calc_tet_err (alphablend_shader_interp.slang:433-599):
// the forward walk from each pixel centre, accumulating per hit into
// tet_err[g, c] (float) the weight T = exp(log T) * a and its products with
// the pixel's error, squared error and SSIM error, the entry / exit points
// and the midpoint of the segment, and into tet_count[g] the hit count and
// the maximum of int(65535 * T).  As in the reference the walk starts from
// log T = 1 (its kern_calc_tet_err initialises the state alpha with 1) and
// stops once log T < -5.5.  Sums are formed per list entry across a work
// item (warp reduce-scatter, shared atomics) before one global atomic per
// (item, entry, column), instead of 16 atomics per (pixel, hit).
constexpr int kErrVals = 14;
__constant__ int kErrCol[kErrVals] = {0, 1, 2, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15};

template <int B>
struct ErrSmem {
    float4 srec[B][kRecFloat4];
    int32_t sid[B];
    float sacc[B][kErrVals];
    int32_t scount[B];
    int32_t smax[B];
};

template <int NT, int B>
__device__ __forceinline__ void err_item(int tile, int sub, const int32_t* __restrict__ ids,
                                         const int2* __restrict__ ranges, const float4* __restrict__ recs,
                                         const rm_camera& cam, const float* __restrict__ pixel_err,
                                         const float* __restrict__ ssim_err, float* __restrict__ tet_err,
                                         int32_t* __restrict__ tet_count, ErrSmem<B>& S, const Queue& lq) {
    constexpr unsigned kMask = WarpShape<NT>::kMask;
    const int tx = tile % cam.grid_width, ty = tile / cam.grid_width;
    int lx, ly;
    strip_pixel<NT>(cam, sub, (int)threadIdx.x, lx, ly);
    const int px = tx * cam.tile_width + lx, py = ty * cam.tile_height + ly;
    const bool inside = px < cam.image_width && py < cam.image_height;
    const int64_t pix = (int64_t)py * cam.image_width + px;
    const int lane = threadIdx.x & 31;
    f3 o = {0.f, 0.f, 0.f}, d = {0.f, 0.f, 1.f};
    float err = 0.f, serr = 0.f;
    if (inside) {
        make_ray(cam, px, py, 0.5f, 0.5f, o, d);  // pixel centre
        err = __ldg(pixel_err + pix);
        serr = __ldg(ssim_err + pix);
    }
    float logT = 1.0f;
    bool active = inside;
    const int2 rg = __ldg(ranges + tile);
    for (int base = rg.x; base < rg.y && __syncthreads_or(active); base += B) {
        const int n = min(B, rg.y - base);
        for (int k = threadIdx.x; k < n; k += NT) {
            S.sid[k] = list_id(ids, base + k, lq);
            S.scount[k] = 0;
            S.smax[k] = 0;
        }
        for (int k = threadIdx.x; k < n * kErrVals; k += NT) (&S.sacc[0][0])[k] = 0.f;
        __syncthreads();
        for (int k = threadIdx.x; k < n * kRecFloat4; k += NT) {
            const int j = k >> 3, c = k & 7;
            S.srec[j][c] = record_part(recs, S.sid[j], c);
        }
        __syncthreads();
        for (int j = 0; j < n; ++j) {
            if (!__any_sync(kMask, active)) break;
            const float4* q = S.srec[j];
            const Isect is = intersect<false>(q, o, d);
            const float dt = fmaxf(is.exit - is.enter, 0.f);
            const float a = q[0].w * dt;
            const bool hit = active && is.geo && a > 0.f;
            float v[kErrVals];
#pragma unroll
            for (int k = 0; k < kErrVals; ++k) v[k] = 0.f;
            int tint = 0;
            if (hit) {
                const float T = expf(logT) * a;
                const float mid = 0.5f * (is.enter + is.exit);
                v[0] = T;
                v[1] = T * err;
                v[2] = T * err * err;
                v[3] = T * serr;
                v[4] = T * fmaf(is.enter, d.x, o.x);
                v[5] = T * fmaf(is.enter, d.y, o.y);
                v[6] = T * fmaf(is.enter, d.z, o.z);
                v[7] = T * fmaf(is.exit, d.x, o.x);
                v[8] = T * fmaf(is.exit, d.y, o.y);
                v[9] = T * fmaf(is.exit, d.z, o.z);
                v[10] = T;
                v[11] = T * fmaf(mid, d.x, o.x);
                v[12] = T * fmaf(mid, d.y, o.y);
                v[13] = T * fmaf(mid, d.z, o.z);
                tint = __float2int_rz(65535.0f * T);
                logT = logT - a;
                if (logT < kTermLogT) active = false;
            }
            if (__any_sync(kMask, hit)) {
                using RS = ReduceScatter<kErrVals, WarpShape<NT>::kTopOffset>;
                int slot = 0;
                RS::template run<kMask>(v, lane, slot);
#pragma unroll
                for (int r = 0; r < RS::R; ++r)
                    if (slot + r < kErrVals && v[r] != 0.f) atomicAdd(&S.sacc[j][slot + r], v[r]);
                const unsigned bal = __ballot_sync(kMask, hit);
#pragma unroll
                for (int off = WarpShape<NT>::kTopOffset; off > 0; off >>= 1)
                    tint = max(tint, __shfl_xor_sync(kMask, tint, off));
                if (lane == 0) {
                    atomicAdd(&S.scount[j], __popc(bal));
                    atomicMax(&S.smax[j], tint);
                }
            }
        }
        __syncthreads();
        for (int jj = threadIdx.x; jj < n; jj += NT) {
            const int cnt = S.scount[jj];
            const int64_t g = S.sid[jj];
            if (cnt == 0 || g < 0) continue;
            float* te = tet_err + 16 * g;
#pragma unroll
            for (int k = 0; k < kErrVals; ++k)
                if (S.sacc[jj][k] != 0.f) atomicAdd(te + kErrCol[k], S.sacc[jj][k]);
            atomicAdd(tet_count + 2 * g, cnt);
            atomicMax(tet_count + 2 * g + 1, S.smax[jj]);
        }
    }
}

template <int NT, int B>
__global__ void __launch_bounds__(NT, (NT >= 64 ? 1024 / NT : 32)) err_kernel(
    const int32_t* __restrict__ ids, const int2* __restrict__ ranges, const float4* __restrict__ recs,
    const rm_camera cam, const float* __restrict__ pixel_err, const float* __restrict__ ssim_err,
    float* __restrict__ tet_err, int32_t* __restrict__ tet_count, const Queue q) {
    __shared__ ErrSmem<B> S;
    __shared__ int s_item;
    const int n_items = queue_items(q);
    for (;;) {
        const int item = next_item(q, &s_item);
        if (item >= n_items) return;
        err_item<NT, B>(queue_tile(q, item), item % q.subs, ids, ranges, recs, cam, pixel_err, ssim_err, tet_err,
                        tet_count, S, q);
    }
}

struct BlendWs {
    float4* recs;
    int32_t* order;
    int32_t* info;
    uint32_t* tickets;
    uint32_t* status;       // the pass's status word when the caller passes none

    uint32_t* mask_header;  // nullptr: the workspace has no room for hit masks
    uint32_t* mask_words;
    int64_t mask_cap;
};

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

// Byte offset of the status word inside the 256-byte header that follows the
// records and the tile order (info at 0, queue tickets at 64).
constexpr size_t kBlendStatusOff = 128;

size_t blend_ws_bytes(int64_t n_tets, int64_t n_tiles) {
    const size_t rec = align256((size_t)(n_tets > 0 ? n_tets : 1) * kRecFloat4 * sizeof(float4));
    const size_t ord = align256((size_t)(n_tiles > 0 ? n_tiles : 1) * sizeof(int32_t));
    return rec + ord + 256;
}

// Hit masks, when the caller's workspace is larger than blend_ws_bytes: a
// 256-byte header, then the mask words (mask_word).
BlendWs blend_ws(void* base, int64_t n_tets, int64_t n_tiles, size_t workspace_bytes) {
    char* p = (char*)base;
    const size_t rec = align256((size_t)(n_tets > 0 ? n_tets : 1) * kRecFloat4 * sizeof(float4));
    const size_t ord = align256((size_t)(n_tiles > 0 ? n_tiles : 1) * sizeof(int32_t));
    BlendWs w = {(float4*)p, (int32_t*)(p + rec), (int32_t*)(p + rec + ord), (uint32_t*)(p + rec + ord + 64),
                 (uint32_t*)(p + rec + ord + kBlendStatusOff), nullptr, nullptr, 0};
    const size_t end = rec + ord + 256;
    if (workspace_bytes >= end + 256 + 64 * sizeof(uint32_t)) {
        w.mask_header = (uint32_t*)(p + end);
        w.mask_words = (uint32_t*)(p + end + 256);
        w.mask_cap = (int64_t)((workspace_bytes - end - 256) / sizeof(uint32_t));
    }
    return w;
}

// Persistent grid: as many CTAs as fit on the device at once (cached per
// kernel instantiation and device).
// Resident CTAs of a persistent kernel on the current device (SMs x CTAs per
// SM), cached per (kernel, device, block shape): kernels of one signature
// differ in their resource use, so the kernel's address is part of the key.
struct GridKey {
    const void* kernel;
    int dev, threads, smem, blocks;
};
std::mutex g_grid_mu;
GridKey g_grid_cache[64];
int g_grid_used = 0;

template <typename K>
int persistent_grid(K kernel, int threads, int smem, int n_items) {
    int dev = 0;
    cudaGetDevice(&dev);
    const void* kp = (const void*)kernel;
    int blocks = -1;
    {
        std::lock_guard<std::mutex> lock(g_grid_mu);
        for (int i = 0; i < g_grid_used; ++i) {
            const GridKey& k = g_grid_cache[i];
            if (k.kernel == kp && k.dev == dev && k.threads == threads && k.smem == smem) blocks = k.blocks;
        }
    }
    if (blocks < 0) {
        int sms = 0, per_sm = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
        blocks = (sms > 0 ? sms : 1) * (per_sm > 0 ? per_sm : 1);
        std::lock_guard<std::mutex> lock(g_grid_mu);
        if (g_grid_used < 64) g_grid_cache[g_grid_used++] = {kp, dev, threads, smem, blocks};
    }
    return n_items < blocks ? n_items : blocks;
}

int sm_count() {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms > 0 ? sms : 1;
}

// When a pass splits its tiles between the two kernels, the pair kernel runs
// on a side stream forked from and joined back into the caller's stream with
// events (capturable in a CUDA graph).  Each (device, caller stream) gets its
// own side stream, so callers on different streams stay independent.
struct SideStream {
    int dev = -1;
    cudaStream_t caller = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
};
constexpr int kSideStreams = 64;
std::mutex g_side_mu;
SideStream g_side[kSideStreams];

// Caller holds g_side_mu.
int side_stream(cudaStream_t caller, SideStream** out) {
    int dev = 0;
    cudaGetDevice(&dev);
    SideStream* free_slot = nullptr;
    for (SideStream& e : g_side) {
        if (e.stream && e.dev == dev && e.caller == caller) {
            *out = &e;
            return RM_OK;
        }
        if (!e.stream && !free_slot) free_slot = &e;
    }
    if (!free_slot) {  // table full: share the first side stream of this device
        for (SideStream& e : g_side)
            if (e.dev == dev) {
                *out = &e;
                return RM_OK;
            }
        return rm_host::fail(RM_ECUDA, "rm_blend: no side stream slot left");
    }
    SideStream& e = *free_slot;
    if (cudaStreamCreateWithFlags(&e.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&e.fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&e.join, cudaEventDisableTiming) != cudaSuccess)
        return rm_host::fail(RM_ECUDA, "rm_blend: side stream: %s", cudaGetErrorString(cudaGetLastError()));
    e.dev = dev;
    e.caller = caller;
    *out = &e;
    return RM_OK;
}

int launch_order(const int32_t* ranges, int G, const BlendWs& w, int heavy_shift, cudaStream_t s,
                 uint32_t* mask_header = nullptr, uint32_t mask_state = 0u) {
    order_kernel<<<1, 1024, 0, s>>>((const int2*)ranges, G, w.order, w.info, w.tickets, heavy_shift, mask_header,
                                    mask_state);
    return rm_host::check_launch("rm_blend order");
}

int fork_side(cudaStream_t s, SideStream* side) {
    if (cudaEventRecord(side->fork, s) != cudaSuccess || cudaStreamWaitEvent(side->stream, side->fork, 0) != cudaSuccess)
        return rm_host::fail(RM_ECUDA, "rm_blend: fork: %s", cudaGetErrorString(cudaGetLastError()));
    return RM_OK;
}

int join_side(cudaStream_t s, SideStream* side) {
    if (cudaEventRecord(side->join, side->stream) != cudaSuccess || cudaStreamWaitEvent(s, side->join, 0) != cudaSuccess)
        return rm_host::fail(RM_ECUDA, "rm_blend: join: %s", cudaGetErrorString(cudaGetLastError()));
    return RM_OK;
}

// Launch tunables carried in the flags word (include/rm_capi.h).
struct Tuning {
    int heavy_shift;       // heavy tiles: list-length bucket >= bucket(mean) + heavy_shift; 1: all tiles
    int pair_ctas_per_sm;  // resident CTAs of the pair kernel per SM
    bool hit_masks;        // RM_BLEND_HIT_MASKS
    bool tma;              // RM_BLEND_STAGE_TMA
    uint32_t* status;      // where a staging wait that gives up is reported
    int64_t n_recs;        // records the list ids may name
};

Tuning tuning_from_flags(int flags, int def_shift, int def_ctas) {
    Tuning t;
    t.tma = (flags & RM_BLEND_STAGE_TMA) != 0;
    t.status = nullptr;
    t.n_recs = 0;
    const int hs = (flags >> RM_BLEND_HEAVY_SHIFT) & 0xf;
    const int pc = (flags >> RM_BLEND_PAIR_CTAS_SHIFT) & 0xf;
    t.heavy_shift = hs ? hs : def_shift;
    t.pair_ctas_per_sm = pc ? pc : def_ctas;
    t.hit_masks = (flags & RM_BLEND_HIT_MASKS) != 0;
    return t;
}

// Shape of one blend launch: G global tiles of tile_px pixels each.
struct Shape {
    int G;
    int tile_px;
};

// Forward pass: order kernel, then the pair kernel (heavy tiles) and the
// dense kernel (other tiles).  When every tile is heavy the pair kernel runs
// alone on the caller's stream; otherwise it runs on the side stream
// concurrently with the dense kernel and is joined back after both launches.
template <int PX, int B_DENSE, int PX_PAIR, int NT_PAIR, int B_PAIR, class V>
int launch_fwd(const int32_t* ids, const int32_t* ranges, const BlendWs& w, const float* jitter, const V& views,
               const Shape& sh, float* img, float* dist, int32_t* nc, const Tuning& tn, cudaStream_t s) {
    const int G = sh.G;
    // hit masks need 64-pixel items in both kernels; the header records whether
    // this forward wrote them, so a backward never reads stale masks
    const bool masks = tn.hit_masks && PX == 64 && PX_PAIR == 64 && w.mask_header;
    int rc = launch_order(ranges, G, w, tn.heavy_shift, s, w.mask_header, masks ? kMaskValid : 0u);
    if (rc) return rc;
    const int subs = sh.tile_px / PX;
    const int subs_pair = sh.tile_px / PX_PAIR;
    const HitMasks hm = {masks ? w.mask_words : nullptr, w.mask_cap, w.mask_header};
    const Queue qd = {w.order, w.info, w.tickets + 0, G, subs, false, hm, tn.status, rm_host::wait_limit(),
                      tn.n_recs};
    const Queue qp = {w.order, w.info, w.tickets + 1, G, subs_pair, true, hm, tn.status, rm_host::wait_limit(),
                      tn.n_recs};
    auto pair_kernel = tn.pair_ctas_per_sm * NT_PAIR >= 1024
                           ? blend_fwd_pair_kernel<PX_PAIR, NT_PAIR, B_PAIR, 1024 / NT_PAIR, V>
                           : blend_fwd_pair_kernel<PX_PAIR, NT_PAIR, B_PAIR, 768 / NT_PAIR, V>;
    const int smem = (int)sizeof(FwdPairSmem<PX_PAIR, B_PAIR>);
    cudaFuncSetAttribute(pair_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    const int pair_cap = tn.pair_ctas_per_sm * sm_count();
    const int pair_grid = G * subs_pair < pair_cap ? G * subs_pair : pair_cap;
    if (tn.heavy_shift == 1) {
        pair_kernel<<<pair_grid, NT_PAIR, smem, s>>>(ids, (const int2*)ranges, w.recs, (const float2*)jitter, views,
                                                     (float4*)img, dist, nc, qp);
        return rm_host::check_launch("rm_blend_fwd (pair)");
    }
    std::lock_guard<std::mutex> lock(g_side_mu);
    SideStream* side = nullptr;
    if ((rc = side_stream(s, &side)) || (rc = fork_side(s, side))) return rc;
    pair_kernel<<<pair_grid, NT_PAIR, smem, side->stream>>>(ids, (const int2*)ranges, w.recs, (const float2*)jitter,
                                                            views, (float4*)img, dist, nc, qp);
    if ((rc = rm_host::check_launch("rm_blend_fwd (pair)"))) return rc;
    auto dense_kernel = blend_fwd_dense_kernel<PX, B_DENSE, V>;
    const int grid = persistent_grid(dense_kernel, PX, 0, G * subs);
    dense_kernel<<<grid, PX, 0, s>>>(ids, (const int2*)ranges, w.recs, (const float2*)jitter, views, (float4*)img,
                                     dist, nc, qd);
    if ((rc = rm_host::check_launch("rm_blend_fwd (dense)"))) return rc;
    return join_side(s, side);
}

template <int PX, int B_DENSE, int PX_PAIR, int NT_PAIR, int B_PAIR, class V>
int launch_bwd(const int32_t* ids, const int32_t* ranges, const BlendWs& w, const int32_t* indices,
               const float* jitter, const V& views, const Shape& sh, const float* img, const float* dist,
               const int32_t* nc, const float* gimg, const float* gdist, float* gverts, float* gcv,
               const Tuning& tn, cudaStream_t s) {
    const int G = sh.G;
    int rc = launch_order(ranges, G, w, tn.heavy_shift, s);
    if (rc) return rc;
    const int subs = sh.tile_px / PX;
    const int subs_pair = sh.tile_px / PX_PAIR;
    const bool masks = tn.hit_masks && PX == 64 && w.mask_header;
    const HitMasks hm = {masks ? w.mask_words : nullptr, w.mask_cap, w.mask_header};
    const Queue qd = {w.order, w.info, w.tickets + 2, G, subs, false, hm, tn.status, rm_host::wait_limit(),
                      tn.n_recs};
    const Queue qp = {w.order, w.info, w.tickets + 3, G, subs_pair, true, HitMasks{nullptr, 0, nullptr},
                      tn.status, rm_host::wait_limit(), tn.n_recs};
    auto pair_kernel = blend_bwd_pair_kernel<PX_PAIR, NT_PAIR, B_PAIR, V>;
    const int smem = (int)sizeof(BwdPairSmem<PX_PAIR, B_PAIR>);
    cudaFuncSetAttribute(pair_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    const int pair_cap = tn.pair_ctas_per_sm * sm_count();
    const int pair_grid = G * subs_pair < pair_cap ? G * subs_pair : pair_cap;
    if (tn.heavy_shift == 1) {
        pair_kernel<<<pair_grid, NT_PAIR, smem, s>>>(ids, (const int2*)ranges, w.recs, (const int4*)indices,
                                                     (const float2*)jitter, views, (const float4*)img, dist, nc,
                                                     (const float4*)gimg, gdist, gverts, gcv, qp);
        return rm_host::check_launch("rm_blend_bwd (pair)");
    }
    std::lock_guard<std::mutex> lock(g_side_mu);
    SideStream* side = nullptr;
    if ((rc = side_stream(s, &side)) || (rc = fork_side(s, side))) return rc;
    pair_kernel<<<pair_grid, NT_PAIR, smem, side->stream>>>(ids, (const int2*)ranges, w.recs, (const int4*)indices,
                                                            (const float2*)jitter, views, (const float4*)img, dist,
                                                            nc, (const float4*)gimg, gdist, gverts, gcv, qp);
    if ((rc = rm_host::check_launch("rm_blend_bwd (pair)"))) return rc;
    if (PX == 64 && tn.tma) {  // records staged by bulk copies, two batches in flight
        auto tma_kernel = blend_bwd_dense_tma_kernel<B_DENSE, V>;
        const int grid = persistent_grid(tma_kernel, 64, 0, G * subs);
        tma_kernel<<<grid, 64, 0, s>>>(ids, (const int2*)ranges, w.recs, (const int4*)indices,
                                       (const float2*)jitter, views, (const float4*)img, dist, nc,
                                       (const float4*)gimg, gdist, gverts, gcv, qd);
        if ((rc = rm_host::check_launch("rm_blend_bwd (dense, bulk-copy staging)"))) return rc;
        return join_side(s, side);
    }
    auto dense_kernel = blend_bwd_dense_kernel<PX, B_DENSE, V>;
    const int grid = persistent_grid(dense_kernel, PX, 0, G * subs);
    dense_kernel<<<grid, PX, 0, s>>>(ids, (const int2*)ranges, w.recs, (const int4*)indices, (const float2*)jitter,
                                     views, (const float4*)img, dist, nc, (const float4*)gimg, gdist, gverts, gcv, qd);
    if ((rc = rm_host::check_launch("rm_blend_bwd (dense)"))) return rc;
    return join_side(s, side);
}

// Strip of pixels handled by one CTA: flags may request 2^k pixels
// (RM_BLEND_STRIP_SHIFT); default 64.  Must divide the tile and be a multiple
// of the tile width.
int strip_pixels(const rm_camera* cam, int flags) {
    const int tile_px = cam->tile_width * cam->tile_height;
    const int req = (flags >> RM_BLEND_STRIP_SHIFT) & 0xff;
    int strip = req ? (1 << req) : 64;
    if (tile_px < strip) strip = tile_px;
    return strip;
}

// Tets per shared-memory batch: flags may request 2^k (RM_BLEND_BATCH_SHIFT).
int batch_size(int flags, int def) {
    const int req = (flags >> RM_BLEND_BATCH_SHIFT) & 0xf;
    return req ? (1 << req) : def;
}

int pack(const int32_t* indices, const float* vertices, int64_t n_verts, const float* cv, int64_t n_tets,
         const int32_t* tiles, float4* recs, cudaStream_t s) {
    const int threads = 256;
    const int64_t blocks = (n_tets + threads - 1) / threads;
    pack_kernel<<<(unsigned)blocks, threads, 0, s>>>((const int4*)indices, vertices, n_verts, cv, n_tets, tiles, recs);
    return rm_host::check_launch("rm_blend pack");
}

// Checks shared by all blend entry points; cam0 is the (first) camera, G the
// total tile count of the launch.
int check_blend_args(const char* who, const int32_t* indices, const float* vertices, const float* cv, int64_t n_tets,
                     const float* jitter, const rm_camera* cam0, int64_t G, void* workspace, size_t workspace_bytes,
                     int flags) {
    int rc = rm_host::check_cam(cam0);
    if (rc) return rc;
    if (n_tets < 0) return rm_host::fail(RM_EINVAL, "%s: negative size", who);
    if (!indices || !vertices || !cv || !jitter || !workspace)
        return rm_host::fail(RM_EINVAL, "%s: NULL pointer", who);
    if ((uintptr_t)indices & 15) return rm_host::fail(RM_EINVAL, "%s: indices must be 16-byte aligned", who);
    if ((uintptr_t)workspace & 15) return rm_host::fail(RM_EINVAL, "%s: workspace must be 16-byte aligned", who);
    if (workspace_bytes < blend_ws_bytes(n_tets, G))
        return rm_host::fail(RM_EINVAL, "%s: workspace %zu < %zu bytes", who, workspace_bytes,
                             blend_ws_bytes(n_tets, G));
    const int nt = cam0->tile_width * cam0->tile_height;
    if (nt != 16 && nt != 64 && nt != 256 && nt != 1024)
        return rm_host::fail(RM_EINVAL, "%s: tile of %d pixels unsupported (16, 64, 256 or 1024)", who, nt);
    const int strip = strip_pixels(cam0, flags);
    if ((strip != 16 && strip != 64) || nt % strip)
        return rm_host::fail(RM_EINVAL, "%s: strip of %d pixels does not fit a %dx%d tile", who, strip,
                             cam0->tile_width, cam0->tile_height);
    return RM_OK;
}

// The pass's status word: the caller's, else the workspace's own (cleared here).
int pass_status(const char* who, BlendWs& w, uint32_t* status_dev, cudaStream_t s, uint32_t** out) {
    if (status_dev) {
        *out = status_dev;
        return RM_OK;
    }
    cudaError_t e = cudaMemsetAsync(w.status, 0, sizeof(uint32_t), s);
    if (e != cudaSuccess) return rm_host::fail(RM_ECUDA, "%s: %s", who, cudaGetErrorString(e));
    *out = w.status;
    return RM_OK;
}

template <class V>
int blend_fwd_any(const char* who, const int32_t* sorted_ids, const int32_t* ranges, const int32_t* indices,
                  const float* vertices, const float* cell_values, int64_t n_tets, int64_t n_verts,
                  const int32_t* tiles_touched,
                  const float* ray_jitter, const rm_camera* cam0, const V& views, const Shape& sh, float* out_img,
                  float* out_distortion, int32_t* n_contrib, const void* records, void* workspace,
                  size_t workspace_bytes, int flags, uint32_t* status_dev, void* stream) {
    int rc = check_blend_args(who, indices, vertices, cell_values, records ? 0 : n_tets, ray_jitter, cam0, sh.G,
                              workspace, workspace_bytes, flags);
    if (rc) return rc;
    if (!ranges || !out_img || !out_distortion || !n_contrib) return rm_host::fail(RM_EINVAL, "%s: NULL pointer", who);
    if (((uintptr_t)out_img & 15) || ((uintptr_t)ranges & 7) || ((uintptr_t)ray_jitter & 7))
        return rm_host::fail(RM_EINVAL, "%s: misaligned image / ranges / jitter", who);
    cudaStream_t s = (cudaStream_t)stream;
    BlendWs w = blend_ws(workspace, records ? 0 : n_tets, sh.G, workspace_bytes);
    if (records) {
        if ((uintptr_t)records & 15) return rm_host::fail(RM_EINVAL, "%s: records must be 16-byte aligned", who);
        w.recs = (float4*)records;  // packed by rm_blend_pack_records
    } else if (!(flags & RM_BLEND_REUSE_RECORDS) && n_tets > 0) {
        rc = pack(indices, vertices, n_verts, cell_values, n_tets, tiles_touched, w.recs, s);
        if (rc) return rc;
    }
    // measured on the 1.3M-tet workload: every tile through the pair kernel, 4 CTAs/SM
    Tuning tn = tuning_from_flags(flags, 1, 4);
    tn.n_recs = n_tets;
    if ((rc = pass_status(who, w, status_dev, s, &tn.status))) return rc;
    // tets per shared-memory batch of the pair kernel: 16, 32 (default) or 64
    const int key = strip_pixels(cam0, flags) * 1000 + batch_size(flags, 32);
#define RM_FWD_CASE(PX, NT, BP)                                                                                  \
    case PX * 1000 + BP:                                                                                         \
        return launch_fwd<PX, 64, PX, NT, BP>(sorted_ids, ranges, w, ray_jitter, views, sh, out_img, out_distortion, \
                                              n_contrib, tn, s);
    switch (key) {
        RM_FWD_CASE(16, 64, 16)
        RM_FWD_CASE(16, 64, 32)
        RM_FWD_CASE(16, 64, 64)
        RM_FWD_CASE(64, 256, 16)
        RM_FWD_CASE(64, 256, 32)
        RM_FWD_CASE(64, 256, 64)
        default:
            return rm_host::fail(RM_EINVAL, "%s: tets per batch %d unsupported (16, 32 or 64)", who, key % 1000);
    }
#undef RM_FWD_CASE
}

template <class V>
int blend_bwd_any(const char* who, const int32_t* sorted_ids, const int32_t* ranges, const int32_t* indices,
                  const float* vertices, const float* cell_values, int64_t n_tets, int64_t n_verts,
                  const int32_t* tiles_touched,
                  const float* ray_jitter, const rm_camera* cam0, const V& views, const Shape& sh,
                  const float* out_img, const float* out_distortion, const int32_t* n_contrib, const float* grad_img,
                  const float* grad_distortion, float* grad_vertices, float* grad_cell_values, const void* records,
                  void* workspace, size_t workspace_bytes, int flags, uint32_t* status_dev, void* stream) {
    int rc = check_blend_args(who, indices, vertices, cell_values, records ? 0 : n_tets, ray_jitter, cam0, sh.G,
                              workspace, workspace_bytes, flags);
    if (rc) return rc;
    if (!ranges || !out_img || !out_distortion || !n_contrib || !grad_img || !grad_vertices || !grad_cell_values)
        return rm_host::fail(RM_EINVAL, "%s: NULL pointer", who);
    if (((uintptr_t)out_img & 15) || ((uintptr_t)grad_img & 15) || ((uintptr_t)ranges & 7) ||
        ((uintptr_t)ray_jitter & 7))
        return rm_host::fail(RM_EINVAL, "%s: misaligned image / grad / ranges / jitter", who);
    cudaStream_t s = (cudaStream_t)stream;
    BlendWs w = blend_ws(workspace, records ? 0 : n_tets, sh.G, workspace_bytes);
    if (records) {
        if ((uintptr_t)records & 15) return rm_host::fail(RM_EINVAL, "%s: records must be 16-byte aligned", who);
        w.recs = (float4*)records;  // packed by rm_blend_pack_records
    } else if (!(flags & RM_BLEND_REUSE_RECORDS) && n_tets > 0) {
        rc = pack(indices, vertices, n_verts, cell_values, n_tets, tiles_touched, w.recs, s);
        if (rc) return rc;
    }
    // measured: the one-thread-per-pixel backward alone is fastest
    Tuning tn = tuning_from_flags(flags, 15, 1);
    tn.n_recs = n_tets;
    if ((rc = pass_status(who, w, status_dev, s, &tn.status))) return rc;
    // tets per shared-memory batch of the dense kernel: 16, 32 or 64 (default)
    const int key = strip_pixels(cam0, flags) * 1000 + batch_size(flags, 64);
#define RM_BWD_CASE(PX, NT, BD)                                                                                  \
    case PX * 1000 + BD:                                                                                         \
        return launch_bwd<PX, BD, PX, NT, 16>(sorted_ids, ranges, w, indices, ray_jitter, views, sh, out_img,       \
                                              out_distortion, n_contrib, grad_img, grad_distortion, grad_vertices,  \
                                              grad_cell_values, tn, s);
    switch (key) {
        RM_BWD_CASE(16, 64, 16)
        RM_BWD_CASE(16, 64, 32)
        RM_BWD_CASE(16, 64, 64)
        RM_BWD_CASE(64, 256, 16)
        RM_BWD_CASE(64, 256, 32)
        RM_BWD_CASE(64, 256, 64)
        default:
            return rm_host::fail(RM_EINVAL, "%s: tets per batch %d unsupported (16, 32 or 64)", who, key % 1000);
    }
#undef RM_BWD_CASE
}

}  // namespace
}  // namespace rm

extern "C" {

size_t rm_blend_workspace_size(int64_t n_tets, int64_t n_tiles) { return rm::blend_ws_bytes(n_tets, n_tiles); }

size_t rm_blend_status_offset(int64_t n_tets, int64_t n_tiles) {
    return rm::blend_ws_bytes(n_tets, n_tiles) - 256 + rm::kBlendStatusOff;
}

size_t rm_blend_hit_mask_bytes(int64_t n_pairs, int64_t n_tiles, int tile_pixels) {
    const int64_t subs = tile_pixels > 64 ? tile_pixels / 64 : 1;
    const int64_t blocks = (n_pairs > 0 ? n_pairs : 0) / 32 + (n_tiles > 0 ? n_tiles : 0) + 2;
    return 256 + (size_t)blocks * (size_t)subs * 64 * sizeof(uint32_t);
}

int rm_calc_tet_err(const int32_t* sorted_ids, const int32_t* ranges, const int32_t* indices, const float* vertices,
                    const float* cell_values, int64_t n_tets, int64_t n_verts, const int32_t* tiles_touched,
                    const rm_camera* cam, const float* pixel_err, const float* ssim_err, float* tet_err,
                    int32_t* tet_count, void* workspace, size_t workspace_bytes, int flags, void* stream) {
    using namespace rm;
    int rc = rm_host::check_cam(cam);
    if (rc) return rc;
    const int64_t G = (int64_t)cam->grid_width * cam->grid_height;
    // the camera check of the blend calls; jitter is unused (pixel centres)
    rc = check_blend_args("rm_calc_tet_err", indices, vertices, cell_values, n_tets, pixel_err, cam, G, workspace,
                          workspace_bytes, flags);
    if (rc) return rc;
    if (!ranges || !ssim_err || !tet_err || !tet_count) return rm_host::fail(RM_EINVAL, "rm_calc_tet_err: NULL pointer");
    cudaStream_t s = (cudaStream_t)stream;
    const BlendWs w = blend_ws(workspace, n_tets, G, workspace_bytes);
    if (!(flags & RM_BLEND_REUSE_RECORDS) && n_tets > 0) {
        rc = pack(indices, vertices, n_verts, cell_values, n_tets, tiles_touched, w.recs, s);
        if (rc) return rc;
    }
    // every tile in one heavy-first queue (heavy_shift 1 marks all tiles heavy)
    if ((rc = launch_order(ranges, (int)G, w, 1, s))) return rc;
    const int strip = strip_pixels(cam, flags);
    const int subs = cam->tile_width * cam->tile_height / strip;
    const Queue qd = {w.order, w.info, w.tickets + 0, (int)G, subs, true, HitMasks{nullptr, 0, nullptr}, nullptr,
                      rm_host::wait_limit(), n_tets};
    if (strip == 16) {
        const int grid = persistent_grid(err_kernel<16, 32>, 16, 0, (int)G * subs);
        err_kernel<16, 32><<<grid, 16, 0, s>>>(sorted_ids, (const int2*)ranges, w.recs, *cam, pixel_err, ssim_err,
                                                tet_err, tet_count, qd);
    } else {
        const int grid = persistent_grid(err_kernel<64, 32>, 64, 0, (int)G * subs);
        err_kernel<64, 32><<<grid, 64, 0, s>>>(sorted_ids, (const int2*)ranges, w.recs, *cam, pixel_err, ssim_err,
                                                tet_err, tet_count, qd);
    }
    return rm_host::check_launch("rm_calc_tet_err");
}

size_t rm_blend_records_size(int64_t n_tets) {
    return (size_t)(n_tets > 0 ? n_tets : 0) * rm::kRecFloat4 * sizeof(float4);
}

int rm_blend_pack_records(const int32_t* indices, const float* vertices, const float* cell_values, int64_t n_tets,
                          int64_t n_verts, const int32_t* tiles_touched, void* records, void* stream) {
    if (n_tets < 0 || n_verts < 0) return rm_host::fail(RM_EINVAL, "rm_blend_pack_records: negative size");
    if (n_tets == 0) return RM_OK;
    if (!indices || !vertices || !cell_values || !records)
        return rm_host::fail(RM_EINVAL, "rm_blend_pack_records: NULL pointer");
    if (((uintptr_t)indices & 15) || ((uintptr_t)records & 15))
        return rm_host::fail(RM_EINVAL, "rm_blend_pack_records: indices and records must be 16-byte aligned");
    return rm::pack(indices, vertices, n_verts, cell_values, n_tets, tiles_touched, (float4*)records,
                    (cudaStream_t)stream);
}

int rm_blend_fwd(const int32_t* sorted_ids, const int32_t* ranges, const int32_t* indices, const float* vertices,
                 const float* cell_values, int64_t n_tets, int64_t n_verts, const int32_t* tiles_touched,
                 const float* ray_jitter, const rm_camera* cam, float* out_img, float* out_distortion,
                 int32_t* n_contrib, void* workspace, size_t workspace_bytes, int flags, uint32_t* status_dev,
                 void* stream) {
    int rc = rm_host::check_cam(cam);
    if (rc) return rc;
    const rm::OneView one = {*cam};
    const rm::Shape sh = {cam->grid_width * cam->grid_height, cam->tile_width * cam->tile_height};
    return rm::blend_fwd_any("rm_blend_fwd", sorted_ids, ranges, indices, vertices, cell_values, n_tets, n_verts,
                             tiles_touched, ray_jitter, cam, one, sh, out_img, out_distortion, n_contrib, nullptr,
                             workspace, workspace_bytes, flags, status_dev, stream);
}

int rm_blend_bwd(const int32_t* sorted_ids, const int32_t* ranges, const int32_t* indices, const float* vertices,
                 const float* cell_values, int64_t n_tets, int64_t n_verts, const int32_t* tiles_touched,
                 const float* ray_jitter, const rm_camera* cam, const float* out_img, const float* out_distortion,
                 const int32_t* n_contrib, const float* grad_img, const float* grad_distortion, float* grad_vertices,
                 float* grad_cell_values, void* workspace, size_t workspace_bytes, int flags, uint32_t* status_dev,
                 void* stream) {
    int rc = rm_host::check_cam(cam);
    if (rc) return rc;
    const rm::OneView one = {*cam};
    const rm::Shape sh = {cam->grid_width * cam->grid_height, cam->tile_width * cam->tile_height};
    return rm::blend_bwd_any("rm_blend_bwd", sorted_ids, ranges, indices, vertices, cell_values, n_tets, n_verts,
                             tiles_touched, ray_jitter, cam, one, sh, out_img, out_distortion, n_contrib, grad_img,
                             grad_distortion, grad_vertices, grad_cell_values, nullptr, workspace, workspace_bytes,
                             flags, status_dev, stream);
}

int rm_blend_fwd_multi(const int32_t* sorted_ids, const int32_t* ranges, const int32_t* indices,
                       const float* vertices, const float* cell_values, int64_t n_tets, int64_t n_verts,
                       const int32_t* tiles_touched, const float* ray_jitter, const rm_camera* cams, int n_views,
                       float* out_img, float* out_distortion, int32_t* n_contrib, const void* records,
                       void* workspace, size_t workspace_bytes, int flags, uint32_t* status_dev, void* stream) {
    rm::ViewSet views;
    int rc = rm_host::make_views("rm_blend_fwd_multi", cams, n_views, &views);
    if (rc) return rc;
    const rm::Shape sh = {views.tiles[n_views], cams[0].tile_width * cams[0].tile_height};
    return rm::blend_fwd_any("rm_blend_fwd_multi", sorted_ids, ranges, indices, vertices, cell_values, n_tets, n_verts,
                             tiles_touched, ray_jitter, cams, views, sh, out_img, out_distortion, n_contrib,
                             records, workspace, workspace_bytes, flags, status_dev, stream);
}

int rm_blend_bwd_multi(const int32_t* sorted_ids, const int32_t* ranges, const int32_t* indices,
                       const float* vertices, const float* cell_values, int64_t n_tets, int64_t n_verts,
                       const int32_t* tiles_touched, const float* ray_jitter, const rm_camera* cams, int n_views,
                       const float* out_img, const float* out_distortion, const int32_t* n_contrib,
                       const float* grad_img, const float* grad_distortion, float* grad_vertices,
                       float* grad_cell_values, const void* records, void* workspace, size_t workspace_bytes,
                       int flags, uint32_t* status_dev, void* stream) {
    rm::ViewSet views;
    int rc = rm_host::make_views("rm_blend_bwd_multi", cams, n_views, &views);
    if (rc) return rc;
    const rm::Shape sh = {views.tiles[n_views], cams[0].tile_width * cams[0].tile_height};
    return rm::blend_bwd_any("rm_blend_bwd_multi", sorted_ids, ranges, indices, vertices, cell_values, n_tets, n_verts,
                             tiles_touched, ray_jitter, cams, views, sh, out_img, out_distortion, n_contrib,
                             grad_img, grad_distortion, grad_vertices, grad_cell_values, records, workspace,
                             workspace_bytes, flags, status_dev, stream);
}

}  // extern "C"
