// rm_blend.cu - stage (d): front-to-back tile blend and its back-to-front
// adjoint.
//
// Forward: splat_tiled / alpha_blend (alphablend_shader_interp.slang:194-271,
// 371-431) with evaluate_tetra_interp and integrate_tetra_segment
// (interp_version.slang:21-98) and ray_tetrahedron_intersect_fused
// (intersect.slang:394-624).  One CTA per screen tile, one thread per pixel.
// The tile's sorted list is walked in batches: each batch's per-tet records
// (128 B, packed once per frame by pack_kernel) are gathered into shared
// memory, then every pixel tests its ray against them in list order.  A pixel
// stops at log T < -5.5; a warp whose pixels are all done skips the batch and
// the CTA leaves the list once every pixel is done.
//
// Backward: bwd_alpha_blend (alphablend_shader_interp.slang:273-369).  Each
// pixel walks its list back to front from the saved final state, skipping list
// offsets >= n_contributors, undoes each hit and back-propagates through the
// segment integral and the ray/plane intersection.  Per hit it produces 25
// partial derivatives (four face-normal gradients, direct v0/v1 gradients and
// the seven cell values); a warp reduce-scatter sums them across the 32 pixels
// of a warp, one shared-memory atomic per value accumulates the CTA's sum per
// list entry, and after each batch the sums are converted to vertex gradients
// and added to global memory with one atomic per (tile, tet, component).
#include "rm_internal.cuh"

namespace rm {
namespace {

constexpr float kTermLogT = -5.5f;  // alphablend_shader_interp.slang:257
constexpr int kNGrad = 25;

// ------------------------------------------------------------------ packing --
__global__ void __launch_bounds__(256) pack_kernel(const int4* __restrict__ indices, const float* __restrict__ verts,
                                                   const float* __restrict__ cv, int64_t n_tets,
                                                   const int32_t* __restrict__ tiles, float4* __restrict__ recs) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_tets) return;
    if (tiles && __ldg(tiles + g) <= 0) return;
    const int4 id = __ldg(indices + g);
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
__device__ __forceinline__ void integrate(const float4* __restrict__ q, f3 o, f3 d, float enter, float exit,
                                          Segment& s) {
    const float density = q[0].w;
    const f3 v0 = xyz(q[4]);
    const f3 grd = {q[4].w, q[5].w, q[6].w};
    s.ve = {fmaf(enter, d.x, o.x) - v0.x, fmaf(enter, d.y, o.y) - v0.y, fmaf(enter, d.z, o.z) - v0.z};
    s.vx = {fmaf(exit, d.x, o.x) - v0.x, fmaf(exit, d.y, o.y) - v0.y, fmaf(exit, d.z, o.z) - v0.z};
    s.ce = dot3(grd, s.ve);
    s.cx = dot3(grd, s.vx);
    s.x = s.dt * density;
    s.w = seg_weights(s.x);
    const float base[3] = {q[1].w, q[2].w, q[3].w};
#pragma unroll
    for (int k = 0; k < 3; ++k) s.rgb[k] = fmaf(s.w.w1, s.ce + base[k], s.w.w0 * (s.cx + base[k]));
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

template <int NT, int B>
__global__ void __launch_bounds__(NT) blend_fwd_kernel(const int32_t* __restrict__ ids,
                                                       const int2* __restrict__ ranges,
                                                       const float4* __restrict__ recs,
                                                       const float2* __restrict__ jitter, const rm_camera cam,
                                                       float4* __restrict__ out_img, float* __restrict__ out_dist,
                                                       int32_t* __restrict__ out_nc) {
    __shared__ float4 srec[B][kRecFloat4];
    __shared__ int32_t sid[B];
    const int tile = blockIdx.x;
    const int tx = tile % cam.grid_width, ty = tile / cam.grid_width;
    const int lx = threadIdx.x % cam.tile_width, ly = threadIdx.x / cam.tile_width;
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
    for (int base = rg.x; base < rg.y; base += B) {
        const int n = min(B, rg.y - base);
        __syncthreads();
        for (int k = threadIdx.x; k < n; k += NT) sid[k] = __ldg(ids + base + k);
        __syncthreads();
        for (int k = threadIdx.x; k < n * kRecFloat4; k += NT) {
            const int j = k >> 3, c = k & 7;
            srec[j][c] = __ldg(recs + (int64_t)kRecFloat4 * sid[j] + c);
        }
        __syncthreads();
        if (__any_sync(WarpShape<NT>::kMask, active)) {
            for (int j = 0; j < n; ++j) {
                if (!active) break;
                ++nc;
                const float4* q = srec[j];
                const Isect is = intersect<false>(q, o, d);
                Segment s;
                s.dt = fmaxf(is.exit - is.enter, 0.f);
                const float density = q[0].w;
                s.a = density * s.dt;
                if (is.geo && s.a > 0.f) {
                    integrate(q, o, d, is.enter, is.exit, s);
                    const float T = __expf(st.logT);
#pragma unroll
                    for (int k = 0; k < 3; ++k) st.c[k] = fmaf(s.rgb[k], T, st.c[k]);
                    st.logT = st.logT - s.a;
                    const float m0 = density;
                    const float m1 = density * (is.exit + is.enter) / 2.0f;
                    const float D2 = st.D[2], D3 = st.D[3];
                    st.D[0] = fmaf(2.0f * m1, D2, st.D[0]);
                    st.D[1] = fmaf(2.0f * m0, D3, st.D[1]);
                    st.D[2] = D2 + m0;
                    st.D[3] = D3 + m1;
                    st.D[4] = st.D[4] + density * density * s.dt / 3.0f;
                    if (st.logT < kTermLogT) active = false;
                }
            }
        }
        if (!__syncthreads_or(active)) break;
    }
    if (inside) {
        out_img[pix] = make_float4(st.c[0], st.c[1], st.c[2], st.logT);
        float* dd = out_dist + 5 * pix;
#pragma unroll
        for (int k = 0; k < 5; ++k) dd[k] = st.D[k];
        out_nc[pix] = nc;
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

template <int NT, int B>
__global__ void __launch_bounds__(NT) blend_bwd_kernel(
    const int32_t* __restrict__ ids, const int2* __restrict__ ranges, const float4* __restrict__ recs,
    const int4* __restrict__ indices, const float2* __restrict__ jitter, const rm_camera cam,
    const float4* __restrict__ img, const float* __restrict__ dist, const int32_t* __restrict__ ncs,
    const float4* __restrict__ gimg, const float* __restrict__ gdist, float* __restrict__ gverts,
    float* __restrict__ gcv) {
    __shared__ float4 srec[B][kRecFloat4];
    __shared__ int32_t sid[B];
    __shared__ float sacc[B][kNGrad];
    __shared__ int32_t smax[WarpShape<NT>::kWarps];
    constexpr unsigned kMask = WarpShape<NT>::kMask;
    const int tile = blockIdx.x;
    const int tx = tile % cam.grid_width, ty = tile / cam.grid_width;
    const int lx = threadIdx.x % cam.tile_width, ly = threadIdx.x / cam.tile_width;
    const int px = tx * cam.tile_width + lx, py = ty * cam.tile_height + ly;
    const bool inside = px < cam.image_width && py < cam.image_height;
    const int64_t pix = (int64_t)py * cam.image_width + px;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    f3 o = {0.f, 0.f, 0.f}, d = {0.f, 0.f, 1.f};
    PixelState st = {{0.f, 0.f, 0.f}, 0.f, {0.f, 0.f, 0.f, 0.f, 0.f}};
    PixelState dS = st;
    int32_t nc = 0;
    if (inside) {
        const float2 j = __ldg(jitter + pix);
        make_ray(cam, px, py, j.x, j.y, o, d);
        const float4 a = __ldg(img + pix);
        st.c[0] = a.x; st.c[1] = a.y; st.c[2] = a.z; st.logT = a.w;
        const float4 g = __ldg(gimg + pix);
        dS.c[0] = g.x; dS.c[1] = g.y; dS.c[2] = g.z; dS.logT = g.w;
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            st.D[k] = __ldg(dist + 5 * pix + k);
            dS.D[k] = gdist ? __ldg(gdist + 5 * pix + k) : 0.f;
        }
        nc = __ldg(ncs + pix);
    }
    int32_t m = nc;
#pragma unroll
    for (int off = WarpShape<NT>::kTopOffset; off > 0; off >>= 1) m = max(m, __shfl_xor_sync(kMask, m, off));
    if (lane == 0) smax[warp] = m;
    __syncthreads();
    int32_t tile_max = 0;
#pragma unroll
    for (int w = 0; w < WarpShape<NT>::kWarps; ++w) tile_max = max(tile_max, smax[w]);
    const int2 rg = __ldg(ranges + tile);
    const int end = min(rg.y, rg.x + tile_max);
    for (int top = end; top > rg.x; top -= B) {
        const int lo = max(rg.x, top - B);
        const int n = top - lo;
        __syncthreads();
        for (int k = threadIdx.x; k < n; k += NT) sid[k] = __ldg(ids + lo + k);
        for (int k = threadIdx.x; k < n * kNGrad; k += NT) (&sacc[0][0])[k] = 0.f;
        __syncthreads();
        for (int k = threadIdx.x; k < n * kRecFloat4; k += NT) {
            const int j = k >> 3, c = k & 7;
            srec[j][c] = __ldg(recs + (int64_t)kRecFloat4 * sid[j] + c);
        }
        __syncthreads();
        for (int jj = n - 1; jj >= 0; --jj) {
            const int off = lo + jj - rg.x;
            const bool act = inside && off < nc;
            if (!__any_sync(kMask, act)) continue;
            const float4* q = srec[jj];
            float gl[kNGrad];
#pragma unroll
            for (int k = 0; k < kNGrad; ++k) gl[k] = 0.f;
            // ---- recompute the forward quantities of this entry
            const f3 a0 = xyz(q[4]) - o;
            const f3 a1 = xyz(q[5]) - o;
            const Isect is = intersect<true>(q, o, d);
            const float te = is.te, tx = is.tx, dene = is.dene, denx = is.denx;
            const int ie = is.ie, ix = is.ix;
            const bool geo = is.geo;
            const float enter = is.enter, exit = is.exit;
            const float density = q[0].w;
            Segment s;
            s.dt = fmaxf(exit - enter, 0.f);
            s.a = density * s.dt;
            const bool hit = act && geo && s.a > 0.f;
            if (hit) {
                integrate(q, o, d, enter, exit, s);
                // ---- undo_alpha_out (alphablend_shader_interp.slang:128-192)
                const float m0 = density;
                const float m1 = density * (exit + enter) / 2.0f;
                const float logT_old = st.logT + s.a;
                const float T = __expf(logT_old);
#pragma unroll
                for (int k = 0; k < 3; ++k) st.c[k] = fmaf(-s.rgb[k], T, st.c[k]);
                st.logT = logT_old;
                st.D[2] = st.D[2] - m0;
                st.D[3] = st.D[3] - m1;
                st.D[0] = st.D[0] - 2.0f * m1 * st.D[2];
                st.D[1] = st.D[1] - 2.0f * m0 * st.D[3];
                st.D[4] = st.D[4] - density * density * s.dt / 3.0f;
                // ---- adjoint of update_distortion_state
                const float dm1 = dS.D[0] * 2.0f * st.D[2] + dS.D[3];
                const float dm0 = dS.D[1] * 2.0f * st.D[3] + dS.D[2];
                const float nD2 = dS.D[2] + dS.D[0] * 2.0f * m1;
                const float nD3 = dS.D[3] + dS.D[1] * 2.0f * m0;
                float d_dens = dm0 + dm1 * (exit + enter) * 0.5f;
                float d_enter = dm1 * density * 0.5f;
                float d_exit = d_enter;
                float d_dt = dS.D[4] * density * density * (1.0f / 3.0f);
                d_dens += dS.D[4] * 2.0f * density * s.dt * (1.0f / 3.0f);
                // ---- adjoint of update_pixel_state
                float d_rgb[3], dT = 0.f, sum_drgb = 0.f;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    d_rgb[k] = dS.c[k] * T;
                    dT = fmaf(dS.c[k], s.rgb[k], dT);
                    sum_drgb += d_rgb[k];
                }
                const float d_a = -dS.logT;
                // safe_exp's clip at log(1e20) never binds: log T <= 0
                const float d_logT_old = dS.logT + dT * T;
                // ---- adjoint of compute_integral / integrate_tetra_segment
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
                d_enter += d_se * dot3(grd, d);
                d_exit += d_sx * dot3(grd, d);
                gl[12] = -grd.x * d_sum;
                gl[13] = -grd.y * d_sum;
                gl[14] = -grd.z * d_sum;
                if (exit - enter > 0.f) {
                    d_exit += d_dt;
                    d_enter -= d_dt;
                }
                gl[18] = density > 0.f ? d_dens : 0.f;
                float d_tx = 0.f;
                if (tx > enter) d_tx = d_exit; else d_enter += d_exit;
                const float d_te = te > 0.f ? d_enter : 0.f;
                // ---- adjoint of the plane intersections t = dot(n, vref - o) / dot(n, d)
                const float ge = d_te / dene, gx = d_tx / denx;
                const f3 ae = ie == 3 ? a1 : a0, ax = ix == 3 ? a1 : a0;
                const f3 dne = {ge * (ae.x - te * d.x), ge * (ae.y - te * d.y), ge * (ae.z - te * d.z)};
                const f3 dnx = {gx * (ax.x - tx * d.x), gx * (ax.y - tx * d.y), gx * (ax.z - tx * d.z)};
#pragma unroll
                for (int p = 0; p < 4; ++p) {
                    const f3 np = xyz(q[p]);
                    const float se = (ie == p) ? ge : 0.f, sx = (ix == p) ? gx : 0.f;
                    gl[3 * p + 0] = (ie == p ? dne.x : 0.f) + (ix == p ? dnx.x : 0.f);
                    gl[3 * p + 1] = (ie == p ? dne.y : 0.f) + (ix == p ? dnx.y : 0.f);
                    gl[3 * p + 2] = (ie == p ? dne.z : 0.f) + (ix == p ? dnx.z : 0.f);
                    const float sref = se + sx;  // gradient of vref = +n * g
                    if (p == 3) {
                        gl[15] += np.x * sref;
                        gl[16] += np.y * sref;
                        gl[17] += np.z * sref;
                    } else {
                        gl[12] += np.x * sref;
                        gl[13] += np.y * sref;
                        gl[14] += np.z * sref;
                    }
                }
                dS.logT = d_logT_old;
                dS.D[2] = nD2;
                dS.D[3] = nD3;
            }
            if (__any_sync(kMask, hit)) {
                using RS = ReduceScatter<kNGrad, WarpShape<NT>::kTopOffset>;
                int slot = 0;
                RS::template run<kMask>(gl, lane, slot);
#pragma unroll
                for (int r = 0; r < RS::R; ++r)
                    if (slot + r < kNGrad && gl[r] != 0.f) atomicAdd(&sacc[jj][slot + r], gl[r]);
            }
        }
        __syncthreads();
        // ---- flush: per list entry, convert to vertex gradients and add to global memory
        for (int jj = threadIdx.x; jj < n; jj += NT) {
            float v[kNGrad];
            bool any = false;
#pragma unroll
            for (int k = 0; k < kNGrad; ++k) {
                v[k] = sacc[jj][k];
                any |= v[k] != 0.f;
            }
            if (!any) continue;
            const float4* q = srec[jj];
            const int g = sid[jj];
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
}

template <int NT, int B>
int launch_fwd(const int32_t* ids, const int32_t* ranges, const float4* recs, const float* jitter,
               const rm_camera& cam, float* img, float* dist, int32_t* nc, cudaStream_t s) {
    const int G = cam.grid_width * cam.grid_height;
    blend_fwd_kernel<NT, B><<<G, NT, 0, s>>>(ids, (const int2*)ranges, recs, (const float2*)jitter, cam,
                                             (float4*)img, dist, nc);
    return rm_host::check_launch("rm_blend_fwd");
}

template <int NT, int B>
int launch_bwd(const int32_t* ids, const int32_t* ranges, const float4* recs, const int32_t* indices,
               const float* jitter, const rm_camera& cam, const float* img, const float* dist, const int32_t* nc,
               const float* gimg, const float* gdist, float* gverts, float* gcv, cudaStream_t s) {
    const int G = cam.grid_width * cam.grid_height;
    blend_bwd_kernel<NT, B><<<G, NT, 0, s>>>(ids, (const int2*)ranges, recs, (const int4*)indices,
                                             (const float2*)jitter, cam, (const float4*)img, dist, nc,
                                             (const float4*)gimg, gdist, gverts, gcv);
    return rm_host::check_launch("rm_blend_bwd");
}

int pack(const int32_t* indices, const float* vertices, const float* cv, int64_t n_tets, const int32_t* tiles,
         float4* recs, cudaStream_t s) {
    const int threads = 256;
    const int64_t blocks = (n_tets + threads - 1) / threads;
    pack_kernel<<<(unsigned)blocks, threads, 0, s>>>((const int4*)indices, vertices, cv, n_tets, tiles, recs);
    return rm_host::check_launch("rm_blend pack");
}

int check_blend_args(const char* who, const int32_t* indices, const float* vertices, const float* cv, int64_t n_tets,
                     const float* jitter, const rm_camera* cam, void* workspace, size_t workspace_bytes) {
    int rc = rm_host::check_cam(cam);
    if (rc) return rc;
    if (n_tets < 0) return rm_host::fail(RM_EINVAL, "%s: negative size", who);
    if (!indices || !vertices || !cv || !jitter || !workspace)
        return rm_host::fail(RM_EINVAL, "%s: NULL pointer", who);
    if ((uintptr_t)indices & 15) return rm_host::fail(RM_EINVAL, "%s: indices must be 16-byte aligned", who);
    if ((uintptr_t)workspace & 15) return rm_host::fail(RM_EINVAL, "%s: workspace must be 16-byte aligned", who);
    if (workspace_bytes < (size_t)n_tets * kRecFloat4 * sizeof(float4))
        return rm_host::fail(RM_EINVAL, "%s: workspace %zu < %zu bytes", who, workspace_bytes,
                             (size_t)n_tets * kRecFloat4 * sizeof(float4));
    const int nt = cam->tile_width * cam->tile_height;
    if (nt != 16 && nt != 64 && nt != 256 && nt != 1024)
        return rm_host::fail(RM_EINVAL, "%s: tile of %d pixels unsupported (16, 64, 256 or 1024)", who, nt);
    return RM_OK;
}

}  // namespace
}  // namespace rm

extern "C" {

size_t rm_blend_workspace_size(int64_t n_tets) {
    return (size_t)(n_tets > 0 ? n_tets : 1) * rm::kRecFloat4 * sizeof(float4);
}

int rm_blend_fwd(const int32_t* sorted_ids, const int32_t* ranges, const int32_t* indices, const float* vertices,
                 const float* cell_values, int64_t n_tets, int64_t n_verts, const int32_t* tiles_touched,
                 const float* ray_jitter, const rm_camera* cam, float* out_img, float* out_distortion,
                 int32_t* n_contrib, void* workspace, size_t workspace_bytes, int flags, void* stream) {
    using namespace rm;
    int rc = check_blend_args("rm_blend_fwd", indices, vertices, cell_values, n_tets, ray_jitter, cam, workspace,
                              workspace_bytes);
    if (rc) return rc;
    if (!ranges || !out_img || !out_distortion || !n_contrib)
        return rm_host::fail(RM_EINVAL, "rm_blend_fwd: NULL pointer");
    if (((uintptr_t)out_img & 15) || ((uintptr_t)ranges & 7) || ((uintptr_t)ray_jitter & 7))
        return rm_host::fail(RM_EINVAL, "rm_blend_fwd: misaligned image / ranges / jitter");
    cudaStream_t s = (cudaStream_t)stream;
    float4* recs = (float4*)workspace;
    if (!(flags & RM_BLEND_REUSE_RECORDS) && n_tets > 0) {
        rc = pack(indices, vertices, cell_values, n_tets, tiles_touched, recs, s);
        if (rc) return rc;
    }
    const int nt = cam->tile_width * cam->tile_height;
    switch (nt) {
        case 16: return launch_fwd<16, 64>(sorted_ids, ranges, recs, ray_jitter, *cam, out_img, out_distortion, n_contrib, s);
        case 64: return launch_fwd<64, 64>(sorted_ids, ranges, recs, ray_jitter, *cam, out_img, out_distortion, n_contrib, s);
        case 256: return launch_fwd<256, 64>(sorted_ids, ranges, recs, ray_jitter, *cam, out_img, out_distortion, n_contrib, s);
        default: return launch_fwd<1024, 64>(sorted_ids, ranges, recs, ray_jitter, *cam, out_img, out_distortion, n_contrib, s);
    }
}

int rm_blend_bwd(const int32_t* sorted_ids, const int32_t* ranges, const int32_t* indices, const float* vertices,
                 const float* cell_values, int64_t n_tets, int64_t n_verts, const int32_t* tiles_touched,
                 const float* ray_jitter, const rm_camera* cam, const float* out_img, const float* out_distortion,
                 const int32_t* n_contrib, const float* grad_img, const float* grad_distortion, float* grad_vertices,
                 float* grad_cell_values, void* workspace, size_t workspace_bytes, int flags, void* stream) {
    using namespace rm;
    int rc = check_blend_args("rm_blend_bwd", indices, vertices, cell_values, n_tets, ray_jitter, cam, workspace,
                              workspace_bytes);
    if (rc) return rc;
    if (!ranges || !out_img || !out_distortion || !n_contrib || !grad_img || !grad_vertices || !grad_cell_values)
        return rm_host::fail(RM_EINVAL, "rm_blend_bwd: NULL pointer");
    if (((uintptr_t)out_img & 15) || ((uintptr_t)grad_img & 15) || ((uintptr_t)ranges & 7) ||
        ((uintptr_t)ray_jitter & 7))
        return rm_host::fail(RM_EINVAL, "rm_blend_bwd: misaligned image / grad / ranges / jitter");
    cudaStream_t s = (cudaStream_t)stream;
    float4* recs = (float4*)workspace;
    if (!(flags & RM_BLEND_REUSE_RECORDS) && n_tets > 0) {
        rc = pack(indices, vertices, cell_values, n_tets, tiles_touched, recs, s);
        if (rc) return rc;
    }
    const int nt = cam->tile_width * cam->tile_height;
    switch (nt) {
        case 16: return launch_bwd<16, 32>(sorted_ids, ranges, recs, indices, ray_jitter, *cam, out_img, out_distortion, n_contrib, grad_img, grad_distortion, grad_vertices, grad_cell_values, s);
        case 64: return launch_bwd<64, 64>(sorted_ids, ranges, recs, indices, ray_jitter, *cam, out_img, out_distortion, n_contrib, grad_img, grad_distortion, grad_vertices, grad_cell_values, s);
        case 256: return launch_bwd<256, 64>(sorted_ids, ranges, recs, indices, ray_jitter, *cam, out_img, out_distortion, n_contrib, grad_img, grad_distortion, grad_vertices, grad_cell_values, s);
        default: return launch_bwd<1024, 64>(sorted_ids, ranges, recs, indices, ray_jitter, *cam, out_img, out_distortion, n_contrib, grad_img, grad_distortion, grad_vertices, grad_cell_values, s);
    }
}

}  // extern "C"
