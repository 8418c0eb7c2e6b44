// rm_internal.cuh - device helpers shared by the rasterizer kernels (sm_100a).
//
// Rounding rules.  This translation unit family is compiled with --fmad=false,
// so the compiler never contracts a*b+c on its own; every fused multiply-add
// below is an explicit fmaf/fma.  Division and sqrt are IEEE correctly rounded
// (-prec-div / -prec-sqrt default on; never -use_fast_math).  The rules are:
//   dot(a,b)     = fma(a.z,b.z, fma(a.y,b.y, a.x*b.x))
//   cross(a,b).x = fma(a.y,b.z, -(a.z*b.y))            (and cyclic)
//   a*b + c      = fma(a,b,c)  where the reference source writes a*b + c
//   lerp(x,y,s)  = fma(y,s, x*(1-s))
//   normalize(v) = v / sqrt(dot(v,v))
// With them the integer outputs of projection and blending (tile counts,
// rectangles, depth keys, n_contributors) and the log-transmittance channel
// are a pure function of the inputs, identical on every run and reproducible
// on the CPU.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/rm_capi.h"

namespace rm {

struct f3 {
    float x, y, z;
};

__device__ __forceinline__ f3 mk3(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ f3 operator-(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ f3 operator+(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ f3 neg3(f3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ f3 scale3(f3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ float dot3(f3 a, f3 b) { return fmaf(a.z, b.z, fmaf(a.y, b.y, a.x * b.x)); }
__device__ __forceinline__ f3 cross3(f3 a, f3 b) {
    return {fmaf(a.y, b.z, -(a.z * b.y)), fmaf(a.z, b.x, -(a.x * b.z)), fmaf(a.x, b.y, -(a.y * b.x))};
}

struct d3 {
    double x, y, z;
};
__device__ __forceinline__ d3 operator-(d3 a, d3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ d3 operator+(d3 a, d3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ d3 scale3(d3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ double dot3(d3 a, d3 b) { return fma(a.z, b.z, fma(a.y, b.y, a.x * b.x)); }
__device__ __forceinline__ d3 cross3(d3 a, d3 b) {
    return {fma(a.y, b.z, -(a.z * b.y)), fma(a.z, b.x, -(a.x * b.z)), fma(a.x, b.y, -(a.y * b.x))};
}
__device__ __forceinline__ double len3(d3 a) { return sqrt(dot3(a, a)); }

// log(1e20) rounded to float: the upper clip of safe_exp (safe-math.slang:137-140).
constexpr float kLogMax = (float)46.051701859880914;

__device__ __forceinline__ float safe_expf(float v) { return expf(fmaxf(fminf(v, kLogMax), -1e20f)); }

// Lens distortion is on when dot(distortion, distortion) >= 1e-9
// (camera.slang:244-246, 359-361).
__device__ __forceinline__ bool cam_distorted(const rm_camera& c) {
    const float* k = c.distortion;
    return k[0] * k[0] + k[1] * k[1] + k[2] * k[2] + k[3] * k[3] >= 1e-9f;
}

// undistort (camera.slang:241-296): 10 Newton steps on the radial (k1, k2)
// and tangential (p1, p2) model, stopping early on a singular Jacobian.  The
// distortion arithmetic is written with plain operations in the reference's
// textual order (no fused multiply-add).
__device__ __forceinline__ void undistort(const rm_camera& c, float& ux, float& uy) {
    const float k1 = c.distortion[0], k2 = c.distortion[1], p1 = c.distortion[2], p2 = c.distortion[3];
    const float pdx = ux, pdy = uy;
    float x = ux, y = uy;
    for (int i = 0; i < 10; ++i) {
        const float r2 = x * x + y * y;
        const float d = 1.0f + r2 * (k1 + r2 * k2);
        const float fx = d * x + 2.0f * p1 * x * y + p2 * (r2 + 2.0f * x * x) - pdx;
        const float fy = d * y + 2.0f * p2 * x * y + p1 * (r2 + 2.0f * y * y) - pdy;
        const float d_r = k1 + r2 * (2.0f * k2);
        const float d_x = 2.0f * x * d_r;
        const float d_y = 2.0f * y * d_r;
        const float fx_x = d + d_x * x + 2.0f * p1 * y + 6.0f * p2 * x;
        const float fx_y = d_y * x + 2.0f * p1 * x + 2.0f * p2 * y;
        const float fy_x = d_x * y + 2.0f * p2 * y + 2.0f * p1 * x;
        const float fy_y = d + d_y * y + 2.0f * p2 * x + 6.0f * p1 * y;
        const float den = fy_x * fx_y - fx_x * fy_y;
        if (fabsf(den) < 1e-9f) break;
        x = x + (fx * fy_y - fy * fx_y) / den;
        y = y + (fy * fx_x - fx * fy_x) / den;
    }
    ux = x;
    uy = y;
}

// Ray direction in world space from a camera-space direction, normalised,
// and the origin min_t along it (get_ray, camera.slang:331-346).
__device__ __forceinline__ void ray_to_world(const rm_camera& c, f3 dc, f3& o, f3& d) {
    const float* M = c.world_view;
    f3 dw = {dot3(mk3(M[0], M[4], M[8]), dc), dot3(mk3(M[1], M[5], M[9]), dc),
             dot3(mk3(M[2], M[6], M[10]), dc)};
    const float l = sqrtf(dot3(dw, dw));
    d = {dw.x / l, dw.y / l, dw.z / l};
    o = {fmaf(d.x, c.min_t, c.cam_pos[0]), fmaf(d.y, c.min_t, c.cam_pos[1]),
         fmaf(d.z, c.min_t, c.cam_pos[2])};
}

// Camera-space direction of a normalised image point for a fisheye or a
// distorted camera: undistorted, then (fisheye) the angle theta = |p| from
// the axis, clamped to pi.  Kept out of line: it runs once per pixel and its
// registers would otherwise count against the blend loops.
static __device__ __noinline__ f3 general_dir(const rm_camera& c, float ux, float uy) {
    const bool fisheye = c.camera_type == 1;
    if (cam_distorted(c)) undistort(c, ux, uy);
    if (fisheye) {
        float theta = sqrtf(ux * ux + uy * uy);
        theta = fminf(3.14159265f, theta);
        const float s = theta < 1e-6f ? 1.0f : sinf(theta) / theta;
        return {ux * s, uy * s, cosf(theta)};
    }
    f3 dc = {ux, uy, 1.0f};
    const float l = sqrtf(dot3(dc, dc));
    return {dc.x / l, dc.y / l, dc.z / l};
}

// get_ray (camera.slang:298-346): pixel -> normalised image point,
// undistorted for perspective (0) and fisheye (1) cameras, then the camera
// ray, rotated to the world and started min_t along the ray.  The pinhole
// path without distortion is exactly the declared-rounding path of the tests.
__device__ __forceinline__ void make_ray(const rm_camera& c, int px, int py, float jx, float jy, f3& o,
                                         f3& d) {
    const float ux = ((float)px + jx - c.K[2]) / c.K[0];
    const float uy = ((float)py + jy - c.K[5]) / c.K[4];
    f3 dc;
    if (c.camera_type == 0 && !cam_distorted(c)) {
        dc = {ux, uy, 1.0f};
        const float l = sqrtf(dot3(dc, dc));
        dc = {dc.x / l, dc.y / l, dc.z / l};
    } else {
        dc = general_dir(c, ux, uy);
    }
    ray_to_world(c, dc, o, d);
}

// Packed per-tet record (128 B = 8 x float4) staged by the blend kernels.
//   q0 = (n0, density)   q1 = (n1, r)   q2 = (n2, g)   q3 = (n3, b)
//   q4 = (v0, gx)        q5 = (v1, gy)  q6 = (v2, gz)  q7 = (v3, flip bits)
// n_i are the outward face normals of ray_tetrahedron_intersect_fused
// (intersect.slang:449-475) after the orientation flip; bit i of the flip word
// records whether n_i was negated.
constexpr int kRecFloat4 = 8;

__device__ __forceinline__ int tile_w_of(const rm_camera& c) { return c.tile_width; }

// Views of one launch, as the blend kernels see them.  Tiles of all views
// share one global, view-major numbering (view v owns the tiles
// [tile_base[v], tile_base[v + 1])) and the per-pixel buffers of all views are
// concatenated (view v's pixel (x, y) is element pixel_base[v] + y * W + x).
// OneView is the single-camera case; ViewSet carries up to RM_MAX_VIEWS
// cameras by value in the kernel parameters, so a captured CUDA graph holds
// its own copy.
struct OneView {
    rm_camera cam;
    __device__ __forceinline__ int find(int) const { return 0; }
    __device__ __forceinline__ const rm_camera& camera(int) const { return cam; }
    __device__ __forceinline__ int tile_base(int) const { return 0; }
    __device__ __forceinline__ int64_t pixel_base(int) const { return 0; }
};

struct ViewSet {
    int n;
    int tiles[RM_MAX_VIEWS + 1];        // tile_base, with tiles[n] = total tiles
    int64_t pixels[RM_MAX_VIEWS + 1];   // pixel_base, with pixels[n] = total pixels
    rm_camera cams[RM_MAX_VIEWS];
    float parallax[RM_MAX_VIEWS];       // rm_host::parallax_px of each camera
    __device__ __forceinline__ int find(int tile) const {
        int lo = 0, hi = n - 1;  // last view whose first tile is <= tile
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (tiles[mid] <= tile) lo = mid;
            else hi = mid - 1;
        }
        return lo;
    }
    __device__ __forceinline__ const rm_camera& camera(int v) const { return cams[v]; }
    __device__ __forceinline__ int tile_base(int v) const { return tiles[v]; }
    __device__ __forceinline__ int64_t pixel_base(int v) const { return pixels[v]; }
};

// Whether a tet can reach a pixel of the tile with pixel columns [x0, x0 + w)
// and rows [y0, y0 + h).  The ray of pixel (px, py) passes through the image
// point (px + jx, py + jy); with the jitter inside jb = (min jx, min jy,
// max jx, max jy) every such point of the tile lies in
// [x0 + jb.x, x0 + w - 1 + jb.z] x [y0 + jb.y, y0 + h - 1 + jb.w] (rounding
// is monotone, so the float sums bound the float sums of the kernels).  A ray
// through a point farther than kBoxMargin from the tet's image-space box
// (rm_project_fwd_fine) misses the tet; the margin covers the rounding of the
// projection against the ray setup many times over.
constexpr float kBoxMargin = 1.0f / 64.0f;

__device__ __forceinline__ bool box_meets_tile(float4 b, float4 jb, int x0, int y0, int w, int h) {
    return b.x - kBoxMargin <= (float)(x0 + w - 1) + jb.z && b.z + kBoxMargin >= (float)x0 + jb.x &&
           b.y - kBoxMargin <= (float)(y0 + h - 1) + jb.w && b.w + kBoxMargin >= (float)y0 + jb.y;
}

// A tet's footprint in the image (rm_project_fwd_fine): its box and, when all
// four vertices lie in front of a pinhole camera (z > 1e-4, so find_extent
// clips nothing) and project within kHullRange pixels of the origin, the four
// projected vertices (p01 = x0 y0 x1 y1, p23 = x2 y2 x3 y3; NaN otherwise).
// The tet's image is then the convex hull of those points, and a ray through
// an image point farther than kHullMargin outside it misses the tet.
struct Footprint {
    float4 box, p01, p23;
};
constexpr float kHullMargin = 1.0f / 16.0f;
constexpr float kHullRange = 8192.0f;

// Bit q (q < F * F) set: the tet with footprint f can reach a pixel ray of
// sub-tile q (column q % F, row q / F; w x h pixels) of the tile whose pixel
// origin is (ox, oy), under the jitter bounds jb.  First the box test
// (box_meets_tile); then, when the projected vertices are given, every edge
// of their convex hull: the 6 vertex pairs, a pair being a hull edge when the
// other two points lie on one side of its line (rounding can only misjudge
// points within rounding distance of the line, far inside the margin).  A
// sub-tile whose jittered footprint lies more than kHullMargin outside one
// hull edge is dropped.  Coordinates are taken relative to (ox, oy); plain
// float operations in this order (no fused multiply-add).
template <int F>
__device__ __forceinline__ uint64_t footprint_bits(const Footprint& f, float4 jb, int ox, int oy, int w, int h) {
    uint64_t bits = 0;
#pragma unroll
    for (int q = 0; q < F * F; ++q)
        if (box_meets_tile(f.box, jb, ox + q % F * w, oy + q / F * h, w, h)) bits |= 1ull << q;
    if (bits == 0 || isnan(f.p01.x)) return bits;
    const float fx = (float)ox, fy = (float)oy;
    const float px[4] = {f.p01.x - fx, f.p01.z - fx, f.p23.x - fx, f.p23.z - fx};
    const float py[4] = {f.p01.y - fy, f.p01.w - fy, f.p23.y - fy, f.p23.w - fy};
    const int ea[6] = {0, 0, 0, 1, 1, 2}, eb[6] = {1, 2, 3, 2, 3, 3};
    const int o1[6] = {2, 1, 1, 0, 0, 0}, o2[6] = {3, 3, 2, 3, 2, 1};
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const int a = ea[k], b = eb[k];
        const float nx = py[b] - py[a], ny = px[a] - px[b];
        const float ca = nx * px[a] + ny * py[a];
        const float s1 = nx * px[o1[k]] + ny * py[o1[k]] - ca;
        const float s2 = nx * px[o2[k]] + ny * py[o2[k]] - ca;
        const bool out_pos = s1 <= 0.f && s2 <= 0.f;  // the others on the negative side: n points out
        const bool out_neg = !out_pos && s1 >= 0.f && s2 >= 0.f;
        if (!out_pos && !out_neg) continue;
        const float sg = out_pos ? 1.0f : -1.0f;
        const float ex = sg * nx, ey = sg * ny, ec = sg * ca;
        const float margin = kHullMargin * (fabsf(ex) + fabsf(ey));
#pragma unroll
        for (int q = 0; q < F * F; ++q) {
            const int dx = q % F * w, dy = q / F * h;
            const float xlo = (float)dx + jb.x, xhi = (float)(dx + w - 1) + jb.z;
            const float ylo = (float)dy + jb.y, yhi = (float)(dy + h - 1) + jb.w;
            const float d = ex * (ex > 0.f ? xlo : xhi) + ey * (ey > 0.f ? ylo : yhi) - ec;
            if (d > margin) bits &= ~(1ull << q);
        }
    }
    return bits;
}

// Whether a tet's four vertex indices lie in [0, n_verts): a tet that fails
// is culled before any vertex load (RM_STATUS_BAD_INDEX).
__device__ __forceinline__ bool tet_indices_ok(int4 id, int64_t n_verts) {
    return id.x >= 0 && id.y >= 0 && id.z >= 0 && id.w >= 0 && (int64_t)id.x < n_verts &&
           (int64_t)id.y < n_verts && (int64_t)id.z < n_verts && (int64_t)id.w < n_verts;
}

// ------------------------------------------------ bulk copies into shared --
// One-dimensional bulk copies (cp.async.bulk, the TMA unit's untiled mode)
// from this GPU's global memory into the issuing CTA's shared memory,
// completing on an mbarrier that counts the bytes; each copy lands in the
// issuing CTA only.
// Source and destination must be 16-byte aligned and the size a multiple of
// 16 bytes (the per-tet records are 128 B).
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Makes mbarrier initialisation visible to the async proxy (the copy unit).
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Orders this thread's earlier shared-memory accesses (after a barrier: the
// CTA's) before async-proxy writes that it issues next (write-after-read on
// a staging buffer).
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Arrive on the barrier (count 1) and expect `bytes` more transaction bytes.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the barrier's phase with the given parity to complete, at most
// `limit` polls (each try_wait itself suspends for a short, hardware-chosen
// time).  Returns false when the limit is reached; the caller then reports
// the timeout and must not read the staged data.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit) {
    for (uint32_t i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Bounded spin helper: returns false once the budget is exhausted.
__device__ __forceinline__ bool spin_budget(uint32_t& left) {
    if (left == 0) return false;
    --left;
    if ((left & 63u) == 0) __nanosleep(64);
    return true;
}

}  // namespace rm

// Host-side helpers (rm_capi.cu).
namespace rm_host {
int fail(int code, const char* fmt, ...);
// Iteration limit of the bounded device-side waits (rm_set_wait_limit); the
// host passes it to every kernel that waits.
uint32_t wait_limit();
// rm_scan_tiles with the timeout / overflow bits or-ed into `status` instead
// of the workspace's own status word (status NULL: the workspace's word).
int scan_tiles_status(const int32_t* tiles_touched, int64_t n_tets, int32_t* offsets, int64_t* total_dev,
                      void* workspace, size_t workspace_bytes, uint32_t* status, void* stream);
// mode 1: inclusive scan of (in[i] > 0); mode 2: of in[order[i]] for i < *n_dev
// (n_dev may be NULL: all n), zero beyond.
int scan_mode(int mode, const int32_t* in, const int32_t* order, int64_t n, const int64_t* n_dev, int32_t* out,
              int64_t* total_dev, void* workspace, size_t workspace_bytes, uint32_t* status, void* stream);
// Checks the launch status of the preceding kernel launches and adds
// `kernels` to the process-wide launch counter.
int check_launch(const char* what, int kernels = 1);
int check_cam(const rm_camera* cam);
// Validates n cameras (n in [1, RM_MAX_VIEWS], one tile size for all) and
// fills the view table.
int make_views(const char* who, const rm_camera* cams, int n, rm::ViewSet* out);
// Pixels by which a ray of the camera can miss the image point its pixel
// names, at the depths rays reach, because rays start from cam_pos while the
// projection uses the centre of world_view: 2 x focal length x offset / min_t
// (rays start min_t along their direction); 0 for a centred camera, infinity
// when the two cannot be reconciled (projective last row, a matrix that is
// not a rotation, or an offset with min_t <= 0).
float parallax_px(const rm_camera& c);
// True unless the camera is a plain perspective one with all distortion
// coefficients zero; kernels instantiated for the plain camera leave out the
// fisheye and distortion code (a conservative test: a camera with tiny
// nonzero coefficients takes the general code, which tests them itself).
inline bool cam_general(const rm_camera& c) {
    return c.camera_type != 0 || c.distortion[0] != 0.f || c.distortion[1] != 0.f || c.distortion[2] != 0.f ||
           c.distortion[3] != 0.f;
}
}  // namespace rm_host
