// rm_project.cu - stage (a): per-tet projection, cull, tile rectangle and the
// FP64 circumsphere-power depth key, plus its adjoint.
//
// Forward follows vertex_shader (vertex_shader.slang:23-89) with find_extent
// (camera.slang:443-508), is_planar (intersect.slang:76-89) and
// power_of_circumsphere (stable_power.slang:18-85).  One thread per tet; the
// [T,4] index row is one 16-byte load and every output row is written once
// (zeros for culled tets), so no separate zero-fill pass is needed.
#include "rm_internal.cuh"

namespace rm {
namespace {

__device__ __forceinline__ float safe_clipf(float v, float lo, float hi) { return fmaxf(fminf(v, hi), lo); }

__device__ __forceinline__ float safe_divf(float a, float b) {  // safe-math.slang:72-79
    const float tiny = 1.0754944e-20f;
    if (fabsf(b) < tiny) return safe_clipf(a / tiny, -1e20f, 1e20f);
    return safe_clipf(a / b, -1e20f, 1e20f);
}

__device__ __forceinline__ f3 point2cam(const rm_camera& c, f3 p) {  // camera.slang:103-108
    const float* M = c.world_view;
    float h0 = fmaf(M[3], 1.0f, fmaf(M[2], p.z, fmaf(M[1], p.y, M[0] * p.x)));
    float h1 = fmaf(M[7], 1.0f, fmaf(M[6], p.z, fmaf(M[5], p.y, M[4] * p.x)));
    float h2 = fmaf(M[11], 1.0f, fmaf(M[10], p.z, fmaf(M[9], p.y, M[8] * p.x)));
    float h3 = fmaf(M[15], 1.0f, fmaf(M[14], p.z, fmaf(M[13], p.y, M[12] * p.x)));
    return {safe_divf(h0, h3), safe_divf(h1, h3), safe_divf(h2, h3)};
}

__device__ __forceinline__ f3 lerp3(f3 a, f3 b, float s) {
    const float w = 1.0f - s;
    return {fmaf(b.x, s, a.x * w), fmaf(b.y, s, a.y * w), fmaf(b.z, s, a.z * w)};
}

struct BBox {
    f3 mn, mx;
};

// GENERAL = false: a perspective camera without distortion (the host picks
// the instantiation with rm_host::cam_general).
template <bool GENERAL>
__device__ __forceinline__ void bbox_add(BBox& b, const rm_camera& c, f3 p) {
    // camspace_to_image (camera.slang:382-412): perspective division or the
    // fisheye angle map, then distort (camera.slang:357-378), then K
    float ux, uy;
    if (GENERAL && c.camera_type == 1) {
        const float l = sqrtf(dot3(p, p));
        const f3 dir = {p.x / l, p.y / l, p.z / l};
        const float theta = acosf(fminf(fmaxf(dir.z, 0.f), 1.f));
        const float st = sinf(theta);
        const float f = st < 1e-6f ? 1.0f : theta / st;
        ux = dir.x * f;
        uy = dir.y * f;
    } else {
        ux = p.x / p.z;
        uy = p.y / p.z;
    }
    if (GENERAL && cam_distorted(c)) {
        const float k1 = c.distortion[0], k2 = c.distortion[1], p1 = c.distortion[2], p2 = c.distortion[3];
        const float r2 = ux * ux + uy * uy;
        const float radial = r2 * (k1 + r2 * k2);
        const float tx = 2.0f * p1 * ux * uy + p2 * (r2 + 2.0f * ux * ux);
        const float ty = 2.0f * p2 * ux * uy + p1 * (r2 + 2.0f * uy * uy);
        const float dx = ux + ux * radial + tx;
        const float dy = uy + uy * radial + ty;
        ux = dx;
        uy = dy;
    }
    const float qx = fmaf(ux, c.K[0], c.K[2]);
    const float qy = fmaf(uy, c.K[4], c.K[5]);
    b.mn = {fminf(b.mn.x, qx), fminf(b.mn.y, qy), fminf(b.mn.z, p.z)};
    b.mx = {fmaxf(b.mx.x, qx), fmaxf(b.mx.y, qy), fmaxf(b.mx.z, p.z)};
}

__device__ __forceinline__ bool eq3(f3 a, f3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }

// One face of find_extent: clip the triangle (a,b,c) against z = 1e-4 and add
// the clipped polygon's vertices to the box when it has more than one vertex.
// Sampling each edge at t = 0 and t = 1 (2 samples) yields exactly the polygon
// vertices (lerp with s = 0 / 1 is exact), so the box is the box of the
// polygon vertices; the de-duplication only matters for the vertex count.
template <bool GENERAL>
__device__ __forceinline__ void clip_face(const rm_camera& c, f3 a, f3 b, f3 cc, BBox& box) {
    const float eps = 1e-4f;
    f3 p[4];
    int n = 0;
    const f3 fv[3] = {a, b, cc};
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const f3 va = fv[j];
        const f3 vb = fv[(j + 1) % 3];
        const bool ain = va.z > eps;
        const bool bin = vb.z > eps;
        if (ain) {
            bool found = false;
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (k < n && eq3(p[k], va)) found = true;
            if (!found) {
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if (k == n) p[k] = va;
                ++n;
            }
        }
        if (ain != bin) {
            const float t = (eps - va.z) / (vb.z - va.z);
            const f3 q = lerp3(va, vb, t);
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (k == n) p[k] = q;
            ++n;
        }
    }
    if (n > 1) {
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (k < n) bbox_add<GENERAL>(box, c, p[k]);
        // update_bounds_from_edge (camera.slang:416-439): 2 samples per edge
        // (its endpoints) for a plain perspective camera, 3 with distortion,
        // 4 for a fisheye; samples at t = i / (n_samples - 1) from each edge's
        // start, so the interior ones are added here
        const int ns = !GENERAL ? 2 : (c.camera_type == 1 ? 4 : (cam_distorted(c) ? 3 : 2));
        if (GENERAL && ns > 2) {
            for (int k = 0; k < n; ++k) {
                f3 a = p[0], b = p[0];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (q == k) a = p[q];
                    if (q == (k + 1) % n) b = p[q];
                }
                for (int i = 1; i < ns - 1; ++i)
                    bbox_add<GENERAL>(box, c, lerp3(a, b, (float)i / (float)(ns - 1)));
            }
        }
    }
}

// Circumsphere of (A,B,C,D) (power_of_circumsphere, stable_power.slang:18-85,
// without the final power): false when the tet is degenerate and not
// collapsed to a point, in which case the reference returns power -1e20.
__device__ bool circumsphere(d3 A, d3 B, d3 C, d3 D, d3& center, double& radius) {
    const d3 a = B - A, b = C - A, c = D - A;
    const double aa = dot3(a, a), bb = dot3(b, b), cc = dot3(c, c);
    const d3 cbc = cross3(b, c), cca = cross3(c, a), cab = cross3(a, b);
    const double den = 2.0 * dot3(a, cbc);
    if (fabs(den) < 1e-10) {
        const double m = fmax(len3(B - A), fmax(len3(C - A), fmax(len3(D - A),
                         fmax(len3(C - B), fmax(len3(D - B), len3(D - C))))));
        if (m < 1e-7) {
            center = scale3(((A + B) + C) + D, 0.25);
            radius = fmin(len3(A - center), fmin(len3(B - center), fmin(len3(C - center), len3(D - center))));
            return true;
        }
        center = {0.0, 0.0, 0.0};
        radius = 0.0;
        return false;
    }
    const d3 rel = {fma(cc, cab.x, fma(bb, cca.x, aa * cbc.x)) / den,
                    fma(cc, cab.y, fma(bb, cca.y, aa * cbc.y)) / den,
                    fma(cc, cab.z, fma(bb, cca.z, aa * cbc.z)) / den};
    center = A + rel;
    radius = len3(rel);
    return true;
}

// Power of P with respect to the sphere: |center - P|^2 - radius^2.
__device__ __forceinline__ double sphere_power(d3 center, double radius, d3 P) {
    const d3 df = center - P;
    return dot3(df, df) - radius * radius;
}

__device__ double power_of_circumsphere(d3 A, d3 B, d3 C, d3 D, d3 P, d3& center) {
    double radius;
    if (!circumsphere(A, B, C, D, center, radius)) return -1e20;
    return sphere_power(center, radius, P);
}

__device__ __forceinline__ f3 load_vertex(const float* __restrict__ v, int i) {
    const float* p = v + 3 * (int64_t)i;
    return {__ldg(p), __ldg(p + 1), __ldg(p + 2)};
}

// View-independent part of vertex_shader: the vertices, the planarity cull
// (is_planar, intersect.slang:76-89) and the circumsphere.  Input checks come
// first: a tet with an index outside [0, n_verts) is culled before any vertex
// load (err = RM_STATUS_BAD_INDEX), one with a NaN or infinite vertex is
// culled too (err = RM_STATUS_NONFINITE; the reference asserts on NaN
// vertices on the host, tile_shader_slang.py:78).  Culling goes through
// `planar`, which every view tests first.
struct TetGeom {
    f3 v[4];
    bool planar;
    bool sphere;  // false: power -1e20 (culled in every view)
    d3 center;
    double radius;
    uint32_t err;
};

__device__ __forceinline__ TetGeom tet_geom(const int4* __restrict__ indices, const float* __restrict__ verts,
                                            int64_t g, int64_t n_verts) {
    TetGeom t;
    t.err = 0u;
    t.sphere = false;
    t.center = {0.0, 0.0, 0.0};
    t.radius = 0.0;
    const int4 id = __ldg(indices + g);
    if (!tet_indices_ok(id, n_verts)) {
#pragma unroll
        for (int i = 0; i < 4; ++i) t.v[i] = {0.f, 0.f, 0.f};
        t.planar = true;
        t.err = RM_STATUS_BAD_INDEX;
        return t;
    }
    t.v[0] = load_vertex(verts, id.x);
    t.v[1] = load_vertex(verts, id.y);
    t.v[2] = load_vertex(verts, id.z);
    t.v[3] = load_vertex(verts, id.w);
    bool finite = true;
#pragma unroll
    for (int i = 0; i < 4; ++i) finite &= isfinite(t.v[i].x) && isfinite(t.v[i].y) && isfinite(t.v[i].z);
    if (!finite) {
        t.planar = true;
        t.err = RM_STATUS_NONFINITE;
        return t;
    }
    f3 nrm = cross3(t.v[1] - t.v[0], t.v[2] - t.v[0]);
    const float l = sqrtf(dot3(nrm, nrm));
    nrm = {nrm.x / l, nrm.y / l, nrm.z / l};
    t.planar = fabsf(dot3(nrm, t.v[3] - t.v[0])) < 1e-3f;
    if (!t.planar)
        t.sphere = circumsphere({(double)t.v[0].x, (double)t.v[0].y, (double)t.v[0].z},
                                {(double)t.v[1].x, (double)t.v[1].y, (double)t.v[1].z},
                                {(double)t.v[2].x, (double)t.v[2].y, (double)t.v[2].z},
                                {(double)t.v[3].x, (double)t.v[3].y, (double)t.v[3].z}, t.center, t.radius);
    return t;
}

// Early cull of tets wholly outside the view: when all four vertices lie in
// the open half-space beyond one side of the image (one pixel of margin) or
// behind the camera, so does their hull, hence every vertex and clipped point
// that find_extent keeps, and the rectangle below would come out empty.  The
// test is linear in the vertices (no divisions) and only ever reports tets
// that the full computation culls, with a tolerance far above its rounding.
// It needs an affine world-to-camera matrix (last row 0 0 0 1).
__device__ __forceinline__ bool outside_view(const rm_camera& c, const TetGeom& t) {
    const float* M = c.world_view;
    if (c.camera_type != 0 || cam_distorted(c)) return false;  // the test assumes the pinhole projection
    if (!(M[12] == 0.f && M[13] == 0.f && M[14] == 0.f && M[15] == 1.f)) return false;
    const float fx = c.K[0], cx = c.K[2], fy = c.K[4], cy = c.K[5];
    const float gw = (float)c.grid_width * (float)c.tile_width, gh = (float)c.grid_height * (float)c.tile_height;
    const float m = 1.0f, tol = 1e-4f;
    bool behind = true, left = true, right = true, top = true, bottom = true;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const f3 p = t.v[i];
        const float x = fmaf(M[3], 1.0f, fmaf(M[2], p.z, fmaf(M[1], p.y, M[0] * p.x)));
        const float y = fmaf(M[7], 1.0f, fmaf(M[6], p.z, fmaf(M[5], p.y, M[4] * p.x)));
        const float z = fmaf(M[11], 1.0f, fmaf(M[10], p.z, fmaf(M[9], p.y, M[8] * p.x)));
        const float az = fabsf(z);
        const float ex = tol * (fabsf(fx * x) + (fabsf(cx) + gw + m) * az) + 1e-6f;
        const float ey = tol * (fabsf(fy * y) + (fabsf(cy) + gh + m) * az) + 1e-6f;
        behind &= z < 0.f;
        left &= fmaf(fx, x, (cx + m) * z) < -ex;
        right &= fmaf(gw + m - cx, z, -(fx * x)) < -ex;
        top &= fmaf(fy, y, (cy + m) * z) < -ey;
        bottom &= fmaf(gh + m - cy, z, -(fy * y)) < -ey;
    }
    return behind || left || right || top || bottom;
}

// Per-view part of vertex_shader (vertex_shader.slang:36-89): camera space,
// find_extent, the depth key and the tile rectangle.  Returns the tile count
// (0: culled, r and depth zero).
// BOX: also return the tet's image footprint (box and projected vertices,
// Footprint; zeros when culled) from which the lists of smaller tiles are cut.
template <bool GENERAL, bool BOX = false>
__device__ __forceinline__ int project_view(const rm_camera& cam, const TetGeom& t, int4& r, float& depth_out,
                                            Footprint* fp = nullptr) {
    r = {0, 0, 0, 0};
    depth_out = 0.f;
    if (BOX) *fp = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
    if (t.planar || outside_view(cam, t)) return 0;
    const f3 cs0 = point2cam(cam, t.v[0]), cs1 = point2cam(cam, t.v[1]);
    const f3 cs2 = point2cam(cam, t.v[2]), cs3 = point2cam(cam, t.v[3]);
    BBox box = {{1e20f, 1e20f, 1e20f}, {-1e20f, -1e20f, -1e20f}};
    clip_face<GENERAL>(cam, cs0, cs1, cs2, box);
    clip_face<GENERAL>(cam, cs0, cs2, cs3, box);
    clip_face<GENERAL>(cam, cs0, cs3, cs1, box);
    clip_face<GENERAL>(cam, cs1, cs3, cs2, box);
    if (box.mx.z <= 0.0f) return 0;
    // depth key: FP64 power of the circumsphere w.r.t. the camera position
    const d3 P = {(double)cam.cam_pos[0], (double)cam.cam_pos[1], (double)cam.cam_pos[2]};
    const double pw = t.sphere ? sphere_power(t.center, t.radius, P) : -1e20;
    const float depth = (float)pw;
    if (depth < -1e19f) return 0;
    const float gw = (float)cam.grid_width, gh = (float)cam.grid_height;
    const float tw = (float)cam.tile_width, th = (float)cam.tile_height;
    r.x = (int)floorf(fmaxf(0.f, fminf(gw, box.mn.x / tw)));
    r.y = (int)floorf(fmaxf(0.f, fminf(gh, box.mn.y / th)));
    r.z = (int)ceilf(fmaxf(0.f, fminf(gw, box.mx.x / tw)));
    r.w = (int)ceilf(fmaxf(0.f, fminf(gh, box.mx.y / th)));
    const int n_tiles = (r.z - r.x) * (r.w - r.y);
    if (n_tiles == 0) {
        r = {0, 0, 0, 0};
        return 0;
    }
    depth_out = fminf(fmaxf(depth, -1e20f), 1e20f);
    if (BOX) {
        fp->box = {box.mn.x, box.mn.y, box.mx.x, box.mx.y};
        // the projected vertices (camspace_to_image as in bbox_add) when no
        // vertex is clipped and the camera is a plain pinhole
        const f3 cs[4] = {cs0, cs1, cs2, cs3};
        float q[8];
        bool ok = !GENERAL;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            q[2 * i] = fmaf(cs[i].x / cs[i].z, cam.K[0], cam.K[2]);
            q[2 * i + 1] = fmaf(cs[i].y / cs[i].z, cam.K[4], cam.K[5]);
            ok &= cs[i].z > 1e-4f && fabsf(q[2 * i]) <= kHullRange && fabsf(q[2 * i + 1]) <= kHullRange;
        }
        const float nan = __int_as_float(0x7fc00000);
        fp->p01 = ok ? make_float4(q[0], q[1], q[2], q[3]) : make_float4(nan, nan, nan, nan);
        fp->p23 = ok ? make_float4(q[4], q[5], q[6], q[7]) : make_float4(nan, nan, nan, nan);
    }
    return n_tiles;
}

template <bool GENERAL>
__global__ void __launch_bounds__(256) project_fwd_kernel(const int4* __restrict__ indices,
                                                          const float* __restrict__ verts, int64_t n_tets,
                                                          int64_t n_verts, const rm_camera cam,
                                                          int32_t* __restrict__ tiles, int4* __restrict__ rect,
                                                          float* __restrict__ vs, float* __restrict__ cc,
                                                          uint32_t* status) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_tets) return;
    const TetGeom t = tet_geom(indices, verts, g, n_verts);
    if (t.err && status) atomicOr(status, t.err);
    int4 r;
    float depth;
    const int n_tiles = project_view<GENERAL>(cam, t, r, depth);
    tiles[g] = n_tiles;
    rect[g] = r;
    vs[3 * g + 0] = 0.f;
    vs[3 * g + 1] = 0.f;
    vs[3 * g + 2] = depth;
    cc[3 * g + 0] = n_tiles ? (float)t.center.x : 0.f;
    cc[3 * g + 1] = n_tiles ? (float)t.center.y : 0.f;
    cc[3 * g + 2] = n_tiles ? (float)t.center.z : 0.f;
}

// Projection plus each tet's image-space bounding box.
template <bool GENERAL>
__global__ void __launch_bounds__(256) project_fwd_fine_kernel(const int4* __restrict__ indices,
                                                               const float* __restrict__ verts, int64_t n_tets,
                                                               int64_t n_verts, const rm_camera cam,
                                                               int32_t* __restrict__ tiles, int4* __restrict__ rect,
                                                               float* __restrict__ vs, float* __restrict__ cc,
                                                               float4* __restrict__ fp, uint32_t* status) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_tets) return;
    const TetGeom t = tet_geom(indices, verts, g, n_verts);
    if (t.err && status) atomicOr(status, t.err);
    int4 r;
    Footprint f;
    float depth;
    const int n_tiles = project_view<GENERAL, true>(cam, t, r, depth, &f);
    tiles[g] = n_tiles;
    rect[g] = r;
    vs[3 * g + 0] = 0.f;
    vs[3 * g + 1] = 0.f;
    vs[3 * g + 2] = depth;
    cc[3 * g + 0] = n_tiles ? (float)t.center.x : 0.f;
    cc[3 * g + 1] = n_tiles ? (float)t.center.y : 0.f;
    cc[3 * g + 2] = n_tiles ? (float)t.center.z : 0.f;
    if (n_tiles) {  // only listed tets' footprints are ever read
        fp[3 * g] = f.box;
        fp[3 * g + 1] = f.p01;
        fp[3 * g + 2] = f.p23;
    }
}

// All views of a batch: each thread loads its tet once and projects it into
// every view; outputs are stacked view-major.
template <bool GENERAL>
__global__ void __launch_bounds__(256) project_fwd_multi_kernel(const int4* __restrict__ indices,
                                                                const float* __restrict__ verts, int64_t n_tets,
                                                                int64_t n_verts,
                                                                const __grid_constant__ ViewSet views,
                                                                int32_t* __restrict__ tiles, int4* __restrict__ rect,
                                                                float* __restrict__ depth, int32_t* __restrict__ any,
                                                                float* __restrict__ cc, float4* __restrict__ fp,
                                                                uint32_t* status) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_tets) return;
    const TetGeom t = tet_geom(indices, verts, g, n_verts);
    if (t.err && status) atomicOr(status, t.err);
    int total = 0;
    for (int v = 0; v < views.n; ++v) {
        int4 r;
        Footprint f;
        float dk;
        const int64_t o = (int64_t)v * n_tets + g;
        int n_tiles;
        if (fp) {
            n_tiles = project_view<GENERAL, true>(views.cams[v], t, r, dk, &f);
        } else {
            n_tiles = project_view<GENERAL>(views.cams[v], t, r, dk);
        }
        tiles[o] = n_tiles;
        // the rows of (view, tet) pairs without tiles are never read: not written
        if (n_tiles) {
            rect[o] = r;
            depth[o] = dk;
            if (fp) {
                fp[3 * o] = f.box;
                fp[3 * o + 1] = f.p01;
                fp[3 * o + 2] = f.p23;
            }
        }
        total += n_tiles;
    }
    if (any) any[g] = total;
    if (cc) {
        cc[3 * g + 0] = total ? (float)t.center.x : 0.f;
        cc[3 * g + 1] = total ? (float)t.center.y : 0.f;
        cc[3 * g + 2] = total ? (float)t.center.z : 0.f;
    }
}

__device__ __forceinline__ void atomic_add3(float* p, d3 g) {
    atomicAdd(p, (float)g.x);
    atomicAdd(p + 1, (float)g.y);
    atomicAdd(p + 2, (float)g.z);
}

// Adjoint of vs[:,2] = clamp(float(power)) and circumcenter = float(center)
// (vertex_shader.bwd, tile_shader_slang.py:128-150), evaluated in FP64.
__global__ void __launch_bounds__(256) project_bwd_kernel(const int4* __restrict__ indices,
                                                          const float* __restrict__ verts, int64_t n_tets,
                                                          int64_t n_verts, const rm_camera cam,
                                                          const int32_t* __restrict__ tiles,
                                                          const float* __restrict__ gvs,
                                                          const float* __restrict__ gcc,
                                                          float* __restrict__ gverts) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_tets) return;
    if (tiles[g] <= 0) return;
    const int4 id = __ldg(indices + g);
    if (!tet_indices_ok(id, n_verts)) return;  // culled by the forward
    const int ids[4] = {id.x, id.y, id.z, id.w};
    d3 X[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const f3 v = load_vertex(verts, ids[i]);
        X[i] = {(double)v.x, (double)v.y, (double)v.z};
    }
    const d3 P = {(double)cam.cam_pos[0], (double)cam.cam_pos[1], (double)cam.cam_pos[2]};
    d3 center;
    const double pw = power_of_circumsphere(X[0], X[1], X[2], X[3], P, center);
    const float pf = (float)pw;
    double gp = gvs ? (double)gvs[3 * g + 2] : 0.0;
    if (!(pf > -1e20f && pf < 1e20f)) gp = 0.0;
    const d3 gC = {gcc ? (double)gcc[3 * g] : 0.0, gcc ? (double)gcc[3 * g + 1] : 0.0,
                   gcc ? (double)gcc[3 * g + 2] : 0.0};
    if (gp == 0.0 && gC.x == 0.0 && gC.y == 0.0 && gC.z == 0.0) return;
    d3 G[4];
    const d3 a = X[1] - X[0], b = X[2] - X[0], c = X[3] - X[0];
    const d3 df = center - P;
    const d3 gcen = {gC.x + 2.0 * gp * df.x, gC.y + 2.0 * gp * df.y, gC.z + 2.0 * gp * df.z};
    const double den = 2.0 * dot3(a, cross3(b, c));
    if (fabs(den) < 1e-10) {
        int im = 0;
        double best = 1e300;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const double l = len3(X[i] - center);
            if (l < best) best = l, im = i;
        }
        const d3 ge = scale3(X[im] - center, -2.0 * gp);
        const d3 share = scale3(gcen - ge, 0.25);
#pragma unroll
        for (int i = 0; i < 4; ++i) G[i] = share;
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (i == im) G[i] = G[i] + ge;
    } else {
        const d3 cbc = cross3(b, c), cca = cross3(c, a), cab = cross3(a, b);
        const double aa = dot3(a, a), bb = dot3(b, b), cc2 = dot3(c, c);
        const d3 N = {aa * cbc.x + bb * cca.x + cc2 * cab.x, aa * cbc.y + bb * cca.y + cc2 * cab.y,
                      aa * cbc.z + bb * cca.z + cc2 * cab.z};
        const d3 rel = center - X[0];
        const d3 grel = {gcen.x - 2.0 * gp * rel.x, gcen.y - 2.0 * gp * rel.y, gcen.z - 2.0 * gp * rel.z};
        const d3 gN = scale3(grel, 1.0 / den);
        const double gden = -dot3(grel, N) / (den * den);
        const double gaa = dot3(gN, cbc), gbb = dot3(gN, cca), gcc = dot3(gN, cab);
        const d3 gcbc = scale3(gN, aa) + scale3(a, 2.0 * gden);
        const d3 gcca = scale3(gN, bb), gcab = scale3(gN, cc2);
        d3 ga = scale3(cbc, 2.0 * gden) + scale3(a, 2.0 * gaa);
        d3 gb = scale3(b, 2.0 * gbb);
        d3 gc = scale3(c, 2.0 * gcc);
        gb = gb + cross3(c, gcbc);
        gc = gc + cross3(gcbc, b);
        gc = gc + cross3(a, gcca);
        ga = ga + cross3(gcca, c);
        ga = ga + cross3(b, gcab);
        gb = gb + cross3(gcab, a);
        G[0] = gcen - ((ga + gb) + gc);
        G[1] = ga;
        G[2] = gb;
        G[3] = gc;
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) atomic_add3(gverts + 3 * (int64_t)ids[i], G[i]);
}

}  // namespace
}  // namespace rm

extern "C" {

int rm_project_fwd(const int32_t* indices, const float* vertices, int64_t n_tets, int64_t n_verts,
                   const rm_camera* cam, int32_t* tiles_touched, int32_t* rect, float* vs,
                   float* circumcenter, uint32_t* status_dev, void* stream) {
    int rc = rm_host::check_cam(cam);
    if (rc) return rc;
    if (n_tets < 0 || n_verts < 0) return rm_host::fail(RM_EINVAL, "rm_project_fwd: negative size");
    if (n_tets == 0) return RM_OK;
    if (!indices || !vertices || !tiles_touched || !rect || !vs || !circumcenter)
        return rm_host::fail(RM_EINVAL, "rm_project_fwd: NULL pointer");
    if (((uintptr_t)indices & 15) || ((uintptr_t)rect & 15))
        return rm_host::fail(RM_EINVAL, "rm_project_fwd: indices and rect must be 16-byte aligned");
    const int threads = 256;
    const int64_t blocks = (n_tets + threads - 1) / threads;
    auto kernel = rm_host::cam_general(*cam) ? rm::project_fwd_kernel<true> : rm::project_fwd_kernel<false>;
    kernel<<<(unsigned)blocks, threads, 0, (cudaStream_t)stream>>>(
        (const int4*)indices, vertices, n_tets, n_verts, *cam, tiles_touched, (int4*)rect, vs, circumcenter,
        status_dev);
    return rm_host::check_launch("rm_project_fwd");
}

int rm_project_fwd_fine(const int32_t* indices, const float* vertices, int64_t n_tets, int64_t n_verts,
                        const rm_camera* cam, int32_t* tiles_touched, int32_t* rect, float* vs, float* circumcenter,
                        float* footprint, uint32_t* status_dev, void* stream) {
    int rc = rm_host::check_cam(cam);
    if (rc) return rc;
    if (n_tets < 0 || n_verts < 0) return rm_host::fail(RM_EINVAL, "rm_project_fwd_fine: negative size");
    if (n_tets == 0) return RM_OK;
    if (!indices || !vertices || !tiles_touched || !rect || !vs || !circumcenter || !footprint)
        return rm_host::fail(RM_EINVAL, "rm_project_fwd_fine: NULL pointer");
    if (((uintptr_t)indices & 15) || ((uintptr_t)rect & 15) || ((uintptr_t)footprint & 15))
        return rm_host::fail(RM_EINVAL, "rm_project_fwd_fine: indices, rect and footprint must be 16-byte aligned");
    const int threads = 256;
    const int64_t blocks = (n_tets + threads - 1) / threads;
    auto kernel =
        rm_host::cam_general(*cam) ? rm::project_fwd_fine_kernel<true> : rm::project_fwd_fine_kernel<false>;
    kernel<<<(unsigned)blocks, threads, 0, (cudaStream_t)stream>>>(
        (const int4*)indices, vertices, n_tets, n_verts, *cam, tiles_touched, (int4*)rect, vs, circumcenter,
        (float4*)footprint, status_dev);
    return rm_host::check_launch("rm_project_fwd_fine");
}

int rm_project_fwd_multi(const int32_t* indices, const float* vertices, int64_t n_tets, int64_t n_verts,
                         const rm_camera* cams, int n_views, int32_t* tiles_touched, int32_t* rect, float* depth,
                         int32_t* tiles_any, float* circumcenter, float* footprint, uint32_t* status_dev,
                         void* stream) {
    rm::ViewSet views;
    int rc = rm_host::make_views("rm_project_fwd_multi", cams, n_views, &views);
    if (rc) return rc;
    if (n_tets < 0 || n_verts < 0) return rm_host::fail(RM_EINVAL, "rm_project_fwd_multi: negative size");
    if (n_tets == 0) return RM_OK;
    if (!indices || !vertices || !tiles_touched || !rect || !depth)
        return rm_host::fail(RM_EINVAL, "rm_project_fwd_multi: NULL pointer");
    if (((uintptr_t)indices & 15) || ((uintptr_t)rect & 15) || ((uintptr_t)footprint & 15))
        return rm_host::fail(RM_EINVAL, "rm_project_fwd_multi: indices, rect and footprint must be 16-byte aligned");
    const int threads = 256;
    const int64_t blocks = (n_tets + threads - 1) / threads;
    bool general = false;
    for (int v = 0; v < n_views; ++v) general |= rm_host::cam_general(cams[v]);
    auto kernel = general ? rm::project_fwd_multi_kernel<true> : rm::project_fwd_multi_kernel<false>;
    kernel<<<(unsigned)blocks, threads, 0, (cudaStream_t)stream>>>(
        (const int4*)indices, vertices, n_tets, n_verts, views, tiles_touched, (int4*)rect, depth, tiles_any,
        circumcenter, (float4*)footprint, status_dev);
    return rm_host::check_launch("rm_project_fwd_multi");
}

int rm_project_bwd(const int32_t* indices, const float* vertices, int64_t n_tets, int64_t n_verts,
                   const rm_camera* cam, const int32_t* tiles_touched, const float* grad_vs,
                   const float* grad_circumcenter, float* grad_vertices, void* stream) {
    int rc = rm_host::check_cam(cam);
    if (rc) return rc;
    if (n_tets < 0 || n_verts < 0) return rm_host::fail(RM_EINVAL, "rm_project_bwd: negative size");
    if (n_tets == 0 || (!grad_vs && !grad_circumcenter)) return RM_OK;
    if (!indices || !vertices || !tiles_touched || !grad_vertices)
        return rm_host::fail(RM_EINVAL, "rm_project_bwd: NULL pointer");
    if ((uintptr_t)indices & 15) return rm_host::fail(RM_EINVAL, "rm_project_bwd: indices must be 16-byte aligned");
    const int threads = 256;
    const int64_t blocks = (n_tets + threads - 1) / threads;
    rm::project_bwd_kernel<<<(unsigned)blocks, threads, 0, (cudaStream_t)stream>>>(
        (const int4*)indices, vertices, n_tets, n_verts, *cam, tiles_touched, grad_vs, grad_circumcenter,
        grad_vertices);
    return rm_host::check_launch("rm_project_bwd");
}

}  // extern "C"
