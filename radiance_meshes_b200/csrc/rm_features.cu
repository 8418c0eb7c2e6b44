// rm_features.cu - the per-tet feature producer that runs before the blend
// on every frame: activate_output (utils/model_util.py:93-105) with
// offset_normalize (:82-91), compute_vertex_colors_from_field (:66-79) and
// eval_sh (utils/eval_sh_py.py:138-200), fused into one pass per tet, and its
// adjoint.  One thread per tet: 4 vertex gathers, the circumcenter, the raw
// attributes and the SH coefficients in, the 7 cell values out.
//
// Per tet (rgb, grd, density, sh_rest, circumcenter cc, vertices v0..v3):
//   m      = min(rgb)                          g  = grd * m
//   r      = |v0 - cc|                         ng = safe_div(g, r)
//   c0     = rgb + dot(ng, v0 - cc)            (the same offset on all channels)
//   dir    = normalize(mean(v) - camera, eps 1e-8)
//   col    = C0 * (c0 - 0.5) / C0 + 0.5 + sum_k Y_k(dir) sh_rest[k]
//   base   = softplus(col, beta 10, threshold 20)
//   out    = (density, base, ng)
// As in the reference, v0 - cc inside c0 carries no gradient (its vertices
// and circumcenter are detached there); r and the mean do.
#include "rm_internal.cuh"

namespace rm {
namespace {

constexpr double kC0 = 0.28209479177387814;

// Forward-mode dual numbers over (x, y, z): the SH basis values and their
// gradients come from one evaluation of the basis polynomials.
struct D3 {
    float v, dx, dy, dz;
};
__device__ __forceinline__ D3 dconst(float c) { return {c, 0.f, 0.f, 0.f}; }
__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return {a.v + b.v, a.dx + b.dx, a.dy + b.dy, a.dz + b.dz}; }
__device__ __forceinline__ D3 operator-(D3 a, D3 b) { return {a.v - b.v, a.dx - b.dx, a.dy - b.dy, a.dz - b.dz}; }
__device__ __forceinline__ D3 operator*(D3 a, D3 b) {
    return {a.v * b.v, a.dx * b.v + a.v * b.dx, a.dy * b.v + a.v * b.dy, a.dz * b.v + a.v * b.dz};
}
__device__ __forceinline__ D3 operator*(float c, D3 a) { return {c * a.v, c * a.dx, c * a.dy, c * a.dz}; }

// Real SH basis of degree 1..4 (the published constants of the
// "hardcoded SH polynomials" evaluation), in the reference's row order and
// sign convention; k indexes sh_rest rows.
template <int DEG>
__device__ __forceinline__ void sh_basis(D3 x, D3 y, D3 z, D3* Y) {
    Y[0] = -0.4886025119029199f * y;
    Y[1] = 0.4886025119029199f * z;
    Y[2] = -0.4886025119029199f * x;
    if (DEG > 1) {
        const D3 xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
        Y[3] = 1.0925484305920792f * xy;
        Y[4] = -1.0925484305920792f * yz;
        Y[5] = 0.31539156525252005f * (2.0f * zz - xx - yy);
        Y[6] = -1.0925484305920792f * xz;
        Y[7] = 0.5462742152960396f * (xx - yy);
        if (DEG > 2) {
            Y[8] = -0.5900435899266435f * y * (3.0f * xx - yy);
            Y[9] = 2.890611442640554f * xy * z;
            Y[10] = -0.4570457994644658f * y * (4.0f * zz - xx - yy);
            Y[11] = 0.3731763325901154f * z * (2.0f * zz - 3.0f * xx - 3.0f * yy);
            Y[12] = -0.4570457994644658f * x * (4.0f * zz - xx - yy);
            Y[13] = 1.445305721320277f * z * (xx - yy);
            Y[14] = -0.5900435899266435f * x * (xx - 3.0f * yy);
            if (DEG > 3) {
                Y[15] = 2.5033429417967046f * xy * (xx - yy);
                Y[16] = -1.7701307697799304f * yz * (3.0f * xx - yy);
                Y[17] = 0.9461746957575601f * xy * (7.0f * zz - dconst(1.f));
                Y[18] = -0.6690465435572892f * yz * (7.0f * zz - dconst(3.f));
                Y[19] = 0.10578554691520431f * (zz * (35.0f * zz - dconst(30.f)) + dconst(3.f));
                Y[20] = -0.6690465435572892f * xz * (7.0f * zz - dconst(3.f));
                Y[21] = 0.47308734787878004f * (xx - yy) * (7.0f * zz - dconst(1.f));
                Y[22] = -1.7701307697799304f * xz * (xx - 3.0f * yy);
                Y[23] = 0.6258357354491761f * (xx * (xx - 3.0f * yy) - yy * (3.0f * xx - yy));
            }
        }
    }
}

constexpr float kFltMax = 3.402823466e38f;
constexpr float kFltTiny = 1.175494351e-38f;

__device__ __forceinline__ f3 vload(const float* p, int i) {
    const float* q = p + 3 * (int64_t)i;
    return {__ldg(q), __ldg(q + 1), __ldg(q + 2)};
}

template <int DEG, bool BWD>
__global__ void __launch_bounds__(128) features_kernel(
    const int4* __restrict__ indices, const float* __restrict__ verts, int64_t n_verts, const float* __restrict__ ccs,
    const float* __restrict__ density, const float* __restrict__ rgb, const float* __restrict__ grd,
    const float* __restrict__ sh, int n_rest, f3 cam, int64_t n_tets, float* __restrict__ feat,
    const float* __restrict__ gfeat, float* __restrict__ g_density, float* __restrict__ g_rgb,
    float* __restrict__ g_grd, float* __restrict__ g_sh, float* __restrict__ g_verts, float* __restrict__ g_cc) {
    constexpr int kRest = (DEG + 1) * (DEG + 1) - 1;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_tets) return;
    const int4 id = __ldg(indices + t);
    if (!tet_indices_ok(id, n_verts)) {  // zero features, no gradients; the vertices are never read
        if (!BWD) {
#pragma unroll
            for (int k = 0; k < 7; ++k) feat[7 * t + k] = 0.f;
        } else {
            g_density[t] = 0.f;
#pragma unroll
            for (int k = 0; k < 3; ++k) g_rgb[3 * t + k] = g_grd[3 * t + k] = g_cc[3 * t + k] = 0.f;
            for (int k = 0; k < 3 * n_rest; ++k) g_sh[(int64_t)3 * n_rest * t + k] = 0.f;
        }
        return;
    }
    if (BWD) {  // a tet that nothing downstream used (e.g. one outside the view): zero gradients, no atomics
        const float* gf = gfeat + 7 * t;
        bool zero = true;
#pragma unroll
        for (int k = 0; k < 7; ++k) zero &= __ldg(gf + k) == 0.f;
        if (zero) {
            g_density[t] = 0.f;
#pragma unroll
            for (int k = 0; k < 3; ++k) g_rgb[3 * t + k] = g_grd[3 * t + k] = g_cc[3 * t + k] = 0.f;
            for (int k = 0; k < 3 * n_rest; ++k) g_sh[(int64_t)3 * n_rest * t + k] = 0.f;
            return;
        }
    }
    const int vid[4] = {id.x, id.y, id.z, id.w};
    f3 v[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) v[i] = vload(verts, vid[i]);
    const f3 c = {__ldg(ccs + 3 * t), __ldg(ccs + 3 * t + 1), __ldg(ccs + 3 * t + 2)};
    float col_in[3], gr[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        col_in[k] = __ldg(rgb + 3 * t + k);
        gr[k] = __ldg(grd + 3 * t + k);
    }
    // offset_normalize
    int kmin = 0;
    float m = col_in[0];
    if (col_in[1] < m) m = col_in[1], kmin = 1;
    if (col_in[2] < m) m = col_in[2], kmin = 2;
    const f3 g = {gr[0] * m, gr[1] * m, gr[2] * m};
    const f3 e0 = v[0] - c;
    const float r = sqrtf(dot3(e0, e0));
    const bool small = fabsf(r) < kFltTiny;
    const float rnz = small ? kFltTiny : r;
    f3 ng = {fminf(fmaxf(g.x / rnz, -kFltMax), kFltMax), fminf(fmaxf(g.y / rnz, -kFltMax), kFltMax),
             fminf(fmaxf(g.z / rnz, -kFltMax), kFltMax)};
    if (small) ng = {0.f, 0.f, 0.f};
    const float off = dot3(ng, e0);
    float c0[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) c0[k] = col_in[k] + off;
    // eval_sh
    const f3 mean = scale3(((v[0] + v[1]) + v[2]) + v[3], 0.25f);
    const f3 u = mean - cam;
    const float un = sqrtf(dot3(u, u));
    const float ud = fmaxf(un, 1e-8f);
    const f3 dir = {u.x / ud, u.y / ud, u.z / ud};
    D3 Y[kRest > 0 ? kRest : 1];
    if (DEG > 0)
        sh_basis<DEG>({dir.x, 1.f, 0.f, 0.f}, {dir.y, 0.f, 1.f, 0.f}, {dir.z, 0.f, 0.f, 1.f}, Y);
    const float* shp = sh + (int64_t)n_rest * 3 * t;
    float col[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float sh0 = (c0[k] - 0.5f) / (float)kC0;
        float acc = (float)kC0 * sh0 + 0.5f;
        for (int j = 0; j < kRest; ++j) acc = acc + Y[j].v * __ldg(shp + 3 * j + k);
        col[k] = acc;
    }
    if (!BWD) {
        float* o = feat + 7 * t;
        o[0] = __ldg(density + t);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float bx = 10.f * col[k];
            o[1 + k] = bx > 20.f ? col[k] : log1pf(expf(bx)) / 10.f;
        }
        o[4] = ng.x;
        o[5] = ng.y;
        o[6] = ng.z;
        return;
    }
    // ---- adjoint
    const float* gf = gfeat + 7 * t;
    g_density[t] = __ldg(gf);
    float dcol[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float bx = 10.f * col[k];
        const float sig = bx > 20.f ? 1.f : 1.f / (1.f + expf(-bx));
        dcol[k] = __ldg(gf + 1 + k) * sig;
    }
    // sh_rest and the direction
    f3 ddir = {0.f, 0.f, 0.f};
    float* gsh = g_sh + (int64_t)n_rest * 3 * t;
    for (int j = 0; j < kRest; ++j) {
        float s = 0.f;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            gsh[3 * j + k] = dcol[k] * Y[j].v;
            s = fmaf(dcol[k], __ldg(shp + 3 * j + k), s);
        }
        ddir = {fmaf(s, Y[j].dx, ddir.x), fmaf(s, Y[j].dy, ddir.y), fmaf(s, Y[j].dz, ddir.z)};
    }
    for (int j = kRest; j < n_rest; ++j)
#pragma unroll
        for (int k = 0; k < 3; ++k) gsh[3 * j + k] = 0.f;
    // normalize(u, eps): (I - dir dir^T) / |u| above eps, I / eps below
    f3 du;
    if (un > 1e-8f) {
        const float p = dot3(ddir, dir);
        du = {(ddir.x - p * dir.x) / un, (ddir.y - p * dir.y) / un, (ddir.z - p * dir.z) / un};
    } else {
        du = {ddir.x / 1e-8f, ddir.y / 1e-8f, ddir.z / 1e-8f};
    }
    f3 gv[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) gv[i] = scale3(du, 0.25f);
    // c0 = rgb + dot(ng, e0) (e0 detached); col = C0 * (c0 - 0.5) / C0 + 0.5 + ...
    float grgb[3], dsum = 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float dc0 = dcol[k] * (float)kC0 / (float)kC0;
        grgb[k] = dc0;
        dsum += dc0;
    }
    f3 dng = {fmaf(dsum, e0.x, __ldg(gf + 4)), fmaf(dsum, e0.y, __ldg(gf + 5)), fmaf(dsum, e0.z, __ldg(gf + 6))};
    // ng = safe_div(g, r): dg = clamp(dng / r'), dr = sum clamp(-dng * ng / r')
    const f3 dg = {fminf(fmaxf(dng.x / rnz, -kFltMax), kFltMax), fminf(fmaxf(dng.y / rnz, -kFltMax), kFltMax),
                   fminf(fmaxf(dng.z / rnz, -kFltMax), kFltMax)};
    const float dr = fminf(fmaxf(-dng.x * ng.x / rnz, -kFltMax), kFltMax) +
                     fminf(fmaxf(-dng.y * ng.y / rnz, -kFltMax), kFltMax) +
                     fminf(fmaxf(-dng.z * ng.z / rnz, -kFltMax), kFltMax);
    // g = grd * m
    float* ogrd = g_grd + 3 * t;
    ogrd[0] = dg.x * m;
    ogrd[1] = dg.y * m;
    ogrd[2] = dg.z * m;
    grgb[kmin] += dot3(dg, mk3(gr[0], gr[1], gr[2]));
#pragma unroll
    for (int k = 0; k < 3; ++k) g_rgb[3 * t + k] = grgb[k];
    // r = |v0 - cc|
    if (r > 0.f) {
        const f3 gr0 = scale3(e0, dr / r);
        gv[0] = gv[0] + gr0;
        float* gcc = g_cc + 3 * t;
        gcc[0] = -gr0.x;
        gcc[1] = -gr0.y;
        gcc[2] = -gr0.z;
    } else {
        float* gcc = g_cc + 3 * t;
        gcc[0] = gcc[1] = gcc[2] = 0.f;
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        float* dst = g_verts + 3 * (int64_t)vid[i];
        atomicAdd(dst, gv[i].x);
        atomicAdd(dst + 1, gv[i].y);
        atomicAdd(dst + 2, gv[i].z);
    }
}

template <bool BWD>
int launch_features(int deg, const int32_t* indices, const float* vertices, int64_t n_verts, const float* ccs,
                    const float* density,
                    const float* rgb, const float* grd, const float* sh, int n_rest, const float* cam, int64_t T,
                    float* feat, const float* gfeat, float* gd, float* grgb, float* ggrd, float* gsh, float* gv,
                    float* gcc, cudaStream_t s) {
    const int threads = 128;
    const int64_t blocks = (T + threads - 1) / threads;
    const f3 c = {cam[0], cam[1], cam[2]};
#define RM_FEAT(D)                                                                                              \
    features_kernel<D, BWD><<<(unsigned)blocks, threads, 0, s>>>((const int4*)indices, vertices, n_verts, ccs,    \
                                                                 density,                                         \
                                                                 rgb, grd, sh, n_rest, c, T, feat, gfeat, gd,      \
                                                                 grgb, ggrd, gsh, gv, gcc)
    switch (deg) {
        case 0: RM_FEAT(0); break;
        case 1: RM_FEAT(1); break;
        case 2: RM_FEAT(2); break;
        case 3: RM_FEAT(3); break;
        default: RM_FEAT(4); break;
    }
#undef RM_FEAT
    return rm_host::check_launch(BWD ? "rm_activate_features_bwd" : "rm_activate_features");
}

int check_features(const char* who, const int32_t* indices, const float* vertices, const float* ccs,
                   const float* density, const float* rgb, const float* grd, const float* sh, int n_rest, int deg,
                   const float* cam, int64_t T) {
    if (T < 0) return rm_host::fail(RM_EINVAL, "%s: negative size", who);
    if (deg < 0 || deg > 4) return rm_host::fail(RM_EINVAL, "%s: SH degree %d (0..4)", who, deg);
    if (n_rest < (deg + 1) * (deg + 1) - 1)
        return rm_host::fail(RM_EINVAL, "%s: %d SH rows for degree %d", who, n_rest, deg);
    if (T == 0) return RM_OK;
    if (!indices || !vertices || !ccs || !density || !rgb || !grd || !cam || (n_rest > 0 && !sh))
        return rm_host::fail(RM_EINVAL, "%s: NULL pointer", who);
    if ((uintptr_t)indices & 15) return rm_host::fail(RM_EINVAL, "%s: indices must be 16-byte aligned", who);
    return RM_OK;
}

}  // namespace
}  // namespace rm

extern "C" {

int rm_activate_features(const int32_t* indices, const float* vertices, int64_t n_verts, const float* circumcenters,
                         const float* density, const float* rgb, const float* grd, const float* sh_rest, int n_rest,
                         int sh_degree, const float* camera_center, int64_t n_tets, float* features, void* stream) {
    int rc = rm::check_features("rm_activate_features", indices, vertices, circumcenters, density, rgb, grd, sh_rest,
                                n_rest, sh_degree, camera_center, n_tets);
    if (rc || n_tets == 0) return rc;
    if (!features) return rm_host::fail(RM_EINVAL, "rm_activate_features: NULL output");
    if (n_verts < 0) return rm_host::fail(RM_EINVAL, "rm_activate_features: negative vertex count");
    return rm::launch_features<false>(sh_degree, indices, vertices, n_verts, circumcenters, density, rgb, grd, sh_rest, n_rest,
                                      camera_center, n_tets, features, nullptr, nullptr, nullptr, nullptr, nullptr,
                                      nullptr, nullptr, (cudaStream_t)stream);
}

int rm_activate_features_bwd(const int32_t* indices, const float* vertices, int64_t n_verts,
                             const float* circumcenters,
                             const float* density, const float* rgb, const float* grd, const float* sh_rest,
                             int n_rest, int sh_degree, const float* camera_center, int64_t n_tets,
                             const float* grad_features, float* grad_density, float* grad_rgb, float* grad_grd,
                             float* grad_sh_rest, float* grad_vertices, float* grad_circumcenters, void* stream) {
    int rc = rm::check_features("rm_activate_features_bwd", indices, vertices, circumcenters, density, rgb, grd,
                                sh_rest, n_rest, sh_degree, camera_center, n_tets);
    if (rc || n_tets == 0) return rc;
    if (!grad_features || !grad_density || !grad_rgb || !grad_grd || !grad_vertices || !grad_circumcenters ||
        (n_rest > 0 && !grad_sh_rest))
        return rm_host::fail(RM_EINVAL, "rm_activate_features_bwd: NULL pointer");
    if (n_verts < 0) return rm_host::fail(RM_EINVAL, "rm_activate_features_bwd: negative vertex count");
    return rm::launch_features<true>(sh_degree, indices, vertices, n_verts, circumcenters, density, rgb, grd, sh_rest, n_rest,
                                     camera_center, n_tets, nullptr, grad_features, grad_density, grad_rgb, grad_grd,
                                     grad_sh_rest, grad_vertices, grad_circumcenters, (cudaStream_t)stream);
}

}  // extern "C"
