// rm_tets.cu - the steps of a Delaunay update that follow the
// tetrahedralisation itself (update_triangulation, models/ingp_color.py:523-558):
//
//   rm_tets_orient  drop rows with an index outside [0, n_verts) (the point at
//                   infinity of gDel3D, :533) and make every kept tet
//                   positively oriented by swapping its vertices 0 and 1 where
//                   the signed volume det(v1 - v0, v2 - v0, v3 - v0) / 6 is
//                   negative (:538-542, topo_utils.tet_volumes);
//   rm_tets_cull    split the tets into those kept (density > threshold or
//                   alpha > threshold, alpha = 1 - exp(-density * shortest
//                   edge), :548-554, base_model.py:82-105) and the empty ones.
//
// Both keep the input order in each output (as the reference's boolean
// indexing does): a flag pass, an inclusive scan of the flags (the decoupled
// look-back scan of rm_scan.cu) and a scatter pass.  The tetrahedralisation
// (gDel3D on the GPU, or scipy's Delaunay on the host in the reference's
// high-precision mode, :526-527) is not part of this library.
#include "rm_internal.cuh"

namespace rm {
namespace {

constexpr int kTetThreads = 256;

__device__ __forceinline__ f3 vload(const float* __restrict__ v, int i) {
    const float* p = v + 3 * (int64_t)i;
    return {__ldg(p), __ldg(p + 1), __ldg(p + 2)};
}

// Sign of det(v1 - v0, v2 - v0, v3 - v0), evaluated in double from the float
// vertices (exact up to double rounding; the reference takes the determinant
// in float32, so the two can disagree only for tets whose volume is at the
// float32 rounding level of their edge products).
__device__ __forceinline__ bool negative_volume(f3 v0, f3 v1, f3 v2, f3 v3) {
    const d3 a = {(double)v1.x - v0.x, (double)v1.y - v0.y, (double)v1.z - v0.z};
    const d3 b = {(double)v2.x - v0.x, (double)v2.y - v0.y, (double)v2.z - v0.z};
    const d3 c = {(double)v3.x - v0.x, (double)v3.y - v0.y, (double)v3.z - v0.z};
    return dot3(a, cross3(b, c)) < 0.0;
}

__global__ void __launch_bounds__(kTetThreads) orient_flags_kernel(const int4* __restrict__ idx, int64_t n,
                                                                  int64_t n_verts, int32_t* __restrict__ keep) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    keep[t] = tet_indices_ok(__ldg(idx + t), n_verts) ? 1 : 0;
}

__global__ void __launch_bounds__(kTetThreads) orient_scatter_kernel(const int4* __restrict__ idx, int64_t n,
                                                                    const float* __restrict__ verts,
                                                                    const int32_t* __restrict__ keep,
                                                                    const int32_t* __restrict__ incl,
                                                                    int4* __restrict__ out) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n || !keep[t]) return;
    int4 r = __ldg(idx + t);
    if (negative_volume(vload(verts, r.x), vload(verts, r.y), vload(verts, r.z), vload(verts, r.w))) {
        const int s = r.x;  // indices[:, [1, 0, 2, 3]]
        r.x = r.y;
        r.y = s;
    }
    out[incl[t] - 1] = r;
}

// alpha = 1 - exp(-density * shortest edge) with the edges' float32 norms,
// as calc_tet_alpha(mode="min") computes them.
__global__ void __launch_bounds__(kTetThreads) cull_flags_kernel(const int4* __restrict__ idx, int64_t n,
                                                                int64_t n_verts, const float* __restrict__ verts,
                                                                const float* __restrict__ density, float d_thr,
                                                                float a_thr, int32_t* __restrict__ keep,
                                                                uint32_t* status) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int4 r = __ldg(idx + t);
    if (!tet_indices_ok(r, n_verts)) {  // never dereferenced: reported, counted as empty
        if (status) atomicOr(status, RM_STATUS_BAD_INDEX);
        keep[t] = 0;
        return;
    }
    const f3 v[4] = {vload(verts, r.x), vload(verts, r.y), vload(verts, r.z), vload(verts, r.w)};
    const int ea[6] = {0, 0, 0, 1, 1, 2}, eb[6] = {1, 2, 3, 2, 3, 3};
    float el = INFINITY;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const f3 e = v[ea[k]] - v[eb[k]];
        el = fminf(el, sqrtf(e.x * e.x + e.y * e.y + e.z * e.z));
    }
    const float dens = __ldg(density + t);
    const float alpha = 1.0f - expf(-dens * el);
    keep[t] = (dens > d_thr || alpha > a_thr) ? 1 : 0;
}

__global__ void __launch_bounds__(kTetThreads) cull_scatter_kernel(const int4* __restrict__ idx, int64_t n,
                                                                  const int32_t* __restrict__ keep,
                                                                  const int32_t* __restrict__ incl,
                                                                  int4* __restrict__ kept, int4* __restrict__ empty) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int4 r = __ldg(idx + t);
    const int32_t c = incl[t];
    if (keep[t]) {
        kept[c - 1] = r;
    } else if (empty) {
        empty[t - c] = r;  // t + 1 - c empty rows up to and including t
    }
}

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

struct TetWs {
    int32_t* keep;
    int32_t* incl;
    void* scan;
    size_t scan_bytes;
};

TetWs tet_ws(void* base, int64_t n) {
    char* p = (char*)base;
    const size_t a = align256(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    return {(int32_t*)p, (int32_t*)(p + a), p + 2 * a, rm_scan_workspace_size(n)};
}

int check_tets(const char* who, const int32_t* idx, int64_t n, const float* verts, int64_t n_verts, void* ws,
               size_t ws_bytes) {
    if (n < 0 || n_verts < 0) return rm_host::fail(RM_EINVAL, "%s: negative size", who);
    if (n >= (int64_t)INT32_MAX) return rm_host::fail(RM_EINVAL, "%s: at most 2^31 - 1 tets", who);
    if (n > 0 && (!idx || !verts || !ws)) return rm_host::fail(RM_EINVAL, "%s: NULL pointer", who);
    if (((uintptr_t)idx & 15) || ((uintptr_t)ws & 255))
        return rm_host::fail(RM_EINVAL, "%s: indices must be 16-byte and the workspace 256-byte aligned", who);
    if (ws_bytes < rm_tets_workspace_size(n))
        return rm_host::fail(RM_EINVAL, "%s: workspace %zu < %zu bytes", who, ws_bytes, rm_tets_workspace_size(n));
    return RM_OK;
}

}  // namespace
}  // namespace rm

extern "C" {

size_t rm_tets_workspace_size(int64_t n_tets) {
    const size_t a = rm::align256(sizeof(int32_t) * (size_t)(n_tets > 0 ? n_tets : 1));
    return 2 * a + rm::align256(rm_scan_workspace_size(n_tets > 0 ? n_tets : 0));
}

int rm_tets_orient(const int32_t* indices_in, int64_t n_tets, const float* vertices, int64_t n_verts,
                   int32_t* indices_out, int64_t* n_out_dev, void* workspace, size_t workspace_bytes,
                   uint32_t* status_dev, void* stream) {
    using namespace rm;
    int rc = check_tets("rm_tets_orient", indices_in, n_tets, vertices, n_verts, workspace, workspace_bytes);
    if (rc) return rc;
    if (!n_out_dev || (n_tets > 0 && !indices_out)) return rm_host::fail(RM_EINVAL, "rm_tets_orient: NULL output");
    if ((uintptr_t)indices_out & 15) return rm_host::fail(RM_EINVAL, "rm_tets_orient: output must be 16-byte aligned");
    cudaStream_t s = (cudaStream_t)stream;
    if (n_tets == 0) {
        cudaError_t e = cudaMemsetAsync(n_out_dev, 0, sizeof(int64_t), s);
        return e == cudaSuccess ? RM_OK : rm_host::fail(RM_ECUDA, "rm_tets_orient: %s", cudaGetErrorString(e));
    }
    const TetWs w = tet_ws(workspace, n_tets);
    const unsigned blocks = (unsigned)((n_tets + kTetThreads - 1) / kTetThreads);
    orient_flags_kernel<<<blocks, kTetThreads, 0, s>>>((const int4*)indices_in, n_tets, n_verts, w.keep);
    if ((rc = rm_host::check_launch("rm_tets_orient (flags)"))) return rc;
    if ((rc = rm_host::scan_tiles_status(w.keep, n_tets, w.incl, n_out_dev, w.scan, w.scan_bytes, status_dev, s)))
        return rc;
    orient_scatter_kernel<<<blocks, kTetThreads, 0, s>>>((const int4*)indices_in, n_tets, vertices, w.keep, w.incl,
                                                         (int4*)indices_out);
    return rm_host::check_launch("rm_tets_orient (scatter)");
}

int rm_tets_cull(const int32_t* indices, int64_t n_tets, const float* vertices, int64_t n_verts,
                 const float* density, float density_threshold, float alpha_threshold, int32_t* kept_out,
                 int32_t* empty_out, int64_t* n_kept_dev, void* workspace, size_t workspace_bytes,
                 uint32_t* status_dev, void* stream) {
    using namespace rm;
    int rc = check_tets("rm_tets_cull", indices, n_tets, vertices, n_verts, workspace, workspace_bytes);
    if (rc) return rc;
    if (!n_kept_dev || (n_tets > 0 && (!kept_out || !density)))
        return rm_host::fail(RM_EINVAL, "rm_tets_cull: NULL pointer");
    if (((uintptr_t)kept_out & 15) || ((uintptr_t)empty_out & 15))
        return rm_host::fail(RM_EINVAL, "rm_tets_cull: outputs must be 16-byte aligned");
    cudaStream_t s = (cudaStream_t)stream;
    if (n_tets == 0) {
        cudaError_t e = cudaMemsetAsync(n_kept_dev, 0, sizeof(int64_t), s);
        return e == cudaSuccess ? RM_OK : rm_host::fail(RM_ECUDA, "rm_tets_cull: %s", cudaGetErrorString(e));
    }
    const TetWs w = tet_ws(workspace, n_tets);
    const unsigned blocks = (unsigned)((n_tets + kTetThreads - 1) / kTetThreads);
    cull_flags_kernel<<<blocks, kTetThreads, 0, s>>>((const int4*)indices, n_tets, n_verts, vertices, density,
                                                     density_threshold, alpha_threshold, w.keep, status_dev);
    if ((rc = rm_host::check_launch("rm_tets_cull (flags)"))) return rc;
    if ((rc = rm_host::scan_tiles_status(w.keep, n_tets, w.incl, n_kept_dev, w.scan, w.scan_bytes, status_dev, s)))
        return rc;
    cull_scatter_kernel<<<blocks, kTetThreads, 0, s>>>((const int4*)indices, n_tets, w.keep, w.incl,
                                                       (int4*)kept_out, (int4*)empty_out);
    return rm_host::check_launch("rm_tets_cull (scatter)");
}

}  // extern "C"
