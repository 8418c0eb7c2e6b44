// rm_capi.cu - error reporting and shared host-side checks of the C ABI.
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "rm_internal.cuh"

namespace {
thread_local char g_last_error[512] = {0};
std::atomic<uint64_t> g_launches{0};
constexpr uint32_t kDefaultWaitLimit = 1u << 22;
std::atomic<uint32_t> g_wait_limit{kDefaultWaitLimit};
}

namespace rm_host {

int fail(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return code;
}

uint32_t wait_limit() { return g_wait_limit.load(std::memory_order_relaxed); }

int check_launch(const char* what, int kernels) {
    g_launches.fetch_add((uint64_t)kernels, std::memory_order_relaxed);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(RM_ECUDA, "%s: %s", what, cudaGetErrorString(e));
    return RM_OK;
}

int check_cam(const rm_camera* cam) {
    if (!cam) return fail(RM_EINVAL, "camera is NULL");
    if (cam->camera_type != 0 && cam->camera_type != 1)
        return fail(RM_EINVAL, "camera_type %d unsupported (0 perspective, 1 fisheye)", cam->camera_type);
    for (int i = 0; i < 4; ++i)
        if (!(cam->distortion[i] == cam->distortion[i])) return fail(RM_EINVAL, "distortion parameter is NaN");
    if (cam->tile_width <= 0 || cam->tile_height <= 0) return fail(RM_EINVAL, "bad tile size");
    if (cam->image_width <= 0 || cam->image_height <= 0) return fail(RM_EINVAL, "bad image size");
    if ((int64_t)cam->grid_width * cam->tile_width < cam->image_width ||
        (int64_t)cam->grid_height * cam->tile_height < cam->image_height)
        return fail(RM_EINVAL, "tile grid does not cover the image");
    if (cam->K[0] == 0.f || cam->K[4] == 0.f) return fail(RM_EINVAL, "zero focal length");
    return RM_OK;
}

int make_views(const char* who, const rm_camera* cams, int n, rm::ViewSet* out) {
    if (!cams) return fail(RM_EINVAL, "%s: cameras are NULL", who);
    if (n < 1 || n > RM_MAX_VIEWS) return fail(RM_EINVAL, "%s: %d views (1..%d)", who, n, RM_MAX_VIEWS);
    out->n = n;
    int64_t tiles = 0, pixels = 0;
    for (int v = 0; v < n; ++v) {
        int rc = check_cam(cams + v);
        if (rc) return rc;
        if (cams[v].tile_width != cams[0].tile_width || cams[v].tile_height != cams[0].tile_height)
            return fail(RM_EINVAL, "%s: view %d has another tile size than view 0", who, v);
        out->tiles[v] = (int)tiles;
        out->pixels[v] = pixels;
        out->cams[v] = cams[v];
        out->parallax[v] = parallax_px(cams[v]);
        tiles += (int64_t)cams[v].grid_width * cams[v].grid_height;
        pixels += (int64_t)cams[v].image_width * cams[v].image_height;
        if (tiles >= (1ll << 31)) return fail(RM_EINVAL, "%s: more than 2^31 tiles", who);
    }
    for (int v = n; v <= RM_MAX_VIEWS; ++v) {
        out->tiles[v] = (int)tiles;
        out->pixels[v] = pixels;
    }
    for (int v = n; v < RM_MAX_VIEWS; ++v) {
        out->cams[v] = cams[0];
        out->parallax[v] = out->parallax[0];
    }
    return RM_OK;
}

float parallax_px(const rm_camera& c) {
    const float* M = c.world_view;
    if (!(M[12] == 0.f && M[13] == 0.f && M[14] == 0.f && M[15] == 1.f)) return INFINITY;
    double R[3][3], t[3];
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) R[i][j] = M[4 * i + j];
        t[i] = M[4 * i + 3];
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            const double d = R[i][0] * R[j][0] + R[i][1] * R[j][1] + R[i][2] * R[j][2] - (i == j ? 1.0 : 0.0);
            if (!(std::fabs(d) <= 1e-5)) return INFINITY;  // not a rotation: rays and projection disagree
        }
    double off2 = 0.0;
    for (int j = 0; j < 3; ++j) {
        const double center = -(R[0][j] * t[0] + R[1][j] * t[1] + R[2][j] * t[2]);
        const double d = (double)c.cam_pos[j] - center;
        off2 += d * d;
    }
    if (off2 == 0.0) return 0.f;
    if (!(c.min_t > 0.f)) return INFINITY;
    const double f = std::fmax(std::fabs((double)c.K[0]), std::fabs((double)c.K[4]));
    return (float)(2.0 * f * std::sqrt(off2) / (double)c.min_t);
}

}  // namespace rm_host

extern "C" {

const char* rm_last_error(void) { return g_last_error; }

int rm_abi_version(void) { return RM_ABI_VERSION; }

uint64_t rm_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

void rm_set_wait_limit(uint32_t polls) {
    g_wait_limit.store(polls ? polls : kDefaultWaitLimit, std::memory_order_relaxed);
}

uint32_t rm_wait_limit(void) { return g_wait_limit.load(std::memory_order_relaxed); }

int rm_read_status(const uint32_t* status_dev, uint32_t* status_host, void* stream) {
    if (!status_dev || !status_host) return rm_host::fail(RM_EINVAL, "rm_read_status: NULL pointer");
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemcpyAsync(status_host, status_dev, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemsetAsync((void*)status_dev, 0, sizeof(uint32_t), s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return rm_host::fail(RM_ECUDA, "rm_read_status: %s", cudaGetErrorString(e));
    return RM_OK;
}

}  // extern "C"
