// capi.cu -- the extern "C" entry points declared in include/pyronn_b200.h.
//
// Each entry point validates its arguments on the host, prepares geometry on
// the device (no host round trip, unlike the reference's blocking D2H copies),
// and enqueues the kernels on the caller's stream.  Errors come back as
// status codes with a per-thread message; nothing exits the process.
#include <stdarg.h>
#include <stdio.h>

#include <string>

#include "internal.h"

namespace pyronn {

size_t dtype_size(int dtype)
{
    switch (dtype) {
    case PYRONN_FLOAT32: return 4;
    case PYRONN_BFLOAT16: return 2;
    case PYRONN_FLOAT16: return 2;
    default: return 0;
    }
}

}  // namespace pyronn

using namespace pyronn;

namespace {
int fail(int status, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
int cuda_fail(cudaError_t e, const char *what);
}  // namespace

namespace pyronn {

int report_error(int status, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return fail(status, "%s", buf);
}

int report_cuda_error(cudaError_t e, const char *what)
{
    return cuda_fail(e, what);
}

}  // namespace pyronn

namespace {

thread_local std::string t_last_error;

int fail(int status, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    t_last_error = buf;
    return status;
}

int ok()
{
    t_last_error.clear();
    return PYRONN_SUCCESS;
}

int cuda_fail(cudaError_t e, const char *what)
{
    return fail(PYRONN_ERROR_CUDA, "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
}

size_t align_up(size_t n, size_t a)
{
    return (n + a - 1) / a * a;
}

// every cone workspace starts with a header whose first word is the device
// error flag of the call (pyronn::DeviceError), cleared at the start of the call
constexpr size_t WS_HEADER = 256;

bool valid_dtype(int dtype)
{
    return dtype == PYRONN_FLOAT32 || dtype == PYRONN_BFLOAT16 || dtype == PYRONN_FLOAT16;
}

int check_common(int in_dtype, int out_dtype, int batch, int geom_batch)
{
    if (!valid_dtype(in_dtype)) return fail(PYRONN_ERROR_INVALID_ARGUMENT, "unknown in_dtype %d", in_dtype);
    if (!valid_dtype(out_dtype)) return fail(PYRONN_ERROR_INVALID_ARGUMENT, "unknown out_dtype %d", out_dtype);
    if (batch <= 0) return fail(PYRONN_ERROR_INVALID_ARGUMENT, "batch must be positive (got %d)", batch);
    if (geom_batch != 1 && geom_batch != batch)
        return fail(PYRONN_ERROR_INVALID_ARGUMENT, "geom_batch must be 1 or batch (%d), got %d", batch, geom_batch);
    return PYRONN_SUCCESS;
}

int check_dims(const char *what, long long a, long long b, long long c, long long d)
{
    if (a <= 0 || b <= 0 || c <= 0 || d <= 0)
        return fail(PYRONN_ERROR_INVALID_ARGUMENT, "%s: every dimension must be positive", what);
    return PYRONN_SUCCESS;
}

// per-batch-element element counts are indexed with 32-bit integers
int check_elements(const char *what, long long n)
{
    if (n >= (1LL << 31) - (1LL << 20))
        return fail(PYRONN_ERROR_UNSUPPORTED, "%s: %lld elements per batch element exceed the 2^31 limit", what, n);
    return PYRONN_SUCCESS;
}

int check_texture_3d(int w, int h, int d)
{
    int dev = 0, mw = 0, mh = 0, md = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&mw, cudaDevAttrMaxTexture3DWidth, dev);
    cudaDeviceGetAttribute(&mh, cudaDevAttrMaxTexture3DHeight, dev);
    cudaDeviceGetAttribute(&md, cudaDevAttrMaxTexture3DDepth, dev);
    if (w > mw || h > mh || d > md || d > 65535 || h > 65535)
        return fail(PYRONN_ERROR_UNSUPPORTED, "hardware_interp: volume %dx%dx%d exceeds the 3D texture limit %dx%dx%d",
                    w, h, d, mw, mh, md);
    return PYRONN_SUCCESS;
}

int check_texture_layered(int w, int h, int layers)
{
    int dev = 0, mw = 0, mh = 0, ml = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&mw, cudaDevAttrMaxTexture2DLayeredWidth, dev);
    cudaDeviceGetAttribute(&mh, cudaDevAttrMaxTexture2DLayeredHeight, dev);
    cudaDeviceGetAttribute(&ml, cudaDevAttrMaxTexture2DLayeredLayers, dev);
    if (w > mw || h > mh || layers > ml || h > 65535)
        return fail(PYRONN_ERROR_UNSUPPORTED,
                    "hardware_interp: sinogram %d views of %dx%d exceeds the layered texture limit %d of %dx%d",
                    layers, w, h, ml, mw, mh);
    return PYRONN_SUCCESS;
}

int run_2d(bool forward, bool fan, const void *in, void *out, int in_dtype, int out_dtype, const Dims2D &d,
           const Geom2D &g, void *workspace, size_t workspace_bytes, void *stream)
{
    const char *name = forward ? (fan ? "fan_projection2d" : "parallel_projection2d")
                               : (fan ? "fan_backprojection2d" : "parallel_backprojection2d");
    int st = check_common(in_dtype, out_dtype, d.batch, d.geom_batch);
    if (st) return st;
    if (!in || !out) return fail(PYRONN_ERROR_INVALID_ARGUMENT, "%s: null data pointer", name);
    if (!g.volume_origin || !g.detector_origin || !g.volume_spacing || !g.detector_spacing || !g.rays ||
        (fan && (!g.sid || !g.sdd)))
        return fail(PYRONN_ERROR_INVALID_ARGUMENT, "%s: null geometry pointer", name);
    st = check_dims(name, d.vol_y, d.vol_x, d.n_proj, d.det_w);
    if (st) return st;
    if (d.n_proj > 65535) return fail(PYRONN_ERROR_UNSUPPORTED, "%s: more than 65535 views", name);
    if (d.batch > 65535) return fail(PYRONN_ERROR_UNSUPPORTED, "%s: batch above 65535", name);
    st = check_elements(name, (long long)d.vol_y * d.vol_x);
    if (st) return st;
    st = check_elements(name, (long long)d.n_proj * d.det_w);
    if (st) return st;
    void *cells = nullptr;
    if (forward && workspace) {
        const size_t need = pyronn_projection2d_workspace_size(d.batch, d.vol_y, d.vol_x, in_dtype);
        if (workspace_bytes < need)
            return fail(PYRONN_ERROR_WORKSPACE_TOO_SMALL, "%s: workspace of %zu bytes needed, %zu given", name, need,
                        workspace_bytes);
        if (((uintptr_t)workspace) % 16 != 0)
            return fail(PYRONN_ERROR_INVALID_ARGUMENT, "%s: workspace must be 16-byte aligned", name);
        cells = workspace;
    }
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = forward ? launch_projection2d(in, out, in_dtype, out_dtype, fan, d, g, cells, s)
                            : launch_backprojection2d(in, out, in_dtype, out_dtype, fan, d, g, s);
    if (e != cudaSuccess) return cuda_fail(e, name);
    return ok();
}

int check_cone(const char *name, const void *in, const void *out, int in_dtype, int out_dtype, const Dims3D &d,
               const float *origin, const float *spacing, const float *P, const float *step, const float *mult)
{
    int st = check_common(in_dtype, out_dtype, d.batch, d.geom_batch);
    if (st) return st;
    if (!in || !out) return fail(PYRONN_ERROR_INVALID_ARGUMENT, "%s: null data pointer", name);
    if (!origin || !spacing || !P || !step || !mult)
        return fail(PYRONN_ERROR_INVALID_ARGUMENT, "%s: null geometry pointer", name);
    st = check_dims(name, d.vol_z, d.vol_y, d.vol_x, d.n_proj);
    if (st) return st;
    st = check_dims(name, d.det_h, d.det_w, 1, 1);
    if (st) return st;
    st = check_elements(name, (long long)d.vol_z * d.vol_y * d.vol_x);
    if (st) return st;
    st = check_elements(name, (long long)d.n_proj * d.det_h * d.det_w + d.det_w + 1);
    if (st) return st;
    if (d.det_h > 65535 * 8 || d.vol_y > 65535 * 4)
        return fail(PYRONN_ERROR_UNSUPPORTED, "%s: grid dimension limit exceeded", name);
    if (d.n_proj > 65535) return fail(PYRONN_ERROR_UNSUPPORTED, "%s: more than 65535 views", name);
    return PYRONN_SUCCESS;
}

}  // namespace

extern "C" {

int pyronn_abi_version(void)
{
    return PYRONN_B200_ABI_VERSION;
}

const char *pyronn_status_string(int status)
{
    switch (status) {
    case PYRONN_SUCCESS: return "success";
    case PYRONN_ERROR_INVALID_ARGUMENT: return "invalid argument";
    case PYRONN_ERROR_UNSUPPORTED: return "unsupported";
    case PYRONN_ERROR_WORKSPACE_TOO_SMALL: return "workspace too small";
    case PYRONN_ERROR_CUDA: return "CUDA error";
    default: return "unknown status";
    }
}

const char *pyronn_last_error(void)
{
    return t_last_error.c_str();
}

int pyronn_debug_starve_tma_wait(int enable)
{
    cone_bp_tma_starve_last_pass(enable);
    return ok();
}

int pyronn_fdk_error(void *stream, int *device_error)
{
    if (!device_error) return fail(PYRONN_ERROR_INVALID_ARGUMENT, "fdk_error: null pointer");
    unsigned flag = 0;
    cudaError_t e = fdk_tc_error((cudaStream_t)stream, &flag);
    if (e != cudaSuccess) return cuda_fail(e, "fdk_error");
    *device_error = (int)flag;
    return ok();
}

int pyronn_release_cached_arrays(void)
{
    const int freed = array_cache_clear();
    if (freed < 0) return fail(PYRONN_ERROR_CUDA, "release_cached_arrays: device synchronise failed");
    return ok();
}

size_t pyronn_projection2d_workspace_size(int batch, int vol_y, int vol_x, int in_dtype)
{
    if (batch <= 0 || vol_y <= 0 || vol_x <= 0 || !valid_dtype(in_dtype)) return 0;
    // two copies of the batch as bilinear cells (4 FP32 taps each, whatever
    // the storage type; zero border of two cells below and one above)
    return 2 * align_up((size_t)batch * (vol_y + 3) * (vol_x + 3) * 4 * sizeof(float), 256);
}

int pyronn_parallel_projection2d(const void *volume, void *sinogram, int in_dtype, int out_dtype, int batch, int vol_y, int vol_x,
                                 int n_proj, int det_w, const float *volume_origin, const float *detector_origin,
                                 const float *volume_spacing, const float *detector_spacing, const float *ray_vectors,
                                 int geom_batch, void *workspace, size_t workspace_bytes, void *stream)
{
    const Dims2D d{batch, vol_y, vol_x, n_proj, det_w, geom_batch};
    const Geom2D g{volume_origin, detector_origin, volume_spacing, detector_spacing, ray_vectors, nullptr, nullptr};
    return run_2d(true, false, volume, sinogram, in_dtype, out_dtype, d, g, workspace, workspace_bytes, stream);
}

int pyronn_parallel_backprojection2d(const void *sinogram, void *volume, int in_dtype, int out_dtype, int batch, int n_proj, int det_w,
                                     int vol_y, int vol_x, const float *volume_origin, const float *detector_origin,
                                     const float *volume_spacing, const float *detector_spacing,
                                     const float *ray_vectors, int geom_batch, void *stream)
{
    const Dims2D d{batch, vol_y, vol_x, n_proj, det_w, geom_batch};
    const Geom2D g{volume_origin, detector_origin, volume_spacing, detector_spacing, ray_vectors, nullptr, nullptr};
    return run_2d(false, false, sinogram, volume, in_dtype, out_dtype, d, g, nullptr, 0, stream);
}

int pyronn_fan_projection2d(const void *volume, void *sinogram, int in_dtype, int out_dtype, int batch, int vol_y, int vol_x,
                            int n_proj, int det_w, const float *volume_origin, const float *detector_origin,
                            const float *volume_spacing, const float *detector_spacing,
                            const float *source_2_isocenter_distance, const float *source_2_detector_distance,
                            const float *central_ray_vectors, int geom_batch, void *workspace,
                            size_t workspace_bytes, void *stream)
{
    const Dims2D d{batch, vol_y, vol_x, n_proj, det_w, geom_batch};
    const Geom2D g{volume_origin, detector_origin, volume_spacing, detector_spacing, central_ray_vectors,
                   source_2_isocenter_distance, source_2_detector_distance};
    return run_2d(true, true, volume, sinogram, in_dtype, out_dtype, d, g, workspace, workspace_bytes, stream);
}

int pyronn_fan_backprojection2d(const void *sinogram, void *volume, int in_dtype, int out_dtype, int batch, int n_proj, int det_w,
                                int vol_y, int vol_x, const float *volume_origin, const float *detector_origin,
                                const float *volume_spacing, const float *detector_spacing,
                                const float *source_2_isocenter_distance, const float *source_2_detector_distance,
                                const float *central_ray_vectors, int geom_batch, void *stream)
{
    const Dims2D d{batch, vol_y, vol_x, n_proj, det_w, geom_batch};
    const Geom2D g{volume_origin, detector_origin, volume_spacing, detector_spacing, central_ray_vectors,
                   source_2_isocenter_distance, source_2_detector_distance};
    return run_2d(false, true, sinogram, volume, in_dtype, out_dtype, d, g, nullptr, 0, stream);
}

size_t pyronn_cone_projection3d_workspace_size(int batch, int vol_z, int vol_y, int vol_x, int n_proj, int det_h,
                                               int det_w, int in_dtype, int hardware_interp, int geom_batch)
{
    if (geom_batch <= 0 || n_proj <= 0 || batch <= 0 || vol_z <= 0 || vol_y <= 0 || vol_x <= 0 ||
        !valid_dtype(in_dtype))
        return 0;
    size_t n = WS_HEADER + align_up((size_t)geom_batch * n_proj * sizeof(ConeFpView), 256);
    const Dims3D d{batch, vol_z, vol_y, vol_x, n_proj, det_h, det_w, geom_batch};
    if (!hardware_interp && cone_fp_padded_supported(d))
        n += align_up(cone_fp_padded_scratch_bytes(vol_z, vol_y, vol_x, in_dtype), 256);
    return n;
}

size_t pyronn_cone_backprojection3d_workspace_size(int batch, int n_proj, int det_h, int det_w, int vol_z, int vol_y,
                                                   int vol_x, int in_dtype, int hardware_interp, int geom_batch)
{
    if (geom_batch <= 0 || n_proj <= 0 || !valid_dtype(in_dtype)) return 0;
    const size_t views = WS_HEADER + align_up((size_t)geom_batch * n_proj * sizeof(ConeBpView), 256);
    if (hardware_interp || batch <= 0 || det_h <= 0 || det_w <= 0) return views;
    // 16-bit sinograms: room for the paired copy the TMA path reads (a
    // workspace of `views` bytes alone is accepted, without the pairing)
    const Dims3D d{batch, vol_z, vol_y, vol_x, n_proj, det_h, det_w, geom_batch};
    return views + align_up(cone_bp_tma_paired_bytes(in_dtype, d), 256);
}

int pyronn_workspace_error(const void *workspace, void *stream, int *device_error)
{
    if (!workspace || !device_error) return fail(PYRONN_ERROR_INVALID_ARGUMENT, "workspace_error: null pointer");
    unsigned flag = 0;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemcpyAsync(&flag, workspace, sizeof(flag), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "workspace_error");
    *device_error = (int)flag;
    return ok();
}

int pyronn_cone_projection3d(const void *volume, void *sinogram, int in_dtype, int out_dtype, int hardware_interp, int batch, int vol_z,
                             int vol_y, int vol_x, int n_proj, int det_h, int det_w, const float *volume_origin,
                             const float *volume_spacing, const float *projection_matrices, const float *step_size,
                             const float *projection_multiplier, int geom_batch, void *workspace,
                             size_t workspace_bytes, void *stream)
{
    const char *name = "cone_projection3d";
    const Dims3D d{batch, vol_z, vol_y, vol_x, n_proj, det_h, det_w, geom_batch};
    int st = check_cone(name, volume, sinogram, in_dtype, out_dtype, d, volume_origin, volume_spacing, projection_matrices,
                        step_size, projection_multiplier);
    if (st) return st;
    const size_t need = pyronn_cone_projection3d_workspace_size(batch, vol_z, vol_y, vol_x, n_proj, det_h, det_w,
                                                                in_dtype, hardware_interp, geom_batch);
    if (!workspace || workspace_bytes < need)
        return fail(PYRONN_ERROR_WORKSPACE_TOO_SMALL, "%s: workspace of %zu bytes needed, %zu given", name, need,
                    workspace ? workspace_bytes : (size_t)0);
    if (((uintptr_t)workspace) % 16 != 0)
        return fail(PYRONN_ERROR_INVALID_ARGUMENT, "%s: workspace must be 16-byte aligned", name);
    if (hardware_interp) {
        st = check_texture_3d(vol_x, vol_y, vol_z);
        if (st) return st;
    }
    cudaStream_t s = (cudaStream_t)stream;
    ConeFpView *views = (ConeFpView *)((char *)workspace + WS_HEADER);
    cudaError_t e = cudaMemsetAsync(workspace, 0, WS_HEADER, s);
    if (e != cudaSuccess) return cuda_fail(e, "cone_projection3d: workspace header");
    e = launch_cone_fp_prepare(projection_matrices, volume_spacing, volume_origin, geom_batch, n_proj, vol_x, vol_y,
                               vol_z, views, s);
    if (e != cudaSuccess) return cuda_fail(e, "cone_projection3d: geometry preparation");
    if (!hardware_interp) {
        if (cone_fp_padded_supported(d)) {
            void *scratch = (char *)workspace + WS_HEADER +
                            align_up((size_t)geom_batch * n_proj * sizeof(ConeFpView), 256);
            e = launch_cone_fp_padded(volume, sinogram, in_dtype, out_dtype, d, views, step_size, volume_spacing,
                                      scratch, (unsigned *)workspace, s);
        } else {
            e = launch_cone_fp(volume, sinogram, in_dtype, out_dtype, d, -1, views, step_size, volume_spacing, 0, s);
        }
        if (e != cudaSuccess) return cuda_fail(e, name);
        return ok();
    }
    CachedArray *arr = nullptr;
    e = array_acquire(ARRAY_VOLUME_3D, vol_x, vol_y, vol_z, in_dtype != PYRONN_FLOAT32, s, &arr);
    if (e != cudaSuccess) return cuda_fail(e, "cone_projection3d: texture array");
    const size_t stride = (size_t)vol_z * vol_y * vol_x * dtype_size(in_dtype);
    for (int b = 0; b < batch && e == cudaSuccess; ++b) {
        e = array_fill(arr, (const char *)volume + b * stride, in_dtype, s);
        if (e == cudaSuccess)
            e = launch_cone_fp(volume, sinogram, in_dtype, out_dtype, d, b, views, step_size, volume_spacing,
                               array_texture(arr), s);
    }
    cudaError_t e2 = array_release(arr, s);
    if (e != cudaSuccess) return cuda_fail(e, name);
    if (e2 != cudaSuccess) return cuda_fail(e2, "cone_projection3d: event record");
    return ok();
}

int pyronn_cone_backprojection3d(const void *sinogram, void *volume, int in_dtype, int out_dtype, int hardware_interp, int batch,
                                 int n_proj, int det_h, int det_w, int vol_z, int vol_y, int vol_x,
                                 const float *volume_origin, const float *volume_spacing,
                                 const float *projection_matrices, const float *step_size,
                                 const float *projection_multiplier, int geom_batch, void *workspace,
                                 size_t workspace_bytes, void *stream)
{
    const char *name = "cone_backprojection3d";
    const Dims3D d{batch, vol_z, vol_y, vol_x, n_proj, det_h, det_w, geom_batch};
    int st = check_cone(name, sinogram, volume, in_dtype, out_dtype, d, volume_origin, volume_spacing, projection_matrices,
                        step_size, projection_multiplier);
    if (st) return st;
    // the views' part is required; the paired copy is used when it fits
    const size_t need = WS_HEADER + align_up((size_t)geom_batch * n_proj * sizeof(ConeBpView), 256);
    if (!workspace || workspace_bytes < need)
        return fail(PYRONN_ERROR_WORKSPACE_TOO_SMALL, "%s: workspace of %zu bytes needed, %zu given", name, need,
                    workspace ? workspace_bytes : (size_t)0);
    if (((uintptr_t)workspace) % 16 != 0)
        return fail(PYRONN_ERROR_INVALID_ARGUMENT, "%s: workspace must be 16-byte aligned", name);
    if (hardware_interp) {
        st = check_texture_layered(det_w, det_h, n_proj);
        if (st) return st;
    }
    cudaStream_t s = (cudaStream_t)stream;
    ConeBpView *views = (ConeBpView *)((char *)workspace + WS_HEADER);
    unsigned *err = (unsigned *)workspace;
    cudaError_t e = cudaMemsetAsync(workspace, 0, WS_HEADER, s);
    if (e != cudaSuccess) return cuda_fail(e, "cone_backprojection3d: workspace header");
    e = launch_cone_bp_prepare(projection_matrices, volume_spacing, volume_origin, geom_batch, n_proj, views, s);
    if (e != cudaSuccess) return cuda_fail(e, "cone_backprojection3d: geometry preparation");
    if (!hardware_interp) {
        if (cone_bp_tma_supported(sinogram, in_dtype, d)) {
            const size_t pb = cone_bp_tma_paired_bytes(in_dtype, d);
            void *paired = (pb > 0 && workspace_bytes >= need + pb) ? (char *)workspace + need : nullptr;
            e = launch_cone_bp_tma(sinogram, volume, in_dtype, out_dtype, d, views, projection_multiplier, err,
                                   paired, s);
        }
        else
            e = launch_cone_bp(sinogram, volume, in_dtype, out_dtype, d, -1, views, projection_multiplier, 0, s);
        if (e != cudaSuccess) return cuda_fail(e, name);
        return ok();
    }
    CachedArray *arr = nullptr;
    e = array_acquire(ARRAY_SINOGRAM_LAYERED, det_w, det_h, n_proj, in_dtype != PYRONN_FLOAT32, s, &arr);
    if (e != cudaSuccess) return cuda_fail(e, "cone_backprojection3d: texture array");
    const size_t stride = (size_t)n_proj * det_h * det_w * dtype_size(in_dtype);
    for (int b = 0; b < batch && e == cudaSuccess; ++b) {
        e = array_fill(arr, (const char *)sinogram + b * stride, in_dtype, s);
        if (e == cudaSuccess)
            e = launch_cone_bp(sinogram, volume, in_dtype, out_dtype, d, b, views, projection_multiplier,
                               array_texture(arr), s);
    }
    cudaError_t e2 = array_release(arr, s);
    if (e != cudaSuccess) return cuda_fail(e, name);
    if (e2 != cudaSuccess) return cuda_fail(e2, "cone_backprojection3d: event record");
    return ok();
}

size_t pyronn_cone_backprojection3d_matched_workspace_size(int geom_batch, int n_proj)
{
    if (geom_batch <= 0 || n_proj <= 0) return 0;
    return WS_HEADER + align_up((size_t)geom_batch * n_proj * sizeof(ConeFpView), 256);
}

int pyronn_cone_backprojection3d_matched(const void *sinogram, float *volume, int in_dtype, int batch, int n_proj,
                                         int det_h, int det_w, int vol_z, int vol_y, int vol_x,
                                         const float *volume_origin, const float *volume_spacing,
                                         const float *projection_matrices, const float *step_size, int geom_batch,
                                         void *workspace, size_t workspace_bytes, void *stream)
{
    const char *name = "cone_backprojection3d_matched";
    const Dims3D d{batch, vol_z, vol_y, vol_x, n_proj, det_h, det_w, geom_batch};
    // the step is the only scalar the scatter reads; pass it as the multiplier
    // slot too so the shared checks see a non-null pointer
    int st = check_cone(name, sinogram, volume, in_dtype, PYRONN_FLOAT32, d, volume_origin, volume_spacing,
                        projection_matrices, step_size, step_size);
    if (st) return st;
    if ((long long)n_proj * batch > 65535)
        return fail(PYRONN_ERROR_UNSUPPORTED, "%s: views x batch above 65535", name);
    const size_t need = pyronn_cone_backprojection3d_matched_workspace_size(geom_batch, n_proj);
    if (!workspace || workspace_bytes < need)
        return fail(PYRONN_ERROR_WORKSPACE_TOO_SMALL, "%s: workspace of %zu bytes needed, %zu given", name, need,
                    workspace ? workspace_bytes : (size_t)0);
    if (((uintptr_t)workspace) % 16 != 0)
        return fail(PYRONN_ERROR_INVALID_ARGUMENT, "%s: workspace must be 16-byte aligned", name);
    cudaStream_t s = (cudaStream_t)stream;
    ConeFpView *views = (ConeFpView *)((char *)workspace + WS_HEADER);
    cudaError_t e = cudaMemsetAsync(workspace, 0, WS_HEADER, s);
    if (e == cudaSuccess)
        e = launch_cone_fp_prepare(projection_matrices, volume_spacing, volume_origin, geom_batch, n_proj, vol_x,
                                   vol_y, vol_z, views, s);
    if (e == cudaSuccess) e = launch_cone_scatter(sinogram, volume, in_dtype, d, views, step_size, volume_spacing, s);
    if (e != cudaSuccess) return cuda_fail(e, name);
    return ok();
}

}  // extern "C"
