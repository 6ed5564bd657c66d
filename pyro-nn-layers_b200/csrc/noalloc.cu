// noalloc.cu -- a cone backprojection entry point that allocates nothing.
//
// pyronn_cone_backprojection3d needs a small scratch area (the per-view
// projection matrices prepared in FP64 on the device, plus an error flag) and
// takes it from a caller-provided workspace.  Some callers cannot hand one
// over: a host framework whose allocator owns all device memory and has no
// way to lend a temporary buffer to a foreign kernel, or a real-time loop
// that must not allocate (cudaMalloc synchronises the device).  For them this
// file keeps that scratch in a fixed-size array in device global memory that
// the library image itself provides: it exists on every GPU that loads the
// library, from load until process exit, and no call ever allocates.
//
// The first word of the scratch is the call's device error flag (cleared at
// the start of every call, set when a bounded wait of the TMA backprojector
// gives up); pyronn_noalloc_error reads it without a workspace pointer.
//
// Limits: geom_batch * n_proj <= PYRONN_NOALLOC_MAX_VIEWS (bigger requests
// are rejected); software interpolation only (hardware_interp needs CUDA
// arrays, which are allocations).  Every call on a device shares the one
// array, so calls that overlap on that GPU (different streams, or host
// threads) race on it and must be serialised by the caller.
#include <mutex>

#include "internal.h"

namespace pyronn {

namespace {

constexpr int MAX_DEVICES = 64;
constexpr size_t NOALLOC_HEADER = 256;  // first word: device error flag

// The scratch itself.  In host code this name is only a host-side stand-in
// for the device symbol; kernels receive the device address obtained from
// cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_HEADER +
                                                                 PYRONN_NOALLOC_MAX_VIEWS * sizeof(ConeBpView)];

std::mutex g_mu;
void *g_scratch_ptr[MAX_DEVICES] = {nullptr};

// Device address of the scratch on the current device; looked up once per
// device (the first call on a device does this, so that call should come
// before any stream capture).
cudaError_t scratch_address(void **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= MAX_DEVICES) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return cudaSuccess;
}

}  // namespace

}  // namespace pyronn

using namespace pyronn;

extern "C" int pyronn_cone_backprojection3d_noalloc(const void *sinogram, void *volume, int in_dtype, int out_dtype,
                                                    int batch, int n_proj, int det_h, int det_w, int vol_z, int vol_y,
                                                    int vol_x, const float *volume_origin,
                                                    const float *volume_spacing, const float *projection_matrices,
                                                    const float *step_size, const float *projection_multiplier,
                                                    int geom_batch, void *stream)
{
    // the shared argument checks of the workspace entry point, with a
    // workspace that is exactly what the views need: the size limit first
    if (geom_batch > 0 && n_proj > 0 && (long long)geom_batch * n_proj > PYRONN_NOALLOC_MAX_VIEWS)
        return report_error(PYRONN_ERROR_UNSUPPORTED,
                            "cone_backprojection3d_noalloc: geom_batch * n_proj = %lld exceeds the fixed scratch of "
                            "%d views (use pyronn_cone_backprojection3d with a workspace)",
                            (long long)geom_batch * n_proj, PYRONN_NOALLOC_MAX_VIEWS);
    void *scratch = nullptr;
    cudaError_t e = scratch_address(&scratch);
    if (e != cudaSuccess) return report_cuda_error(e, "cone_backprojection3d_noalloc: scratch address");
    const size_t bytes = NOALLOC_HEADER + (size_t)PYRONN_NOALLOC_MAX_VIEWS * sizeof(ConeBpView);
    // hardware_interp = 0: the software path allocates nothing
    return pyronn_cone_backprojection3d(sinogram, volume, in_dtype, out_dtype, 0, batch, n_proj, det_h, det_w, vol_z,
                                        vol_y, vol_x, volume_origin, volume_spacing, projection_matrices, step_size,
                                        projection_multiplier, geom_batch, scratch, bytes, stream);
}

extern "C" int pyronn_noalloc_error(void *stream, int *device_error)
{
    if (!device_error) return report_error(PYRONN_ERROR_INVALID_ARGUMENT, "noalloc_error: null pointer");
    void *scratch = nullptr;
    cudaError_t e = scratch_address(&scratch);
    if (e != cudaSuccess) return report_cuda_error(e, "noalloc_error: scratch address");
    // the header word (a pageable host copy: synchronous for the host)
    unsigned flag = 0;
    cudaStream_t s = (cudaStream_t)stream;
    e = cudaMemcpyAsync(&flag, scratch, sizeof(flag), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return report_cuda_error(e, "noalloc_error");
    *device_error = (int)flag;
    return report_error(PYRONN_SUCCESS, "%s", "");
}
