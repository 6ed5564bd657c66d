// internal.h -- launcher interfaces between the C-ABI layer and the kernels.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../../include/pyronn_b200.h"

namespace pyronn {

// Per-view cone forward geometry in voxel-index space, built in FP64 on the
// device from P = [M | p4]: inv_ar = diag(1/spacing) M^-1 (row major) and
// src = (C - origin) / spacing with C = -M^-1 p4 the camera centre.
struct ConeFpView {
    double inv_ar[9];
    double src[3];
    // detector footprint of the volume box [-0.5, N] per axis, in pixel
    // indices (u_min, u_max, v_min, v_max), widened by 2 pixels: a ray whose
    // pixel lies outside misses the box; unbounded (+-inf) when the box's
    // corners do not all lie on one side of the source
    float foot[4];
};

// Per-view cone backprojection matrix in voxel-index space:
// row r = (P[r,0] sx, P[r,1] sy, P[r,2] sz, P[r,:] . (ox, oy, oz, 1)).
struct ConeBpView {
    float4 row[3];
};

struct Dims2D {
    int batch, vol_y, vol_x, n_proj, det_w, geom_batch;
};

struct Geom2D {
    const float *volume_origin, *detector_origin, *volume_spacing, *detector_spacing;
    const float *rays, *sid, *sdd;  // sid/sdd null for parallel beam
};

struct Dims3D {
    int batch, vol_z, vol_y, vol_x, n_proj, det_h, det_w, geom_batch;
};

// geometry preparation (geometry.cu)
cudaError_t launch_cone_fp_prepare(const float *P, const float *spacing, const float *origin, int geom_batch,
                                   int n_proj, int vol_x, int vol_y, int vol_z, ConeFpView *out, cudaStream_t stream);
cudaError_t launch_cone_bp_prepare(const float *P, const float *spacing, const float *origin, int geom_batch,
                                   int n_proj, ConeBpView *out, cudaStream_t stream);

// 2D (proj2d.cu)
// workspace: room for the two cell copies (pyronn_projection2d_workspace_size), or null
cudaError_t launch_projection2d(const void *volume, void *sinogram, int in_dtype, int out_dtype, bool fan,
                                const Dims2D &d, const Geom2D &g, void *workspace, cudaStream_t stream);
cudaError_t launch_backprojection2d(const void *sinogram, void *volume, int in_dtype, int out_dtype, bool fan,
                                    const Dims2D &d, const Geom2D &g, cudaStream_t stream);

// cone (cone_fp.cu / cone_bp.cu); tex == 0 selects the software path
cudaError_t launch_cone_fp(const void *volume, void *sinogram, int in_dtype, int out_dtype, const Dims3D &d,
                           int batch_index, const ConeFpView *views, const float *step, const float *spacing,
                           cudaTextureObject_t tex, cudaStream_t stream);
cudaError_t launch_cone_bp(const void *sinogram, void *volume, int in_dtype, int out_dtype, const Dims3D &d,
                           int batch_index, const ConeBpView *views, const float *mult, cudaTextureObject_t tex,
                           cudaStream_t stream);

// software forward projector over padded, view-oriented copies (cone_fp_padded.cu)
size_t cone_fp_padded_scratch_bytes(int vol_z, int vol_y, int vol_x, int in_dtype);
bool cone_fp_padded_supported(const Dims3D &d);
// flags: zeroed header words of the workspace (the kernel records which copies it needs)
cudaError_t launch_cone_fp_padded(const void *volume, void *sinogram, int in_dtype, int out_dtype, const Dims3D &d,
                                  const ConeFpView *views, const float *step, const float *spacing, void *scratch,
                                  unsigned *flags, cudaStream_t stream);

// matched (exact-adjoint) scatter backprojector (cone_matched.cu); FP32 output
// FDK weighting + ramp filtering of `rows` detector rows (fdk.cu)
cudaError_t launch_fdk_filter(const void *in, void *out, int in_dtype, int out_dtype, long long rows, int det_h,
                              int W, float sdd, float dv, float du, float cv, float cu, int kind, int weight_output,
                              cudaStream_t stream);
// the same on the tensor cores (fdk_tc.cu): rows of at most 2048 pixels, a
// multiple of 4, 16-byte aligned buffers, at most 65535 * 128 rows
bool fdk_tc_supported(long long rows, int W, const void *in, const void *out);
cudaError_t launch_fdk_filter_tc(const void *in, void *out, int in_dtype, int out_dtype, long long rows, int det_h,
                                 int W, float sdd, float dv, float du, float cv, float cu, int kind,
                                 int weight_output, cudaStream_t stream);
// reads the filter's sticky device error word on the current device (and
// clears it when set); synchronises the stream
cudaError_t fdk_tc_error(cudaStream_t stream, unsigned *device_error);

cudaError_t launch_cone_scatter(const void *sinogram, float *volume, int in_dtype, const Dims3D &d,
                                const ConeFpView *views, const float *step, const float *spacing,
                                cudaStream_t stream);

// TMA-staged software backprojector (cone_bp_tma.cu); err = device error flag
bool cone_bp_tma_supported(const void *sinogram, int in_dtype, const Dims3D &d);
// Bytes of the paired copy of a 16-bit sinogram (0 for FP32, or where the
// copy does not pay): with it the TMA backprojector stages 32-bit tap pairs,
// one shared-memory load per lerp.
size_t cone_bp_tma_paired_bytes(int in_dtype, const Dims3D &d);
// `paired` (device, 16-byte aligned, cone_bp_tma_paired_bytes) or null.
cudaError_t launch_cone_bp_tma(const void *sinogram, void *volume, int in_dtype, int out_dtype, const Dims3D &d,
                               const ConeBpView *views, const float *mult, unsigned *err, void *paired,
                               cudaStream_t stream);
// testing hook (pyronn_debug_starve_tma_wait): while enabled, the last pass of
// every TMA backprojector block issues no copies and expects bytes that never
// arrive, so its bounded wait runs out and the block reports the timeout
void cone_bp_tma_starve_last_pass(int enable);

// texture-array cache (texcache.cu)
struct CachedArray;
enum ArrayKind { ARRAY_VOLUME_3D = 0, ARRAY_SINOGRAM_LAYERED = 1 };
// Returns an array of the given kind/extent whose previous users are done
// (or were on the same stream).  half_texels selects an FP16 texel format.
cudaError_t array_acquire(int kind, int w, int h, int d, bool half_texels, cudaStream_t stream, CachedArray **out);
cudaTextureObject_t array_texture(CachedArray *a);
// Copies one batch element (w*h*d elements of dtype) into the array on stream.
cudaError_t array_fill(CachedArray *a, const void *src, int dtype, cudaStream_t stream);
// Marks the array as in use by work already enqueued on stream.
cudaError_t array_release(CachedArray *a, cudaStream_t stream);
int array_cache_clear();

size_t dtype_size(int dtype);

// record a failure as the calling thread's last error (capi.cu); return status
int report_error(int status, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
int report_cuda_error(cudaError_t e, const char *what);

}  // namespace pyronn
