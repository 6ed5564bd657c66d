/*
 * pyronn_b200.h -- C ABI of the B200-native PYRO-NN-Layers projector operators.
 *
 * One entry point per reference operator.  Every entry point
 *   - takes caller-owned DEVICE buffers for the data (volume / sinogram) and for
 *     the geometry tensors, exactly the tensors the reference TF op receives
 *     (the reference op kernels read geometry from device memory too);
 *   - takes the shapes as host integers (the reference copies its int32 shape
 *     tensor device->host with a blocking cudaMemcpy inside Compute);
 *   - launches on the caller's stream and never synchronises it;
 *   - allocates no device memory for the linear data path: scratch comes from
 *     a caller-provided workspace (16-byte aligned) whose size the
 *     *_workspace_size() query returns (the hardware_interp paths keep their
 *     CUDA arrays in a library-owned, stream-aware cache; see
 *     pyronn_release_cached_arrays);
 *   - returns a pyronn_status_t and never exits the process (the reference
 *     calls exit() from gpuErrchk, cc/kernels/cone_projector_3D_CudaKernel.cu.cc:32-40).
 *
 * Geometry tensors are batch-major: row b of a [geom_batch, ...] tensor holds
 * the geometry of batch element b, like the reference's flat_outer_dims(index)
 * rows (e.g. cc/ops/cone_projector_3D_OPKernel.cc:235).  geom_batch may be 1
 * (one geometry shared by every batch element) or equal to batch.
 * Vector-valued geometry keeps the reference's [z, y, x] (3D) / [y, x] (2D)
 * order; ray vectors are (x, y) pairs as the reference kernels read them.
 *
 * Storage dtypes: in_dtype and out_dtype (PYRONN_FLOAT32, PYRONN_BFLOAT16,
 * PYRONN_FLOAT16) give the element type of the data input and of the data
 * output independently (e.g. BF16 volumes gathered, FP32 sinograms written);
 * every sum accumulates in FP32 and geometry is always FP32 on input
 * (prepared in FP64 on the device).
 */
#ifndef PYRONN_B200_H
#define PYRONN_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PYRONN_B200_ABI_VERSION 1

#if defined(__GNUC__)
#define PYRONN_API __attribute__((visibility("default")))
#else
#define PYRONN_API
#endif

typedef enum {
    PYRONN_FLOAT32 = 0,
    PYRONN_BFLOAT16 = 1,
    PYRONN_FLOAT16 = 2
} pyronn_dtype_t;

typedef enum {
    PYRONN_SUCCESS = 0,
    PYRONN_ERROR_INVALID_ARGUMENT = 1,
    PYRONN_ERROR_UNSUPPORTED = 2,
    PYRONN_ERROR_WORKSPACE_TOO_SMALL = 3,
    PYRONN_ERROR_CUDA = 4
} pyronn_status_t;

/* ABI version of the loaded library (PYRONN_B200_ABI_VERSION). */
PYRONN_API int pyronn_abi_version(void);

/* Static text for a status code. */
PYRONN_API const char *pyronn_status_string(int status);

/* Detail of the last failing call on the calling host thread ("" if none). */
PYRONN_API const char *pyronn_last_error(void);

/* Device error flags (the kernels' bounded waits never hang: a wait that
 * gives up records this, and the affected output is invalid). */
#define PYRONN_DEVICE_ERROR_NONE 0
#define PYRONN_DEVICE_ERROR_WAIT_TIMEOUT 1

/* Reads the device error flag a cone call left in its workspace
 * (PYRONN_DEVICE_ERROR_NONE, or PYRONN_DEVICE_ERROR_WAIT_TIMEOUT: a bounded
 * wait for a TMA transfer timed out and the volume is invalid).
 * Synchronises the stream.  No counterpart in the reference (which has no
 * asynchronous error reporting). */
PYRONN_API int pyronn_workspace_error(const void *workspace, void *stream, int *device_error);

/* Testing hook, not for production use.  While enable != 0, every block of the
 * TMA-staged cone backprojector (the software-interpolation path of
 * pyronn_cone_backprojection3d and of pyronn_cone_backprojection3d_noalloc for
 * 16-byte aligned detector rows) starves the bounded wait of its last pass of
 * views: that pass issues no copy and waits, with a short spin limit, for
 * bytes that never arrive.  The wait runs out and the call's device error
 * flag becomes PYRONN_DEVICE_ERROR_WAIT_TIMEOUT (the volume is invalid).  No
 * copy is in flight when the wait gives up, so the device stays usable.
 * Process-wide; affects calls enqueued while it is set.  No counterpart in
 * the reference. */
PYRONN_API int pyronn_debug_starve_tma_wait(int enable);

/* Frees the CUDA arrays the hardware_interp paths cached on the current
 * device.  Waits for the work that still reads them (device synchronise). */
PYRONN_API int pyronn_release_cached_arrays(void);

/* ---------------------------------------------------------------------------
 * ParallelProjection2D
 *   replaces REGISTER_OP("ParallelProjection2D")  cc/ops/par_projector_2D_OPKernel.cc:30-56
 *   and Parallel_Projection2D_Kernel_Launcher     cc/kernels/par_projector_2D_CudaKernel.cu.cc:149-178
 *   volume   [batch, vol_y, vol_x]     -> sinogram [batch, n_proj, det_w]
 *   volume_origin [g,2], detector_origin [g,1], volume_spacing [g,2],
 *   detector_spacing [g,1], ray_vectors [g, n_proj, 2]   (g = geom_batch)
 * ------------------------------------------------------------------------- */
PYRONN_API int pyronn_parallel_projection2d(const void *volume, void *sinogram, int in_dtype, int out_dtype,
                                 int batch, int vol_y, int vol_x, int n_proj, int det_w,
                                 const float *volume_origin, const float *detector_origin,
                                 const float *volume_spacing, const float *detector_spacing,
                                 const float *ray_vectors, int geom_batch,
                                 void *workspace, size_t workspace_bytes, void *stream);

/* Workspace bytes of a 2D forward projection (parallel or fan): two copies
 * of the batch as bilinear cells (the four taps of each cell together, as
 * FP32 for every in_dtype, zero border), one x-fastest and one y-fastest, so
 * that a sample is one load and a warp's loads stay on few cache lines
 * whatever the view direction: 2 * align256(batch * (vol_y+3) * (vol_x+3) * 16)
 * bytes.
 * workspace may also be NULL: the call then reads the caller's volume with a
 * bounds test per tap (same results, slower). */
PYRONN_API size_t pyronn_projection2d_workspace_size(int batch, int vol_y, int vol_x, int in_dtype);

/* ---------------------------------------------------------------------------
 * ParallelBackprojection2D
 *   replaces REGISTER_OP("ParallelBackprojection2D") cc/ops/par_backprojector_2D_OPKernel.cc:26-51
 *   and Parallel_Backprojection2D_Kernel_Launcher     cc/kernels/par_backprojector_2D_CudaKernel.cu.cc:77-105
 *   sinogram [batch, n_proj, det_w]    -> volume [batch, vol_y, vol_x]
 * ------------------------------------------------------------------------- */
PYRONN_API int pyronn_parallel_backprojection2d(const void *sinogram, void *volume, int in_dtype, int out_dtype,
                                     int batch, int n_proj, int det_w, int vol_y, int vol_x,
                                     const float *volume_origin, const float *detector_origin,
                                     const float *volume_spacing, const float *detector_spacing,
                                     const float *ray_vectors, int geom_batch, void *stream);

/* ---------------------------------------------------------------------------
 * FanProjection2D
 *   replaces REGISTER_OP("FanProjection2D")  cc/ops/fan_projector_2D_OPKernel.cc:26-53
 *   and Fan_Projection_Kernel_Launcher       cc/kernels/fan_projector_2D_CudaKernel.cu.cc:165-194
 *   source_2_isocenter_distance [g,1], source_2_detector_distance [g,1],
 *   central_ray_vectors [g, n_proj, 2]
 * ------------------------------------------------------------------------- */
PYRONN_API int pyronn_fan_projection2d(const void *volume, void *sinogram, int in_dtype, int out_dtype,
                            int batch, int vol_y, int vol_x, int n_proj, int det_w,
                            const float *volume_origin, const float *detector_origin,
                            const float *volume_spacing, const float *detector_spacing,
                            const float *source_2_isocenter_distance,
                            const float *source_2_detector_distance,
                            const float *central_ray_vectors, int geom_batch,
                            void *workspace, size_t workspace_bytes, void *stream);

/* ---------------------------------------------------------------------------
 * FanBackprojection2D
 *   replaces REGISTER_OP("FanBackprojection2D") cc/ops/fan_backprojector_2D_OPKernel.cc:26-53
 *   and Fan_Backprojection2D_Kernel_Launcher    cc/kernels/fan_backprojector_2D_CudaKernel.cu.cc:83-113
 * ------------------------------------------------------------------------- */
PYRONN_API int pyronn_fan_backprojection2d(const void *sinogram, void *volume, int in_dtype, int out_dtype,
                                int batch, int n_proj, int det_w, int vol_y, int vol_x,
                                const float *volume_origin, const float *detector_origin,
                                const float *volume_spacing, const float *detector_spacing,
                                const float *source_2_isocenter_distance,
                                const float *source_2_detector_distance,
                                const float *central_ray_vectors, int geom_batch, void *stream);

/* ---------------------------------------------------------------------------
 * ConeProjection3D
 *   replaces REGISTER_OP("ConeProjection3D")       cc/ops/cone_projector_3D_OPKernel.cc:34-60,
 *   its host DecomposeProjectionMatrices           cc/ops/cone_projector_3D_OPKernel.cc:96-182
 *   (done here in FP64 on the device, into the workspace),
 *   Cone_Projection_Kernel_Launcher                cc/kernels/cone_projector_3D_CudaKernel.cu.cc:225-257
 *   and Cone_Projection_Kernel_Tex_Interp_Launcher cc/kernels/cone_projector_3D_CudaKernel_hardware_interp.cu.cc:199-262
 *   volume [batch, vol_z, vol_y, vol_x] -> sinogram [batch, n_proj, det_h, det_w]
 *   volume_origin [g,3], volume_spacing [g,3], projection_matrices [g, n_proj, 3, 4],
 *   step_size [g,1], projection_multiplier [g,1] (unused by the forward op, as
 *   in the reference)
 * ------------------------------------------------------------------------- */
/* Workspace bytes a pyronn_cone_projection3d call with these arguments needs
 * (prepared geometry; for hardware_interp = 0 also a copy of one volume as
 * trilinear cells -- the 8 taps of each cell together -- and two zero-padded
 * copies for views whose detector v axis does not run along z, all in the
 * input dtype). */
PYRONN_API size_t pyronn_cone_projection3d_workspace_size(int batch, int vol_z, int vol_y, int vol_x, int n_proj,
                                                          int det_h, int det_w, int in_dtype, int hardware_interp,
                                                          int geom_batch);

PYRONN_API int pyronn_cone_projection3d(const void *volume, void *sinogram, int in_dtype, int out_dtype, int hardware_interp,
                             int batch, int vol_z, int vol_y, int vol_x,
                             int n_proj, int det_h, int det_w,
                             const float *volume_origin, const float *volume_spacing,
                             const float *projection_matrices, const float *step_size,
                             const float *projection_multiplier, int geom_batch,
                             void *workspace, size_t workspace_bytes, void *stream);

/* ---------------------------------------------------------------------------
 * ConeBackprojection3D
 *   replaces REGISTER_OP("ConeBackprojection3D")       cc/ops/cone_backprojector_3D_OPKernel.cc:27-53,
 *   Cone_Backprojection3D_Kernel_Launcher              cc/kernels/cone_backprojector_3D_CudaKernel.cu.cc:121-146
 *   and Cone_Backprojection3D_Kernel_Tex_Interp_Launcher cc/kernels/cone_backprojector_3D_CudaKernel_hardware_interp.cu.cc:104-160
 *   sinogram [batch, n_proj, det_h, det_w] -> volume [batch, vol_z, vol_y, vol_x]
 *   step_size is accepted and unused, as in the reference.
 * ------------------------------------------------------------------------- */
/* Workspace bytes for a pyronn_cone_backprojection3d call with these
 * arguments: the per-view geometry and, for a 16-bit sinogram on the software
 * path with at least 100 voxels per detector pixel, a paired copy of the
 * sinogram (tap u and tap u + 1 in one 32-bit element; one shared-memory load
 * per lerp, the same results).  A workspace
 * of the per-view part alone -- this size with batch = 0 -- is accepted: the
 * call then stages the sinogram itself. */
PYRONN_API size_t pyronn_cone_backprojection3d_workspace_size(int batch, int n_proj, int det_h, int det_w, int vol_z,
                                                              int vol_y, int vol_x, int in_dtype,
                                                              int hardware_interp, int geom_batch);

PYRONN_API int pyronn_cone_backprojection3d(const void *sinogram, void *volume, int in_dtype, int out_dtype, int hardware_interp,
                                 int batch, int n_proj, int det_h, int det_w,
                                 int vol_z, int vol_y, int vol_x,
                                 const float *volume_origin, const float *volume_spacing,
                                 const float *projection_matrices, const float *step_size,
                                 const float *projection_multiplier, int geom_batch,
                                 void *workspace, size_t workspace_bytes, void *stream);

/* ---------------------------------------------------------------------------
 * Matched cone backprojection: the exact transpose of the software-interpolation
 * ConeProjection3D (ray-driven scatter with the projector's own samples and
 * weights, FP32 atomics).  No counterpart in the reference, whose voxel-driven
 * ConeBackprojection3D is not the transpose of its projector; this is the
 * adjoint a dot-product test <A x, y> = <x, A^T y> holds for (exact for every
 * ray whose line integral is > 0, e.g. any non-negative volume).
 *   sinogram [batch, n_proj, det_h, det_w] (in_dtype) -> volume [batch, vol_z,
 *   vol_y, vol_x] FP32 (overwritten); projection_multiplier is not applied.
 * ------------------------------------------------------------------------- */
PYRONN_API size_t pyronn_cone_backprojection3d_matched_workspace_size(int geom_batch, int n_proj);

PYRONN_API int pyronn_cone_backprojection3d_matched(const void *sinogram, float *volume, int in_dtype, int batch,
                                                    int n_proj, int det_h, int det_w, int vol_z, int vol_y,
                                                    int vol_x, const float *volume_origin,
                                                    const float *volume_spacing, const float *projection_matrices,
                                                    const float *step_size, int geom_batch, void *workspace,
                                                    size_t workspace_bytes, void *stream);

/* ---------------------------------------------------------------------------
 * Cone backprojection that allocates nothing.  No counterpart in the
 * reference (whose launchers cudaMalloc per call, the out-of-memory trap its
 * README warns about when TensorFlow's allocator owns the GPU).
 *
 * For callers that cannot provide a workspace or call cudaMalloc: a host
 * framework whose allocator owns the device memory and cannot lend a buffer
 * to foreign code, or a real-time loop that must not allocate (cudaMalloc
 * synchronises the device).  Same arguments and result as
 * pyronn_cone_backprojection3d with hardware_interp = 0, minus the workspace:
 * the scratch (prepared projection matrices and the error flag) lives in a
 * fixed array of device global memory inside the library, which every GPU
 * that loads the library holds until process exit.
 *   - geom_batch * n_proj must not exceed PYRONN_NOALLOC_MAX_VIEWS (8192
 *     views, 384 KiB of scratch); larger requests return
 *     PYRONN_ERROR_UNSUPPORTED;
 *   - software interpolation only (texture arrays would be allocations);
 *   - the first call on a device looks up the array's device address, so make
 *     that call before capturing a stream;
 *   - all calls on a device share the array (it keeps the last call's
 *     contents; each call rewrites what it reads): calls that overlap on the
 *     same GPU race and must be serialised by the caller.
 * ------------------------------------------------------------------------- */
#define PYRONN_NOALLOC_MAX_VIEWS 8192

/* Reads the device error flag that the last
 * pyronn_cone_backprojection3d_noalloc call on the current device left in the
 * fixed scratch (PYRONN_DEVICE_ERROR_NONE, or
 * PYRONN_DEVICE_ERROR_WAIT_TIMEOUT: the volume is invalid).
 * Synchronises the stream; allocates nothing.  No counterpart in the
 * reference. */
PYRONN_API int pyronn_noalloc_error(void *stream, int *device_error);

PYRONN_API int pyronn_cone_backprojection3d_noalloc(const void *sinogram, void *volume, int in_dtype,
                                                    int out_dtype, int batch, int n_proj, int det_h, int det_w,
                                                    int vol_z, int vol_y, int vol_x, const float *volume_origin,
                                                    const float *volume_spacing,
                                                    const float *projection_matrices, const float *step_size,
                                                    const float *projection_multiplier, int geom_batch,
                                                    void *stream);

/* ---------------------------------------------------------------------------
 * Geometry of circular trajectories, built on the device in FP64 on `stream`
 * (no counterpart in the reference, whose ops receive these tensors from the
 * PYRO-NN package, which builds them on the host): view n at angle
 * start_angle + n * angular_range / n_proj.
 *
 * pyronn_circular_projection_matrices writes [n_proj, 3, 4] FP32 matrices P
 * of a cone-beam scan: source at -SID (cos a, sin a, 0) mm, principal ray
 * (cos a, sin a, 0), detector columns along (-sin a, cos a, 0), rows along +z,
 * principal point (principal_v, principal_u) in pixel indices ((H-1)/2,
 * (W-1)/2 for a centred detector); P maps world mm (x, y, z, 1) to
 * (u w, v w, w) -- the projection_matrices input of the cone ops.
 * pyronn_circular_ray_vectors_2d writes [n_proj, 2] FP32 (cos a, sin a), the
 * ray_vectors / central_ray_vectors input of the 2D ops.
 * ------------------------------------------------------------------------- */
PYRONN_API int pyronn_circular_projection_matrices(float *projection_matrices, int n_proj, double sid, double sdd,
                                                   double det_spacing_v, double det_spacing_u, double principal_v,
                                                   double principal_u, double angular_range, double start_angle,
                                                   void *stream);

PYRONN_API int pyronn_circular_ray_vectors_2d(float *ray_vectors, int n_proj, double angular_range,
                                              double start_angle, void *stream);

/* ---------------------------------------------------------------------------
 * FDK / FBP pre-processing (no counterpart in the reference's ops; the
 * PYRO-NN package filters in Python).  For every detector row of
 * projections [batch, n_proj, det_h, det_w]:
 *   g[k] = p[k] * SDD / sqrt(SDD^2 + u_k^2 + v^2)     (Feldkamp cosine weight;
 *          u_k = (k - principal_u) * det_spacing_u, v = (row - principal_v) *
 *          det_spacing_v; no weight when sdd == 0, i.e. parallel beam)
 *   q[j] = tau * sum_k h[j - k] g[k]                   (linear convolution,
 *          tau = det_spacing_u, h the Ram-Lak or Shepp-Logan ramp kernel of
 *          Kak & Slaney ch. 3)
 * weight_output = 1 applies the weight after the filter instead (the adjoint
 * of the weight-then-filter operator, the kernel being symmetric).  FDK =
 * this, then pyronn_cone_backprojection3d with projection_multiplier
 * SID * SDD * pi / n_proj (full circle).  projections and filtered may be
 * the same buffer.  det_w <= PYRONN_FDK_MAX_WIDTH.  Distinct buffers with
 * det_w a multiple of 4 up to 2048 (16-byte aligned) run on the tensor cores
 * (the Toeplitz product in 3xTF32, FP32-accurate: within a few 1e-6 relative
 * of the CUDA-core kernel); in-place calls and other widths on the CUDA
 * cores (FP32 FMAs).
 * ------------------------------------------------------------------------- */
#define PYRONN_FILTER_RAM_LAK 0
#define PYRONN_FILTER_SHEPP_LOGAN 1
#define PYRONN_FDK_MAX_WIDTH 4096

PYRONN_API int pyronn_fdk_filter(const void *projections, void *filtered, int in_dtype, int out_dtype, int batch,
                                 int n_proj, int det_h, int det_w, double sdd, double det_spacing_v,
                                 double det_spacing_u, double principal_v, double principal_u, int filter,
                                 int weight_output, void *stream);

/* Reads and clears the device error flag of the tensor-core filter on the
 * current device: PYRONN_DEVICE_ERROR_WAIT_TIMEOUT if a bounded wait of any
 * pyronn_fdk_filter call since the last read gave up (that call's rows of the
 * affected tile were not written), else PYRONN_DEVICE_ERROR_NONE.
 * Synchronises the stream. */
PYRONN_API int pyronn_fdk_error(void *stream, int *device_error);

#ifdef __cplusplus
}
#endif

#endif /* PYRONN_B200_H */
