// ref_driver.cu -- restates the reference's TF op layer (cc/ops/*_OPKernel.cc)
// around the reference's own, unmodified kernel launchers so tests can run
// them.  TEST INFRASTRUCTURE ONLY: linked into oracle/_ref/libpyronn_ref.so,
// never into the product.
//
// Each ref_* function takes device pointers laid out like the op inputs
// (batch-major geometry rows, one per batch element) and, like the op's
// Compute, loops over the batch calling the launcher for each element
// (e.g. cc/ops/cone_projector_3D_OPKernel.cc:234-247).  The cone forward
// op's DecomposeProjectionMatrices (cc/ops/cone_projector_3D_OPKernel.cc:96-182,
// FP32 Eigen SVD) is restated in FP64 on the host and rounded to FP32.
#include <cuda_runtime.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

// launcher prototypes as the reference op files declare them
void Parallel_Projection2D_Kernel_Launcher(const float *volume_ptr, float *out, const float *ray_vectors,
                                           const int number_of_projections, const int volume_size_x,
                                           const int volume_size_y, const float *volume_spacing_ptr,
                                           const float *volume_origin_ptr, const int detector_size,
                                           const float *detector_spacing, const float *detector_origin);
void Parallel_Backprojection2D_Kernel_Launcher(const float *sinogram_ptr, float *out, const float *ray_vectors,
                                               const int number_of_projections, const int volume_size_x,
                                               const int volume_size_y, const float *volume_spacing_ptr,
                                               const float *volume_origin_ptr, const int detector_size,
                                               const float *detector_spacing, const float *detector_origin);
void Fan_Projection_Kernel_Launcher(const float *volume_ptr, float *out, const float *ray_vectors,
                                    const int number_of_projections, const int volume_size_x,
                                    const int volume_size_y, const float *volume_spacing_ptr,
                                    const float *volume_origin_ptr, const int detector_size,
                                    const float *detector_spacing, const float *detector_origin, const float *sid,
                                    const float *sdd);
void Fan_Backprojection2D_Kernel_Launcher(const float *sinogram_ptr, float *out, const float *ray_vectors,
                                          const int number_of_projections, const int volume_size_x,
                                          const int volume_size_y, const float *volume_spacing,
                                          const float *volume_origin, const int detector_size,
                                          const float *detector_spacing, const float *detector_origin,
                                          const float *sid, const float *sdd);
void Cone_Projection_Kernel_Launcher(const float *volume_ptr, float *out, const float *inv_AR_matrix,
                                     const float *src_points, const int number_of_projections,
                                     const int volume_width, const int volume_height, const int volume_depth,
                                     const float *volume_spacing, const int detector_width,
                                     const int detector_height, const float *step_size);
void Cone_Projection_Kernel_Tex_Interp_Launcher(const float *volume_ptr, float *out, const float *inv_AR_matrix,
                                                const float *src_points, const int number_of_projections,
                                                const int volume_width, const int volume_height,
                                                const int volume_depth, const float *volume_spacing,
                                                const int detector_width, const int detector_height,
                                                const float *step_size);
void Cone_Backprojection3D_Kernel_Launcher(const float *sinogram_ptr, float *out, const float *projection_matrices,
                                           const int number_of_projections, const int volume_width,
                                           const int volume_height, const int volume_depth,
                                           const float *volume_spacing, const float *volume_origin,
                                           const int detector_width, const int detector_height,
                                           const float *projection_multiplier);
void Cone_Backprojection3D_Kernel_Tex_Interp_Launcher(const float *sinogram_ptr, float *out,
                                                      const float *projection_matrix,
                                                      const int number_of_projections, const int volume_width,
                                                      const int volume_height, const int volume_depth,
                                                      const float *volume_spacing, const float *volume_origin,
                                                      const int detector_width, const int detector_height,
                                                      const float *projection_multiplier);

static int finish()
{
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaGetLastError();
    return (int)e;
}

extern "C" {

int ref_parallel_projection2d(const float *vol, float *sino, int batch, int Y, int X, int n_proj, int W,
                              const float *vol_origin, const float *det_origin, const float *vol_spacing,
                              const float *det_spacing, const float *rays)
{
    for (int b = 0; b < batch; ++b)
        Parallel_Projection2D_Kernel_Launcher(vol + (size_t)b * Y * X, sino + (size_t)b * n_proj * W,
                                              rays + (size_t)b * n_proj * 2, n_proj, X, Y, vol_spacing + 2 * b,
                                              vol_origin + 2 * b, W, det_spacing + b, det_origin + b);
    return finish();
}

int ref_parallel_backprojection2d(const float *sino, float *vol, int batch, int n_proj, int W, int Y, int X,
                                  const float *vol_origin, const float *det_origin, const float *vol_spacing,
                                  const float *det_spacing, const float *rays)
{
    for (int b = 0; b < batch; ++b)
        Parallel_Backprojection2D_Kernel_Launcher(sino + (size_t)b * n_proj * W, vol + (size_t)b * Y * X,
                                                  rays + (size_t)b * n_proj * 2, n_proj, X, Y, vol_spacing + 2 * b,
                                                  vol_origin + 2 * b, W, det_spacing + b, det_origin + b);
    return finish();
}

int ref_fan_projection2d(const float *vol, float *sino, int batch, int Y, int X, int n_proj, int W,
                         const float *vol_origin, const float *det_origin, const float *vol_spacing,
                         const float *det_spacing, const float *sid, const float *sdd, const float *rays)
{
    for (int b = 0; b < batch; ++b)
        Fan_Projection_Kernel_Launcher(vol + (size_t)b * Y * X, sino + (size_t)b * n_proj * W,
                                       rays + (size_t)b * n_proj * 2, n_proj, X, Y, vol_spacing + 2 * b,
                                       vol_origin + 2 * b, W, det_spacing + b, det_origin + b, sid + b, sdd + b);
    return finish();
}

int ref_fan_backprojection2d(const float *sino, float *vol, int batch, int n_proj, int W, int Y, int X,
                             const float *vol_origin, const float *det_origin, const float *vol_spacing,
                             const float *det_spacing, const float *sid, const float *sdd, const float *rays)
{
    for (int b = 0; b < batch; ++b)
        Fan_Backprojection2D_Kernel_Launcher(sino + (size_t)b * n_proj * W, vol + (size_t)b * Y * X,
                                             rays + (size_t)b * n_proj * 2, n_proj, X, Y, vol_spacing + 2 * b,
                                             vol_origin + 2 * b, W, det_spacing + b, det_origin + b, sid + b,
                                             sdd + b);
    return finish();
}

// FP64 restatement of DecomposeProjectionMatrices for one batch element;
// host inputs, FP32 outputs in the launcher's layout
static void decompose(const float *P, const float *spacing, const float *origin, int n_proj, float *inv_ar,
                      float *src)
{
    const double s[3] = {spacing[2], spacing[1], spacing[0]};
    const double o[3] = {origin[2], origin[1], origin[0]};
    for (int n = 0; n < n_proj; ++n) {
        const float *m = P + 12 * n;
        const double a = m[0], b = m[1], c = m[2], d = m[4], e = m[5], f = m[6], g = m[8], h = m[9], i = m[10];
        const double A = e * i - f * h, B = -(d * i - f * g), C = d * h - e * g;
        const double det = a * A + b * B + c * C;
        double inv[9] = {A / det, -(b * i - c * h) / det, (b * f - c * e) / det,
                         B / det, (a * i - c * g) / det,  -(a * f - c * d) / det,
                         C / det, -(a * h - b * g) / det, (a * e - b * d) / det};
        const double p4[3] = {m[3], m[7], m[11]};
        for (int r = 0; r < 3; ++r) {
            const double cc = -(inv[3 * r] * p4[0] + inv[3 * r + 1] * p4[1] + inv[3 * r + 2] * p4[2]);
            src[3 * n + r] = (float)((cc - o[r]) / s[r]);
            for (int k = 0; k < 3; ++k) inv_ar[9 * n + 3 * r + k] = (float)(inv[3 * r + k] / s[r]);
        }
    }
}

int ref_cone_projection3d(const float *vol, float *sino, int hardware_interp, int batch, int Z, int Y, int X,
                          int n_proj, int H, int W, const float *vol_origin, const float *vol_spacing,
                          const float *P, const float *step)
{
    float *hP = (float *)malloc(sizeof(float) * 12 * (size_t)n_proj);
    float *inv_ar = (float *)malloc(sizeof(float) * 9 * (size_t)n_proj);
    float *src = (float *)malloc(sizeof(float) * 3 * (size_t)n_proj);
    float hs[3], ho[3];
    int rc = 0;
    for (int b = 0; b < batch && rc == 0; ++b) {
        // the op copies spacing, origin and P device->host (:118-147)
        rc = (int)cudaMemcpy(hs, vol_spacing + 3 * b, sizeof(hs), cudaMemcpyDeviceToHost);
        if (rc == 0) rc = (int)cudaMemcpy(ho, vol_origin + 3 * b, sizeof(ho), cudaMemcpyDeviceToHost);
        if (rc == 0)
            rc = (int)cudaMemcpy(hP, P + (size_t)b * n_proj * 12, sizeof(float) * 12 * n_proj,
                                 cudaMemcpyDeviceToHost);
        if (rc) break;
        decompose(hP, hs, ho, n_proj, inv_ar, src);
        const float *v = vol + (size_t)b * Z * Y * X;
        float *o = sino + (size_t)b * n_proj * H * W;
        if (hardware_interp)
            Cone_Projection_Kernel_Tex_Interp_Launcher(v, o, inv_ar, src, n_proj, X, Y, Z, vol_spacing + 3 * b, W, H,
                                                       step + b);
        else
            Cone_Projection_Kernel_Launcher(v, o, inv_ar, src, n_proj, X, Y, Z, vol_spacing + 3 * b, W, H, step + b);
    }
    free(hP);
    free(inv_ar);
    free(src);
    return rc ? rc : finish();
}

int ref_cone_backprojection3d(const float *sino, float *vol, int hardware_interp, int batch, int n_proj, int H,
                              int W, int Z, int Y, int X, const float *vol_origin, const float *vol_spacing,
                              const float *P, const float *mult)
{
    for (int b = 0; b < batch; ++b) {
        const float *s = sino + (size_t)b * n_proj * H * W;
        float *v = vol + (size_t)b * Z * Y * X;
        if (hardware_interp)
            Cone_Backprojection3D_Kernel_Tex_Interp_Launcher(s, v, P + (size_t)b * n_proj * 12, n_proj, X, Y, Z,
                                                             vol_spacing + 3 * b, vol_origin + 3 * b, W, H, mult + b);
        else
            Cone_Backprojection3D_Kernel_Launcher(s, v, P + (size_t)b * n_proj * 12, n_proj, X, Y, Z,
                                                  vol_spacing + 3 * b, vol_origin + 3 * b, W, H, mult + b);
    }
    return finish();
}

}  // extern "C"
