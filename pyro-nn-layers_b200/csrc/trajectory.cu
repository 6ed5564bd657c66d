// trajectory.cu -- geometry of circular trajectories built on the device in
// FP64: the 3x4 projection matrices of a cone-beam scan and the (cos, sin)
// ray vectors of a 2D scan, the tensors the projector ops take as geometry.
//
// The reference ops receive these tensors from their caller (PYRO-NN builds
// them on the host in Python); building them on the stream lets a serving
// caller make geometry without a host round trip.  Conventions are those of
// pyronn_layers/geometry.py, computed with the same FP64 expressions:
//   theta_n = start + n * (range / n_proj)
//   source at -SID (cos theta, sin theta, 0); rotation rows (-s, c, 0),
//   (0, 0, 1), (c, s, 0); t = -R source; P = K [R | t] with
//   K = [[SDD/du, 0, cu], [0, SDD/dv, cv], [0, 0, 1]].
#include "internal.h"

namespace pyronn {

namespace {

__global__ void circular_pm_kernel(float *__restrict__ P, int n_proj, double sid, double sdd, double dv, double du,
                                   double cv, double cu, double range, double start)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= n_proj) return;
    const double th = start + (double)n * (range / n_proj);
    double s, c;
    sincos(th, &s, &c);
    const double src[3] = {-sid * c, -sid * s, 0.0};
    const double R[3][3] = {{-s, c, 0.0}, {0.0, 0.0, 1.0}, {c, s, 0.0}};
    double Rt[3][4];
    for (int r = 0; r < 3; ++r) {
        Rt[r][0] = R[r][0], Rt[r][1] = R[r][1], Rt[r][2] = R[r][2];
        Rt[r][3] = -(R[r][0] * src[0] + R[r][1] * src[1] + R[r][2] * src[2]);
    }
    const double K[3][3] = {{sdd / du, 0.0, cu}, {0.0, sdd / dv, cv}, {0.0, 0.0, 1.0}};
    float *out = P + (size_t)n * 12;
    for (int r = 0; r < 3; ++r)
        for (int col = 0; col < 4; ++col)
            out[r * 4 + col] = (float)(K[r][0] * Rt[0][col] + K[r][1] * Rt[1][col] + K[r][2] * Rt[2][col]);
}

__global__ void circular_rays_2d_kernel(float *__restrict__ rays, int n_proj, double range, double start)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= n_proj) return;
    const double th = start + (double)n * (range / n_proj);
    double s, c;
    sincos(th, &s, &c);
    rays[2 * (size_t)n] = (float)c;
    rays[2 * (size_t)n + 1] = (float)s;
}

bool finite_positive(double x)
{
    return x > 0.0 && x < 1.0e300;
}

bool finite_value(double x)
{
    return x == x && x > -1.0e300 && x < 1.0e300;
}

}  // namespace

}  // namespace pyronn

using namespace pyronn;

extern "C" int pyronn_circular_projection_matrices(float *projection_matrices, int n_proj, double sid, double sdd,
                                                   double det_spacing_v, double det_spacing_u, double principal_v,
                                                   double principal_u, double angular_range, double start_angle,
                                                   void *stream)
{
    if (!projection_matrices) return report_error(PYRONN_ERROR_INVALID_ARGUMENT, "circular_projection_matrices: null output");
    if (n_proj <= 0) return report_error(PYRONN_ERROR_INVALID_ARGUMENT, "circular_projection_matrices: n_proj must be positive");
    if (!finite_positive(sid) || !finite_positive(sdd) || !finite_positive(det_spacing_v) ||
        !finite_positive(det_spacing_u))
        return report_error(PYRONN_ERROR_INVALID_ARGUMENT,
                            "circular_projection_matrices: SID, SDD and the detector spacing must be positive");
    if (!finite_value(principal_v) || !finite_value(principal_u) || !finite_value(angular_range) || !finite_value(start_angle))
        return report_error(PYRONN_ERROR_INVALID_ARGUMENT,
                            "circular_projection_matrices: principal point and angles must be finite");
    circular_pm_kernel<<<(n_proj + 127) / 128, 128, 0, (cudaStream_t)stream>>>(
        projection_matrices, n_proj, sid, sdd, det_spacing_v, det_spacing_u, principal_v, principal_u, angular_range,
        start_angle);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return report_cuda_error(e, "circular_projection_matrices");
    return PYRONN_SUCCESS;
}

extern "C" int pyronn_circular_ray_vectors_2d(float *ray_vectors, int n_proj, double angular_range,
                                              double start_angle, void *stream)
{
    if (!ray_vectors) return report_error(PYRONN_ERROR_INVALID_ARGUMENT, "circular_ray_vectors_2d: null output");
    if (n_proj <= 0) return report_error(PYRONN_ERROR_INVALID_ARGUMENT, "circular_ray_vectors_2d: n_proj must be positive");
    if (!finite_value(angular_range) || !finite_value(start_angle))
        return report_error(PYRONN_ERROR_INVALID_ARGUMENT, "circular_ray_vectors_2d: angles must be finite");
    circular_rays_2d_kernel<<<(n_proj + 127) / 128, 128, 0, (cudaStream_t)stream>>>(ray_vectors, n_proj,
                                                                                    angular_range, start_angle);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return report_cuda_error(e, "circular_ray_vectors_2d");
    return PYRONN_SUCCESS;
}
