// geometry.cu -- FP64 device preparation of the cone-beam projection matrices.
//
// The reference decomposes P on the host in FP32 (JacobiSVD null space for the
// camera centre, Eigen inverse for M) once per call and per batch element,
// after blocking device->host copies (cc/ops/cone_projector_3D_OPKernel.cc:96-182,
// cc/helper_headers/helper_geometry_cpu.h:30-43).  Here one thread per view
// does it in FP64 on the stream: C = -M^-1 p4 is the right null vector of
// P = [M | p4] already normalised to C[3] = 1, so no SVD is needed.
#include "internal.h"

namespace pyronn {

namespace {

__device__ void invert3x3(const double *m, double *inv)
{
    // cofactor expansion; m and inv row major
    const double a = m[0], b = m[1], c = m[2], d = m[3], e = m[4], f = m[5], g = m[6], h = m[7], i = m[8];
    const double A = e * i - f * h, B = -(d * i - f * g), C = d * h - e * g;
    const double inv_det = 1.0 / (a * A + b * B + c * C);
    inv[0] = A * inv_det;
    inv[1] = -(b * i - c * h) * inv_det;
    inv[2] = (b * f - c * e) * inv_det;
    inv[3] = B * inv_det;
    inv[4] = (a * i - c * g) * inv_det;
    inv[5] = -(a * f - c * d) * inv_det;
    inv[6] = C * inv_det;
    inv[7] = -(a * h - b * g) * inv_det;
    inv[8] = (a * e - b * d) * inv_det;
}

// spacing/origin rows are in (z, y, x) order, as the reference op receives them
__global__ void cone_fp_prepare_kernel(const float *__restrict__ P, const float *__restrict__ spacing,
                                       const float *__restrict__ origin, int geom_batch, int n_proj,
                                       ConeFpView *__restrict__ out)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= geom_batch * n_proj) return;
    const int g = t / n_proj;
    const float *p = P + (size_t)t * 12;
    const double s[3] = {spacing[g * 3 + 2], spacing[g * 3 + 1], spacing[g * 3 + 0]};
    const double o[3] = {origin[g * 3 + 2], origin[g * 3 + 1], origin[g * 3 + 0]};
    double m[9] = {p[0], p[1], p[2], p[4], p[5], p[6], p[8], p[9], p[10]};
    const double p4[3] = {p[3], p[7], p[11]};
    double inv[9];
    invert3x3(m, inv);
    ConeFpView v;
    for (int r = 0; r < 3; ++r) {
        const double c = -(inv[3 * r] * p4[0] + inv[3 * r + 1] * p4[1] + inv[3 * r + 2] * p4[2]);
        v.src[r] = (c - o[r]) / s[r];
        for (int k = 0; k < 3; ++k) v.inv_ar[3 * r + k] = inv[3 * r + k] / s[r];
    }
    out[t] = v;
}

__global__ void cone_bp_prepare_kernel(const float *__restrict__ P, const float *__restrict__ spacing,
                                       const float *__restrict__ origin, int geom_batch, int n_proj,
                                       ConeBpView *__restrict__ out)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= geom_batch * n_proj) return;
    const int g = t / n_proj;
    const float *p = P + (size_t)t * 12;
    const double sx = spacing[g * 3 + 2], sy = spacing[g * 3 + 1], sz = spacing[g * 3 + 0];
    const double ox = origin[g * 3 + 2], oy = origin[g * 3 + 1], oz = origin[g * 3 + 0];
    ConeBpView v;
    float *r = reinterpret_cast<float *>(v.row);
    for (int k = 0; k < 3; ++k) {
        const double a = p[4 * k], b = p[4 * k + 1], c = p[4 * k + 2], d = p[4 * k + 3];
        r[4 * k + 0] = (float)(a * sx);
        r[4 * k + 1] = (float)(b * sy);
        r[4 * k + 2] = (float)(c * sz);
        r[4 * k + 3] = (float)(a * ox + b * oy + c * oz + d);
    }
    out[t] = v;
}

}  // namespace

cudaError_t launch_cone_fp_prepare(const float *P, const float *spacing, const float *origin, int geom_batch,
                                   int n_proj, ConeFpView *out, cudaStream_t stream)
{
    const int n = geom_batch * n_proj;
    cone_fp_prepare_kernel<<<(n + 127) / 128, 128, 0, stream>>>(P, spacing, origin, geom_batch, n_proj, out);
    return cudaGetLastError();
}

cudaError_t launch_cone_bp_prepare(const float *P, const float *spacing, const float *origin, int geom_batch,
                                   int n_proj, ConeBpView *out, cudaStream_t stream)
{
    const int n = geom_batch * n_proj;
    cone_bp_prepare_kernel<<<(n + 127) / 128, 128, 0, stream>>>(P, spacing, origin, geom_batch, n_proj, out);
    return cudaGetLastError();
}

}  // namespace pyronn
