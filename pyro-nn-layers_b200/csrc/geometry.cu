// geometry.cu -- FP64 device preparation of the cone-beam projection matrices.
//
// The reference decomposes P on the host in FP32 (JacobiSVD null space for the
// camera centre, Eigen inverse for M) once per call and per batch element,
// after blocking device->host copies (cc/ops/cone_projector_3D_OPKernel.cc:96-182,
// cc/helper_headers/helper_geometry_cpu.h:30-43).  Here one thread per view
// does it in FP64 on the stream: C = -M^-1 p4 is the right null vector of
// P = [M | p4] already normalised to C[3] = 1, so no SVD is needed.
#include <math_constants.h>

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
                                       const float *__restrict__ origin, int geom_batch, int n_proj, int X, int Y,
                                       int Z, ConeFpView *__restrict__ out)
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
    // footprint: the eight corners of the box [-0.5, N] (index space, the
    // union of the software [0, N] and texture [-0.5, N - 0.5] boxes) through
    // P; the box is convex and, with every corner on one side of the source,
    // its image is the convex hull of the corners' images
    double u0 = CUDART_INF, u1 = -CUDART_INF, v0 = CUDART_INF, v1 = -CUDART_INF;
    int pos = 0, neg = 0;
    for (int c = 0; c < 8; ++c) {
        const double ix = (c & 1) ? (double)X : -0.5, iy = (c & 2) ? (double)Y : -0.5, iz = (c & 4) ? (double)Z : -0.5;
        const double wx = o[0] + s[0] * ix, wy = o[1] + s[1] * iy, wz = o[2] + s[2] * iz;
        const double hu = (double)p[0] * wx + (double)p[1] * wy + (double)p[2] * wz + (double)p[3];
        const double hv = (double)p[4] * wx + (double)p[5] * wy + (double)p[6] * wz + (double)p[7];
        const double hw = (double)p[8] * wx + (double)p[9] * wy + (double)p[10] * wz + (double)p[11];
        pos += hw > 0.0;
        neg += hw < 0.0;
        const double cu = hu / hw, cv = hv / hw;
        u0 = fmin(u0, cu), u1 = fmax(u1, cu), v0 = fmin(v0, cv), v1 = fmax(v1, cv);
    }
    const bool bounded = (pos == 8 || neg == 8) && isfinite(u0) && isfinite(u1) && isfinite(v0) && isfinite(v1);
    v.foot[0] = bounded ? (float)(u0 - 2.0) : -CUDART_INF_F;
    v.foot[1] = bounded ? (float)(u1 + 2.0) : CUDART_INF_F;
    v.foot[2] = bounded ? (float)(v0 - 2.0) : -CUDART_INF_F;
    v.foot[3] = bounded ? (float)(v1 + 2.0) : CUDART_INF_F;
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
                                   int n_proj, int vol_x, int vol_y, int vol_z, ConeFpView *out, cudaStream_t stream)
{
    const int n = geom_batch * n_proj;
    cone_fp_prepare_kernel<<<(n + 127) / 128, 128, 0, stream>>>(P, spacing, origin, geom_batch, n_proj, vol_x, vol_y,
                                                                vol_z, out);
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
