// proj2d.cu -- 2D parallel-beam and fan-beam projector / backprojector.
//
// Forward (ParallelProjection2D / FanProjection2D): one thread per detector
// pixel, blockIdx.y = view, blockIdx.z = batch element; the ray march follows
// kernel_project2D (par_projector_2D_CudaKernel.cu.cc:28-102): box edges
// index_to_physical(0|N) - 0.5 in mm, first sample at the entry with weight
// 1/2, alpha advanced in a float, step 0.2 * min(spacing) mm, end correction
// only when the sum is > 0, result scaled by |ray (.) spacing| (:141).
// The reference samples a border/linear texture at index + 0.5; here the
// same bilinear interpolation is done with exact FP32 weights.
//
// Backward (ParallelBackprojection2D / FanBackprojection2D): one thread per
// pixel, loop over views, linear interpolation along the detector row.
#include <math_constants.h>

#include "common.cuh"
#include "internal.h"

namespace pyronn {

namespace {

constexpr float PI_REF = 3.14159265359f;  // par_backprojector_2D_CudaKernel.cu.cc:32
constexpr int FP2_BLOCK = 128;
constexpr int BP2_BLOCK_X = 32;
constexpr int BP2_BLOCK_Y = 8;

template <typename T>
__device__ __forceinline__ float interp2d_border(const T *__restrict__ img, float x, float y, int X, int Y)
{
    // sample positions stay inside the box (|x|, |y| << 2^22): exact FADD floor
    const FloorFrac ffx = floor_frac(x), ffy = floor_frac(y);
    const int x0 = ffx.i, y0 = ffy.i;
    const float tx = ffx.f, ty = ffy.f;
    const bool vx0 = (unsigned)x0 < (unsigned)X, vx1 = (unsigned)(x0 + 1) < (unsigned)X;
    const bool vy0 = (unsigned)y0 < (unsigned)Y, vy1 = (unsigned)(y0 + 1) < (unsigned)Y;
    const int base = y0 * X + x0;
    const float p00 = (vy0 && vx0) ? load_as_float(img + base) : 0.0f;
    const float p01 = (vy0 && vx1) ? load_as_float(img + base + 1) : 0.0f;
    const float p10 = (vy1 && vx0) ? load_as_float(img + base + X) : 0.0f;
    const float p11 = (vy1 && vx1) ? load_as_float(img + base + X + 1) : 0.0f;
    const float p0 = lerp_ref(p00, p01, tx);
    const float p1 = lerp_ref(p10, p11, tx);
    return lerp_ref(p0, p1, ty);
}

template <typename T, typename Tout, bool FAN>
__global__ void __launch_bounds__(FP2_BLOCK)
    projection2d_kernel(const T *__restrict__ vol, Tout *__restrict__ sino, Geom2D geo, int X, int Y, int W,
                        int n_proj, int geom_batch)
{
    const int u = blockIdx.x * FP2_BLOCK + threadIdx.x;
    const int p = blockIdx.y;
    const int b = blockIdx.z;
    if (u >= W) return;
    const int g = geom_batch == 1 ? 0 : b;
    const float sx = geo.volume_spacing[2 * g + 1], sy = geo.volume_spacing[2 * g + 0];
    const float ox = geo.volume_origin[2 * g + 1], oy = geo.volume_origin[2 * g + 0];
    const float ds = geo.detector_spacing[g], dorg = geo.detector_origin[g];
    const float2 ray_in = reinterpret_cast<const float2 *>(geo.rays)[(size_t)g * n_proj + p];
    const float uu = (float)u * ds + dorg;

    double srcx, srcy, rx, ry;
    if (!FAN) {
        // par_projector_2D_CudaKernel.cu.cc:120-132
        const float sid = sqrtf((float)((float)X * sx * (float)X * sx) + ((float)Y * sy * (float)Y * sy)) * 1.2f;
        rx = ray_in.x;
        ry = ray_in.y;
        srcx = (double)ray_in.x * -(double)sid + (double)(-ray_in.y) * (double)uu;
        srcy = (double)ray_in.y * -(double)sid + (double)ray_in.x * (double)uu;
    } else {
        // fan_projector_2D_CudaKernel.cu.cc:122-133
        const double sid = geo.sid[g], sdd = geo.sdd[g];
        srcx = ray_in.x * -sid;
        srcy = ray_in.y * -sid;
        const double lx = ray_in.x * sdd + (double)(-ray_in.y) * uu;
        const double ly = ray_in.y * sdd + (double)ray_in.x * uu;
        const double inv = 1.0 / sqrt(lx * lx + ly * ly);
        rx = lx * inv;
        ry = ly * inv;
    }

    // box in mm (the reference's -0.5 is in mm, :38-39,50-51), FP64
    double amin = 0.0, amax = CUDART_INF;
    if (rx != 0.0) {
        const double e0 = (double)ox - 0.5, e1 = (double)X * sx + ox - 0.5;
        const double rc = 1.0 / rx;
        const double a0 = (e0 - srcx) * rc, a1 = (e1 - srcx) * rc;
        amin = fmin(a0, a1);
        amax = fmax(a0, a1);
    }
    if (ry != 0.0) {
        const double e0 = (double)oy - 0.5, e1 = (double)Y * sy + oy - 0.5;
        const double rc = 1.0 / ry;
        const double a0 = (e0 - srcy) * rc, a1 = (e1 - srcy) * rc;
        amin = fmax(amin, fmin(a0, a1));
        amax = fmin(amax, fmax(a0, a1));
    }

    const float step = 0.2f * fminf(sx, sy);
    const float dx = (float)rx, dy = (float)ry;
    float pixel = 0.0f;
    if (step > 0.0f && amin < amax) {
        const T *img = vol + (size_t)b * X * Y;
        // sample positions in index space: idx = (src + a r - o) / s
        const float isx = 1.0f / sx, isy = 1.0f / sy;
        const float bx = (float)((srcx - ox) / sx), by = (float)((srcy - oy) / sy);
        const float gx = dx * isx, gy = dy * isy;
        float a = (float)amin;
        const float am = (float)amax;
        const double bound = ((double)am - (double)a) / (double)step + 4.0;
        const int max_iter = bound > 1.0e8 ? 100000000 : (int)bound;
        float px = 0.0f, py = 0.0f;
        int iter = 0;
        if (a < am) {
            px = fmaf(a, gx, bx);
            py = fmaf(a, gy, by);
            pixel += 0.5f * interp2d_border<T>(img, px, py, X, Y);
            a += step;
            ++iter;
        }
        // two samples per iteration (their gathers overlap); same alpha
        // sequence and the same order of additions as one at a time
        while (a < am && iter < max_iter) {
            const float a1 = a + step;
            if (a1 < am && iter + 1 < max_iter) {
                const float qx = fmaf(a, gx, bx), qy = fmaf(a, gy, by);
                px = fmaf(a1, gx, bx);
                py = fmaf(a1, gy, by);
                const float v0 = interp2d_border<T>(img, qx, qy, X, Y);
                const float v1 = interp2d_border<T>(img, px, py, X, Y);
                pixel += v0;
                pixel += v1;
                a = a1 + step;
                iter += 2;
            } else {
                px = fmaf(a, gx, bx);
                py = fmaf(a, gy, by);
                pixel += interp2d_border<T>(img, px, py, X, Y);
                a += step;
                ++iter;
            }
        }
        pixel *= step;
        if (pixel > 0.0f) {  // :88-100
            const float last_val = interp2d_border<T>(img, px, py, X, Y);
            pixel -= 0.5f * step * last_val;
            a -= step;
            const float last_step = am - a;
            pixel += 0.5f * last_step * last_val;
            px = fmaf(am, gx, bx);
            py = fmaf(am, gy, by);
            pixel += 0.5f * last_step * interp2d_border<T>(img, px, py, X, Y);
        }
        pixel *= sqrtf((dx * sx) * (dx * sx) + (dy * sy) * (dy * sy));  // :141
    }
    store_from_float(sino + ((size_t)b * n_proj + p) * W + u, pixel);
}

template <typename T, typename Tout, bool FAN>
__global__ void __launch_bounds__(BP2_BLOCK_X *BP2_BLOCK_Y)
    backprojection2d_kernel(const T *__restrict__ sino, Tout *__restrict__ vol, Geom2D geo, int X, int Y, int W,
                            int n_proj, int geom_batch)
{
    const int i = blockIdx.x * BP2_BLOCK_X + threadIdx.x;
    const int j = blockIdx.y * BP2_BLOCK_Y + threadIdx.y;
    const int b = blockIdx.z;
    if (i >= X || j >= Y) return;
    const int g = geom_batch == 1 ? 0 : b;
    const float sx = geo.volume_spacing[2 * g + 1], sy = geo.volume_spacing[2 * g + 0];
    const float ox = geo.volume_origin[2 * g + 1], oy = geo.volume_origin[2 * g + 0];
    const float ds = geo.detector_spacing[g], dorg = geo.detector_origin[g];
    const float ids = 1.0f / ds;
    const float cx = (float)i * sx + ox, cy = (float)j * sy + oy;
    const float2 *rays = reinterpret_cast<const float2 *>(geo.rays) + (size_t)g * n_proj;
    const T *sino_b = sino + (size_t)b * n_proj * W;
    float sid = 0.0f, sdd = 0.0f;
    if (FAN) {
        sid = geo.sid[g];
        sdd = geo.sdd[g];
    }
    float acc = 0.0f;
    for (int n = 0; n < n_proj; ++n) {
        const float2 r = __ldg(&rays[n]);
        // detector direction (-r.y, r.x), par_backprojector_2D_CudaKernel.cu.cc:48-49
        float s, w = 1.0f;
        if (!FAN) {
            s = cx * -r.y + cy * r.x;  // :51
        } else {
            // intersectLines2D(pixel, source, centre, centre + det) of
            // fan_backprojector_2D_CudaKernel.cu.cc:52-57 in closed form:
            // s = SDD |r|^2 <c, d> / (<c, r> + SID |r|^2), weight 1 / |c - src|^2
            const float rr = r.x * r.x + r.y * r.y;
            const float cd = cx * -r.y + cy * r.x;
            const float cr = cx * r.x + cy * r.y;
            s = sdd * rr * cd / fmaf(sid, rr, cr);
            const float ex = fmaf(r.x, sid, cx), ey = fmaf(r.y, sid, cy);
            w = 1.0f / fmaf(ex, ex, ey * ey);
        }
        const float sidx = (s - dorg) * ids;
        const float fu = floorf(sidx);
        const float t = sidx - fu;
        const int x0 = __float2int_rz(fu);
        const T *row = sino_b + (size_t)n * W;
        const float p0 = (unsigned)x0 < (unsigned)W ? load_as_float(row + x0) : 0.0f;
        const float p1 = (unsigned)(x0 + 1) < (unsigned)W ? load_as_float(row + x0 + 1) : 0.0f;
        acc = fmaf(lerp_ref(p0, p1, t), w, acc);
    }
    float out;
    if (!FAN)
        out = PI_REF * acc / (float)n_proj;  // :58
    else
        out = sid * sdd * PI_REF * acc / (float)n_proj;  // fan_backprojector_2D_CudaKernel.cu.cc:64
    store_from_float(vol + ((size_t)b * Y + j) * X + i, out);
}

template <typename Tin, typename Tout>
cudaError_t fp_typed(const void *volume, void *sinogram, bool fan, const Dims2D &d, const Geom2D &g,
                     cudaStream_t stream)
{
    const dim3 grid((d.det_w + FP2_BLOCK - 1) / FP2_BLOCK, d.n_proj, d.batch);
    if (fan)
        projection2d_kernel<Tin, Tout, true><<<grid, FP2_BLOCK, 0, stream>>>(
            (const Tin *)volume, (Tout *)sinogram, g, d.vol_x, d.vol_y, d.det_w, d.n_proj, d.geom_batch);
    else
        projection2d_kernel<Tin, Tout, false><<<grid, FP2_BLOCK, 0, stream>>>(
            (const Tin *)volume, (Tout *)sinogram, g, d.vol_x, d.vol_y, d.det_w, d.n_proj, d.geom_batch);
    return cudaGetLastError();
}

template <typename Tin, typename Tout>
cudaError_t bp_typed(const void *sinogram, void *volume, bool fan, const Dims2D &d, const Geom2D &g,
                     cudaStream_t stream)
{
    const dim3 block(BP2_BLOCK_X, BP2_BLOCK_Y);
    const dim3 grid((d.vol_x + BP2_BLOCK_X - 1) / BP2_BLOCK_X, (d.vol_y + BP2_BLOCK_Y - 1) / BP2_BLOCK_Y,
                    d.batch);
    if (fan)
        backprojection2d_kernel<Tin, Tout, true><<<grid, block, 0, stream>>>(
            (const Tin *)sinogram, (Tout *)volume, g, d.vol_x, d.vol_y, d.det_w, d.n_proj, d.geom_batch);
    else
        backprojection2d_kernel<Tin, Tout, false><<<grid, block, 0, stream>>>(
            (const Tin *)sinogram, (Tout *)volume, g, d.vol_x, d.vol_y, d.det_w, d.n_proj, d.geom_batch);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_projection2d(const void *volume, void *sinogram, int in_dtype, int out_dtype, bool fan,
                                const Dims2D &d, const Geom2D &g, cudaStream_t stream)
{
    return dispatch_dtypes(in_dtype, out_dtype, [&](auto tin, auto tout) {
        using Tin = typename decltype(tin)::type;
        using Tout = typename decltype(tout)::type;
        return fp_typed<Tin, Tout>(volume, sinogram, fan, d, g, stream);
    });
}

cudaError_t launch_backprojection2d(const void *sinogram, void *volume, int in_dtype, int out_dtype, bool fan,
                                    const Dims2D &d, const Geom2D &g, cudaStream_t stream)
{
    return dispatch_dtypes(in_dtype, out_dtype, [&](auto tin, auto tout) {
        using Tin = typename decltype(tin)::type;
        using Tout = typename decltype(tout)::type;
        return bp_typed<Tin, Tout>(sinogram, volume, fan, d, g, stream);
    });
}

}  // namespace pyronn
