/*
 * oracle.c -- CPU oracle for the PYRO-NN-Layers projector ops.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (the pyro-nn-layers_b200
 * package, its CUDA library or its C ABI) links or calls this file; only the
 * tests, __graft_entry__.smoke() and bench.py's CPU-baseline / reference legs
 * do, and only to check or to time against it.
 *
 * It restates, in FP64 C, the arithmetic of the reference CUDA kernels
 * (file:line citations are relative to the PYRO-NN-Layers source tree), with
 * the reference's discretisation kept on purpose:
 *   - the ray parameter alpha advances in FP32 (`min_alpha += step_size` on a
 *     float), so the oracle samples exactly where the reference samples;
 *     every other quantity is FP64;
 *   - the 2D box is index_to_physical(0|N) - 0.5 in mm and the final 2D scale
 *     is |ray (.) spacing| (par_projector_2D_CudaKernel.cu.cc:38-39,141);
 *   - the trapezoid end correction only runs when the sum is > 0
 *     (cone_projector_3D_CudaKernel.cu.cc:164, par_projector_2D_CudaKernel.cu.cc:88);
 *   - software-interp cone box is [0, N] and starts half a step in
 *     (cone_projector_3D_CudaKernel.cu.cc:96-135); hardware-interp box is
 *     [-0.5, N-0.5] (cone_projector_3D_CudaKernel_hardware_interp.cu.cc:53-89);
 *   - interp2D of the software cone backprojector accepts taps up to x == W and
 *     y == H and reads them from the flat buffer (next row / next view), the
 *     `>` bounds of cone_backprojector_3D_CudaKernel.cu.cc:68-71; a tap past
 *     the end of the whole sinogram buffer (undefined in the reference) reads 0;
 *   - texture fetches (border address mode, linear filter, unnormalised
 *     coordinates at p + 0.5) are bilinear/trilinear interpolation at p with
 *     zero outside the grid and EXACT weights (the hardware's 8-bit weights
 *     are the reason hardware-interp parity is 5e-3, not 1e-5).
 *
 * Compile: gcc -O2 -ffp-contract=off -fPIC -shared -pthread -o liboracle.so oracle.c -lm
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define PI_F 3.14159265359f /* par_backprojector_2D_CudaKernel.cu.cc:32 */

/* ------------------------------------------------------------------ threads */

typedef void (*work_fn)(void *ctx, long item);
typedef struct {
    work_fn fn;
    void *ctx;
    long n_items;
    long next;
    pthread_mutex_t lock;
} pool_t;

static void *pool_worker(void *arg)
{
    pool_t *p = (pool_t *)arg;
    for (;;) {
        pthread_mutex_lock(&p->lock);
        long it = p->next++;
        pthread_mutex_unlock(&p->lock);
        if (it >= p->n_items) break;
        p->fn(p->ctx, it);
    }
    return NULL;
}

static void parallel_for(long n_items, int nthreads, work_fn fn, void *ctx)
{
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 512) nthreads = 512;
    if (nthreads > n_items) nthreads = (int)(n_items > 0 ? n_items : 1);
    pool_t p;
    p.fn = fn;
    p.ctx = ctx;
    p.n_items = n_items;
    p.next = 0;
    pthread_mutex_init(&p.lock, NULL);
    if (nthreads == 1) {
        pool_worker(&p);
    } else {
        pthread_t th[512];
        for (int i = 0; i < nthreads; ++i) pthread_create(&th[i], NULL, pool_worker, &p);
        for (int i = 0; i < nthreads; ++i) pthread_join(th[i], NULL);
    }
    pthread_mutex_destroy(&p.lock);
}

/* -------------------------------------------------------- interpolation */

/* Texture fetch of a 2D border/linear texture at (x + 0.5, y + 0.5): bilinear
 * at (x, y), texel centres at integers, zero outside [0,W-1] x [0,H-1]. */
static double bilinear_border(const float *img, long W, long H, double x, double y)
{
    double xf = floor(x), yf = floor(y);
    double fx = x - xf, fy = y - yf;
    long x0 = (long)xf, y0 = (long)yf;
    double t[2][2];
    for (int dy = 0; dy < 2; ++dy)
        for (int dx = 0; dx < 2; ++dx) {
            long xx = x0 + dx, yy = y0 + dy;
            t[dy][dx] = (xx < 0 || xx >= W || yy < 0 || yy >= H) ? 0.0 : (double)img[yy * W + xx];
        }
    double r0 = t[0][0] + fx * (t[0][1] - t[0][0]);
    double r1 = t[1][0] + fx * (t[1][1] - t[1][0]);
    return r0 + fy * (r1 - r0);
}

/* interp3D, cone_projector_3D_CudaKernel.cu.cc:42-85 (and tex3D(p+0.5) of the
 * hardware path, which has the same taps): trilinear at (x,y,z), zero outside. */
static double trilinear_border(const float *vol, long X, long Y, long Z, double x, double y, double z)
{
    double xf = floor(x), yf = floor(y), zf = floor(z);
    double fx = x - xf, fy = y - yf, fz = z - zf;
    long x0 = (long)xf, y0 = (long)yf, z0 = (long)zf;
    double c[2][2][2];
    for (int dz = 0; dz < 2; ++dz)
        for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx) {
                long xx = x0 + dx, yy = y0 + dy, zz = z0 + dz;
                c[dz][dy][dx] = (xx < 0 || xx >= X || yy < 0 || yy >= Y || zz < 0 || zz >= Z)
                                    ? 0.0
                                    : (double)vol[(zz * Y + yy) * X + xx];
            }
    /* same lerp order as the reference: z first, then y, then x */
    double c00 = c[0][0][0] + fz * (c[1][0][0] - c[0][0][0]);
    double c01 = c[0][0][1] + fz * (c[1][0][1] - c[0][0][1]);
    double c10 = c[0][1][0] + fz * (c[1][1][0] - c[0][1][0]);
    double c11 = c[0][1][1] + fz * (c[1][1][1] - c[0][1][1]);
    double c0 = c00 + fy * (c10 - c00);
    double c1 = c01 + fy * (c11 - c01);
    return c0 + fx * (c1 - c0);
}

/* interp2D, cone_backprojector_3D_CudaKernel.cu.cc:55-82, with its `>` bounds:
 * taps with 0 <= x <= W and 0 <= y <= H are read from the flat sinogram at
 * n*H*W + y*W + x (so x == W reads the next row, y == H the next view). */
static double bilinear_quirk(const float *sino, long W, long H, long total, long n, double x, double y)
{
    double xf = floor(x), yf = floor(y);
    double fx = x - xf, fy = y - yf;
    long x0 = (long)xf, y0 = (long)yf;
    double t[2][2];
    for (int dy = 0; dy < 2; ++dy)
        for (int dx = 0; dx < 2; ++dx) {
            long xx = x0 + dx, yy = y0 + dy;
            long idx = n * H * W + yy * W + xx;
            t[dy][dx] = (xx < 0 || xx > W || yy < 0 || yy > H || idx >= total) ? 0.0 : (double)sino[idx];
        }
    double r0 = t[0][0] + fx * (t[0][1] - t[0][0]);
    double r1 = t[1][0] + fx * (t[1][1] - t[1][0]);
    return r0 + fy * (r1 - r0);
}

/* ------------------------------------------------------------- 2D forward */

typedef struct {
    const float *img;
    long X, Y;
    double ox, oy, sx, sy;
} grid2d_t;

static double tex2d_mm(const grid2d_t *g, double px, double py)
{
    return bilinear_border(g->img, g->X, g->Y, (px - g->ox) / g->sx, (py - g->oy) / g->sy);
}

/* kernel_project2D, par_projector_2D_CudaKernel.cu.cc:28-102 (identical in
 * fan_projector_2D_CudaKernel.cu.cc:27-102).  Returns the sum and, if
 * n_samples != NULL, adds the number of samples taken. */
static double project2d(const grid2d_t *g, double srcx, double srcy, double rx, double ry, float step,
                        long long *n_samples)
{
    double min_a = 0.0, max_a = INFINITY;
    if (rx != 0.0) {
        double e0 = 0.0 * g->sx + g->ox - 0.5;
        double e1 = (double)g->X * g->sx + g->ox - 0.5;
        double r = 1.0 / rx;
        double a0 = (e0 - srcx) * r, a1 = (e1 - srcx) * r;
        min_a = fmin(a0, a1);
        max_a = fmax(a0, a1);
    }
    if (ry != 0.0) {
        double e0 = 0.0 * g->sy + g->oy - 0.5;
        double e1 = (double)g->Y * g->sy + g->oy - 0.5;
        double r = 1.0 / ry;
        double a0 = (e0 - srcy) * r, a1 = (e1 - srcy) * r;
        min_a = fmax(min_a, fmin(a0, a1));
        max_a = fmin(max_a, fmax(a0, a1));
    }
    /* the reference keeps alpha in a float */
    float a = (float)min_a;
    float amax = (float)max_a;
    double pixel = 0.0, px = 0.0, py = 0.0;
    long long cnt = 0;
    if (a < amax) {
        px = srcx + (double)a * rx;
        py = srcy + (double)a * ry;
        pixel += 0.5 * tex2d_mm(g, px, py);
        a += step;
        ++cnt;
    }
    while (a < amax) {
        px = srcx + (double)a * rx;
        py = srcy + (double)a * ry;
        pixel += tex2d_mm(g, px, py);
        a += step;
        ++cnt;
    }
    pixel *= (double)step;
    if (pixel > 0.0) {
        double last_val = tex2d_mm(g, px, py);
        pixel -= 0.5 * (double)step * last_val;
        a -= step;
        double last = (double)amax - (double)a;
        pixel += 0.5 * last * last_val;
        px = srcx + (double)amax * rx;
        py = srcy + (double)amax * ry;
        pixel += 0.5 * last * tex2d_mm(g, px, py);
    }
    if (n_samples) *n_samples += cnt;
    return pixel;
}

typedef struct {
    const float *vol;
    double *sino;
    int batch, Y, X, n_proj, W, geom_batch, fan;
    const float *vol_origin, *det_origin, *vol_spacing, *det_spacing, *rays, *sid, *sdd;
    long long *counts; /* per (b, view) sample counts, may be NULL */
} fp2d_ctx;

static void fp2d_item(void *vctx, long item)
{
    fp2d_ctx *c = (fp2d_ctx *)vctx;
    int b = (int)(item / c->n_proj), p = (int)(item % c->n_proj);
    int gb = c->geom_batch == 1 ? 0 : b;
    grid2d_t g;
    g.img = c->vol + (long)b * c->Y * c->X;
    g.X = c->X;
    g.Y = c->Y;
    g.sx = c->vol_spacing[gb * 2 + 1];
    g.sy = c->vol_spacing[gb * 2 + 0];
    g.ox = c->vol_origin[gb * 2 + 1];
    g.oy = c->vol_origin[gb * 2 + 0];
    double ds = c->det_spacing[gb], dorg = c->det_origin[gb];
    double rx = c->rays[((long)gb * c->n_proj + p) * 2 + 0];
    double ry = c->rays[((long)gb * c->n_proj + p) * 2 + 1];
    float step = 0.2f * fminf((float)g.sx, (float)g.sy); /* :136,166 / fan :138,182 */
    long long cnt = 0;
    for (int u = 0; u < c->W; ++u) {
        double uu = (double)u * ds + dorg;
        double sx, sy, dx, dy;
        if (!c->fan) {
            /* par_projector_2D_CudaKernel.cu.cc:120-132: the virtual source
             * point is formed in FP32 as the reference forms it (its sid, the
             * detector coordinate, and ray * (-sid) + u_vec * u with the
             * second product fused): a ray that grazes the box -- e.g. along
             * an axis with a 1e-17 cross component -- enters or misses on
             * that rounding */
            float fsx = (float)g.sx, fsy = (float)g.sy, fX = (float)c->X, fY = (float)c->Y;
            float fsid = sqrtf((fX * fsx * fX * fsx) + (fY * fsy * fY * fsy)) * 1.2f;
            float fu = fmaf((float)u, (float)ds, (float)dorg);
            float frx = (float)rx, fry = (float)ry;
            sx = (double)fmaf(-fry, fu, frx * -fsid);
            sy = (double)fmaf(frx, fu, fry * -fsid);
            dx = rx;
            dy = ry;
        } else {
            /* fan_projector_2D_CudaKernel.cu.cc:122-133 */
            double sid = c->sid[gb], sdd = c->sdd[gb];
            sx = rx * (-sid);
            sy = ry * (-sid);
            double px = sx + rx * sdd + (-ry) * uu;
            double py = sy + ry * sdd + rx * uu;
            double lx = px - sx, ly = py - sy;
            double inv = 1.0 / sqrt(lx * lx + ly * ly);
            dx = lx * inv;
            dy = ly * inv;
        }
        double pix = project2d(&g, sx, sy, dx, dy, step, &cnt);
        pix *= sqrt((dx * g.sx) * (dx * g.sx) + (dy * g.sy) * (dy * g.sy));
        c->sino[((long)b * c->n_proj + p) * c->W + u] = pix;
    }
    if (c->counts) c->counts[item] = cnt;
}

/* ParallelProjection2D: par_projector_2D_CudaKernel.cu.cc:104-147 */
void oracle_parallel_projection2d(const float *vol, double *sino, int batch, int Y, int X, int n_proj, int W,
                                  const float *vol_origin, const float *det_origin, const float *vol_spacing,
                                  const float *det_spacing, const float *rays, int geom_batch, int nthreads,
                                  long long *counts)
{
    fp2d_ctx c = {vol, sino, batch, Y, X, n_proj, W, geom_batch, 0, vol_origin, det_origin, vol_spacing,
                  det_spacing, rays, NULL, NULL, counts};
    parallel_for((long)batch * n_proj, nthreads, fp2d_item, &c);
}

/* FanProjection2D: fan_projector_2D_CudaKernel.cu.cc:104-149 */
void oracle_fan_projection2d(const float *vol, double *sino, int batch, int Y, int X, int n_proj, int W,
                             const float *vol_origin, const float *det_origin, const float *vol_spacing,
                             const float *det_spacing, const float *sid, const float *sdd, const float *rays,
                             int geom_batch, int nthreads, long long *counts)
{
    fp2d_ctx c = {vol, sino, batch, Y, X, n_proj, W, geom_batch, 1, vol_origin, det_origin, vol_spacing,
                  det_spacing, rays, sid, sdd, counts};
    parallel_for((long)batch * n_proj, nthreads, fp2d_item, &c);
}

/* ---------------------------------------------------------- 2D backprojection */

typedef struct {
    const float *sino;
    double *vol;
    int batch, n_proj, W, Y, X, geom_batch, fan;
    const float *vol_origin, *det_origin, *vol_spacing, *det_spacing, *rays, *sid, *sdd;
} bp2d_ctx;

/* intersectLines2D, helper_geometry_gpu.h:28-44 (NaN when near-parallel) */
static void intersect_lines(double p1x, double p1y, double p2x, double p2y, double p3x, double p3y, double p4x,
                            double p4y, double *ox, double *oy)
{
    double dn = (p1x - p2x) * (p3y - p4y) - (p1y - p2y) * (p3x - p4x);
    if (dn < 0.000001 && dn > -0.000001) {
        *ox = NAN;
        *oy = NAN;
        return;
    }
    double a = p1x * p2y - p1y * p2x, bq = p3x * p4y - p3y * p4x;
    *ox = (a * (p3x - p4x) - (p1x - p2x) * bq) / dn;
    *oy = (a * (p3y - p4y) - (p1y - p2y) * bq) / dn;
}

/* Detector index of pixel (cx, cy) for a fan view by the reference's FP32
 * steps (fan_backprojector_2D_CudaKernel.cu.cc:47-59 with intersectLines2D,
 * helper_geometry_gpu.h:28-44), each operation rounded once (this file is
 * built with -ffp-contract=off): near the source's depth the reference's FP32
 * intersection is far from the exact one -- NaN below its 1e-6 threshold,
 * which its texture samples as coordinate 0 (index -0.5), a far-off point
 * just above.  The GPU kernel takes the same steps there. */
static double fan_index_reference_steps(float cx, float cy, float rx, float ry, float sid, float sdd, float dorg,
                                        float ds)
{
    float srcx = rx * -sid, srcy = ry * -sid;
    float cpx = srcx + rx * sdd, cpy = srcy + ry * sdd;
    float detx = -ry, dety = rx;
    float p4x = cpx + detx, p4y = cpy + dety;
    float a1 = cx - srcx, b1 = cpy - p4y, a2 = cy - srcy, b2 = cpx - p4x;
    float dn = a1 * b1 - a2 * b2;
    if (dn < 0.000001f && dn > -0.000001f) return -0.5;
    float x12 = cx * srcy - cy * srcx, x34 = cpx * p4y - cpy * p4x;
    float x = (x12 * b2 - a1 * x34) / dn, y = (x12 * b1 - a2 * x34) / dn;
    float s = x * detx + y * dety;
    return (double)((s - dorg) / ds);
}

static void bp2d_item(void *vctx, long item)
{
    bp2d_ctx *c = (bp2d_ctx *)vctx;
    int b = (int)(item / c->Y), y = (int)(item % c->Y);
    int gb = c->geom_batch == 1 ? 0 : b;
    double sx = c->vol_spacing[gb * 2 + 1], sy = c->vol_spacing[gb * 2 + 0];
    double ox = c->vol_origin[gb * 2 + 1], oy = c->vol_origin[gb * 2 + 0];
    double ds = c->det_spacing[gb], dorg = c->det_origin[gb];
    const float *sino = c->sino + (long)b * c->n_proj * c->W;
    const float *rays = c->rays + (long)gb * c->n_proj * 2;
    for (int x = 0; x < c->X; ++x) {
        double cx = x * sx + ox, cy = y * sy + oy;
        double acc = 0.0;
        for (int n = 0; n < c->n_proj; ++n) {
            double rx = rays[2 * n], ry = rays[2 * n + 1];
            double dvx = -ry, dvy = rx;
            double s, w = 1.0;
            if (!c->fan) {
                /* par_backprojector_2D_CudaKernel.cu.cc:46-55 */
                s = cx * dvx + cy * dvy;
            } else {
                /* fan_backprojector_2D_CudaKernel.cu.cc:47-61 */
                double sid = c->sid[gb], sdd = c->sdd[gb];
                double srx = rx * (-sid), sry = ry * (-sid);
                double cpx = srx + rx * sdd, cpy = sry + ry * sdd;
                double ix, iy;
                intersect_lines(cx, cy, srx, sry, cpx, cpy, cpx + dvx, cpy + dvy, &ix, &iy);
                double dx = cx - srx, dy = cy - sry;
                w = 1.0 / sqrt(dx * dx + dy * dy);
                w = w * w;
                s = ix * dvx + iy * dvy;
            }
            double sidx = (s - dorg) / ds;
            if (c->fan) {
                /* within 1e-2 mm of the source's depth the reference's FP32
                 * steps decide (see fan_index_reference_steps) */
                double sid = c->sid[gb], sdd = c->sdd[gb];
                double depth = (cx + rx * sid) * rx + (cy + ry * sid) * ry;
                if (fabs(depth) < 1e-2)
                    sidx = fan_index_reference_steps((float)cx, (float)cy, (float)rx, (float)ry, (float)sid, (float)sdd,
                                                     (float)dorg, (float)ds);
            }
            /* tex2D(s_idx + 0.5, n + 0.5): row n exactly, linear along u */
            acc += bilinear_border(sino, c->W, c->n_proj, sidx, (double)n) * w;
        }
        double scale = (double)PI_F / (double)c->n_proj;
        if (c->fan) scale *= (double)c->sid[gb] * (double)c->sdd[gb];
        c->vol[((long)b * c->Y + y) * c->X + x] = acc * scale;
    }
}

/* ParallelBackprojection2D: par_backprojector_2D_CudaKernel.cu.cc:28-61 */
void oracle_parallel_backprojection2d(const float *sino, double *vol, int batch, int n_proj, int W, int Y, int X,
                                      const float *vol_origin, const float *det_origin, const float *vol_spacing,
                                      const float *det_spacing, const float *rays, int geom_batch, int nthreads)
{
    bp2d_ctx c = {sino, vol, batch, n_proj, W, Y, X, geom_batch, 0, vol_origin, det_origin, vol_spacing,
                  det_spacing, rays, NULL, NULL};
    parallel_for((long)batch * Y, nthreads, bp2d_item, &c);
}

/* FanBackprojection2D: fan_backprojector_2D_CudaKernel.cu.cc:29-67 */
void oracle_fan_backprojection2d(const float *sino, double *vol, int batch, int n_proj, int W, int Y, int X,
                                 const float *vol_origin, const float *det_origin, const float *vol_spacing,
                                 const float *det_spacing, const float *sid, const float *sdd, const float *rays,
                                 int geom_batch, int nthreads)
{
    bp2d_ctx c = {sino, vol, batch, n_proj, W, Y, X, geom_batch, 1, vol_origin, det_origin, vol_spacing,
                  det_spacing, rays, sid, sdd};
    parallel_for((long)batch * Y, nthreads, bp2d_item, &c);
}

/* ---------------------------------------------- cone geometry decomposition */

/* DecomposeProjectionMatrices, cone_projector_3D_OPKernel.cc:96-182, in FP64.
 * P = [M | p4]; the camera centre C (right null vector of P normalised to
 * C[3] = 1, helper_geometry_cpu.h:30-43) is -M^-1 p4; the source in voxel
 * index space is (C - origin) / spacing (:165-169) and
 * invAR = diag(1/sx, 1/sy, 1/sz) M^-1 (:148-152, 171).
 * P: [n,3,4]; spacing/origin: [3] in (z,y,x) order; out invAR [n,9], src [n,3]. */
void oracle_cone_decompose(const float *P, const float *spacing, const float *origin, int n_proj, double *invAR,
                           double *src)
{
    double s[3] = {spacing[2], spacing[1], spacing[0]};
    double o[3] = {origin[2], origin[1], origin[0]};
    for (int n = 0; n < n_proj; ++n) {
        const float *m = P + 12 * n;
        double a = m[0], b = m[1], c = m[2], d = m[4], e = m[5], f = m[6], g = m[8], h = m[9], i = m[10];
        double A = e * i - f * h, B = -(d * i - f * g), C = d * h - e * g;
        double det = a * A + b * B + c * C;
        double inv[9];
        inv[0] = A / det;
        inv[1] = -(b * i - c * h) / det;
        inv[2] = (b * f - c * e) / det;
        inv[3] = B / det;
        inv[4] = (a * i - c * g) / det;
        inv[5] = -(a * f - c * d) / det;
        inv[6] = C / det;
        inv[7] = -(a * h - b * g) / det;
        inv[8] = (a * e - b * d) / det;
        double p4[3] = {m[3], m[7], m[11]};
        for (int r = 0; r < 3; ++r) {
            double cc = -(inv[3 * r] * p4[0] + inv[3 * r + 1] * p4[1] + inv[3 * r + 2] * p4[2]);
            src[3 * n + r] = (cc - o[r]) / s[r];
            for (int k = 0; k < 3; ++k) invAR[9 * n + 3 * r + k] = inv[3 * r + k] / s[r];
        }
    }
}

/* ----------------------------------------------------------- cone forward */

typedef struct {
    const float *vol;
    double *sino;
    int batch, Z, Y, X, n_proj, H, W, geom_batch, hw;
    const float *vol_origin, *vol_spacing, *P, *step;
    double *invAR, *src; /* [geom_batch, n_proj, 9|3] */
    long long *counts;
} fp3d_ctx;

static void fp3d_item(void *vctx, long item)
{
    fp3d_ctx *c = (fp3d_ctx *)vctx;
    int b = (int)(item / c->n_proj), p = (int)(item % c->n_proj);
    int gb = c->geom_batch == 1 ? 0 : b;
    const double *M = c->invAR + ((long)gb * c->n_proj + p) * 9;
    const double *S = c->src + ((long)gb * c->n_proj + p) * 3;
    const float *vol = c->vol + (long)b * c->Z * c->Y * c->X;
    double sp[3] = {c->vol_spacing[gb * 3 + 2], c->vol_spacing[gb * 3 + 1], c->vol_spacing[gb * 3 + 0]};
    float step = c->step[gb];
    long N[3] = {c->X, c->Y, c->Z};
    double lo = c->hw ? -0.5 : 0.0, hi_off = c->hw ? -0.5 : 0.0;
    long long cnt = 0;
    for (int v = 0; v < c->H; ++v)
        for (int u = 0; u < c->W; ++u) {
            /* cone_projector_3D_CudaKernel.cu.cc:200-205 */
            double r[3];
            for (int k = 0; k < 3; ++k) r[k] = M[3 * k + 2] + v * M[3 * k + 1] + u * M[3 * k + 0];
            double len = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
            for (int k = 0; k < 3; ++k) r[k] /= len;
            /* box, :96-132 (sw) / hardware_interp :51-86 */
            double min_a = 0.0, max_a = INFINITY;
            for (int k = 0; k < 3; ++k) {
                if (r[k] != 0.0) {
                    double e0 = lo, e1 = (double)N[k] + hi_off;
                    double rc = 1.0 / r[k];
                    double a0 = (e0 - S[k]) * rc, a1 = (e1 - S[k]) * rc;
                    if (k == 0) { /* the x test assigns, y and z intersect */
                        min_a = fmin(a0, a1);
                        max_a = fmax(a0, a1);
                    } else {
                        min_a = fmax(min_a, fmin(a0, a1));
                        max_a = fmin(max_a, fmax(a0, a1));
                    }
                }
            }
            float a = (float)min_a;
            a += step * 0.5f; /* :135 */
            float amax = (float)max_a;
            double pixel = 0.0, pt[3] = {0, 0, 0};
            if (a < amax) {
                for (int k = 0; k < 3; ++k) pt[k] = S[k] + (double)a * r[k];
                pixel += 0.5 * trilinear_border(vol, c->X, c->Y, c->Z, pt[0], pt[1], pt[2]);
                a += step;
                ++cnt;
            }
            while (a < amax) {
                for (int k = 0; k < 3; ++k) pt[k] = S[k] + (double)a * r[k];
                pixel += trilinear_border(vol, c->X, c->Y, c->Z, pt[0], pt[1], pt[2]);
                a += step;
                ++cnt;
            }
            pixel *= (double)step;
            if (pixel > 0.0) { /* :164-179 */
                double lv = trilinear_border(vol, c->X, c->Y, c->Z, pt[0], pt[1], pt[2]);
                pixel -= 0.5 * (double)step * lv;
                a -= step;
                double last = (double)amax - (double)a;
                pixel += 0.5 * last * lv;
                for (int k = 0; k < 3; ++k) pt[k] = S[k] + (double)amax * r[k];
                pixel += 0.5 * last * trilinear_border(vol, c->X, c->Y, c->Z, pt[0], pt[1], pt[2]);
            }
            /* :217-219 */
            pixel *= sqrt((r[0] * sp[0]) * (r[0] * sp[0]) + (r[1] * sp[1]) * (r[1] * sp[1]) +
                          (r[2] * sp[2]) * (r[2] * sp[2]));
            c->sino[(((long)b * c->n_proj + p) * c->H + v) * c->W + u] = pixel;
        }
    if (c->counts) c->counts[item] = cnt;
}

/* ConeProjection3D: cone_projector_3D_CudaKernel.cu.cc:182-223 (hardware_interp=0)
 * and cone_projector_3D_CudaKernel_hardware_interp.cu.cc:144-182 (=1), after
 * the per-batch-element decomposition of cone_projector_3D_OPKernel.cc:234-247. */
void oracle_cone_projection3d(const float *vol, double *sino, int hardware_interp, int batch, int Z, int Y, int X,
                              int n_proj, int H, int W, const float *vol_origin, const float *vol_spacing,
                              const float *P, const float *step, int geom_batch, int nthreads, long long *counts)
{
    double *invAR = (double *)malloc(sizeof(double) * 9 * (size_t)geom_batch * n_proj);
    double *src = (double *)malloc(sizeof(double) * 3 * (size_t)geom_batch * n_proj);
    for (int g = 0; g < geom_batch; ++g)
        oracle_cone_decompose(P + (size_t)g * n_proj * 12, vol_spacing + 3 * g, vol_origin + 3 * g, n_proj,
                              invAR + (size_t)g * n_proj * 9, src + (size_t)g * n_proj * 3);
    fp3d_ctx c = {vol, sino, batch, Z, Y, X, n_proj, H, W, geom_batch, hardware_interp, vol_origin, vol_spacing,
                  P, step, invAR, src, counts};
    parallel_for((long)batch * n_proj, nthreads, fp3d_item, &c);
    free(invAR);
    free(src);
}

/* ------------------------------------------------------ cone backprojection */

typedef struct {
    const float *sino;
    double *vol;
    int batch, n_proj, H, W, Z, Y, X, geom_batch, hw;
    const float *vol_origin, *vol_spacing, *P, *mult;
} bp3d_ctx;

static void bp3d_item(void *vctx, long item)
{
    bp3d_ctx *c = (bp3d_ctx *)vctx;
    int b = (int)(item / c->Z), k = (int)(item % c->Z);
    int gb = c->geom_batch == 1 ? 0 : b;
    double sx = c->vol_spacing[gb * 3 + 2], sy = c->vol_spacing[gb * 3 + 1], sz = c->vol_spacing[gb * 3 + 0];
    double ox = c->vol_origin[gb * 3 + 2], oy = c->vol_origin[gb * 3 + 1], oz = c->vol_origin[gb * 3 + 0];
    const float *sino = c->sino + (long)b * c->n_proj * c->H * c->W;
    long total = (long)c->n_proj * c->H * c->W;
    const float *P = c->P + (long)gb * c->n_proj * 12;
    double mult = c->mult[gb];
    for (int j = 0; j < c->Y; ++j)
        for (int i = 0; i < c->X; ++i) {
            double x = i * sx + ox, y = j * sy + oy, z = k * sz + oz;
            double acc = 0.0;
            for (int n = 0; n < c->n_proj; ++n) {
                const float *m = P + 12 * n;
                double un = m[0] * x + m[1] * y + m[2] * z + m[3];
                double vn = m[4] * x + m[5] * y + m[6] * z + m[7];
                double wn = m[8] * x + m[9] * y + m[10] * z + m[11];
                double rw = 1.0 / wn;
                double u = un * rw, v = vn * rw;
                double val = c->hw ? bilinear_border(sino + (long)n * c->H * c->W, c->W, c->H, u, v)
                                   : bilinear_quirk(sino, c->W, c->H, total, n, u, v);
                acc += val * rw * rw;
            }
            c->vol[(((long)b * c->Z + k) * c->Y + j) * c->X + i] = acc * mult;
        }
}

/* ConeBackprojection3D: cone_backprojector_3D_CudaKernel.cu.cc:84-118
 * (hardware_interp=0) and cone_backprojector_3D_CudaKernel_hardware_interp.cu.cc:55-87 (=1). */
void oracle_cone_backprojection3d(const float *sino, double *vol, int hardware_interp, int batch, int n_proj, int H,
                                  int W, int Z, int Y, int X, const float *vol_origin, const float *vol_spacing,
                                  const float *P, const float *mult, int geom_batch, int nthreads)
{
    bp3d_ctx c = {sino, vol, batch, n_proj, H, W, Z, Y, X, geom_batch, hardware_interp, vol_origin, vol_spacing,
                  P, mult};
    parallel_for((long)batch * Z, nthreads, bp3d_item, &c);
}

/* Runs fn over items [first, first + n) of another work function. */
typedef struct {
    work_fn fn;
    void *ctx;
    long first;
} offset_ctx;

static void offset_item(void *v, long it)
{
    offset_ctx *o = (offset_ctx *)v;
    o->fn(o->ctx, o->first + it);
}

/* Same as oracle_cone_backprojection3d but only for the z-slices
 * [z_begin, z_end) of batch element 0 (bounded CPU-baseline samples). */
void oracle_cone_backprojection3d_slab(const float *sino, double *vol, int hardware_interp, int n_proj, int H, int W,
                                       int Z, int Y, int X, int z_begin, int z_end, const float *vol_origin,
                                       const float *vol_spacing, const float *P, const float *mult, int nthreads)
{
    bp3d_ctx c = {sino, vol, 1, n_proj, H, W, Z, Y, X, 1, hardware_interp, vol_origin, vol_spacing, P, mult};
    offset_ctx o = {bp3d_item, &c, z_begin};
    parallel_for((long)(z_end - z_begin), nthreads, offset_item, &o);
}

/* Same as oracle_cone_projection3d but only for views [p_begin, p_end) of
 * batch element 0; sino holds all n_proj views, only the subset is written. */
void oracle_cone_projection3d_views(const float *vol, double *sino, int hardware_interp, int Z, int Y, int X,
                                    int n_proj, int H, int W, int p_begin, int p_end, const float *vol_origin,
                                    const float *vol_spacing, const float *P, const float *step, int nthreads,
                                    long long *counts)
{
    double *invAR = (double *)malloc(sizeof(double) * 9 * (size_t)n_proj);
    double *src = (double *)malloc(sizeof(double) * 3 * (size_t)n_proj);
    oracle_cone_decompose(P, vol_spacing, vol_origin, n_proj, invAR, src);
    fp3d_ctx c = {vol, sino, 1, Z, Y, X, n_proj, H, W, 1, hardware_interp, vol_origin, vol_spacing, P, step, invAR,
                  src, counts};
    offset_ctx o = {fp3d_item, &c, p_begin};
    parallel_for((long)(p_end - p_begin), nthreads, offset_item, &o);
    free(invAR);
    free(src);
}

/* ------------------------------------------- matched (transpose) backprojection */

static void scatter_trilinear(double *vol, long X, long Y, long Z, double x, double y, double z, double val)
{
    double xf = floor(x), yf = floor(y), zf = floor(z);
    double fx = x - xf, fy = y - yf, fz = z - zf;
    long x0 = (long)xf, y0 = (long)yf, z0 = (long)zf;
    double wx[2] = {1.0 - fx, fx}, wy[2] = {1.0 - fy, fy}, wz[2] = {1.0 - fz, fz};
    for (int dz = 0; dz < 2; ++dz)
        for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx) {
                long xx = x0 + dx, yy = y0 + dy, zz = z0 + dz;
                if (xx < 0 || xx >= X || yy < 0 || yy >= Y || zz < 0 || zz >= Z) continue;
                vol[(zz * Y + yy) * X + xx] += val * wz[dz] * wy[dy] * wx[dx];
            }
}

/* Transpose of the software forward projector with the end correction always
 * applied (the linear form of cone_projector_3D_CudaKernel.cu.cc:135-179):
 * every sample scatters sino * (its trapezoid weight) * |ray (.) spacing|
 * into its 8 trilinear taps.  Single-threaded per batch element (test sizes). */
void oracle_cone_backprojection3d_matched(const float *sino, double *vol, int batch, int n_proj, int H, int W, int Z,
                                          int Y, int X, const float *vol_origin, const float *vol_spacing,
                                          const float *P, const float *step, int geom_batch)
{
    double *invAR = (double *)malloc(sizeof(double) * 9 * (size_t)geom_batch * n_proj);
    double *src = (double *)malloc(sizeof(double) * 3 * (size_t)geom_batch * n_proj);
    for (int g = 0; g < geom_batch; ++g)
        oracle_cone_decompose(P + (size_t)g * n_proj * 12, vol_spacing + 3 * g, vol_origin + 3 * g, n_proj,
                              invAR + (size_t)g * n_proj * 9, src + (size_t)g * n_proj * 3);
    long N[3] = {X, Y, Z};
    memset(vol, 0, sizeof(double) * (size_t)batch * Z * Y * X);
    for (int b = 0; b < batch; ++b) {
        int gb = geom_batch == 1 ? 0 : b;
        double sp[3] = {vol_spacing[gb * 3 + 2], vol_spacing[gb * 3 + 1], vol_spacing[gb * 3 + 0]};
        float h = step[gb];
        double *vb = vol + (size_t)b * Z * Y * X;
        for (int p = 0; p < n_proj; ++p) {
            const double *M = invAR + ((size_t)gb * n_proj + p) * 9;
            const double *S = src + ((size_t)gb * n_proj + p) * 3;
            for (int v = 0; v < H; ++v)
                for (int u = 0; u < W; ++u) {
                    double yv = sino[(((size_t)b * n_proj + p) * H + v) * W + u];
                    if (yv == 0.0) continue;
                    double r[3];
                    for (int k = 0; k < 3; ++k) r[k] = M[3 * k + 2] + v * M[3 * k + 1] + u * M[3 * k + 0];
                    double len = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
                    for (int k = 0; k < 3; ++k) r[k] /= len;
                    double min_a = 0.0, max_a = INFINITY;
                    for (int k = 0; k < 3; ++k)
                        if (r[k] != 0.0) {
                            double rc = 1.0 / r[k], a0 = (0.0 - S[k]) * rc, a1 = ((double)N[k] - S[k]) * rc;
                            if (k == 0) {
                                min_a = fmin(a0, a1);
                                max_a = fmax(a0, a1);
                            } else {
                                min_a = fmax(min_a, fmin(a0, a1));
                                max_a = fmin(max_a, fmax(a0, a1));
                            }
                        }
                    float a = (float)min_a;
                    a += h * 0.5f;
                    float amax = (float)max_a;
                    if (!(a < amax)) continue;
                    double scale = yv * sqrt((r[0] * sp[0]) * (r[0] * sp[0]) + (r[1] * sp[1]) * (r[1] * sp[1]) +
                                             (r[2] * sp[2]) * (r[2] * sp[2]));
                    double held = 0.5 * (double)h, pt[3];
                    for (int k = 0; k < 3; ++k) pt[k] = S[k] + (double)a * r[k];
                    a += h;
                    while (a < amax) {
                        scatter_trilinear(vb, X, Y, Z, pt[0], pt[1], pt[2], held * scale);
                        for (int k = 0; k < 3; ++k) pt[k] = S[k] + (double)a * r[k];
                        held = (double)h;
                        a += h;
                    }
                    a -= h;
                    double last = (double)amax - (double)a;
                    scatter_trilinear(vb, X, Y, Z, pt[0], pt[1], pt[2], (held - 0.5 * (double)h + 0.5 * last) * scale);
                    for (int k = 0; k < 3; ++k) pt[k] = S[k] + (double)amax * r[k];
                    scatter_trilinear(vb, X, Y, Z, pt[0], pt[1], pt[2], 0.5 * last * scale);
                }
        }
    }
    free(invAR);
    free(src);
}
