// pyronn_tf_ops.cc -- TensorFlow custom-op shim over the C ABI of
// include/pyronn_b200.h.  Registers the six ops under the reference's names,
// inputs, attrs and shape functions, so graphs written against
// PYRO-NN-Layers load this library instead (tf.load_op_library).
//
// Build (needs TensorFlow headers; tests/test_tf_shim_cpu.py compile-checks this
// file against stub declarations of the TensorFlow names it uses), one command:
//   TF_CFLAGS=$(python -c 'import tensorflow as tf; print(" ".join(tf.sysconfig.get_compile_flags()))')
//   TF_LFLAGS=$(python -c 'import tensorflow as tf; print(" ".join(tf.sysconfig.get_link_flags()))')
//   g++ -std=c++17 -shared -fPIC pyronn_tf_ops.cc -o _pyronn_layers_ops.so $TF_CFLAGS $TF_LFLAGS
//       -I../../include -DGOOGLE_CUDA=1 -I/usr/local/cuda/include -L../pyronn_layers -lpyronn_b200
//
// Differences from the reference op kernels, all invisible to graph code:
//   * the shape inputs are HostMemory, so Compute needs no blocking
//     device->host copy (the reference cudaMemcpy's them, e.g.
//     cc/ops/cone_projector_3D_OPKernel.cc:219-223);
//   * one call per op handles the whole batch on TF's compute stream (the
//     reference loops over the batch and launches on the legacy default stream);
//   * the cone workspace comes from allocate_temp (the reference cudaMalloc's
//     outside TF's allocator, README.rst:127-130);
//   * CUDA failures become op errors instead of exit().
#define EIGEN_USE_GPU
#include "tensorflow/core/framework/op.h"
#include "tensorflow/core/framework/op_kernel.h"
#include "tensorflow/core/framework/shape_inference.h"

#include "pyronn_b200.h"

using namespace tensorflow;  // NOLINT(build/namespaces)
using shape_inference::InferenceContext;
using shape_inference::ShapeHandle;

namespace {

// output = [batch] ++ value of the shape tensor (input 1), as the reference's
// shape functions (e.g. cc/ops/cone_projector_3D_OPKernel.cc:44-54)
Status BatchPlusShapeTensor(InferenceContext *c)
{
    ShapeHandle batch, dims, out;
    TF_RETURN_IF_ERROR(c->MakeShapeFromShapeTensor(1, &dims));
    TF_RETURN_IF_ERROR(c->Subshape(c->input(0), 0, 1, &batch));
    TF_RETURN_IF_ERROR(c->Concatenate(batch, dims, &out));
    c->set_output(0, out);
    return OkStatus();
}

// rows of a geometry tensor: 1 (shared) or batch (one per batch element)
int GeomRows(const Tensor &t, int batch, int64_t row_elems)
{
    return t.NumElements() == row_elems ? 1 : batch;
}

Status CheckRows(const char *what, const Tensor &t, int batch, int64_t row_elems)
{
    if (t.NumElements() == row_elems || t.NumElements() == row_elems * batch) return OkStatus();
    return errors::InvalidArgument(what, ": expected ", row_elems, " values per batch element, got ",
                                   t.NumElements());
}

Status FromStatus(int st, const char *op)
{
    if (st == PYRONN_SUCCESS) return OkStatus();
    return errors::Internal(op, ": ", pyronn_status_string(st), ": ", pyronn_last_error());
}

cudaStream_t StreamOf(OpKernelContext *ctx)
{
    return ctx->eigen_device<Eigen::GpuDevice>().stream();
}

std::vector<int> ShapeValues(const Tensor &t)
{
    auto v = t.flat<int32>();
    return std::vector<int>(v.data(), v.data() + v.size());
}

}  // namespace

REGISTER_OP("ParallelProjection2D")
    .Input("volume: float")
    .Input("projection_shape: int32")
    .Input("volume_origin : float")
    .Input("detector_origin : float")
    .Input("volume_spacing : float")
    .Input("detector_spacing : float")
    .Input("ray_vectors : float")
    .Output("output: float")
    .SetShapeFn(BatchPlusShapeTensor)
    .Doc("output = A x (2D parallel beam)");

REGISTER_OP("ParallelBackprojection2D")
    .Input("sinogram: float")
    .Input("volume_shape: int32")
    .Input("volume_origin : float")
    .Input("detector_origin : float")
    .Input("volume_spacing : float")
    .Input("detector_spacing : float")
    .Input("ray_vectors : float")
    .Output("output: float")
    .SetShapeFn(BatchPlusShapeTensor)
    .Doc("output = A^T p (2D parallel beam)");

REGISTER_OP("FanProjection2D")
    .Input("volume: float")
    .Input("projection_shape: int32")
    .Input("volume_origin : float")
    .Input("detector_origin : float")
    .Input("volume_spacing : float")
    .Input("detector_spacing : float")
    .Input("source_2_isocenter_distance : float")
    .Input("source_2_detector_distance : float")
    .Input("central_ray_vectors : float")
    .Output("output: float")
    .SetShapeFn(BatchPlusShapeTensor)
    .Doc("output = A_fan x (2D fan beam, flat detector)");

REGISTER_OP("FanBackprojection2D")
    .Input("sinogram: float")
    .Input("volume_shape: int32")
    .Input("volume_origin : float")
    .Input("detector_origin : float")
    .Input("volume_spacing : float")
    .Input("detector_spacing : float")
    .Input("source_2_isocenter_distance : float")
    .Input("source_2_detector_distance : float")
    .Input("central_ray_vectors : float")
    .Output("output: float")
    .SetShapeFn(BatchPlusShapeTensor)
    .Doc("output = A_fan^T p (distance-weighted fan-beam backprojection)");

REGISTER_OP("ConeProjection3D")
    .Input("volume: float")
    .Input("projection_shape: int32")
    .Input("volume_origin : float")
    .Input("volume_spacing : float")
    .Input("projection_matrices : float")
    .Input("step_size: float")
    .Input("projection_multiplier : float")
    .Attr("hardware_interp : bool = false")
    .Output("output: float")
    .SetShapeFn(BatchPlusShapeTensor)
    .Doc("output = A_cone x (3D cone beam, ray driven)");

REGISTER_OP("ConeBackprojection3D")
    .Input("sinogram: float")
    .Input("volume_shape: int32")
    .Input("volume_origin : float")
    .Input("volume_spacing : float")
    .Input("projection_matrices : float")
    .Input("step_size : float")
    .Input("projection_multiplier : float")
    .Attr("hardware_interp : bool = false")
    .Output("output: float")
    .SetShapeFn(BatchPlusShapeTensor)
    .Doc("output = A_cone^T p (3D cone beam, voxel driven)");

template <bool kForward, bool kFan>
class Op2D : public OpKernel {
  public:
    explicit Op2D(OpKernelConstruction *c) : OpKernel(c) {}

    void Compute(OpKernelContext *ctx) override
    {
        const Tensor &in = ctx->input(0);
        OP_REQUIRES(ctx, in.dims() == 3, errors::InvalidArgument("expected [batch, ., .] input"));
        const int batch = in.dim_size(0);
        const std::vector<int> shp = ShapeValues(ctx->input(1));
        OP_REQUIRES(ctx, shp.size() == 2, errors::InvalidArgument("shape input must have 2 values"));
        const int n_proj = kForward ? shp[0] : in.dim_size(1);
        const int det_w = kForward ? shp[1] : in.dim_size(2);
        const int vol_y = kForward ? in.dim_size(1) : shp[0];
        const int vol_x = kForward ? in.dim_size(2) : shp[1];
        const int rays_in = kFan ? 8 : 6;
        const Tensor &vo = ctx->input(2), &dor = ctx->input(3), &vs = ctx->input(4), &ds = ctx->input(5),
                     &rays = ctx->input(rays_in);
        OP_REQUIRES_OK(ctx, CheckRows("volume_origin", vo, batch, 2));
        OP_REQUIRES_OK(ctx, CheckRows("detector_origin", dor, batch, 1));
        OP_REQUIRES_OK(ctx, CheckRows("volume_spacing", vs, batch, 2));
        OP_REQUIRES_OK(ctx, CheckRows("detector_spacing", ds, batch, 1));
        OP_REQUIRES_OK(ctx, CheckRows("ray_vectors", rays, batch, 2LL * n_proj));
        const int g = GeomRows(rays, batch, 2LL * n_proj);
        OP_REQUIRES(ctx, GeomRows(vo, batch, 2) == g && GeomRows(dor, batch, 1) == g &&
                             GeomRows(vs, batch, 2) == g && GeomRows(ds, batch, 1) == g,
                    errors::InvalidArgument("geometry tensors must be all shared or all batched"));
        Tensor *out = nullptr;
        const TensorShape os = kForward ? TensorShape({batch, n_proj, det_w}) : TensorShape({batch, vol_y, vol_x});
        OP_REQUIRES_OK(ctx, ctx->allocate_output(0, os, &out));
        // forward: the transposed slice copy (see pyronn_projection2d_workspace_size)
        Tensor ws;
        const size_t ws_bytes = kForward ? pyronn_projection2d_workspace_size(batch, vol_y, vol_x, PYRONN_FLOAT32) : 0;
        if (ws_bytes)
            OP_REQUIRES_OK(ctx, ctx->allocate_temp(DT_UINT8, TensorShape({(int64_t)ws_bytes}), &ws));
        void *ws_ptr = ws_bytes ? (void *)ws.flat<uint8>().data() : nullptr;
        const float *p_vo = vo.flat<float>().data(), *p_do = dor.flat<float>().data();
        const float *p_vs = vs.flat<float>().data(), *p_ds = ds.flat<float>().data();
        const float *p_r = rays.flat<float>().data();
        int st;
        if (kFan) {
            const float *sid = ctx->input(6).flat<float>().data(), *sdd = ctx->input(7).flat<float>().data();
            st = kForward ? pyronn_fan_projection2d(in.flat<float>().data(), out->flat<float>().data(),
                                                    PYRONN_FLOAT32, PYRONN_FLOAT32, batch, vol_y, vol_x, n_proj,
                                                    det_w, p_vo, p_do, p_vs, p_ds, sid, sdd, p_r, g, ws_ptr, ws_bytes,
                                                    StreamOf(ctx))
                          : pyronn_fan_backprojection2d(in.flat<float>().data(), out->flat<float>().data(),
                                                        PYRONN_FLOAT32, PYRONN_FLOAT32, batch, n_proj, det_w, vol_y,
                                                        vol_x, p_vo, p_do, p_vs, p_ds, sid, sdd, p_r, g,
                                                        StreamOf(ctx));
        } else {
            st = kForward ? pyronn_parallel_projection2d(in.flat<float>().data(), out->flat<float>().data(),
                                                         PYRONN_FLOAT32, PYRONN_FLOAT32, batch, vol_y, vol_x, n_proj,
                                                         det_w, p_vo, p_do, p_vs, p_ds, p_r, g, ws_ptr, ws_bytes,
                                                         StreamOf(ctx))
                          : pyronn_parallel_backprojection2d(in.flat<float>().data(), out->flat<float>().data(),
                                                             PYRONN_FLOAT32, PYRONN_FLOAT32, batch, n_proj, det_w,
                                                             vol_y, vol_x, p_vo, p_do, p_vs, p_ds, p_r, g,
                                                             StreamOf(ctx));
        }
        OP_REQUIRES_OK(ctx, FromStatus(st, name().c_str()));
    }
};

template <bool kForward>
class OpCone : public OpKernel {
  public:
    explicit OpCone(OpKernelConstruction *c) : OpKernel(c)
    {
        OP_REQUIRES_OK(c, c->GetAttr("hardware_interp", &hardware_interp_));
    }

    void Compute(OpKernelContext *ctx) override
    {
        const Tensor &in = ctx->input(0);
        OP_REQUIRES(ctx, in.dims() == 4, errors::InvalidArgument("expected [batch, ., ., .] input"));
        const int batch = in.dim_size(0);
        const std::vector<int> shp = ShapeValues(ctx->input(1));
        OP_REQUIRES(ctx, shp.size() == 3, errors::InvalidArgument("shape input must have 3 values"));
        const int n_proj = kForward ? shp[0] : in.dim_size(1);
        const int det_h = kForward ? shp[1] : in.dim_size(2);
        const int det_w = kForward ? shp[2] : in.dim_size(3);
        const int vol_z = kForward ? in.dim_size(1) : shp[0];
        const int vol_y = kForward ? in.dim_size(2) : shp[1];
        const int vol_x = kForward ? in.dim_size(3) : shp[2];
        const Tensor &vo = ctx->input(2), &vs = ctx->input(3), &P = ctx->input(4), &step = ctx->input(5),
                     &mult = ctx->input(6);
        OP_REQUIRES_OK(ctx, CheckRows("volume_origin", vo, batch, 3));
        OP_REQUIRES_OK(ctx, CheckRows("volume_spacing", vs, batch, 3));
        OP_REQUIRES_OK(ctx, CheckRows("projection_matrices", P, batch, 12LL * n_proj));
        OP_REQUIRES_OK(ctx, CheckRows("step_size", step, batch, 1));
        OP_REQUIRES_OK(ctx, CheckRows("projection_multiplier", mult, batch, 1));
        const int g = GeomRows(P, batch, 12LL * n_proj);
        OP_REQUIRES(ctx, GeomRows(vo, batch, 3) == g && GeomRows(vs, batch, 3) == g &&
                             GeomRows(step, batch, 1) == g && GeomRows(mult, batch, 1) == g,
                    errors::InvalidArgument("geometry tensors must be all shared or all batched"));
        Tensor *out = nullptr;
        const TensorShape os = kForward ? TensorShape({batch, n_proj, det_h, det_w})
                                        : TensorShape({batch, vol_z, vol_y, vol_x});
        OP_REQUIRES_OK(ctx, ctx->allocate_output(0, os, &out));
        const int hw = hardware_interp_ ? 1 : 0;
        const size_t ws_bytes =
            kForward ? pyronn_cone_projection3d_workspace_size(batch, vol_z, vol_y, vol_x, n_proj, det_h, det_w,
                                                               PYRONN_FLOAT32, hw, g)
                     : pyronn_cone_backprojection3d_workspace_size(batch, n_proj, det_h, det_w, vol_z, vol_y, vol_x,
                                                                   PYRONN_FLOAT32, hw, g);
        OP_REQUIRES(ctx, ws_bytes > 0, errors::InvalidArgument(name(), ": invalid problem size"));
        Tensor ws;
        OP_REQUIRES_OK(ctx, ctx->allocate_temp(DT_UINT8, TensorShape({(int64_t)ws_bytes}), &ws));
        const int st =
            kForward ? pyronn_cone_projection3d(in.flat<float>().data(), out->flat<float>().data(), PYRONN_FLOAT32,
                                                PYRONN_FLOAT32, hw, batch, vol_z, vol_y, vol_x,
                                                n_proj, det_h, det_w, vo.flat<float>().data(), vs.flat<float>().data(),
                                                P.flat<float>().data(), step.flat<float>().data(),
                                                mult.flat<float>().data(), g, ws.flat<uint8>().data(), ws_bytes,
                                                StreamOf(ctx))
                     : pyronn_cone_backprojection3d(in.flat<float>().data(), out->flat<float>().data(),
                                                    PYRONN_FLOAT32, PYRONN_FLOAT32, hw, batch,
                                                    n_proj, det_h, det_w, vol_z, vol_y, vol_x,
                                                    vo.flat<float>().data(), vs.flat<float>().data(),
                                                    P.flat<float>().data(), step.flat<float>().data(),
                                                    mult.flat<float>().data(), g, ws.flat<uint8>().data(), ws_bytes,
                                                    StreamOf(ctx));
        OP_REQUIRES_OK(ctx, FromStatus(st, name().c_str()));
    }

  private:
    bool hardware_interp_ = false;
};

REGISTER_KERNEL_BUILDER(Name("ParallelProjection2D").Device(DEVICE_GPU).HostMemory("projection_shape"),
                        (Op2D<true, false>));
REGISTER_KERNEL_BUILDER(Name("ParallelBackprojection2D").Device(DEVICE_GPU).HostMemory("volume_shape"),
                        (Op2D<false, false>));
REGISTER_KERNEL_BUILDER(Name("FanProjection2D").Device(DEVICE_GPU).HostMemory("projection_shape"),
                        (Op2D<true, true>));
REGISTER_KERNEL_BUILDER(Name("FanBackprojection2D").Device(DEVICE_GPU).HostMemory("volume_shape"),
                        (Op2D<false, true>));
REGISTER_KERNEL_BUILDER(Name("ConeProjection3D").Device(DEVICE_GPU).HostMemory("projection_shape"),
                        OpCone<true>);
REGISTER_KERNEL_BUILDER(Name("ConeBackprojection3D").Device(DEVICE_GPU).HostMemory("volume_shape"),
                        OpCone<false>);
