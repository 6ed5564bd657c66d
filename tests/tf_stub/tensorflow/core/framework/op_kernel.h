// Compile-check stub (see tests/tf_stub/README.txt): OpKernel, its contexts,
// the kernel registration builder and OP_REQUIRES / OP_REQUIRES_OK.
#pragma once
#include <string>

#include "tensorflow/core/framework/types.h"

namespace Eigen {
struct GpuDevice {
    const cudaStream_t &stream() const;
};
}  // namespace Eigen

namespace tensorflow {

class OpKernelConstruction {
  public:
    template <class T>
    Status GetAttr(const char *attr_name, T *value) const;
    void CtxFailure(const Status &s);
};

class OpKernelContext {
  public:
    const Tensor &input(int index) const;
    Status allocate_output(int index, const TensorShape &shape, Tensor **tensor);
    Status allocate_temp(DataType type, const TensorShape &shape, Tensor *out_temp);
    template <typename EigenDeviceType>
    const EigenDeviceType &eigen_device() const;
    void CtxFailure(const Status &s);
};

class OpKernel {
  public:
    explicit OpKernel(OpKernelConstruction *context);
    virtual ~OpKernel();
    virtual void Compute(OpKernelContext *context) = 0;
    const std::string &name() const;
};

constexpr const char *DEVICE_GPU = "GPU";

class KernelDefBuilder {
  public:
    KernelDefBuilder &Device(const char *device_type);
    KernelDefBuilder &HostMemory(const char *arg_name);
};
KernelDefBuilder Name(const char *op);

namespace kernel_factory {
// TensorFlow's registration: a factory that runs `new <kernel class>(context)`
struct OpKernelRegistrar {
    OpKernelRegistrar(const KernelDefBuilder &builder, OpKernel *(*create)(OpKernelConstruction *));
};
}  // namespace kernel_factory

}  // namespace tensorflow

#define REGISTER_KERNEL_BUILDER(kernel_builder, ...)                                                    \
    static ::tensorflow::kernel_factory::OpKernelRegistrar TF_STUB_CONCAT(kernel_reg_, __COUNTER__)(       \
        kernel_builder,                                                                                 \
        [](::tensorflow::OpKernelConstruction *context) -> ::tensorflow::OpKernel * {                   \
            return new __VA_ARGS__(context);                                                            \
        })

#define OP_REQUIRES(CTX, EXP, STATUS) \
    do {                              \
        if (!(EXP)) {                 \
            (CTX)->CtxFailure(STATUS); \
            return;                   \
        }                             \
    } while (0)

#define OP_REQUIRES_OK(CTX, ...)                          \
    do {                                                  \
        const ::tensorflow::Status _s(__VA_ARGS__);       \
        if (!_s.ok()) {                                   \
            (CTX)->CtxFailure(_s);                        \
            return;                                       \
        }                                                 \
    } while (0)

#ifndef TF_STUB_CONCAT
#define TF_STUB_CONCAT_(a, b) a##b
#define TF_STUB_CONCAT(a, b) TF_STUB_CONCAT_(a, b)
#endif
