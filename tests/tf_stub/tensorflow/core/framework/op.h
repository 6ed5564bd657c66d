// Compile-check stub (see tests/tf_stub/README.txt): REGISTER_OP and its builder.
#pragma once
#include <string>

#include "tensorflow/core/framework/shape_inference.h"

namespace tensorflow {
namespace register_op {

class OpDefBuilderWrapper {
  public:
    explicit OpDefBuilderWrapper(const char *name);
    OpDefBuilderWrapper &Input(std::string spec);
    OpDefBuilderWrapper &Output(std::string spec);
    OpDefBuilderWrapper &Attr(std::string spec);
    OpDefBuilderWrapper &Doc(std::string text);
    OpDefBuilderWrapper &SetShapeFn(Status (*fn)(shape_inference::InferenceContext *));
};

}  // namespace register_op
}  // namespace tensorflow

#define TF_STUB_CONCAT_(a, b) a##b
#define TF_STUB_CONCAT(a, b) TF_STUB_CONCAT_(a, b)
#define REGISTER_OP(name)                                                                               \
    static ::tensorflow::register_op::OpDefBuilderWrapper TF_STUB_CONCAT(register_op_, __COUNTER__) = \
        ::tensorflow::register_op::OpDefBuilderWrapper(name)
