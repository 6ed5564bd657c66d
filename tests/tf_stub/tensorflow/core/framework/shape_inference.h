// Compile-check stub (see tests/tf_stub/README.txt): shape_inference::InferenceContext.
#pragma once
#include "tensorflow/core/framework/types.h"

namespace tensorflow {
namespace shape_inference {

class ShapeHandle {
  public:
    ShapeHandle() = default;

  private:
    const void *ptr_ = nullptr;
};

class InferenceContext {
  public:
    ShapeHandle input(int64_t idx) const;
    void set_output(int idx, ShapeHandle shape);
    Status MakeShapeFromShapeTensor(int input_idx, ShapeHandle *out);
    Status Subshape(ShapeHandle s, int64_t start, int64_t end, ShapeHandle *out);
    Status Concatenate(ShapeHandle s1, ShapeHandle s2, ShapeHandle *out);
};

}  // namespace shape_inference
}  // namespace tensorflow
