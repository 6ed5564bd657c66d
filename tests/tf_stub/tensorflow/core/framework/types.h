// Compile-check stub (see tests/tf_stub/README.txt): core value types, Status
// and the error / requirement macros with TensorFlow 2.x signatures.
#pragma once
#include <cuda_runtime_api.h>
#include <stdint.h>

#include <initializer_list>
#include <sstream>
#include <string>
#include <vector>

namespace tensorflow {

using int32 = int32_t;
using uint8 = uint8_t;

enum DataType { DT_FLOAT = 1, DT_INT32 = 3, DT_UINT8 = 4 };

class Status {
  public:
    Status() = default;
    Status(int code, std::string msg) : code_(code), msg_(std::move(msg)) {}
    bool ok() const { return code_ == 0; }
    const std::string &message() const { return msg_; }

  private:
    int code_ = 0;
    std::string msg_;
};

inline Status OkStatus() { return Status(); }

namespace errors {
template <typename... Args>
Status InvalidArgument(Args... args)
{
    std::ostringstream s;
    (s << ... << args);
    return Status(3, s.str());
}
template <typename... Args>
Status Internal(Args... args)
{
    std::ostringstream s;
    (s << ... << args);
    return Status(13, s.str());
}
}  // namespace errors

class TensorShape {
  public:
    TensorShape(std::initializer_list<int64_t> dims) : dims_(dims) {}
    int dims() const { return (int)dims_.size(); }
    int64_t dim_size(int d) const { return dims_[d]; }

  private:
    std::vector<int64_t> dims_;
};

// an Eigen::TensorMap-like flat view: data() and size()
template <typename T>
struct FlatView {
    T *ptr;
    int64_t n;
    T *data() const { return ptr; }
    int64_t size() const { return n; }
};

class Tensor {
  public:
    int dims() const;
    int64_t dim_size(int d) const;
    int64_t NumElements() const;
    template <typename T>
    FlatView<T> flat();
    template <typename T>
    FlatView<const T> flat() const;
};

}  // namespace tensorflow

#define TF_RETURN_IF_ERROR(expr)                        \
    do {                                                \
        const ::tensorflow::Status _tf_status = (expr); \
        if (!_tf_status.ok()) return _tf_status;        \
    } while (0)
