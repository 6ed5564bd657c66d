// Declarations only: the reference kernel files include Eigen and TensorFlow
// headers but instantiate nothing from them (helper_eigen.h holds two
// uninstantiated templates).  Test infrastructure for building the reference.
#pragma once
namespace Eigen {
const int Dynamic = -1;
template <typename S, int R, int C, int O = 0, int MR = R, int MC = C> class Matrix;
template <typename M, int O = 0, typename St = void> class Map;
template <typename S, int N, int O = 0, typename I = long> class Tensor;
template <typename T, int O = 0> class TensorMap;
}  // namespace Eigen
