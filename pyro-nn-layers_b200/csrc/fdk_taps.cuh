// fdk_taps.cuh -- the spatial ramp-filter kernels of the FDK / FBP filter,
// shared by its CUDA-core and tensor-core implementations.
//
// tau * h[m] for the Ram-Lak and Shepp-Logan kernels of Kak & Slaney (1988,
// ch. 3), tau the detector column pitch: Ram-Lak h[0] = 1 / (4 tau^2),
// h[m] = -1 / (pi^2 m^2 tau^2) for odd m and 0 for even m != 0; Shepp-Logan
// h[m] = -2 / (pi^2 tau^2 (4 m^2 - 1)).  Evaluated in FP64, rounded once.
#pragma once

namespace pyronn {

__device__ __forceinline__ float fdk_tap(int kind, int m_int, float du)
{
    const double pi2 = 9.869604401089358;  // pi^2
    const double m = (double)m_int;
    double t;
    if (kind == 0)
        t = (m_int == 0) ? 0.25 / du : ((m_int & 1) ? -1.0 / (pi2 * m * m * du) : 0.0);
    else
        t = -2.0 / (pi2 * du * (4.0 * m * m - 1.0));
    return (float)t;
}

}  // namespace pyronn
