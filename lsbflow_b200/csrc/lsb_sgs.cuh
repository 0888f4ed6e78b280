// Pointwise pieces of the SGS models shared by the SGS kernels and the fused row pass of the
// dynamic model (src/sgsterm.f90:130-190): the symmetric-tensor index, products rounded one
// at a time, and |S| in the reference's summation order.
#pragma once

#include <cuda_runtime.h>

namespace lsb {

__host__ __device__ __forceinline__ int sym6(int l, int m) {
    // (1,1)=0 (1,2)=1 (1,3)=2 (2,2)=3 (2,3)=4 (3,3)=5
    const int a = l < m ? l : m, b = l < m ? m : l;
    return a == 0 ? b : (a == 1 ? 2 + b : 5);
}

// products rounded one at a time, so that no multiply-add contraction changes them
__device__ __forceinline__ double mul_rn(double x, double y) { return __dmul_rn(x, y); }
__device__ __forceinline__ float mul_rn(float x, float y) { return __fmul_rn(x, y); }

// |S| = sqrt(2 S_ij S_ij) from the six independent components
template <class T>
__device__ __forceinline__ T snorm6(const T (&s6)[6]) {
    T sn = (T)0;
    for (int m = 0; m < 3; ++m)
        for (int l = 0; l < 3; ++l) {
            const T v = s6[sym6(l, m)];
            sn = sn + (T)2 * v * v;
        }
    return sqrt(sn);
}

// the first pass of the dynamic model at one point: S_lm (l <= m) from the gradients
// g_lm = du_l/dx_m and g_ml, and L'_lm = delta^2 |S| S_lm
template <class T>
__device__ __forceinline__ T dyn_sij(T g_lm, T g_ml) { return (T)0.5 * (g_lm + g_ml); }
template <class T>
__device__ __forceinline__ T dyn_lij(T dl, T sn, T s) { return mul_rn(mul_rn(mul_rn(dl, dl), sn), s); }

}  // namespace lsb
