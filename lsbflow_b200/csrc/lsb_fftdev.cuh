// Device helpers shared by the FFT kernels: complex arithmetic, exactly rounded twiddle
// constants for the small register DFTs, and the register DFT of 1..16 points.
#pragma once
#include <cuda_runtime.h>

namespace lsb {

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }

// scalar type and constructor of a complex vector type (double2 / float2)
template <class V> struct CT;
template <> struct CT<double2> {
    using S = double;
    __device__ static double2 make(double x, double y) { return make_double2(x, y); }
};
template <> struct CT<float2> {
    using S = float;
    __device__ static float2 make(float x, float y) { return make_float2(x, y); }
};

// cos and sin of 2 pi j / 48, j = 0..47, correctly rounded (computed from the series
// definitions in exact decimal arithmetic)
static __device__ constexpr double kC48[48] = {0x1.0000000000000p+0, 0x1.fb9ea92ec689bp-1, 0x1.ee8dd4748bf15p-1, 0x1.d906bcf328d46p-1, 0x1.bb67ae8584caap-1, 0x1.963268b572492p-1, 0x1.6a09e667f3bcdp-1, 0x1.37af93f9513eap-1, 0x1.0000000000000p-1, 0x1.87de2a6aea963p-2, 0x1.0907dc1930690p-2, 0x1.0b5150f6da2d1p-3, 0x0.0p+0, -0x1.0b5150f6da2d1p-3, -0x1.0907dc1930690p-2, -0x1.87de2a6aea963p-2, -0x1.0000000000000p-1, -0x1.37af93f9513eap-1, -0x1.6a09e667f3bcdp-1, -0x1.963268b572492p-1, -0x1.bb67ae8584caap-1, -0x1.d906bcf328d46p-1, -0x1.ee8dd4748bf15p-1, -0x1.fb9ea92ec689bp-1, -0x1.0000000000000p+0, -0x1.fb9ea92ec689bp-1, -0x1.ee8dd4748bf15p-1, -0x1.d906bcf328d46p-1, -0x1.bb67ae8584caap-1, -0x1.963268b572492p-1, -0x1.6a09e667f3bcdp-1, -0x1.37af93f9513eap-1, -0x1.0000000000000p-1, -0x1.87de2a6aea963p-2, -0x1.0907dc1930690p-2, -0x1.0b5150f6da2d1p-3, 0x0.0p+0, 0x1.0b5150f6da2d1p-3, 0x1.0907dc1930690p-2, 0x1.87de2a6aea963p-2, 0x1.0000000000000p-1, 0x1.37af93f9513eap-1, 0x1.6a09e667f3bcdp-1, 0x1.963268b572492p-1, 0x1.bb67ae8584caap-1, 0x1.d906bcf328d46p-1, 0x1.ee8dd4748bf15p-1, 0x1.fb9ea92ec689bp-1};
static __device__ constexpr double kS48[48] = {0x0.0p+0, 0x1.0b5150f6da2d1p-3, 0x1.0907dc1930690p-2, 0x1.87de2a6aea963p-2, 0x1.0000000000000p-1, 0x1.37af93f9513eap-1, 0x1.6a09e667f3bcdp-1, 0x1.963268b572492p-1, 0x1.bb67ae8584caap-1, 0x1.d906bcf328d46p-1, 0x1.ee8dd4748bf15p-1, 0x1.fb9ea92ec689bp-1, 0x1.0000000000000p+0, 0x1.fb9ea92ec689bp-1, 0x1.ee8dd4748bf15p-1, 0x1.d906bcf328d46p-1, 0x1.bb67ae8584caap-1, 0x1.963268b572492p-1, 0x1.6a09e667f3bcdp-1, 0x1.37af93f9513eap-1, 0x1.0000000000000p-1, 0x1.87de2a6aea963p-2, 0x1.0907dc1930690p-2, 0x1.0b5150f6da2d1p-3, 0x0.0p+0, -0x1.0b5150f6da2d1p-3, -0x1.0907dc1930690p-2, -0x1.87de2a6aea963p-2, -0x1.0000000000000p-1, -0x1.37af93f9513eap-1, -0x1.6a09e667f3bcdp-1, -0x1.963268b572492p-1, -0x1.bb67ae8584caap-1, -0x1.d906bcf328d46p-1, -0x1.ee8dd4748bf15p-1, -0x1.fb9ea92ec689bp-1, -0x1.0000000000000p+0, -0x1.fb9ea92ec689bp-1, -0x1.ee8dd4748bf15p-1, -0x1.d906bcf328d46p-1, -0x1.bb67ae8584caap-1, -0x1.963268b572492p-1, -0x1.6a09e667f3bcdp-1, -0x1.37af93f9513eap-1, -0x1.0000000000000p-1, -0x1.87de2a6aea963p-2, -0x1.0907dc1930690p-2, -0x1.0b5150f6da2d1p-3};

// e^{SIGN 2 pi i m / R} for R dividing 48
template <int R, int SIGN, class V = double2>
__device__ __forceinline__ V omega(int m) {
    using S = typename CT<V>::S;
    const int j = (m * (48 / R)) % 48;
    return CT<V>::make((S)kC48[j], (S)(SIGN < 0 ? -kS48[j] : kS48[j]));
}

// R-point DFT in registers, R in {1,2,3,4,6,8,12,16}: 2, 3, 4 directly, the others as
// R = A*B (A in {4,3}) by one four-step split with constant twiddles.
template <int R, int SIGN, class V>
__device__ __forceinline__ void dft_reg(V (&v)[R]) {
    using S = typename CT<V>::S;
    if constexpr (R == 1) {
    } else if constexpr (R == 2) {
        const V a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (R == 3) {
        const S h = (S)kS48[16];  // sin(2 pi / 3)
        const V t1 = cadd(v[1], v[2]);
        const V t2 = CT<V>::make(v[0].x - (S)0.5 * t1.x, v[0].y - (S)0.5 * t1.y);
        const V d = csub(v[1], v[2]);
        // SIGN < 0: X1 = t2 - i h d, X2 = t2 + i h d
        const V ihd = CT<V>::make(-h * d.y, h * d.x);
        v[0] = cadd(v[0], t1);
        if (SIGN < 0) {
            v[1] = csub(t2, ihd);
            v[2] = cadd(t2, ihd);
        } else {
            v[1] = cadd(t2, ihd);
            v[2] = csub(t2, ihd);
        }
    } else if constexpr (R == 4) {
        const V a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
        const V c = cadd(v[1], v[3]), d = csub(v[1], v[3]);
        v[0] = cadd(a, c);
        v[2] = csub(a, c);
        if (SIGN < 0) {
            v[1] = CT<V>::make(b.x + d.y, b.y - d.x);
            v[3] = CT<V>::make(b.x - d.y, b.y + d.x);
        } else {
            v[1] = CT<V>::make(b.x - d.y, b.y + d.x);
            v[3] = CT<V>::make(b.x + d.y, b.y - d.x);
        }
    } else {
        constexpr int A = (R % 4 == 0) ? 4 : 3;
        constexpr int B = R / A;
        V w[B][A];
#pragma unroll
        for (int b = 0; b < B; ++b) {
            V u[A];
#pragma unroll
            for (int a = 0; a < A; ++a) u[a] = v[B * a + b];
            dft_reg<A, SIGN>(u);
#pragma unroll
            for (int ka = 0; ka < A; ++ka) w[b][ka] = (b > 0 && ka > 0) ? cmul(u[ka], omega<R, SIGN, V>(b * ka)) : u[ka];
        }
#pragma unroll
        for (int ka = 0; ka < A; ++ka) {
            V u[B];
#pragma unroll
            for (int b = 0; b < B; ++b) u[b] = w[b][ka];
            dft_reg<B, SIGN>(u);
#pragma unroll
            for (int kb = 0; kb < B; ++kb) v[ka + A * kb] = u[kb];
        }
    }
}


}  // namespace lsb
