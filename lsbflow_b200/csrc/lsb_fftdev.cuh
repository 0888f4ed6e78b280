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

// cos and sin of 2 pi j / 48, j = 0..47, correctly rounded (computed from the series
// definitions in exact decimal arithmetic)
static __device__ constexpr double kC48[48] = {0x1.0000000000000p+0, 0x1.fb9ea92ec689bp-1, 0x1.ee8dd4748bf15p-1, 0x1.d906bcf328d46p-1, 0x1.bb67ae8584caap-1, 0x1.963268b572492p-1, 0x1.6a09e667f3bcdp-1, 0x1.37af93f9513eap-1, 0x1.0000000000000p-1, 0x1.87de2a6aea963p-2, 0x1.0907dc1930690p-2, 0x1.0b5150f6da2d1p-3, 0x0.0p+0, -0x1.0b5150f6da2d1p-3, -0x1.0907dc1930690p-2, -0x1.87de2a6aea963p-2, -0x1.0000000000000p-1, -0x1.37af93f9513eap-1, -0x1.6a09e667f3bcdp-1, -0x1.963268b572492p-1, -0x1.bb67ae8584caap-1, -0x1.d906bcf328d46p-1, -0x1.ee8dd4748bf15p-1, -0x1.fb9ea92ec689bp-1, -0x1.0000000000000p+0, -0x1.fb9ea92ec689bp-1, -0x1.ee8dd4748bf15p-1, -0x1.d906bcf328d46p-1, -0x1.bb67ae8584caap-1, -0x1.963268b572492p-1, -0x1.6a09e667f3bcdp-1, -0x1.37af93f9513eap-1, -0x1.0000000000000p-1, -0x1.87de2a6aea963p-2, -0x1.0907dc1930690p-2, -0x1.0b5150f6da2d1p-3, 0x0.0p+0, 0x1.0b5150f6da2d1p-3, 0x1.0907dc1930690p-2, 0x1.87de2a6aea963p-2, 0x1.0000000000000p-1, 0x1.37af93f9513eap-1, 0x1.6a09e667f3bcdp-1, 0x1.963268b572492p-1, 0x1.bb67ae8584caap-1, 0x1.d906bcf328d46p-1, 0x1.ee8dd4748bf15p-1, 0x1.fb9ea92ec689bp-1};
static __device__ constexpr double kS48[48] = {0x0.0p+0, 0x1.0b5150f6da2d1p-3, 0x1.0907dc1930690p-2, 0x1.87de2a6aea963p-2, 0x1.0000000000000p-1, 0x1.37af93f9513eap-1, 0x1.6a09e667f3bcdp-1, 0x1.963268b572492p-1, 0x1.bb67ae8584caap-1, 0x1.d906bcf328d46p-1, 0x1.ee8dd4748bf15p-1, 0x1.fb9ea92ec689bp-1, 0x1.0000000000000p+0, 0x1.fb9ea92ec689bp-1, 0x1.ee8dd4748bf15p-1, 0x1.d906bcf328d46p-1, 0x1.bb67ae8584caap-1, 0x1.963268b572492p-1, 0x1.6a09e667f3bcdp-1, 0x1.37af93f9513eap-1, 0x1.0000000000000p-1, 0x1.87de2a6aea963p-2, 0x1.0907dc1930690p-2, 0x1.0b5150f6da2d1p-3, 0x0.0p+0, -0x1.0b5150f6da2d1p-3, -0x1.0907dc1930690p-2, -0x1.87de2a6aea963p-2, -0x1.0000000000000p-1, -0x1.37af93f9513eap-1, -0x1.6a09e667f3bcdp-1, -0x1.963268b572492p-1, -0x1.bb67ae8584caap-1, -0x1.d906bcf328d46p-1, -0x1.ee8dd4748bf15p-1, -0x1.fb9ea92ec689bp-1, -0x1.0000000000000p+0, -0x1.fb9ea92ec689bp-1, -0x1.ee8dd4748bf15p-1, -0x1.d906bcf328d46p-1, -0x1.bb67ae8584caap-1, -0x1.963268b572492p-1, -0x1.6a09e667f3bcdp-1, -0x1.37af93f9513eap-1, -0x1.0000000000000p-1, -0x1.87de2a6aea963p-2, -0x1.0907dc1930690p-2, -0x1.0b5150f6da2d1p-3};

// e^{SIGN 2 pi i m / R} for R dividing 48
template <int R, int SIGN>
__device__ __forceinline__ double2 omega(int m) {
    const int j = (m * (48 / R)) % 48;
    return make_double2(kC48[j], SIGN < 0 ? -kS48[j] : kS48[j]);
}

// R-point DFT in registers, R in {1,2,3,4,6,8,12,16}: 2, 3, 4 directly, the others as
// R = A*B (A in {4,3}) by one four-step split with constant twiddles.
template <int R, int SIGN>
__device__ __forceinline__ void dft_reg(double2 (&v)[R]) {
    if constexpr (R == 1) {
    } else if constexpr (R == 2) {
        const double2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (R == 3) {
        const double h = kS48[16];  // sin(2 pi / 3)
        const double2 t1 = cadd(v[1], v[2]);
        const double2 t2 = make_double2(v[0].x - 0.5 * t1.x, v[0].y - 0.5 * t1.y);
        const double2 d = csub(v[1], v[2]);
        // SIGN < 0: X1 = t2 - i h d, X2 = t2 + i h d
        const double2 ihd = make_double2(-h * d.y, h * d.x);
        v[0] = cadd(v[0], t1);
        if (SIGN < 0) {
            v[1] = csub(t2, ihd);
            v[2] = cadd(t2, ihd);
        } else {
            v[1] = cadd(t2, ihd);
            v[2] = csub(t2, ihd);
        }
    } else if constexpr (R == 4) {
        const double2 a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
        const double2 c = cadd(v[1], v[3]), d = csub(v[1], v[3]);
        v[0] = cadd(a, c);
        v[2] = csub(a, c);
        if (SIGN < 0) {
            v[1] = make_double2(b.x + d.y, b.y - d.x);
            v[3] = make_double2(b.x - d.y, b.y + d.x);
        } else {
            v[1] = make_double2(b.x - d.y, b.y + d.x);
            v[3] = make_double2(b.x + d.y, b.y - d.x);
        }
    } else {
        constexpr int A = (R % 4 == 0) ? 4 : 3;
        constexpr int B = R / A;
        double2 w[B][A];
#pragma unroll
        for (int b = 0; b < B; ++b) {
            double2 u[A];
#pragma unroll
            for (int a = 0; a < A; ++a) u[a] = v[B * a + b];
            dft_reg<A, SIGN>(u);
#pragma unroll
            for (int ka = 0; ka < A; ++ka) w[b][ka] = (b > 0 && ka > 0) ? cmul(u[ka], omega<R, SIGN>(b * ka)) : u[ka];
        }
#pragma unroll
        for (int ka = 0; ka < A; ++ka) {
            double2 u[B];
#pragma unroll
            for (int b = 0; b < B; ++b) u[b] = w[b][ka];
            dft_reg<B, SIGN>(u);
#pragma unroll
            for (int kb = 0; kb < B; ++kb) v[ka + A * kb] = u[kb];
        }
    }
}


}  // namespace lsb
