// Register-resident small DFTs with compile-time sizes, for the two-level
// FFT of pass 2 (a length L = R1 * R2 transform done as R2 DFTs of size R1
// per column held in registers, one shared-memory exchange, then R1 DFTs of
// size R2).  All index arithmetic is compile-time; the only runtime inputs
// are the data and the twiddle table.
#pragma once

#include "fft_fast.cuh"

namespace tdda {

constexpr int inv_mod(int a, int m) {
    for (int x = 1; x < m; ++x)
        if ((a * x) % m == 1) return x;
    return 0;
}

// Prime-factor (Good-Thomas) DFT of N = N1 * N2 with gcd(N1, N2) = 1: inputs
// re-indexed n = (N2 n1 + N1 n2) mod N, N1-point DFTs over n1, N2-point DFTs
// over n2, outputs at k = (N2 u k1 + N1 v k2) mod N (u = N2^-1 mod N1,
// v = N1^-1 mod N2).  No twiddle factors.
template <int N1, int N2, int SIGN, typename C> __device__ __forceinline__ void dft_pfa(C (&a)[N1 * N2]) {
    constexpr int N = N1 * N2;
    constexpr int u = inv_mod(N2 % N1, N1), v = inv_mod(N1 % N2, N2);
    C m[N2][N1];
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) {
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1) m[n2][n1] = a[(N2 * n1 + N1 * n2) % N];
        dftR<N1, SIGN>(m[n2]);
    }
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) {
        C col[N2];
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) col[n2] = m[n2][k1];
        dftR<N2, SIGN>(col);
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) a[(N2 * u * k1 + N1 * v * k2) % N] = col[k2];
    }
}

// N-point DFT in natural order, N in {2, 3, 4, 6, 8, 12, 16}
template <int N, int SIGN, typename C> __device__ __forceinline__ void dft_reg(C (&a)[N]) {
    if constexpr (N == 16) dft16<SIGN>(a);
    else if constexpr (N == 12) dft_pfa<4, 3, SIGN>(a);
    else if constexpr (N == 6) dft_pfa<2, 3, SIGN>(a);
    else dftR<N, SIGN>(a);
}

// DFT of size 2H whose inputs n >= H are zero: with b[n] = a[n] W_2H^n,
// X[2k] = DFT_H(a)[k] and X[2k + 1] = DFT_H(b)[k].  On return a holds the
// even outputs and b the odd ones.  twN: table stride of W_2H (Lmax / 2H).
template <int H, int SIGN, typename C>
__device__ __forceinline__ void dft_half_in(C (&a)[H], C (&b)[H], const C *__restrict__ tw, int twN) {
    b[0] = a[0];
#pragma unroll
    for (int n = 1; n < H; ++n) b[n] = a[n] * twiddle<SIGN>(tw, n * twN);
    dft_reg<H, SIGN>(a);
    dft_reg<H, SIGN>(b);
}

// First H outputs of a DFT of size 2H: X[k] = E[k] + W_2H^k O[k] with E, O the
// DFTs of the even and odd inputs (held in e and o, overwritten; the result is
// left in e).
template <int H, int SIGN, typename C>
__device__ __forceinline__ void dft_half_out(C (&e)[H], C (&o)[H], const C *__restrict__ tw, int twN) {
    dft_reg<H, SIGN>(e);
    dft_reg<H, SIGN>(o);
    e[0] = e[0] + o[0];
#pragma unroll
    for (int k = 1; k < H; ++k) e[k] = e[k] + o[k] * twiddle<SIGN>(tw, k * twN);
}

}  // namespace tdda
