// Batched complex FFTs on data staged in shared memory.
//
// Mixed-radix Stockham autosort (radix 8/4/2/3): each stage, every work item
// reads R elements spaced L/R apart, twiddles them by w^(r*k), k = i mod P,
// runs an R-point DFT in registers and writes them P apart from
// j = (i - k) * R + k.  The stage is in place: all items of a thread are held
// in registers across one __syncthreads() between the reads and the writes.
//
// Element (batch b, position n) lives at buf[b * bstr + n * pstr].  Work items
// are numbered with the batch index fastest, so consecutive threads touch
// consecutive batches; callers pick an odd element pitch for the strided
// direction, which keeps every access pattern free of bank conflicts.
//
// Twiddles come from a table of Lmax entries exp(-2 pi i j / Lmax) in global
// memory (read through the L1/texture path); a length-L transform uses every
// (Lmax / L)-th entry.
#pragma once

#include "tdda_common.cuh"

namespace tdda {

template <int SIGN, typename C>
__device__ __forceinline__ C twiddle(const C *tw, int j) {
    C w = __ldg(tw + j);
    if (SIGN > 0) w.y = -w.y;
    return w;
}

template <int SIGN, typename C> __device__ __forceinline__ void dft2(C &a0, C &a1) {
    C t = a0 - a1;
    a0 = a0 + a1;
    a1 = t;
}

template <int SIGN, typename C> __device__ __forceinline__ void dft4(C &a0, C &a1, C &a2, C &a3) {
    C t0 = a0 + a2, t1 = a0 - a2, t2 = a1 + a3, t3 = mul_i(a1 - a3, SIGN);
    a0 = t0 + t2;
    a2 = t0 - t2;
    a1 = t1 + t3;
    a3 = t1 - t3;
}

template <int SIGN, typename C> __device__ __forceinline__ void dft3(C &a0, C &a1, C &a2) {
    using R = typename RealOf<C>::type;
    const R h = (R)0.86602540378443864676;  // sqrt(3)/2
    C t = a1 + a2, s = a1 - a2;
    C m = a0 - (R)0.5 * t;
    C q = mul_i(h * s, SIGN);
    a0 = a0 + t;
    a1 = m + q;
    a2 = m - q;
}

template <int SIGN, typename C> __device__ __forceinline__ void dft8(C (&a)[8]) {
    using R = typename RealOf<C>::type;
    const R s = (R)0.70710678118654752440;
    // even / odd 4-point transforms
    dft4<SIGN>(a[0], a[2], a[4], a[6]);
    dft4<SIGN>(a[1], a[3], a[5], a[7]);
    // twiddles w8^k, w8 = exp(SIGN * 2 pi i / 8)
    C o1 = a[3], o2 = a[5], o3 = a[7];
    // w8^1 = (1 + SIGN i) s
    C w1o;
    w1o.x = s * (o1.x - SIGN * o1.y);
    w1o.y = s * (o1.y + SIGN * o1.x);
    C w2o = mul_i(o2, SIGN);
    // w8^3 = (-1 + SIGN i) s
    C w3o;
    w3o.x = s * (-o3.x - SIGN * o3.y);
    w3o.y = s * (-o3.y + SIGN * o3.x);
    C e0 = a[0], e1 = a[2], e2 = a[4], e3 = a[6], o0 = a[1];
    a[0] = e0 + o0;
    a[4] = e0 - o0;
    a[1] = e1 + w1o;
    a[5] = e1 - w1o;
    a[2] = e2 + w2o;
    a[6] = e2 - w2o;
    a[3] = e3 + w3o;
    a[7] = e3 - w3o;
}

template <int R, int SIGN, typename C> __device__ __forceinline__ void dftR(C (&a)[R]) {
    if constexpr (R == 2) dft2<SIGN>(a[0], a[1]);
    else if constexpr (R == 3) dft3<SIGN>(a[0], a[1], a[2]);
    else if constexpr (R == 4) dft4<SIGN>(a[0], a[1], a[2], a[3]);
    else dft8<SIGN>(a);
}

template <int R, int SIGN, int MAXI, typename C>
__device__ __forceinline__ void fft_stage(C *buf, int L, int P, int nb, int pstr, int bstr,
                                          const C *tw, int twstep) {
    const int LR = L / R;
    const int W = nb * LR;
    const int tstep = (L / (P * R)) * twstep;
    C a[MAXI][R];
    int pos[MAXI];
#pragma unroll
    for (int it = 0; it < MAXI; ++it) {
        int w = threadIdx.x + it * blockDim.x;
        pos[it] = -1;
        if (w < W) {
            int b = w % nb, i = w / nb;
            int k = i % P;
            C *base = buf + (size_t)b * bstr;
#pragma unroll
            for (int r = 0; r < R; ++r) a[it][r] = base[(size_t)(i + r * LR) * pstr];
            if (k != 0) {
                int j1 = k * tstep;
#pragma unroll
                for (int r = 1; r < R; ++r) a[it][r] = a[it][r] * twiddle<SIGN>(tw, r * j1);
            }
            dftR<R, SIGN>(a[it]);
            pos[it] = b * bstr + ((i - k) * R + k) * pstr;
        }
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < MAXI; ++it) {
        if (pos[it] >= 0) {
            C *o = buf + pos[it];
#pragma unroll
            for (int r = 0; r < R; ++r) o[(size_t)r * P * pstr] = a[it][r];
        }
    }
    __syncthreads();
}

__host__ __device__ __forceinline__ int pick_radix(int rem) {
    if (rem % 8 == 0 && rem != 16) return 8;
    if (rem % 4 == 0) return 4;
    if (rem % 2 == 0) return 2;
    return 3;
}

// number of items one thread must hold for a stage of radix R (host helper)
__host__ __device__ __forceinline__ int fft_max_items(int L, int nb, int nthreads) {
    int worst = 0, P = 1;
    while (P < L) {
        int R = pick_radix(L / P);
        int W = nb * (L / R);
        int items = (W + nthreads - 1) / nthreads;
        if (items > worst) worst = items;
        P *= R;
    }
    return worst;
}

// In-place batched FFT of nb sequences of length L (SIGN=-1 forward, +1 inverse,
// unnormalised).  Must be called by every thread of the block.
template <int SIGN, int MAXI, typename C>
__device__ void fft_smem(C *buf, int L, int nb, int pstr, int bstr, const C *tw, int Lmax) {
    const int twstep = Lmax / L;
    int P = 1;
    while (P < L) {
        int R = pick_radix(L / P);
        switch (R) {
            case 8: fft_stage<8, SIGN, MAXI>(buf, L, P, nb, pstr, bstr, tw, twstep); break;
            case 4: fft_stage<4, SIGN, MAXI>(buf, L, P, nb, pstr, bstr, tw, twstep); break;
            case 2: fft_stage<2, SIGN, MAXI>(buf, L, P, nb, pstr, bstr, tw, twstep); break;
            default: fft_stage<3, SIGN, MAXI>(buf, L, P, nb, pstr, bstr, tw, twstep); break;
        }
        P *= R;
    }
}

}  // namespace tdda
