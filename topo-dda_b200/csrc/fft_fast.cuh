// Compile-time-length batched FFTs in shared memory (ping-pong Stockham).
//
// Same mixed-radix Stockham autosort as fft_smem.cuh, specialised for one
// transform length L known at compile time: the radix of every stage, the
// span P and the twiddle strides are constants, so the per-item index math is
// shifts and masks.  Stages are out of place (buffer a -> buffer b -> a ...),
// so a thread holds one radix-R butterfly at a time and any batch size works
// with any thread count: each thread owns one batch column b and walks the
// butterflies i0, i0 + istep, ... of that column.
// Radix plan: 256 = 16*16, 128 = 16*8, 64 = 8*8, 32 = 8*4, 16 = 16, and
// 8/4/2/3 for the rest (lengths 2^a 3^b, e.g. 192 = 16*4*3, 96 = 8*4*3).
#pragma once

#include "fft_smem.cuh"

namespace tdda {

__host__ __device__ constexpr int fast_radix(int rem) {
    return (rem == 64 || rem == 32) ? 8
           : (rem >= 128 && rem % 16 == 0) ? 16
           : (rem == 16) ? 16
           : (rem % 8 == 0) ? 8
           : (rem % 4 == 0) ? 4
           : (rem % 2 == 0) ? 2
                            : 3;
}

__host__ __device__ constexpr int fast_stages(int L) {
    int s = 0, P = 1;
    while (P < L) {
        P *= fast_radix(L / P);
        ++s;
    }
    return s;
}

// 16-point DFT as 4 x 4 (index n = 4 n1 + n2, k = k1 + 4 k2)
template <int SIGN, typename C> __device__ __forceinline__ void dft16(C (&a)[16]) {
    using Rl = typename RealOf<C>::type;
    // columns n2: 4-point DFTs over n1
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) dft4<SIGN>(a[n2], a[n2 + 4], a[n2 + 8], a[n2 + 12]);
    // after dft4 in place: a[n2 + 4 k1] = y[n2][k1]; twiddle by W16^(n2 k1)
    const Rl c1 = (Rl)0.92387953251128675613, s1 = (Rl)0.38268343236508977173;  // cos/sin(pi/8)
    const Rl r2 = (Rl)0.70710678118654752440;
    auto tw = [&](C v, int j) -> C {  // v * exp(SIGN * 2 pi i j / 16)
        Rl c, s;
        switch (j) {
            case 1: c = c1; s = s1; break;
            case 2: c = r2; s = r2; break;
            case 3: c = s1; s = c1; break;
            case 4: c = 0; s = 1; break;
            case 6: c = -r2; s = r2; break;
            case 9: c = -c1; s = -s1; break;
            default: c = 1; s = 0; break;
        }
        s = SIGN * s;
        C r;
        r.x = v.x * c - v.y * s;
        r.y = v.x * s + v.y * c;
        return r;
    };
#pragma unroll
    for (int n2 = 1; n2 < 4; ++n2)
#pragma unroll
        for (int k1 = 1; k1 < 4; ++k1) a[n2 + 4 * k1] = tw(a[n2 + 4 * k1], n2 * k1);
    // rows k1: 4-point DFTs over n2 -> X[k1 + 4 k2]
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) dft4<SIGN>(a[4 * k1], a[4 * k1 + 1], a[4 * k1 + 2], a[4 * k1 + 3]);
    // now a[4 k1 + k2] = X[k1 + 4 k2]: transpose the 4 x 4 index grid
    C t[16];
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1)
#pragma unroll
        for (int k2 = 0; k2 < 4; ++k2) t[k1 + 4 * k2] = a[4 * k1 + k2];
#pragma unroll
    for (int q = 0; q < 16; ++q) a[q] = t[q];
}

template <int R, int SIGN, typename C> __device__ __forceinline__ void dft_fast(C (&a)[R]) {
    if constexpr (R == 16) dft16<SIGN>(a);
    else dftR<R, SIGN>(a);
}

// One out-of-place stage of span P and radix R for the column this thread owns.
// nvalid: inputs at n >= nvalid are zero and not read (first stage);
// nkeep: outputs at n >= nkeep are not needed and not written (last stage).
template <int L, int P, int SIGN, typename C>
__device__ __forceinline__ void fast_stage(const C *__restrict__ in, C *__restrict__ out, int b, int i0,
                                           int istep, int pstr, int bstr, const C *__restrict__ tw,
                                           int twstep, int nvalid, int nkeep) {
    constexpr int R = fast_radix(L / P);
    constexpr int LR = L / R;
    constexpr int TS = L / (P * R);
    constexpr bool first = (P == 1), last = (P * R == L);
    if (b >= 0) {
        const C *ib = in + b * bstr;
        C *ob = out + b * bstr;
        for (int i = i0; i < LR; i += istep) {
            const int k = i % P;
            C a[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int n = i + r * LR;
                a[r] = (first && n >= nvalid) ? czero<C>() : ib[n * pstr];
            }
            if (P > 1 && k != 0) {
                const int j1 = k * TS * twstep;
#pragma unroll
                for (int r = 1; r < R; ++r) a[r] = a[r] * twiddle<SIGN>(tw, r * j1);
            }
            dft_fast<R, SIGN>(a);
            const int j = (i - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int n = j + r * P;
                if (!last || n < nkeep) ob[n * pstr] = a[r];
            }
        }
    }
    __syncthreads();
}

template <int L, int P, int SIGN, typename C>
__device__ __forceinline__ C *fast_stages_from(C *a, C *b, int col, int i0, int istep, int pstr, int bstr,
                                               const C *tw, int twstep, int nvalid, int nkeep) {
    if constexpr (P >= L) {
        return a;
    } else {
        fast_stage<L, P, SIGN>(a, b, col, i0, istep, pstr, bstr, tw, twstep, nvalid, nkeep);
        return fast_stages_from<L, P * fast_radix(L / P), SIGN>(b, a, col, i0, istep, pstr, bstr, tw, twstep,
                                                                nvalid, nkeep);
    }
}

// In-place variant: every butterfly of a stage is loaded into registers,
// transformed, and stored after a barrier.  Thread t owns butterflies
// t, t + NTH, ... (at most K per stage, K = ceil(NBMAX * (L / R) / NTH) for a
// batch of at most NBMAX columns).  In the first stage, positions n >= nvalid
// are read as zero (zero-padded input), so they need not be initialised.
template <int L, int P, int SIGN, int NBMAX, int NTH, typename C>
__device__ __forceinline__ void ip_stage(C *buf, int nb, int pstr, int bstr, const C *__restrict__ tw, int twstep,
                                         int nvalid, int nkeep) {
    constexpr int R = fast_radix(L / P);
    constexpr int LR = L / R;
    constexpr int TS = L / (P * R);
    constexpr bool last = (P * R == L);
    constexpr int K = (NBMAX * LR + NTH - 1) / NTH;
    C a[K][R];
    int base[K], jpos[K];
#pragma unroll
    for (int q = 0; q < K; ++q) {
        const int w = threadIdx.x + q * NTH;
        base[q] = -1;
        jpos[q] = 0;
        if (w < nb * LR) {
            const int b = w % nb, i = w / nb;
            const int k = i % P;
            const C *col = buf + b * bstr;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int n = i + r * LR;
                if (P == 1 && n >= nvalid) a[q][r] = czero<C>();
                else a[q][r] = col[n * pstr];
            }
            if (P > 1 && k != 0) {
                const int j1 = k * TS * twstep;
#pragma unroll
                for (int r = 1; r < R; ++r) a[q][r] = a[q][r] * twiddle<SIGN>(tw, r * j1);
            }
            dft_fast<R, SIGN>(a[q]);
            jpos[q] = (i - k) * R + k;
            base[q] = b * bstr + jpos[q] * pstr;
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < K; ++q) {
        if (base[q] >= 0) {
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (!last || jpos[q] + r * P < nkeep) buf[base[q] + r * P * pstr] = a[q][r];
        }
    }
    __syncthreads();
}

template <int L, int P, int SIGN, int NBMAX, int NTH, typename C>
__device__ __forceinline__ void ip_stages_from(C *buf, int nb, int pstr, int bstr, const C *tw, int twstep,
                                               int nvalid, int nkeep) {
    if constexpr (P < L) {
        ip_stage<L, P, SIGN, NBMAX, NTH>(buf, nb, pstr, bstr, tw, twstep, nvalid, nkeep);
        ip_stages_from<L, P * fast_radix(L / P), SIGN, NBMAX, NTH>(buf, nb, pstr, bstr, tw, twstep, nvalid, nkeep);
    }
}

// nb <= NBMAX columns, blockDim.x == NTH; nvalid: inputs at n >= nvalid are
// zero (never read); nkeep: only outputs n < nkeep are written by the last stage.
template <int L, int SIGN, int NBMAX, int NTH, typename C>
__device__ __forceinline__ void fft_ip(C *buf, int nb, int pstr, int bstr, const C *tw, int Lmax, int nvalid,
                                       int nkeep = L) {
    ip_stages_from<L, 1, SIGN, NBMAX, NTH>(buf, nb, pstr, bstr, tw, Lmax / L, nvalid, nkeep);
}

// largest number of butterflies any stage of a length-L transform needs per column
__host__ __device__ constexpr int fast_max_items(int L) {
    int m = 0, P = 1;
    while (P < L) {
        int R = fast_radix(L / P);
        if (L / R > m) m = L / R;
        P *= R;
    }
    return m;
}

// Batched length-L FFT of nb columns held in buffer a (element (b, n) at
// b * bstr + n * pstr); buffer b is scratch of the same shape.  Returns the
// buffer that holds the result.  Every thread of the block must call it.
template <int L, int SIGN, typename C>
__device__ __forceinline__ C *fft_fast(C *a, C *b, int nb, int pstr, int bstr, const C *tw, int Lmax,
                                       int nvalid = L, int nkeep = L) {
    const int istep = blockDim.x / nb;
    const int col = (int)threadIdx.x < istep * nb ? (int)threadIdx.x % nb : -1;
    const int i0 = (int)threadIdx.x / (nb > 0 ? nb : 1);
    return fast_stages_from<L, 1, SIGN>(a, b, col, i0, istep, pstr, bstr, tw, Lmax / L, nvalid, nkeep);
}

}  // namespace tdda
