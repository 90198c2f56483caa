// Fused zero-padded FFT convolution A.x and the BiCGSTAB built on it.
//
// One application of the interaction operator runs as three kernels:
//   pass 1  k_fwd_zy : per (x-slab, component): load the ny*nz slab (with a
//            fused prologue that can form the slab from several solver
//            vectors), z-FFT (zero padded), y-FFT (zero padded), store the
//            populated x-half of the spectrum to T.
//   pass 2  k_xconv  : per (ky, kz-chunk): x-FFT of all three components of
//            every right-hand side, symmetric 3x3 multiply by the cached
//            folded Green-tensor spectrum, inverse x-FFT, store back to T
//            (only x < nx is kept).
//   pass 3  k_inv_yz : per (x-slab, component): inverse y-FFT, crop y < ny,
//            inverse z-FFT, crop z < nz, fused epilogue (polarisability
//            diagonal, residual / vector updates, dot products with a
//            deterministic last-block reduction that also computes the
//            BiCGSTAB scalars on the device).
// Reference: AProductCore::Aproduct (src/AProductCore.cpp:461-515) with the
// element-wise kernels of src/Kernel.cu:44-125, plus DDAModel::Aproductwithalb
// (src/DDAModel.cpp:1194-1203) and DDAModel::bicgstab (src/DDAModel.cpp:899-1009).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "fft_fast.cuh"
#include "fft_reg.cuh"
#include "operator.cuh"

namespace tdda {

constexpr int NT = 512;          // threads per CTA of the convolution passes
constexpr int MAXI = 2;          // FFT work items a thread holds per stage
constexpr int SMEM_MAX = 200 * 1024;
constexpr int UPD_BLOCKS = 296;  // 2 x 148 SMs for the element-wise update

// ----------------------------------------------------------------------------
// deterministic reductions
// ----------------------------------------------------------------------------
template <int NQ> __device__ __forceinline__ void block_sum(double2 (&v)[NQ]) {
    __shared__ double2 red[NQ > 0 ? NQ : 1][32];
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NQ; ++q)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            v[q].x += __shfl_xor_sync(0xffffffffu, v[q].x, off);
            v[q].y += __shfl_xor_sync(0xffffffffu, v[q].y, off);
        }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < NQ; ++q) red[q][wid] = v[q];
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            v[q] = lane < nw ? red[q][lane] : make_double2(0.0, 0.0);
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                v[q].x += __shfl_xor_sync(0xffffffffu, v[q].x, off);
                v[q].y += __shfl_xor_sync(0xffffffffu, v[q].y, off);
            }
        }
    }
}

// Every block contributes NQ complex sums; the last block to finish adds the
// per-block partials in block order and calls fin(rhs, totals) on thread 0.
// The partials of one RHS take nblk * NQ entries: the scratch holds
// max(6 nx, UPD_BLOCKS) * kMaxNQ per RHS (pass 3 runs nx * 3 blocks per RHS,
// 2 nx * 3 in the complex128 cluster form,
// the vector kernels UPD_BLOCKS), and no reduction uses more than kMaxNQ sums.
constexpr int kMaxNQ = 4;
template <int NQ, class Fin>
__device__ __forceinline__ void reduce_finalize(double2 (&v)[NQ], double2 *part, unsigned *counter,
                                                int bid, int nblk, const Fin &fin, int rhs) {
    block_sum<NQ>(v);
    __shared__ int am_last;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) part[(size_t)bid * NQ + q] = v[q];
        __threadfence();
        unsigned prev = atomicAdd(counter, 1u);
        am_last = (prev == (unsigned)nblk - 1u);
    }
    __syncthreads();
    if (!am_last) return;
    __threadfence();
    double2 s[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) s[q] = make_double2(0.0, 0.0);
    for (int b = threadIdx.x; b < nblk; b += blockDim.x)
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            double2 w = __ldcg(part + (size_t)b * NQ + q);
            s[q].x += w.x;
            s[q].y += w.y;
        }
    block_sum<NQ>(s);
    if (threadIdx.x == 0) {
        fin(rhs, s);
        *counter = 0u;
    }
}

__device__ __forceinline__ bool dzero(double2 a) { return a.x == 0.0 && a.y == 0.0; }
__device__ __forceinline__ bool dfinite(double2 a) { return isfinite(a.x) && isfinite(a.y); }

// ----------------------------------------------------------------------------
// the three passes
// ----------------------------------------------------------------------------
template <typename C, class Pro>
__global__ void __launch_bounds__(NT) k_fwd_zy(ConvGeom g, C *__restrict__ T, const C *__restrict__ tw,
                                               Pro pro) {
    pdl_wait();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *A = reinterpret_cast<C *>(smem_raw);
    C *B = A + (size_t)g.ny * g.pA;
    const int x = blockIdx.x, c = blockIdx.y, rhs = blockIdx.z;
    if (pro.skip(rhs)) return;
    const int nyz = g.ny * g.nz;
    const long long cell0 = (long long)x * nyz;
    for (int e = threadIdx.x; e < nyz; e += NT) {
        int y = e / g.nz, z = e - y * g.nz;
        A[y * g.pA + z] = pro.load(rhs, c, cell0 + e);
    }
    const int zpad = g.Lz - g.nz;
    for (int e = threadIdx.x; e < g.ny * zpad; e += NT) {
        int y = e / zpad, z = g.nz + (e - y * zpad);
        A[y * g.pA + z] = czero<C>();
    }
    __syncthreads();
    for (int y0 = 0; y0 < g.ny; y0 += g.YC)
        fft_smem<-1, MAXI>(A + y0 * g.pA, g.Lz, min(g.YC, g.ny - y0), 1, g.pA, tw, g.Lmax);
    C *Tc = T + ((size_t)(rhs * 3 + c) * g.nx + x) * (size_t)g.Ly * g.Lz;
    for (int kz0 = 0; kz0 < g.Lz; kz0 += g.CK) {
        for (int e = threadIdx.x; e < g.ny * g.CK; e += NT) {
            int y = e / g.CK, kl = e - y * g.CK;
            B[y * g.pB + kl] = A[y * g.pA + kz0 + kl];
        }
        for (int e = threadIdx.x; e < (g.Ly - g.ny) * g.CK; e += NT) {
            int yy = e / g.CK, kl = e - yy * g.CK;
            B[(g.ny + yy) * g.pB + kl] = czero<C>();
        }
        __syncthreads();
        fft_smem<-1, MAXI>(B, g.Ly, g.CK, g.pB, 1, tw, g.Lmax);
        for (int e = threadIdx.x; e < g.Ly * g.CK; e += NT) {
            int ky = e / g.CK, kl = e - ky * g.CK;
            Tc[(size_t)ky * g.Lz + kz0 + kl] = B[ky * g.pB + kl];
        }
        __syncthreads();
    }
}

__device__ __forceinline__ void fold(int k, int L, int &fk, int &sgn) {
    if (2 * k <= L) { fk = k; sgn = 1; }
    else { fk = L - k; sgn = -1; }
}

// The 6 entries of one folded tensor point (xx, xy, xz, yy, yz, zz; 16-byte
// aligned): three 16-byte loads in complex64, six in complex128.
template <typename C> __device__ __forceinline__ void load6(const C *__restrict__ a, C (&t)[6]) {
    if constexpr (sizeof(C) == 8) {
        const float4 *q = reinterpret_cast<const float4 *>(a);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const float4 v = q[i];
            t[2 * i].x = v.x; t[2 * i].y = v.y;
            t[2 * i + 1].x = v.z; t[2 * i + 1].y = v.w;
        }
    } else {
#pragma unroll
        for (int i = 0; i < 6; ++i) t[i] = a[i];
    }
}

// w (the 3 components of one right-hand side, CKx apart) <- A w for the folded
// symmetric tensor entry a[6], with the parity signs of its off-diagonal terms
template <typename C>
__device__ __forceinline__ void mul_sym3(const C *__restrict__ a, typename RealOf<C>::type sxy,
                                         typename RealOf<C>::type sxz, typename RealOf<C>::type syz, C *w, int CKx) {
    C e[6];
    load6(a, e);
    C axx = e[0], axy = sxy * e[1], axz = sxz * e[2];
    C ayy = e[3], ayz = syz * e[4], azz = e[5];
    C bx = w[0], by = w[CKx], bz = w[2 * CKx];
    w[0] = axx * bx + axy * by + axz * bz;
    w[CKx] = axy * bx + ayy * by + ayz * bz;
    w[2 * CKx] = axz * bx + ayz * by + azz * bz;
}

// Pass 2: x transforms, tensor multiply, inverse x transforms for one ky and
// a chunk of kz.  tab != nullptr: right-hand side r uses its own tensor tab[r]
// (same grid, another wavelength or period); else every one uses ahat.
template <typename C>
__global__ void __launch_bounds__(NT) k_xconv(ConvGeom g, C *__restrict__ T, const C *__restrict__ ahat,
                                              const C *const *__restrict__ tab, const C *__restrict__ tw, int nrhs,
                                              const SolverState *__restrict__ st) {
    pdl_wait();
    using R = typename RealOf<C>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *Cb = reinterpret_cast<C *>(smem_raw);
    if (st != nullptr) {
        bool any = false;
        for (int r = 0; r < nrhs; ++r) any |= (st[r].done == 0);
        if (!any) return;
    }
    const int ky = blockIdx.x, kz0 = blockIdx.y * g.CKx;
    const int CKx = g.CKx, nbat = nrhs * 3 * CKx, pC = g.pC;
    const size_t plane = (size_t)g.Ly * g.Lz;
    const size_t off = (size_t)ky * g.Lz + kz0;
    for (int e = threadIdx.x; e < g.nx * nbat; e += NT) {
        int x = e / nbat, rem = e - x * nbat;
        int rc = rem / CKx, kl = rem - rc * CKx;
        Cb[x * pC + rem] = T[((size_t)rc * g.nx + x) * plane + off + kl];
    }
    for (int e = threadIdx.x; e < (g.Lx - g.nx) * nbat; e += NT) {
        int xx = e / nbat, rem = e - xx * nbat;
        Cb[(g.nx + xx) * pC + rem] = czero<C>();
    }
    __syncthreads();
    fft_smem<-1, MAXI>(Cb, g.Lx, nbat, pC, 1, tw, g.Lmax);
    int fky, sy;
    fold(ky, g.Ly, fky, sy);
    for (int e = threadIdx.x; e < g.Lx * CKx; e += NT) {
        int kx = e / CKx, kl = e - kx * CKx;
        int fkx, sx, fkz, sz;
        fold(kx, g.Lx, fkx, sx);
        fold(kz0 + kl, g.Lz, fkz, sz);
        const size_t ti = (((size_t)fky * g.hx + fkx) * g.hz + fkz) * 6;
        C *v = Cb + kx * pC + kl;
        if (tab != nullptr) {
            for (int r = 0; r < nrhs; ++r)
                mul_sym3(tab[r] + ti, (R)(sx * sy), (R)(sx * sz), (R)(sy * sz), v + r * 3 * CKx, CKx);
            continue;
        }
        C e6[6];
        load6(ahat + ti, e6);
        C axx = e6[0], axy = (R)(sx * sy) * e6[1], axz = (R)(sx * sz) * e6[2];
        C ayy = e6[3], ayz = (R)(sy * sz) * e6[4], azz = e6[5];
        for (int r = 0; r < nrhs; ++r) {
            C *w = v + r * 3 * CKx;
            C bx = w[0], by = w[CKx], bz = w[2 * CKx];
            w[0] = axx * bx + axy * by + axz * bz;
            w[CKx] = axy * bx + ayy * by + ayz * bz;
            w[2 * CKx] = axz * bx + ayz * by + azz * bz;
        }
    }
    __syncthreads();
    fft_smem<+1, MAXI>(Cb, g.Lx, nbat, pC, 1, tw, g.Lmax);
    for (int e = threadIdx.x; e < g.nx * nbat; e += NT) {
        int x = e / nbat, rem = e - x * nbat;
        int rc = rem / CKx, kl = rem - rc * CKx;
        T[((size_t)rc * g.nx + x) * plane + off + kl] = Cb[x * pC + rem];
    }
}

// Pass 2 for a compile-time x length L: same work as k_xconv, with the x
// transforms on the ping-pong compile-time FFT (256-thread CTAs, several CTAs
// per SM so one CTA's loads overlap another's transforms).
constexpr int NT2 = 256;

template <typename C, int L>
__global__ void __launch_bounds__(NT2) k_xconv_fast(ConvGeom g, C *__restrict__ T, const C *__restrict__ ahat,
                                                    const C *const *__restrict__ tab, const C *__restrict__ tw,
                                                    int nrhs, const SolverState *__restrict__ st) {
    pdl_wait();
    using R = typename RealOf<C>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (st != nullptr) {
        bool any = false;
        for (int r = 0; r < nrhs; ++r) any |= (st[r].done == 0);
        if (!any) return;
    }
    const int CKx = g.CKx2, nbat = nrhs * 3 * CKx;
    C *b0 = reinterpret_cast<C *>(smem_raw);
    C *b1 = b0 + L * nbat;
    const int ky = blockIdx.x, kz0 = blockIdx.y * CKx;
    const size_t plane = (size_t)g.Ly * g.Lz;
    const size_t off = (size_t)ky * g.Lz + kz0;
    for (int e = threadIdx.x; e < g.nx * nbat; e += NT2) {
        int x = e / nbat, rem = e - x * nbat;
        int rc = rem / CKx, kl = rem - rc * CKx;
        b0[x * nbat + rem] = T[((size_t)rc * g.nx + x) * plane + off + kl];
    }
    __syncthreads();
    C *f = fft_fast<L, -1>(b0, b1, nbat, nbat, 1, tw, g.Lmax, g.nx, L);
    int fky, sy;
    fold(ky, g.Ly, fky, sy);
    for (int e = threadIdx.x; e < L * CKx; e += NT2) {
        int kx = e / CKx, kl = e - kx * CKx;
        int fkx, sx, fkz, sz;
        fold(kx, L, fkx, sx);
        fold(kz0 + kl, g.Lz, fkz, sz);
        const size_t ti = (((size_t)fky * g.hx + fkx) * g.hz + fkz) * 6;
        C *v = f + kx * nbat + kl;
        if (tab != nullptr) {
            for (int r = 0; r < nrhs; ++r)
                mul_sym3(tab[r] + ti, (R)(sx * sy), (R)(sx * sz), (R)(sy * sz), v + r * 3 * CKx, CKx);
            continue;
        }
        C e6[6];
        load6(ahat + ti, e6);
        C axx = e6[0], axy = (R)(sx * sy) * e6[1], axz = (R)(sx * sz) * e6[2];
        C ayy = e6[3], ayz = (R)(sy * sz) * e6[4], azz = e6[5];
        for (int r = 0; r < nrhs; ++r) {
            C *w = v + r * 3 * CKx;
            C bx = w[0], by = w[CKx], bz = w[2 * CKx];
            w[0] = axx * bx + axy * by + axz * bz;
            w[CKx] = axy * bx + ayy * by + ayz * bz;
            w[2 * CKx] = axz * bx + ayz * by + azz * bz;
        }
    }
    __syncthreads();
    C *res = fft_fast<L, +1>(f, f == b0 ? b1 : b0, nbat, nbat, 1, tw, g.Lmax, L, g.nx);
    for (int e = threadIdx.x; e < g.nx * nbat; e += NT2) {
        int x = e / nbat, rem = e - x * nbat;
        int rc = rem / CKx, kl = rem - rc * CKx;
        T[((size_t)rc * g.nx + x) * plane + off + kl] = res[x * nbat + rem];
    }
}

template <typename C>
static bool launch_xconv_fast(const ConvGeom &g, C *T, const C *ahat, const C *const *tab, const C *tw, int nrhs,
                              const SolverState *st, cudaStream_t s) {
    dim3 grid(g.Ly, g.Lz / g.CKx2, 1);
    switch (g.Lx) {
        case 256: launch_dep((k_xconv_fast<C, 256>), grid, dim3(NT2), g.smem_x2, s, g, T, ahat, tab, tw, nrhs, st); return true;
        case 128: launch_dep((k_xconv_fast<C, 128>), grid, dim3(NT2), g.smem_x2, s, g, T, ahat, tab, tw, nrhs, st); return true;
        case 64: launch_dep((k_xconv_fast<C, 64>), grid, dim3(NT2), g.smem_x2, s, g, T, ahat, tab, tw, nrhs, st); return true;
        case 32: launch_dep((k_xconv_fast<C, 32>), grid, dim3(NT2), g.smem_x2, s, g, T, ahat, tab, tw, nrhs, st); return true;
        case 192: launch_dep((k_xconv_fast<C, 192>), grid, dim3(NT2), g.smem_x2, s, g, T, ahat, tab, tw, nrhs, st); return true;
        case 96: launch_dep((k_xconv_fast<C, 96>), grid, dim3(NT2), g.smem_x2, s, g, T, ahat, tab, tw, nrhs, st); return true;
        default: return false;
    }
}

// Pass 2 as a register-resident two-level FFT, for Lx = L = R1 * 8 with
// nx = L / 2 (the zero padding is exactly the upper half):
//   forward: thread (column, n2) loads x = 8 n1 + n2 (n1 < R1 / 2) straight
//   from T, runs the half-input R1-point DFT, twiddles by W_L^(n2 k1) and
//   writes to shared memory; thread (rhs, kz, k1) reads the 8 values of each
//   of the 3 components, runs 8-point DFTs (X at kx = k1 + R1 k2), applies the
//   3x3 tensor in registers, runs the inverse 8-point DFTs, twiddles by
//   W_L^(-n1 k1) and writes back; thread (column, n1) finishes with the
//   half-output R1-point inverse DFT and stores x = n1 + 8 n2 < nx to T.
// One shared-memory exchange per direction; every thread holds one task.
// Tasks run with the kz index fastest, then component / right-hand side, so a
// half-warp touches consecutive columns of a row (or rows 8 x odd pitch apart):
// the exchanges are free of bank conflicts.
// With g.pair_x a CTA takes ky and its mirror Ly - ky (ky = 0 and ky = Ly / 2
// alone): both read the same folded tensor entries (the mirror with the sign
// of the y parity), so the tensor slice one CTA reads is half as large and
// stays in L1 for the second member.  Columns are then (member, rhs, component,
// kz) with kz fastest.
constexpr int NTR = 256;

template <typename C, int L, bool P>
__global__ void __launch_bounds__(NTR, sizeof(C) == 8 ? 3 : 1) k_xconv_reg(ConvGeom g, C *__restrict__ T, const C *__restrict__ ahat,
                                                   const C *const *__restrict__ tab, const C *__restrict__ tw,
                                                   int nrhs, const SolverState *__restrict__ st) {
    pdl_wait();
    using R = typename RealOf<C>::type;
    constexpr int R2 = 8, R1 = L / R2, H1 = R1 / 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *S = reinterpret_cast<C *>(smem_raw);
    if (st != nullptr) {
        bool any = false;
        for (int r = 0; r < nrhs; ++r) any |= (st[r].done == 0);
        if (!any) return;
    }
    const int CK = g.CKr, kyA = blockIdx.x, kz0 = blockIdx.y * CK;
    const int nky = (P && kyA != 0 && 2 * kyA != g.Ly) ? 2 : 1;   // P: g.pair_x
    const int nrc = nrhs * 3;                 // columns per kz and member
    const int ncomp = nrc * nky;
    const int ncol = ncomp * CK, ncolP = ncol | 1;
    const size_t plane = (size_t)g.Ly * g.Lz;
    const int twL = g.Lmax / L, twR1 = g.Lmax / R1;
    const int t = threadIdx.x;
    const int tasks1 = ncol * R2, tasks2 = nrhs * nky * CK * R1;
    // complex64: threads without a first-level task bring the tensor entries of
    // the multiply (one folded ky, the folded kz of the chunk, every folded kx)
    // into L1 while the others transform (shared tensor only).  B200,
    // 128x128x32: 67.0 -> 65.1 us per launch; complex128 (paired ky) measured
    // 140.4 -> 142.1 us with it, so it is left out there.
    if (sizeof(C) == 8 && t >= tasks1 && tab == nullptr) {
        int fky, sgn, lo = g.Lz, hi = 0;
        fold(kyA, g.Ly, fky, sgn);
        for (int kl = 0; kl < CK; ++kl) {
            int fz;
            fold(kz0 + kl, g.Lz, fz, sgn);
            lo = min(lo, fz);
            hi = max(hi, fz);
        }
        const int run = (hi - lo + 1) * 6 * (int)sizeof(C);  // bytes per folded kx
        const int lines = (run + 127) / 128 + 1;
        const char *base = reinterpret_cast<const char *>(ahat + ((size_t)fky * g.hx * g.hz + lo) * 6);
        for (int i = t - tasks1; i < g.hx * lines; i += NTR - tasks1) {
            const int fkx = i / lines, l = i - fkx * lines;
            const char *p0 = base + (size_t)fkx * g.hz * 6 * sizeof(C);
            const char *q = reinterpret_cast<const char *>(reinterpret_cast<uintptr_t>(p0) & ~(uintptr_t)127) + 128 * l;
            if (q < p0 + run && q >= reinterpret_cast<const char *>(ahat))
                asm volatile("prefetch.global.L1 [%0];" ::"l"(q));
        }
    }
    // forward, first level: the column's R1-point DFT over x = 8 n1 + n2
    if (t < tasks1) {
        const int kl = t % CK, rest = t / CK, rc = rest % ncomp, n2 = rest / ncomp;
        const int col = rc * CK + kl;
        const int m = P ? rc / nrc : 0, ky = m ? g.Ly - kyA : kyA;
        const C *src = T + (size_t)(rc - m * nrc) * g.nx * plane + (size_t)ky * g.Lz + kz0 + kl;
        C a[H1], b[H1];
#pragma unroll
        for (int n1 = 0; n1 < H1; ++n1) a[n1] = src[(size_t)(R2 * n1 + n2) * plane];
        dft_half_in<H1, -1>(a, b, tw, twR1);
#pragma unroll
        for (int q = 0; q < H1; ++q) {
            const int k1 = 2 * q;
            C y0 = a[q], y1 = b[q];
            if (n2 != 0) {
                if (k1 != 0) y0 = y0 * twiddle<-1>(tw, n2 * k1 * twL);
                y1 = y1 * twiddle<-1>(tw, n2 * (k1 + 1) * twL);
            }
            S[(k1 * R2 + n2) * ncolP + col] = y0;
            S[((k1 + 1) * R2 + n2) * ncolP + col] = y1;
        }
    }
    __syncthreads();
    // second level, tensor, inverse first level
    C v[3][R2];
    int kl2 = 0, k1 = 0, rm = 0, rhs = 0, m = 0;
    if (t < tasks2) {
        kl2 = t % CK;
        const int rest = t / CK;
        if constexpr (P) {
            rm = rest % (nrhs * nky);
            k1 = rest / (nrhs * nky);
            m = rm / nrhs;
            rhs = rm - m * nrhs;
        } else {
            rm = rhs = rest % nrhs;
            k1 = rest / nrhs;
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int col = (rm * 3 + c) * CK + kl2;
#pragma unroll
            for (int n2 = 0; n2 < R2; ++n2) v[c][n2] = S[(k1 * R2 + n2) * ncolP + col];
        }
    }
    __syncthreads();
    if (t < tasks2) {
#pragma unroll
        for (int c = 0; c < 3; ++c) dftR<R2, -1>(v[c]);
        int fky, sy, fkz, sz;
        fold(m ? g.Ly - kyA : kyA, g.Ly, fky, sy);
        fold(kz0 + kl2, g.Lz, fkz, sz);
        const C *A = (tab != nullptr) ? tab[rhs] : ahat;
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) {
            int fkx, sx;
            fold(k1 + R1 * k2, L, fkx, sx);
            C e6[6];
            load6(A + (((size_t)fky * g.hx + fkx) * g.hz + fkz) * 6, e6);
            C axx = e6[0], axy = (R)(sx * sy) * e6[1], axz = (R)(sx * sz) * e6[2];
            C ayy = e6[3], ayz = (R)(sy * sz) * e6[4], azz = e6[5];
            C bx = v[0][k2], by = v[1][k2], bz = v[2][k2];
            v[0][k2] = axx * bx + axy * by + axz * bz;
            v[1][k2] = axy * bx + ayy * by + ayz * bz;
            v[2][k2] = axz * bx + ayz * by + azz * bz;
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) dftR<R2, +1>(v[c]);
        if (k1 != 0) {
#pragma unroll
            for (int n1 = 1; n1 < R2; ++n1) {
                const C w = twiddle<+1>(tw, k1 * n1 * twL);
#pragma unroll
                for (int c = 0; c < 3; ++c) v[c][n1] = v[c][n1] * w;
            }
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int col = (rm * 3 + c) * CK + kl2;
#pragma unroll
            for (int n1 = 0; n1 < R2; ++n1) S[(k1 * R2 + n1) * ncolP + col] = v[c][n1];
        }
    }
    __syncthreads();
    // inverse, second level: outputs x = n1 + 8 n2 for n2 < R1 / 2 (x < nx)
    if (t < tasks1) {
        const int kl = t % CK, rest = t / CK, rc = rest % ncomp, n1 = rest / ncomp;
        const int col = rc * CK + kl;
        const int mm = P ? rc / nrc : 0, ky = mm ? g.Ly - kyA : kyA;
        C e[H1], o[H1];
#pragma unroll
        for (int q = 0; q < H1; ++q) {
            e[q] = S[((2 * q) * R2 + n1) * ncolP + col];
            o[q] = S[((2 * q + 1) * R2 + n1) * ncolP + col];
        }
        dft_half_out<H1, +1>(e, o, tw, twR1);
        C *dst = T + (size_t)(rc - mm * nrc) * g.nx * plane + (size_t)ky * g.Lz + kz0 + kl;
#pragma unroll
        for (int n2 = 0; n2 < H1; ++n2) dst[(size_t)(n1 + R2 * n2) * plane] = e[n2];
    }
}

template <typename C, bool P>
static bool launch_xconv_reg_t(const ConvGeom &g, dim3 grid, C *T, const C *ahat, const C *const *tab,
                               const C *tw, int nrhs, const SolverState *st, cudaStream_t s) {
    switch (g.Lx) {
        case 256: launch_dep((k_xconv_reg<C, 256, P>), grid, dim3(NTR), g.smem_r, s, g, T, ahat, tab, tw, nrhs, st); return true;
        case 192: launch_dep((k_xconv_reg<C, 192, P>), grid, dim3(NTR), g.smem_r, s, g, T, ahat, tab, tw, nrhs, st); return true;
        case 128: launch_dep((k_xconv_reg<C, 128, P>), grid, dim3(NTR), g.smem_r, s, g, T, ahat, tab, tw, nrhs, st); return true;
        case 96: launch_dep((k_xconv_reg<C, 96, P>), grid, dim3(NTR), g.smem_r, s, g, T, ahat, tab, tw, nrhs, st); return true;
        case 64: launch_dep((k_xconv_reg<C, 64, P>), grid, dim3(NTR), g.smem_r, s, g, T, ahat, tab, tw, nrhs, st); return true;
        default: return false;
    }
}

template <typename C>
static bool launch_xconv_reg(const ConvGeom &g, C *T, const C *ahat, const C *const *tab, const C *tw, int nrhs,
                             const SolverState *st, cudaStream_t s) {
    if (!g.reg_x) return false;
    dim3 grid(g.pair_x ? g.Ly / 2 + 1 : g.Ly, g.Lz / g.CKr, 1);
    if constexpr (sizeof(C) == 16) {
        if (g.pair_x) return launch_xconv_reg_t<C, true>(g, grid, T, ahat, tab, tw, nrhs, st, s);
    }
    return launch_xconv_reg_t<C, false>(g, grid, T, ahat, tab, tw, nrhs, st, s);
}

static bool reg_x_length(int L) { return L == 256 || L == 192 || L == 128 || L == 96 || L == 64; }

static bool fast_x_length(int L) { return L == 256 || L == 192 || L == 128 || L == 96 || L == 64 || L == 32; }

// Passes 1 and 3 for complex64 with compile-time (Lz, Ly): the whole padded
// (x, component) slab [Ly][Lz + 1] sits in shared memory and 1024 threads
// transform it in place, one butterfly each per stage; zero-padded inputs are
// never stored (the first stage of each transform reads them as zero).
constexpr int NT3 = 1024;
constexpr int kSmemFast = 224 * 1024;  // dynamic SMEM opt-in of the slab kernels

template <typename C, int LZ, int LY, class Pro>
__global__ void __launch_bounds__(NT3, 1) k_fwd_zy_fast(ConvGeom g, C *__restrict__ T, const C *__restrict__ tw,
                                                        Pro pro) {
    pdl_wait();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *S = reinterpret_cast<C *>(smem_raw);
    constexpr int pS = LZ + 1;
    const int x = blockIdx.x, c = blockIdx.y, rhs = blockIdx.z;
    if (pro.skip(rhs)) return;
    const int nyz = g.ny * g.nz;
    const long long cell0 = (long long)x * nyz;
    for (int e = threadIdx.x; e < nyz; e += NT3) {
        int y = e / g.nz, z = e - y * g.nz;
        S[y * pS + z] = pro.load(rhs, c, cell0 + e);
    }
    __syncthreads();
    // ny <= (LY + 1) / 2 columns of z, LZ columns of y
    fft_ip<LZ, -1, (LY + 1) / 2, NT3>(S, g.ny, 1, pS, tw, g.Lmax, g.nz);
    fft_ip<LY, -1, LZ, NT3>(S, LZ, pS, 1, tw, g.Lmax, g.ny);
    C *Tc = T + ((size_t)(rhs * 3 + c) * g.nx + x) * (size_t)(LY * LZ);
    for (int e = threadIdx.x; e < LY * LZ; e += NT3) Tc[e] = S[(e / LZ) * pS + (e % LZ)];
}

template <typename C, int LZ, int LY, class Epi>
__global__ void __launch_bounds__(NT3, 1) k_inv_yz_fast(ConvGeom g, const C *__restrict__ T,
                                                        const C *__restrict__ tw, Epi epi) {
    pdl_wait();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *S = reinterpret_cast<C *>(smem_raw);
    constexpr int pS = LZ + 1;
    const int x = blockIdx.x, c = blockIdx.y, rhs = blockIdx.z;
    if (epi.skip(rhs)) return;
    const C *Tc = T + ((size_t)(rhs * 3 + c) * g.nx + x) * (size_t)(LY * LZ);
    {
        // every load of this thread in flight before the first shared-memory store
        constexpr int NPER = (LY * LZ + NT3 - 1) / NT3;
        C v[NPER];
#pragma unroll
        for (int q = 0; q < NPER; ++q) {
            const int e = threadIdx.x + q * NT3;
            if (e < LY * LZ) v[q] = Tc[e];
        }
#pragma unroll
        for (int q = 0; q < NPER; ++q) {
            const int e = threadIdx.x + q * NT3;
            if (e < LY * LZ) S[(e / LZ) * pS + (e % LZ)] = v[q];
        }
    }
    __syncthreads();
    fft_ip<LY, +1, LZ, NT3>(S, LZ, pS, 1, tw, g.Lmax, LY, g.ny);
    fft_ip<LZ, +1, (LY + 1) / 2, NT3>(S, g.ny, 1, pS, tw, g.Lmax, LZ, g.nz);
    const int nyz = g.ny * g.nz;
    const long long cell0 = (long long)x * nyz;
    double2 acc[Epi::NQ > 0 ? Epi::NQ : 1];
#pragma unroll
    for (int q = 0; q < (Epi::NQ > 0 ? Epi::NQ : 1); ++q) acc[q] = make_double2(0.0, 0.0);
    for (int e = threadIdx.x; e < nyz; e += NT3) {
        int y = e / g.nz, z = e - y * g.nz;
        epi.apply(rhs, c, cell0 + e, S[y * pS + z], acc);
    }
    if constexpr (Epi::NQ > 0) {
        reduce_finalize<Epi::NQ>(acc, epi.part + (size_t)rhs * epi.pstride, epi.counter + rhs,
                                 blockIdx.y * gridDim.x + blockIdx.x, gridDim.x * gridDim.y, epi, rhs);
    }
}

// (Lz, Ly) pairs with a compile-time slab kernel
#define TDDA_YZ_PAIRS(X) X(64, 256) X(32, 128) X(16, 64) X(16, 32) X(24, 96) X(32, 192) X(48, 192) X(32, 256)

static bool fast_yz_pair(int Lz, int Ly) {
#define TDDA_PAIR_TEST(a, b) if (Lz == a && Ly == b) return true;
    TDDA_YZ_PAIRS(TDDA_PAIR_TEST)
#undef TDDA_PAIR_TEST
    return false;
}

template <typename C, class Pro>
static bool launch_fwd_fast(const ConvGeom &g, dim3 grid, C *T, const C *tw, const Pro &pro, cudaStream_t s) {
    if constexpr (!std::is_same<C, float2>::value) {
        return false;
    } else {
#define TDDA_FWD_CASE(a, b)                                                                  \
    if (g.Lz == a && g.Ly == b) {                                                            \
        launch_dep((k_fwd_zy_fast<C, a, b, Pro>), grid, dim3(NT3), g.smem_yz2, s, g, T, tw, pro);           \
        return true;                                                                         \
    }
        TDDA_YZ_PAIRS(TDDA_FWD_CASE)
#undef TDDA_FWD_CASE
        return false;
    }
}

template <typename C, class Epi>
static bool launch_inv_fast(const ConvGeom &g, dim3 grid, const C *T, const C *tw, const Epi &epi, cudaStream_t s) {
    if constexpr (!std::is_same<C, float2>::value) {
        return false;
    } else {
#define TDDA_INV_CASE(a, b)                                                                  \
    if (g.Lz == a && g.Ly == b) {                                                            \
        launch_dep((k_inv_yz_fast<C, a, b, Epi>), grid, dim3(NT3), g.smem_yz2, s, g, T, tw, epi);           \
        return true;                                                                         \
    }
        TDDA_YZ_PAIRS(TDDA_INV_CASE)
#undef TDDA_INV_CASE
        return false;
    }
}

}  // namespace tdda
#include "slab_reg.cuh"
#include "slab_cluster.cuh"
namespace tdda {

template <typename C, class Epi>
__global__ void __launch_bounds__(NT) k_inv_yz(ConvGeom g, const C *__restrict__ T,
                                               const C *__restrict__ tw, Epi epi) {
    pdl_wait();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *A = reinterpret_cast<C *>(smem_raw);
    C *B = A + (size_t)g.ny * g.pA;
    const int x = blockIdx.x, c = blockIdx.y, rhs = blockIdx.z;
    if (epi.skip(rhs)) return;
    const C *Tc = T + ((size_t)(rhs * 3 + c) * g.nx + x) * (size_t)g.Ly * g.Lz;
    for (int kz0 = 0; kz0 < g.Lz; kz0 += g.CK) {
        for (int e = threadIdx.x; e < g.Ly * g.CK; e += NT) {
            int ky = e / g.CK, kl = e - ky * g.CK;
            B[ky * g.pB + kl] = Tc[(size_t)ky * g.Lz + kz0 + kl];
        }
        __syncthreads();
        fft_smem<+1, MAXI>(B, g.Ly, g.CK, g.pB, 1, tw, g.Lmax);
        for (int e = threadIdx.x; e < g.ny * g.CK; e += NT) {
            int y = e / g.CK, kl = e - y * g.CK;
            A[y * g.pA + kz0 + kl] = B[y * g.pB + kl];
        }
        __syncthreads();
    }
    for (int y0 = 0; y0 < g.ny; y0 += g.YC)
        fft_smem<+1, MAXI>(A + y0 * g.pA, g.Lz, min(g.YC, g.ny - y0), 1, g.pA, tw, g.Lmax);
    const int nyz = g.ny * g.nz;
    const long long cell0 = (long long)x * nyz;
    double2 acc[Epi::NQ > 0 ? Epi::NQ : 1];
#pragma unroll
    for (int q = 0; q < (Epi::NQ > 0 ? Epi::NQ : 1); ++q) acc[q] = make_double2(0.0, 0.0);
    for (int e = threadIdx.x; e < nyz; e += NT) {
        int y = e / g.nz, z = e - y * g.nz;
        epi.apply(rhs, c, cell0 + e, A[y * g.pA + z], acc);
    }
    if constexpr (Epi::NQ > 0) {
        reduce_finalize<Epi::NQ>(acc, epi.part + (size_t)rhs * epi.pstride, epi.counter + rhs,
                                 blockIdx.y * gridDim.x + blockIdx.x, gridDim.x * gridDim.y, epi, rhs);
    }
}

// ----------------------------------------------------------------------------
// prologues (what pass 1 transforms) and epilogues (what pass 3 produces)
// ----------------------------------------------------------------------------
// Optional diagonal (Jacobi) scaling: with sc = D^(-1/2) per cell the passes
// apply S A S + diag(alS) (alS = sc^2 al) instead of A + diag(al): pass 1
// scales what it transforms, pass 3 scales the convolution.  sc == nullptr is
// the unscaled operator of the reference.  The diagonal (al, sc) is shared by
// every right-hand side (dstride = 0) or held per right-hand side at
// [rhs][cell] (dstride = nbox): the polarisabilities of one structure differ
// between incident polarisations (src/Tools.cpp:353-366 depends on n_E0).
template <typename C> struct VecBase {
    long long nbox;
    const C *sc = nullptr;
    size_t dstride = 0;
    __device__ __forceinline__ size_t idx(int rhs, int c, long long cell) const {
        return ((size_t)rhs * 3 + c) * (size_t)nbox + (size_t)cell;
    }
    __device__ __forceinline__ size_t didx(int rhs, long long cell) const {
        return (size_t)rhs * dstride + (size_t)cell;
    }
    __device__ __forceinline__ C scaled(int rhs, long long cell, C v) const {
        return sc != nullptr ? __ldg(sc + didx(rhs, cell)) * v : v;
    }
};
// Operands that a pass only reads are loaded through the non-coherent path
// (__ldg): nothing the same kernel stores can alias them (every element is
// read and written by one thread), so the compiler may issue the loads of
// several elements ahead of the stores of earlier ones.

template <typename C> struct ProLoad : VecBase<C> {
    const C *x;
    const SolverState *st;  // optional
    __device__ bool skip(int rhs) const { return st != nullptr && st[rhs].done; }
    __device__ C load(int rhs, int c, long long cell) const {
        return this->scaled(rhs, cell, __ldg(x + this->idx(rhs, c, cell)));
    }
};

// p = r + beta (p - zeta Ap)   (first step: p = r)       src/DDAModel.cpp:929,972-973
template <typename C> struct ProP : VecBase<C> {
    const C *r;
    C *p;
    const C *Ap;
    const SolverState *st;
    int first;
    __device__ bool skip(int rhs) const { return st[rhs].done; }
    __device__ C load(int rhs, int c, long long cell) const {
        size_t i = this->idx(rhs, c, cell);
        C v = __ldg(r + i);
        if (!first) {
            C beta = from_d<C>(__ldg(&st[rhs].beta)), zeta = from_d<C>(__ldg(&st[rhs].zeta));
            v = v + beta * (__ldg(p + i) - zeta * __ldg(Ap + i));
        }
        p[i] = v;
        return this->scaled(rhs, cell, v);
    }
};

// t = r - alpha Ap                                          src/DDAModel.cpp:933,976
template <typename C> struct ProT : VecBase<C> {
    const C *r;
    const C *Ap;
    C *t;
    const SolverState *st;
    __device__ bool skip(int rhs) const { return st[rhs].done; }
    __device__ C load(int rhs, int c, long long cell) const {
        size_t i = this->idx(rhs, c, cell);
        C alpha = from_d<C>(__ldg(&st[rhs].alpha));
        C v = __ldg(r + i) - alpha * __ldg(Ap + i);
        t[i] = v;
        return this->scaled(rhs, cell, v);
    }
};

template <typename C> struct EpiBase : VecBase<C> {
    const unsigned char *mask;  // nullptr: every cell is a dipole
    double2 *part;
    unsigned *counter;
    size_t pstride;
    __device__ __forceinline__ C masked(int rhs, long long cell, C conv) const {
        if (mask != nullptr && __ldg(mask + cell) == 0) return czero<C>();
        return this->scaled(rhs, cell, conv);
    }
};

// y = conv (+ al o x)
template <typename C> struct EpiMatvec : EpiBase<C> {
    static constexpr int NQ = 0;
    C *y;
    const C *x;
    const C *al;  // per cell, or nullptr
    __device__ bool skip(int) const { return false; }
    __device__ void apply(int rhs, int c, long long cell, C conv, double2 *) const {
        size_t i = this->idx(rhs, c, cell);
        C v = this->masked(rhs, cell, conv);
        if (al != nullptr) v = v + __ldg(al + this->didx(rhs, cell)) * __ldg(x + i);
        y[i] = v;
    }
    __device__ void operator()(int, const double2 *) const {}
};

// One factor of the polynomial preconditioner of the GMRES solver (gmres.cuh):
// Ar = conv + al o r (the operator the passes apply), r' = r - c Ar, and
// y = c r (first) or y += c r when y is given; r' goes to rout (may alias rin:
// every element is read and written by one thread), or wout = v0 - r'.
template <typename C> struct EpiPoly : EpiBase<C> {
    static constexpr int NQ = 0;
    const C *rin, *al, *v0;
    C *rout, *y, *wout;
    double2 c;
    int first;
    __device__ bool skip(int) const { return false; }
    __device__ void apply(int rhs, int comp, long long cell, C conv, double2 *) const {
        const size_t i = this->idx(rhs, comp, cell);
        const C r = rin[i];
        const C Ar = this->masked(rhs, cell, conv) + __ldg(al + this->didx(rhs, cell)) * r;
        const C cc = from_d<C>(c);
        const C rn = r - cc * Ar;
        if (y != nullptr) y[i] = first ? cc * r : y[i] + cc * r;
        if (wout != nullptr) wout[i] = __ldg(v0 + i) - rn;
        else if (rout != nullptr) rout[i] = rn;
    }
    __device__ void operator()(int, const double2 *) const {}
};

// r = B - (A x0 + al o x0); r0 = r;  sums: r0.r, ||B||^2   src/DDAModel.cpp:925-928
template <typename C> struct EpiInit : EpiBase<C> {
    static constexpr int NQ = 3;
    const C *x0, *b, *al;
    C *r, *r0;
    SolverState *st;
    ResidualPost post;   // E_int and the objective sum of right-hand side 0 (off when post.eres is null)
    __device__ bool skip(int rhs) const { return false; }
    __device__ void apply(int rhs, int c, long long cell, C conv, double2 *acc) const {
        size_t i = this->idx(rhs, c, cell);
        const C alx = __ldg(al + this->didx(rhs, cell)) * __ldg(x0 + i);
        C ax = this->masked(rhs, cell, conv) + alx;
        C bb = __ldg(b + i);
        C v = bb - ax;
        r[i] = v;
        r0[i] = v;
        double2 vd = to_d(v), bd = to_d(bb);
        double2 d = cdot1(vd, vd);
        acc[0].x += d.x;
        acc[0].y += d.y;
        acc[1].x += bd.x * bd.x + bd.y * bd.y;
        if (post.eres != nullptr && rhs == 0) {
            const double2 a = to_d(alx);
            const double2 e = __ldg(post.diel + cell);
            post.eres[(size_t)c * this->nbox + cell] = cdiv(a, make_double2((2.0 + e.x) / 3.0, e.y / 3.0));
            if (post.mask == nullptr || __ldg(post.mask + cell) != 0) {
                const double m = hypot(a.x, a.y);
                acc[2].x += post.q == 2 ? m * m : pow(m, (double)post.q);
            }
        }
    }
    __device__ void operator()(int rhs, const double2 *s) const {
        SolverState &S = st[rhs];
        S.post_sum = s[2].x;
        S.rho = s[0];
        S.rho_prev = make_double2(0.0, 0.0);
        S.enorm = sqrt(s[1].x);
        S.err = S.enorm > 0 ? sqrt(s[0].x) / S.enorm : 0.0;
        S.it = -1;
        if (S.enorm == 0.0) {
            S.done = 1;
            S.status = TDDA_SOLVE_ZERO_RHS;
            S.iters = 0;
        }
    }
};

// Ap = conv + al o p;  sum r0.Ap -> alpha = rho / (r0.Ap)    src/DDAModel.cpp:931-932,974-975
template <typename C> struct EpiAp : EpiBase<C> {
    static constexpr int NQ = 1;
    const C *p, *al, *r0;
    C *Ap;
    SolverState *st;
    __device__ bool skip(int rhs) const { return st[rhs].done; }
    __device__ void apply(int rhs, int c, long long cell, C conv, double2 *acc) const {
        size_t i = this->idx(rhs, c, cell);
        C v = this->masked(rhs, cell, conv) + __ldg(al + this->didx(rhs, cell)) * __ldg(p + i);
        Ap[i] = v;
        double2 d = cdot1(to_d(__ldg(r0 + i)), to_d(v));
        acc[0].x += d.x;
        acc[0].y += d.y;
    }
    __device__ void operator()(int rhs, const double2 *s) const {
        SolverState &S = st[rhs];
        S.alpha = cdiv(S.rho, s[0]);
    }
};

// At = conv + al o t;  sums At.t, At.At -> zeta              src/DDAModel.cpp:935-936,977-979
template <typename C> struct EpiAt : EpiBase<C> {
    static constexpr int NQ = 2;
    const C *t, *al;
    C *At;
    SolverState *st;
    __device__ bool skip(int rhs) const { return st[rhs].done; }
    __device__ void apply(int rhs, int c, long long cell, C conv, double2 *acc) const {
        size_t i = this->idx(rhs, c, cell);
        C tv = __ldg(t + i);
        C v = this->masked(rhs, cell, conv) + __ldg(al + this->didx(rhs, cell)) * tv;
        At[i] = v;
        double2 vd = to_d(v);
        double2 d = cdot1(vd, to_d(tv));
        acc[0].x += d.x;
        acc[0].y += d.y;
        double2 d2 = cdot1(vd, vd);
        acc[1].x += d2.x;
        acc[1].y += d2.y;
    }
    __device__ void operator()(int rhs, const double2 *s) const {
        SolverState &S = st[rhs];
        S.zeta = cdiv(s[0], s[1]);
    }
};

// Finalize after the P/r update: bookkeeping of src/DDAModel.cpp:940-1008.
// Fused variant of the At epilogue: also r0.t, r0.At and ||t||^2, from which
// the finalize forms the next recursive residual without the update pass:
//   r = t - zeta At,  r0.r = r0.t - zeta r0.At,
//   ||r||^2 = ||t||^2 - 2 Re(conj(zeta) <At, t>) + |zeta|^2 ||At||^2
// (FP64 sums; the vectors r and P are formed by the next iteration's first
// pass, ProPF, or by k_flush after the last iteration).
template <typename C> struct EpiAtF : EpiBase<C> {
    static constexpr int NQ = 4;
    static_assert(NQ <= kMaxNQ, "reduction scratch holds kMaxNQ sums per block");
    const C *t, *al, *r0;
    C *At;
    SolverState *st;
    __device__ bool skip(int rhs) const { return st[rhs].done; }
    __device__ void apply(int rhs, int c, long long cell, C conv, double2 *acc) const {
        size_t i = this->idx(rhs, c, cell);
        const C tv = __ldg(t + i);
        const C v = this->masked(rhs, cell, conv) + __ldg(al + this->didx(rhs, cell)) * tv;
        At[i] = v;
        const double2 vd = to_d(v), td = to_d(tv), r0d = to_d(__ldg(r0 + i));
        const double2 d0 = cdot1(vd, td);
        acc[0].x += d0.x;
        acc[0].y += d0.y;
        acc[1].x += vd.x * vd.x + vd.y * vd.y;
        acc[1].y += td.x * td.x + td.y * td.y;
        const double2 d2 = cdot1(r0d, td), d3 = cdot1(r0d, vd);
        acc[2].x += d2.x;
        acc[2].y += d2.y;
        acc[3].x += d3.x;
        acc[3].y += d3.y;
    }
    __device__ void operator()(int rhs, const double2 *s) const;
};

// One loop pass's bookkeeping after the new r: stopping tests and beta.
__device__ __forceinline__ void finish_iteration(SolverState &S, double2 rho_new, double rnorm2) {
    {
        S.rho_prev = S.rho;
        S.rho = rho_new;
        S.err = sqrt(rnorm2) / S.enorm;
        const int it = S.it;
        if (S.stall_limit > 0 && it >= 0 && S.err < 0.9 * S.best_err) {
            S.best_err = S.err;
            S.best_it = it;
        }
        if (it >= 0 && S.err <= S.tol) {
            S.done = 1;
            S.status = TDDA_SOLVE_CONVERGED;
            S.iters = it + 1;
        } else if (!isfinite(S.err)) {
            S.done = 1;
            S.status = TDDA_SOLVE_NONFINITE;
            S.iters = it + 1;
        } else if (it + 1 >= S.max_iter) {
            S.done = 1;
            S.status = TDDA_SOLVE_MAXITER;
            S.iters = S.max_iter;
        } else if (S.stall_limit > 0 && it >= 0 && it - S.best_it >= S.stall_limit) {
            S.done = 1;
            S.status = TDDA_SOLVE_STAGNATED;
            S.iters = it + 1;
        } else if (dzero(S.rho_prev)) {
            S.done = 1;
            S.status = TDDA_SOLVE_BREAKDOWN;
            S.iters = it + 2;
        } else {
            // beta = (alpha / zeta) * (r0.r) / (r0.rl)
            double2 az = cdiv(S.alpha, S.zeta);
            double2 num = make_double2(az.x * S.rho.x - az.y * S.rho.y, az.x * S.rho.y + az.y * S.rho.x);
            S.beta = cdiv(num, S.rho_prev);
        }
        S.it = it + 1;
    }
}

struct FinUpdate {
    SolverState *st;
    __device__ void operator()(int rhs, const double2 *s) const { finish_iteration(st[rhs], s[0], s[1].x); }
};

template <typename C> __device__ void EpiAtF<C>::operator()(int rhs, const double2 *s) const {
    SolverState &S = st[rhs];
    const double2 atat = make_double2(s[1].x, 0.0);
    S.zeta = cdiv(s[0], atat);
    const double2 z = S.zeta;
    // Re(conj(zeta) <At,t>) and |zeta|^2
    const double re = z.x * s[0].x + z.y * s[0].y;
    const double z2 = z.x * z.x + z.y * z.y;
    const double rn2 = fmax(s[1].y - 2.0 * re + z2 * s[1].x, 0.0);
    const double2 rho_new = make_double2(s[2].x - (z.x * s[3].x - z.y * s[3].y),
                                         s[2].y - (z.x * s[3].y + z.y * s[3].x));
    S.pending = 1;
    finish_iteration(S, rho_new, rn2);
}

// Fused first pass: the previous iteration's r = t - zeta At and
// P += alpha p + zeta t, then p = r + beta (p - zeta Ap)  (first step: p = r)
template <typename C> struct ProPF : VecBase<C> {
    C *r, *P, *p;
    const C *t, *At, *Ap;
    const SolverState *st;
    int first;
    __device__ bool skip(int rhs) const { return st[rhs].done; }
    __device__ C load(int rhs, int c, long long cell) const {
        const size_t i = this->idx(rhs, c, cell);
        C v;
        if (first) {
            v = __ldg(r + i);
        } else {
            const C alpha = from_d<C>(__ldg(&st[rhs].alpha)), zeta = from_d<C>(__ldg(&st[rhs].zeta));
            const C beta = from_d<C>(__ldg(&st[rhs].beta));
            const C tv = __ldg(t + i), pv = __ldg(p + i);
            const C rn = tv - zeta * __ldg(At + i);
            r[i] = rn;
            P[i] = P[i] + alpha * pv + zeta * tv;
            v = rn + beta * (pv - zeta * __ldg(Ap + i));
        }
        p[i] = v;
        return this->scaled(rhs, cell, v);
    }
};

// After a fused solve: the last iteration's P += alpha p + zeta t
template <typename C>
__global__ void __launch_bounds__(NT) k_flush(long long n, C *__restrict__ P, const C *__restrict__ p,
                                              const C *__restrict__ t, const SolverState *st) {
    const int rhs = blockIdx.y;
    if (!st[rhs].pending) return;
    const C alpha = from_d<C>(st[rhs].alpha), zeta = from_d<C>(st[rhs].zeta);
    const size_t base = (size_t)rhs * n;
    for (long long i = (long long)blockIdx.x * NT + threadIdx.x; i < n; i += (long long)gridDim.x * NT) {
        const size_t k = base + i;
        P[k] = P[k] + alpha * __ldg(p + k) + zeta * __ldg(t + k);
    }
}

// P += alpha p + zeta t;  r = t - zeta At;  sums r0.r, ||r||^2
// (src/DDAModel.cpp:937-941,980-984, with alpha p + zeta r - alpha zeta Ap
//  regrouped as alpha p + zeta t, which is the same vector since t = r - alpha Ap)
template <typename C>
__global__ void __launch_bounds__(NT) k_update(long long n, C *__restrict__ P, const C *__restrict__ p,
                                               const C *__restrict__ t, const C *__restrict__ At,
                                               C *__restrict__ r, const C *__restrict__ r0,
                                               SolverState *st, double2 *part, unsigned *counter,
                                               size_t pstride) {
    pdl_wait();
    const int rhs = blockIdx.y;
    if (st[rhs].done) return;
    const C alpha = from_d<C>(st[rhs].alpha), zeta = from_d<C>(st[rhs].zeta);
    const size_t base = (size_t)rhs * n;
    double2 acc[2] = {make_double2(0.0, 0.0), make_double2(0.0, 0.0)};
    for (long long i = (long long)blockIdx.x * NT + threadIdx.x; i < n; i += (long long)gridDim.x * NT) {
        size_t k = base + i;
        C tv = __ldg(t + k);
        P[k] = P[k] + alpha * __ldg(p + k) + zeta * tv;
        C rn = tv - zeta * __ldg(At + k);
        r[k] = rn;
        double2 rd = to_d(rn);
        double2 d = cdot1(to_d(__ldg(r0 + k)), rd);
        acc[0].x += d.x;
        acc[0].y += d.y;
        acc[1].x += rd.x * rd.x + rd.y * rd.y;
    }
    FinUpdate fin{st};
    reduce_finalize<2>(acc, part + (size_t)rhs * pstride, counter + rhs, blockIdx.x, gridDim.x, fin, rhs);
}

// r = B, r0 = B, X = 0; sums r0.r, ||B||^2 (zero initial guess)
template <typename C>
__global__ void __launch_bounds__(NT) k_init_zero(long long n, const C *__restrict__ B, C *__restrict__ X,
                                                  C *__restrict__ r, C *__restrict__ r0,
                                                  SolverState *st, double2 *part, unsigned *counter,
                                                  size_t pstride) {
    const int rhs = blockIdx.y;
    const size_t base = (size_t)rhs * n;
    double2 acc[2] = {make_double2(0.0, 0.0), make_double2(0.0, 0.0)};
    for (long long i = (long long)blockIdx.x * NT + threadIdx.x; i < n; i += (long long)gridDim.x * NT) {
        size_t k = base + i;
        C b = B[k];
        r[k] = b;
        r0[k] = b;
        X[k] = czero<C>();
        double2 bd = to_d(b);
        double2 d = cdot1(bd, bd);
        acc[0].x += d.x;
        acc[0].y += d.y;
        acc[1].x += bd.x * bd.x + bd.y * bd.y;
    }
    EpiInit<C> fin{};
    fin.st = st;
    reduce_finalize<2>(acc, part + (size_t)rhs * pstride, counter + rhs, blockIdx.x, gridDim.x, fin, rhs);
}

// The device-driven iteration loop (a CUDA graph whose while-node repeats the
// BiCGSTAB iterations): the start kernel zeroes the pass counter and records
// the start time; the condition kernel, last in the loop body, keeps the loop
// going while some right-hand side runs.  Past `cap` passes or `limit_ns`
// nanoseconds the running right-hand sides end (MAXITER / TIMEOUT), so the
// loop ends after at most `cap` passes whatever the states hold.
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__global__ void k_loop_start(unsigned long long *loop) {
    if (threadIdx.x == 0) {
        loop[0] = 0;
        loop[1] = global_ns();
    }
}

__global__ void k_loop_cond(cudaGraphConditionalHandle h, SolverState *st, int nrhs, unsigned long long *loop,
                            unsigned long long cap, unsigned long long limit_ns) {
    if (threadIdx.x != 0) return;
    const unsigned long long c = ++loop[0];
    const bool over_time = limit_ns > 0 && global_ns() - loop[1] > limit_ns;
    const bool over_cap = c >= cap;
    int running = 0;
    for (int k = 0; k < nrhs; ++k) {
        if (st[k].done) continue;
        if (over_time) {
            st[k].done = 1;
            st[k].status = TDDA_SOLVE_TIMEOUT;
        } else if (over_cap) {
            st[k].done = 1;
            st[k].status = TDDA_SOLVE_MAXITER;
        } else {
            running = 1;
        }
    }
    cudaGraphSetConditional(h, running ? 1u : 0u);
}

// ----------------------------------------------------------------------------
// host side
// ----------------------------------------------------------------------------
static int gcd_i(int a, int b) { while (b) { int t = a % b; a = b; b = t; } return a; }
static int lcm_i(int a, int b) { return a / gcd_i(a, b) * b; }

int next_fft_len(int minlen) {
    if (minlen <= 1) return 1;
    int best = 1 << 30;
    for (long long p2 = 1; p2 < (1LL << 30); p2 *= 2)
        for (long long p3 = 1; p2 * p3 < (1LL << 30); p3 *= 3) {
            long long v = p2 * p3;
            if (v >= minlen && v < best) best = (int)v;
        }
    return best;
}

template <typename C> static void set_smem_attrs(int yz, int x) {
    // the opt-in dynamic shared memory limit is a per-function attribute
    cudaFuncSetAttribute(k_fwd_zy<C, ProLoad<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, yz);
    cudaFuncSetAttribute(k_fwd_zy<C, ProP<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, yz);
    cudaFuncSetAttribute(k_fwd_zy<C, ProT<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, yz);
    cudaFuncSetAttribute(k_fwd_zy<C, ProPF<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, yz);
    cudaFuncSetAttribute(k_inv_yz<C, EpiAtF<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, yz);
    cudaFuncSetAttribute(k_inv_yz<C, EpiMatvec<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, yz);
    cudaFuncSetAttribute(k_inv_yz<C, EpiPoly<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, yz);
    cudaFuncSetAttribute(k_inv_yz<C, EpiInit<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, yz);
    cudaFuncSetAttribute(k_inv_yz<C, EpiAp<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, yz);
    cudaFuncSetAttribute(k_inv_yz<C, EpiAt<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, yz);
    cudaFuncSetAttribute(k_xconv<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, x);
    cudaFuncSetAttribute(k_xconv_fast<C, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize, x);
    cudaFuncSetAttribute(k_xconv_fast<C, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize, x);
    cudaFuncSetAttribute(k_xconv_fast<C, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize, x);
    cudaFuncSetAttribute(k_xconv_fast<C, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, x);
    cudaFuncSetAttribute(k_xconv_fast<C, 192>, cudaFuncAttributeMaxDynamicSharedMemorySize, x);
    cudaFuncSetAttribute(k_xconv_fast<C, 96>, cudaFuncAttributeMaxDynamicSharedMemorySize, x);
    cudaFuncSetAttribute(k_xconv_reg<C, 256, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, x);
    cudaFuncSetAttribute(k_xconv_reg<C, 192, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, x);
    cudaFuncSetAttribute(k_xconv_reg<C, 128, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, x);
    cudaFuncSetAttribute(k_xconv_reg<C, 96, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, x);
    cudaFuncSetAttribute(k_xconv_reg<C, 64, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, x);
    if constexpr (sizeof(C) == 16) {
        cudaFuncSetAttribute(k_xconv_reg<C, 256, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, x);
        cudaFuncSetAttribute(k_xconv_reg<C, 192, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, x);
        cudaFuncSetAttribute(k_xconv_reg<C, 128, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, x);
        cudaFuncSetAttribute(k_xconv_reg<C, 96, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, x);
        cudaFuncSetAttribute(k_xconv_reg<C, 64, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, x);
    }
    if constexpr (std::is_same<C, float2>::value) {
        // dynamic + static shared memory must stay within the 227 KB opt-in limit;
        // the epilogue kernels carry ~1 KB of static reduction scratch
#define TDDA_ATTR(a, b)                                                                                            \
    cudaFuncSetAttribute(k_fwd_zy_fast<C, a, b, ProLoad<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemFast);   \
    cudaFuncSetAttribute(k_fwd_zy_fast<C, a, b, ProP<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemFast);      \
    cudaFuncSetAttribute(k_fwd_zy_fast<C, a, b, ProT<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemFast);      \
    cudaFuncSetAttribute(k_fwd_zy_fast<C, a, b, ProPF<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemFast);     \
    cudaFuncSetAttribute(k_inv_yz_fast<C, a, b, EpiAtF<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemFast);    \
    cudaFuncSetAttribute(k_inv_yz_fast<C, a, b, EpiMatvec<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemFast); \
    cudaFuncSetAttribute(k_inv_yz_fast<C, a, b, EpiPoly<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemFast);   \
    cudaFuncSetAttribute(k_inv_yz_fast<C, a, b, EpiInit<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemFast);   \
    cudaFuncSetAttribute(k_inv_yz_fast<C, a, b, EpiAp<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemFast);     \
    cudaFuncSetAttribute(k_inv_yz_fast<C, a, b, EpiAt<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemFast);
        TDDA_YZ_PAIRS(TDDA_ATTR)
#undef TDDA_ATTR
#define TDDA_ATTR_REG(a, b)                                                                                          \
    cudaFuncSetAttribute(k_fwd_zy_reg<C, a, b, ProLoad<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemFast);    \
    cudaFuncSetAttribute(k_fwd_zy_reg<C, a, b, ProP<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemFast);       \
    cudaFuncSetAttribute(k_fwd_zy_reg<C, a, b, ProT<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemFast);       \
    cudaFuncSetAttribute(k_fwd_zy_reg<C, a, b, ProPF<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemFast);      \
    cudaFuncSetAttribute(k_inv_yz_reg<C, a, b, EpiAtF<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemFast);     \
    cudaFuncSetAttribute(k_inv_yz_reg<C, a, b, EpiMatvec<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemFast);  \
    cudaFuncSetAttribute(k_inv_yz_reg<C, a, b, EpiPoly<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemFast);    \
    cudaFuncSetAttribute(k_inv_yz_reg<C, a, b, EpiInit<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemFast);    \
    cudaFuncSetAttribute(k_inv_yz_reg<C, a, b, EpiAp<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemFast);      \
    cudaFuncSetAttribute(k_inv_yz_reg<C, a, b, EpiAt<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemFast);
        TDDA_YZ_REG_PAIRS(TDDA_ATTR_REG)
#undef TDDA_ATTR_REG
    }
    if constexpr (sizeof(C) == 16) {
#define TDDA_ATTR_CL(a, b)                                                                                           \
    cudaFuncSetAttribute(k_fwd_zy_cl<C, a, b, ProLoad<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, ClGeom<a, b>::SMEM); \
    cudaFuncSetAttribute(k_fwd_zy_cl<C, a, b, ProP<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, ClGeom<a, b>::SMEM);    \
    cudaFuncSetAttribute(k_fwd_zy_cl<C, a, b, ProT<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, ClGeom<a, b>::SMEM);    \
    cudaFuncSetAttribute(k_fwd_zy_cl<C, a, b, ProPF<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, ClGeom<a, b>::SMEM);   \
    cudaFuncSetAttribute(k_inv_yz_cl<C, a, b, EpiAtF<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, ClGeom<a, b>::SMEM);  \
    cudaFuncSetAttribute(k_inv_yz_cl<C, a, b, EpiMatvec<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, ClGeom<a, b>::SMEM); \
    cudaFuncSetAttribute(k_inv_yz_cl<C, a, b, EpiPoly<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, ClGeom<a, b>::SMEM); \
    cudaFuncSetAttribute(k_inv_yz_cl<C, a, b, EpiInit<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, ClGeom<a, b>::SMEM); \
    cudaFuncSetAttribute(k_inv_yz_cl<C, a, b, EpiAp<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, ClGeom<a, b>::SMEM);   \
    cudaFuncSetAttribute(k_inv_yz_cl<C, a, b, EpiAt<C>>, cudaFuncAttributeMaxDynamicSharedMemorySize, ClGeom<a, b>::SMEM);
        TDDA_YZ_CL_PAIRS(TDDA_ATTR_CL)
#undef TDDA_ATTR_CL
    }
    cudaGetLastError();  // a refused opt-in shows up at launch time, not here
}

static bool plan_geom(int nx, int ny, int nz, int nrhs, int esize, ConvGeom &g, std::string &why) {
    g.nx = nx; g.ny = ny; g.nz = nz;
    g.Lx = next_fft_len(2 * nx - 1);
    g.Ly = next_fft_len(2 * ny - 1);
    g.Lz = next_fft_len(2 * nz - 1);
    g.hx = g.Lx / 2 + 1; g.hy = g.Ly / 2 + 1; g.hz = g.Lz / 2 + 1;
    g.Lmax = lcm_i(lcm_i(g.Lx, g.Ly), g.Lz);
    g.nbox = (long long)nx * ny * nz;
    g.tcomp = (long long)nx * g.Ly * g.Lz;
    g.nrhs = nrhs;
    g.pA = (g.Lz % 2 == 0) ? g.Lz + 1 : g.Lz;
    // z transforms of the slab in chunks of YC columns (as many as fit the block)
    g.YC = ny;
    while (g.YC > 1 && fft_max_items(g.Lz, g.YC, NT) > MAXI) g.YC = (g.YC + 1) / 2;
    if (fft_max_items(g.Lz, g.YC, NT) > MAXI) { why = "Lz too large for the z transform"; return false; }
    g.CK = 0;
    for (int ck = g.Lz; ck >= 1; --ck) {
        if (g.Lz % ck) continue;
        long long bytes = ((long long)ny * g.pA + (long long)g.Ly * ck) * esize;
        if (bytes > SMEM_MAX) continue;
        if (fft_max_items(g.Ly, ck, NT) > MAXI) continue;
        g.CK = ck;
        break;
    }
    if (g.CK == 0) { why = "slab does not fit in shared memory"; return false; }
    g.pB = g.CK;
    g.smem_yz = (int)(((long long)ny * g.pA + (long long)g.Ly * g.CK) * esize);
    const int ckcap = esize == 16 ? 8 : 16;
    g.CKx = 0;
    for (int ck = std::min(g.Lz, ckcap); ck >= 1; --ck) {
        if (g.Lz % ck) continue;
        int nbat = nrhs * 3 * ck;
        long long bytes = (long long)g.Lx * nbat * esize;
        if (bytes > SMEM_MAX) continue;
        if (fft_max_items(g.Lx, nbat, NT) > MAXI) continue;
        g.CKx = ck;
        break;
    }
    // (CKx == 0: the generic x pass cannot hold this batch; a compile-time
    // x pass below may still take it)
    g.pC = nrhs * 3 * g.CKx;
    g.smem_x = g.Lx * g.pC * esize;
    // compile-time slab kernels for passes 1 and 3 (complex64 only)
    g.smem_yz2 = (int)((long long)g.Ly * (g.Lz + 1) * esize);
    g.fast_yz = (esize == 8 && fast_yz_pair(g.Lz, g.Ly) && g.smem_yz2 <= kSmemFast) ? 1 : 0;
    // register two-level slab kernels: half padding on both axes
    g.reg_yz = 0;
    if (esize == 8 && 2 * ny == g.Ly && 2 * nz == g.Lz && reg_yz_pair(g.Lz, g.Ly)) {
        g.smem_fr = slab_reg_smem(ny, g.Lz, g.Ly, true, esize);
        g.smem_ir = slab_reg_smem(ny, g.Lz, g.Ly, false, esize);
        g.reg_yz = (g.smem_fr <= kSmemFast && g.smem_ir <= kSmemFast) ? 1 : 0;
    }
    // complex128: the slab split over a two-CTA cluster
    g.cl_yz = (esize == 16 && 2 * ny == g.Ly && 2 * nz == g.Lz && cl_yz_pair(g.Lz, g.Ly) &&
               cl_smem(g.Lz, g.Ly) <= kSmemFast) ? 1 : 0;
    // compile-time-length pass 2: two ping-pong buffers, at most ~100 KB so
    // that two CTAs share an SM; runs of >= 64 bytes along kz
    g.fast_x = fast_x_length(g.Lx) ? 1 : 0;
    g.CKx2 = 0;
    for (int ck = std::min(g.Lz, esize == 16 ? 4 : 8); ck >= 1 && g.fast_x; --ck) {
        if (g.Lz % ck) continue;
        long long bytes = 2LL * g.Lx * nrhs * 3 * ck * esize;
        if (bytes > 100 * 1024 && ck > 1) continue;
        g.CKx2 = ck;
        g.smem_x2 = (int)bytes;
        break;
    }
    if (g.CKx2 == 0 || g.smem_x2 > SMEM_MAX) g.fast_x = 0;
    // register-resident pass 2: one task per thread at every step.  In
    // complex128 ky is paired with its mirror where a kz chunk of at least 2
    // fits the CTA that way (B200, 128x128x32: 144.0 -> 138.6 us); in complex64
    // the halved kz chunk and the extra registers cost more than the tensor
    // reuse gains (67.0 -> 71.2 us), so it stays unpaired.
    g.reg_x = 0;
    g.CKr = 0;
    g.pair_x = 0;
    if (reg_x_length(g.Lx) && 2 * nx == g.Lx) {
        const int R1 = g.Lx / 8;
        for (int pair = (esize == 16) ? 1 : 0; pair >= 0 && !g.reg_x; --pair) {
            const int nky = pair ? 2 : 1;
            for (int ck = g.Lz; ck >= (pair ? 2 : 1); --ck) {
                if (g.Lz % ck) continue;
                const int ncol = nky * nrhs * 3 * ck;
                const long long bytes = (long long)g.Lx * (ncol | 1) * esize;
                if (nky * nrhs * ck * R1 > NTR || ncol * 8 > NTR || bytes > SMEM_MAX) continue;
                g.CKr = ck;
                g.smem_r = (int)bytes;
                g.reg_x = 1;
                g.pair_x = pair;
                break;
            }
        }
    }
    if (g.CKx == 0 && !g.fast_x && !g.reg_x) { why = "x pencils do not fit in shared memory"; return false; }
    return true;
}

template <typename C> tdda_status ConvOperator<C>::init(int nx, int ny, int nz, int nrhs_cap_) {
    nrhs_cap = nrhs_cap_;
    set_smem_attrs<C>(SMEM_MAX, SMEM_MAX);
    std::string why;
    if (!plan_geom(nx, ny, nz, 1, (int)sizeof(C), g, why)) {
        set_error("unsupported grid " + std::to_string(nx) + "x" + std::to_string(ny) + "x" +
                  std::to_string(nz) + ": " + why);
        return TDDA_ERR_UNSUPPORTED;
    }
    // twiddles in double, rounded once to C
    std::vector<C> h(g.Lmax);
    for (int j = 0; j < g.Lmax; ++j) {
        long double ang = -2.0L * 3.141592653589793238462643383279502884L * (long double)j / g.Lmax;
        h[j] = from_d<C>(make_double2((double)cosl(ang), (double)sinl(ang)));
    }
    TDDA_CUDA_TRY(cudaMalloc(&tw, sizeof(C) * g.Lmax));
    TDDA_CUDA_TRY(cudaMemcpy(tw, h.data(), sizeof(C) * g.Lmax, cudaMemcpyHostToDevice));
    TDDA_CUDA_TRY(cudaMalloc(&T, sizeof(C) * (size_t)nrhs_cap * 3 * g.tcomp));
    partial_cap = std::max(6 * nx, UPD_BLOCKS) * kMaxNQ;
    TDDA_CUDA_TRY(cudaMalloc(&partials, sizeof(double2) * (size_t)partial_cap * nrhs_cap));
    TDDA_CUDA_TRY(cudaMalloc(&counters, sizeof(unsigned) * (size_t)nrhs_cap));
    TDDA_CUDA_TRY(cudaMemset(counters, 0, sizeof(unsigned) * (size_t)nrhs_cap));
    return TDDA_OK;
}

size_t conv_workspace_bytes(int nx, int ny, int nz, int nrhs_cap, int esize) {
    ConvGeom g;
    std::string why;
    if (!plan_geom(nx, ny, nz, 1, esize, g, why)) return 0;
    const size_t partial_cap = (size_t)std::max(6 * nx, UPD_BLOCKS) * kMaxNQ;
    return (size_t)esize * g.Lmax + (size_t)esize * nrhs_cap * 3 * g.tcomp + sizeof(double2) * partial_cap * nrhs_cap +
           sizeof(unsigned) * nrhs_cap;
}

bool conv_supported(int nx, int ny, int nz, int nrhs, int esize, std::string &why) {
    ConvGeom g;
    return plan_geom(nx, ny, nz, nrhs, esize, g, why);
}

template <typename C> void ConvOperator<C>::release() {
    cudaFree(ahat); cudaFree(tw); cudaFree(T); cudaFree(partials); cudaFree(counters);
    ahat = nullptr; tw = nullptr; T = nullptr; partials = nullptr; counters = nullptr;
}

template <typename C> static bool geom_for(const ConvOperator<C> &op, int nrhs, ConvGeom &g) {
    std::string why;
    if (nrhs == op.g.nrhs) { g = op.g; return true; }
    return plan_geom(op.g.nx, op.g.ny, op.g.nz, nrhs, (int)sizeof(C), g, why);
}

template <typename C, class Pro, class Epi>
static tdda_status run_conv(ConvOperator<C> &op, const ConvGeom &g, int nrhs, const Pro &pro,
                            const Epi &epi, const SolverState *st, cudaStream_t s) {
    dim3 g13(g.nx, 3, nrhs);
    count_launches(1);
    if (!launch_fwd_reg<C, Pro>(g, g13, op.T, op.tw, pro, s) && !launch_fwd_cl<C, Pro>(g, g13, op.T, op.tw, pro, s) &&
        !(g.fast_yz && launch_fwd_fast<C, Pro>(g, g13, op.T, op.tw, pro, s)))
        launch_dep((k_fwd_zy<C, Pro>), g13, dim3(NT), g.smem_yz, s, g, op.T, op.tw, pro);
    dim3 g2(g.Ly, g.CKx > 0 ? g.Lz / g.CKx : 1, 1);
    count_launches(1);
    if (!launch_xconv_reg<C>(g, op.T, op.ahat, op.ahat_rhs, op.tw, nrhs, st, s) &&
        !(g.fast_x && launch_xconv_fast<C>(g, op.T, op.ahat, op.ahat_rhs, op.tw, nrhs, st, s)))
        launch_dep(k_xconv<C>, g2, dim3(NT), g.smem_x, s, g, op.T, op.ahat, op.ahat_rhs, op.tw, nrhs, st);
    count_launches(1);
    if (!launch_inv_reg<C, Epi>(g, g13, op.T, op.tw, epi, s) && !launch_inv_cl<C, Epi>(g, g13, op.T, op.tw, epi, s) &&
        !(g.fast_yz && launch_inv_fast<C, Epi>(g, g13, op.T, op.tw, epi, s)))
        launch_dep((k_inv_yz<C, Epi>), g13, dim3(NT), g.smem_yz, s, g, op.T, op.tw, epi);
    return TDDA_OK;
}

template <typename C>
tdda_status ConvOperator<C>::apply(const C *x, C *y, const C *al, int nrhs, cudaStream_t s) {
    if (nrhs > nrhs_cap) { set_error("nrhs exceeds operator capacity"); return TDDA_ERR_BAD_ARG; }
    ConvGeom gg;
    if (!geom_for(*this, nrhs, gg)) { set_error("batch does not fit the x pass"); return TDDA_ERR_UNSUPPORTED; }
    ProLoad<C> pro{};
    pro.nbox = g.nbox; pro.x = x; pro.st = nullptr;
    EpiMatvec<C> epi{};
    epi.nbox = g.nbox; epi.mask = mask; epi.y = y; epi.x = x; epi.al = al;
    run_conv(*this, gg, nrhs, pro, epi, nullptr, s);
    TDDA_CUDA_TRY(cudaGetLastError());
    return TDDA_OK;
}

template <typename C>
tdda_status apply_scaled(ConvOperator<C> &op, const C *sc, const C *al, const C *x, C *y, int nrhs, size_t dstride,
                         cudaStream_t s) {
    if (nrhs > op.nrhs_cap) { set_error("nrhs exceeds operator capacity"); return TDDA_ERR_BAD_ARG; }
    ConvGeom gg;
    if (!geom_for(op, nrhs, gg)) { set_error("batch does not fit the x pass"); return TDDA_ERR_UNSUPPORTED; }
    ProLoad<C> pro{};
    pro.nbox = op.g.nbox; pro.x = x; pro.st = nullptr; pro.sc = sc; pro.dstride = dstride;
    EpiMatvec<C> epi{};
    epi.nbox = op.g.nbox; epi.mask = op.mask; epi.y = y; epi.x = x; epi.al = al; epi.sc = sc; epi.dstride = dstride;
    run_conv(op, gg, nrhs, pro, epi, nullptr, s);
    TDDA_CUDA_TRY(cudaGetLastError());
    return TDDA_OK;
}

template <typename C>
tdda_status poly_factor(ConvOperator<C> &op, const C *sc, const C *al, const C *rin, C *rout, C *y, bool first,
                        const C *v0, C *wout, double2 c, int nrhs, size_t dstride, cudaStream_t s) {
    if (nrhs > op.nrhs_cap) { set_error("nrhs exceeds operator capacity"); return TDDA_ERR_BAD_ARG; }
    ConvGeom gg;
    if (!geom_for(op, nrhs, gg)) { set_error("batch does not fit the x pass"); return TDDA_ERR_UNSUPPORTED; }
    ProLoad<C> pro{};
    pro.nbox = op.g.nbox; pro.x = rin; pro.st = nullptr; pro.sc = sc; pro.dstride = dstride;
    EpiPoly<C> epi{};
    epi.nbox = op.g.nbox; epi.mask = op.mask; epi.sc = sc; epi.dstride = dstride;
    epi.rin = rin; epi.al = al; epi.v0 = v0; epi.rout = rout; epi.y = y; epi.wout = wout; epi.c = c;
    epi.first = first ? 1 : 0;
    run_conv(op, gg, nrhs, pro, epi, nullptr, s);
    TDDA_CUDA_TRY(cudaGetLastError());
    return TDDA_OK;
}

template tdda_status apply_scaled<float2>(ConvOperator<float2> &, const float2 *, const float2 *, const float2 *,
                                          float2 *, int, size_t, cudaStream_t);
template tdda_status apply_scaled<double2>(ConvOperator<double2> &, const double2 *, const double2 *,
                                           const double2 *, double2 *, int, size_t, cudaStream_t);
template tdda_status poly_factor<float2>(ConvOperator<float2> &, const float2 *, const float2 *, const float2 *,
                                         float2 *, float2 *, bool, const float2 *, float2 *, double2, int, size_t,
                                         cudaStream_t);
template tdda_status poly_factor<double2>(ConvOperator<double2> &, const double2 *, const double2 *,
                                          const double2 *, double2 *, double2 *, bool, const double2 *, double2 *,
                                          double2, int, size_t, cudaStream_t);

template <typename C>
tdda_status apply_external_scratch(const ConvOperator<C> &op, C *T_ext, const C *x, C *y, const C *al,
                                   cudaStream_t s) {
    ConvOperator<C> view = op;  // same tensor, twiddles and plan; only the intermediate moves
    view.T = T_ext;
    ProLoad<C> pro{};
    pro.nbox = op.g.nbox; pro.x = x; pro.st = nullptr;
    EpiMatvec<C> epi{};
    epi.nbox = op.g.nbox; epi.mask = op.mask; epi.y = y; epi.x = x; epi.al = al;
    run_conv(view, op.g, 1, pro, epi, nullptr, s);
    TDDA_CUDA_TRY(cudaGetLastError());
    return TDDA_OK;
}

template tdda_status apply_external_scratch<double2>(const ConvOperator<double2> &, double2 *, const double2 *,
                                                     double2 *, const double2 *, cudaStream_t);

template <typename C> tdda_status Krylov<C>::init(long long n3, int nrhs_) {
    nrhs = nrhs_;
    n = n3;
    size_t bytes = sizeof(C) * (size_t)n * nrhs;
    C **bufs[6] = {&r, &r0, &p, &t, &Ap, &At};
    for (auto b : bufs) TDDA_CUDA_TRY(cudaMalloc(b, bytes));
    TDDA_CUDA_TRY(cudaMalloc(&st, sizeof(SolverState) * nrhs));
    TDDA_CUDA_TRY(cudaMallocHost(&st_host, sizeof(SolverState) * nrhs));
    TDDA_CUDA_TRY(cudaMalloc(&loop, sizeof(unsigned long long) * 4));
    return TDDA_OK;
}

template <typename C> void Krylov<C>::release() {
    C *bufs[6] = {r, r0, p, t, Ap, At};
    for (auto b : bufs) cudaFree(b);
    cudaFree(st);
    cudaFreeHost(st_host);
    cudaFree(loop);
    r = r0 = p = t = Ap = At = nullptr;
    st = nullptr;
    st_host = nullptr;
    loop = nullptr;
}

template <typename C>
tdda_status bicgstab_device(ConvOperator<C> &op, Krylov<C> &kv, const C *al, const C *sc, const C *B, C *X,
                            int nrhs, bool x0_zero, int max_iter, double tol, cudaStream_t s,
                            tdda_solve_info *info, const KrylovOptions &o) {
    if (nrhs > kv.nrhs || nrhs > op.nrhs_cap) { set_error("nrhs exceeds workspace"); return TDDA_ERR_BAD_ARG; }
    ConvGeom g;
    if (!geom_for(op, nrhs, g)) { set_error("batch does not fit the x pass"); return TDDA_ERR_UNSUPPORTED; }
    const long long n = 3 * g.nbox;
    for (int k = 0; k < nrhs; ++k) {
        SolverState &S = kv.st_host[k];
        std::memset(&S, 0, sizeof(S));
        S.it = -1;
        S.max_iter = max_iter;
        S.tol = o.tols != nullptr ? o.tols[k] : tol;
        S.stall_limit = o.stall_limit;
        S.best_it = 0;
        S.best_err = 1e300;
        S.status = TDDA_SOLVE_RUNNING;
    }
    TDDA_CUDA_TRY(cudaMemcpyAsync(kv.st, kv.st_host, sizeof(SolverState) * nrhs, cudaMemcpyHostToDevice, s));
    const size_t ps = (size_t)op.partial_cap;
    if (x0_zero) {
        dim3 gi(UPD_BLOCKS, nrhs);
        count_launches(1);
        k_init_zero<C><<<gi, NT, 0, s>>>(n, B, X, kv.r, kv.r0, kv.st, op.partials, op.counters, ps);
    } else {
        ProLoad<C> pro{};
        pro.nbox = g.nbox; pro.x = X; pro.st = nullptr; pro.sc = sc; pro.dstride = o.dstride;
        EpiInit<C> epi{};
        epi.nbox = g.nbox; epi.mask = op.mask; epi.part = op.partials; epi.counter = op.counters;
        epi.pstride = ps; epi.x0 = X; epi.b = B; epi.al = al; epi.r = kv.r; epi.r0 = kv.r0; epi.st = kv.st;
        epi.sc = sc; epi.dstride = o.dstride;
        run_conv(op, g, nrhs, pro, epi, nullptr, s);
    }
    TDDA_CUDA_TRY(cudaGetLastError());

    // one BiCGSTAB step: Ap, alpha, t, At, zeta, P/r update, beta (7 launches;
    // 6 fused, the P/r update riding in the next step's first pass)
    const int kLaunchesPerStep = o.fused ? 6 : 7;
    auto step_fused = [&](bool first) {
        ProPF<C> pp{};
        pp.nbox = g.nbox; pp.r = kv.r; pp.P = X; pp.p = kv.p; pp.t = kv.t; pp.At = kv.At; pp.Ap = kv.Ap;
        pp.st = kv.st; pp.first = first ? 1 : 0; pp.sc = sc; pp.dstride = o.dstride;
        EpiAp<C> ea{};
        ea.nbox = g.nbox; ea.mask = op.mask; ea.part = op.partials; ea.counter = op.counters; ea.pstride = ps;
        ea.p = kv.p; ea.al = al; ea.r0 = kv.r0; ea.Ap = kv.Ap; ea.st = kv.st;
        ea.sc = sc; ea.dstride = o.dstride;
        run_conv(op, g, nrhs, pp, ea, kv.st, s);
        ProT<C> pt{};
        pt.nbox = g.nbox; pt.r = kv.r; pt.Ap = kv.Ap; pt.t = kv.t; pt.st = kv.st;
        pt.sc = sc; pt.dstride = o.dstride;
        EpiAtF<C> et{};
        et.nbox = g.nbox; et.mask = op.mask; et.part = op.partials; et.counter = op.counters; et.pstride = ps;
        et.t = kv.t; et.al = al; et.r0 = kv.r0; et.At = kv.At; et.st = kv.st;
        et.sc = sc; et.dstride = o.dstride;
        run_conv(op, g, nrhs, pt, et, kv.st, s);
    };
    auto step = [&](bool first) {
        if (o.fused) {
            step_fused(first);
            return;
        }
        ProP<C> pp{};
        pp.nbox = g.nbox; pp.r = kv.r; pp.p = kv.p; pp.Ap = kv.Ap; pp.st = kv.st; pp.first = first ? 1 : 0;
        pp.sc = sc; pp.dstride = o.dstride;
        EpiAp<C> ea{};
        ea.nbox = g.nbox; ea.mask = op.mask; ea.part = op.partials; ea.counter = op.counters; ea.pstride = ps;
        ea.p = kv.p; ea.al = al; ea.r0 = kv.r0; ea.Ap = kv.Ap; ea.st = kv.st;
        ea.sc = sc; ea.dstride = o.dstride;
        run_conv(op, g, nrhs, pp, ea, kv.st, s);
        ProT<C> pt{};
        pt.nbox = g.nbox; pt.r = kv.r; pt.Ap = kv.Ap; pt.t = kv.t; pt.st = kv.st;
        pt.sc = sc; pt.dstride = o.dstride;
        EpiAt<C> et{};
        et.nbox = g.nbox; et.mask = op.mask; et.part = op.partials; et.counter = op.counters; et.pstride = ps;
        et.t = kv.t; et.al = al; et.At = kv.At; et.st = kv.st;
        et.sc = sc; et.dstride = o.dstride;
        run_conv(op, g, nrhs, pt, et, kv.st, s);
        dim3 gu(UPD_BLOCKS, nrhs);
        count_launches(1);
        launch_dep(k_update<C>, gu, dim3(NT), 0, s, n, X, kv.p, kv.t, kv.At, kv.r, kv.r0, kv.st, op.partials, op.counters, ps);
    };

    // Optional CUDA graph of graph_steps consecutive iterations, replayed
    // between polls: every launch reads its scalars from the device states and
    // returns at once for a finished right-hand side, so a replay past
    // convergence is harmless.
    cudaGraphExec_t exec = nullptr;
    struct GraphGuard {
        cudaGraphExec_t *e;
        ~GraphGuard() { if (*e) cudaGraphExecDestroy(*e); }
    } guard{&exec};
    auto capture = [&]() -> tdda_status {
        cudaGraph_t graph = nullptr;
        set_capturing(true);
        cudaError_t err = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
        if (err == cudaSuccess) {
            for (int k = 0; k < o.graph_steps; ++k) step(false);
            err = cudaStreamEndCapture(s, &graph);
        }
        set_capturing(false);
        if (err == cudaSuccess) err = cudaGraphInstantiate(&exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (err != cudaSuccess) {
            set_error(std::string("graph capture: ") + cudaGetErrorString(err));
            return TDDA_ERR_CUDA;
        }
        return TDDA_OK;
    };

    // One launch for the whole solve: the first step (p = r) directly, then a
    // graph whose while-node repeats graph_steps iterations and the condition
    // kernel until every right-hand side is done or the pass cap / time limit
    // ends it.  Falls back to host-polled chunks when conditional nodes are
    // unavailable.
    if (o.graph_steps > 0 && o.device_loop && kv.loop != nullptr) {
        step(true);
        count_launches(1);
        k_loop_start<<<1, 32, 0, s>>>(kv.loop);
        cudaGraph_t graph = nullptr;
        cudaGraphConditionalHandle handle;
        bool ok = cudaGraphCreate(&graph, 0) == cudaSuccess &&
                  cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault) == cudaSuccess;
        cudaGraphNodeParams np = {};
        cudaGraphNode_t node;
        if (ok) {
            np.type = cudaGraphNodeTypeConditional;
            np.conditional.handle = handle;
            np.conditional.type = cudaGraphCondTypeWhile;
            np.conditional.size = 1;
            ok = cudaGraphAddNode(&node, graph, nullptr, 0, &np) == cudaSuccess;
        }
        if (ok) {
            cudaGraph_t body = np.conditional.phGraph_out[0];
            const unsigned long long cap = (unsigned long long)max_iter / o.graph_steps + 2;
            const unsigned long long limit_ns =
                o.time_limit_s > 0 ? (unsigned long long)(o.time_limit_s * 1e9) : 0ull;
            set_capturing(true);
            cudaError_t err = cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
            if (err == cudaSuccess) {
                for (int k = 0; k < o.graph_steps; ++k) step(false);
                k_loop_cond<<<1, 32, 0, s>>>(handle, kv.st, nrhs, kv.loop, cap, limit_ns);
                err = cudaStreamEndCapture(s, &body);
            }
            set_capturing(false);
            if (err == cudaSuccess) err = cudaGraphInstantiate(&exec, graph, 0);
            ok = err == cudaSuccess;
            if (!ok) cudaGetLastError();
        }
        if (graph) cudaGraphDestroy(graph);
        if (ok) {
            TDDA_CUDA_TRY(cudaGraphLaunch(exec, s));
            TDDA_CUDA_TRY(cudaMemcpyAsync(kv.st_host, kv.st, sizeof(SolverState) * nrhs, cudaMemcpyDeviceToHost, s));
            unsigned long long passes = 0;
            TDDA_CUDA_TRY(cudaMemcpyAsync(&passes, kv.loop, sizeof(passes), cudaMemcpyDeviceToHost, s));
            TDDA_CUDA_TRY(cudaStreamSynchronize(s));
            count_launches((long long)passes * (o.graph_steps * kLaunchesPerStep + 1));
            if (o.fused) {
                dim3 gu(UPD_BLOCKS, nrhs);
                count_launches(1);
                k_flush<C><<<gu, NT, 0, s>>>(n, X, kv.p, kv.t, kv.st);
                TDDA_CUDA_TRY(cudaGetLastError());
            }
            if (info != nullptr)
                for (int k = 0; k < nrhs; ++k) {
                    const SolverState &S = kv.st_host[k];
                    info[k].iterations = S.iters;
                    info[k].error = S.err;
                    info[k].status = S.status;
                    info[k].refinements = 0;
                    info[k].inner_iterations = S.iters;
                    info[k].true_error = -1.0;
                }
            return TDDA_OK;
        }
        if (exec) { cudaGraphExecDestroy(exec); exec = nullptr; }
        // fall back: the first step is done; continue with polled chunks
    }

    long long launched = 0;
    bool first = !(o.graph_steps > 0 && o.device_loop && kv.loop != nullptr);
    int chunk = 2;
    for (;;) {
        if (o.graph_steps > 0 && !first) {
            if (exec == nullptr) { tdda_status st = capture(); if (st != TDDA_OK) return st; }
            const int reps = std::max(1, chunk / o.graph_steps);
            for (int k = 0; k < reps; ++k) TDDA_CUDA_TRY(cudaGraphLaunch(exec, s));
            count_launches((long long)reps * o.graph_steps * kLaunchesPerStep);
            launched += (long long)reps * o.graph_steps;
        } else {
            const int steps = (o.graph_steps > 0) ? 1 : chunk;  // the first step sets p = r
            for (int k = 0; k < steps; ++k) {
                step(first);
                first = false;
            }
            launched += steps;
        }
        TDDA_CUDA_TRY(cudaGetLastError());
        TDDA_CUDA_TRY(cudaMemcpyAsync(kv.st_host, kv.st, sizeof(SolverState) * nrhs, cudaMemcpyDeviceToHost, s));
        TDDA_CUDA_TRY(cudaStreamSynchronize(s));
        bool all = true;
        for (int k = 0; k < nrhs; ++k) all &= (kv.st_host[k].done != 0);
        if (all) break;
        if (launched > (long long)max_iter + 64) {
            set_error("solver did not report completion");
            return TDDA_ERR_STATE;
        }
        chunk = std::min(chunk * 2, 16);
    }
    if (o.fused) {
        dim3 gu(UPD_BLOCKS, nrhs);
        count_launches(1);
        k_flush<C><<<gu, NT, 0, s>>>(n, X, kv.p, kv.t, kv.st);
        TDDA_CUDA_TRY(cudaGetLastError());
    }
    if (info != nullptr)
        for (int k = 0; k < nrhs; ++k) {
            const SolverState &S = kv.st_host[k];
            info[k].iterations = S.iters;
            info[k].error = S.err;
            info[k].status = S.status;
            info[k].refinements = 0;
            info[k].inner_iterations = S.iters;
            info[k].true_error = -1.0;
        }
    return TDDA_OK;
}

template struct ConvOperator<double2>;
template struct ConvOperator<float2>;
template struct Krylov<double2>;
template struct Krylov<float2>;
template tdda_status bicgstab_device<double2>(ConvOperator<double2> &, Krylov<double2> &, const double2 *,
                                              const double2 *, const double2 *, double2 *, int, bool, int, double,
                                              cudaStream_t, tdda_solve_info *, const KrylovOptions &);
template tdda_status bicgstab_device<float2>(ConvOperator<float2> &, Krylov<float2> &, const float2 *,
                                             const float2 *, const float2 *, float2 *, int, bool, int, double,
                                             cudaStream_t, tdda_solve_info *, const KrylovOptions &);

template <typename C>
tdda_status profile_apply(ConvOperator<C> &op, const C *x, C *y, const C *al, int nrhs, int iters,
                          cudaStream_t s, double *ms_total, double *ms_pass) {
    ConvGeom g;
    if (nrhs > op.nrhs_cap || !geom_for(op, nrhs, g)) { set_error("batch does not fit"); return TDDA_ERR_UNSUPPORTED; }
    if (iters < 1) iters = 1;
    ProLoad<C> pro{};
    pro.nbox = g.nbox; pro.x = x; pro.st = nullptr;
    EpiMatvec<C> epi{};
    epi.nbox = g.nbox; epi.mask = op.mask; epi.y = y; epi.x = x; epi.al = al;
    cudaEvent_t e0, e1;
    TDDA_CUDA_TRY(cudaEventCreate(&e0));
    TDDA_CUDA_TRY(cudaEventCreate(&e1));
    dim3 g13(g.nx, 3, nrhs), g2(g.Ly, g.CKx > 0 ? g.Lz / g.CKx : 1, 1);
    auto timed = [&](auto &&fn) -> double {
        fn();  // warm
        cudaEventRecord(e0, s);
        for (int i = 0; i < iters; ++i) fn();
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        return (double)ms / iters;
    };
    *ms_total = timed([&] { run_conv(op, g, nrhs, pro, epi, nullptr, s); });
    ms_pass[0] = timed([&] {
        count_launches(1);
        if (!launch_fwd_reg<C, ProLoad<C>>(g, g13, op.T, op.tw, pro, s) &&
            !launch_fwd_cl<C, ProLoad<C>>(g, g13, op.T, op.tw, pro, s) &&
            !(g.fast_yz && launch_fwd_fast<C, ProLoad<C>>(g, g13, op.T, op.tw, pro, s)))
            k_fwd_zy<C, ProLoad<C>><<<g13, NT, g.smem_yz, s>>>(g, op.T, op.tw, pro);
    });
    ms_pass[1] = timed([&] {
        count_launches(1);
        if (!launch_xconv_reg<C>(g, op.T, op.ahat, op.ahat_rhs, op.tw, nrhs, nullptr, s) &&
            !(g.fast_x && launch_xconv_fast<C>(g, op.T, op.ahat, op.ahat_rhs, op.tw, nrhs, nullptr, s)))
            k_xconv<C><<<g2, NT, g.smem_x, s>>>(g, op.T, op.ahat, op.ahat_rhs, op.tw, nrhs, nullptr);
    });
    ms_pass[2] = timed([&] {
        count_launches(1);
        if (!launch_inv_reg<C, EpiMatvec<C>>(g, g13, op.T, op.tw, epi, s) &&
            !launch_inv_cl<C, EpiMatvec<C>>(g, g13, op.T, op.tw, epi, s) &&
            !(g.fast_yz && launch_inv_fast<C, EpiMatvec<C>>(g, g13, op.T, op.tw, epi, s)))
            k_inv_yz<C, EpiMatvec<C>><<<g13, NT, g.smem_yz, s>>>(g, op.T, op.tw, epi);
    });
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    TDDA_CUDA_TRY(cudaGetLastError());
    return TDDA_OK;
}

template tdda_status profile_apply<double2>(ConvOperator<double2> &, const double2 *, double2 *, const double2 *,
                                            int, int, cudaStream_t, double *, double *);
template tdda_status profile_apply<float2>(ConvOperator<float2> &, const float2 *, float2 *, const float2 *, int,
                                           int, cudaStream_t, double *, double *);

tdda_status residual_c128(ConvOperator<double2> &op, const double2 *al, const double2 *B, const double2 *X,
                          double2 *R, SolverState *st, int nrhs, cudaStream_t s, size_t dstride,
                          const ResidualPost *post) {
    ConvGeom g;
    if (nrhs > op.nrhs_cap || !geom_for(op, nrhs, g)) { set_error("batch does not fit"); return TDDA_ERR_UNSUPPORTED; }
    ProLoad<double2> pro{};
    pro.nbox = g.nbox; pro.x = X; pro.st = nullptr;
    EpiInit<double2> epi{};
    epi.nbox = g.nbox; epi.mask = op.mask; epi.part = op.partials; epi.counter = op.counters;
    epi.pstride = (size_t)op.partial_cap; epi.x0 = X; epi.b = B; epi.al = al; epi.r = R; epi.r0 = R; epi.st = st;
    epi.dstride = dstride;
    if (post != nullptr) epi.post = *post;
    run_conv(op, g, nrhs, pro, epi, nullptr, s);
    TDDA_CUDA_TRY(cudaGetLastError());
    return TDDA_OK;
}

}  // namespace tdda
