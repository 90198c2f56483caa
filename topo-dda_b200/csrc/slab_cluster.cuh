// Passes 1 and 3 for complex128 slabs, one (x, component, RHS) slab per
// cluster of two CTAs that share it through distributed shared memory
// (included by operator.cu; uses its prologue/epilogue functors and
// reduce_finalize).
//
// A complex128 slab after its z transforms is LZ x ny x 16 bytes (128 KB at
// 128x128x32): with the exchange buffer it does not fit one CTA's shared
// memory, so the generic runtime-length kernels took these passes.  Here the
// two CTAs of a cluster split the slab:
//   forward  z stage: CTA r transforms the rows y in [r ny/2, (r+1) ny/2)
//            (two-level LZ = R1z x 8: half-input R1z-point DFTs from the
//            fused prologue, one exchange, 8-point DFTs) into its half S_r;
//            cluster barrier;
//            y stage: CTA r transforms the columns kz in [r LZ/2, (r+1) LZ/2)
//            reading y from both halves (LY = RA x 16: half-input RA-point
//            DFTs over y = 16 n1 + n2, one exchange, 16-point DFTs written
//            straight to T as ky = k1 + RA k2).
//   inverse  the same stages the other way round: 16-point inverse DFTs from
//            T, half-output RA-point DFTs written into the half S_r that holds
//            each y (peer writes through distributed shared memory), cluster
//            barrier, inverse z transforms into the fused epilogue.
// The y split by 16 keeps the largest register set of one task at 16
// complex128 values (the complex64 kernels' 32-point half-input DFTs would
// need 32).  Pitches make the shared-memory patterns conflict-free for
// 16-byte elements: eight consecutive lanes touch either consecutive
// elements or elements an odd pitch apart.
#pragma once

#include <cooperative_groups.h>

namespace tdda {

namespace cgx = cooperative_groups;

template <int LZ, int LY> struct ClGeom {
    static constexpr int NY = LY / 2, NZ = LZ / 2;     // grid extents (half padding on both axes)
    static constexpr int NYH = NY / 2, KZH = LZ / 2;   // rows per CTA (z stage), columns per CTA (y stage)
    static constexpr int R1z = LZ / 8, H1z = R1z / 2;  // z: LZ = R1z x 8
    static constexpr int RA = LY / 16, HA = RA / 2;    // y: LY = RA x 16
    static constexpr int PS = NYH + 1, PZ = NYH + 1, PY = KZH + 1;
    static constexpr int NT = LZ == 64 ? 512 : (LZ == 48 ? 384 : 256);
    static constexpr int MINB = LZ >= 48 ? 1 : 2;
    static constexpr int S_ELEMS = LZ * PS;
    static constexpr int X_ELEMS = (LZ * PZ > LY * PY) ? LZ * PZ : LY * PY;
    static constexpr int SMEM = (S_ELEMS + X_ELEMS) * 16;
    static_assert(NYH % 16 == 0, "each half of y must hold whole groups of 16 rows");
    static_assert(LZ % 16 == 0 && LY % 32 == 0, "unsupported slab shape");
};

template <typename C, int LZ, int LY, class Pro>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(ClGeom<LZ, LY>::NT, ClGeom<LZ, LY>::MINB)
    k_fwd_zy_cl(ConvGeom g, C *__restrict__ T, const C *__restrict__ tw, Pro pro) {
    using G = ClGeom<LZ, LY>;
    pdl_wait();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cgx::cluster_group cl = cgx::this_cluster();
    const int r = (int)cl.block_rank();
    const int x = blockIdx.x >> 1, c = blockIdx.y, rhs = blockIdx.z;
    if (pro.skip(rhs)) return;  // the same for both CTAs of the cluster
    C *S = reinterpret_cast<C *>(smem_raw);  // [kz][PS]: rows y0 .. y0 + NYH
    C *X = S + G::S_ELEMS;                   // exchange
    C *peer = cl.map_shared_rank(S, r ^ 1);
    const C *S0 = r == 0 ? S : peer;
    const C *S1 = r == 0 ? peer : S;
    const long long cell0 = (long long)x * G::NY * G::NZ;
    const int twz = g.Lmax / LZ, twy = g.Lmax / LY, twz1 = g.Lmax / G::R1z, twy1 = g.Lmax / G::RA;
    const int y0 = r * G::NYH, kz0 = r * G::KZH;
    // z, first level: task (n2, yl), z = 8 n1 + n2 from the prologue
    for (int t = threadIdx.x; t < 8 * G::NYH; t += G::NT) {
        const int n2 = t & 7, yl = t >> 3;
        C a[G::H1z], b[G::H1z];
#pragma unroll
        for (int n1 = 0; n1 < G::H1z; ++n1)
            a[n1] = pro.load(rhs, c, cell0 + (long long)(y0 + yl) * G::NZ + 8 * n1 + n2);
        dft_half_in<G::H1z, -1>(a, b, tw, twz1);
#pragma unroll
        for (int q = 0; q < G::H1z; ++q) {
            const int k1 = 2 * q;
            C v0 = a[q], v1 = b[q];
            if (n2 != 0) {
                if (k1 != 0) v0 = v0 * twiddle<-1>(tw, n2 * k1 * twz);
                v1 = v1 * twiddle<-1>(tw, n2 * (k1 + 1) * twz);
            }
            X[(k1 * 8 + n2) * G::PZ + yl] = v0;
            X[((k1 + 1) * 8 + n2) * G::PZ + yl] = v1;
        }
    }
    __syncthreads();
    // z, second level: task (yl, k1), kz = k1 + R1z k2 into this CTA's half
    for (int t = threadIdx.x; t < G::NYH * G::R1z; t += G::NT) {
        const int yl = t % G::NYH, k1 = t / G::NYH;
        C v[8];
#pragma unroll
        for (int n2 = 0; n2 < 8; ++n2) v[n2] = X[(k1 * 8 + n2) * G::PZ + yl];
        dftR<8, -1>(v);
#pragma unroll
        for (int k2 = 0; k2 < 8; ++k2) S[(k1 + G::R1z * k2) * G::PS + yl] = v[k2];
    }
    cl.sync();  // both halves of the slab are complete
    // y, first level: task (n2, kzl), y = 16 n1 + n2 (n1 < HA) from the half holding it
    for (int t = threadIdx.x; t < 16 * G::KZH; t += G::NT) {
        const int n2 = t & 15, kzl = t >> 4, kz = kz0 + kzl;
        C a[G::HA], b[G::HA];
#pragma unroll
        for (int n1 = 0; n1 < G::HA; ++n1) {
            const int src = (16 * n1) / G::NYH;  // compile-time once unrolled
            const C *Ssrc = src == 0 ? S0 : S1;
            a[n1] = Ssrc[kz * G::PS + 16 * n1 - src * G::NYH + n2];
        }
        dft_half_in<G::HA, -1>(a, b, tw, twy1);
#pragma unroll
        for (int q = 0; q < G::HA; ++q) {
            const int k1 = 2 * q;
            C v0 = a[q], v1 = b[q];
            if (n2 != 0) {
                if (k1 != 0) v0 = v0 * twiddle<-1>(tw, n2 * k1 * twy);
                v1 = v1 * twiddle<-1>(tw, n2 * (k1 + 1) * twy);
            }
            X[(k1 * 16 + n2) * G::PY + kzl] = v0;
            X[((k1 + 1) * 16 + n2) * G::PY + kzl] = v1;
        }
    }
    cl.sync();  // the peer has read this CTA's half; the exchange is complete
    // y, second level: task (kzl, k1), ky = k1 + RA k2 straight to T[ky][kz]
    C *Tc = T + ((size_t)(rhs * 3 + c) * g.nx + x) * (size_t)(LY * LZ);
    for (int t = threadIdx.x; t < G::KZH * G::RA; t += G::NT) {
        const int kzl = t % G::KZH, k1 = t / G::KZH;
        C v[16];
#pragma unroll
        for (int n2 = 0; n2 < 16; ++n2) v[n2] = X[(k1 * 16 + n2) * G::PY + kzl];
        dft_reg<16, -1>(v);
#pragma unroll
        for (int k2 = 0; k2 < 16; ++k2) Tc[(size_t)(k1 + G::RA * k2) * LZ + kz0 + kzl] = v[k2];
    }
}

template <typename C, int LZ, int LY, class Epi>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(ClGeom<LZ, LY>::NT, ClGeom<LZ, LY>::MINB)
    k_inv_yz_cl(ConvGeom g, const C *__restrict__ T, const C *__restrict__ tw, Epi epi) {
    using G = ClGeom<LZ, LY>;
    pdl_wait();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cgx::cluster_group cl = cgx::this_cluster();
    const int r = (int)cl.block_rank();
    const int x = blockIdx.x >> 1, c = blockIdx.y, rhs = blockIdx.z;
    if (epi.skip(rhs)) return;  // the same for both CTAs of the cluster
    C *S = reinterpret_cast<C *>(smem_raw);  // [kz][PS]: rows y0 .. y0 + NYH
    C *X = S + G::S_ELEMS;
    C *peer = cl.map_shared_rank(S, r ^ 1);
    C *S0 = r == 0 ? S : peer;
    C *S1 = r == 0 ? peer : S;
    const int twz = g.Lmax / LZ, twy = g.Lmax / LY, twz1 = g.Lmax / G::R1z, twy1 = g.Lmax / G::RA;
    const int y0 = r * G::NYH, kz0 = r * G::KZH;
    const C *Tc = T + ((size_t)(rhs * 3 + c) * g.nx + x) * (size_t)(LY * LZ);
    // y, inverse first level: task (kzl, k1) over ky = k1 + RA k2 from T
    for (int t = threadIdx.x; t < G::KZH * G::RA; t += G::NT) {
        const int kzl = t % G::KZH, k1 = t / G::KZH;
        C v[16];
#pragma unroll
        for (int k2 = 0; k2 < 16; ++k2) v[k2] = Tc[(size_t)(k1 + G::RA * k2) * LZ + kz0 + kzl];
        dft_reg<16, +1>(v);
        if (k1 != 0) {
#pragma unroll
            for (int n1 = 1; n1 < 16; ++n1) v[n1] = v[n1] * twiddle<+1>(tw, k1 * n1 * twy);
        }
#pragma unroll
        for (int n1 = 0; n1 < 16; ++n1) X[(k1 * 16 + n1) * G::PY + kzl] = v[n1];
    }
    cl.sync();  // the exchange is complete and the peer CTA is running
    // y, inverse second level: task (kzl, n1), y = n1 + 16 n2 < ny into the half holding y
    for (int t = threadIdx.x; t < G::KZH * 16; t += G::NT) {
        const int kzl = t % G::KZH, n1 = t / G::KZH, kz = kz0 + kzl;
        C e[G::HA], o[G::HA];
#pragma unroll
        for (int q = 0; q < G::HA; ++q) {
            e[q] = X[((2 * q) * 16 + n1) * G::PY + kzl];
            o[q] = X[((2 * q + 1) * 16 + n1) * G::PY + kzl];
        }
        dft_half_out<G::HA, +1>(e, o, tw, twy1);
#pragma unroll
        for (int n2 = 0; n2 < G::HA; ++n2) {
            const int dst = (16 * n2) / G::NYH;  // compile-time once unrolled
            C *Sd = dst == 0 ? S0 : S1;
            Sd[kz * G::PS + 16 * n2 - dst * G::NYH + n1] = e[n2];
        }
    }
    cl.sync();  // both halves hold every kz of their rows (peer writes visible)
    // z, inverse first level: task (yl, k1) over kz = k1 + R1z k2
    for (int t = threadIdx.x; t < G::NYH * G::R1z; t += G::NT) {
        const int yl = t % G::NYH, k1 = t / G::NYH;
        C v[8];
#pragma unroll
        for (int k2 = 0; k2 < 8; ++k2) v[k2] = S[(k1 + G::R1z * k2) * G::PS + yl];
        dftR<8, +1>(v);
        if (k1 != 0) {
#pragma unroll
            for (int n1 = 1; n1 < 8; ++n1) v[n1] = v[n1] * twiddle<+1>(tw, k1 * n1 * twz);
        }
#pragma unroll
        for (int n1 = 0; n1 < 8; ++n1) X[(k1 * 8 + n1) * G::PZ + yl] = v[n1];
    }
    __syncthreads();
    // z, inverse second level: task (n1, yl), z = n1 + 8 n2 < nz into the epilogue
    const long long cell0 = (long long)x * G::NY * G::NZ;
    double2 acc[Epi::NQ > 0 ? Epi::NQ : 1];
#pragma unroll
    for (int q = 0; q < (Epi::NQ > 0 ? Epi::NQ : 1); ++q) acc[q] = make_double2(0.0, 0.0);
    for (int t = threadIdx.x; t < 8 * G::NYH; t += G::NT) {
        const int n1 = t & 7, yl = t >> 3;
        C e[G::H1z], o[G::H1z];
#pragma unroll
        for (int q = 0; q < G::H1z; ++q) {
            e[q] = X[((2 * q) * 8 + n1) * G::PZ + yl];
            o[q] = X[((2 * q + 1) * 8 + n1) * G::PZ + yl];
        }
        dft_half_out<G::H1z, +1>(e, o, tw, twz1);
#pragma unroll
        for (int n2 = 0; n2 < G::H1z; ++n2)
            epi.apply(rhs, c, cell0 + (long long)(y0 + yl) * G::NZ + n1 + 8 * n2, e[n2], acc);
    }
    if constexpr (Epi::NQ > 0) {
        reduce_finalize<Epi::NQ>(acc, epi.part + (size_t)rhs * epi.pstride, epi.counter + rhs,
                                 blockIdx.y * gridDim.x + blockIdx.x, gridDim.x * gridDim.y, epi, rhs);
    }
}

// (Lz, Ly) pairs with complex128 cluster slab kernels
#define TDDA_YZ_CL_PAIRS(X) X(64, 256) X(48, 192) X(32, 128) X(32, 192) X(32, 256)

static bool cl_yz_pair(int Lz, int Ly) {
#define TDDA_CL_PAIR_TEST(a, b) if (Lz == a && Ly == b) return true;
    TDDA_YZ_CL_PAIRS(TDDA_CL_PAIR_TEST)
#undef TDDA_CL_PAIR_TEST
    return false;
}

static int cl_smem(int Lz, int Ly) {
#define TDDA_CL_SMEM(a, b) if (Lz == a && Ly == b) return ClGeom<a, b>::SMEM;
    TDDA_YZ_CL_PAIRS(TDDA_CL_SMEM)
#undef TDDA_CL_SMEM
    return 0;
}

template <typename C, class Pro>
static bool launch_fwd_cl(const ConvGeom &g, dim3 grid, C *T, const C *tw, const Pro &pro, cudaStream_t s) {
    if constexpr (!std::is_same<C, double2>::value) {
        return false;
    } else {
        if (!g.cl_yz) return false;
        const dim3 gc(2 * grid.x, grid.y, grid.z);
#define TDDA_FWD_CL_CASE(a, b)                                                                            \
    if (g.Lz == a && g.Ly == b) {                                                                         \
        launch_dep((k_fwd_zy_cl<C, a, b, Pro>), gc, dim3(ClGeom<a, b>::NT), ClGeom<a, b>::SMEM, s, g, T, tw, pro); \
        return true;                                                                                      \
    }
        TDDA_YZ_CL_PAIRS(TDDA_FWD_CL_CASE)
#undef TDDA_FWD_CL_CASE
        return false;
    }
}

template <typename C, class Epi>
static bool launch_inv_cl(const ConvGeom &g, dim3 grid, const C *T, const C *tw, const Epi &epi, cudaStream_t s) {
    if constexpr (!std::is_same<C, double2>::value) {
        return false;
    } else {
        if (!g.cl_yz) return false;
        const dim3 gc(2 * grid.x, grid.y, grid.z);
#define TDDA_INV_CL_CASE(a, b)                                                                            \
    if (g.Lz == a && g.Ly == b) {                                                                         \
        launch_dep((k_inv_yz_cl<C, a, b, Epi>), gc, dim3(ClGeom<a, b>::NT), ClGeom<a, b>::SMEM, s, g, T, tw, epi); \
        return true;                                                                                      \
    }
        TDDA_YZ_CL_PAIRS(TDDA_INV_CL_CASE)
#undef TDDA_INV_CL_CASE
        return false;
    }
}

}  // namespace tdda
