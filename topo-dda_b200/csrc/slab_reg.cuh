// Passes 1 and 3 for complex64 slabs as register-resident two-level FFTs
// (included by operator.cu; uses its prologue/epilogue functors and
// reduce_finalize).  For one (x, component, RHS) slab with nz = LZ / 2 and
// ny = LY / 2 (the zero padding is exactly the upper half of each axis), every
// transform of length L = R1 * 8 runs as:
//   half-input R1-point DFTs in registers (inputs n = 8 n1 + n2, n1 < R1/2),
//   twiddle W_L^(n2 k1), one shared-memory exchange, 8-point DFTs
//   (outputs k = k1 + R1 k2),
// and the inverses the other way round with half-output R1-point DFTs.
// Forward: z transforms straight from the fused prologue, the spectra
// into an [kz][y] slab, y transforms, the 8-point stage written straight to T.
// Inverse: the 8-point stage straight from T, ... , the last half-output
// z transform straight into the fused epilogue.  Three barriers per kernel.
// Row pitches make every shared-memory access pattern conflict-free: a
// half-warp touches either 16 consecutive elements or 8 x 2 elements whose
// pitch is 2 (mod 16) or 8 (mod 16) elements (8-byte elements, 16 bank pairs).
#pragma once

namespace tdda {

constexpr int NTS = 512;

__host__ __device__ constexpr int pitch_mod16(int n, int r) { return n + (((r - n) % 16) + 16) % 16; }

struct SlabPitch {
    int PS, PZ, PY;  // slab [kz][PS], z exchange [LZ][PZ], y exchange [LY][PY]
};

__host__ __device__ inline SlabPitch slab_pitch_fwd(int ny, int LZ) {
    return {pitch_mod16(ny, 8), pitch_mod16(ny, 2), pitch_mod16(LZ, 2)};
}

__host__ __device__ inline SlabPitch slab_pitch_inv(int ny, int LZ) {
    return {ny | 1, pitch_mod16(ny, 2), LZ};
}

__host__ inline int slab_reg_smem(int ny, int LZ, int LY, bool fwd, int esize) {
    const SlabPitch p = fwd ? slab_pitch_fwd(ny, LZ) : slab_pitch_inv(ny, LZ);
    const long long x = std::max((long long)LZ * p.PZ, (long long)LY * p.PY);
    return (int)(((long long)LZ * p.PS + x) * esize);
}

template <typename C, int LZ, int LY, class Pro>
__global__ void __launch_bounds__(NTS, 1) k_fwd_zy_reg(ConvGeom g, C *__restrict__ T, const C *__restrict__ tw,
                                                       Pro pro) {
    pdl_wait();
    constexpr int R1z = LZ / 8, H1z = R1z / 2, R1y = LY / 8, H1y = R1y / 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int x = blockIdx.x, c = blockIdx.y, rhs = blockIdx.z;
    if (pro.skip(rhs)) return;
    const int ny = g.ny, nz = g.nz;
    const SlabPitch p = slab_pitch_fwd(ny, LZ);
    C *S = reinterpret_cast<C *>(smem_raw);  // [kz][y]
    C *X = S + LZ * p.PS;                     // exchange
    const long long cell0 = (long long)x * ny * nz;
    const int twz = g.Lmax / LZ, twy = g.Lmax / LY, twz1 = g.Lmax / R1z, twy1 = g.Lmax / R1y;
    // z, first level: task (n2, y), z = 8 n1 + n2 from the prologue
    for (int t = threadIdx.x; t < ny * 8; t += NTS) {
        const int n2 = t & 7, y = t >> 3;
        C a[H1z], b[H1z];
#pragma unroll
        for (int n1 = 0; n1 < H1z; ++n1) a[n1] = pro.load(rhs, c, cell0 + (long long)y * nz + 8 * n1 + n2);
        dft_half_in<H1z, -1>(a, b, tw, twz1);
#pragma unroll
        for (int q = 0; q < H1z; ++q) {
            const int k1 = 2 * q;
            C y0 = a[q], y1 = b[q];
            if (n2 != 0) {
                if (k1 != 0) y0 = y0 * twiddle<-1>(tw, n2 * k1 * twz);
                y1 = y1 * twiddle<-1>(tw, n2 * (k1 + 1) * twz);
            }
            X[(k1 * 8 + n2) * p.PZ + y] = y0;
            X[((k1 + 1) * 8 + n2) * p.PZ + y] = y1;
        }
    }
    __syncthreads();
    // z, second level: task (y, k1), kz = k1 + R1z k2 into the slab
    for (int t = threadIdx.x; t < ny * R1z; t += NTS) {
        const int y = t % ny, k1 = t / ny;
        C v[8];
#pragma unroll
        for (int n2 = 0; n2 < 8; ++n2) v[n2] = X[(k1 * 8 + n2) * p.PZ + y];
        dftR<8, -1>(v);
#pragma unroll
        for (int k2 = 0; k2 < 8; ++k2) S[(k1 + R1z * k2) * p.PS + y] = v[k2];
    }
    __syncthreads();
    // y, first level: task (n2, kz), y = 8 n1 + n2
    for (int t = threadIdx.x; t < LZ * 8; t += NTS) {
        const int n2 = t & 7, kz = t >> 3;
        C a[H1y], b[H1y];
#pragma unroll
        for (int n1 = 0; n1 < H1y; ++n1) a[n1] = S[kz * p.PS + 8 * n1 + n2];
        dft_half_in<H1y, -1>(a, b, tw, twy1);
#pragma unroll
        for (int q = 0; q < H1y; ++q) {
            const int k1 = 2 * q;
            C y0 = a[q], y1 = b[q];
            if (n2 != 0) {
                if (k1 != 0) y0 = y0 * twiddle<-1>(tw, n2 * k1 * twy);
                y1 = y1 * twiddle<-1>(tw, n2 * (k1 + 1) * twy);
            }
            X[(k1 * 8 + n2) * p.PY + kz] = y0;
            X[((k1 + 1) * 8 + n2) * p.PY + kz] = y1;
        }
    }
    __syncthreads();
    // y, second level: task (kz, k1), ky = k1 + R1y k2 straight to T[ky][kz]
    C *Tc = T + ((size_t)(rhs * 3 + c) * g.nx + x) * (size_t)(LY * LZ);
    for (int t = threadIdx.x; t < LZ * R1y; t += NTS) {
        const int kz = t % LZ, k1 = t / LZ;
        C v[8];
#pragma unroll
        for (int n2 = 0; n2 < 8; ++n2) v[n2] = X[(k1 * 8 + n2) * p.PY + kz];
        dftR<8, -1>(v);
#pragma unroll
        for (int k2 = 0; k2 < 8; ++k2) Tc[(size_t)(k1 + R1y * k2) * LZ + kz] = v[k2];
    }
}

template <typename C, int LZ, int LY, class Epi>
__global__ void __launch_bounds__(NTS, 1) k_inv_yz_reg(ConvGeom g, const C *__restrict__ T, const C *__restrict__ tw,
                                                       Epi epi) {
    pdl_wait();
    constexpr int R1z = LZ / 8, H1z = R1z / 2, R1y = LY / 8, H1y = R1y / 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int x = blockIdx.x, c = blockIdx.y, rhs = blockIdx.z;
    if (epi.skip(rhs)) return;
    const int ny = g.ny, nz = g.nz;
    const SlabPitch p = slab_pitch_inv(ny, LZ);
    C *S = reinterpret_cast<C *>(smem_raw);  // [kz][y]
    C *X = S + LZ * p.PS;
    const int twz = g.Lmax / LZ, twy = g.Lmax / LY, twz1 = g.Lmax / R1z, twy1 = g.Lmax / R1y;
    const C *Tc = T + ((size_t)(rhs * 3 + c) * g.nx + x) * (size_t)(LY * LZ);
    // y, inverse first level: task (kz, k1) over ky = k1 + R1y k2 from T; a
    // thread loads the values of two tasks before transforming either, so two
    // tasks' loads are in flight at once
    for (int t0 = threadIdx.x; t0 < LZ * R1y; t0 += 2 * NTS) {
        C v[2][8];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int t = t0 + u * NTS, kz = t % LZ, k1 = t / LZ;
            if (t < LZ * R1y) {
#pragma unroll
                for (int k2 = 0; k2 < 8; ++k2) v[u][k2] = Tc[(size_t)(k1 + R1y * k2) * LZ + kz];
            }
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int t = t0 + u * NTS, kz = t % LZ, k1 = t / LZ;
            if (t < LZ * R1y) {
                dftR<8, +1>(v[u]);
                if (k1 != 0) {
#pragma unroll
                    for (int n1 = 1; n1 < 8; ++n1) v[u][n1] = v[u][n1] * twiddle<+1>(tw, k1 * n1 * twy);
                }
#pragma unroll
                for (int n1 = 0; n1 < 8; ++n1) X[(k1 * 8 + n1) * p.PY + kz] = v[u][n1];
            }
        }
    }
    __syncthreads();
    // y, inverse second level: task (kz, n1), y = n1 + 8 n2 < ny into the slab
    for (int t = threadIdx.x; t < LZ * 8; t += NTS) {
        const int kz = t % LZ, n1 = t / LZ;
        C e[H1y], o[H1y];
#pragma unroll
        for (int q = 0; q < H1y; ++q) {
            e[q] = X[((2 * q) * 8 + n1) * p.PY + kz];
            o[q] = X[((2 * q + 1) * 8 + n1) * p.PY + kz];
        }
        dft_half_out<H1y, +1>(e, o, tw, twy1);
#pragma unroll
        for (int n2 = 0; n2 < H1y; ++n2) S[kz * p.PS + n1 + 8 * n2] = e[n2];
    }
    __syncthreads();
    // z, inverse first level: task (y, k1) over kz = k1 + R1z k2
    for (int t = threadIdx.x; t < ny * R1z; t += NTS) {
        const int y = t % ny, k1 = t / ny;
        C v[8];
#pragma unroll
        for (int k2 = 0; k2 < 8; ++k2) v[k2] = S[(k1 + R1z * k2) * p.PS + y];
        dftR<8, +1>(v);
        if (k1 != 0) {
#pragma unroll
            for (int n1 = 1; n1 < 8; ++n1) v[n1] = v[n1] * twiddle<+1>(tw, k1 * n1 * twz);
        }
#pragma unroll
        for (int n1 = 0; n1 < 8; ++n1) X[(k1 * 8 + n1) * p.PZ + y] = v[n1];
    }
    __syncthreads();
    // z, inverse second level: task (n1, y), z = n1 + 8 n2 < nz into the epilogue
    const long long cell0 = (long long)x * ny * nz;
    double2 acc[Epi::NQ > 0 ? Epi::NQ : 1];
#pragma unroll
    for (int q = 0; q < (Epi::NQ > 0 ? Epi::NQ : 1); ++q) acc[q] = make_double2(0.0, 0.0);
    for (int t = threadIdx.x; t < ny * 8; t += NTS) {
        const int n1 = t & 7, y = t >> 3;
        C e[H1z], o[H1z];
#pragma unroll
        for (int q = 0; q < H1z; ++q) {
            e[q] = X[((2 * q) * 8 + n1) * p.PZ + y];
            o[q] = X[((2 * q + 1) * 8 + n1) * p.PZ + y];
        }
        dft_half_out<H1z, +1>(e, o, tw, twz1);
#pragma unroll
        for (int n2 = 0; n2 < H1z; ++n2) epi.apply(rhs, c, cell0 + (long long)y * nz + n1 + 8 * n2, e[n2], acc);
    }
    if constexpr (Epi::NQ > 0) {
        reduce_finalize<Epi::NQ>(acc, epi.part + (size_t)rhs * epi.pstride, epi.counter + rhs,
                                 blockIdx.y * gridDim.x + blockIdx.x, gridDim.x * gridDim.y, epi, rhs);
    }
}

// (Lz, Ly) pairs with register slab kernels (both lengths 8 x an even R1 >= 4)
#define TDDA_YZ_REG_PAIRS(X) X(64, 256) X(48, 192) X(32, 128) X(32, 192) X(32, 256)

template <typename C, class Pro>
static bool launch_fwd_reg(const ConvGeom &g, dim3 grid, C *T, const C *tw, const Pro &pro, cudaStream_t s) {
    if constexpr (!std::is_same<C, float2>::value) {
        return false;
    } else {
        if (!g.reg_yz) return false;
#define TDDA_FWD_REG_CASE(a, b)                                                                  \
    if (g.Lz == a && g.Ly == b) {                                                                \
        launch_dep((k_fwd_zy_reg<C, a, b, Pro>), grid, dim3(NTS), g.smem_fr, s, g, T, tw, pro);                 \
        return true;                                                                             \
    }
        TDDA_YZ_REG_PAIRS(TDDA_FWD_REG_CASE)
#undef TDDA_FWD_REG_CASE
        return false;
    }
}

template <typename C, class Epi>
static bool launch_inv_reg(const ConvGeom &g, dim3 grid, const C *T, const C *tw, const Epi &epi, cudaStream_t s) {
    if constexpr (!std::is_same<C, float2>::value) {
        return false;
    } else {
        if (!g.reg_yz) return false;
#define TDDA_INV_REG_CASE(a, b)                                                                  \
    if (g.Lz == a && g.Ly == b) {                                                                \
        launch_dep((k_inv_yz_reg<C, a, b, Epi>), grid, dim3(NTS), g.smem_ir, s, g, T, tw, epi);                 \
        return true;                                                                             \
    }
        TDDA_YZ_REG_PAIRS(TDDA_INV_REG_CASE)
#undef TDDA_INV_REG_CASE
        return false;
    }
}

static bool reg_yz_pair(int Lz, int Ly) {
#define TDDA_REG_PAIR_TEST(a, b) if (Lz == a && Ly == b) return true;
    TDDA_YZ_REG_PAIRS(TDDA_REG_PAIR_TEST)
#undef TDDA_REG_PAIR_TEST
    return false;
}

}  // namespace tdda
