// Shared device/host helpers for libtdda: complex arithmetic on double2/float2,
// error handling, and the geometry of the padded FFT convolution.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <string>

namespace tdda {

// ----------------------------------------------------------------------------
// complex arithmetic on CUDA vector types (real part .x, imaginary part .y)
// ----------------------------------------------------------------------------
template <typename R> struct CplxOf;
template <> struct CplxOf<double> { using type = double2; };
template <> struct CplxOf<float> { using type = float2; };

template <typename C> struct RealOf;
template <> struct RealOf<double2> { using type = double; };
template <> struct RealOf<float2> { using type = float; };

__host__ __device__ __forceinline__ double2 cmake(double a, double b) { return make_double2(a, b); }
__host__ __device__ __forceinline__ float2 cmake(float a, float b) { return make_float2(a, b); }

template <typename C> __host__ __device__ __forceinline__ C czero() { C z; z.x = 0; z.y = 0; return z; }

#define TDDA_CPLX_OPS(C, R)                                                                         \
    __host__ __device__ __forceinline__ C operator+(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; } \
    __host__ __device__ __forceinline__ C operator-(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; } \
    __host__ __device__ __forceinline__ C operator-(C a) { C r; r.x = -a.x; r.y = -a.y; return r; }                \
    __host__ __device__ __forceinline__ C operator*(C a, C b) {                                    \
        C r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r; }                  \
    __host__ __device__ __forceinline__ C operator*(R s, C a) { C r; r.x = s * a.x; r.y = s * a.y; return r; }     \
    __host__ __device__ __forceinline__ C conj(C a) { C r; r.x = a.x; r.y = -a.y; return r; }      \
    /* multiply by +i (s=+1) or -i (s=-1) */                                                       \
    __host__ __device__ __forceinline__ C mul_i(C a, int s) {                                      \
        C r; r.x = s > 0 ? -a.y : a.y; r.y = s > 0 ? a.x : -a.x; return r; }                        \
    __host__ __device__ __forceinline__ R cabs2(C a) { return a.x * a.x + a.y * a.y; }

TDDA_CPLX_OPS(double2, double)
TDDA_CPLX_OPS(float2, float)
#undef TDDA_CPLX_OPS

__host__ __device__ __forceinline__ double2 to_d(double2 a) { return a; }
__host__ __device__ __forceinline__ double2 to_d(float2 a) { return make_double2(a.x, a.y); }
template <typename C> __host__ __device__ __forceinline__ C from_d(double2 a);
template <> __host__ __device__ __forceinline__ double2 from_d<double2>(double2 a) { return a; }
template <> __host__ __device__ __forceinline__ float2 from_d<float2>(double2 a) {
    return make_float2((float)a.x, (float)a.y);
}

// conjugate-first product conj(a) * b, accumulated in double
__host__ __device__ __forceinline__ double2 cdot1(double2 a, double2 b) {
    return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

// complex division a / b (Smith's algorithm, scaled to avoid overflow)
__host__ __device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
    double ar = a.x, ai = a.y, br = b.x, bi = b.y;
    if (fabs(br) >= fabs(bi)) {
        if (br == 0.0 && bi == 0.0) return make_double2(NAN, NAN);
        double q = bi / br, den = br + bi * q;
        return make_double2((ar + ai * q) / den, (ai - ar * q) / den);
    }
    double q = br / bi, den = bi + br * q;
    return make_double2((ar * q + ai) / den, (ai * q - ar) / den);
}

// ----------------------------------------------------------------------------
// convolution geometry
// ----------------------------------------------------------------------------
// The box holds nx*ny*nz cells; a dipole vector is stored per component as
// [c][x][y][z] (z fastest).  The zero-padded convolution grid is Lx*Ly*Lz with
// L >= 2n-1 on each axis; offset o of the interaction tensor sits at o mod L.
// The spectral intermediate T keeps only the populated x-half of the grid
// after the y/z transforms: [rhs][c][x < nx][ky < Ly][kz < Lz].
struct ConvGeom {
    int nx, ny, nz;     // box
    int Lx, Ly, Lz;     // padded FFT lengths
    int hx, hy, hz;     // folded spectral extents L/2+1 (tensor parity symmetry)
    int Lmax;           // common multiple of Lx, Ly, Lz (twiddle table length)
    long long nbox;     // nx*ny*nz
    long long tcomp;    // nx*Ly*Lz (one component of T)
    int pA;             // SMEM row pitch of the [y][z] slab buffer (elements)
    int YC;             // y columns per z transform call (passes 1 and 3)
    int reg_x;          // pass 2 on the register-resident two-level FFT
    int CKr;            // kz chunk of that kernel
    int pair_x;         // 1: that kernel takes ky and Ly - ky in one CTA
    int smem_r;         // its dynamic SMEM bytes
    int reg_yz;         // passes 1 and 3 on the register two-level slab kernels
    int smem_fr, smem_ir;  // their dynamic SMEM bytes (forward, inverse)
    int CK;             // kz chunk for the y transforms (passes 1 and 3)
    int pB;             // SMEM row pitch of the [ky][kz-chunk] buffer
    int CKx;            // kz chunk for the x pass (pass 2)
    int nrhs;           // right-hand sides per launch
    int pC;             // SMEM row pitch of the [kx][batch] buffer
    int smem_yz;        // dynamic SMEM bytes, passes 1 and 3
    int smem_x;         // dynamic SMEM bytes, pass 2
    int fast_yz;        // 1: passes 1 and 3 use the compile-time (Lz, Ly) slab kernels
    int cl_yz;          // 1: complex128 passes 1 and 3 use the two-CTA cluster slab kernels
    int smem_yz2;       // their dynamic SMEM bytes
    int fast_x;         // 1: pass 2 uses the compile-time-length kernel for Lx
    int CKx2;           // kz chunk of that kernel
    int smem_x2;        // its dynamic SMEM bytes (two ping-pong buffers)
};

// ----------------------------------------------------------------------------
// programmatic dependent launch
// ----------------------------------------------------------------------------
// The operator's passes and the solver's step kernels are launched with
// programmatic stream serialization (launch_dep): the stream's next kernel may
// be launched before the current one has fully retired.  Every kernel
// launched through launch_dep calls pdl_wait() before its first global-memory
// access: it returns once the previous kernel of the stream has completed and
// its writes are visible (at once for a kernel launched without the
// attribute, or after a copy).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline void launch_dep(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                       const Args &...args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kern, args...);
}

int next_fft_len(int minlen);   // smallest 2^a 3^b >= minlen

// number of kernels this library has launched (all devices, all models)
void count_launches(long long n);
// while a CUDA graph is being captured on this thread its launches are counted at replay
void set_capturing(bool on);
long long launches_total();

// error state (thread-local message for tdda_last_error)
void set_error(const std::string &msg);
const char *get_error();

}  // namespace tdda

#define TDDA_CUDA_TRY(expr)                                                                       \
    do {                                                                                           \
        cudaError_t _e = (expr);                                                                   \
        if (_e != cudaSuccess) {                                                                   \
            ::tdda::set_error(std::string(#expr) + ": " + cudaGetErrorString(_e));               \
            return _e == cudaErrorMemoryAllocation ? TDDA_ERR_OOM : TDDA_ERR_CUDA;               \
        }                                                                                          \
    } while (0)
