// Allocation-free application of the interaction operator.
//
// Some callers cannot let a library allocate device memory while they run:
// a serving loop that admits work against a fixed device-memory budget, a
// host thread with a latency deadline (cudaMalloc and cudaFree may wait for
// the whole device), or an application that plans every device byte up front.
// For them, tdda_matvec_device_noalloc applies A (+ 1/alpha) to one vector
// using only the memory it is given (the model, the input and the output) and
// a fixed scratch area that is part of the library image.
//
// The scratch is a file-scope __device__ array of kScratchBytes (32 MiB).
// Every GPU that loads the library holds it until the process exits.  It
// holds the input and output in the operator's internal layout and the
// spectral intermediate, so a call fits when
//     2 * 3 * nx*ny*nz * 16 B  +  3 * nx * Ly * Lz * 16 B  <=  32 MiB
// (e.g. 64 x 64 x 16 dipoles use 18 MiB; 64 x 64 x 32 need 36 MiB and are
// rejected).
//
// Host code cannot use the array's name as a device address.  The first call
// on each device looks the address up with cudaGetSymbolAddress while that
// device is current and caches it together with the unique id of the device's
// current context; a call made in another context (the primary context was
// destroyed by cudaDeviceReset and created again, which reloads the library's
// module, possibly at another address) looks it up again.  Under lazy module
// loading (the CUDA default) the first call on a model may also load the
// operator kernels of its grid, which allocates device memory: make one
// warm-up call per model before the allocation-free region and before any
// stream capture begins.  All calls share the one array: calls that overlap
// on the GPU (different streams, or different host threads) race on it and
// must be serialised by the caller.
#include <cuda.h>

#include <algorithm>
#include <cstdio>
#include <mutex>
#include <string>

#include "model_view.cuh"

namespace tdda {

constexpr size_t kScratchBytes = size_t(32) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

std::mutex g_scratch_mu;

// device address of g_noalloc_scratch per device, valid in the context whose
// id is stored beside it
struct ScratchSlot {
    unsigned long long ctx_id;
    void *addr;
};
ScratchSlot g_scratch[kMaxDevices];

typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long *);
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;

// Unique id of the calling thread's current context (the runtime's primary
// context of the current device).  Context ids are never reused within a
// process, unlike context handles.  Called with g_scratch_mu held.
tdda_status current_context_id(unsigned long long *id) {
    if (g_ctx_get_current == nullptr || g_ctx_get_id == nullptr) {
        cudaDriverEntryPointQueryResult q1, q2;
        void *f1 = nullptr, *f2 = nullptr;
        cudaError_t e1 = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1);
        cudaError_t e2 = cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2);
        if (e1 != cudaSuccess || e2 != cudaSuccess || q1 != cudaDriverEntryPointSuccess ||
            q2 != cudaDriverEntryPointSuccess || f1 == nullptr || f2 == nullptr) {
            set_error("cuCtxGetCurrent / cuCtxGetId are not available from the driver");
            return TDDA_ERR_CUDA;
        }
        g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(f1);
        g_ctx_get_id = reinterpret_cast<CtxGetIdFn>(f2);
    }
    CUcontext ctx = nullptr;
    if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr || g_ctx_get_id(ctx, id) != CUDA_SUCCESS) {
        set_error("no current CUDA context");
        return TDDA_ERR_CUDA;
    }
    return TDDA_OK;
}

// The device address of the scratch array on device `dev` (current), looked
// up once per device and context.
tdda_status scratch_address(int dev, unsigned char **out) {
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    unsigned long long ctx_id = 0;
    tdda_status st = current_context_id(&ctx_id);
    if (st != TDDA_OK) return st;
    ScratchSlot &slot = g_scratch[dev];
    if (slot.addr == nullptr || slot.ctx_id != ctx_id) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            set_error(std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
            return TDDA_ERR_CUDA;
        }
        slot.addr = p;
        slot.ctx_id = ctx_id;
    }
    *out = static_cast<unsigned char *>(slot.addr);
    return TDDA_OK;
}

size_t round256(size_t b) { return (b + 255) & ~size_t(255); }

// dipole order (3 i + c) <-> internal [c][cell]
__global__ void k_noalloc_scatter(long long N, long long nbox, const long long *__restrict__ cell_of,
                                  const double2 *__restrict__ ext, double2 *__restrict__ in) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < 3 * N; e += (long long)gridDim.x * blockDim.x) {
        long long i = e / 3;
        int c = (int)(e - 3 * i);
        in[(size_t)c * nbox + cell_of[i]] = ext[e];
    }
}

__global__ void k_noalloc_gather(long long N, long long nbox, const long long *__restrict__ cell_of,
                                 const double2 *__restrict__ in, double2 *__restrict__ ext) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < 3 * N; e += (long long)gridDim.x * blockDim.x) {
        long long i = e / 3;
        int c = (int)(e - 3 * i);
        ext[e] = in[(size_t)c * nbox + cell_of[i]];
    }
}

}  // namespace
}  // namespace tdda

using namespace tdda;

extern "C" tdda_status tdda_matvec_device_noalloc(tdda_model *m, const void *x_dev, void *y_dev, int with_al,
                                                  void *stream) {
    if (m == nullptr || x_dev == nullptr || y_dev == nullptr) {
        set_error("null argument");
        return TDDA_ERR_BAD_ARG;
    }
    const ModelView v = model_view(m);
    const ConvGeom &g = v.op->g;
    const size_t vec_bytes = round256(sizeof(double2) * 3 * (size_t)v.nbox);
    const size_t t_bytes = round256(sizeof(double2) * 3 * (size_t)g.tcomp);
    const size_t need = 2 * vec_bytes + t_bytes;
    if (need > kScratchBytes) {
        char msg[256];
        snprintf(msg, sizeof msg,
                 "grid %dx%dx%d needs %.1f MiB of scratch; the allocation-free matvec has %zu MiB "
                 "(use tdda_matvec_device)",
                 g.nx, g.ny, g.nz, need / 1048576.0, kScratchBytes >> 20);
        set_error(msg);
        return TDDA_ERR_BAD_ARG;
    }
    int dev = 0;
    TDDA_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("device index beyond the scratch table");
        return TDDA_ERR_UNSUPPORTED;
    }
    cudaPointerAttributes at{};
    TDDA_CUDA_TRY(cudaPointerGetAttributes(&at, v.al));
    if (at.device != dev) {
        set_error("the model lives on another device than the current one");
        return TDDA_ERR_BAD_ARG;
    }
    unsigned char *base = nullptr;
    tdda_status st = scratch_address(dev, &base);
    if (st != TDDA_OK) return st;
    double2 *xin = reinterpret_cast<double2 *>(base);
    double2 *yin = reinterpret_cast<double2 *>(base + vec_bytes);
    double2 *T = reinterpret_cast<double2 *>(base + 2 * vec_bytes);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // cells without a dipole must read as zero; the previous call may have left data there
    if (v.mask != nullptr) TDDA_CUDA_TRY(cudaMemsetAsync(xin, 0, sizeof(double2) * 3 * (size_t)v.nbox, s));
    const long long n3 = 3 * v.N;
    const unsigned blocks = (unsigned)std::min<long long>((n3 + 255) / 256, 148 * 16);
    count_launches(1);
    k_noalloc_scatter<<<blocks, 256, 0, s>>>(v.N, v.nbox, v.cell_of, static_cast<const double2 *>(x_dev), xin);
    TDDA_CUDA_TRY(cudaGetLastError());
    st = apply_external_scratch<double2>(*v.op, T, xin, yin, with_al ? v.al : nullptr, s);
    if (st != TDDA_OK) return st;
    count_launches(1);
    k_noalloc_gather<<<blocks, 256, 0, s>>>(v.N, v.nbox, v.cell_of, yin, static_cast<double2 *>(y_dev));
    TDDA_CUDA_TRY(cudaGetLastError());
    return TDDA_OK;
}
