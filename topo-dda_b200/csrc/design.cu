// Design-density chain on the device: the radius-R cone filter and the tanh
// projection that turn a raw design field into per-dipole densities, and
// their adjoints (no counterpart in the reference, whose Python paths disable
// its own in-plane filter; that legacy filter is in legacy_filter.cu).
//
//   filtered[x,y,z] = sum_o w_o raw[(x-dx) mod nx, (y-dy) mod ny, z-dz] / sum_o w_o
//       over the integer offsets o = (dx,dy,dz) with w_o = R - |o| > 0 and
//       0 <= z - dz < nz (periodic in x and y, truncated and renormalised in z)
//   rho = (tanh(beta eta) + tanh(beta (filtered - eta))) /
//         (tanh(beta eta) + tanh(beta (1 - eta))), clamped to [0, 1]
//
// The raw field and the filtered field are [x][y][z] (z fastest); the
// densities are in dipole order (x fastest), the order the model takes.
// Products and sums are rounded one at a time in the offset order
// dx, dy, dz ascending, as a plain elementwise evaluation does.
#include <cmath>
#include <string>

#include "tdda_common.cuh"
#include "../../include/tdda.h"

namespace tdda {

constexpr int kMaxConeRadius = 6;

__device__ __forceinline__ int wrap(int v, int n) {
    v %= n;
    return v < 0 ? v + n : v;
}

__device__ __forceinline__ double cone_w(double R, int dx, int dy, int dz) {
    return __dsub_rn(R, sqrt((double)(dx * dx + dy * dy + dz * dz)));
}

// the filter's denominator at height z (it depends on z only)
__device__ double cone_den(double R, int r, int z, int nz) {
    double den = 0.0;
    for (int dx = -r; dx <= r; ++dx)
        for (int dy = -r; dy <= r; ++dy)
            for (int dz = -r; dz <= r; ++dz) {
                const double w = cone_w(R, dx, dy, dz);
                if (!(w > 0.0)) continue;
                const int zs = z - dz;
                if (zs < 0 || zs >= nz) continue;
                den = __dadd_rn(den, w);
            }
    return den;
}

__global__ void k_design_forward(int nx, int ny, int nz, double R, int r, double beta, double eta,
                                 const double *__restrict__ raw, double *__restrict__ filtered,
                                 double *__restrict__ rho) {
    const long long n = (long long)nx * ny * nz;
    const double tbe = tanh(beta * eta), pden = tbe + tanh(beta * (1.0 - eta));
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const int z = (int)(c % nz), y = (int)((c / nz) % ny), x = (int)(c / ((long long)nz * ny));
        double num = 0.0, den = 0.0;
        for (int dx = -r; dx <= r; ++dx)
            for (int dy = -r; dy <= r; ++dy) {
                const int xs = wrap(x - dx, nx), ys = wrap(y - dy, ny);
                const double *col = raw + ((long long)xs * ny + ys) * nz;
                for (int dz = -r; dz <= r; ++dz) {
                    const double w = cone_w(R, dx, dy, dz);
                    if (!(w > 0.0)) continue;
                    const int zs = z - dz;
                    if (zs < 0 || zs >= nz) continue;
                    num = __dadd_rn(num, __dmul_rn(w, __ldg(col + zs)));
                    den = __dadd_rn(den, w);
                }
            }
        const double f = num / den;
        filtered[c] = f;
        const double p = (tbe + tanh(beta * (f - eta))) / pden;
        rho[x + (long long)nx * (y + (long long)ny * z)] = fmin(fmax(p, 0.0), 1.0);
    }
}

// t[x,y,z] = grad_rho[dipole(x,y,z)] * dproj/dfiltered / den(z)
__global__ void k_design_back1(int nx, int ny, int nz, double R, int r, double beta, double eta,
                               const double *__restrict__ filtered, const double *__restrict__ grad_rho,
                               double *__restrict__ t) {
    const long long n = (long long)nx * ny * nz;
    const double tbe = tanh(beta * eta), pden = tbe + tanh(beta * (1.0 - eta));
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const int z = (int)(c % nz), y = (int)((c / nz) % ny), x = (int)(c / ((long long)nz * ny));
        const double g = __ldg(grad_rho + x + (long long)nx * (y + (long long)ny * z));
        const double th = tanh(beta * (__ldg(filtered + c) - eta));
        const double p = (tbe + th) / pden;
        // the clamp to [0, 1] passes no gradient where it is active
        const double dp = (p < 0.0 || p > 1.0) ? 0.0 : beta * (1.0 - th * th) / pden;
        t[c] = g * dp / cone_den(R, r, z, nz);
    }
}

// grad_raw[x',y',z'] = sum_o w_o t[(x'+dx) mod nx, (y'+dy) mod ny, z'+dz]
__global__ void k_design_back2(int nx, int ny, int nz, double R, int r, const double *__restrict__ t,
                               double *__restrict__ grad_raw) {
    const long long n = (long long)nx * ny * nz;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const int z = (int)(c % nz), y = (int)((c / nz) % ny), x = (int)(c / ((long long)nz * ny));
        double s = 0.0;
        for (int dx = -r; dx <= r; ++dx)
            for (int dy = -r; dy <= r; ++dy) {
                const int xs = wrap(x + dx, nx), ys = wrap(y + dy, ny);
                const double *col = t + ((long long)xs * ny + ys) * nz;
                for (int dz = -r; dz <= r; ++dz) {
                    const double w = cone_w(R, dx, dy, dz);
                    if (!(w > 0.0)) continue;
                    const int zs = z + dz;
                    if (zs < 0 || zs >= nz) continue;
                    s = __dadd_rn(s, __dmul_rn(w, __ldg(col + zs)));
                }
            }
        grad_raw[c] = s;
    }
}

static unsigned design_blocks(long long n) {
    long long b = (n + 255) / 256;
    return (unsigned)(b < 1 ? 1 : (b < 148 * 16 ? b : 148 * 16));
}

static tdda_status design_args(int nx, int ny, int nz, double radius, double beta, double eta, int &r) {
    if (nx < 1 || ny < 1 || nz < 1) { set_error("grid must be at least 1x1x1"); return TDDA_ERR_BAD_ARG; }
    if (!(radius > 0.0) || radius > kMaxConeRadius) {
        set_error("filter radius must be in (0, " + std::to_string(kMaxConeRadius) + "] cells");
        return TDDA_ERR_BAD_ARG;
    }
    if (!(beta > 0.0) || !(eta > 0.0 && eta < 1.0)) { set_error("need beta > 0 and 0 < eta < 1"); return TDDA_ERR_BAD_ARG; }
    r = (int)std::ceil(radius);
    return TDDA_OK;
}

}  // namespace tdda

using namespace tdda;

extern "C" tdda_status tdda_design_forward_device(int nx, int ny, int nz, double radius, double beta, double eta,
                                                  const double *raw_dev, double *filtered_dev, double *rho_dev,
                                                  void *stream) {
    if (!raw_dev || !filtered_dev || !rho_dev) { set_error("null argument"); return TDDA_ERR_BAD_ARG; }
    int r = 0;
    tdda_status st = design_args(nx, ny, nz, radius, beta, eta, r);
    if (st != TDDA_OK) return st;
    const long long n = (long long)nx * ny * nz;
    count_launches(1);
    k_design_forward<<<design_blocks(n), 256, 0, (cudaStream_t)stream>>>(nx, ny, nz, radius, r, beta, eta, raw_dev,
                                                                        filtered_dev, rho_dev);
    TDDA_CUDA_TRY(cudaGetLastError());
    return TDDA_OK;
}

extern "C" tdda_status tdda_design_backward_device(int nx, int ny, int nz, double radius, double beta, double eta,
                                                   const double *filtered_dev, const double *grad_rho_dev,
                                                   double *grad_raw_dev, double *scratch_dev, void *stream) {
    if (!filtered_dev || !grad_rho_dev || !grad_raw_dev || !scratch_dev) {
        set_error("null argument");
        return TDDA_ERR_BAD_ARG;
    }
    int r = 0;
    tdda_status st = design_args(nx, ny, nz, radius, beta, eta, r);
    if (st != TDDA_OK) return st;
    const long long n = (long long)nx * ny * nz;
    cudaStream_t s = (cudaStream_t)stream;
    count_launches(2);
    k_design_back1<<<design_blocks(n), 256, 0, s>>>(nx, ny, nz, radius, r, beta, eta, filtered_dev, grad_rho_dev,
                                                    scratch_dev);
    k_design_back2<<<design_blocks(n), 256, 0, s>>>(nx, ny, nz, radius, r, scratch_dev, grad_raw_dev);
    TDDA_CUDA_TRY(cudaGetLastError());
    return TDDA_OK;
}
