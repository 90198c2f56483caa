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
#include <algorithm>
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

// ----------------------------------------------------------------------------
// One iteration's update of the topology-optimisation loop on the device
// (calculation_scripts/TopoOptCalculation.py:165-209): penalty and its
// gradient (python_bindings/dda_model/binarizers.py:5-34), the penalised
// gradient, Adam with its bias correction inside the moving averages
// (optimizers.py:3-23), the clipped ascent step.  Every product, sum, quotient
// and square root is rounded on its own, in the order the reference's numpy
// expressions evaluate, so the update is the host loop's to the last bit
// (exp in the gaussian penalty aside).
// ----------------------------------------------------------------------------
namespace tdda {

__device__ __forceinline__ void penalty_of(const tdda_ascent_step &c, double x, double &pen, double &pg) {
    if (c.penalty == 0) {            // parabolic: x - x^2, 1 - 2x
        pen = __dsub_rn(x, __dmul_rn(x, x));
        pg = __dsub_rn(1.0, __dmul_rn(2.0, x));
    } else if (c.penalty == 1) {     // gaussian
        const double t = __ddiv_rn(__dsub_rn(x, c.mu), c.sigma);
        pen = __dmul_rn(c.sigma, exp(__dadd_rn(-__ddiv_rn(__dmul_rn(t, t), 2.0), 0.5)));
        pg = __ddiv_rn(__dmul_rn(-__dsub_rn(x, c.mu), pen), __dmul_rn(c.sigma, c.sigma));
    } else {                         // triangular
        pen = x > 0.5 ? __dsub_rn(c.slope, __dmul_rn(c.slope, x)) : __dmul_rn(c.slope, x);
        pg = x > 0.5 ? -c.slope : c.slope;
    }
}

__global__ void k_ascent(long long n, double *__restrict__ x, double *__restrict__ V, double *__restrict__ S,
                         const double *__restrict__ gobj, tdda_ascent_step c, double *__restrict__ pen_out,
                         double *__restrict__ pg_out) {
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x) {
        const double xj = x[j];
        double pen, pg;
        penalty_of(c, xj, pen, pg);
        if (pen_out) pen_out[j] = pen;
        if (pg_out) pg_out[j] = pg;
        const double g = __dsub_rn(__dmul_rn(c.one_minus_coeff, gobj[j]), __dmul_rn(c.coeff, pg));
        const double v = __dadd_rn(__dmul_rn(c.beta1, V[j]), __ddiv_rn(__dmul_rn(c.one_minus_beta1, g), c.bias1));
        const double sq = __dadd_rn(__dmul_rn(c.beta2, S[j]),
                                    __ddiv_rn(__dmul_rn(__dmul_rn(c.one_minus_beta2, g), g), c.bias2));
        V[j] = v;
        S[j] = sq;
        const double stp = __ddiv_rn(v, __dadd_rn(__dsqrt_rn(sq), 1e-8));
        x[j] = fmin(fmax(__dadd_rn(xj, __dmul_rn(c.step, stp)), 0.0), 1.0);
    }
}

// mean of pen[0..n) by one CTA: per-thread strided sums, then a fixed tree
__global__ void k_mean(long long n, const double *__restrict__ v, double *__restrict__ out) {
    __shared__ double sm[256];
    double s = 0.0;
    for (long long j = threadIdx.x; j < n; j += blockDim.x) s += v[j];
    sm[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sm[threadIdx.x] += sm[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sm[0] / (double)n;
}

}  // namespace tdda

extern "C" tdda_status tdda_ascent_step_device(int64_t n, double *params, double *adam_v, double *adam_s,
                                               const double *grad_obj, const tdda_ascent_step *cfg,
                                               double *penalty_out, double *penalty_grad_out,
                                               double *penalty_mean_out, void *stream) {
    using namespace tdda;
    if (n < 1 || !params || !adam_v || !adam_s || !grad_obj || !cfg) {
        set_error("tdda_ascent_step_device: bad argument");
        return TDDA_ERR_BAD_ARG;
    }
    if (cfg->penalty < 0 || cfg->penalty > 2) {
        set_error("penalty must be 0 (parabolic), 1 (gaussian) or 2 (triangular)");
        return TDDA_ERR_BAD_ARG;
    }
    if (penalty_mean_out != nullptr && penalty_out == nullptr) {
        set_error("the penalty mean needs penalty_out");
        return TDDA_ERR_BAD_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned nb = (unsigned)std::min<long long>((n + 255) / 256, 148 * 8);
    count_launches(1);
    k_ascent<<<nb, 256, 0, s>>>(n, params, adam_v, adam_s, grad_obj, *cfg, penalty_out, penalty_grad_out);
    if (penalty_mean_out) {
        count_launches(1);
        k_mean<<<1, 256, 0, s>>>(n, penalty_out, penalty_mean_out);
    }
    TDDA_CUDA_TRY(cudaGetLastError());
    return TDDA_OK;
}

