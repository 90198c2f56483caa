// Iterative refinement driver (see refine.cuh).
#include <algorithm>
#include <cmath>
#include <vector>

#include "refine.cuh"

namespace tdda {

static unsigned blocks_for(long long n, int bs = 256, unsigned cap = 148 * 16) {
    long long b = (n + bs - 1) / bs;
    return (unsigned)std::max<long long>(1, std::min<long long>(b, cap));
}

// Rin[k] = sc[k] o R[k] * scale[k] in the inner precision (scale 0 parks a
// finished right-hand side; sc == nullptr: no Jacobi scaling)
template <typename C>
__global__ void k_to_inner(long long n, long long nbox, int nrhs, size_t dstride, const double2 *__restrict__ a,
                           const double *__restrict__ scale, const double2 *__restrict__ sc, C *__restrict__ b) {
    long long tot = n * nrhs;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
        const long long k = i / n;
        double s = scale[k];
        double2 v = make_double2(a[i].x * s, a[i].y * s);
        if (sc != nullptr) v = sc[k * dstride + (i % n) % nbox] * v;
        b[i] = from_d<C>(v);
    }
}

// X[k] += w[k] * sc[k] o D[k]
template <typename C>
__global__ void k_axpy_inner(long long n, long long nbox, int nrhs, size_t dstride, const double *__restrict__ w,
                             const double2 *__restrict__ sc, const C *__restrict__ d, double2 *__restrict__ x) {
    long long tot = n * nrhs;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
        const long long k = i / n;
        double s = w[k];
        double2 v = to_d(d[i]);
        if (sc != nullptr) v = sc[k * dstride + (i % n) % nbox] * v;
        x[i].x += s * v.x;
        x[i].y += s * v.y;
    }
}

template <typename C>
void launch_to_inner(long long n, long long nbox, int nrhs, size_t dstride, const double2 *a, const double *scale,
                     const double2 *sc, C *b, cudaStream_t s) {
    count_launches(1);
    k_to_inner<C><<<blocks_for(n * nrhs), 256, 0, s>>>(n, nbox, nrhs, dstride, a, scale, sc, b);
}

template <typename C>
void launch_axpy_inner(long long n, long long nbox, int nrhs, size_t dstride, const double *w, const double2 *sc,
                       const C *d, double2 *x, cudaStream_t s) {
    count_launches(1);
    k_axpy_inner<C><<<blocks_for(n * nrhs), 256, 0, s>>>(n, nbox, nrhs, dstride, w, sc, d, x);
}

template <typename C>
tdda_status refine_solve(const RefineWork<C> &w, const double2 *B, double2 *X, int nrhs, bool x0_zero,
                         int max_iter, double tol, tdda_solve_info *info) {
    const bool single = sizeof(C) == sizeof(float2);
    const long long n = 3 * w.nbox;
    cudaStream_t s = w.s;
    if (x0_zero) TDDA_CUDA_TRY(cudaMemsetAsync(X, 0, sizeof(double2) * n * nrhs, s));
    std::vector<int> done(nrhs, 0), refine(nrhs, 0), inner(nrhs, 0);
    std::vector<double> err(nrhs, 0.0);
    std::vector<int> status(nrhs, TDDA_SOLVE_RUNNING), slow(nrhs, 0);
    std::vector<double> prev(nrhs, 1e300);
    const int max_refine = 12;
    // an inner complex64 solve that has not cut its residual by 10% in this many
    // iterations has reached what single precision can give; refinement takes over
    const int kInnerStall = 150;
    double *h = w.h_part;
    for (int outer = 0; outer <= max_refine; ++outer) {
        tdda_status st = residual_c128(*w.op64, w.al64, B, X, w.Rm, w.st_res, nrhs, s, w.dstride,
                                        w.post.eres != nullptr ? &w.post : nullptr);
        if (st != TDDA_OK) return st;
        TDDA_CUDA_TRY(cudaMemcpyAsync(w.st_res_host, w.st_res, sizeof(SolverState) * nrhs, cudaMemcpyDeviceToHost, s));
        TDDA_CUDA_TRY(cudaStreamSynchronize(s));
        bool all = true;
        for (int k = 0; k < nrhs; ++k) {
            if (done[k]) continue;
            const SolverState &S = w.st_res_host[k];
            err[k] = S.err;
            if (S.enorm == 0.0) {
                TDDA_CUDA_TRY(cudaMemsetAsync(X + (size_t)k * n, 0, sizeof(double2) * n, s));
                done[k] = 1; status[k] = TDDA_SOLVE_ZERO_RHS; err[k] = 0.0;
            } else if (S.err <= tol) {
                done[k] = 1; status[k] = TDDA_SOLVE_CONVERGED;
            } else if (!std::isfinite(S.err)) {
                done[k] = 1; status[k] = TDDA_SOLVE_NONFINITE;
            } else if (outer == max_refine || inner[k] >= max_iter) {
                done[k] = 1; status[k] = TDDA_SOLVE_MAXITER;
            } else {
                // two refinements in a row that do not halve the true residual: stop
                slow[k] = (S.err > 0.5 * prev[k]) ? slow[k] + 1 : 0;
                if (slow[k] >= 2) { done[k] = 1; status[k] = TDDA_SOLVE_STAGNATED; }
            }
            prev[k] = S.err;
            all &= (done[k] != 0);
        }
        if (all) break;
        // one batched inner solve over every unfinished right-hand side, each
        // normalised by its own residual norm (finished ones get a zero RHS)
        std::fill(h, h + 3 * (size_t)nrhs, 0.0);
        int budget = 1;
        for (int k = 0; k < nrhs; ++k) {
            if (done[k]) continue;
            const SolverState &S = w.st_res_host[k];
            const double rn = S.err * S.enorm;
            h[k] = 1.0 / rn;         // scale into the inner RHS
            h[nrhs + k] = rn;        // scale of the correction
            // inner tolerance: what this step must gain, floored where single
            // precision stops paying off
            h[2 * nrhs + k] = std::max(0.5 * tol / S.err, single ? 2e-6 : 0.0);
            budget = std::max(budget, max_iter - inner[k]);
        }
        TDDA_CUDA_TRY(cudaMemcpyAsync(w.d_part, h, sizeof(double) * 3 * nrhs, cudaMemcpyHostToDevice, s));
        launch_to_inner<C>(n, w.nbox, nrhs, w.dstride, w.Rm, w.d_part, w.sc64, w.R, s);
        std::vector<tdda_solve_info> ii(nrhs);
        KrylovOptions o;
        o.tols = h + 2 * nrhs;
        o.stall_limit = kInnerStall;
        o.dstride = w.dstride;
        o.graph_steps = w.graph_steps;
        o.time_limit_s = w.time_limit_s;
        o.fused = true;
        st = bicgstab_device<C>(*w.op, *w.kv, w.al, w.sc, w.R, w.D, nrhs, true, budget, h[2 * nrhs], s, ii.data(), o);
        if (st != TDDA_OK) return st;
        launch_axpy_inner<C>(n, w.nbox, nrhs, w.dstride, w.d_part + nrhs, w.sc64, w.D, X, s);
        TDDA_CUDA_TRY(cudaGetLastError());
        for (int k = 0; k < nrhs; ++k) {
            if (done[k]) continue;
            inner[k] += ii[k].iterations;
            refine[k] += 1;
            if (ii[k].status == TDDA_SOLVE_TIMEOUT) { done[k] = 1; status[k] = TDDA_SOLVE_TIMEOUT; }
        }
    }
    if (info)
        for (int k = 0; k < nrhs; ++k) {
            info[k].iterations = inner[k];
            info[k].error = err[k];
            info[k].status = status[k];
            info[k].refinements = refine[k];
            info[k].inner_iterations = inner[k];
            info[k].true_error = err[k];
        }
    return TDDA_OK;
}

template void launch_to_inner<float2>(long long, long long, int, size_t, const double2 *, const double *,
                                      const double2 *, float2 *, cudaStream_t);
template void launch_to_inner<double2>(long long, long long, int, size_t, const double2 *, const double *,
                                       const double2 *, double2 *, cudaStream_t);
template void launch_axpy_inner<float2>(long long, long long, int, size_t, const double *, const double2 *,
                                        const float2 *, double2 *, cudaStream_t);
template void launch_axpy_inner<double2>(long long, long long, int, size_t, const double *, const double2 *,
                                         const double2 *, double2 *, cudaStream_t);
template tdda_status refine_solve<float2>(const RefineWork<float2> &, const double2 *, double2 *, int, bool, int,
                                          double, tdda_solve_info *);
template tdda_status refine_solve<double2>(const RefineWork<double2> &, const double2 *, double2 *, int, bool, int,
                                           double, tdda_solve_info *);

}  // namespace tdda
