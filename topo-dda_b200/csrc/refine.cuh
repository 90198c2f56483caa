// Iterative refinement on the true complex128 residual around an inner
// BiCGSTAB in complex64 (mixed precision) or complex128, optionally
// Jacobi-scaled.  Shared by the DDAModel state machine and the serving engine.
#pragma once

#include "operator.cuh"

namespace tdda {

template <typename C> struct RefineWork {
    ConvOperator<double2> *op64 = nullptr;  // the true operator (complex128)
    const double2 *al64 = nullptr;          // its diagonal 1/alpha
    ConvOperator<C> *op = nullptr;          // inner operator (its tensor in precision C)
    Krylov<C> *kv = nullptr;
    const C *al = nullptr;                  // inner diagonal (sc^2 al under Jacobi scaling)
    const C *sc = nullptr;                  // inner Jacobi scale, or nullptr
    const double2 *sc64 = nullptr;          // the same scale in complex128, or nullptr
    C *R = nullptr, *D = nullptr;           // inner right-hand sides / corrections [nrhs][3][nbox]
    double2 *Rm = nullptr;                  // true residual [nrhs][3][nbox]
    SolverState *st_res = nullptr;          // device, nrhs
    SolverState *st_res_host = nullptr;     // pinned, nrhs
    double *d_part = nullptr;               // device, >= 3 nrhs doubles
    double *h_part = nullptr;               // pinned, >= 3 nrhs doubles
    long long nbox = 0;
    size_t dstride = 0;                     // diagonals per rhs ([rhs][cell]) when nbox
    int graph_steps = 0;                    // inner BiCGSTAB: iterations per CUDA graph (0: none)
    double time_limit_s = 0.0;              // inner BiCGSTAB: device-side time limit (0: none)
    cudaStream_t s = nullptr;
    // E_int and the objective sum of X[0], fused into every true-residual
    // evaluation (the last one evaluates the returned solution); off when
    // post.eres is null
    ResidualPost post{};
};

// Solves (A + diag al) X = B to a TRUE relative residual <= tol per
// right-hand side: R = B - A X in complex128, inner solve A D = R / ||R|| in
// precision C, X += ||R|| D, repeated.  info[k].iterations counts inner
// iterations, info[k].refinements the corrections.
template <typename C>
tdda_status refine_solve(const RefineWork<C> &w, const double2 *B, double2 *X, int nrhs, bool x0_zero,
                         int max_iter, double tol, tdda_solve_info *info);

// b[k] = sc[k] o a[k] * scale[k] in precision C (scale: device, one per rhs;
// sc: complex128 scale per cell or nullptr), for nrhs vectors of n = 3 nbox
template <typename C>
void launch_to_inner(long long n, long long nbox, int nrhs, size_t dstride, const double2 *a, const double *scale,
                     const double2 *sc, C *b, cudaStream_t s);
// x[k] += w[k] * sc[k] o d[k] with d in precision C, x in complex128
template <typename C>
void launch_axpy_inner(long long n, long long nbox, int nrhs, size_t dstride, const double *w, const double2 *sc,
                       const C *d, double2 *x, cudaStream_t s);

}  // namespace tdda
