// Host-side interface of the fused interaction operator and the BiCGSTAB
// driver built on it.
#pragma once

#include "tdda_common.cuh"
#include "../../include/tdda.h"

namespace tdda {

// Per right-hand side solver scalars, resident in device memory.
struct SolverState {
    double2 rho;        // r0 . r   (current r)
    double2 rho_prev;   // r0 . rl  (previous r)
    double2 alpha, zeta, beta;
    double enorm;       // ||E||
    double err;         // ||r|| / ||E|| (recursive residual)
    int it;             // index of the next loop iteration (-1: pre-loop step pending)
    int done;           // 1 once finished
    int status;         // tdda_solve_status
    int iters;          // loop passes executed, as the reference counts them
    int max_iter;
    double tol;
    int stall_limit;    // >0: stop when err has not dropped 10% in this many iterations
    int best_it;
    double best_err;
    int pending;        // fused steps: the last iteration's P update is not applied yet
    int pad_;
    double post_sum;    // true-residual evaluation with ResidualPost: sum over dipole cells of |al x_c|^q
};

// Post-processing fused into the true-residual evaluation of right-hand side 0
// (the last kernel of a refinement solve evaluates the final solution X): the
// internal field E_int = al X / ((2 + eps) / 3) (DDAModel::solveElectricField's
// EResult, src/DDAModel.cpp:1153-1192) and the IntegratedE sum
// S = sum over dipole cells of sum_c |al X_c|^q (src/ObjDDAModel.cpp:103-218).
struct ResidualPost {
    double2 *eres = nullptr;              // [3][nbox] in the box layout, or nullptr: off
    const double2 *diel = nullptr;        // permittivity per cell
    const unsigned char *mask = nullptr;  // dipole cells (nullptr: every cell)
    int q = 2;
};

// Geometry + device buffers of one operator instance (one precision).
template <typename C> struct ConvOperator {
    ConvGeom g{};
    C *ahat = nullptr;     // folded spectral tensor [hy][hx][hz][6], scaled by 1/(Lx Ly Lz)
    const C *const *ahat_rhs = nullptr;  // device table of one tensor per right-hand side, or nullptr
    C *tw = nullptr;       // twiddles exp(-2 pi i j / Lmax), j < Lmax
    C *T = nullptr;        // spectral intermediate, nrhs_cap * 3 * tcomp
    int nrhs_cap = 0;
    double2 *partials = nullptr;  // reduction scratch
    unsigned *counters = nullptr; // last-block counters
    int partial_cap = 0;          // per rhs, per quantity
    const unsigned char *mask = nullptr;  // cell -> in geometry (nullptr: full box)

    tdda_status init(int nx, int ny, int nz, int nrhs_cap);
    void release();
    // y = A x (+ al o x when al != nullptr); x, y: [nrhs][3][nbox]
    tdda_status apply(const C *x, C *y, const C *al, int nrhs, cudaStream_t s);
};

// Device bytes ConvOperator<C>::init allocates (twiddles, spectral
// intermediate, reduction scratch; not the tensor) for esize = sizeof(C).
size_t conv_workspace_bytes(int nx, int ny, int nz, int nrhs_cap, int esize);
// Whether the fused operator supports this grid with nrhs right-hand sides.
bool conv_supported(int nx, int ny, int nz, int nrhs, int esize, std::string &why);

// Vectors of one BiCGSTAB instance ([nrhs][3][nbox] each) + states.
template <typename C> struct Krylov {
    int nrhs = 0;
    long long n = 0;     // 3 * nbox
    C *r = nullptr, *r0 = nullptr, *p = nullptr, *t = nullptr, *Ap = nullptr, *At = nullptr;
    SolverState *st = nullptr;   // device
    SolverState *st_host = nullptr;  // pinned mirror
    unsigned long long *loop = nullptr;  // device loop: passes, start time (device), and a pinned copy
    tdda_status init(long long n3, int nrhs);
    void release();
};

// Options of the device BiCGSTAB driver.
struct KrylovOptions {
    const double *tols = nullptr;  // tolerance per right-hand side (host), or nullptr: one tol for all
    int stall_limit = 0;           // 0: off (reference semantics); else stop after this many
                                   // iterations without a 10% drop of the residual
    size_t dstride = 0;            // diagonal (al, sc) per rhs at [rhs][cell] when nbox, shared when 0
    int graph_steps = 0;           // > 0: capture this many iterations in a CUDA graph and replay it
    bool device_loop = true;       // with graph_steps: one launch of a graph whose while-node repeats the
                                   // iterations until every right-hand side is done (no host polls)
    double time_limit_s = 0.0;     // device loop: end running right-hand sides with TIMEOUT after this long
    bool fused = false;            // fold the P/r update into the next iteration's first pass
                                   // (recursive residual norm from dot products; not the
                                   // reference's exact bookkeeping)
};

// BiCGSTAB of DDAModel::bicgstab on the fused operator: solves
// (A + diag(al)) X = B for nrhs right-hand sides, X holds the initial guess
// (zero when x0_zero).  With sc (Jacobi scale per cell) the operator is
// S A S + diag(al) and al must already be sc^2 al.  Runs fully on the device;
// the host polls the done flags once per chunk of iterations.
template <typename C>
tdda_status bicgstab_device(ConvOperator<C> &op, Krylov<C> &kv, const C *al, const C *sc, const C *B, C *X,
                            int nrhs, bool x0_zero, int max_iter, double tol, cudaStream_t s,
                            tdda_solve_info *info, const KrylovOptions &opts);

// One operator application for one right-hand side whose spectral
// intermediate lives in T_ext (3 * g.tcomp elements) instead of op.T.
template <typename C>
tdda_status apply_external_scratch(const ConvOperator<C> &op, C *T_ext, const C *x, C *y, const C *al,
                                   cudaStream_t s);

// R = B - (A + diag al) X in complex128 (one fused convolution); st receives
// enorm = ||B|| and err = ||R|| / ||B|| per right-hand side; with post
// (eres != nullptr) also E_int of X[0] and st[0].post_sum.
tdda_status residual_c128(ConvOperator<double2> &op, const double2 *al, const double2 *B, const double2 *X,
                          double2 *R, SolverState *st, int nrhs, cudaStream_t s, size_t dstride = 0,
                          const ResidualPost *post = nullptr);

// Times `iters` back-to-back applications of the operator, then each pass
// alone, with CUDA events on stream s: ms_total = mean per application,
// ms_pass[0..2] = mean per launch of pass 1, 2, 3.
template <typename C>
tdda_status profile_apply(ConvOperator<C> &op, const C *x, C *y, const C *al, int nrhs, int iters,
                          cudaStream_t s, double *ms_total, double *ms_pass);

}  // namespace tdda
