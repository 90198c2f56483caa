// Polynomial-preconditioned restarted GMRES inside complex128 iterative
// refinement: the solver for the systems where BiCGSTAB stalls (periodic
// structures that fill their unit cell, where the lattice sums couple every
// cell to thousands of images and the spectrum of the scaled operator
// reaches towards zero).
//
//   outer (complex128): R = B - (A + diag al) X, one restart per outer step
//   inner (precision C, Jacobi-scaled operator Ah = S A S + diag(S^2 al)):
//     one GMRES cycle of `restart` steps on Ah p(Ah) u = R^ (right
//     preconditioning), correction D = p(Ah) u, X += ||R|| S D.
//   p is the GMRES polynomial of `degree` Arnoldi steps of Ah on the first
//   residual, applied in product form over its roots (the harmonic Ritz values
//   theta_i, in modified Leja order): 1 - z p(z) = prod (1 - z / theta_i).
//   Each factor is one fused operator application (r <- r - Ah r / theta_i).
//
// The reference solves every system with BiCGSTAB (src/DDAModel.cpp:899-1009);
// this is an alternative solver for the same system, stopping on the same
// relative residual ||E - A P|| / ||E|| (here the true residual).
#pragma once

#include <complex>
#include <vector>

#include "refine.cuh"

namespace tdda {

using cplx = std::complex<double>;

// Device vectors of one polynomial-preconditioned GMRES instance.
template <typename C> struct GmresWork {
    int restart = 0, degree = 0, deflate = 0, nrhs = 0;
    long long n = 0;            // 3 * nbox
    C *V = nullptr, *V2 = nullptr;  // basis and the deflated restart's new basis [restart + 1][nrhs][n]
    C *U = nullptr;             // inner solution accumulated over cycles [nrhs][n]
    C *W = nullptr, *Y = nullptr;  // polynomial work vector and accumulator [nrhs][n]
    double2 *part = nullptr;    // block partial sums
    double2 *h = nullptr;       // device sums [2][nrhs][restart + 1]
    double *nrm = nullptr;      // device norms / reciprocals [2][nrhs]
    double2 *coef = nullptr;    // device [nrhs][restart + 1] combination weights
    double2 *P = nullptr;       // device [nrhs][restart + 1][deflate + 1 + 4] restart combinations
    double2 *h_host = nullptr;  // pinned mirror of h, nrm
    double2 *c_host = nullptr;  // pinned staging of coef
    tdda_status init(long long n3, int nrhs, int restart, int degree, int deflate);
    void release();
    size_t bytes() const;
};

// Options of the solver.
struct GmresOptions {
    int degree = 24;        // polynomial degree (operator applications per preconditioned step)
    int restart = 40;       // GMRES steps per cycle
    int deflate = 0;        // harmonic Ritz vectors kept across restarts (GMRES-DR), < restart
    double floor = 0.0;     // an inner solve stops once it has cut its residual by this much
    // carry the deflation space from one refinement step's inner solve to the
    // next (needs deflate > 0): the next inner solve starts from that space
    // with the new residual added to it, instead of from the residual alone
    bool recycle = false;
};

// Solves (A + diag al) X = B to a TRUE relative residual <= tol per
// right-hand side (w: the refinement workspace of the inner precision C).
// Each refinement step recomputes the true residual R in complex128 and runs
// an inner solve of (deflated) restarted GMRES cycles on the scaled operator
// times the polynomial until the inner residual has dropped by
// max(tol / (2 ||R||/||B||), floor).  info[k].iterations = GMRES steps,
// inner_iterations = inner operator applications, refinements = refinement
// steps.  max_iter bounds the inner operator applications.
template <typename C>
tdda_status pgmres_solve(const RefineWork<C> &w, GmresWork<C> &gw, const double2 *B, double2 *X, int nrhs,
                         bool x0_zero, int max_iter, double tol, const GmresOptions &o, tdda_solve_info *info);

// Mean time of the Gram-Schmidt projection kernel (ms[0], with the block-sum
// kernel) and of the update kernel (ms[1]) against nv basis vectors of n3
// elements, on a scratch basis (measurement support).
template <typename C> tdda_status profile_gram_schmidt(long long n3, int nv, int iters, cudaStream_t s, double *ms);

// --- host linear algebra of the polynomial ----------------------------------
// Eigenvalues of the n x n upper-Hessenberg matrix H (column-major, ld;
// destroyed) by shifted QR; false if it did not converge.
bool hessenberg_eigenvalues(cplx *H, int n, int ld, std::vector<cplx> &ev);
// Harmonic Ritz values of d Arnoldi steps from the (d+1) x d Hessenberg
// matrix Hbar (column-major, ld >= d + 1).
bool harmonic_ritz(const cplx *Hbar, int d, int ld, std::vector<cplx> &theta);
// Modified Leja order, plus extra copies of roots with a large product of
// other factors (stability of the product form).
void leja_order(std::vector<cplx> &theta);

// --- operator pieces the solver uses (operator.cu) ---------------------------
// One factor of the polynomial: r' = r - c (S A S + diag al) r for nrhs
// vectors (sc: Jacobi scale or nullptr).  rin -> rout (may alias), or, when
// wout != nullptr, wout = v0 - r' instead of rout.  y != nullptr:
// y = c r (first) or y += c r.  dstride: the diagonal (sc, al) per
// right-hand side at [rhs][cell] when nonzero, shared when 0.
template <typename C>
tdda_status poly_factor(ConvOperator<C> &op, const C *sc, const C *al, const C *rin, C *rout, C *y, bool first,
                        const C *v0, C *wout, double2 c, int nrhs, size_t dstride, cudaStream_t s);
// y = (S A S + diag al) x for nrhs vectors (sc: Jacobi scale or nullptr).
template <typename C>
tdda_status apply_scaled(ConvOperator<C> &op, const C *sc, const C *al, const C *x, C *y, int nrhs, size_t dstride,
                         cudaStream_t s);

}  // namespace tdda
