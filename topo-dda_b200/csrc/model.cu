// The DDAModel state machine behind the C ABI (include/tdda.h).
//
// Reference: src/DDAModel.cpp (constructor :79-333, parameter map :163-247,
// polarisability :319-328/:1122-1151, solve :874-885, E_int :1185-1192,
// objective via src/ObjDDAModel.cpp:103-218, gradient :398-578).  Host code
// keeps the O(N) bookkeeping (parameter map, segmented sums over the
// parameter -> dipole lists); everything on the solve path runs on the device.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "lattice.cuh"
#include "physics.cuh"
#include "model_view.cuh"
#include "operator.cuh"
#include "refine.cuh"
#include "gmres.cuh"
#include "legacy_filter.cuh"

namespace tdda {

static std::atomic<long long> g_launches{0};
static thread_local bool g_capturing = false;
void count_launches(long long n) {
    if (!g_capturing) g_launches.fetch_add(n, std::memory_order_relaxed);
}
void set_capturing(bool on) { g_capturing = on; }
long long launches_total() { return g_launches.load(std::memory_order_relaxed); }

static thread_local std::string g_err;
void set_error(const std::string &msg) { g_err = msg; }
const char *get_error() { return g_err.c_str(); }

// ----------------------------------------------------------------------------
// device helpers of the model layer
// ----------------------------------------------------------------------------
__global__ void k_alpha(long long nbox, const double *__restrict__ rho, const unsigned char *__restrict__ mask,
                        AlphaParams A, double2 *__restrict__ al, float2 *__restrict__ al32,
                        double2 *__restrict__ diel) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nbox; i += (long long)gridDim.x * blockDim.x) {
        double2 a, e;
        if (mask != nullptr && mask[i] == 0) {
            a = make_double2(1.0, 0.0);
            e = make_double2(1.0, 0.0);
        } else {
            e = diel_of(rho[i], A);
            a = inv_alpha(e, A);
        }
        al[i] = a;
        diel[i] = e;
        if (al32 != nullptr) al32[i] = make_float2((float)a.x, (float)a.y);
    }
}

// dipole order (3*i + c, interleaved complex) <-> internal [rhs][c][cell]
__global__ void k_scatter(int nrhs, long long N, long long nbox, const long long *__restrict__ cell_of,
                          const double2 *__restrict__ ext, double2 *__restrict__ in) {
    long long tot = (long long)nrhs * N * 3;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x) {
        long long k = e / (3 * N), rem = e - k * 3 * N;
        long long i = rem / 3;
        int c = (int)(rem - i * 3);
        in[((size_t)k * 3 + c) * nbox + cell_of[i]] = ext[e];
    }
}

// count of densities outside [0, 1] (NaN included)
__global__ void k_rho_check(long long N, const double *__restrict__ rho, unsigned *__restrict__ bad) {
    unsigned c = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        const double v = rho[i];
        if (!(v >= 0.0 && v <= 1.0)) ++c;
    }
    if (c) atomicAdd(bad, c);
}

// density per cell from per-dipole densities (cells without a dipole keep 0)
__global__ void k_rho_scatter(long long N, const long long *__restrict__ cell_of, const double *__restrict__ rho,
                              double *__restrict__ d_rho) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
        d_rho[cell_of[i]] = rho[i];
}

// per-dipole values from per-cell values
__global__ void k_cell_to_dipole(long long N, const long long *__restrict__ cell_of, const double *__restrict__ v,
                                 double *__restrict__ out) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
        out[i] = v[cell_of[i]];
}

__global__ void k_gather(int nrhs, long long N, long long nbox, const long long *__restrict__ cell_of,
                         const double2 *__restrict__ in, double2 *__restrict__ ext) {
    long long tot = (long long)nrhs * N * 3;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x) {
        long long k = e / (3 * N), rem = e - k * 3 * N;
        long long i = rem / 3;
        int c = (int)(rem - i * 3);
        ext[e] = in[((size_t)k * 3 + c) * nbox + cell_of[i]];
    }
}

// EResult = E_int = al P / ((2 + eps) / 3)   (src/DDAModel.cpp:1185-1192)
__global__ void k_eresult(long long nbox, const double2 *__restrict__ P, const double2 *__restrict__ al,
                          const double2 *__restrict__ diel, double2 *__restrict__ Eres) {
    long long tot = 3 * nbox;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x) {
        long long cell = e % nbox;
        double2 lf = make_double2((2.0 + diel[cell].x) / 3.0, diel[cell].y / 3.0);
        Eres[e] = cdiv(cmul_d(al[cell], P[e]), lf);
    }
}

__device__ __forceinline__ double powabs(double2 z, int q) {
    double a = hypot(z.x, z.y);
    if (q == 2) return a * a;
    return pow(a, (double)q);
}

// per-block partial sums of sum_c |al P_c|^q over dipole cells
__global__ void k_objective(long long nbox, const double2 *__restrict__ P, const double2 *__restrict__ al,
                            const unsigned char *__restrict__ mask, int q, double *__restrict__ part) {
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nbox; i += (long long)gridDim.x * blockDim.x) {
        if (mask != nullptr && mask[i] == 0) continue;
        double2 a = al[i];
        for (int c = 0; c < 3; ++c) s += powabs(cmul_d(a, P[(size_t)c * nbox + i]), q);
    }
    __shared__ double red[32];
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
        if (threadIdx.x == 0) part[blockIdx.x] = s;
    }
}

// Finite-difference partials of the reference gradient
// (devx_and_Adevxp src/DDAModel.cpp:471-536, devp :538-578), per dipole cell:
//   dS[cell]     = sum_c |al' P_c|^q - |al P_c|^q  with al' = al(rho + sign eps)
//   change[cell] = (al' - al) / (sign eps)
//   devp[c][cell]= (log(S - base + c_re) - J0)/eps + (log(S - base + c_im) - J0)/(i eps)
struct GradFD {
    AlphaParams A;
    double eps, J0, S;
    int q;
};

__global__ void k_grad_fd(long long nbox, const double *__restrict__ rho, const unsigned char *__restrict__ mask,
                          const double2 *__restrict__ P, const double2 *__restrict__ al, GradFD G,
                          double *__restrict__ dS, double2 *__restrict__ change, double2 *__restrict__ devp) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nbox; i += (long long)gridDim.x * blockDim.x) {
        if (mask != nullptr && mask[i] == 0) {
            dS[i] = 0.0;
            change[i] = make_double2(0.0, 0.0);
            for (int c = 0; c < 3; ++c) devp[(size_t)c * nbox + i] = make_double2(0.0, 0.0);
            continue;
        }
        const double r0 = rho[i];
        const double sgn = r0 >= G.eps ? -1.0 : 1.0;
        const double2 a = al[i];
        const double2 an = inv_alpha(diel_of(r0 + sgn * G.eps, G.A), G.A);
        double old = 0.0, nw = 0.0;
        double2 Pc[3];
        double cold[3];
        for (int c = 0; c < 3; ++c) {
            Pc[c] = P[(size_t)c * nbox + i];
            cold[c] = powabs(cmul_d(a, Pc[c]), G.q);
            old += cold[c];
            nw += powabs(cmul_d(an, Pc[c]), G.q);
        }
        dS[i] = nw - old;
        const double se = sgn * G.eps;
        change[i] = make_double2((an.x - a.x) / se, (an.y - a.y) / se);
        const double base = G.S - old;
        for (int c = 0; c < 3; ++c) {
            double cre = old - cold[c] + powabs(cmul_d(a, make_double2(Pc[c].x + G.eps, Pc[c].y)), G.q);
            double cim = old - cold[c] + powabs(cmul_d(a, make_double2(Pc[c].x, Pc[c].y + G.eps)), G.q);
            double fre = (log(base + cre) - G.J0) / G.eps;
            double fim = (log(base + cim) - G.J0) / G.eps;
            // fre + fim / (i) = fre - i fim
            devp[(size_t)c * nbox + i] = make_double2(fre, -fim);
        }
    }
}

// prod[cell] = change[cell] * sum_c lambda_c P_c  (non-conjugated, src/DDAModel.cpp:445-455)
__global__ void k_grad_mult(long long nbox, const double2 *__restrict__ lam, const double2 *__restrict__ P,
                            const double2 *__restrict__ change, double2 *__restrict__ prod) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nbox; i += (long long)gridDim.x * blockDim.x) {
        double2 s = make_double2(0.0, 0.0);
        for (int c = 0; c < 3; ++c) {
            double2 v = cmul_d(lam[(size_t)c * nbox + i], P[(size_t)c * nbox + i]);
            s.x += v.x;
            s.y += v.y;
        }
        prod[i] = cmul_d(s, change[i]);
    }
}

// Jacobi scaling of the operator A + diag(al): D = al + a0 (a0: mean of the
// diagonal of the zero-offset lattice entry), sc = D^(-1/2), alS = sc^2 al.
__global__ void k_jacobi(long long nbox, const double2 *__restrict__ al, const unsigned char *__restrict__ mask,
                         double2 a0, double2 *__restrict__ sc, double2 *__restrict__ alS,
                         float2 *__restrict__ sc32, float2 *__restrict__ alS32) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nbox; i += (long long)gridDim.x * blockDim.x) {
        double2 s = make_double2(1.0, 0.0), a = al[i];
        if (mask == nullptr || mask[i] != 0) s = jacobi_scale(a, a0);
        double2 as = cmul_d(cmul_d(s, s), a);
        sc[i] = s;
        alS[i] = as;
        if (sc32 != nullptr) {
            sc32[i] = make_float2((float)s.x, (float)s.y);
            alS32[i] = make_float2((float)as.x, (float)as.y);
        }
    }
}


// adjoint right-hand side dJ/dx - i dJ/dy of J = log S, S = sum |al P|^q:
// q |al|^q |P|^(q-2) conj(P) / S
__global__ void k_adjoint_rhs(long long nbox, const double2 *__restrict__ P, const double2 *__restrict__ al,
                              const unsigned char *__restrict__ mask, int q, double S, double2 *__restrict__ rhs) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nbox; i += (long long)gridDim.x * blockDim.x) {
        const bool on = mask == nullptr || mask[i] != 0;
        const double2 a = al[i];
        const double aq = pow(hypot(a.x, a.y), (double)q);
        for (int c = 0; c < 3; ++c) {
            double2 p = P[(size_t)c * nbox + i];
            double w = 0.0;
            if (on) {
                double ap = hypot(p.x, p.y);
                w = q == 2 ? 2.0 * aq / S : (ap > 0 ? q * aq * pow(ap, (double)(q - 2)) / S : 0.0);
            }
            rhs[(size_t)c * nbox + i] = make_double2(w * p.x, -w * p.y);
        }
    }
}

// grad = explicit - Re(sum_c lambda_c al' P_c), explicit = sum_c q |al|^(q-2) |P_c|^q Re(conj(al) al') / S
__global__ void k_grad_analytic(long long nbox, const double *__restrict__ rho, const unsigned char *__restrict__ mask,
                                const double2 *__restrict__ P, const double2 *__restrict__ al,
                                const double2 *__restrict__ diel, const double2 *__restrict__ lam, AlphaParams A,
                                int q, double S, double *__restrict__ grad) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nbox; i += (long long)gridDim.x * blockDim.x) {
        if (mask != nullptr && mask[i] == 0) { grad[i] = 0.0; continue; }
        const double2 a = al[i];
        const double2 da = dal_drho(diel[i], A);
        const double ra = a.x * da.x + a.y * da.y;  // Re(conj(a) a')
        const double am = hypot(a.x, a.y);
        double ex = 0.0, im = 0.0;
        for (int c = 0; c < 3; ++c) {
            double2 p = P[(size_t)c * nbox + i];
            double ap = hypot(p.x, p.y);
            ex += (q == 2 ? 2.0 * ap * ap : q * pow(am, (double)(q - 2)) * pow(ap, (double)q)) * ra;
            double2 v = cmul_d(lam[(size_t)c * nbox + i], cmul_d(da, p));
            im += v.x;
        }
        grad[i] = ex / S - im;
    }
}

// ---- observation patch -----------------------------------------------------
// E_obs = E_inc(r_o) - sum_j G(r_o - r_j) P_j with G the same damped lattice
// sum as the operator (offsets in grid units, tensor on the offset box).
struct PatchGeo {
    int nx, ny, nz;
    int lox, loy, loz, bx, by, bz;
};

__device__ __forceinline__ const double2 *gobs_at(const double2 *G, const PatchGeo &pg, int dx, int dy, int dz) {
    return G + ((size_t)((dx - pg.lox) * pg.by + (dy - pg.loy)) * pg.bz + (dz - pg.loz)) * 6;
}

// G (symmetric, components xx xy xz yy yz zz) times v, row c
__device__ __forceinline__ double2 grow(const double2 *g, int c, double2 vx, double2 vy, double2 vz) {
    const int i0 = c == 0 ? 0 : c == 1 ? 1 : 2;
    const int i1 = c == 0 ? 1 : c == 1 ? 3 : 4;
    const int i2 = c == 0 ? 2 : c == 1 ? 4 : 5;
    double2 a = cmul_d(g[i0], vx), b = cmul_d(g[i1], vy), d = cmul_d(g[i2], vz);
    return make_double2(a.x + b.x + d.x, a.y + b.y + d.y);
}

// one block per observation point; deterministic block reduction
__global__ void k_patch_field(int nobs, const int *__restrict__ obs, PatchGeo pg, const unsigned char *__restrict__ mask,
                              const double2 *__restrict__ P, long long nbox, const double2 *__restrict__ G,
                              const double2 *__restrict__ Einc_obs, double2 *__restrict__ Eobs) {
    const int o = blockIdx.x;
    const int ox = obs[3 * o], oy = obs[3 * o + 1], oz = obs[3 * o + 2];
    double2 acc[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
    const int nyz = pg.ny * pg.nz;
    for (long long cell = threadIdx.x; cell < nbox; cell += blockDim.x) {
        if (mask != nullptr && mask[cell] == 0) continue;
        const int x = (int)(cell / nyz), rem = (int)(cell - (long long)x * nyz);
        const int y = rem / pg.nz, z = rem - y * pg.nz;
        const double2 *g = gobs_at(G, pg, ox - x, oy - y, oz - z);
        const double2 px = P[cell], py = P[nbox + cell], pz = P[2 * nbox + cell];
        for (int c = 0; c < 3; ++c) {
            double2 v = grow(g, c, px, py, pz);
            acc[c].x += v.x;
            acc[c].y += v.y;
        }
    }
    __shared__ double2 red[3][32];
    for (int c = 0; c < 3; ++c)
        for (int off = 16; off > 0; off >>= 1) {
            acc[c].x += __shfl_xor_sync(0xffffffffu, acc[c].x, off);
            acc[c].y += __shfl_xor_sync(0xffffffffu, acc[c].y, off);
        }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (lane == 0)
        for (int c = 0; c < 3; ++c) red[c][wid] = acc[c];
    __syncthreads();
    if (wid == 0) {
        for (int c = 0; c < 3; ++c) {
            double2 v = lane < nw ? red[c][lane] : make_double2(0, 0);
            for (int off = 16; off > 0; off >>= 1) {
                v.x += __shfl_xor_sync(0xffffffffu, v.x, off);
                v.y += __shfl_xor_sync(0xffffffffu, v.y, off);
            }
            if (lane == 0) {
                const double2 e = Einc_obs[3 * o + c];
                Eobs[3 * o + c] = make_double2(e.x - v.x, e.y - v.y);
            }
        }
    }
}

// adjoint right-hand side of J = (1/nobs) sum_o |E_o|^2:
// dJ/dx - i dJ/dy at dipole j = -(2/nobs) sum_o G(r_o - r_j) conj(E_o)
__global__ void k_patch_adjoint_rhs(int nobs, const int *__restrict__ obs, PatchGeo pg,
                                    const unsigned char *__restrict__ mask, long long nbox,
                                    const double2 *__restrict__ G, const double2 *__restrict__ Eobs,
                                    double2 *__restrict__ rhs) {
    const int nyz = pg.ny * pg.nz;
    const double w = -2.0 / nobs;
    for (long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x; cell < nbox;
         cell += (long long)gridDim.x * blockDim.x) {
        double2 acc[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
        if (mask == nullptr || mask[cell] != 0) {
            const int x = (int)(cell / nyz), rem = (int)(cell - (long long)x * nyz);
            const int y = rem / pg.nz, z = rem - y * pg.nz;
            for (int o = 0; o < nobs; ++o) {
                const double2 *g = gobs_at(G, pg, obs[3 * o] - x, obs[3 * o + 1] - y, obs[3 * o + 2] - z);
                const double2 ex = conj(Eobs[3 * o]), ey = conj(Eobs[3 * o + 1]), ez = conj(Eobs[3 * o + 2]);
                for (int c = 0; c < 3; ++c) {
                    double2 v = grow(g, c, ex, ey, ez);
                    acc[c].x += v.x;
                    acc[c].y += v.y;
                }
            }
        }
        for (int c = 0; c < 3; ++c) rhs[(size_t)c * nbox + cell] = make_double2(w * acc[c].x, w * acc[c].y);
    }
}

// gradient of an objective without explicit density dependence:
// dJ/drho_j = -Re(sum_c lambda_jc al'_j P_jc)
__global__ void k_grad_implicit(long long nbox, const unsigned char *__restrict__ mask, const double2 *__restrict__ P,
                                const double2 *__restrict__ diel, const double2 *__restrict__ lam, AlphaParams A,
                                double *__restrict__ grad) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nbox; i += (long long)gridDim.x * blockDim.x) {
        if (mask != nullptr && mask[i] == 0) { grad[i] = 0.0; continue; }
        const double2 da = dal_drho(diel[i], A);
        double s = 0.0;
        for (int c = 0; c < 3; ++c) s += cmul_d(lam[(size_t)c * nbox + i], cmul_d(da, P[(size_t)c * nbox + i])).x;
        grad[i] = -s;
    }
}

static unsigned grid_for(long long n, int bs = 256, unsigned cap = 148 * 16) {
    long long g = (n + bs - 1) / bs;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (unsigned)g;
}

}  // namespace tdda

using namespace tdda;

// ----------------------------------------------------------------------------
// the model
// ----------------------------------------------------------------------------
struct tdda_model {
    // constructor arguments
    int Nx = 0, Ny = 0, Nz = 0, N = 0;
    double d = 0, lam = 0, nback = 1, K = 0, E0 = 1;
    double nK[3]{}, nE0[3]{};
    double2 mat[2]{};
    int MAXm = 0, MAXn = 0;
    double Lm = 0, Ln = 0;  // lengths (d included)
    int method = 0;
    double delta = 0.1;
    int powNum = 2;
    int precision = TDDA_PREC_C128;
    int verbose = 0;
    AlphaParams ap{};
    // host bookkeeping
    long long nbox = 0;
    std::vector<int32_t> geometry;
    std::vector<long long> cell_of;       // dipole -> cell
    std::vector<int> geometryPara;        // dipole -> parameter
    std::vector<int> p2g_off, p2g_idx;    // parameter -> dipoles (CSR)
    int NFpara = 0;
    std::vector<double> parameters;
    double E_int = 0.0;                   // objective state of the last calculateObjective
    bool per_dipole = false;              // densities set per dipole (tdda_set_densities)
    std::vector<double> rho_dipole;       // per-dipole densities when per_dipole
    bool rho_host_stale = false;          // set on the device since: rho_dipole must be read back
    // device
    cudaStream_t stream = nullptr;
    ConvOperator<double2> op;
    ConvOperator<float2> op32;
    Krylov<double2> kv;
    Krylov<float2> kv32;
    int kv_nrhs = 0, kv32_nrhs = 0;
    long long *d_cell = nullptr;
    unsigned char *d_mask = nullptr;
    double *d_rho = nullptr;        // density per cell
    double2 *al = nullptr, *diel = nullptr;
    float2 *al32 = nullptr;
    double2 *Einc = nullptr;        // incident field [3][nbox]
    double2 *P = nullptr;           // polarisation [3][nbox]
    double2 *Eres = nullptr;        // EResult [3][nbox]
    // Generation of (P, 1/alpha): bumped by every solve into P and every
    // polarisability update.  post_gen == gen: Eres and post_obj (the
    // IntegratedE sum of P) came from the solve's last true-residual kernel.
    unsigned long long gen = 1, post_gen = 0;
    double post_obj = 0.0;
    double2 *ext = nullptr;         // dipole-order staging, 3N (grows for batches)
    long long ext_cap = 0;
    double2 *bufB = nullptr, *bufX = nullptr;  // batch staging [nrhs][3][nbox]
    int buf_nrhs = 0;
    // refinement workspace (mixed precision, or preconditioned complex128)
    double2 *Rm = nullptr;
    float2 *R32 = nullptr, *D32 = nullptr;
    int mixed_nrhs = 0;
    double2 *R64 = nullptr, *D64 = nullptr;
    int refine64_nrhs = 0, res_nrhs = 0;
    // Jacobi scaling: 0 off (the reference's plain BiCGSTAB), 1 on
    int precond = 0;
    double2 a0{};                          // mean diagonal of the zero-offset tensor entry
    double2 *sc64 = nullptr, *alS64 = nullptr;
    float2 *sc32 = nullptr, *alS32 = nullptr;
    double *d_grad = nullptr;              // per-cell gradient scratch
    // the parameter map on the device (built on first use): parameter of each
    // dipole, and each parameter's dipoles in dipole order (CSR)
    int32_t *d_pmap = nullptr, *d_pptr = nullptr, *d_pidx = nullptr;
    unsigned *d_flag = nullptr, *h_flag = nullptr;  // density check count (device, pinned)
    SolverState *st_res = nullptr, *st_res_host = nullptr;
    double *d_part = nullptr, *h_part = nullptr;
    // lattice inputs kept for later tensors (observation patches)
    LatticeParams lat{};
    std::vector<double> si_h, ci_h;
    // observation patch: E_obs = E_inc(r_obs) - sum_j G(r_obs - r_j) P_j
    int nobs = 0;
    int *d_obs = nullptr;        // 3 ints per observation point (grid units)
    double2 *Gobs = nullptr;     // lattice sums on the offset box [bx][by][bz][6]
    int obs_lo[3]{}, obs_n[3]{};
    double2 *Einc_obs = nullptr; // [nobs][3]
    double2 *Eobs = nullptr;     // [nobs][3]
    // the reference's legacy design filter (use_filter)
    LegacyFilter lfilter;
    double time_limit_s = 0.0;             // device-side time limit of BiCGSTAB solves
    // solver of later solves: 0 BiCGSTAB, 1 polynomial-preconditioned GMRES
    int solver = 0;
    GmresOptions gopt{};
    GmresWork<double2> gw64;
    GmresWork<float2> gw32;
    // stats
    double lattice_ms = 0, fft_ms = 0;
    long long device_bytes = 0;

    ~tdda_model() {
        op.release();
        op32.release();
        kv.release();
        kv32.release();
        gw64.release();
        gw32.release();
        void *bufs[] = {d_cell, d_mask, d_rho,  al,  diel, al32,  Einc, P,     Eres,  ext,   bufB,     bufX,
                        Rm,     R32,    D32,    st_res, d_part, R64, D64,  sc64, alS64, sc32, alS32, d_obs,
                        Gobs,   Einc_obs, Eobs, d_grad, d_flag, d_pmap, d_pptr, d_pidx};
        for (void *b : bufs) cudaFree(b);
        cudaFreeHost(h_flag);
        cudaFreeHost(st_res_host);
        cudaFreeHost(h_part);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace tdda {
ModelView model_view(const tdda_model *m) {
    return {&m->op, m->al, m->d_cell, m->d_mask, (long long)m->N, m->nbox};
}
}  // namespace tdda

#define TRY(x)                                \
    do {                                      \
        tdda_status _s = (x);                 \
        if (_s != TDDA_OK) return _s;         \
    } while (0)

static tdda_status bad(const std::string &msg) {
    set_error(msg);
    return TDDA_ERR_BAD_ARG;
}

static tdda_status ensure_ext(tdda_model *m, long long n) {
    if (m->ext_cap >= n) return TDDA_OK;
    cudaFree(m->ext);
    m->ext = nullptr;
    TDDA_CUDA_TRY(cudaMalloc(&m->ext, sizeof(double2) * n));
    m->ext_cap = n;
    return TDDA_OK;
}

static tdda_status ensure_batch(tdda_model *m, int nrhs) {
    if (m->buf_nrhs >= nrhs) return TDDA_OK;
    cudaFree(m->bufB);
    cudaFree(m->bufX);
    m->bufB = m->bufX = nullptr;
    size_t bytes = sizeof(double2) * 3 * (size_t)m->nbox * nrhs;
    TDDA_CUDA_TRY(cudaMalloc(&m->bufB, bytes));
    TDDA_CUDA_TRY(cudaMalloc(&m->bufX, bytes));
    if (m->N < m->nbox) {
        TDDA_CUDA_TRY(cudaMemset(m->bufB, 0, bytes));
        TDDA_CUDA_TRY(cudaMemset(m->bufX, 0, bytes));
    }
    m->buf_nrhs = nrhs;
    return TDDA_OK;
}

static tdda_status ensure_op_cap(tdda_model *m, int nrhs) {
    if (m->op.nrhs_cap >= nrhs) return TDDA_OK;
    // grow the spectral intermediate and the reduction scratch
    cudaFree(m->op.T);
    m->op.T = nullptr;
    TDDA_CUDA_TRY(cudaMalloc(&m->op.T, sizeof(double2) * (size_t)nrhs * 3 * m->op.g.tcomp));
    cudaFree(m->op.partials);
    cudaFree(m->op.counters);
    m->op.partials = nullptr;
    m->op.counters = nullptr;
    TDDA_CUDA_TRY(cudaMalloc(&m->op.partials, sizeof(double2) * (size_t)m->op.partial_cap * nrhs));
    TDDA_CUDA_TRY(cudaMalloc(&m->op.counters, sizeof(unsigned) * nrhs));
    TDDA_CUDA_TRY(cudaMemset(m->op.counters, 0, sizeof(unsigned) * nrhs));
    m->op.nrhs_cap = nrhs;
    return TDDA_OK;
}

static tdda_status ensure_krylov(tdda_model *m, int nrhs) {
    if (m->kv_nrhs < nrhs) {
        m->kv.release();
        TRY(m->kv.init(3 * m->nbox, nrhs));
        if (m->N < m->nbox) {
            size_t bytes = sizeof(double2) * 3 * (size_t)m->nbox * nrhs;
            double2 *b[6] = {m->kv.r, m->kv.r0, m->kv.p, m->kv.t, m->kv.Ap, m->kv.At};
            for (auto p : b) TDDA_CUDA_TRY(cudaMemset(p, 0, bytes));
        }
        m->kv_nrhs = nrhs;
    }
    return ensure_op_cap(m, nrhs);
}

static tdda_status ensure_mixed(tdda_model *m, int nrhs) {
    TRY(ensure_op_cap(m, nrhs));  // the complex128 residual runs on the batch too
    if (m->kv32_nrhs < nrhs) {
        m->kv32.release();
        TRY(m->kv32.init(3 * m->nbox, nrhs));
        if (m->N < m->nbox) {
            size_t bytes = sizeof(float2) * 3 * (size_t)m->nbox * nrhs;
            float2 *b[6] = {m->kv32.r, m->kv32.r0, m->kv32.p, m->kv32.t, m->kv32.Ap, m->kv32.At};
            for (auto p : b) TDDA_CUDA_TRY(cudaMemset(p, 0, bytes));
        }
        m->kv32_nrhs = nrhs;
    }
    if (m->op32.nrhs_cap < nrhs) {
        cudaFree(m->op32.T);
        m->op32.T = nullptr;
        TDDA_CUDA_TRY(cudaMalloc(&m->op32.T, sizeof(float2) * (size_t)nrhs * 3 * m->op32.g.tcomp));
        cudaFree(m->op32.partials);
        cudaFree(m->op32.counters);
        TDDA_CUDA_TRY(cudaMalloc(&m->op32.partials, sizeof(double2) * (size_t)m->op32.partial_cap * nrhs));
        TDDA_CUDA_TRY(cudaMalloc(&m->op32.counters, sizeof(unsigned) * nrhs));
        TDDA_CUDA_TRY(cudaMemset(m->op32.counters, 0, sizeof(unsigned) * nrhs));
        m->op32.nrhs_cap = nrhs;
    }
    if (m->mixed_nrhs < nrhs) {
        cudaFree(m->R32); cudaFree(m->D32);
        m->R32 = m->D32 = nullptr;
        size_t n = 3 * (size_t)m->nbox * nrhs;
        TDDA_CUDA_TRY(cudaMalloc(&m->R32, sizeof(float2) * n));
        TDDA_CUDA_TRY(cudaMalloc(&m->D32, sizeof(float2) * n));
        TDDA_CUDA_TRY(cudaMemset(m->R32, 0, sizeof(float2) * n));
        TDDA_CUDA_TRY(cudaMemset(m->D32, 0, sizeof(float2) * n));
        m->mixed_nrhs = nrhs;
    }
    return TDDA_OK;
}

// complex128 residual + per-RHS states shared by both refinement variants
static tdda_status ensure_residual(tdda_model *m, int nrhs) {
    static_assert(sizeof(SolverState) % 8 == 0, "SolverState layout");
    TRY(ensure_op_cap(m, nrhs));
    if (m->st_res != nullptr && m->res_nrhs >= nrhs) return TDDA_OK;
    cudaFree(m->Rm); cudaFree(m->st_res); cudaFreeHost(m->st_res_host);
    m->Rm = nullptr; m->st_res = nullptr; m->st_res_host = nullptr;
    size_t n = 3 * (size_t)m->nbox * nrhs;
    TDDA_CUDA_TRY(cudaMalloc(&m->Rm, sizeof(double2) * n));
    TDDA_CUDA_TRY(cudaMemset(m->Rm, 0, sizeof(double2) * n));
    TDDA_CUDA_TRY(cudaMalloc(&m->st_res, sizeof(SolverState) * nrhs));
    TDDA_CUDA_TRY(cudaMallocHost(&m->st_res_host, sizeof(SolverState) * nrhs));
    m->res_nrhs = nrhs;
    return TDDA_OK;
}

static tdda_status ensure_refine(tdda_model *m, int nrhs, float2 *) {
    TRY(ensure_residual(m, nrhs));
    return ensure_mixed(m, nrhs);
}

static tdda_status ensure_refine(tdda_model *m, int nrhs, double2 *) {
    TRY(ensure_residual(m, nrhs));
    TRY(ensure_krylov(m, nrhs));
    if (m->refine64_nrhs >= nrhs) return TDDA_OK;
    cudaFree(m->R64); cudaFree(m->D64);
    m->R64 = m->D64 = nullptr;
    size_t n = 3 * (size_t)m->nbox * nrhs;
    TDDA_CUDA_TRY(cudaMalloc(&m->R64, sizeof(double2) * n));
    TDDA_CUDA_TRY(cudaMalloc(&m->D64, sizeof(double2) * n));
    TDDA_CUDA_TRY(cudaMemset(m->R64, 0, sizeof(double2) * n));
    TDDA_CUDA_TRY(cudaMemset(m->D64, 0, sizeof(double2) * n));
    m->refine64_nrhs = nrhs;
    return TDDA_OK;
}

static tdda_status update_alpha(tdda_model *m) {
    ++m->gen;
    // rho per cell from the parameters (src/DDAModel.cpp:762-770)
    std::vector<double> rho(m->nbox, 0.0);
    for (int i = 0; i < m->N; ++i)
        rho[m->cell_of[i]] = m->per_dipole ? m->rho_dipole[i] : m->parameters[m->geometryPara[i]];
    for (int i = 0; i < m->N; ++i) {
        double v = rho[m->cell_of[i]];
        if (!(v >= 0.0 && v <= 1.0)) return bad("design density outside [0, 1]");
    }
    TDDA_CUDA_TRY(cudaMemcpyAsync(m->d_rho, rho.data(), sizeof(double) * m->nbox, cudaMemcpyHostToDevice, m->stream));
    count_launches(1);
    k_alpha<<<grid_for(m->nbox), 256, 0, m->stream>>>(m->nbox, m->d_rho, m->d_mask, m->ap, m->al, m->al32, m->diel);
    count_launches(1);
    k_jacobi<<<grid_for(m->nbox), 256, 0, m->stream>>>(m->nbox, m->al, m->d_mask, m->a0, m->sc64, m->alS64,
                                                        m->sc32, m->alS32);
    TDDA_CUDA_TRY(cudaGetLastError());
    TDDA_CUDA_TRY(cudaStreamSynchronize(m->stream));
    return TDDA_OK;
}

// BiCGSTAB iterations per CUDA graph: the solver replays them between polls
// of the done flags instead of launching their 7 kernels one by one.
constexpr int kGraphSteps = 4;

static tdda_status solve_c128(tdda_model *m, const double2 *B, double2 *X, int nrhs, bool x0_zero,
                              int max_iter, double tol, tdda_solve_info *info) {
    TRY(ensure_krylov(m, nrhs));
    KrylovOptions o;
    o.graph_steps = kGraphSteps;
    o.time_limit_s = m->time_limit_s;
    return bicgstab_device<double2>(m->op, m->kv, m->al, nullptr, B, X, nrhs, x0_zero, max_iter, tol, m->stream,
                                    info, o);
}

// A refinement solve into the model's own P (one right-hand side) computes
// E_int and the IntegratedE sum in its last kernel, the true-residual
// evaluation of the returned solution.
static bool post_fused(const tdda_model *m, const double2 *X, int nrhs) { return X == m->P && nrhs == 1; }
static void set_post(tdda_model *m, ResidualPost &p, const double2 *X, int nrhs) {
    if (!post_fused(m, X, nrhs)) return;
    p.eres = m->Eres;
    p.diel = m->diel;
    p.mask = m->d_mask;
    p.q = m->powNum;
}

// Refinement workspace of the model, per inner precision.
static RefineWork<float2> refine_work(tdda_model *m, float2 *) {
    const bool j = m->precond != 0;
    RefineWork<float2> w;
    w.op = &m->op32; w.kv = &m->kv32; w.al = j ? m->alS32 : m->al32; w.sc = j ? m->sc32 : nullptr;
    w.R = m->R32; w.D = m->D32;
    return w;
}

static RefineWork<double2> refine_work(tdda_model *m, double2 *) {
    const bool j = m->precond != 0;
    RefineWork<double2> w;
    w.op = &m->op; w.kv = &m->kv; w.al = j ? m->alS64 : m->al; w.sc = j ? m->sc64 : nullptr;
    w.R = m->R64; w.D = m->D64;
    return w;
}

// Iterative refinement on the complex128 residual with inner solves in C
// (complex64 for mixed precision), Jacobi-scaled when precond is on.
template <typename C>
static tdda_status solve_refined(tdda_model *m, const double2 *B, double2 *X, int nrhs, bool x0_zero,
                                 int max_iter, double tol, tdda_solve_info *info) {
    TRY(ensure_refine(m, nrhs, (C *)nullptr));
    RefineWork<C> w = refine_work(m, (C *)nullptr);
    w.op64 = &m->op; w.al64 = m->al; w.sc64 = m->precond ? m->sc64 : nullptr;
    w.Rm = m->Rm; w.st_res = m->st_res; w.st_res_host = m->st_res_host;
    w.d_part = m->d_part; w.h_part = m->h_part;
    w.nbox = m->nbox; w.s = m->stream; w.graph_steps = kGraphSteps; w.time_limit_s = m->time_limit_s;
    set_post(m, w.post, X, nrhs);
    return refine_solve<C>(w, B, X, nrhs, x0_zero, max_iter, tol, info);
}

static GmresWork<float2> &gmres_work(tdda_model *m, float2 *) { return m->gw32; }
static GmresWork<double2> &gmres_work(tdda_model *m, double2 *) { return m->gw64; }

// Polynomial-preconditioned GMRES in complex128 refinement, inner solves in C
// (complex64 for mixed precision), always Jacobi-scaled.
template <typename C>
static tdda_status solve_pgmres(tdda_model *m, const double2 *B, double2 *X, int nrhs, bool x0_zero, int max_iter,
                                double tol, tdda_solve_info *info) {
    TRY(ensure_refine(m, nrhs, (C *)nullptr));
    GmresWork<C> &gw = gmres_work(m, (C *)nullptr);
    if (gw.nrhs != nrhs || gw.restart != m->gopt.restart || gw.degree != m->gopt.degree ||
        gw.deflate != m->gopt.deflate) {
        gw.release();
        TRY(gw.init(3 * m->nbox, nrhs, m->gopt.restart, m->gopt.degree, m->gopt.deflate));
    }
    const int saved = m->precond;
    m->precond = 1;
    RefineWork<C> w = refine_work(m, (C *)nullptr);
    m->precond = saved;
    w.op64 = &m->op; w.al64 = m->al; w.sc64 = m->sc64;
    w.Rm = m->Rm; w.st_res = m->st_res; w.st_res_host = m->st_res_host;
    w.d_part = m->d_part; w.h_part = m->h_part;
    w.nbox = m->nbox; w.s = m->stream;
    set_post(m, w.post, X, nrhs);
    GmresOptions o = m->gopt;
    o.floor = sizeof(C) == sizeof(float2) ? 2e-6 : 0.0;
    return pgmres_solve<C>(w, gw, B, X, nrhs, x0_zero, max_iter, tol, o, info);
}

static tdda_status solve_dispatch(tdda_model *m, const double2 *B, double2 *X, int nrhs, bool x0_zero,
                                  int max_iter, double tol, tdda_solve_info *info) {
    if (max_iter < 0) return bad("max_iter must be >= 0");
    if (!(tol >= 0.0)) return bad("tolerance must be >= 0");
    if (m->solver == 1) {
        if (m->precision == TDDA_PREC_MIXED)
            return solve_pgmres<float2>(m, B, X, nrhs, x0_zero, max_iter, tol, info);
        return solve_pgmres<double2>(m, B, X, nrhs, x0_zero, max_iter, tol, info);
    }
    if (m->precision == TDDA_PREC_MIXED)
        return solve_refined<float2>(m, B, X, nrhs, x0_zero, max_iter, tol, info);
    if (m->precond != 0) return solve_refined<double2>(m, B, X, nrhs, x0_zero, max_iter, tol, info);
    return solve_c128(m, B, X, nrhs, x0_zero, max_iter, tol, info);
}

static tdda_status solve_internal(tdda_model *m, const double2 *B, double2 *X, int nrhs, bool x0_zero,
                                  int max_iter, double tol, tdda_solve_info *info) {
    if (X == m->P) ++m->gen;
    const bool refinement = m->solver == 1 || m->precision == TDDA_PREC_MIXED || m->precond != 0;
    tdda_status st = solve_dispatch(m, B, X, nrhs, x0_zero, max_iter, tol, info);
    // a zero right-hand side ends with X cleared after its residual evaluation
    if (st == TDDA_OK && refinement && post_fused(m, X, nrhs) && info != nullptr &&
        info[0].status != TDDA_SOLVE_ZERO_RHS) {
        m->post_gen = m->gen;
        m->post_obj = m->st_res_host[0].post_sum;
    }
    return st;
}

// ----------------------------------------------------------------------------
// C ABI
// ----------------------------------------------------------------------------
extern "C" {

const char *tdda_status_string(tdda_status s) {
    switch (s) {
        case TDDA_OK: return "ok";
        case TDDA_ERR_BAD_ARG: return "bad argument";
        case TDDA_ERR_OOM: return "out of device memory";
        case TDDA_ERR_NOT_CONVERGED: return "not converged";
        case TDDA_ERR_BREAKDOWN: return "breakdown";
        case TDDA_ERR_CUDA: return "CUDA error";
        case TDDA_ERR_TIMEOUT: return "timeout";
        case TDDA_ERR_UNSUPPORTED: return "unsupported";
        case TDDA_ERR_STATE: return "invalid state";
    }
    return "unknown";
}

const char *tdda_last_error(void) { return get_error(); }
int tdda_abi_version(void) { return 1; }

tdda_status tdda_model_create(const tdda_params *p, const int32_t *geometry, const double *input_dielectrics,
                              const double *si, const double *ci, int64_t ntab, tdda_model **out) {
    if (out == nullptr || p == nullptr || geometry == nullptr || input_dielectrics == nullptr)
        return bad("null argument");
    *out = nullptr;
    std::unique_ptr<tdda_model> m(new tdda_model());
    m->Nx = p->num_x; m->Ny = p->num_y; m->Nz = p->num_z; m->N = p->num_total;
    if (m->Nx < 1 || m->Ny < 1 || m->Nz < 1 || m->N < 1) return bad("grid sizes must be positive");
    m->nbox = (long long)m->Nx * m->Ny * m->Nz;
    if (m->N > m->nbox) return bad("num_total exceeds num_x*num_y*num_z");
    if (p->d <= 0 || p->lam <= 0 || p->nback <= 0) return bad("d, lam and nback must be positive");
    if (p->use_filter) {
        if (p->n_filters < 1 || p->filter_radii == nullptr) return bad("useFilter needs at least one filter radius");
        if (p->is_periodic && (p->Lm != std::floor(p->Lm) || p->Ln != std::floor(p->Ln)))
            return bad("the periodic legacy filter needs whole-cell periods Lm, Ln");
    }
    std::string sym = p->symmetry_type ? p->symmetry_type : "";
    int dividesym;
    if (sym == "None") dividesym = 1;
    else if (sym == "4fold") dividesym = 4;
    else return bad("symmetryType must be \"None\" or \"4fold\" (src/DDAModel.cpp:163-173)");
    std::string meth = p->matrix_method ? p->matrix_method : "";
    if (meth == "FCD") m->method = 0;
    else if (meth == "LDR") m->method = 1;
    else return bad("\"" + meth + "\" is not a valid polarizabiliy calculation method.");
    if (m->method == 0 && (si == nullptr || ci == nullptr || ntab < 2)) return bad("FCD needs SiCi tables");
    if (p->n_obj_para < 1 || p->obj_para == nullptr) return bad("objPara needs at least the power");
    if (p->MAXm < 0 || p->MAXn < 0) return bad("MAXm, MAXn must be >= 0");
    m->powNum = (int)std::lround(p->obj_para[0]);
    m->d = p->d; m->lam = p->lam; m->nback = p->nback; m->E0 = p->E0;
    for (int c = 0; c < 3; ++c) { m->nK[c] = p->n_K[c]; m->nE0[c] = p->n_E0[c]; }
    m->MAXm = p->MAXm; m->MAXn = p->MAXn;
    m->Lm = p->Lm * p->d; m->Ln = p->Ln * p->d;
    m->delta = p->integral_delta;
    m->precision = p->precision;
    m->verbose = p->verbose;
    // src/AProductCore.cpp:25-33: K, rescale materials
    m->K = 2.0 * M_PI / (m->lam / m->nback);
    for (int i = 0; i < 2; ++i) {
        std::complex<double> v(p->material[2 * i], p->material[2 * i + 1]);
        v = v / (m->nback * m->nback);
        if (std::sqrt(std::norm(v)) < 1.01) v = v + 0.01;
        m->mat[i] = make_double2(v.real(), v.imag());
    }
    m->ap.lam = m->lam; m->ap.K = m->K; m->ap.d = m->d; m->ap.m0 = m->mat[0]; m->ap.m1 = m->mat[1];
    m->ap.S = std::pow(m->nE0[0] * m->nK[0], 2) + std::pow(m->nE0[1] * m->nK[1], 2) + std::pow(m->nE0[2] * m->nK[2], 2);
    // geometry -> cells
    m->geometry.assign(geometry, geometry + 3 * (size_t)m->N);
    m->cell_of.resize(m->N);
    std::vector<unsigned char> mask(m->nbox, 0);
    for (int i = 0; i < m->N; ++i) {
        int x = geometry[3 * i], y = geometry[3 * i + 1], z = geometry[3 * i + 2];
        if (x < 0 || x >= m->Nx || y < 0 || y >= m->Ny || z < 0 || z >= m->Nz)
            return bad("geometry coordinate outside the num_x*num_y*num_z box");
        long long cell = ((long long)x * m->Ny + y) * m->Nz + z;
        if (mask[cell]) return bad("duplicate geometry coordinate");
        mask[cell] = 1;
        m->cell_of[i] = cell;
    }
    // parameter map (src/DDAModel.cpp:181-247, FCurrentinsert :37-64)
    m->NFpara = (int)std::lround((double)(3 * m->N / 3 / m->Nz / dividesym));
    std::map<std::pair<int, int>, int> cur;
    int pos = 0;
    m->geometryPara.resize(m->N);
    for (int i = 0; i < m->N; ++i) {
        std::pair<int, int> xy(geometry[3 * i], geometry[3 * i + 1]);
        auto it = cur.find(xy);
        if (it == cur.end()) {
            if (dividesym == 1) {
                cur[xy] = pos++;
            } else {
                auto mir = [](double ax, int v) { return (int)std::lround(2 * ax - v); };
                std::pair<int, int> s1(mir(p->symmetry_axis[0], xy.first), xy.second);
                std::pair<int, int> s2(mir(p->symmetry_axis[0], xy.first), mir(p->symmetry_axis[1], xy.second));
                std::pair<int, int> s3(xy.first, mir(p->symmetry_axis[1], xy.second));
                if (cur.count(s1)) cur[xy] = cur[s1];
                else if (cur.count(s2)) cur[xy] = cur[s2];
                else if (cur.count(s3)) cur[xy] = cur[s3];
                else cur[xy] = pos++;
            }
        }
        m->geometryPara[i] = cur[xy];
    }
    if (pos != m->NFpara)
        return bad("symmetry map yields " + std::to_string(pos) + " free parameters, expected NFpara=" +
                   std::to_string(m->NFpara));
    m->p2g_off.assign(m->NFpara + 1, 0);
    for (int i = 0; i < m->N; ++i) m->p2g_off[m->geometryPara[i] + 1]++;
    for (int k = 0; k < m->NFpara; ++k) m->p2g_off[k + 1] += m->p2g_off[k];
    m->p2g_idx.resize(m->N);
    {
        std::vector<int> fill(m->p2g_off.begin(), m->p2g_off.end() - 1);
        for (int i = 0; i < m->N; ++i) m->p2g_idx[fill[m->geometryPara[i]]++] = i;
    }
    // initial parameters: value of the first dipole of each parameter (src/DDAModel.cpp:227-247)
    m->parameters.resize(m->NFpara);
    for (int k = 0; k < m->NFpara; ++k) m->parameters[k] = input_dielectrics[3 * (size_t)m->p2g_idx[m->p2g_off[k]]];

    // device state
    TDDA_CUDA_TRY(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
    if (p->use_filter) {
        // src/DDAModel.cpp:255-264: raw = filtered = the initial parameters, weights built once
        LegacyFilterConfig fc;
        fc.beta_min = p->beta_min; fc.beta_max = p->beta_max; fc.ita = p->ita;
        fc.beta_type = p->beta_type ? p->beta_type : "";
        fc.rfilter = p->filter_radii[0];
        fc.periodic = p->is_periodic != 0;
        fc.Lm = (int)p->Lm; fc.Ln = (int)p->Ln;
        TRY(m->lfilter.build(fc, m->geometry, m->p2g_off, m->p2g_idx, m->parameters));
    }
    TRY(m->op.init(m->Nx, m->Ny, m->Nz, 1));
    const ConvGeom &g = m->op.g;
    const size_t nfold = (size_t)g.hx * g.hy * g.hz * 6;
    TDDA_CUDA_TRY(cudaMalloc(&m->op.ahat, sizeof(double2) * nfold));
    float2 *ahat32 = nullptr;
    if (m->precision == TDDA_PREC_MIXED) {
        TRY(m->op32.init(m->Nx, m->Ny, m->Nz, 1));
        TDDA_CUDA_TRY(cudaMalloc(&m->op32.ahat, sizeof(float2) * nfold));
        ahat32 = m->op32.ahat;
    } else if (m->precision != TDDA_PREC_C128) {
        return bad("precision must be 0 (complex128) or 1 (mixed)");
    }
    const bool full = (m->N == m->nbox);
    if (!full) {
        TDDA_CUDA_TRY(cudaMalloc(&m->d_mask, m->nbox));
        TDDA_CUDA_TRY(cudaMemcpy(m->d_mask, mask.data(), m->nbox, cudaMemcpyHostToDevice));
        m->op.mask = m->d_mask;
        m->op32.mask = m->d_mask;
    }
    TDDA_CUDA_TRY(cudaMalloc(&m->d_cell, sizeof(long long) * m->N));
    TDDA_CUDA_TRY(cudaMemcpy(m->d_cell, m->cell_of.data(), sizeof(long long) * m->N, cudaMemcpyHostToDevice));
    TDDA_CUDA_TRY(cudaMalloc(&m->d_rho, sizeof(double) * m->nbox));
    TDDA_CUDA_TRY(cudaMemset(m->d_rho, 0, sizeof(double) * m->nbox));
    TDDA_CUDA_TRY(cudaMalloc(&m->al, sizeof(double2) * m->nbox));
    TDDA_CUDA_TRY(cudaMalloc(&m->diel, sizeof(double2) * m->nbox));
    TDDA_CUDA_TRY(cudaMalloc(&m->sc64, sizeof(double2) * m->nbox));
    TDDA_CUDA_TRY(cudaMalloc(&m->alS64, sizeof(double2) * m->nbox));
    if (m->precision == TDDA_PREC_MIXED) {
        TDDA_CUDA_TRY(cudaMalloc(&m->al32, sizeof(float2) * m->nbox));
        TDDA_CUDA_TRY(cudaMalloc(&m->sc32, sizeof(float2) * m->nbox));
        TDDA_CUDA_TRY(cudaMalloc(&m->alS32, sizeof(float2) * m->nbox));
        m->precond = 1;  // mixed precision refines Jacobi-scaled complex64 solves
    }
    const size_t nvec = 3 * (size_t)m->nbox;
    TDDA_CUDA_TRY(cudaMalloc(&m->Einc, sizeof(double2) * nvec));
    TDDA_CUDA_TRY(cudaMalloc(&m->P, sizeof(double2) * nvec));
    TDDA_CUDA_TRY(cudaMalloc(&m->Eres, sizeof(double2) * nvec));
    TDDA_CUDA_TRY(cudaMemset(m->Einc, 0, sizeof(double2) * nvec));
    TDDA_CUDA_TRY(cudaMemset(m->P, 0, sizeof(double2) * nvec));
    TDDA_CUDA_TRY(cudaMemset(m->Eres, 0, sizeof(double2) * nvec));
    TDDA_CUDA_TRY(cudaMalloc(&m->d_part, sizeof(double) * 1024));
    TDDA_CUDA_TRY(cudaMallocHost(&m->h_part, sizeof(double) * 1024));
    TRY(ensure_ext(m.get(), 3 * (long long)m->N));

    // interaction tensor
    LatticeParams L{};
    L.nx = m->Nx; L.ny = m->Ny; L.nz = m->Nz;
    L.Lx = g.Lx; L.Ly = g.Ly; L.Lz = g.Lz;
    L.d = m->d; L.K = m->K; L.Kf = M_PI / m->d; L.Lm = m->Lm; L.Ln = m->Ln;
    L.MAXm = m->MAXm; L.MAXn = m->MAXn; L.method = m->method; L.gamma = 0.01; L.delta = m->delta;
    std::vector<double> dummy(2, 0.0);
    const double *tsi = si ? si : dummy.data(), *tci = ci ? ci : dummy.data();
    long nt = (si && ci) ? (long)ntab : 2;
    double2 a0[6];
    TRY(build_tensor(L, tsi, tci, nt, m->op.ahat, ahat32, m->stream, &m->lattice_ms, &m->fft_ms, a0));
    m->lat = L;
    m->si_h.assign(tsi, tsi + nt);
    m->ci_h.assign(tci, tci + nt);
    m->a0 = make_double2((a0[0].x + a0[3].x + a0[5].x) / 3.0, (a0[0].y + a0[3].y + a0[5].y) / 3.0);

    // incident field (src/DDAModel.cpp:312-316), internal layout
    {
        std::vector<double2> e(nvec, make_double2(0.0, 0.0));
        for (int i = 0; i < m->N; ++i) {
            const int32_t *gi = &geometry[3 * i];
            double ph = m->K * m->d * (m->nK[0] * gi[0] + m->nK[1] * gi[1] + m->nK[2] * gi[2]);
            double cr = std::cos(ph), sn = std::sin(ph);
            for (int c = 0; c < 3; ++c)
                e[(size_t)c * m->nbox + m->cell_of[i]] = make_double2(m->E0 * m->nE0[c] * cr, m->E0 * m->nE0[c] * sn);
        }
        TDDA_CUDA_TRY(cudaMemcpy(m->Einc, e.data(), sizeof(double2) * nvec, cudaMemcpyHostToDevice));
    }
    TRY(update_alpha(m.get()));
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    m->device_bytes = (long long)(sizeof(double2) * nfold + sizeof(double2) * nvec * 3 +
                                  sizeof(double2) * 3 * g.tcomp);
    *out = m.release();
    return TDDA_OK;
}

void tdda_model_destroy(tdda_model *m) { delete m; }

tdda_status tdda_model_get_info(const tdda_model *m, tdda_model_info *info) {
    if (!m || !info) return bad("null argument");
    info->N = m->N; info->NFpara = m->NFpara;
    info->nx = m->Nx; info->ny = m->Ny; info->nz = m->Nz;
    info->Lx = m->op.g.Lx; info->Ly = m->op.g.Ly; info->Lz = m->op.g.Lz;
    info->K = m->K;
    for (int i = 0; i < 2; ++i) { info->material[2 * i] = m->mat[i].x; info->material[2 * i + 1] = m->mat[i].y; }
    info->device_bytes = m->device_bytes;
    info->lattice_ms = m->lattice_ms;
    info->tensor_fft_ms = m->fft_ms;
    return TDDA_OK;
}

static tdda_status to_internal(tdda_model *m, const double *host, double2 *dst, int nrhs) {
    const long long n = 3 * (long long)m->N * nrhs;
    TRY(ensure_ext(m, n));
    TDDA_CUDA_TRY(cudaMemcpyAsync(m->ext, host, sizeof(double2) * n, cudaMemcpyHostToDevice, m->stream));
    count_launches(1);
    k_scatter<<<grid_for(n), 256, 0, m->stream>>>(nrhs, m->N, m->nbox, m->d_cell, m->ext, dst);
    TDDA_CUDA_TRY(cudaGetLastError());
    return TDDA_OK;
}

static tdda_status to_host(tdda_model *m, const double2 *src, double *host, int nrhs) {
    const long long n = 3 * (long long)m->N * nrhs;
    TRY(ensure_ext(m, n));
    count_launches(1);
    k_gather<<<grid_for(n), 256, 0, m->stream>>>(nrhs, m->N, m->nbox, m->d_cell, src, m->ext);
    TDDA_CUDA_TRY(cudaGetLastError());
    TDDA_CUDA_TRY(cudaMemcpyAsync(host, m->ext, sizeof(double2) * n, cudaMemcpyDeviceToHost, m->stream));
    TDDA_CUDA_TRY(cudaStreamSynchronize(m->stream));
    return TDDA_OK;
}

tdda_status tdda_solve_electric_field(tdda_model *m, const double *P0, int max_iter, double tol,
                                      tdda_solve_info *info) {
    if (!m) return bad("null model");
    bool zero = (P0 == nullptr);
    if (!zero) {
        zero = true;
        for (long long i = 0; i < 6LL * m->N && zero; ++i) zero = (P0[i] == 0.0);
        if (!zero) TRY(to_internal(m, P0, m->P, 1));
    }
    tdda_solve_info inf{};
    TRY(solve_internal(m, m->Einc, m->P, 1, zero, max_iter, tol, &inf));
    if (m->post_gen != m->gen) {
        // the reference-semantics solve ends on its recursive residual: E_int here
        count_launches(1);
        k_eresult<<<grid_for(3 * m->nbox), 256, 0, m->stream>>>(m->nbox, m->P, m->al, m->diel, m->Eres);
        TDDA_CUDA_TRY(cudaGetLastError());
    }
    TDDA_CUDA_TRY(cudaStreamSynchronize(m->stream));
    if (m->verbose)
        fprintf(stderr, "[tdda] solve: %d iterations, error %.3e, status %d\n", inf.iterations, inf.error, inf.status);
    if (info) *info = inf;
    return TDDA_OK;
}

static tdda_status objective_sum(tdda_model *m, const double2 *P, double *S) {
    if (P == m->P && m->post_gen == m->gen) {   // summed by the solve's last kernel
        *S = m->post_obj;
        return TDDA_OK;
    }
    const int nb = 512;
    count_launches(1);
    k_objective<<<nb, 256, 0, m->stream>>>(m->nbox, P, m->al, m->d_mask, m->powNum, m->d_part);
    TDDA_CUDA_TRY(cudaGetLastError());
    TDDA_CUDA_TRY(cudaMemcpyAsync(m->h_part, m->d_part, sizeof(double) * nb, cudaMemcpyDeviceToHost, m->stream));
    TDDA_CUDA_TRY(cudaStreamSynchronize(m->stream));
    double s = 0.0;
    for (int b = 0; b < nb; ++b) s += m->h_part[b];
    *S = s;
    return TDDA_OK;
}

tdda_status tdda_calculate_objective(tdda_model *m, double *out) {
    if (!m || !out) return bad("null argument");
    double S;
    TRY(objective_sum(m, m->P, &S));
    m->E_int = S;
    *out = std::log(S);
    return TDDA_OK;
}

tdda_status tdda_calculate_gradients(tdda_model *m, double eps, double J0, int max_iter, double tol, double *grad,
                                     int64_t n) {
    if (!m || !grad) return bad("null argument");
    if (n != m->NFpara) return bad("gradient buffer must hold NFpara values");
    if (!(eps != 0.0)) return bad("epsilon_partial must be non-zero");
    if (m->per_dipole) {
        set_error("densities were set per dipole: use tdda_gradient_densities");
        return TDDA_ERR_STATE;
    }
    const long long nbox = m->nbox;
    TRY(ensure_batch(m, 1));
    double *dS = nullptr;
    double2 *change = nullptr, *prod = nullptr;
    TDDA_CUDA_TRY(cudaMalloc(&dS, sizeof(double) * nbox));
    std::unique_ptr<void, void (*)(void *)> g1(dS, [](void *p) { cudaFree(p); });
    TDDA_CUDA_TRY(cudaMalloc(&change, sizeof(double2) * nbox));
    std::unique_ptr<void, void (*)(void *)> g2(change, [](void *p) { cudaFree(p); });
    TDDA_CUDA_TRY(cudaMalloc(&prod, sizeof(double2) * nbox));
    std::unique_ptr<void, void (*)(void *)> g3(prod, [](void *p) { cudaFree(p); });
    GradFD G{m->ap, eps, J0, m->E_int, m->powNum};
    double2 *devp = m->bufB;
    count_launches(1);
    k_grad_fd<<<grid_for(nbox), 256, 0, m->stream>>>(nbox, m->d_rho, m->d_mask, m->P, m->al, G, dS, change, devp);
    TDDA_CUDA_TRY(cudaGetLastError());
    std::vector<double> hdS(nbox);
    TDDA_CUDA_TRY(cudaMemcpyAsync(hdS.data(), dS, sizeof(double) * nbox, cudaMemcpyDeviceToHost, m->stream));
    // adjoint solve with the same complex-symmetric operator (src/DDAModel.cpp:429-435)
    double2 *lam = m->bufX;
    tdda_solve_info inf{};
    TRY(solve_internal(m, devp, lam, 1, true, max_iter, tol, &inf));
    count_launches(1);
    k_grad_mult<<<grid_for(nbox), 256, 0, m->stream>>>(nbox, lam, m->P, change, prod);
    TDDA_CUDA_TRY(cudaGetLastError());
    std::vector<double2> hprod(nbox);
    TDDA_CUDA_TRY(cudaMemcpyAsync(hprod.data(), prod, sizeof(double2) * nbox, cudaMemcpyDeviceToHost, m->stream));
    TDDA_CUDA_TRY(cudaStreamSynchronize(m->stream));
    for (int k = 0; k < m->NFpara; ++k) {
        const double rho = m->parameters[k];
        const double se = (rho >= eps ? -1.0 : 1.0) * eps;
        double dsum = 0.0, mult = 0.0;
        for (int q = m->p2g_off[k]; q < m->p2g_off[k + 1]; ++q) {
            long long cell = m->cell_of[m->p2g_idx[q]];
            dsum += hdS[cell];
            mult += hprod[cell].x;
        }
        const double devx = (std::log(m->E_int + dsum) - J0) / se;
        grad[k] = devx - mult;
    }
    // as in the reference, the model's polarisation now holds the adjoint solution
    ++m->gen;
    TDDA_CUDA_TRY(cudaMemcpyAsync(m->P, lam, sizeof(double2) * 3 * nbox, cudaMemcpyDeviceToDevice, m->stream));
    TDDA_CUDA_TRY(cudaStreamSynchronize(m->stream));
    if (m->verbose)
        fprintf(stderr, "[tdda] adjoint: %d iterations, error %.3e\n", inf.iterations, inf.error);
    return TDDA_OK;
}

tdda_status tdda_set_parameters(tdda_model *m, const double *values, int64_t n) {
    if (!m || !values) return bad("null argument");
    if (n != m->NFpara) return bad("ERROR: In CoreStructure::UpdateStr(VectorXd step), step.size!=FreePara.size");
    std::vector<double> old = m->parameters;
    const bool old_pd = m->per_dipole;
    m->parameters.assign(values, values + n);
    m->per_dipole = false;
    tdda_status s = update_alpha(m);
    if (s != TDDA_OK) {
        m->parameters = old;
        m->per_dipole = old_pd;
    }
    return s;
}

tdda_status tdda_get_parameters(const tdda_model *m, double *out, int64_t n) {
    if (!m || !out) return bad("null argument");
    if (n != m->NFpara) return bad("buffer must hold NFpara values");
    std::copy(m->parameters.begin(), m->parameters.end(), out);
    return TDDA_OK;
}

tdda_status tdda_lattice_offsets_device(tdda_model *m, const int32_t *lo, const int32_t *nb, void *out_dev,
                                        void *stream) {
    if (!m || !lo || !nb || !out_dev) return bad("null argument");
    if (nb[0] < 1 || nb[1] < 1 || nb[2] < 1) return bad("box extents must be positive");
    if ((long long)nb[0] * nb[1] * nb[2] > (1LL << 28)) return bad("at most 2^28 offsets");
    cudaStream_t user = (cudaStream_t)stream;
    TDDA_CUDA_TRY(cudaStreamSynchronize(user));
    TRY(build_offset_tensor(m->lat, m->si_h.data(), m->ci_h.data(), (long)m->si_h.size(), lo[0], lo[1], lo[2], nb[0],
                            nb[1], nb[2], reinterpret_cast<double2 *>(out_dev), m->stream));
    return TDDA_OK;
}

tdda_status tdda_get_parameter_map(const tdda_model *m, int32_t *map, int64_t n) {
    if (!m || !map) return bad("null argument");
    if (n != m->N) return bad("map buffer must hold num_total entries");
    for (int i = 0; i < m->N; ++i) map[i] = m->geometryPara[i];
    return TDDA_OK;
}

tdda_status tdda_get_dielectrics(const tdda_model *cm, double *out, int64_t n) {
    if (!cm || !out) return bad("null argument");
    if (n != 3LL * cm->N) return bad("buffer must hold 3N values");
    tdda_model *m = const_cast<tdda_model *>(cm);  // refreshes the host mirror of device-set densities
    if (m->rho_host_stale) {
        std::vector<double> cells(m->nbox);
        TDDA_CUDA_TRY(cudaMemcpyAsync(cells.data(), m->d_rho, sizeof(double) * m->nbox, cudaMemcpyDeviceToHost,
                                      m->stream));
        TDDA_CUDA_TRY(cudaStreamSynchronize(m->stream));
        m->rho_dipole.resize(m->N);
        for (int i = 0; i < m->N; ++i) m->rho_dipole[i] = cells[m->cell_of[i]];
        m->rho_host_stale = false;
    }
    for (int i = 0; i < m->N; ++i) {
        double v = m->per_dipole ? m->rho_dipole[i] : m->parameters[m->geometryPara[i]];
        out[3 * i] = out[3 * i + 1] = out[3 * i + 2] = v;
    }
    return TDDA_OK;
}

tdda_status tdda_get_electric_field(const tdda_model *m, double *out, int64_t n) {
    if (!m || !out) return bad("null argument");
    if (n != 3LL * m->N) return bad("buffer must hold 3N complex values");
    return to_host(const_cast<tdda_model *>(m), m->Eres, out, 1);
}

tdda_status tdda_get_polarization(const tdda_model *m, double *out, int64_t n) {
    if (!m || !out) return bad("null argument");
    if (n != 3LL * m->N) return bad("buffer must hold 3N complex values");
    return to_host(const_cast<tdda_model *>(m), m->P, out, 1);
}

tdda_status tdda_matvec(tdda_model *m, const double *x, double *y, int with_al) {
    if (!m || !x || !y) return bad("null argument");
    TRY(ensure_batch(m, 1));
    TRY(to_internal(m, x, m->bufB, 1));
    TRY(m->op.apply(m->bufB, m->bufX, with_al ? m->al : nullptr, 1, m->stream));
    return to_host(m, m->bufX, y, 1);
}

tdda_status tdda_matvec_c64(tdda_model *m, const double *x, double *y, int with_al) {
    if (!m || !x || !y) return bad("null argument");
    if (m->op32.ahat == nullptr) {
        set_error("complex64 operator exists only in models created mixed");
        return TDDA_ERR_UNSUPPORTED;
    }
    TRY(ensure_batch(m, 1));
    TRY(ensure_mixed(m, 1));
    const long long n = 3 * m->nbox;
    TRY(to_internal(m, x, m->bufB, 1));
    const double one = 1.0;
    TDDA_CUDA_TRY(cudaMemcpyAsync(m->d_part, &one, sizeof(double), cudaMemcpyHostToDevice, m->stream));
    launch_to_inner<float2>(n, m->nbox, 1, 0, m->bufB, m->d_part, nullptr, m->R32, m->stream);
    TRY(m->op32.apply(m->R32, m->D32, with_al ? m->al32 : nullptr, 1, m->stream));
    TDDA_CUDA_TRY(cudaMemsetAsync(m->bufX, 0, sizeof(double2) * n, m->stream));
    launch_axpy_inner<float2>(n, m->nbox, 1, 0, m->d_part, nullptr, m->D32, m->bufX, m->stream);
    TDDA_CUDA_TRY(cudaGetLastError());
    return to_host(m, m->bufX, y, 1);
}

tdda_status tdda_solve_batch_device(tdda_model *m, const void *B_dev, void *X_dev, int nrhs, int x0_zero,
                                    int max_iter, double tol, void *stream, tdda_solve_info *infos) {
    if (!m || !X_dev || nrhs < 1) return bad("bad argument");
    cudaStream_t user = (cudaStream_t)stream;
    cudaEvent_t ev;
    TDDA_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    std::unique_ptr<CUevent_st, void (*)(cudaEvent_t)> evg(ev, [](cudaEvent_t e) { cudaEventDestroy(e); });
    // order the model stream after the caller's stream
    TDDA_CUDA_TRY(cudaEventRecord(ev, user));
    TDDA_CUDA_TRY(cudaStreamWaitEvent(m->stream, ev, 0));
    TRY(ensure_batch(m, nrhs));
    const long long n3 = 3 * (long long)m->N;
    const size_t nvec = 3 * (size_t)m->nbox;
    if (B_dev) {
        count_launches(1);
        k_scatter<<<grid_for(n3 * nrhs), 256, 0, m->stream>>>(nrhs, m->N, m->nbox, m->d_cell,
                                                             (const double2 *)B_dev, m->bufB);
    } else {
        for (int k = 0; k < nrhs; ++k)
            TDDA_CUDA_TRY(cudaMemcpyAsync(m->bufB + k * nvec, m->Einc, sizeof(double2) * nvec,
                                          cudaMemcpyDeviceToDevice, m->stream));
    }
    if (!x0_zero) {
        count_launches(1);
        k_scatter<<<grid_for(n3 * nrhs), 256, 0, m->stream>>>(nrhs, m->N, m->nbox, m->d_cell,
                                                             (const double2 *)X_dev, m->bufX);
    }
    TDDA_CUDA_TRY(cudaGetLastError());
    TRY(solve_internal(m, m->bufB, m->bufX, nrhs, x0_zero != 0, max_iter, tol, infos));
    count_launches(1);
    k_gather<<<grid_for(n3 * nrhs), 256, 0, m->stream>>>(nrhs, m->N, m->nbox, m->d_cell, m->bufX, (double2 *)X_dev);
    TDDA_CUDA_TRY(cudaGetLastError());
    TDDA_CUDA_TRY(cudaEventRecord(ev, m->stream));
    TDDA_CUDA_TRY(cudaStreamWaitEvent(user, ev, 0));
    return TDDA_OK;
}

tdda_status tdda_matvec_device(tdda_model *m, const void *x_dev, void *y_dev, int nrhs, int with_al, void *stream) {
    if (!m || !x_dev || !y_dev || nrhs < 1) return bad("bad argument");
    cudaStream_t user = (cudaStream_t)stream;
    cudaEvent_t ev;
    TDDA_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    std::unique_ptr<CUevent_st, void (*)(cudaEvent_t)> evg(ev, [](cudaEvent_t e) { cudaEventDestroy(e); });
    TDDA_CUDA_TRY(cudaEventRecord(ev, user));
    TDDA_CUDA_TRY(cudaStreamWaitEvent(m->stream, ev, 0));
    TRY(ensure_batch(m, nrhs));
    TRY(ensure_op_cap(m, nrhs));
    const long long n3 = 3 * (long long)m->N;
    count_launches(1);
    k_scatter<<<grid_for(n3 * nrhs), 256, 0, m->stream>>>(nrhs, m->N, m->nbox, m->d_cell, (const double2 *)x_dev, m->bufB);
    TRY(m->op.apply(m->bufB, m->bufX, with_al ? m->al : nullptr, nrhs, m->stream));
    count_launches(1);
    k_gather<<<grid_for(n3 * nrhs), 256, 0, m->stream>>>(nrhs, m->N, m->nbox, m->d_cell, m->bufX, (double2 *)y_dev);
    TDDA_CUDA_TRY(cudaGetLastError());
    TDDA_CUDA_TRY(cudaEventRecord(ev, m->stream));
    TDDA_CUDA_TRY(cudaStreamWaitEvent(user, ev, 0));
    return TDDA_OK;
}

tdda_status tdda_set_densities(tdda_model *m, const double *rho, int64_t n) {
    if (!m || !rho) return bad("null argument");
    if (n != m->N) return bad("densities must hold N values");
    std::vector<double> old = m->rho_dipole;
    const bool old_pd = m->per_dipole;
    m->rho_dipole.assign(rho, rho + n);
    m->per_dipole = true;
    const bool old_stale = m->rho_host_stale;
    m->rho_host_stale = false;
    tdda_status s = update_alpha(m);
    if (s != TDDA_OK) {
        m->rho_dipole = old;
        m->per_dipole = old_pd;
        m->rho_host_stale = old_stale;
    }
    return s;
}

// Makes `to` wait for the work queued so far on `from`.
static tdda_status join_streams(cudaStream_t from, cudaStream_t to) {
    cudaEvent_t ev;
    TDDA_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    cudaError_t e1 = cudaEventRecord(ev, from);
    cudaError_t e2 = e1 == cudaSuccess ? cudaStreamWaitEvent(to, ev, 0) : e1;
    cudaEventDestroy(ev);
    TDDA_CUDA_TRY(e2);
    return TDDA_OK;
}

static tdda_status ensure_grad_scratch(tdda_model *m) {
    if (m->d_grad == nullptr) TDDA_CUDA_TRY(cudaMalloc(&m->d_grad, sizeof(double) * m->nbox));
    if (m->d_flag == nullptr) {
        TDDA_CUDA_TRY(cudaMalloc(&m->d_flag, sizeof(unsigned)));
        TDDA_CUDA_TRY(cudaMallocHost(&m->h_flag, sizeof(unsigned)));
    }
    return TDDA_OK;
}

tdda_status tdda_set_densities_device(tdda_model *m, const double *rho_dev, void *stream) {
    if (!m || !rho_dev) return bad("null argument");
    TRY(ensure_grad_scratch(m));
    cudaStream_t user = (cudaStream_t)stream;
    TRY(join_streams(user, m->stream));
    TDDA_CUDA_TRY(cudaMemsetAsync(m->d_flag, 0, sizeof(unsigned), m->stream));
    count_launches(1);
    k_rho_check<<<grid_for(m->N), 256, 0, m->stream>>>(m->N, rho_dev, m->d_flag);
    TDDA_CUDA_TRY(cudaMemcpyAsync(m->h_flag, m->d_flag, sizeof(unsigned), cudaMemcpyDeviceToHost, m->stream));
    TDDA_CUDA_TRY(cudaStreamSynchronize(m->stream));
    if (*m->h_flag != 0) return bad("design density outside [0, 1]");
    count_launches(3);
    k_rho_scatter<<<grid_for(m->N), 256, 0, m->stream>>>(m->N, m->d_cell, rho_dev, m->d_rho);
    ++m->gen;
    k_alpha<<<grid_for(m->nbox), 256, 0, m->stream>>>(m->nbox, m->d_rho, m->d_mask, m->ap, m->al, m->al32, m->diel);
    k_jacobi<<<grid_for(m->nbox), 256, 0, m->stream>>>(m->nbox, m->al, m->d_mask, m->a0, m->sc64, m->alS64,
                                                        m->sc32, m->alS32);
    TDDA_CUDA_TRY(cudaGetLastError());
    m->per_dipole = true;
    m->rho_host_stale = true;
    return join_streams(m->stream, user);
}

// The exact adjoint gradient of IntegratedE per cell into m->d_grad.
static tdda_status gradient_cells(tdda_model *m, int max_iter, double tol, tdda_solve_info *info) {
    double S;
    TRY(objective_sum(m, m->P, &S));
    if (!(S > 0.0)) return bad("objective sum is zero: solve first");
    TRY(ensure_batch(m, 1));
    TRY(ensure_grad_scratch(m));
    const long long nbox = m->nbox;
    k_adjoint_rhs<<<grid_for(nbox), 256, 0, m->stream>>>(nbox, m->P, m->al, m->d_mask, m->powNum, S, m->bufB);
    count_launches(1);
    TDDA_CUDA_TRY(cudaGetLastError());
    tdda_solve_info inf{};
    TRY(solve_internal(m, m->bufB, m->bufX, 1, true, max_iter, tol, &inf));
    k_grad_analytic<<<grid_for(nbox), 256, 0, m->stream>>>(nbox, m->d_rho, m->d_mask, m->P, m->al, m->diel, m->bufX,
                                                           m->ap, m->powNum, S, m->d_grad);
    count_launches(1);
    TDDA_CUDA_TRY(cudaGetLastError());
    if (info) *info = inf;
    return TDDA_OK;
}

static tdda_status cells_to_host(tdda_model *m, const double *cells, double *out) {
    std::vector<double> h(m->nbox);
    TDDA_CUDA_TRY(cudaMemcpyAsync(h.data(), cells, sizeof(double) * m->nbox, cudaMemcpyDeviceToHost, m->stream));
    TDDA_CUDA_TRY(cudaStreamSynchronize(m->stream));
    for (int i = 0; i < m->N; ++i) out[i] = h[m->cell_of[i]];
    return TDDA_OK;
}

// rho[i] = params[pmap[i]] (free parameters -> per-dipole densities)
__global__ void k_param_gather(long long n, const int32_t *__restrict__ pmap, const double *__restrict__ params,
                               double *__restrict__ rho) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        rho[i] = params[pmap[i]];
}

// out[j] = sum of g over parameter j's dipoles, added one at a time in dipole
// order (the order of a sequential scatter-add over the dipoles)
__global__ void k_param_sum(long long np, const int32_t *__restrict__ ptr, const int32_t *__restrict__ idx,
                            const double *__restrict__ g, double *__restrict__ out) {
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < np; j += (long long)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int k = ptr[j]; k < ptr[j + 1]; ++k) s = __dadd_rn(s, g[idx[k]]);
        out[j] = s;
    }
}

static tdda_status ensure_pmap(tdda_model *m) {
    if (m->d_pmap != nullptr) return TDDA_OK;
    const int np = m->NFpara;
    std::vector<int32_t> ptr(np + 1, 0), idx(m->N), map(m->geometryPara.begin(), m->geometryPara.end());
    for (int i = 0; i < m->N; ++i) ptr[map[i] + 1] += 1;
    for (int j = 0; j < np; ++j) ptr[j + 1] += ptr[j];
    std::vector<int32_t> fill(ptr.begin(), ptr.end() - 1);
    for (int i = 0; i < m->N; ++i) idx[fill[map[i]]++] = i;
    int32_t *a = nullptr, *b = nullptr, *c = nullptr;
    TDDA_CUDA_TRY(cudaMalloc(&a, sizeof(int32_t) * m->N));
    TDDA_CUDA_TRY(cudaMalloc(&b, sizeof(int32_t) * (np + 1)));
    TDDA_CUDA_TRY(cudaMalloc(&c, sizeof(int32_t) * m->N));
    TDDA_CUDA_TRY(cudaMemcpy(a, map.data(), sizeof(int32_t) * m->N, cudaMemcpyHostToDevice));
    TDDA_CUDA_TRY(cudaMemcpy(b, ptr.data(), sizeof(int32_t) * (np + 1), cudaMemcpyHostToDevice));
    TDDA_CUDA_TRY(cudaMemcpy(c, idx.data(), sizeof(int32_t) * m->N, cudaMemcpyHostToDevice));
    m->d_pmap = a; m->d_pptr = b; m->d_pidx = c;
    return TDDA_OK;
}

static tdda_status cells_to_device(tdda_model *m, const double *cells, double *out_dev, cudaStream_t user) {
    count_launches(1);
    k_cell_to_dipole<<<grid_for(m->N), 256, 0, m->stream>>>(m->N, m->d_cell, cells, out_dev);
    TDDA_CUDA_TRY(cudaGetLastError());
    return join_streams(m->stream, user);
}

tdda_status tdda_gradient_densities(tdda_model *m, int max_iter, double tol, double *grad, int64_t n,
                                    tdda_solve_info *info) {
    if (!m || !grad) return bad("null argument");
    if (n != m->N) return bad("gradient buffer must hold N values");
    TRY(gradient_cells(m, max_iter, tol, info));
    return cells_to_host(m, m->d_grad, grad);
}

tdda_status tdda_gradient_densities_device(tdda_model *m, int max_iter, double tol, double *grad_dev, void *stream,
                                           tdda_solve_info *info) {
    if (!m || !grad_dev) return bad("null argument");
    TRY(join_streams((cudaStream_t)stream, m->stream));
    TRY(gradient_cells(m, max_iter, tol, info));
    return cells_to_device(m, m->d_grad, grad_dev, (cudaStream_t)stream);
}

tdda_status tdda_params_to_densities_device(tdda_model *m, const double *params_dev, double *rho_dev,
                                           void *stream) {
    if (!m || !params_dev || !rho_dev) return bad("null argument");
    TRY(ensure_pmap(m));
    cudaStream_t user = (cudaStream_t)stream;
    TRY(join_streams(user, m->stream));
    count_launches(1);
    k_param_gather<<<grid_for(m->N), 256, 0, m->stream>>>(m->N, m->d_pmap, params_dev, rho_dev);
    TDDA_CUDA_TRY(cudaGetLastError());
    return join_streams(m->stream, user);
}

tdda_status tdda_densities_to_params_device(tdda_model *m, const double *grad_dev, double *grad_params_dev,
                                           void *stream) {
    if (!m || !grad_dev || !grad_params_dev) return bad("null argument");
    TRY(ensure_pmap(m));
    cudaStream_t user = (cudaStream_t)stream;
    TRY(join_streams(user, m->stream));
    count_launches(1);
    k_param_sum<<<grid_for(m->NFpara), 256, 0, m->stream>>>(m->NFpara, m->d_pptr, m->d_pidx, grad_dev,
                                                            grad_params_dev);
    TDDA_CUDA_TRY(cudaGetLastError());
    return join_streams(m->stream, user);
}

tdda_status tdda_solve_electric_field_warm(tdda_model *m, int max_iter, double tol, tdda_solve_info *info) {
    if (!m) return bad("null model");
    tdda_solve_info inf{};
    TRY(solve_internal(m, m->Einc, m->P, 1, false, max_iter, tol, &inf));
    if (m->post_gen != m->gen) {
        count_launches(1);
        k_eresult<<<grid_for(3 * m->nbox), 256, 0, m->stream>>>(m->nbox, m->P, m->al, m->diel, m->Eres);
        TDDA_CUDA_TRY(cudaGetLastError());
    }
    TDDA_CUDA_TRY(cudaStreamSynchronize(m->stream));
    if (info) *info = inf;
    return TDDA_OK;
}

tdda_status tdda_profile_matvec(tdda_model *m, int precision, int nrhs, int iters, double *ms_matvec,
                                double *ms_pass) {
    if (!m || !ms_matvec || !ms_pass || nrhs < 1) return bad("bad argument");
    if (precision == 0) {
        TRY(ensure_batch(m, nrhs));
        TRY(ensure_op_cap(m, nrhs));
        return profile_apply<double2>(m->op, m->bufB, m->bufX, m->al, nrhs, iters, m->stream, ms_matvec, ms_pass);
    }
    if (m->op32.ahat == nullptr) {
        set_error("complex64 operator exists only in models created mixed");
        return TDDA_ERR_UNSUPPORTED;
    }
    TRY(ensure_mixed(m, nrhs));
    return profile_apply<float2>(m->op32, m->kv32.r, m->kv32.p, m->al32, nrhs, iters, m->stream, ms_matvec, ms_pass);
}

tdda_status tdda_profile_gram_schmidt(tdda_model *m, int precision, int nv, int iters, double *ms) {
    if (!m || !ms || nv < 1 || nv > 1024 || iters < 1) return bad("bad argument");
    if (precision == 0) return profile_gram_schmidt<double2>(3 * m->nbox, nv, iters, m->stream, ms);
    if (precision == 1) return profile_gram_schmidt<float2>(3 * m->nbox, nv, iters, m->stream, ms);
    return bad("precision must be 0 or 1");
}

long long tdda_kernel_launches(void) { return launches_total(); }

tdda_status tdda_set_precision(tdda_model *m, int precision) {
    if (!m) return bad("null model");
    if (precision == TDDA_PREC_C128) { m->precision = TDDA_PREC_C128; return TDDA_OK; }
    if (precision == TDDA_PREC_MIXED) {
        if (m->op32.ahat == nullptr) {
            set_error("model was created in complex128: no complex64 operator");
            return TDDA_ERR_STATE;
        }
        m->precision = TDDA_PREC_MIXED;
        return TDDA_OK;
    }
    return bad("precision must be 0 or 1");
}

tdda_status tdda_set_time_limit(tdda_model *m, double seconds) {
    if (m == nullptr) return bad("null model");
    if (!(seconds >= 0.0)) return bad("time limit must be >= 0");
    m->time_limit_s = seconds;
    return TDDA_OK;
}

tdda_status tdda_filter_update(tdda_model *m, const double *step, int64_t n, int it, int max_it) {
    if (!m || !step) return bad("null argument");
    if (n != m->NFpara) return bad("step must hold NFpara values");
    std::vector<double> phys;
    TRY(m->lfilter.update(step, it, max_it, m->stream, phys));
    const std::vector<double> old = m->parameters;
    const bool old_pd = m->per_dipole;
    m->parameters = phys;
    m->per_dipole = false;
    tdda_status st = update_alpha(m);
    if (st != TDDA_OK) {
        m->parameters = old;
        m->per_dipole = old_pd;
    }
    return st;
}

tdda_status tdda_filter_gradients(tdda_model *m, const double *grad, int64_t n, int it, int max_it, double *out) {
    if (!m || !grad || !out) return bad("null argument");
    if (n != m->NFpara) return bad("gradients must hold NFpara values");
    return m->lfilter.gradients(grad, it, max_it, m->stream, out);
}

tdda_status tdda_filter_state(tdda_model *m, double *raw, double *filtered, int64_t n, double *beta) {
    if (!m) return bad("null argument");
    if (n != m->NFpara) return bad("buffers must hold NFpara values");
    TRY(m->lfilter.state(raw, filtered, m->stream));
    if (beta) *beta = m->lfilter.beta();
    return TDDA_OK;
}

tdda_status tdda_set_solver(tdda_model *m, int kind, int degree, int restart, int deflate) {
    if (m == nullptr) return bad("null model");
    if (kind < 0 || kind > 2)
        return bad("solver must be 0 (BiCGSTAB), 1 (polynomial-preconditioned GMRES) or 2 (GMRES carrying its "
                   "deflation space across refinement steps)");
    if (kind >= 1) {
        if (degree < 1 || degree > 64) return bad("polynomial degree must be in [1, 64]");
        if (restart < 2 || restart > 1024) return bad("GMRES restart must be in [2, 1024]");
        if (deflate < 0 || deflate >= restart) return bad("deflation vectors must be in [0, restart)");
        if (kind == 2 && (deflate < 1 || deflate + 6 > restart))
            return bad("carrying the deflation space needs 1 <= deflate <= restart - 6");
        m->gopt.degree = degree;
        m->gopt.restart = restart;
        m->gopt.deflate = deflate;
        m->gopt.recycle = kind == 2;
    }
    m->solver = kind == 0 ? 0 : 1;
    return TDDA_OK;
}

tdda_status tdda_set_preconditioner(tdda_model *m, int kind) {
    if (!m) return bad("null model");
    if (kind != 0 && kind != 1) return bad("preconditioner must be 0 (none) or 1 (Jacobi)");
    m->precond = kind;
    return TDDA_OK;
}

tdda_status tdda_set_observation_points(tdda_model *m, const int32_t *xyz, int64_t nobs) {
    if (!m || !xyz || nobs < 1) return bad("bad argument");
    if (nobs > 1 << 20) return bad("too many observation points");
    int lo[3], hi[3];
    const int nb[3] = {m->Nx, m->Ny, m->Nz};
    for (int a = 0; a < 3; ++a) {
        lo[a] = INT32_MAX;
        hi[a] = INT32_MIN;
    }
    std::vector<double2> einc(3 * (size_t)nobs);
    std::vector<char> occupied;  // built on the first point inside the box
    for (int64_t o = 0; o < nobs; ++o) {
        bool inside = true;
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], xyz[3 * o + a] - (nb[a] - 1));
            hi[a] = std::max(hi[a], (int)xyz[3 * o + a]);
            inside &= (xyz[3 * o + a] >= 0 && xyz[3 * o + a] < nb[a]);
        }
        if (inside) {
            if (occupied.empty()) {
                occupied.assign(m->nbox, 0);
                for (long long c : m->cell_of) occupied[c] = 1;
            }
            const long long cell = ((long long)xyz[3 * o] * m->Ny + xyz[3 * o + 1]) * m->Nz + xyz[3 * o + 2];
            if (occupied[cell]) return bad("observation point on a dipole");
        }
        // incident plane wave at the point (src/DDAModel.cpp:312-316 for a grid position)
        const double ph = m->K * m->d * (m->nK[0] * xyz[3 * o] + m->nK[1] * xyz[3 * o + 1] + m->nK[2] * xyz[3 * o + 2]);
        for (int c = 0; c < 3; ++c)
            einc[3 * o + c] = make_double2(m->E0 * m->nE0[c] * std::cos(ph), m->E0 * m->nE0[c] * std::sin(ph));
    }
    int n[3];
    long long total = 1;
    for (int a = 0; a < 3; ++a) {
        n[a] = hi[a] - lo[a] + 1;
        total *= n[a];
    }
    if (total > (1LL << 27)) return bad("observation points span too large an offset box");
    cudaFree(m->d_obs); cudaFree(m->Gobs); cudaFree(m->Einc_obs); cudaFree(m->Eobs);
    m->d_obs = nullptr; m->Gobs = m->Einc_obs = m->Eobs = nullptr; m->nobs = 0;
    TDDA_CUDA_TRY(cudaMalloc(&m->d_obs, sizeof(int) * 3 * nobs));
    TDDA_CUDA_TRY(cudaMemcpy(m->d_obs, xyz, sizeof(int) * 3 * nobs, cudaMemcpyHostToDevice));
    TDDA_CUDA_TRY(cudaMalloc(&m->Gobs, sizeof(double2) * 6 * total));
    TDDA_CUDA_TRY(cudaMalloc(&m->Einc_obs, sizeof(double2) * 3 * nobs));
    TDDA_CUDA_TRY(cudaMalloc(&m->Eobs, sizeof(double2) * 3 * nobs));
    TDDA_CUDA_TRY(cudaMemcpy(m->Einc_obs, einc.data(), sizeof(double2) * 3 * nobs, cudaMemcpyHostToDevice));
    TRY(build_offset_tensor(m->lat, m->si_h.data(), m->ci_h.data(), (long)m->si_h.size(), lo[0], lo[1], lo[2], n[0],
                            n[1], n[2], m->Gobs, m->stream));
    for (int a = 0; a < 3; ++a) {
        m->obs_lo[a] = lo[a];
        m->obs_n[a] = n[a];
    }
    m->nobs = (int)nobs;
    return TDDA_OK;
}

static PatchGeo patch_geo(const tdda_model *m) {
    return {m->Nx, m->Ny, m->Nz, m->obs_lo[0], m->obs_lo[1], m->obs_lo[2], m->obs_n[0], m->obs_n[1], m->obs_n[2]};
}

static tdda_status patch_field(tdda_model *m) {
    if (m->nobs == 0) {
        set_error("no observation points: call tdda_set_observation_points first");
        return TDDA_ERR_STATE;
    }
    count_launches(1);
    k_patch_field<<<m->nobs, 256, 0, m->stream>>>(m->nobs, m->d_obs, patch_geo(m), m->d_mask, m->P, m->nbox,
                                                  m->Gobs, m->Einc_obs, m->Eobs);
    TDDA_CUDA_TRY(cudaGetLastError());
    return TDDA_OK;
}

tdda_status tdda_observation_field(tdda_model *m, double *E, int64_t n) {
    if (!m || !E) return bad("null argument");
    if (n != 3LL * m->nobs) return bad("buffer must hold 3 complex values per observation point");
    TRY(patch_field(m));
    TDDA_CUDA_TRY(cudaMemcpyAsync(E, m->Eobs, sizeof(double2) * 3 * m->nobs, cudaMemcpyDeviceToHost, m->stream));
    TDDA_CUDA_TRY(cudaStreamSynchronize(m->stream));
    return TDDA_OK;
}

tdda_status tdda_patch_objective(tdda_model *m, double *out) {
    if (!m || !out) return bad("null argument");
    std::vector<double2> e(3 * (size_t)m->nobs);
    TRY(tdda_observation_field(m, reinterpret_cast<double *>(e.data()), 3LL * m->nobs));
    double s = 0.0;
    for (const double2 &v : e) s += v.x * v.x + v.y * v.y;
    *out = s / m->nobs;
    return TDDA_OK;
}

// The exact adjoint gradient of the patch objective per cell into m->d_grad.
static tdda_status patch_gradient_cells(tdda_model *m, int max_iter, double tol, tdda_solve_info *info) {
    TRY(patch_field(m));
    TRY(ensure_batch(m, 1));
    TRY(ensure_grad_scratch(m));
    const long long nbox = m->nbox;
    count_launches(1);
    k_patch_adjoint_rhs<<<grid_for(nbox), 256, 0, m->stream>>>(m->nobs, m->d_obs, patch_geo(m), m->d_mask, nbox,
                                                                m->Gobs, m->Eobs, m->bufB);
    TDDA_CUDA_TRY(cudaGetLastError());
    tdda_solve_info inf{};
    TRY(solve_internal(m, m->bufB, m->bufX, 1, true, max_iter, tol, &inf));
    count_launches(1);
    k_grad_implicit<<<grid_for(nbox), 256, 0, m->stream>>>(nbox, m->d_mask, m->P, m->diel, m->bufX, m->ap, m->d_grad);
    TDDA_CUDA_TRY(cudaGetLastError());
    if (info) *info = inf;
    return TDDA_OK;
}

tdda_status tdda_patch_gradient(tdda_model *m, int max_iter, double tol, double *grad, int64_t n,
                                tdda_solve_info *info) {
    if (!m || !grad) return bad("null argument");
    if (n != m->N) return bad("gradient buffer must hold N values");
    TRY(patch_gradient_cells(m, max_iter, tol, info));
    return cells_to_host(m, m->d_grad, grad);
}

tdda_status tdda_patch_gradient_device(tdda_model *m, int max_iter, double tol, double *grad_dev, void *stream,
                                       tdda_solve_info *info) {
    if (!m || !grad_dev) return bad("null argument");
    TRY(join_streams((cudaStream_t)stream, m->stream));
    TRY(patch_gradient_cells(m, max_iter, tol, info));
    return cells_to_device(m, m->d_grad, grad_dev, (cudaStream_t)stream);
}

}  // extern "C"
