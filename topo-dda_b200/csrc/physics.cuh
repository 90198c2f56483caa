// Per-dipole physics shared by the model and the serving engine: material
// interpolation, the lattice-dispersion-relation polarisability and its
// derivative, the Jacobi scale of the operator diagonal.
#pragma once

#include "tdda_common.cuh"

namespace tdda {

// polarisability of the lattice dispersion relation, 1/alpha
// (src/Tools.cpp:353-366; interpolation src/DDAModel.cpp:319-328)
struct AlphaParams {
    double lam, K, d;
    double2 m0, m1;   // rescaled materials
    double S;         // sum_c (n_E0,c n_K,c)^2
};

__host__ __device__ inline double2 cmul_d(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__host__ __device__ inline double2 diel_of(double rho, const AlphaParams &A) {
    // labelfloor = floor(rho), labelnext = floor+1 unless floor >= 1
    double lf = floor(rho);
    double2 mf = lf >= 1.0 ? A.m1 : A.m0;
    double2 mn = (lf >= 1.0 || lf + 1.0 >= 1.0) ? A.m1 : A.m0;
    double w = rho - lf;
    return make_double2(mf.x + w * (mn.x - mf.x), mf.y + w * (mn.y - mf.y));
}

__host__ __device__ inline double2 inv_alpha(double2 eps, const AlphaParams &A) {
    // same operation order as Get_Alpha (src/Tools.cpp:353-366)
    const double b1 = -1.891531, b2 = 0.1648469, b3 = -1.7700004;
    const double d3 = A.d * A.d * A.d;
    const double pre = 3.0 * d3 / (4.0 * M_PI);
    double2 num = make_double2(pre * (eps.x - 1.0), pre * eps.y);
    double2 a1 = cdiv(num, make_double2(eps.x + 2.0, eps.y));
    const double kd = A.K * A.d;
    const double kd2 = kd * kd;
    double2 rad = make_double2(0.0, (2.0 / 3.0) * (kd * kd * kd));
    // (b1 + eps b2 + eps b3 S) (Kd)^2 - rad
    double2 poly = make_double2(b1 + eps.x * b2 + (eps.x * b3) * A.S, eps.y * b2 + (eps.y * b3) * A.S);
    double2 t = make_double2(poly.x * kd2 - rad.x, poly.y * kd2 - rad.y);
    double2 a1d = make_double2(a1.x / d3, a1.y / d3);
    double2 res = cmul_d(a1d, t);
    res.x = 1.0 + res.x;
    double2 alpha = cdiv(a1, res);
    return cdiv(make_double2(1.0, 0.0), alpha);
}

// principal square root
__host__ __device__ inline double2 csqrt_d(double2 z) {
    double r = hypot(z.x, z.y);
    double re = sqrt(0.5 * (r + z.x));
    double im = sqrt(0.5 * fmax(r - z.x, 0.0));
    return make_double2(re, z.y < 0 ? -im : im);
}

// Jacobi scale of one diagonal entry: D = al + a0 (a0: mean of the diagonal of
// the zero-offset lattice entry), sc = D^(-1/2).
__host__ __device__ inline double2 jacobi_scale(double2 al, double2 a0) {
    return cdiv(make_double2(1.0, 0.0), csqrt_d(make_double2(al.x + a0.x, al.y + a0.y)));
}

// d(1/alpha)/d rho: (-3 / (c (eps - 1)^2) + (b2 + b3 S) K^2 / d) (m1 - m0),
// c = 3 d^3 / (4 pi) -- the closed-form derivative of Get_Alpha's inverse.
__host__ __device__ inline double2 dal_drho(double2 eps, const AlphaParams &A) {
    const double b2 = 0.1648469, b3 = -1.7700004;
    const double c = 3.0 * A.d * A.d * A.d / (4.0 * M_PI);
    double2 em1 = make_double2(eps.x - 1.0, eps.y);
    double2 sq = cmul_d(em1, em1);
    double2 t = cdiv(make_double2(-3.0 / c, 0.0), sq);
    t.x += (b2 + b3 * A.S) * A.K * A.K / A.d;
    return cmul_d(t, make_double2(A.m1.x - A.m0.x, A.m1.y - A.m0.y));
}

}  // namespace tdda
