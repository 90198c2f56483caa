/*
 * ORACLE — test infrastructure only.  Nothing in the product links this file;
 * it is built into oracle/_build/liboracle_lattice.so and loaded by the tests,
 * by __graft_entry__.smoke() and by bench.py's CPU-baseline leg, as the
 * checker for the CUDA lattice-sum kernel.
 *
 * Plain-C restatement of Topo-DDA's interaction-tensor assembly:
 *   - SiCi::get_Si / SiCi::get_Ci           src/SiCi.cpp:12-44
 *   - AProductCore::FCD_inter                src/AProductCore.cpp:388-459
 *   - AProductCore::LDR_inter                src/AProductCore.cpp:351-386
 *   - AProductCore::A_dic_generator(x,y,z,m,n) (image shift + damping)
 *                                            src/AProductCore.cpp:335-349
 *   - the 8 octant loops that fill AHos      src/AProductCore.cpp:62-244
 *
 * Output layout is the reference's AHos: double[12*NFFT], index
 *   2*l + {0,1} + 12*(k + NzFFT*(j + NyFFT*i)),  l in {xx,xy,xz,yy,yz,zz},
 * with NxFFT = 2Nx-1 etc. (src/AProductCore.cpp:50-53,81-82).
 *
 * Two documented departures, both about undefined behaviour in the reference:
 *   1. r == 0: FCD_inter/LDR_inter set only the diagonal to 0 and leave the
 *      off-diagonals uninitialised (src/AProductCore.cpp:395-400,356-361).
 *      Here the whole self term is 0 (in the periodic reference build the
 *      reused stack slot holds the previous image's off-diagonals, which are
 *      exactly 0 for the (0,0,0) entry, so this matches it).
 *   2. SiCi lookup with x/delta an exact integer gives 0/0 = NaN in the
 *      reference (src/SiCi.cpp:23-27) and x < delta reads index -1.  Here the
 *      exact-integer case returns the table value itself (the limit of the
 *      interpolant) and x < delta clamps to the first entry; the flag counter
 *      `oracle_sici_guard_hits` records how often either happened.
 *
 * `full != 0` evaluates every padded entry exactly as the reference does
 * (m outer, n inner).  `full == 0` evaluates only the non-negative octant and
 * fills the rest by parity (xx,yy,zz even in every axis; xy odd in x and y;
 * xz odd in x and z; yz odd in y and z): the image set of a mirrored offset is
 * the mirrored image set, so this is the same sum taken in reversed m/n order
 * (equal up to rounding).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#include <stdlib.h>
#include <pthread.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

long oracle_sici_guard_hits = 0;

static double sici_lookup(const double *tab, long n, double delta, double x)
{
    /* src/SiCi.cpp:12-28 */
    double q = x / delta;
    long pos1 = (long)floor(q) - 1;
    long pos2 = (long)ceil(q) - 1;
    if (pos2 >= n) return tab[n - 1];
    if (pos1 < 0) {
        __atomic_fetch_add(&oracle_sici_guard_hits, 1, __ATOMIC_RELAXED);
        pos1 = 0;
        if (pos2 < 0) pos2 = 0;
    }
    double val1 = tab[pos1];
    double val2 = tab[pos2];
    if (pos1 == pos2) {
        __atomic_fetch_add(&oracle_sici_guard_hits, 1, __ATOMIC_RELAXED);
        return val1;
    }
    double axis1 = (double)(pos1 + 1) * delta;
    double axis2 = (double)(pos2 + 1) * delta;
    return val1 + ((val2 - val1) / (axis2 - axis1)) * (x - axis1);
}

/* 6 complex components (re,im interleaved): xx,xy,xz,yy,yz,zz */
static void fcd_inter(double x, double y, double z, double K, double d,
                      const double *si, const double *ci, long ntab, double delta,
                      double out[12])
{
    double xs = x * x, ys = y * y, zs = z * z;
    double r = sqrt(xs + ys + zs);
    memset(out, 0, 12 * sizeof(double));
    if (r == 0.0) return;
    double xy = x * y, yz = y * z, zx = z * x;
    double r2 = r * r;
    double r3 = r * r * r;
    double Kf = M_PI / d;
    double Cz = sici_lookup(ci, ntab, delta, (Kf + K) * r);
    double Cf = sici_lookup(ci, ntab, delta, (Kf - K) * r);
    double Sz = sici_lookup(si, ntab, delta, (Kf + K) * r);
    double Sf = sici_lookup(si, ntab, delta, (Kf - K) * r);
    double ap = (Kf + K) * r, am = (Kf - K) * r;
    double Cz1 = cos(ap) / r;
    double Cf1 = cos(am) / r;
    double Sz1 = sin(ap) / r;
    double Sf1 = sin(am) / r;
    double Cz2 = (-ap * sin(ap) - cos(ap)) / r2;
    double Cf2 = (-am * sin(am) - cos(am)) / r2;
    double Sz2 = (ap * cos(ap) - sin(ap)) / r2;
    double Sf2 = (am * cos(am) - sin(am)) / r2;
    double kr = K * r;
    double sikr = sin(kr), cskr = cos(kr);
    double sikfr = sin(Kf * r), cskfr = cos(Kf * r);
    /* CC = i*pi + Cf - Cz (complex), everything else real */
    double CCr = Cf - Cz, CCi = M_PI;
    double C1C1 = Cf1 - Cz1;
    double C2C2 = Cf2 - Cz2;
    double SS = Sz + Sf;
    double S1S1 = Sz1 + Sf1;
    double S2S2 = Sz2 + Sf2;
    /* gf = (sikr*CC + cskr*SS) / (pi r) */
    double gfr = (sikr * CCr + cskr * SS) / (M_PI * r);
    double gfi = (sikr * CCi) / (M_PI * r);
    /* const1 = (kr cskr - sikr) CC - (kr sikr + cskr) SS + r sikr C1C1 + r cskr S1S1 */
    double a1 = kr * cskr - sikr;
    double c1r = a1 * CCr - (kr * sikr + cskr) * SS + r * sikr * C1C1 + r * cskr * S1S1;
    double c1i = a1 * CCi;
    /* const2 = (-K kr sikr) CC - (K kr cskr) SS + 2 kr cskr C1C1 - 2 kr sikr S1S1
     *          + r sikr C2C2 + r cskr S2S2 */
    double a2 = -K * kr * sikr;
    double c2r = a2 * CCr - (K * kr * cskr) * SS + (2 * kr * cskr) * C1C1 - (2 * kr * sikr) * S1S1
                 + r * sikr * C2C2 + r * cskr * S2S2;
    double c2i = a2 * CCi;
    double gf1r = c1r / (M_PI * r2), gf1i = c1i / (M_PI * r2);
    double gf2r = (r * c2r - 2.0 * c1r) / (M_PI * r3);
    double gf2i = (r * c2i - 2.0 * c1i) / (M_PI * r3);
    double hr = (sikfr - Kf * r * cskfr) / (2.0 * M_PI * M_PI * r3);
    double t1r = K * K * gfr + gf1r / r + (4.0 * M_PI / 3.0) * hr;
    double t1i = K * K * gfi + gf1i / r;
    double t2r = (gf2r - gf1r / r) / r2;
    double t2i = (gf2i - gf1i / r) / r2;
    /* result = -(term1*I + rr^T term2) */
    out[0] = -(t1r + xs * t2r);  out[1] = -(t1i + xs * t2i);
    out[2] = -(xy * t2r);        out[3] = -(xy * t2i);
    out[4] = -(zx * t2r);        out[5] = -(zx * t2i);
    out[6] = -(t1r + ys * t2r);  out[7] = -(t1i + ys * t2i);
    out[8] = -(yz * t2r);        out[9] = -(yz * t2i);
    out[10] = -(t1r + zs * t2r); out[11] = -(t1i + zs * t2i);
}

static void ldr_inter(double x, double y, double z, double K, double out[12])
{
    /* src/AProductCore.cpp:351-386 */
    double xs = x * x, ys = y * y, zs = z * z;
    double r = sqrt(xs + ys + zs);
    memset(out, 0, 12 * sizeof(double));
    if (r == 0.0) return;
    double xy = x * y, yz = y * z, zx = z * x;
    double r2 = r * r, r3 = r * r * r;
    /* const1 = exp(i K r) / r^3 */
    double k1r = cos(K * r) / r3, k1i = sin(K * r) / r3;
    /* const2 = (1 - i K r) / r^2 */
    double k2r = 1.0 / r2, k2i = -K * r / r2;
    /* const3 = K^2 - 3 const2 */
    double k3r = K * K - 3.0 * k2r, k3i = -3.0 * k2i;
    double m[12];
    m[0] = k2r * (r2 - 3 * xs) - K * K * (ys + zs); m[1] = k2i * (r2 - 3 * xs);
    m[2] = xy * k3r; m[3] = xy * k3i;
    m[4] = zx * k3r; m[5] = zx * k3i;
    m[6] = k2r * (r2 - 3 * ys) - K * K * (zs + xs); m[7] = k2i * (r2 - 3 * ys);
    m[8] = yz * k3r; m[9] = yz * k3i;
    m[10] = k2r * (r2 - 3 * zs) - K * K * (xs + ys); m[11] = k2i * (r2 - 3 * zs);
    for (int l = 0; l < 6; l++) {
        double ar = m[2 * l], ai = m[2 * l + 1];
        out[2 * l] = k1r * ar - k1i * ai;
        out[2 * l + 1] = k1r * ai + k1i * ar;
    }
}

/* AProductCore::A_dic_generator(x,y,z) (method 0 = FCD, 1 = LDR) */
void oracle_green(int method, double x, double y, double z, double K, double d,
                  const double *si, const double *ci, long ntab, double delta, double out[12])
{
    if (method == 0) fcd_inter(x, y, z, K, d, si, ci, ntab, delta, out);
    else ldr_inter(x, y, z, K, out);
}

/* AProductCore::A_dic_generator(x,y,z,m,n): shift by the lattice vector and damp */
void oracle_green_image(int method, double x, double y, double z, int m, int n, double Lm, double Ln,
                        double K, double d, const double *si, const double *ci, long ntab,
                        double delta, double out[12])
{
    const double gamma = 0.01;
    x = x + m * Lm;
    y = y + n * Ln;
    oracle_green(method, x, y, z, K, d, si, ci, ntab, delta, out);
    double damp = exp(-pow(gamma * K * sqrt(x * x + y * y + z * z), 4));
    for (int l = 0; l < 12; l++) out[l] *= damp;
}

static void entry_sum(int method, double x, double y, double z, int MAXm, int MAXn, double Lm,
                      double Ln, double K, double d, const double *si, const double *ci, long ntab,
                      double delta, double acc[12])
{
    double g[12];
    memset(acc, 0, 12 * sizeof(double));
    for (int m = -MAXm; m <= MAXm; m++)
        for (int n = -MAXn; n <= MAXn; n++) {
            oracle_green_image(method, x, y, z, m, n, Lm, Ln, K, d, si, ci, ntab, delta, g);
            for (int l = 0; l < 12; l++) acc[l] += g[l];
        }
}

/* parity sign of component l under mirroring of the axes in `mir` (bit0=x, bit1=y, bit2=z) */
static int parity_sign(int l, int mir)
{
    static const int odd_axes[6] = {0, 3, 5, 0, 6, 0}; /* xx,xy(x|y),xz(x|z),yy,yz(y|z),zz */
    int bits = odd_axes[l] & mir;
    int s = 1;
    while (bits) { s = -s; bits &= bits - 1; }
    return s;
}

/*
 * Fill AHos (reference layout, double[12 * NFFT]).  Lm, Ln are lengths (already
 * multiplied by d, as DDAModel passes them: src/DDAModel.cpp:281).  The padded
 * entries are split over `nthreads` POSIX threads (work unit: one i-plane).
 */
typedef struct {
    int Nx, Ny, Nz, MAXm, MAXn, method, full;
    double d, K, Lm, Ln, delta;
    const double *si, *ci;
    long ntab;
    double *AHos;
    int next; /* next i-plane to take (atomic) */
} lattice_job;

static void lattice_plane(lattice_job *J, int i)
{
    int Nx = J->Nx, Ny = J->Ny, Nz = J->Nz;
    int NxF = 2 * Nx - 1, NyF = 2 * Ny - 1, NzF = 2 * Nz - 1;
    double acc[12];
    if (J->full) {
        for (int j = 0; j < NyF; j++)
            for (int k = 0; k < NzF; k++) {
                double x = J->d * (i < Nx ? i : i - NxF);
                double y = J->d * (j < Ny ? j : j - NyF);
                double z = J->d * (k < Nz ? k : k - NzF);
                entry_sum(J->method, x, y, z, J->MAXm, J->MAXn, J->Lm, J->Ln, J->K, J->d, J->si, J->ci,
                          J->ntab, J->delta, acc);
                long idx = (long)k + (long)NzF * ((long)j + (long)NyF * i);
                memcpy(J->AHos + 12 * idx, acc, sizeof(acc));
            }
        return;
    }
    for (int j = 0; j < Ny; j++)
        for (int k = 0; k < Nz; k++) {
            entry_sum(J->method, J->d * i, J->d * j, J->d * k, J->MAXm, J->MAXn, J->Lm, J->Ln, J->K, J->d,
                      J->si, J->ci, J->ntab, J->delta, acc);
            for (int mir = 0; mir < 8; mir++) {
                if ((mir & 1) && i == 0) continue;
                if ((mir & 2) && j == 0) continue;
                if ((mir & 4) && k == 0) continue;
                int ii = (mir & 1) ? NxF - i : i;
                int jj = (mir & 2) ? NyF - j : j;
                int kk = (mir & 4) ? NzF - k : k;
                long idx = (long)kk + (long)NzF * ((long)jj + (long)NyF * ii);
                for (int l = 0; l < 6; l++) {
                    int s = parity_sign(l, mir);
                    J->AHos[12 * idx + 2 * l] = s * acc[2 * l];
                    J->AHos[12 * idx + 2 * l + 1] = s * acc[2 * l + 1];
                }
            }
        }
}

static void *lattice_worker(void *arg)
{
    lattice_job *J = (lattice_job *)arg;
    int nplanes = J->full ? 2 * J->Nx - 1 : J->Nx;
    for (;;) {
        int i = __atomic_fetch_add(&J->next, 1, __ATOMIC_RELAXED);
        if (i >= nplanes) break;
        lattice_plane(J, i);
    }
    return NULL;
}

int oracle_lattice(int Nx, int Ny, int Nz, double d, double K, double Lm, double Ln, int MAXm,
                   int MAXn, int method, const double *si, const double *ci, long ntab,
                   double delta, int full, int nthreads, double *AHos)
{
    lattice_job J = {Nx, Ny, Nz, MAXm, MAXn, method, full, d, K, Lm, Ln, delta, si, ci, ntab, AHos, 0};
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    int started = 0;
    for (int t = 1; t < nthreads; t++)
        if (pthread_create(&th[started], NULL, lattice_worker, &J) == 0) started++;
    lattice_worker(&J);
    for (int t = 0; t < started; t++) pthread_join(th[t], NULL);
    return 0;
}

/* the 4 lookups FCD uses, exposed for tests of the table quirks */
double oracle_get_si(const double *si, long n, double delta, double x) { return sici_lookup(si, n, delta, x); }
double oracle_get_ci(const double *ci, long n, double delta, double x) { return sici_lookup(ci, n, delta, x); }
long oracle_guard_hits(void) { return oracle_sici_guard_hits; }

/* Lattice sums (same images and damping as the tensor entries) at arbitrary
 * offsets xyz[3*npts] (lengths): out[12*npts], components xx,xy,xz,yy,yz,zz.
 * Used for fields at observation points outside the dipole grid. */
int oracle_lattice_points(int method, long npts, const double *xyz, int MAXm, int MAXn, double Lm, double Ln,
                          double K, double d, const double *si, const double *ci, long ntab, double delta,
                          double *out)
{
    for (long p = 0; p < npts; p++)
        entry_sum(method, xyz[3 * p], xyz[3 * p + 1], xyz[3 * p + 2], MAXm, MAXn, Lm, Ln, K, d, si, ci, ntab,
                  delta, out + 12 * p);
    return 0;
}
