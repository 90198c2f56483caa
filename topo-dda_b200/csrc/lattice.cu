// Interaction-tensor assembly on the device (FP64).
//
// Reference: the AProductCore constructor (src/AProductCore.cpp:12-298): for
// every signed grid offset, A = sum over periodic images (m, n) of the damped
// Green tensor A_dic_generator(x + m Lm, y + n Ln, z) (:335-349), with the
// filtered-coupled-dipole (FCD_inter :388-459, sine/cosine integrals from the
// SiCi tables of src/SiCi.cpp:12-44) or point-dipole (LDR_inter :351-386)
// kernel; then the six tensor components are FFT'd once (:262-279).
//
// Device design:
//   k_lattice  one group of `lanes` threads per non-negative offset (the
//              octant); lanes split the image loop, their partial sums are
//              combined by a fixed shuffle tree, and lane 0 writes the sum
//              into all eight mirrored slots of the padded grid with the
//              parity sign of each component (xx, yy, zz even in every axis;
//              xy odd in x,y; xz odd in x,z; yz odd in y,z) -- 8x less work
//              than evaluating each signed offset.
//   k_fft_lines_*  batched FP64 line FFTs of the padded grid along z, y, x.
//   k_fold     keeps the folded spectral octant [hy][hx][hz][6] (the spectrum
//              has the same parity), scaled by 1/(Lx Ly Lz) so the inverse
//              transforms of the matvec need no normalisation.
#include <cmath>
#include <vector>

#include "fft_smem.cuh"
#include "lattice.cuh"

namespace tdda {

constexpr int LNT = 256;

// SiCi::get_Si / get_Ci (src/SiCi.cpp:12-44) on a table of (si, ci) pairs.
// Guards: x/delta an exact integer returns the table value (the reference
// divides 0 by 0 there); x < delta clamps to the first entry (the reference
// reads index -1).
__device__ __forceinline__ void sici_pair(const double2 *__restrict__ tab, long ntab, double delta,
                                          double x, double &si, double &ci) {
    double q = x / delta;
    long pos1 = (long)floor(q) - 1;
    long pos2 = (long)ceil(q) - 1;
    if (pos2 >= ntab) {
        double2 v = __ldg(tab + ntab - 1);
        si = v.x;
        ci = v.y;
        return;
    }
    if (pos1 < 0) {
        pos1 = 0;
        if (pos2 < 0) pos2 = 0;
    }
    double2 v1 = __ldg(tab + pos1);
    if (pos1 == pos2) {
        si = v1.x;
        ci = v1.y;
        return;
    }
    double2 v2 = __ldg(tab + pos2);
    double axis1 = __dmul_rn((double)(pos1 + 1), delta);
    double axis2 = __dmul_rn((double)(pos2 + 1), delta);
    double den = __dsub_rn(axis2, axis1);
    double dx = __dsub_rn(x, axis1);
    si = __dadd_rn(v1.x, __dmul_rn(__ddiv_rn(__dsub_rn(v2.x, v1.x), den), dx));
    ci = __dadd_rn(v1.y, __dmul_rn(__ddiv_rn(__dsub_rn(v2.y, v1.y), den), dx));
}

// One undamped Green-tensor term, accumulated as acc += damp * (-G).
// Components xx, xy, xz, yy, yz, zz as (re, im) pairs.
__device__ __forceinline__ void fcd_term(double x, double y, double z, double r, double damp,
                                         const LatticeParams &P, double (&acc)[12]) {
    const double K = P.K, Kf = P.Kf;
    const double xs = x * x, ys = y * y, zs = z * z;
    const double r2 = r * r, r3 = r2 * r;
    const double ap = (Kf + K) * r, am = (Kf - K) * r;
    double Sz, Cz, Sf, Cf;
    sici_pair(P.sc, P.ntab, P.delta, ap, Sz, Cz);
    sici_pair(P.sc, P.ntab, P.delta, am, Sf, Cf);
    double sap, cap, sam, cam, sikr, cskr, sikfr, cskfr;
    sincos(ap, &sap, &cap);
    sincos(am, &sam, &cam);
    sincos(K * r, &sikr, &cskr);
    sincos(Kf * r, &sikfr, &cskfr);
    const double ir = 1.0 / r, ir2 = 1.0 / r2;
    const double Cz1 = cap * ir, Cf1 = cam * ir, Sz1 = sap * ir, Sf1 = sam * ir;
    const double Cz2 = (-ap * sap - cap) * ir2;
    const double Cf2 = (-am * sam - cam) * ir2;
    const double Sz2 = (ap * cap - sap) * ir2;
    const double Sf2 = (am * cam - sam) * ir2;
    const double kr = K * r;
    const double CCr = Cf - Cz, CCi = M_PI;
    const double C1C1 = Cf1 - Cz1, C2C2 = Cf2 - Cz2;
    const double SS = Sz + Sf, S1S1 = Sz1 + Sf1, S2S2 = Sz2 + Sf2;
    const double ipr = 1.0 / (M_PI * r);
    const double gfr = (sikr * CCr + cskr * SS) * ipr;
    const double gfi = (sikr * CCi) * ipr;
    const double a1 = kr * cskr - sikr;
    const double c1r = a1 * CCr - (kr * sikr + cskr) * SS + r * sikr * C1C1 + r * cskr * S1S1;
    const double c1i = a1 * CCi;
    const double a2 = -K * kr * sikr;
    const double c2r = a2 * CCr - (K * kr * cskr) * SS + (2 * kr * cskr) * C1C1 - (2 * kr * sikr) * S1S1 +
                       r * sikr * C2C2 + r * cskr * S2S2;
    const double c2i = a2 * CCi;
    const double ipr2 = 1.0 / (M_PI * r2), ipr3 = 1.0 / (M_PI * r3);
    const double gf1r = c1r * ipr2, gf1i = c1i * ipr2;
    const double gf2r = (r * c2r - 2.0 * c1r) * ipr3;
    const double gf2i = (r * c2i - 2.0 * c1i) * ipr3;
    const double hr = (sikfr - Kf * r * cskfr) / (2.0 * M_PI * M_PI * r3);
    const double t1r = K * K * gfr + gf1r * ir + (4.0 * M_PI / 3.0) * hr;
    const double t1i = K * K * gfi + gf1i * ir;
    const double t2r = (gf2r - gf1r * ir) * ir2;
    const double t2i = (gf2i - gf1i * ir) * ir2;
    const double md = -damp;
    acc[0] += md * (t1r + xs * t2r);  acc[1] += md * (t1i + xs * t2i);
    acc[2] += md * (x * y * t2r);     acc[3] += md * (x * y * t2i);
    acc[4] += md * (z * x * t2r);     acc[5] += md * (z * x * t2i);
    acc[6] += md * (t1r + ys * t2r);  acc[7] += md * (t1i + ys * t2i);
    acc[8] += md * (y * z * t2r);     acc[9] += md * (y * z * t2i);
    acc[10] += md * (t1r + zs * t2r); acc[11] += md * (t1i + zs * t2i);
}

__device__ __forceinline__ void ldr_term(double x, double y, double z, double r, double damp,
                                         const LatticeParams &P, double (&acc)[12]) {
    const double K = P.K;
    const double xs = x * x, ys = y * y, zs = z * z;
    const double r2 = r * r, r3 = r2 * r;
    double s, c;
    sincos(K * r, &s, &c);
    const double k1r = c / r3, k1i = s / r3;
    const double k2r = 1.0 / r2, k2i = -K * r / r2;
    const double k3r = K * K - 3.0 * k2r, k3i = -3.0 * k2i;
    double m[12];
    m[0] = k2r * (r2 - 3 * xs) - K * K * (ys + zs); m[1] = k2i * (r2 - 3 * xs);
    m[2] = x * y * k3r; m[3] = x * y * k3i;
    m[4] = z * x * k3r; m[5] = z * x * k3i;
    m[6] = k2r * (r2 - 3 * ys) - K * K * (zs + xs); m[7] = k2i * (r2 - 3 * ys);
    m[8] = y * z * k3r; m[9] = y * z * k3i;
    m[10] = k2r * (r2 - 3 * zs) - K * K * (xs + ys); m[11] = k2i * (r2 - 3 * zs);
#pragma unroll
    for (int l = 0; l < 6; ++l) {
        double ar = m[2 * l], ai = m[2 * l + 1];
        acc[2 * l] += damp * (k1r * ar - k1i * ai);
        acc[2 * l + 1] += damp * (k1r * ai + k1i * ar);
    }
}

__device__ __forceinline__ int parity_sign(int l, int mir) {
    // odd axes per component: xx -, xy x|y, xz x|z, yy -, yz y|z, zz -
    const int odd = (l == 1) ? 3 : (l == 2) ? 5 : (l == 4) ? 6 : 0;
    return (__popc(odd & mir) & 1) ? -1 : 1;
}

__global__ void __launch_bounds__(LNT) k_lattice(LatticeParams P, double2 *__restrict__ G, int lanes) {
    const long long gid = (long long)blockIdx.x * LNT + threadIdx.x;
    const long long entry = gid / lanes;
    const int lane = (int)(gid % lanes);
    const long long nent = (long long)P.nx * P.ny * P.nz;
    const bool valid = entry < nent;
    int i = 0, j = 0, k = 0;
    if (valid) {
        i = (int)(entry / ((long long)P.ny * P.nz));
        int rem = (int)(entry - (long long)i * P.ny * P.nz);
        j = rem / P.nz;
        k = rem - j * P.nz;
    }
    double acc[12];
#pragma unroll
    for (int l = 0; l < 12; ++l) acc[l] = 0.0;
    if (valid) {
        const double x0 = P.d * i, y0 = P.d * j, z = P.d * k;
        const int nm = 2 * P.MAXm + 1, nn = 2 * P.MAXn + 1;
        const int nimg = nm * nn;
        const double gk = P.gamma * P.K;
        for (int q = lane; q < nimg; q += lanes) {
            const int m = q / nn - P.MAXm;
            const int n = q % nn - P.MAXn;
            const double x = x0 + m * P.Lm;
            const double y = y0 + n * P.Ln;
            const double r = sqrt(x * x + y * y + z * z);
            if (r == 0.0) continue;  // self term: zero (see oracle header)
            const double e = gk * r;
            const double e2 = e * e, e4 = e2 * e2;
            if (e4 > 746.0) continue;  // exp(-e4) == 0 in double: the term is exactly 0
            const double damp = exp(-e4);
            if (P.method == 0) fcd_term(x, y, z, r, damp, P, acc);
            else ldr_term(x, y, z, r, damp, P, acc);
        }
    }
    // fixed-shape tree over the lanes of one entry (lanes is a power of two)
    for (int off = lanes >> 1; off > 0; off >>= 1)
#pragma unroll
        for (int l = 0; l < 12; ++l) acc[l] += __shfl_down_sync(0xffffffffu, acc[l], off, lanes);
    if (!valid || lane != 0) return;
    const size_t Lyz = (size_t)P.Ly * P.Lz, Lxyz = (size_t)P.Lx * Lyz;
    for (int mir = 0; mir < 8; ++mir) {
        if ((mir & 1) && i == 0) continue;
        if ((mir & 2) && j == 0) continue;
        if ((mir & 4) && k == 0) continue;
        const int ii = (mir & 1) ? P.Lx - i : i;
        const int jj = (mir & 2) ? P.Ly - j : j;
        const int kk = (mir & 4) ? P.Lz - k : k;
        const size_t idx = (size_t)ii * Lyz + (size_t)jj * P.Lz + kk;
#pragma unroll
        for (int l = 0; l < 6; ++l) {
            const double s = parity_sign(l, mir);
            G[(size_t)l * Lxyz + idx] = make_double2(s * acc[2 * l], s * acc[2 * l + 1]);
        }
    }
}

// Lines along a strided axis: data viewed as [outer][L][inner], CTA = one
// outer index and a tile of TI consecutive inner indices.
__global__ void __launch_bounds__(LNT) k_fft_lines_strided(double2 *__restrict__ data, int L, long long inner,
                                                           int TI, const double2 *__restrict__ tw, int Lmax,
                                                           long long comp_stride) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *S = reinterpret_cast<double2 *>(smem_raw);
    const long long o = blockIdx.y;
    const long long i0 = (long long)blockIdx.x * TI;
    const int nb = (int)min((long long)TI, inner - i0);
    double2 *base = data + (size_t)blockIdx.z * comp_stride + (size_t)o * L * inner + i0;
    for (int e = threadIdx.x; e < L * nb; e += LNT) {
        int pos = e / nb, il = e - pos * nb;
        S[pos * nb + il] = base[(size_t)pos * inner + il];
    }
    __syncthreads();
    fft_smem<-1, 4>(S, L, nb, nb, 1, tw, Lmax);
    for (int e = threadIdx.x; e < L * nb; e += LNT) {
        int pos = e / nb, il = e - pos * nb;
        base[(size_t)pos * inner + il] = S[pos * nb + il];
    }
}

// Lines along the contiguous axis: CTA = TO consecutive lines of length L.
__global__ void __launch_bounds__(LNT) k_fft_lines_contig(double2 *__restrict__ data, int L, long long nlines,
                                                          int TO, const double2 *__restrict__ tw, int Lmax,
                                                          long long comp_stride) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *S = reinterpret_cast<double2 *>(smem_raw);
    const long long o0 = (long long)blockIdx.x * TO;
    const int nb = (int)min((long long)TO, nlines - o0);
    const int pT = (nb % 2 == 0) ? nb + 1 : nb;
    double2 *base = data + (size_t)blockIdx.z * comp_stride + (size_t)o0 * L;
    for (int e = threadIdx.x; e < L * nb; e += LNT) {
        int ol = e / L, pos = e - ol * L;
        S[pos * pT + ol] = base[e];
    }
    __syncthreads();
    fft_smem<-1, 4>(S, L, nb, pT, 1, tw, Lmax);
    for (int e = threadIdx.x; e < L * nb; e += LNT) {
        int ol = e / L, pos = e - ol * L;
        base[e] = S[pos * pT + ol];
    }
}

__global__ void k_fold(const double2 *__restrict__ G, int Lx, int Ly, int Lz, int hx, int hy, int hz, double scale,
                       double2 *__restrict__ ahat, float2 *__restrict__ ahat32) {
    const long long n = (long long)hx * hy * hz;
    const size_t Lxyz = (size_t)Lx * Ly * Lz;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        int fky = (int)(e / ((long long)hx * hz));
        int rem = (int)(e - (long long)fky * hx * hz);
        int fkx = rem / hz, fkz = rem - fkx * hz;
        size_t src = ((size_t)fkx * Ly + fky) * Lz + fkz;
#pragma unroll
        for (int l = 0; l < 6; ++l) {
            double2 v = G[(size_t)l * Lxyz + src];
            v.x *= scale;
            v.y *= scale;
            ahat[(size_t)e * 6 + l] = v;
            if (ahat32 != nullptr) ahat32[(size_t)e * 6 + l] = make_float2((float)v.x, (float)v.y);
        }
    }
}

static int pick_tile(int L, int want) {
    int t = want;
    while (t > 1 && fft_max_items(L, t, LNT) > 4) t >>= 1;
    return t;
}

static int lmax_of(int Lx, int Ly, int Lz) {
    auto g = [](int a, int b) { while (b) { int t = a % b; a = b; b = t; } return a; };
    int L = Lx;
    L = L / g(L, Ly) * Ly;
    L = L / g(L, Lz) * Lz;
    return L;
}

tdda_status TensorScratch::init_tables(const double *si, const double *ci, long n) {
    std::vector<double2> h(n > 0 ? n : 1, make_double2(0.0, 0.0));
    for (long q = 0; q < n; ++q) h[q] = make_double2(si[q], ci[q]);
    if (cudaMalloc(&sc, sizeof(double2) * h.size()) != cudaSuccess ||
        cudaMemcpy(sc, h.data(), sizeof(double2) * h.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
        set_error("cannot upload the SiCi tables");
        return TDDA_ERR_OOM;
    }
    ntab = n;
    owns_tables = true;
    return TDDA_OK;
}

tdda_status TensorScratch::reserve(size_t Lxyz, int Lmax) {
    if (G_elems < 6 * Lxyz) {
        cudaFree(G);
        G = nullptr;
        G_elems = 0;
        if (cudaMalloc(&G, sizeof(double2) * 6 * Lxyz) != cudaSuccess) {
            set_error("cannot allocate the padded tensor grid");
            return TDDA_ERR_OOM;
        }
        G_elems = 6 * Lxyz;
    }
    for (auto &t : tw)
        if (t.first == Lmax) return TDDA_OK;
    std::vector<double2> h(Lmax);
    for (int j = 0; j < Lmax; ++j) {
        long double ang = -2.0L * 3.141592653589793238462643383279502884L * (long double)j / Lmax;
        h[j] = make_double2((double)cosl(ang), (double)sinl(ang));
    }
    double2 *d = nullptr;
    if (cudaMalloc(&d, sizeof(double2) * Lmax) != cudaSuccess ||
        cudaMemcpy(d, h.data(), sizeof(double2) * Lmax, cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(d);
        set_error("cannot upload twiddles");
        return TDDA_ERR_OOM;
    }
    tw.emplace_back(Lmax, d);
    return TDDA_OK;
}

const double2 *TensorScratch::twiddles(int Lmax) const {
    for (auto &t : tw)
        if (t.first == Lmax) return t.second;
    return nullptr;
}

size_t TensorScratch::bytes() const {
    return sizeof(double2) * (G_elems + (owns_tables ? (size_t)ntab : 0)) +
           [&] { size_t b = 0; for (auto &t : tw) b += sizeof(double2) * t.first; return b; }();
}

void TensorScratch::release() {
    cudaFree(G);
    if (owns_tables) cudaFree(sc);
    for (auto &t : tw) cudaFree(t.second);
    G = nullptr;
    sc = nullptr;
    tw.clear();
    G_elems = 0;
    ntab = 0;
}

tdda_status build_tensor_async(const LatticeParams &P0, TensorScratch &ws, double2 *ahat, float2 *ahat32,
                               cudaStream_t s, double2 *a0, cudaEvent_t ev_sums, cudaEvent_t ev_done) {
    LatticeParams P = P0;
    const size_t Lxyz = (size_t)P.Lx * P.Ly * P.Lz;
    const int Lmax = lmax_of(P.Lx, P.Ly, P.Lz);
    tdda_status st = ws.reserve(Lxyz, Lmax);
    if (st != TDDA_OK) return st;
    P.sc = ws.sc;
    P.ntab = ws.ntab;
    double2 *G = ws.G;
    const double2 *tw = ws.twiddles(Lmax);
    cudaMemsetAsync(G, 0, sizeof(double2) * 6 * Lxyz, s);
    const long long nent = (long long)P.nx * P.ny * P.nz;
    const long long nimg = (long long)(2 * P.MAXm + 1) * (2 * P.MAXn + 1);
    int lanes = 1;
    while (lanes < 32 && lanes < nimg) lanes <<= 1;
    const long long threads = nent * lanes;
    count_launches(1);
    k_lattice<<<(unsigned)((threads + LNT - 1) / LNT), LNT, 0, s>>>(P, G, lanes);
    if (ev_sums) cudaEventRecord(ev_sums, s);
    if (a0 != nullptr)
        for (int l = 0; l < 6; ++l)
            cudaMemcpyAsync(a0 + l, G + (size_t)l * Lxyz, sizeof(double2), cudaMemcpyDeviceToHost, s);
    // FFT along z (contiguous), y, x; the 6 components ride on grid.z
    {
        int TO = pick_tile(P.Lz, 16);
        long long nlines = (long long)P.Lx * P.Ly;
        int smem = (int)(sizeof(double2) * (size_t)P.Lz * (TO + 1));
        cudaFuncSetAttribute(k_fft_lines_contig, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        dim3 grid((unsigned)((nlines + TO - 1) / TO), 1, 6);
        count_launches(1);
        k_fft_lines_contig<<<grid, LNT, smem, s>>>(G, P.Lz, nlines, TO, tw, Lmax, (long long)Lxyz);
    }
    cudaFuncSetAttribute(k_fft_lines_strided, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    {
        long long inner = P.Lz;
        int TI = pick_tile(P.Ly, (int)std::min<long long>(16, inner));
        int smem = (int)(sizeof(double2) * (size_t)P.Ly * TI);
        dim3 grid((unsigned)((inner + TI - 1) / TI), (unsigned)P.Lx, 6);
        count_launches(1);
        k_fft_lines_strided<<<grid, LNT, smem, s>>>(G, P.Ly, inner, TI, tw, Lmax, (long long)Lxyz);
    }
    {
        long long inner = (long long)P.Ly * P.Lz;
        int TI = pick_tile(P.Lx, (int)std::min<long long>(16, inner));
        int smem = (int)(sizeof(double2) * (size_t)P.Lx * TI);
        dim3 grid((unsigned)((inner + TI - 1) / TI), 1, 6);
        count_launches(1);
        k_fft_lines_strided<<<grid, LNT, smem, s>>>(G, P.Lx, inner, TI, tw, Lmax, (long long)Lxyz);
    }
    const double scale = 1.0 / ((double)P.Lx * P.Ly * P.Lz);
    count_launches(1);
    k_fold<<<1184, 256, 0, s>>>(G, P.Lx, P.Ly, P.Lz, P.Lx / 2 + 1, P.Ly / 2 + 1, P.Lz / 2 + 1, scale, ahat, ahat32);
    if (ev_done) cudaEventRecord(ev_done, s);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) {
        set_error(std::string("tensor build: ") + cudaGetErrorString(err));
        return TDDA_ERR_CUDA;
    }
    return TDDA_OK;
}

tdda_status build_tensor(const LatticeParams &P, const double *si, const double *ci, long ntab,
                         double2 *ahat, float2 *ahat32, cudaStream_t s, double *lattice_ms,
                         double *fft_ms, double2 *a0) {
    TensorScratch ws;
    cudaEvent_t e0, e1, e2;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventCreate(&e2);
    auto cleanup = [&]() {
        ws.release();
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaEventDestroy(e2);
    };
    tdda_status st = ws.init_tables(si, ci, ntab);
    if (st == TDDA_OK) st = ws.reserve((size_t)P.Lx * P.Ly * P.Lz, lmax_of(P.Lx, P.Ly, P.Lz));
    if (st != TDDA_OK) {
        cleanup();
        return st;
    }
    cudaEventRecord(e0, s);
    st = build_tensor_async(P, ws, ahat, ahat32, s, a0, e1, e2);
    cudaError_t err = cudaStreamSynchronize(s);
    if (st == TDDA_OK && err != cudaSuccess) {
        set_error(std::string("tensor build: ") + cudaGetErrorString(err));
        st = TDDA_ERR_CUDA;
    }
    if (st != TDDA_OK) {
        cleanup();
        return st;
    }
    float a = 0, b = 0;
    cudaEventElapsedTime(&a, e0, e1);
    cudaEventElapsedTime(&b, e1, e2);
    if (lattice_ms) *lattice_ms = a;
    if (fft_ms) *fft_ms = b;
    cleanup();
    return TDDA_OK;
}

// Lattice sums on an arbitrary box of integer offsets [lo, lo + n) (no
// parity folding): out[((ix * ny) + iy) * nz + iz][6] for offset lo + (ix, iy, iz).
// Used for fields at observation points outside the dipole box.
__global__ void __launch_bounds__(LNT) k_lattice_box(LatticeParams P, int lox, int loy, int loz, int nbx, int nby,
                                                     int nbz, double2 *__restrict__ out, int lanes) {
    const long long gid = (long long)blockIdx.x * LNT + threadIdx.x;
    const long long entry = gid / lanes;
    const int lane = (int)(gid % lanes);
    const long long nent = (long long)nbx * nby * nbz;
    const bool valid = entry < nent;
    int i = 0, j = 0, k = 0;
    if (valid) {
        i = (int)(entry / ((long long)nby * nbz));
        int rem = (int)(entry - (long long)i * nby * nbz);
        j = rem / nbz;
        k = rem - j * nbz;
    }
    double acc[12];
#pragma unroll
    for (int l = 0; l < 12; ++l) acc[l] = 0.0;
    if (valid) {
        const double x0 = P.d * (lox + i), y0 = P.d * (loy + j), z = P.d * (loz + k);
        const int nn = 2 * P.MAXn + 1;
        const int nimg = (2 * P.MAXm + 1) * nn;
        const double gk = P.gamma * P.K;
        for (int q = lane; q < nimg; q += lanes) {
            const int m = q / nn - P.MAXm;
            const int n = q % nn - P.MAXn;
            const double x = x0 + m * P.Lm, y = y0 + n * P.Ln;
            const double r = sqrt(x * x + y * y + z * z);
            if (r == 0.0) continue;
            const double e = gk * r;
            const double e2 = e * e, e4 = e2 * e2;
            if (e4 > 746.0) continue;
            const double damp = exp(-e4);
            if (P.method == 0) fcd_term(x, y, z, r, damp, P, acc);
            else ldr_term(x, y, z, r, damp, P, acc);
        }
    }
    for (int off = lanes >> 1; off > 0; off >>= 1)
#pragma unroll
        for (int l = 0; l < 12; ++l) acc[l] += __shfl_down_sync(0xffffffffu, acc[l], off, lanes);
    if (!valid || lane != 0) return;
#pragma unroll
    for (int l = 0; l < 6; ++l) out[(size_t)entry * 6 + l] = make_double2(acc[2 * l], acc[2 * l + 1]);
}

tdda_status build_offset_tensor(const LatticeParams &P0, const double *si, const double *ci, long ntab, int lox,
                                int loy, int loz, int nbx, int nby, int nbz, double2 *out, cudaStream_t s) {
    LatticeParams P = P0;
    double2 *sc = nullptr;
    std::vector<double2> h(ntab > 0 ? ntab : 1);
    for (long q = 0; q < ntab; ++q) h[q] = make_double2(si[q], ci[q]);
    if (cudaMalloc(&sc, sizeof(double2) * h.size()) != cudaSuccess) {
        set_error("cannot upload the SiCi tables");
        return TDDA_ERR_OOM;
    }
    cudaMemcpy(sc, h.data(), sizeof(double2) * h.size(), cudaMemcpyHostToDevice);
    P.sc = sc;
    P.ntab = ntab;
    const long long nent = (long long)nbx * nby * nbz;
    const long long nimg = (long long)(2 * P.MAXm + 1) * (2 * P.MAXn + 1);
    int lanes = 1;
    while (lanes < 32 && lanes < nimg) lanes <<= 1;
    const long long threads = nent * lanes;
    count_launches(1);
    k_lattice_box<<<(unsigned)((threads + LNT - 1) / LNT), LNT, 0, s>>>(P, lox, loy, loz, nbx, nby, nbz, out, lanes);
    cudaError_t err = cudaStreamSynchronize(s);
    if (err == cudaSuccess) err = cudaGetLastError();
    cudaFree(sc);
    if (err != cudaSuccess) {
        set_error(std::string("offset tensor: ") + cudaGetErrorString(err));
        return TDDA_ERR_CUDA;
    }
    return TDDA_OK;
}

// Green tensor at arbitrary offsets (for tests of the lattice kernel against
// the oracle's single-term evaluation): out[6] complex per offset.
__global__ void k_green_points(LatticeParams P, const double *__restrict__ xyz, int npts, int m, int n,
                               double2 *__restrict__ out) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npts) return;
    double acc[12];
#pragma unroll
    for (int l = 0; l < 12; ++l) acc[l] = 0.0;
    double x = xyz[3 * q] + m * P.Lm, y = xyz[3 * q + 1] + n * P.Ln, z = xyz[3 * q + 2];
    double r = sqrt(x * x + y * y + z * z);
    if (r != 0.0) {
        double e = P.gamma * P.K * r;
        double damp = exp(-(e * e) * (e * e));
        if (P.method == 0) fcd_term(x, y, z, r, damp, P, acc);
        else ldr_term(x, y, z, r, damp, P, acc);
    }
#pragma unroll
    for (int l = 0; l < 6; ++l) out[(size_t)q * 6 + l] = make_double2(acc[2 * l], acc[2 * l + 1]);
}

}  // namespace tdda
