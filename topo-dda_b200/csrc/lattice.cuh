// Interaction-tensor assembly (lattice sums + FFT) on the device.
#pragma once

#include <utility>
#include <vector>

#include "tdda_common.cuh"
#include "../../include/tdda.h"

namespace tdda {

struct LatticeParams {
    int nx, ny, nz;       // box (octant extents)
    int Lx, Ly, Lz;       // padded grid
    double d;             // dipole spacing
    double K;             // 2 pi nback / lam
    double Kf;            // pi / d
    double Lm, Ln;        // periods as lengths (d included)
    int MAXm, MAXn;
    int method;           // 0 FCD, 1 LDR
    double gamma;         // damping exp(-(gamma K r)^4), 0.01 in the reference
    double delta;         // SiCi table spacing
    const double2 *sc;    // device (si, ci) pairs
    long ntab;
};

// Device scratch of repeated tensor builds: SiCi table, padded grid and
// twiddle tables, kept between builds so that a build allocates nothing once
// its sizes have been seen.  The table may be shared (owns_tables = false).
struct TensorScratch {
    double2 *sc = nullptr;
    long ntab = 0;
    bool owns_tables = false;
    double2 *G = nullptr;
    size_t G_elems = 0;
    std::vector<std::pair<int, double2 *>> tw;  // (Lmax, table)
    tdda_status init_tables(const double *si, const double *ci, long ntab);
    tdda_status reserve(size_t Lxyz, int Lmax);
    const double2 *twiddles(int Lmax) const;
    size_t bytes() const;
    void release();
};

// Enqueues one tensor build on stream s without synchronising: lattice sums
// into ws.G, FP64 FFT, fold into ahat (and ahat32).  a0 (pinned host
// double2[6], optional) receives the zero-offset entry once s reaches it;
// ev_sums / ev_done (optional) are recorded after the sums and at the end.
tdda_status build_tensor_async(const LatticeParams &P, TensorScratch &ws, double2 *ahat, float2 *ahat32,
                               cudaStream_t s, double2 *a0, cudaEvent_t ev_sums, cudaEvent_t ev_done);

// Lattice sums -> padded grid -> FP64 FFT -> folded spectral tensor
// [hy][hx][hz][6] (scaled by 1/(Lx Ly Lz)); ahat32 optional complex64 copy.
// a0 (optional, host double2[6]) receives the zero-offset tensor entry (the
// sum over periodic images seen by every dipole itself).
tdda_status build_tensor(const LatticeParams &P, const double *si, const double *ci, long ntab,
                         double2 *ahat, float2 *ahat32, cudaStream_t s, double *lattice_ms,
                         double *fft_ms, double2 *a0);

// Lattice sums (same periodic images and damping) for every integer offset
// lo + (i, j, k), i < nbx, j < nby, k < nbz: out[((i*nby + j)*nbz + k)*6 + l].
tdda_status build_offset_tensor(const LatticeParams &P, const double *si, const double *ci, long ntab, int lox,
                                int loy, int loz, int nbx, int nby, int nbz, double2 *out, cudaStream_t s);

}  // namespace tdda
