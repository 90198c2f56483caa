// Interaction-tensor assembly (lattice sums + FFT) on the device.
#pragma once

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
