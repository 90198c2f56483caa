// The reference's legacy design filter: an in-plane cone filter over the free
// parameters followed by an exponential (smoothed Heaviside) projection, with
// the reference's gradient rule (src/DDAModel.cpp:340-396,580-838,
// src/FilterOption.cpp:23-62).  In the reference it is reachable only from
// C++ (DDAModel::UpdateStr, gradients_filtered); here it is a device-side
// component of the model behind the tdda_filter_* entry points.
#pragma once

#include <string>
#include <vector>

#include "tdda_common.cuh"
#include "../../include/tdda.h"

namespace tdda {

struct LegacyFilterConfig {
    double beta_min = 0, beta_max = 0, ita = 0.5;
    std::string beta_type;       // "exp", "piecewise" or "linear"
    double rfilter = 0;          // radius of the first entry of the radius list
    bool periodic = false;
    int Lm = 0, Ln = 0;          // periods in grid units (the images of the periodic filter)
};

class LegacyFilter {
public:
    // Weights of every free parameter (src/DDAModel.cpp:580-712): geometry is
    // int[3N] (x, y, z per dipole), p2g_off/p2g_idx the parameter -> dipoles
    // CSR, parameters the initial values (raw = filtered = parameters).
    tdda_status build(const LegacyFilterConfig &cfg, const std::vector<int32_t> &geometry,
                      const std::vector<int> &p2g_off, const std::vector<int> &p2g_idx,
                      const std::vector<double> &parameters);
    // UpdateStr's filter branch: raw += step (clamped to [0, 1]), filtered =
    // weighted mean, physical = SmoothDensity(filtered) at the scheduled beta.
    tdda_status update(const double *step_host, int it, int max_it, cudaStream_t s, std::vector<double> &physical);
    // gradients_filtered: out_i = (sum over the filters parameter i enters of
    // its normalised weight) * projection derivative at filtered_i * grad_i.
    tdda_status gradients(const double *grad_host, int it, int max_it, cudaStream_t s, double *out_host);
    tdda_status state(double *raw, double *filtered, cudaStream_t s) const;
    double beta() const { return beta_; }
    int nfpara() const { return nf_; }
    bool active() const { return nf_ > 0; }
    void release();
    ~LegacyFilter() { release(); }

private:
    LegacyFilterConfig cfg_;
    int nf_ = 0;
    size_t nnz_ = 0;
    double beta_ = 0;
    int *d_int_ = nullptr;       // off [nf+1], col [nnz], toff [nf+1], trow [nnz]
    double *d_dbl_ = nullptr;    // w [nnz], tw [nnz], raw, filtered, in, rowsum, out, flag [nf each]
    double schedule(int it, int max_it) const;
};

// FilterOption::update_beta's schedules (src/Tools.cpp:473-516); false for an
// unknown schedule name.
bool legacy_beta(const std::string &type, int it, int max_it, double bmin, double bmax, double *beta);

}  // namespace tdda
