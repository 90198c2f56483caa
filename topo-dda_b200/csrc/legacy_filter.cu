// The reference's legacy design filter on the device (see legacy_filter.cuh).
#include <algorithm>
#include <cmath>
#include <map>
#include <tuple>

#include "legacy_filter.cuh"

namespace tdda {

bool legacy_beta(const std::string &type, int it, int max_it, double bmin, double bmax, double *beta) {
    const double x = (double)it, xm = (double)max_it;
    if (type == "exp") {
        *beta = x <= 300 ? bmin + (bmax - bmin) * (std::pow(100.0, x / xm) - 1) / (100 - 1) : 0.5;
    } else if (type == "piecewise") {
        if (x <= 0.5 * xm) *beta = bmin;
        else if (x <= 0.7 * xm) *beta = bmin + (bmax - bmin) / 5;
        else if (x <= 0.8 * xm) *beta = bmin + (bmax - bmin) / 2.5;
        else *beta = bmax;
    } else if (type == "linear") {
        *beta = bmin + (bmax - bmin) * x / xm;
    } else {
        return false;
    }
    return true;
}

// SmoothDensity (src/FilterOption.cpp:48-62); inputs outside [0, 1] are
// flagged (the reference throws)
__device__ double lf_smooth(double x, double beta, double ita, int *bad) {
    if (x >= 0.0 && x <= ita) return ita * (exp(-beta * (1 - x / ita)) - (1 - x / ita) * exp(-beta));
    if (x > ita && x <= 1.0)
        return (1 - ita) * (1 - exp(-beta * (x - ita) / (1 - ita)) + (x - ita) / (1 - ita) * exp(-beta)) + ita;
    atomicExch(bad, 1);
    return 0.0;
}

// PtoFderivative (src/DDAModel.cpp:340-352), as the reference writes it
__device__ double lf_smooth_d(double x, double beta, double ita, int *bad) {
    if (x >= 0.0 && x <= ita) return beta * exp(-beta * (1 - x / ita)) + exp(-beta);
    if (x > ita && x <= 1.0) return beta * exp(-beta * (x - ita) / (1 - ita)) + exp(-beta);
    atomicExch(bad, 1);
    return 0.0;
}

// raw = clamp(raw + step, 0, 1)   (src/DDAModel.cpp:789-797)
__global__ void k_lf_step(int nf, const double *__restrict__ step, double *__restrict__ raw) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nf; i += gridDim.x * blockDim.x) {
        double v = raw[i] + step[i];
        if (v >= 1) v = 1;
        if (v <= 0) v = 0;
        raw[i] = v;
    }
}

// filtered_i = sum_k w_k raw[col_k] / sum_k w_k in list order; physical_i =
// SmoothDensity(filtered_i)   (src/DDAModel.cpp:803-815)
__global__ void k_lf_filter(int nf, const int *__restrict__ off, const int *__restrict__ col,
                            const double *__restrict__ w, const double *__restrict__ raw, double beta, double ita,
                            double *__restrict__ filt, double *__restrict__ phys, int *bad) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nf; i += gridDim.x * blockDim.x) {
        double num = 0.0, den = 0.0;
        for (int k = off[i]; k < off[i + 1]; ++k) {
            num = __dadd_rn(num, __dmul_rn(w[k], raw[col[k]]));
            den = __dadd_rn(den, w[k]);
        }
        const double f = num / den;
        filt[i] = f;
        phys[i] = lf_smooth(f, beta, ita, bad);
    }
}

// out_j = (sum over the rows i that hold j of w / rowsum_i, in row order) *
// PtoFderivative(filtered_j) * grad_j   (src/DDAModel.cpp:365-393): each
// thread gathers its column from the transposed lists, so the sum keeps the
// reference's order
__global__ void k_lf_grad(int nf, const int *__restrict__ toff, const int *__restrict__ trow,
                          const double *__restrict__ tw, const double *__restrict__ rowsum,
                          const double *__restrict__ filt, const double *__restrict__ grad, double beta, double ita,
                          double *__restrict__ out, int *bad) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nf; j += gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int k = toff[j]; k < toff[j + 1]; ++k) acc = __dadd_rn(acc, tw[k] / rowsum[trow[k]]);
        out[j] = __dmul_rn(__dmul_rn(acc, lf_smooth_d(filt[j], beta, ita, bad)), grad[j]);
    }
}

tdda_status LegacyFilter::build(const LegacyFilterConfig &cfg, const std::vector<int32_t> &geo,
                                const std::vector<int> &p2g_off, const std::vector<int> &p2g_idx,
                                const std::vector<double> &parameters) {
    release();
    cfg_ = cfg;
    double b0;
    if (!legacy_beta(cfg.beta_type, 0, 1, cfg.beta_min, cfg.beta_max, &b0)) {
        set_error("betaType must be exp, piecewise or linear (src/FilterOption.cpp:26-44)");
        return TDDA_ERR_BAD_ARG;
    }
    if (!(cfg.rfilter > 0.0)) { set_error("the legacy filter needs a positive radius"); return TDDA_ERR_BAD_ARG; }
    if (!(cfg.ita > 0.0 && cfg.ita < 1.0)) { set_error("the legacy filter needs 0 < ita < 1"); return TDDA_ERR_BAD_ARG; }
    const int nf = (int)p2g_off.size() - 1;
    const int N = (int)geo.size() / 3;
    // dipole at (x, y, z); parameter of each dipole and its rank in that parameter's list
    std::map<std::tuple<int, int, int>, int> at;
    for (int i = 0; i < N; ++i) at[{geo[3 * i], geo[3 * i + 1], geo[3 * i + 2]}] = i;
    std::vector<int> par(N, -1), rank(N, 0);
    for (int j = 0; j < nf; ++j)
        for (int k = p2g_off[j]; k < p2g_off[j + 1]; ++k) {
            par[p2g_idx[k]] = j;
            rank[p2g_idx[k]] = k - p2g_off[j];
        }
    // image shifts in the reference's order (src/DDAModel.cpp:616-704)
    std::vector<std::pair<int, int>> sh = {{0, 0}};
    if (cfg.periodic) {
        const int Lm = cfg.Lm, Ln = cfg.Ln;
        sh.insert(sh.end(), {{0, -Ln}, {-Lm, -Ln}, {-Lm, 0}, {-Lm, Ln}, {0, Ln}, {Lm, Ln}, {Lm, 0}, {Lm, -Ln}});
    }
    const double r = cfg.rfilter, r2 = r * r - 0.01;
    const int ri = (int)std::ceil(r) + 1;
    std::vector<int> off(1, 0), col;
    std::vector<double> w;
    for (int i = 0; i < nf; ++i) {
        const int o = p2g_idx[p2g_off[i]];
        const int xo = geo[3 * o], yo = geo[3 * o + 1], zo = geo[3 * o + 2];
        // (parameter j, rank in j, shift index, weight): the reference visits
        // the parameters j, then the dipoles of j, then the shifts
        std::vector<std::tuple<int, int, int, double>> hits;
        for (int si = 0; si < (int)sh.size(); ++si)
            for (int x = xo - ri; x <= xo + ri; ++x)
                for (int y = yo - ri; y <= yo + ri; ++y) {
                    const double d2 = double(x - xo) * double(x - xo) + double(y - yo) * double(y - yo);
                    if (!(d2 <= r2)) continue;
                    auto it = at.find({x - sh[si].first, y - sh[si].second, zo});
                    if (it == at.end() || par[it->second] < 0) continue;
                    hits.emplace_back(par[it->second], rank[it->second], si, r - std::sqrt(d2));
                }
        std::sort(hits.begin(), hits.end(), [](const auto &a, const auto &b) {
            return std::make_tuple(std::get<0>(a), std::get<1>(a), std::get<2>(a)) <
                   std::make_tuple(std::get<0>(b), std::get<1>(b), std::get<2>(b));
        });
        for (auto &hh : hits) {
            col.push_back(std::get<0>(hh));
            w.push_back(std::get<3>(hh));
        }
        off.push_back((int)col.size());
        if (off[i + 1] == off[i]) {
            set_error("legacy filter: a parameter has no weight");
            return TDDA_ERR_BAD_ARG;
        }
    }
    // transposed lists (rows in order within each column) and row sums
    const size_t nnz = col.size();
    std::vector<double> rowsum(nf, 0.0);
    for (int i = 0; i < nf; ++i)
        for (int k = off[i]; k < off[i + 1]; ++k) rowsum[i] += w[k];
    std::vector<int> toff(nf + 1, 0), trow(nnz);
    std::vector<double> tw(nnz);
    for (size_t k = 0; k < nnz; ++k) toff[col[k] + 1]++;
    for (int j = 0; j < nf; ++j) toff[j + 1] += toff[j];
    std::vector<int> fill(toff.begin(), toff.end() - 1);
    for (int i = 0; i < nf; ++i)
        for (int k = off[i]; k < off[i + 1]; ++k) {
            const int p = fill[col[k]]++;
            trow[p] = i;
            tw[p] = w[k];
        }
    std::vector<int> ib;
    ib.insert(ib.end(), off.begin(), off.end());
    ib.insert(ib.end(), col.begin(), col.end());
    ib.insert(ib.end(), toff.begin(), toff.end());
    ib.insert(ib.end(), trow.begin(), trow.end());
    std::vector<double> db;
    db.insert(db.end(), w.begin(), w.end());
    db.insert(db.end(), tw.begin(), tw.end());
    db.insert(db.end(), parameters.begin(), parameters.end());   // raw
    db.insert(db.end(), parameters.begin(), parameters.end());   // filtered
    db.insert(db.end(), (size_t)nf, 0.0);                        // in (step or gradient)
    db.insert(db.end(), rowsum.begin(), rowsum.end());
    db.insert(db.end(), (size_t)nf + 1, 0.0);                    // out, flag
    TDDA_CUDA_TRY(cudaMalloc(&d_int_, sizeof(int) * ib.size()));
    TDDA_CUDA_TRY(cudaMalloc(&d_dbl_, sizeof(double) * db.size()));
    TDDA_CUDA_TRY(cudaMemcpy(d_int_, ib.data(), sizeof(int) * ib.size(), cudaMemcpyHostToDevice));
    TDDA_CUDA_TRY(cudaMemcpy(d_dbl_, db.data(), sizeof(double) * db.size(), cudaMemcpyHostToDevice));
    nf_ = nf;
    nnz_ = nnz;
    beta_ = cfg.beta_min;
    return TDDA_OK;
}

double LegacyFilter::schedule(int it, int max_it) const {
    double b = beta_;
    legacy_beta(cfg_.beta_type, it, max_it, cfg_.beta_min, cfg_.beta_max, &b);
    return b;
}

static unsigned lf_blocks(int n) { return (unsigned)std::max(1, std::min((n + 255) / 256, 148 * 8)); }

tdda_status LegacyFilter::update(const double *step, int it, int max_it, cudaStream_t s,
                                 std::vector<double> &physical) {
    if (!active()) { set_error("the model was created without the legacy filter (useFilter)"); return TDDA_ERR_STATE; }
    beta_ = schedule(it, max_it);
    const int *off = d_int_, *col = d_int_ + nf_ + 1;
    const double *w = d_dbl_;
    double *raw = d_dbl_ + 2 * nnz_, *filt = raw + nf_, *in = filt + nf_, *out = in + 2 * (size_t)nf_;
    int *bad = reinterpret_cast<int *>(out + nf_);
    TDDA_CUDA_TRY(cudaMemsetAsync(bad, 0, sizeof(int), s));
    TDDA_CUDA_TRY(cudaMemcpyAsync(in, step, sizeof(double) * nf_, cudaMemcpyHostToDevice, s));
    count_launches(2);
    k_lf_step<<<lf_blocks(nf_), 256, 0, s>>>(nf_, in, raw);
    k_lf_filter<<<lf_blocks(nf_), 256, 0, s>>>(nf_, off, col, w, raw, beta_, cfg_.ita, filt, out, bad);
    TDDA_CUDA_TRY(cudaGetLastError());
    physical.resize(nf_);
    int hbad = 0;
    TDDA_CUDA_TRY(cudaMemcpyAsync(physical.data(), out, sizeof(double) * nf_, cudaMemcpyDeviceToHost, s));
    TDDA_CUDA_TRY(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    TDDA_CUDA_TRY(cudaStreamSynchronize(s));
    if (hbad) { set_error("legacy filter: filtered density outside [0, 1]"); return TDDA_ERR_BAD_ARG; }
    return TDDA_OK;
}

tdda_status LegacyFilter::gradients(const double *grad, int it, int max_it, cudaStream_t s, double *out_host) {
    if (!active()) { set_error("the model was created without the legacy filter (useFilter)"); return TDDA_ERR_STATE; }
    beta_ = schedule(it, max_it);
    const int *toff = d_int_ + (nf_ + 1) + nnz_, *trow = toff + (nf_ + 1);
    const double *tw = d_dbl_ + nnz_;
    double *raw = d_dbl_ + 2 * nnz_, *filt = raw + nf_, *in = filt + nf_, *rowsum = in + nf_, *out = rowsum + nf_;
    int *bad = reinterpret_cast<int *>(out + nf_);
    TDDA_CUDA_TRY(cudaMemsetAsync(bad, 0, sizeof(int), s));
    TDDA_CUDA_TRY(cudaMemcpyAsync(in, grad, sizeof(double) * nf_, cudaMemcpyHostToDevice, s));
    count_launches(1);
    k_lf_grad<<<lf_blocks(nf_), 256, 0, s>>>(nf_, toff, trow, tw, rowsum, filt, in, beta_, cfg_.ita, out, bad);
    TDDA_CUDA_TRY(cudaGetLastError());
    int hbad = 0;
    TDDA_CUDA_TRY(cudaMemcpyAsync(out_host, out, sizeof(double) * nf_, cudaMemcpyDeviceToHost, s));
    TDDA_CUDA_TRY(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
    TDDA_CUDA_TRY(cudaStreamSynchronize(s));
    if (hbad) { set_error("legacy filter: filtered density outside [0, 1]"); return TDDA_ERR_BAD_ARG; }
    return TDDA_OK;
}

tdda_status LegacyFilter::state(double *raw_h, double *filt_h, cudaStream_t s) const {
    if (!active()) { set_error("the model was created without the legacy filter (useFilter)"); return TDDA_ERR_STATE; }
    const double *raw = d_dbl_ + 2 * nnz_, *filt = raw + nf_;
    if (raw_h) TDDA_CUDA_TRY(cudaMemcpyAsync(raw_h, raw, sizeof(double) * nf_, cudaMemcpyDeviceToHost, s));
    if (filt_h) TDDA_CUDA_TRY(cudaMemcpyAsync(filt_h, filt, sizeof(double) * nf_, cudaMemcpyDeviceToHost, s));
    TDDA_CUDA_TRY(cudaStreamSynchronize(s));
    return TDDA_OK;
}

void LegacyFilter::release() {
    cudaFree(d_int_);
    cudaFree(d_dbl_);
    d_int_ = nullptr;
    d_dbl_ = nullptr;
    nf_ = 0;
    nnz_ = 0;
}

}  // namespace tdda
