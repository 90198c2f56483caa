// Serving engine of libtdda (include/tdda.h, tdda_server_*): a request loop
// with continuous batching on one GPU.
//
// The reference solves one structure per DDAModel and has no request loop;
// each request here is the solve of src/DDAModel.cpp:874-885 for a full box
// (incident field :312-316, polarisability src/Tools.cpp:353-366 with the
// material rescale of src/AProductCore.cpp:25-33), one right-hand side per
// incident polarisation, solved to a true complex128 residual by iterative
// refinement around complex64 (or complex128) BiCGSTAB.
//
// Structure:
//   * worker threads, each with a CUDA stream, a tensor-build scratch and one
//     solve workspace per grid shape it has served (sized for max_rhs);
//   * one FIFO queue; an idle worker admits the first request whose device
//     memory (tensor if not resident + its workspace if not yet allocated) fits
//     the budget, evicting idle tensors (LRU) and idle workspaces of other
//     shapes when short, then merges queued requests of the same grid (and
//     precision, tolerance, iteration limit) into the batch, up to the most
//     right-hand sides the operator takes for that grid.  Each right-hand side
//     keeps its own tensor (its wavelength and period); requests with equal
//     tensor keys share one;
//   * a tensor is built once per key on the admitting worker's stream; other
//     workers needing it wait until it is ready and then share it read-only.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "lattice.cuh"
#include "operator.cuh"
#include "physics.cuh"
#include "refine.cuh"

using namespace tdda;
using Clock = std::chrono::steady_clock;

namespace {

constexpr int kMaxRhs = 16;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

// identity of an interaction tensor: everything the lattice sums depend on
struct TensorKey {
    int nx, ny, nz, method, MAXm, MAXn;
    double d, lam, nback, Lm, Ln;
    bool operator<(const TensorKey &o) const {
        return std::tie(nx, ny, nz, method, MAXm, MAXn, d, lam, nback, Lm, Ln) <
               std::tie(o.nx, o.ny, o.nz, o.method, o.MAXm, o.MAXn, o.d, o.lam, o.nback, o.Lm, o.Ln);
    }
    bool operator==(const TensorKey &o) const { return !(*this < o) && !(o < *this); }
};

struct Tensor {
    TensorKey key{};
    double2 *ahat64 = nullptr;
    float2 *ahat32 = nullptr;
    double2 a0{};           // mean diagonal of the zero-offset entry
    size_t bytes = 0;
    int users = 0;
    bool ready = false;
    bool failed = false;
};

size_t tensor_bytes(int nx, int ny, int nz) {
    const long long hx = next_fft_len(2 * nx - 1) / 2 + 1, hy = next_fft_len(2 * ny - 1) / 2 + 1,
                    hz = next_fft_len(2 * nz - 1) / 2 + 1;
    return (size_t)hx * hy * hz * 6 * (sizeof(double2) + sizeof(float2));
}

// per-right-hand-side inputs of the setup kernel
struct RhsParams {
    AlphaParams A;
    double2 a0;
    double kd;        // K d
    double nK[3];
    double e[3];      // E0 n_E0
    int job;          // index of the density field
};

struct SetupArgs {
    int nrhs, nx, ny, nz;
    RhsParams r[kMaxRhs];
};

// per right-hand side k and cell: eps, 1/alpha, Jacobi scale, incident field
__global__ void k_serve_setup(SetupArgs a, const double *__restrict__ rho, double2 *__restrict__ al64,
                              float2 *__restrict__ al32, double2 *__restrict__ sc64, float2 *__restrict__ sc32,
                              float2 *__restrict__ alS32, double2 *__restrict__ alS64,
                              double2 *__restrict__ diel, double2 *__restrict__ B) {
    const long long nbox = (long long)a.nx * a.ny * a.nz;
    const long long tot = nbox * a.nrhs;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(e / nbox);
        const long long cell = e - (long long)k * nbox;
        const int z = (int)(cell % a.nz);
        const int y = (int)((cell / a.nz) % a.ny);
        const int x = (int)(cell / ((long long)a.nz * a.ny));
        const RhsParams &p = a.r[k];
        const long long dip = x + (long long)a.nx * (y + (long long)a.ny * z);
        const double2 eps = diel_of(rho[(size_t)p.job * nbox + dip], p.A);
        const double2 al = inv_alpha(eps, p.A);
        const double2 s = jacobi_scale(al, p.a0);
        const double2 as = cmul_d(cmul_d(s, s), al);
        al64[e] = al;
        al32[e] = make_float2((float)al.x, (float)al.y);
        sc64[e] = s;
        sc32[e] = make_float2((float)s.x, (float)s.y);
        alS32[e] = make_float2((float)as.x, (float)as.y);
        if (alS64 != nullptr) alS64[e] = as;
        diel[e] = eps;
        double sn, cs;
        sincos(p.kd * (p.nK[0] * x + p.nK[1] * y + p.nK[2] * z), &sn, &cs);
        for (int c = 0; c < 3; ++c)
            B[((size_t)k * 3 + c) * nbox + cell] = make_double2(p.e[c] * cs, p.e[c] * sn);
    }
}

// X [k][c][cell] -> P (dipole order, interleaved) and E_int = al P / ((2 + eps) / 3)
__global__ void k_serve_out(int nrhs, int nx, int ny, int nz, const double2 *__restrict__ X,
                            const double2 *__restrict__ al, const double2 *__restrict__ diel,
                            double2 *__restrict__ P, double2 *__restrict__ E) {
    const long long nbox = (long long)nx * ny * nz;
    const long long tot = nbox * 3 * nrhs;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(e / (3 * nbox));
        const long long rem = e - (long long)k * 3 * nbox;
        const long long dip = rem / 3;
        const int c = (int)(rem - dip * 3);
        const int x = (int)(dip % nx);
        const int y = (int)((dip / nx) % ny);
        const int z = (int)(dip / ((long long)nx * ny));
        const long long cell = ((long long)x * ny + y) * nz + z;
        const double2 p = X[((size_t)k * 3 + c) * nbox + cell];
        const double2 ev = diel[(size_t)k * nbox + cell];
        const double2 lf = make_double2((2.0 + ev.x) / 3.0, ev.y / 3.0);
        P[e] = p;
        E[e] = cdiv(cmul_d(al[(size_t)k * nbox + cell], p), lf);
    }
}

unsigned blocks_for(long long n) {
    long long b = (n + 255) / 256;
    return (unsigned)std::max<long long>(1, std::min<long long>(b, 148 * 16));
}

// solve workspace of one worker for one grid shape, sized for `cap` right-hand sides
struct Workspace {
    int nx = 0, ny = 0, nz = 0, cap = 0;
    long long nbox = 0;
    ConvOperator<double2> op64;
    ConvOperator<float2> op32;
    Krylov<float2> kv32;
    Krylov<double2> kv64;  // complex128 requests only (has64)
    bool has64 = false;
    double2 *B = nullptr, *X = nullptr, *Rm = nullptr, *al64 = nullptr, *sc64 = nullptr, *diel = nullptr;
    double2 *alS64 = nullptr, *R64 = nullptr, *D64 = nullptr;
    float2 *al32 = nullptr, *sc32 = nullptr, *alS32 = nullptr, *R32 = nullptr, *D32 = nullptr;
    SolverState *st_res = nullptr, *st_res_host = nullptr;
    double *d_part = nullptr, *h_part = nullptr;
    double *d_rho = nullptr, *h_rho = nullptr;
    double2 *d_out = nullptr, *h_out = nullptr;  // P then E, [cap][3 nbox] each
    const double2 **h_tab64 = nullptr, **d_tab64 = nullptr;  // tensor of each right-hand side
    const float2 **h_tab32 = nullptr, **d_tab32 = nullptr;
    bool want64 = false;  // complex128 part reserved, allocated at first use
    size_t bytes = 0;

    static size_t bytes_for(int nx, int ny, int nz, int cap) {
        const size_t nbox = (size_t)nx * ny * nz, v = 3 * nbox * cap;
        size_t b = conv_workspace_bytes(nx, ny, nz, cap, 16) + conv_workspace_bytes(nx, ny, nz, cap, 8);
        b += 6 * v * sizeof(float2) + cap * sizeof(SolverState);          // kv32
        b += 3 * v * sizeof(double2);                                      // B, X, Rm
        b += 3 * nbox * cap * sizeof(double2);                             // al64, sc64, diel
        b += 3 * nbox * cap * sizeof(float2);                              // al32, sc32, alS32
        b += 2 * v * sizeof(float2);                                       // R32, D32
        b += cap * sizeof(SolverState) + 1024 * sizeof(double);            // st_res, d_part
        b += nbox * cap * sizeof(double);                                  // d_rho
        b += 2 * v * sizeof(double2);                                      // d_out
        // the worker's tensor-build grid (6 padded components, complex128)
        b += 6 * sizeof(double2) * (size_t)next_fft_len(2 * nx - 1) * next_fft_len(2 * ny - 1) *
             next_fft_len(2 * nz - 1);
        return b;
    }
    static size_t bytes64_for(int nx, int ny, int nz, int cap) {
        const size_t nbox = (size_t)nx * ny * nz, v = 3 * nbox * cap;
        return 6 * v * sizeof(double2) + cap * sizeof(SolverState) + nbox * cap * sizeof(double2) +
               2 * v * sizeof(double2);
    }

    tdda_status init(int nx_, int ny_, int nz_, int cap_) {
        nx = nx_; ny = ny_; nz = nz_; cap = cap_;
        nbox = (long long)nx * ny * nz;
        tdda_status st = op64.init(nx, ny, nz, cap);
        if (st != TDDA_OK) return st;
        st = op32.init(nx, ny, nz, cap);
        if (st != TDDA_OK) return st;
        st = kv32.init(3 * nbox, cap);
        if (st != TDDA_OK) return st;
        const size_t v = 3 * (size_t)nbox * cap, d = (size_t)nbox * cap;
        double2 **b64[] = {&B, &X, &Rm};
        for (auto p : b64) TDDA_CUDA_TRY(cudaMalloc(p, sizeof(double2) * v));
        double2 **d64[] = {&al64, &sc64, &diel};
        for (auto p : d64) TDDA_CUDA_TRY(cudaMalloc(p, sizeof(double2) * d));
        float2 **d32[] = {&al32, &sc32, &alS32};
        for (auto p : d32) TDDA_CUDA_TRY(cudaMalloc(p, sizeof(float2) * d));
        TDDA_CUDA_TRY(cudaMalloc(&R32, sizeof(float2) * v));
        TDDA_CUDA_TRY(cudaMalloc(&D32, sizeof(float2) * v));
        TDDA_CUDA_TRY(cudaMalloc(&st_res, sizeof(SolverState) * cap));
        TDDA_CUDA_TRY(cudaMallocHost(&st_res_host, sizeof(SolverState) * cap));
        TDDA_CUDA_TRY(cudaMalloc(&d_part, sizeof(double) * 1024));
        TDDA_CUDA_TRY(cudaMallocHost(&h_part, sizeof(double) * 1024));
        TDDA_CUDA_TRY(cudaMalloc(&d_rho, sizeof(double) * d));
        TDDA_CUDA_TRY(cudaMallocHost(&h_rho, sizeof(double) * d));
        TDDA_CUDA_TRY(cudaMalloc(&d_out, sizeof(double2) * 2 * v));
        TDDA_CUDA_TRY(cudaMallocHost(&h_out, sizeof(double2) * 2 * v));
        TDDA_CUDA_TRY(cudaMalloc(&d_tab64, sizeof(void *) * cap));
        TDDA_CUDA_TRY(cudaMalloc(&d_tab32, sizeof(void *) * cap));
        TDDA_CUDA_TRY(cudaMallocHost(&h_tab64, sizeof(void *) * cap));
        TDDA_CUDA_TRY(cudaMallocHost(&h_tab32, sizeof(void *) * cap));
        bytes = bytes_for(nx, ny, nz, cap);
        return TDDA_OK;
    }

    tdda_status init64() {
        if (has64) return TDDA_OK;
        tdda_status st = kv64.init(3 * nbox, cap);
        if (st != TDDA_OK) return st;
        const size_t v = 3 * (size_t)nbox * cap;
        TDDA_CUDA_TRY(cudaMalloc(&alS64, sizeof(double2) * (size_t)nbox * cap));
        TDDA_CUDA_TRY(cudaMalloc(&R64, sizeof(double2) * v));
        TDDA_CUDA_TRY(cudaMalloc(&D64, sizeof(double2) * v));
        has64 = true;
        bytes += bytes64_for(nx, ny, nz, cap);
        return TDDA_OK;
    }

    ~Workspace() {
        op64.ahat = nullptr;  // tensors belong to the cache
        op32.ahat = nullptr;
        op64.release();
        op32.release();
        kv32.release();
        kv64.release();
        void *dev[] = {B, X, Rm, al64, sc64, diel, alS64, R64, D64, al32, sc32, alS32, R32, D32, st_res, d_part,
                       d_rho, d_out, (void *)d_tab64, (void *)d_tab32};
        for (void *p : dev) cudaFree(p);
        void *host[] = {st_res_host, h_part, h_rho, h_out, (void *)h_tab64, (void *)h_tab32};
        for (void *p : host) cudaFreeHost(p);
    }
};

struct Job {
    long long ticket = 0;
    tdda_request req{};
    std::vector<double> rho;
    TensorKey key{};
    Clock::time_point t_submit, t_admit, t_done;
    tdda_request_result res{};
    std::string error;
    int rhs_cap = 1;  // most right-hand sides a batch of this grid may hold
    bool done = false;
    std::shared_ptr<Tensor> tensor;  // held from admission to the end of its batch
    bool hit = false;
};

using Shape = std::tuple<int, int, int>;

Shape shape_of(const tdda_request &r) { return Shape{r.num_x, r.num_y, r.num_z}; }

struct Worker {
    int id = 0;
    cudaStream_t stream = nullptr;
    TensorScratch scratch;
    std::map<Shape, std::unique_ptr<Workspace>> ws;
    double2 *a0_host = nullptr;  // pinned [6]
    std::thread th;
};

}  // namespace

struct tdda_server {
    tdda_server_config cfg{};
    int device = 0;
    double2 *d_sici = nullptr;
    long ntab = 0;
    double delta = 0.1;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<Job>> queue;
    std::unordered_map<long long, std::shared_ptr<Job>> jobs;
    std::list<std::shared_ptr<Tensor>> cache;  // least recently used first
    std::vector<std::unique_ptr<Worker>> workers;
    long long next_ticket = 1;
    size_t in_use = 0;
    int inflight = 0;
    bool stop = false;
    tdda_server_stats stats{};

    using FreeList = std::vector<std::unique_ptr<Workspace>>;
    using EvictList = std::vector<std::shared_ptr<Tensor>>;

    std::shared_ptr<Tensor> find(const TensorKey &k) {
        for (auto &t : cache)
            if (t->key == k) return t;
        return nullptr;
    }
    long long need_of(Worker *w, const Job &j, bool with_ws);
    bool make_room(Worker *w, size_t need, const Shape &keep, FreeList &to_free, EvictList &evicted);
    void take(Worker *w, Job &j, bool with_ws, size_t need);
    void run(Worker *w);
    void run_batch(Worker *w, std::vector<std::shared_ptr<Job>> &batch);
};

// Under the lock: device bytes job j still needs on worker w -- its tensor if
// not resident, and (with_ws) the worker's workspace for its grid if missing
// or without the complex128 part a complex128 request needs.  -1: its tensor
// is being built by another worker right now.
long long tdda_server::need_of(Worker *w, const Job &j, bool with_ws) {
    const tdda_request &r = j.req;
    auto t = find(j.key);
    if (t && (!t->ready || t->failed)) return -1;
    size_t need = t ? 0 : tensor_bytes(r.num_x, r.num_y, r.num_z);
    if (with_ws) {
        auto it = w->ws.find(shape_of(r));
        const bool missing = it == w->ws.end();
        if (missing) need += Workspace::bytes_for(r.num_x, r.num_y, r.num_z, cfg.max_rhs);
        if (r.precision == TDDA_PREC_C128 && (missing || (!it->second->has64 && !it->second->want64)))
            need += Workspace::bytes64_for(r.num_x, r.num_y, r.num_z, cfg.max_rhs);
    }
    return (long long)need;
}

// Under the lock: evict until `need` more bytes fit the budget -- idle
// tensors least recently used first, then this worker's workspaces of other
// grids, then, with no batch in flight, other workers' workspaces.
bool tdda_server::make_room(Worker *w, size_t need, const Shape &keep, FreeList &to_free, EvictList &evicted) {
    const size_t budget = (size_t)cfg.hbm_budget_bytes;
    for (auto c = cache.begin(); in_use + need > budget && c != cache.end();) {
        if ((*c)->users == 0 && (*c)->ready) {
            in_use -= (*c)->bytes;
            evicted.push_back(*c);
            c = cache.erase(c);
            stats.evictions++;
        } else {
            ++c;
        }
    }
    for (auto c = w->ws.begin(); in_use + need > budget && c != w->ws.end();) {
        if (c->first != keep) {
            in_use -= c->second->bytes;
            to_free.push_back(std::move(c->second));
            c = w->ws.erase(c);
        } else {
            ++c;
        }
    }
    for (auto &ow : workers) {
        if (in_use + need <= budget || inflight > 0) break;
        if (ow.get() == w) continue;
        for (auto c = ow->ws.begin(); in_use + need > budget && c != ow->ws.end();) {
            in_use -= c->second->bytes;
            to_free.push_back(std::move(c->second));
            c = ow->ws.erase(c);
        }
    }
    return in_use + need <= budget;
}

// Under the lock, after need_of/make_room: take job j's reservation of `need` bytes.
void tdda_server::take(Worker *w, Job &j, bool with_ws, size_t need) {
    const tdda_request &r = j.req;
    in_use += need;
    stats.peak_bytes = std::max<int64_t>(stats.peak_bytes, (int64_t)in_use);
    auto t = find(j.key);
    if (t) {
        j.hit = true;
        t->users++;
        stats.cache_hits++;
    } else {
        j.hit = false;
        t = std::make_shared<Tensor>();
        t->key = j.key;
        t->bytes = tensor_bytes(r.num_x, r.num_y, r.num_z);
        t->users = 1;
        cache.push_back(t);
        stats.cache_misses++;
    }
    j.tensor = t;
    if (with_ws) {
        auto &slot = w->ws[shape_of(r)];
        if (!slot) {
            // reserved now, allocated by the worker outside the lock
            slot.reset(new Workspace());
            slot->bytes = Workspace::bytes_for(r.num_x, r.num_y, r.num_z, cfg.max_rhs);
        }
        if (r.precision == TDDA_PREC_C128 && !slot->has64 && !slot->want64) {
            slot->want64 = true;
            slot->bytes += Workspace::bytes64_for(r.num_x, r.num_y, r.num_z, cfg.max_rhs);
        }
    }
}

void tdda_server::run(Worker *w) {
    cudaSetDevice(device);
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        if (stop && queue.empty()) return;
        FreeList to_free;
        EvictList evicted;
        std::vector<std::shared_ptr<Job>> batch;
        for (auto q = queue.begin(); q != queue.end(); ++q) {
            const long long need = need_of(w, **q, true);
            if (need >= 0 && make_room(w, (size_t)need, shape_of((*q)->req), to_free, evicted)) {
                take(w, **q, true, (size_t)need);
                batch.push_back(*q);
                queue.erase(q);
                break;
            }
            if (q == queue.begin()) stats.admission_waits++;
        }
        auto release = [&]() {
            to_free.clear();
            for (auto &e : evicted) {
                cudaFreeAsync(e->ahat64, w->stream);
                cudaFreeAsync(e->ahat32, w->stream);
            }
            evicted.clear();
        };
        if (batch.empty()) {
            if (!to_free.empty() || !evicted.empty()) {
                lk.unlock();
                release();
                cudaStreamSynchronize(w->stream);
                lk.lock();
                continue;
            }
            cv_work.wait(lk);
            continue;
        }
        // continuous batching: queued requests of the same grid join as further
        // right-hand sides, each with its own tensor (shared when the keys match)
        const tdda_request &r0 = batch[0]->req;
        const Shape sh = shape_of(r0);
        int rhs = r0.npol;
        // a tensor that this batch itself is about to build is shared, not waited for
        auto built_here = [&](const Job &j) {
            auto t = find(j.key);
            if (!t || t->ready) return false;
            for (auto &b : batch)
                if (b->tensor == t) return true;
            return false;
        };
        for (auto q = queue.begin(); q != queue.end();) {
            const tdda_request &r = (*q)->req;
            bool joined = false;
            if (shape_of(r) == sh && r.precision == r0.precision && r.tol == r0.tol && r.max_iter == r0.max_iter &&
                rhs + r.npol <= batch[0]->rhs_cap) {
                const long long need = built_here(**q) ? 0 : need_of(w, **q, false);
                if (need >= 0 && make_room(w, (size_t)need, sh, to_free, evicted)) {
                    take(w, **q, false, (size_t)need);
                    rhs += r.npol;
                    batch.push_back(*q);
                    q = queue.erase(q);
                    stats.merged_requests++;
                    joined = true;
                }
            }
            if (!joined) ++q;
        }
        const auto now = Clock::now();
        for (auto &j : batch) j->t_admit = now;
        stats.batches++;
        inflight++;
        stats.max_concurrent = std::max(stats.max_concurrent, inflight);
        lk.unlock();
        release();
        run_batch(w, batch);
        lk.lock();
        inflight--;
        for (auto &j : batch) {
            std::shared_ptr<Tensor> t = j->tensor;
            j->tensor.reset();
            t->users--;
            for (auto c = cache.begin(); c != cache.end(); ++c)
                if (*c == t) {
                    cache.erase(c);
                    if (t->failed) in_use -= t->bytes;
                    else cache.push_back(t);  // most recently used last
                    break;
                }
            j->done = true;
            stats.completed++;
            if (j->res.status != TDDA_OK) stats.failed++;
        }
        stats.cached_tensors = (int64_t)cache.size();
        stats.bytes_in_use = (int64_t)in_use;
        cv_done.notify_all();
        cv_work.notify_all();
    }
}

void tdda_server::run_batch(Worker *w, std::vector<std::shared_ptr<Job>> &batch) {
    const tdda_request &r0 = batch[0]->req;
    const int nx = r0.num_x, ny = r0.num_y, nz = r0.num_z;
    const long long nbox = (long long)nx * ny * nz;
    cudaStream_t s = w->stream;
    auto fail = [&](tdda_status st, const std::string &msg) {
        for (auto &j : batch) {
            j->res.status = st;
            j->error = msg;
            j->t_done = Clock::now();
        }
    };
    Workspace *ws = nullptr;
    {
        std::lock_guard<std::mutex> g(mu);
        ws = w->ws[shape_of(r0)].get();
    }
    tdda_status st = TDDA_OK;
    if (ws->cap == 0) {
        const size_t reserved = ws->bytes;
        st = ws->init(nx, ny, nz, cfg.max_rhs);
        ws->bytes = reserved;
        if (st != TDDA_OK) {
            const std::string msg = get_error();
            std::lock_guard<std::mutex> g(mu);
            in_use -= ws->bytes;
            w->ws.erase(shape_of(r0));
            for (auto &j : batch)
                if (!j->hit) j->tensor->failed = true;
            fail(st, msg);
            return;
        }
    }
    const bool c128 = r0.precision == TDDA_PREC_C128;
    if (c128 && !ws->has64) {
        const size_t reserved = ws->bytes;
        st = ws->init64();
        ws->bytes = reserved;
        if (st != TDDA_OK) {
            fail(st, get_error());
            return;
        }
    }
    // tensors of the requests that missed the cache, one after another on this stream
    const ConvGeom &g = ws->op64.g;
    const size_t nfold = (size_t)g.hx * g.hy * g.hz * 6;
    std::vector<double> build_ms(batch.size(), 0.0);
    for (size_t jj = 0; jj < batch.size(); ++jj) {
        Job &j = *batch[jj];
        if (j.hit) continue;
        Tensor &t = *j.tensor;
        const auto tb0 = Clock::now();
        const tdda_request &r = j.req;
        bool ok = cudaMallocAsync(&t.ahat64, sizeof(double2) * nfold, s) == cudaSuccess &&
                  cudaMallocAsync(&t.ahat32, sizeof(float2) * nfold, s) == cudaSuccess;
        LatticeParams L{};
        L.nx = nx; L.ny = ny; L.nz = nz;
        L.Lx = g.Lx; L.Ly = g.Ly; L.Lz = g.Lz;
        L.d = r.d; L.K = 2.0 * M_PI / (r.lam / r.nback); L.Kf = M_PI / r.d;
        L.Lm = r.Lm * r.d; L.Ln = r.Ln * r.d;
        L.MAXm = r.MAXm; L.MAXn = r.MAXn; L.method = r.method; L.gamma = 0.01; L.delta = delta;
        if (ok) {
            w->scratch.sc = d_sici;
            w->scratch.ntab = ntab;
            ok = build_tensor_async(L, w->scratch, t.ahat64, t.ahat32, s, w->a0_host, nullptr, nullptr) == TDDA_OK &&
                 cudaStreamSynchronize(s) == cudaSuccess;
        }
        std::lock_guard<std::mutex> g2(mu);
        if (!ok) {
            // every tensor of this batch not built yet is abandoned with it
            for (auto &o : batch)
                if (!o->tensor->ready) o->tensor->failed = true;
            cudaFreeAsync(t.ahat64, s);
            cudaFreeAsync(t.ahat32, s);
            t.ahat64 = nullptr;
            t.ahat32 = nullptr;
            fail(TDDA_ERR_CUDA, std::string("tensor build failed: ") + get_error());
            cv_work.notify_all();
            return;
        }
        const double2 *a = w->a0_host;
        t.a0 = make_double2((a[0].x + a[3].x + a[5].x) / 3.0, (a[0].y + a[3].y + a[5].y) / 3.0);
        t.ready = true;
        cv_work.notify_all();  // workers waiting for this tensor
        build_ms[jj] = ms_between(tb0, Clock::now());
    }
    const auto ts0 = Clock::now();
    // per right-hand side parameters, densities and tensors
    SetupArgs sa{};
    sa.nx = nx; sa.ny = ny; sa.nz = nz;
    int k = 0;
    bool shared = true;
    for (size_t jj = 0; jj < batch.size(); ++jj) {
        const tdda_request &r = batch[jj]->req;
        const Tensor &t = *batch[jj]->tensor;
        shared &= (batch[jj]->tensor == batch[0]->tensor);
        std::memcpy(ws->h_rho + jj * (size_t)nbox, batch[jj]->rho.data(), sizeof(double) * nbox);
        const double K = 2.0 * M_PI / (r.lam / r.nback);
        double2 m[2];
        for (int i = 0; i < 2; ++i) {
            std::complex<double> v(r.material[2 * i], r.material[2 * i + 1]);
            v = v / (r.nback * r.nback);
            if (std::sqrt(std::norm(v)) < 1.01) v = v + 0.01;
            m[i] = make_double2(v.real(), v.imag());
        }
        for (int q = 0; q < r.npol; ++q, ++k) {
            RhsParams &p = sa.r[k];
            p.A.lam = r.lam; p.A.K = K; p.A.d = r.d; p.A.m0 = m[0]; p.A.m1 = m[1];
            p.A.S = 0.0;
            for (int c = 0; c < 3; ++c) p.A.S += std::pow(r.n_E0[q][c] * r.n_K[c], 2);
            p.a0 = t.a0;
            p.kd = K * r.d;
            for (int c = 0; c < 3; ++c) {
                p.nK[c] = r.n_K[c];
                p.e[c] = r.E0 * r.n_E0[q][c];
            }
            p.job = (int)jj;
            ws->h_tab64[k] = t.ahat64;
            ws->h_tab32[k] = t.ahat32;
        }
    }
    const int nrhs = k;
    sa.nrhs = nrhs;
    ws->op64.ahat = batch[0]->tensor->ahat64;
    ws->op32.ahat = batch[0]->tensor->ahat32;
    ws->op64.ahat_rhs = shared ? nullptr : ws->d_tab64;
    ws->op32.ahat_rhs = shared ? nullptr : ws->d_tab32;
    std::vector<tdda_solve_info> info(nrhs);
    st = TDDA_OK;
    if (cudaMemcpyAsync(ws->d_rho, ws->h_rho, sizeof(double) * nbox * batch.size(), cudaMemcpyHostToDevice, s) !=
            cudaSuccess ||
        (!shared && (cudaMemcpyAsync(ws->d_tab64, ws->h_tab64, sizeof(void *) * nrhs, cudaMemcpyHostToDevice, s) !=
                         cudaSuccess ||
                     cudaMemcpyAsync(ws->d_tab32, ws->h_tab32, sizeof(void *) * nrhs, cudaMemcpyHostToDevice, s) !=
                         cudaSuccess)))
        st = TDDA_ERR_CUDA;
    if (st == TDDA_OK) {
        count_launches(1);
        k_serve_setup<<<blocks_for(nbox * nrhs), 256, 0, s>>>(sa, ws->d_rho, ws->al64, ws->al32, ws->sc64, ws->sc32,
                                                             ws->alS32, c128 ? ws->alS64 : nullptr, ws->diel, ws->B);
        if (cudaGetLastError() != cudaSuccess) st = TDDA_ERR_CUDA;
    }
    if (st == TDDA_OK) {
        const int gsteps = cfg.use_graphs ? (cfg.graph_steps > 0 ? cfg.graph_steps : 4) : 0;
        if (c128) {
            RefineWork<double2> rw;
            rw.op64 = &ws->op64; rw.al64 = ws->al64; rw.op = &ws->op64; rw.kv = &ws->kv64;
            rw.al = ws->alS64; rw.sc = ws->sc64; rw.sc64 = ws->sc64; rw.R = ws->R64; rw.D = ws->D64;
            rw.Rm = ws->Rm; rw.st_res = ws->st_res; rw.st_res_host = ws->st_res_host;
            rw.d_part = ws->d_part; rw.h_part = ws->h_part;
            rw.nbox = nbox; rw.dstride = (size_t)nbox; rw.graph_steps = gsteps; rw.s = s;
            st = refine_solve<double2>(rw, ws->B, ws->X, nrhs, true, r0.max_iter, r0.tol, info.data());
        } else {
            RefineWork<float2> rw;
            rw.op64 = &ws->op64; rw.al64 = ws->al64; rw.op = &ws->op32; rw.kv = &ws->kv32;
            rw.al = ws->alS32; rw.sc = ws->sc32; rw.sc64 = ws->sc64; rw.R = ws->R32; rw.D = ws->D32;
            rw.Rm = ws->Rm; rw.st_res = ws->st_res; rw.st_res_host = ws->st_res_host;
            rw.d_part = ws->d_part; rw.h_part = ws->h_part;
            rw.nbox = nbox; rw.dstride = (size_t)nbox; rw.graph_steps = gsteps; rw.s = s;
            st = refine_solve<float2>(rw, ws->B, ws->X, nrhs, true, r0.max_iter, r0.tol, info.data());
        }
    }
    if (st == TDDA_OK) {
        const size_t v = 3 * (size_t)nbox * nrhs;
        count_launches(1);
        k_serve_out<<<blocks_for((long long)v), 256, 0, s>>>(nrhs, nx, ny, nz, ws->X, ws->al64, ws->diel, ws->d_out,
                                                              ws->d_out + v);
        if (cudaMemcpyAsync(ws->h_out, ws->d_out, sizeof(double2) * 2 * v, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            st = TDDA_ERR_CUDA;
    }
    if (st != TDDA_OK) {
        std::string msg = get_error();
        if (msg.empty()) msg = cudaGetErrorString(cudaGetLastError());
        fail(st, msg);
        return;
    }
    const size_t v = 3 * (size_t)nbox * nrhs;
    const auto done = Clock::now();
    k = 0;
    for (size_t jj = 0; jj < batch.size(); ++jj) {
        Job &j = *batch[jj];
        const tdda_request &r = j.req;
        const size_t n3 = 3 * (size_t)nbox;
        if (r.P_out) std::memcpy(r.P_out, ws->h_out + (size_t)k * n3, sizeof(double2) * n3 * r.npol);
        if (r.E_out) std::memcpy(r.E_out, ws->h_out + v + (size_t)k * n3, sizeof(double2) * n3 * r.npol);
        for (int q = 0; q < r.npol; ++q) j.res.info[q] = info[k + q];
        k += r.npol;
        j.res.status = TDDA_OK;
        j.res.batch_rhs = nrhs;
        j.res.batch_requests = (int)batch.size();
        j.res.cache_hit = j.hit ? 1 : 0;
        j.res.worker = w->id;
        j.res.queue_ms = ms_between(j.t_submit, j.t_admit);
        j.res.build_ms = build_ms[jj];
        j.res.solve_ms = ms_between(ts0, done);
        j.t_done = Clock::now();
        j.res.total_ms = ms_between(j.t_submit, j.t_done);
    }
}

static tdda_status sbad(const std::string &m) {
    set_error(m);
    return TDDA_ERR_BAD_ARG;
}

extern "C" {

tdda_status tdda_server_create(const tdda_server_config *cfg, const double *si, const double *ci, int64_t ntab,
                               tdda_server **out) {
    if (!cfg || !out) return sbad("null argument");
    *out = nullptr;
    if (cfg->workers < 1 || cfg->workers > 64) return sbad("workers must be in 1..64");
    if (cfg->max_rhs < 1 || cfg->max_rhs > kMaxRhs) return sbad("max_rhs must be in 1..16");
    if (cfg->hbm_budget_bytes <= 0) return sbad("hbm_budget_bytes must be positive");
    if (cfg->graph_steps < 0 || cfg->graph_steps > 64) return sbad("graph_steps must be in 0..64");
    std::unique_ptr<tdda_server> S(new tdda_server());
    S->cfg = *cfg;
    TDDA_CUDA_TRY(cudaGetDevice(&S->device));
    std::vector<double2> h(ntab > 0 ? ntab : 1, make_double2(0.0, 0.0));
    for (int64_t q = 0; q < ntab; ++q) h[q] = make_double2(si[q], ci[q]);
    TDDA_CUDA_TRY(cudaMalloc(&S->d_sici, sizeof(double2) * h.size()));
    TDDA_CUDA_TRY(cudaMemcpy(S->d_sici, h.data(), sizeof(double2) * h.size(), cudaMemcpyHostToDevice));
    S->ntab = (long)(si && ci ? ntab : 0);
    for (int i = 0; i < cfg->workers; ++i) {
        std::unique_ptr<Worker> w(new Worker());
        w->id = i;
        TDDA_CUDA_TRY(cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking));
        TDDA_CUDA_TRY(cudaMallocHost(&w->a0_host, sizeof(double2) * 6));
        S->workers.push_back(std::move(w));
    }
    for (auto &w : S->workers) {
        Worker *wp = w.get();
        tdda_server *sp = S.get();
        w->th = std::thread([sp, wp] { sp->run(wp); });
    }
    *out = S.release();
    return TDDA_OK;
}

tdda_status tdda_server_submit(tdda_server *s, const tdda_request *req, int64_t *ticket) {
    if (!s || !req || !ticket) return sbad("null argument");
    const tdda_request &r = *req;
    if (r.num_x < 1 || r.num_y < 1 || r.num_z < 1) return sbad("grid sizes must be positive");
    if (r.npol < 1 || r.npol > TDDA_SERVER_MAX_POL) return sbad("npol must be in 1..4");
    if (r.npol > s->cfg.max_rhs) return sbad("npol exceeds the server's max_rhs");
    if (!(r.d > 0) || !(r.lam > 0) || !(r.nback > 0)) return sbad("d, lam and nback must be positive");
    if (r.method != 0 && r.method != 1) return sbad("method must be 0 (FCD) or 1 (LDR)");
    if (r.method == 0 && s->ntab < 2) return sbad("FCD needs the SiCi tables at server creation");
    if (r.MAXm < 0 || r.MAXn < 0) return sbad("MAXm, MAXn must be >= 0");
    if (r.precision != TDDA_PREC_MIXED && r.precision != TDDA_PREC_C128) return sbad("precision must be 0 or 1");
    if (!(r.tol > 0) || r.max_iter < 1) return sbad("tol must be > 0 and max_iter >= 1");
    if (!r.rho) return sbad("rho is required");
    // the largest batch the fused operator takes for this grid (the x pass
    // holds every right-hand side of a pencil group in one block)
    std::string why;
    int cap = 0;
    for (int k = s->cfg.max_rhs; k >= 1 && cap == 0; --k)
        if (conv_supported(r.num_x, r.num_y, r.num_z, k, 8, why) && conv_supported(r.num_x, r.num_y, r.num_z, k, 16, why))
            cap = k;
    if (cap < r.npol) return sbad("grid not supported with " + std::to_string(r.npol) + " right-hand sides: " + why);
    const long long nbox = (long long)r.num_x * r.num_y * r.num_z;
    auto j = std::make_shared<Job>();
    j->rho.assign(r.rho, r.rho + nbox);
    for (double v : j->rho)
        if (!(v >= 0.0 && v <= 1.0)) return sbad("design density outside [0, 1]");
    size_t worst = Workspace::bytes_for(r.num_x, r.num_y, r.num_z, s->cfg.max_rhs) +
                   tensor_bytes(r.num_x, r.num_y, r.num_z);
    if (r.precision == TDDA_PREC_C128) worst += Workspace::bytes64_for(r.num_x, r.num_y, r.num_z, s->cfg.max_rhs);
    if (worst > (size_t)s->cfg.hbm_budget_bytes) {
        set_error("request needs " + std::to_string(worst) + " bytes, more than the HBM budget");
        return TDDA_ERR_OOM;
    }
    j->req = r;
    j->req.rho = nullptr;
    j->rhs_cap = cap;
    j->key = TensorKey{r.num_x, r.num_y, r.num_z, r.method, r.MAXm, r.MAXn, r.d, r.lam, r.nback,
                       (r.MAXm > 0 ? r.Lm : 0.0), (r.MAXn > 0 ? r.Ln : 0.0)};
    j->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> g(s->mu);
        if (s->stop) return sbad("server is shutting down");
        j->ticket = s->next_ticket++;
        s->jobs[j->ticket] = j;
        s->queue.push_back(j);
        s->stats.submitted++;
    }
    s->cv_work.notify_all();
    *ticket = j->ticket;
    return TDDA_OK;
}

tdda_status tdda_server_wait(tdda_server *s, int64_t ticket, double timeout_s, tdda_request_result *result) {
    if (!s || !result) return sbad("null argument");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->jobs.find(ticket);
    if (it == s->jobs.end()) return sbad("unknown ticket");
    std::shared_ptr<Job> j = it->second;
    auto ready = [&] { return j->done; };
    if (timeout_s < 0) {
        s->cv_done.wait(lk, ready);
    } else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) {
        set_error("request not finished");
        return TDDA_ERR_TIMEOUT;
    }
    *result = j->res;
    s->jobs.erase(ticket);
    if (j->res.status != TDDA_OK) set_error(j->error);
    return TDDA_OK;
}

tdda_status tdda_server_reserve(tdda_server *s, int32_t nx, int32_t ny, int32_t nz, int32_t precision) {
    if (!s) return sbad("null argument");
    if (nx < 1 || ny < 1 || nz < 1) return sbad("grid sizes must be positive");
    if (precision != TDDA_PREC_MIXED && precision != TDDA_PREC_C128) return sbad("precision must be 0 or 1");
    std::string why;
    if (!conv_supported(nx, ny, nz, 1, 8, why) || !conv_supported(nx, ny, nz, 1, 16, why))
        return sbad("grid not supported: " + why);
    std::lock_guard<std::mutex> g(s->mu);
    if (!s->queue.empty() || s->inflight > 0) return sbad("reserve before submitting requests");
    const Shape sh{nx, ny, nz};
    for (auto &w : s->workers) {
        auto it = w->ws.find(sh);
        const bool missing = it == w->ws.end();
        size_t need = missing ? Workspace::bytes_for(nx, ny, nz, s->cfg.max_rhs) : 0;
        const bool want64 = precision == TDDA_PREC_C128 && (missing || !it->second->has64);
        if (want64) need += Workspace::bytes64_for(nx, ny, nz, s->cfg.max_rhs);
        if (s->in_use + need > (size_t)s->cfg.hbm_budget_bytes) {
            set_error("reserving workspaces for this grid exceeds the HBM budget");
            return TDDA_ERR_OOM;
        }
        if (missing) {
            std::unique_ptr<Workspace> ws(new Workspace());
            tdda_status st = ws->init(nx, ny, nz, s->cfg.max_rhs);
            if (st != TDDA_OK) return st;
            it = w->ws.emplace(sh, std::move(ws)).first;
        }
        if (want64) {
            const size_t keep = it->second->bytes;
            tdda_status st = it->second->init64();
            it->second->bytes = keep + Workspace::bytes64_for(nx, ny, nz, s->cfg.max_rhs);
            if (st != TDDA_OK) return st;
        }
        s->in_use += need;
        s->stats.peak_bytes = std::max<int64_t>(s->stats.peak_bytes, (int64_t)s->in_use);
    }
    s->stats.bytes_in_use = (int64_t)s->in_use;
    return TDDA_OK;
}

tdda_status tdda_server_get_stats(tdda_server *s, tdda_server_stats *out) {
    if (!s || !out) return sbad("null argument");
    std::lock_guard<std::mutex> g(s->mu);
    s->stats.bytes_in_use = (int64_t)s->in_use;
    s->stats.cached_tensors = (int64_t)s->cache.size();
    *out = s->stats;
    return TDDA_OK;
}

void tdda_server_destroy(tdda_server *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto &w : s->workers)
        if (w->th.joinable()) w->th.join();
    for (auto &w : s->workers) cudaStreamSynchronize(w->stream);
    for (auto &t : s->cache) {
        cudaFree(t->ahat64);
        cudaFree(t->ahat32);
    }
    s->cache.clear();
    for (auto &w : s->workers) {
        w->ws.clear();
        w->scratch.sc = nullptr;  // the shared table is freed below
        w->scratch.release();
        cudaFreeHost(w->a0_host);
        cudaStreamDestroy(w->stream);
    }
    cudaFree(s->d_sici);
    delete s;
}

}  // extern "C"
