// Polynomial-preconditioned GMRES in complex128 refinement (see gmres.cuh).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "dense_eig.h"
#include "gmres.cuh"

namespace tdda {

// ----------------------------------------------------------------------------
// Gram-Schmidt kernels: all sums in FP64, block partials added in block order
// (deterministic).  Vectors of right-hand side k start at k * rstr; basis
// vector i starts at i * vstr.
// ----------------------------------------------------------------------------
constexpr int kGsThreads = 256;
constexpr int kGsBlocks = 148 * 4;
constexpr int kGsChunk = 8;   // basis vectors per multi-dot CTA
// directions beyond the residual's that a recycled start may carry (each
// refinement step that starts from a recycled space adds one)
constexpr int kMaxAug = 4;
// Gram-Schmidt: a second projection pass runs when the first leaves
// ||w'||^2 < kReorth ||w||^2 (||w'|| < 0.32 ||w||).  On the periodic
// 128x128x32 structure 0.1 measured faster than 0.25 in both precisions (fewer
// second passes, no more operator applications).
constexpr double kReorth = 0.1;

// The nv basis vectors split into nch = gridDim.y chunks of near-equal size
// (at most kGsChunk each, the first nv % nch one larger), so that the CTAs of
// every chunk stream about the same bytes: chunk c holds [i0, i0 + nb).
__device__ __forceinline__ void chunk_of(int nv, int c, int nch, int &i0, int &nb) {
    const int base = nv / nch, rem = nv % nch;
    nb = base + (c < rem ? 1 : 0);
    i0 = c * base + min(c, rem);
}

template <int NV> __device__ __forceinline__ void block_sum_v(double2 (&v)[NV], double2 *sm) {
    // sm: NV * (kGsThreads / 32) double2
#pragma unroll
    for (int k = 0; k < NV; ++k)
        for (int o = 16; o > 0; o >>= 1) {
            v[k].x += __shfl_down_sync(0xffffffffu, v[k].x, o);
            v[k].y += __shfl_down_sync(0xffffffffu, v[k].y, o);
        }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) sm[k * (kGsThreads / 32) + warp] = v[k];
    __syncthreads();
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double2 t = sm[k * (kGsThreads / 32)];
            for (int w = 1; w < kGsThreads / 32; ++w) {
                t.x += sm[k * (kGsThreads / 32) + w].x;
                t.y += sm[k * (kGsThreads / 32) + w].y;
            }
            v[k] = t;
        }
}

// The two streaming Gram-Schmidt kernels move 16-byte packs: two complex64
// elements (float4) or one complex128 element.  Vectors whose length or
// starts are not 16-byte multiples take the element-wise variants.
template <typename C> struct Pack;
template <> struct Pack<float2> {
    using T = float4;
    static constexpr int E = 2;
    __device__ static T zero() { return make_float4(0.f, 0.f, 0.f, 0.f); }
    __device__ static double2 get(const T &p, int i) {
        return i == 0 ? make_double2(p.x, p.y) : make_double2(p.z, p.w);
    }
    __device__ static T make(const double2 (&d)[2]) {
        return make_float4((float)d[0].x, (float)d[0].y, (float)d[1].x, (float)d[1].y);
    }
};
template <> struct Pack<double2> {
    using T = double2;
    static constexpr int E = 1;
    __device__ static T zero() { return make_double2(0.0, 0.0); }
    __device__ static double2 get(const T &p, int) { return p; }
    __device__ static T make(const double2 (&d)[1]) { return d[0]; }
};

// part[(k * no + i) * gridDim.x + blk] = this block's share of conj(V_i[k]) . w[k]
// for i < nv; with no = nv + 1 the CTAs of the first chunk also sum ||w[k]||^2
// into entry i = nv.
// The same sums with the vectors streamed into shared memory by the bulk-copy
// engine (cp.async.bulk, global -> shared, completion on an mbarrier): tiles
// of kBdTile packs of w and of every basis vector of the CTA's chunk, kBdStages
// tiles in a ring, kBdStages - 1 of them in flight while the threads work on
// the oldest.  The bytes in flight do not cost registers, so two CTAs per SM
// keep ~144 KB of loads outstanding.  CTA (x, chunk, rhs) takes the tiles
// x, x + gridDim.x, ... of its chunk; partials as in k_multidot.  A wait that
// has not completed after kBdSpin polls marks the CTA's partials NaN (the host
// rejects non-finite sums) and stops the CTA; every copy issued before has
// been waited for by then or belongs to the stalled tile.
constexpr int kBdTile = 256;    // packs per vector per tile (4 KB)
constexpr int kBdStages = 3;
constexpr long long kBdSpin = 1ll << 22;
constexpr size_t kBdSmem = (size_t)kBdStages * (kGsChunk + 1) * kBdTile * 16;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

template <typename C>
__global__ void __launch_bounds__(kGsThreads, 2) k_multidot_bulk(long long np, int nv, int no,
                                                                 const typename Pack<C>::T *__restrict__ V,
                                                                 size_t vstr, size_t rstr,
                                                                 const typename Pack<C>::T *__restrict__ w,
                                                                 double2 *__restrict__ part) {
    using PK = Pack<C>;
    using PT = typename PK::T;
    extern __shared__ __align__(128) unsigned char bd_smem[];
    __shared__ __align__(8) unsigned long long full[kBdStages];
    __shared__ double2 sm[(kGsChunk + 1) * (kGsThreads / 32)];
    PT *tiles = reinterpret_cast<PT *>(bd_smem);   // [stage][vector (w last)][kBdTile]
    const int k = blockIdx.z;
    int i0, nb;
    chunk_of(nv, blockIdx.y, gridDim.y, i0, nb);
    const bool norm = no > nv && blockIdx.y == 0;
    const long long ntiles = (np + kBdTile - 1) / kBdTile;
    const PT *wk = w + (size_t)k * rstr;
    const PT *Vk = V + (size_t)k * rstr + (size_t)i0 * vstr;
    if (threadIdx.x == 0) {
        for (int st = 0; st < kBdStages; ++st)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full[st])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    pdl_wait();
    // tile t into ring slot st (thread 0)
    auto issue = [&](long long t, int st) {
        const long long p0 = t * kBdTile;
        const uint32_t bytes = (uint32_t)(min((long long)kBdTile, np - p0) * 16);
        const uint32_t bar = smem_u32(&full[st]);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes * (nb + 1))
                     : "memory");
        PT *slot = tiles + (size_t)st * (kGsChunk + 1) * kBdTile;
        for (int q = 0; q <= nb; ++q) {
            const PT *src = (q < nb ? Vk + (size_t)q * vstr : wk) + p0;
            PT *dst = slot + (size_t)(q < nb ? q : kGsChunk) * kBdTile;
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
                             "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(bar)
                         : "memory");
        }
    };
    double2 acc[kGsChunk + 1];
#pragma unroll
    for (int q = 0; q <= kGsChunk; ++q) acc[q] = make_double2(0.0, 0.0);
    const long long t0 = blockIdx.x, dt = gridDim.x;
    if (threadIdx.x == 0)
        for (int st = 0; st < kBdStages - 1; ++st)
            if (t0 + st * dt < ntiles) issue(t0 + st * dt, st);
    bool stalled = false;
    long long it = 0;
    for (long long t = t0; t < ntiles; t += dt, ++it) {
        const int st = (int)(it % kBdStages);
        const uint32_t parity = (uint32_t)((it / kBdStages) & 1);
        if (threadIdx.x == 0) {
            // the slot refilled here was read in iteration it - 1, which every
            // thread has left (barrier at the end of the loop)
            const long long tn = t + (kBdStages - 1) * dt;
            if (tn < ntiles) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                issue(tn, (int)((it + kBdStages - 1) % kBdStages));
            }
        }
        uint32_t ok = 0;
        for (long long spin = 0; !ok; ++spin) {
            asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                         " selp.u32 %0, 1, 0, p;\n}"
                         : "=r"(ok)
                         : "r"(smem_u32(&full[st])), "r"(parity)
                         : "memory");
            if (!ok && spin > kBdSpin) break;
        }
        if (!__syncthreads_and((int)ok)) {
            stalled = true;
            // let the copies already issued land (bounded) before the CTA ends
            if (threadIdx.x == 0)
                for (int a = 0; a < kBdStages - 1; ++a) {
                    const long long ia = it + a;
                    if (t + a * dt >= ntiles) break;
                    const uint32_t par = (uint32_t)((ia / kBdStages) & 1);
                    uint32_t got = 0;
                    for (long long spin = 0; !got && spin <= kBdSpin; ++spin)
                        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                                     " selp.u32 %0, 1, 0, p;\n}"
                                     : "=r"(got)
                                     : "r"(smem_u32(&full[(int)(ia % kBdStages)])), "r"(par)
                                     : "memory");
                }
            __syncthreads();
            break;
        }
        const PT *slot = tiles + (size_t)st * (kGsChunk + 1) * kBdTile;
        const long long cnt = min((long long)kBdTile, np - t * kBdTile);
        for (int p = threadIdx.x; p < cnt; p += kGsThreads) {
            const PT wv = slot[(size_t)kGsChunk * kBdTile + p];
            PT v[kGsChunk];
#pragma unroll
            for (int q = 0; q < kGsChunk; ++q) v[q] = q < nb ? slot[(size_t)q * kBdTile + p] : PK::zero();
#pragma unroll
            for (int e = 0; e < PK::E; ++e) {
                const double2 wd = PK::get(wv, e);
#pragma unroll
                for (int q = 0; q < kGsChunk; ++q) {
                    const double2 d = cdot1(PK::get(v[q], e), wd);
                    acc[q].x += d.x;
                    acc[q].y += d.y;
                }
                if (norm) acc[kGsChunk].x += wd.x * wd.x + wd.y * wd.y;
            }
        }
        __syncthreads();
    }
    block_sum_v<kGsChunk + 1>(acc, sm);
    if (threadIdx.x == 0) {
        const double bad = __longlong_as_double(0x7ff8000000000000ll);
#pragma unroll
        for (int q = 0; q <= kGsChunk; ++q)
            if (stalled) acc[q] = make_double2(bad, bad);
#pragma unroll
        for (int q = 0; q < kGsChunk; ++q)
            if (q < nb) part[((size_t)k * no + i0 + q) * gridDim.x + blockIdx.x] = acc[q];
        if (norm) part[((size_t)k * no + nv) * gridDim.x + blockIdx.x] = acc[kGsChunk];
    }
}

// The same sums element by element (any length and alignment).
template <typename C>
__global__ void __launch_bounds__(kGsThreads) k_multidot_e(long long n, int nv, int no, const C *__restrict__ V,
                                                           size_t vstr, size_t rstr, const C *__restrict__ w,
                                                           double2 *__restrict__ part) {
    pdl_wait();
    __shared__ double2 sm[(kGsChunk + 1) * (kGsThreads / 32)];
    const int k = blockIdx.z;
    int i0, nb;
    chunk_of(nv, blockIdx.y, gridDim.y, i0, nb);
    const bool norm = no > nv && blockIdx.y == 0;
    double2 acc[kGsChunk + 1];
#pragma unroll
    for (int q = 0; q <= kGsChunk; ++q) acc[q] = make_double2(0.0, 0.0);
    const C *wk = w + (size_t)k * rstr;
    const C *Vk = V + (size_t)k * rstr + (size_t)i0 * vstr;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const double2 wd = to_d(__ldg(wk + e));
        C v[kGsChunk];
#pragma unroll
        for (int q = 0; q < kGsChunk; ++q) v[q] = q < nb ? __ldg(Vk + (size_t)q * vstr + e) : czero<C>();
#pragma unroll
        for (int q = 0; q < kGsChunk; ++q) {
            const double2 d = cdot1(to_d(v[q]), wd);
            acc[q].x += d.x;
            acc[q].y += d.y;
        }
        if (norm) acc[kGsChunk].x += wd.x * wd.x + wd.y * wd.y;
    }
    block_sum_v<kGsChunk + 1>(acc, sm);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < kGsChunk; ++q)
            if (q < nb) part[((size_t)k * no + i0 + q) * gridDim.x + blockIdx.x] = acc[q];
        if (norm) part[((size_t)k * no + nv) * gridDim.x + blockIdx.x] = acc[kGsChunk];
    }
}

// out[k] = (w[k] - sum_{i < nv} c[k][i] V_i[k]) * c[k][nv].x: one Gram-Schmidt
// update and the normalisation in one pass (c: device, rows of nv + 1).
// Lengths and strides in packs; one pack per thread, the loads of four basis
// vectors issued together, 16 CTAs per SM.
template <typename C>
__global__ void __launch_bounds__(kGsThreads) k_gs_update_scale(long long np, int nv,
                                                                const typename Pack<C>::T *__restrict__ V,
                                                                size_t vstr, size_t rstr,
                                                                const double2 *__restrict__ c,
                                                                typename Pack<C>::T *__restrict__ w) {
    using PK = Pack<C>;
    using PT = typename PK::T;
    pdl_wait();
    extern __shared__ double2 cs[];
    const int k = blockIdx.z;
    for (int i = threadIdx.x; i <= nv; i += blockDim.x) cs[i] = c[(size_t)k * (nv + 1) + i];
    __syncthreads();
    const double f = cs[nv].x;
    PT *wk = w + (size_t)k * rstr;
    const PT *Vk = V + (size_t)k * rstr;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < np; p += (long long)gridDim.x * blockDim.x) {
        double2 acc[PK::E];
        const PT w0 = wk[p];
#pragma unroll
        for (int e = 0; e < PK::E; ++e) acc[e] = PK::get(w0, e);
        int i = 0;
        for (; i + 4 <= nv; i += 4) {
            PT b[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) b[q] = __ldg(Vk + (size_t)(i + q) * vstr + p);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const double2 h = cs[i + q];
#pragma unroll
                for (int e = 0; e < PK::E; ++e) {
                    const double2 bb = PK::get(b[q], e);
                    acc[e].x -= h.x * bb.x - h.y * bb.y;
                    acc[e].y -= h.x * bb.y + h.y * bb.x;
                }
            }
        }
        for (; i < nv; ++i) {
            const double2 h = cs[i];
            const PT b = __ldg(Vk + (size_t)i * vstr + p);
#pragma unroll
            for (int e = 0; e < PK::E; ++e) {
                const double2 bb = PK::get(b, e);
                acc[e].x -= h.x * bb.x - h.y * bb.y;
                acc[e].y -= h.x * bb.y + h.y * bb.x;
            }
        }
#pragma unroll
        for (int e = 0; e < PK::E; ++e) acc[e] = make_double2(f * acc[e].x, f * acc[e].y);
        wk[p] = PK::make(acc);
    }
}

// The same update element by element (any length and alignment).
template <typename C>
__global__ void __launch_bounds__(kGsThreads) k_gs_update_scale_e(long long n, int nv, const C *__restrict__ V,
                                                                  size_t vstr, size_t rstr,
                                                                  const double2 *__restrict__ c, C *__restrict__ w) {
    pdl_wait();
    extern __shared__ double2 cs[];
    const int k = blockIdx.z;
    for (int i = threadIdx.x; i <= nv; i += blockDim.x) cs[i] = c[(size_t)k * (nv + 1) + i];
    __syncthreads();
    const double f = cs[nv].x;
    C *wk = w + (size_t)k * rstr;
    const C *Vk = V + (size_t)k * rstr;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        double2 acc = to_d(wk[e]);
        int i = 0;
        for (; i + 4 <= nv; i += 4) {
            C b[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) b[q] = __ldg(Vk + (size_t)(i + q) * vstr + e);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const double2 h = cs[i + q], bb = to_d(b[q]);
                acc.x -= h.x * bb.x - h.y * bb.y;
                acc.y -= h.x * bb.y + h.y * bb.x;
            }
        }
        for (; i < nv; ++i) {
            const double2 h = cs[i], bb = to_d(__ldg(Vk + (size_t)i * vstr + e));
            acc.x -= h.x * bb.x - h.y * bb.y;
            acc.y -= h.x * bb.y + h.y * bb.x;
        }
        wk[e] = from_d<C>(make_double2(f * acc.x, f * acc.y));
    }
}

// out[j] = sum over blocks (in order) of part[j * nblk + b], one warp per j;
// with nrm != nullptr the entries are squared norms (real part): nrm[j] gets
// the square root of the sum and inv[j] its reciprocal (0 for a zero norm).
__global__ void k_sum_parts(int nout, int nblk, const double2 *__restrict__ part, double2 *__restrict__ out,
                            double *__restrict__ nrm, double *__restrict__ inv) {
    pdl_wait();
    const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (j >= nout) return;
    double2 t = make_double2(0.0, 0.0);
    for (int b = lane; b < nblk; b += 32) {
        t.x += part[(size_t)j * nblk + b].x;
        t.y += part[(size_t)j * nblk + b].y;
    }
    for (int o = 16; o > 0; o >>= 1) {
        t.x += __shfl_down_sync(0xffffffffu, t.x, o);
        t.y += __shfl_down_sync(0xffffffffu, t.y, o);
    }
    if (lane == 0) {
        if (out != nullptr) out[j] = t;
        if (nrm != nullptr) {
            const double r = sqrt(fmax(t.x, 0.0));
            nrm[j] = r;
            inv[j] = r > 0.0 ? 1.0 / r : 0.0;
        }
    }
}

// w[k] -= sum_{i < nv} h[k * hstr + i] V_i[k]; with part != nullptr also the
// block's share of ||w[k]||^2 (after the update) into part[k * gridDim.x + blk]
template <typename C>
__global__ void __launch_bounds__(kGsThreads) k_gs_update(long long n, int nv, const C *__restrict__ V, size_t vstr,
                                                          size_t rstr, const double2 *__restrict__ h, int hstr,
                                                          C *__restrict__ w, double2 *__restrict__ part) {
    pdl_wait();
    extern __shared__ double2 hs[];
    __shared__ double2 sm[kGsThreads / 32];
    const int k = blockIdx.z;
    for (int i = threadIdx.x; i < nv; i += blockDim.x) hs[i] = h[(size_t)k * hstr + i];
    __syncthreads();
    C *wk = w + (size_t)k * rstr;
    const C *Vk = V + (size_t)k * rstr;
    double2 acc[1] = {make_double2(0.0, 0.0)};
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        double2 v = to_d(wk[e]);
        for (int i = 0; i < nv; ++i) {
            const double2 b = to_d(__ldg(Vk + (size_t)i * vstr + e));
            const double2 c = hs[i];
            v.x -= c.x * b.x - c.y * b.y;
            v.y -= c.x * b.y + c.y * b.x;
        }
        const C vc = from_d<C>(v);
        wk[e] = vc;
        const double2 vd = to_d(vc);
        acc[0].x += vd.x * vd.x + vd.y * vd.y;
    }
    if (part != nullptr) {
        block_sum_v<1>(acc, sm);
        if (threadIdx.x == 0) part[(size_t)k * gridDim.x + blockIdx.x] = acc[0];
    }
}

// out[k] = s[k] * x[k]   (s: device reals, one per right-hand side)
template <typename C>
__global__ void __launch_bounds__(kGsThreads) k_scale_vec(long long n, size_t rstr, const double *__restrict__ s,
                                                          const C *__restrict__ x, C *__restrict__ out) {
    pdl_wait();
    const int k = blockIdx.z;
    const double f = s[k];
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const double2 v = to_d(x[(size_t)k * rstr + e]);
        out[(size_t)k * rstr + e] = from_d<C>(make_double2(f * v.x, f * v.y));
    }
}

// out_l[k] = sum_{i < nin} P[k][i * ldp + l] V_i[k] for l < nout (in chunks of
// kGsChunk outputs per CTA row): the deflated restart's new basis
template <typename C>
__global__ void __launch_bounds__(kGsThreads) k_lincomb_multi(long long n, int nin, int nout, const C *__restrict__ V,
                                                              size_t vstr, size_t rstr, const double2 *__restrict__ P,
                                                              int ldp, size_t pstr, C *__restrict__ out) {
    pdl_wait();
    const int k = blockIdx.z, l0 = blockIdx.y * kGsChunk;
    const int nb = min(kGsChunk, nout - l0);
    const C *Vk = V + (size_t)k * rstr;
    const double2 *Pk = P + (size_t)k * pstr;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        double2 acc[kGsChunk];
#pragma unroll
        for (int q = 0; q < kGsChunk; ++q) acc[q] = make_double2(0.0, 0.0);
        for (int i = 0; i < nin; ++i) {
            const double2 b = to_d(__ldg(Vk + (size_t)i * vstr + e));
#pragma unroll
            for (int q = 0; q < kGsChunk; ++q)
                if (q < nb) {
                    const double2 c = __ldg(Pk + (size_t)i * ldp + l0 + q);
                    acc[q].x += c.x * b.x - c.y * b.y;
                    acc[q].y += c.x * b.y + c.y * b.x;
                }
        }
#pragma unroll
        for (int q = 0; q < kGsChunk; ++q)
            if (q < nb) out[(size_t)(l0 + q) * vstr + (size_t)k * rstr + e] = from_d<C>(acc[q]);
    }
}

// out_l[k] = sum_{i < nin} P[k * pstr + i * ldp + l] V_i[k] for l < nout, in
// 16-byte packs: one pack per thread and NB outputs per CTA row, the
// coefficients of the CTA's outputs in shared memory (read as broadcasts),
// the loads of four inputs issued before their products.  Used by the
// deflated restart (NB = 8) and the cycle correction (NB = 1); lengths and
// strides in packs.
template <typename C, int NB>
__global__ void __launch_bounds__(kGsThreads) k_lincomb_pack(long long np, int nin, int nout,
                                                             const typename Pack<C>::T *__restrict__ V, size_t vstr,
                                                             size_t rstr, const double2 *__restrict__ P, int ldp,
                                                             size_t pstr, typename Pack<C>::T *__restrict__ out) {
    using PK = Pack<C>;
    using PT = typename PK::T;
    constexpr int E = PK::E;
    pdl_wait();
    extern __shared__ double2 cs[];   // [nin][NB]
    const int k = blockIdx.z, l0 = blockIdx.y * NB;
    const int nb = min(NB, nout - l0);
    for (int t = threadIdx.x; t < nin * NB; t += blockDim.x) {
        const int i = t / NB, q = t % NB;
        cs[t] = q < nb ? P[(size_t)k * pstr + (size_t)i * ldp + l0 + q] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    const PT *Vk = V + (size_t)k * rstr;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < np; p += (long long)gridDim.x * blockDim.x) {
        double2 acc[E][NB];
#pragma unroll
        for (int e = 0; e < E; ++e)
#pragma unroll
            for (int q = 0; q < NB; ++q) acc[e][q] = make_double2(0.0, 0.0);
        int i = 0;
        for (; i + 4 <= nin; i += 4) {
            PT b[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) b[u] = __ldg(Vk + (size_t)(i + u) * vstr + p);
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const double2 bd = PK::get(b[u], e);
#pragma unroll
                    for (int q = 0; q < NB; ++q) {
                        const double2 c = cs[(i + u) * NB + q];
                        acc[e][q].x += c.x * bd.x - c.y * bd.y;
                        acc[e][q].y += c.x * bd.y + c.y * bd.x;
                    }
                }
        }
        for (; i < nin; ++i) {
            const PT b = __ldg(Vk + (size_t)i * vstr + p);
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const double2 bd = PK::get(b, e);
#pragma unroll
                for (int q = 0; q < NB; ++q) {
                    const double2 c = cs[i * NB + q];
                    acc[e][q].x += c.x * bd.x - c.y * bd.y;
                    acc[e][q].y += c.x * bd.y + c.y * bd.x;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < NB; ++q)
            if (q < nb) {
                double2 d[E];
#pragma unroll
                for (int e = 0; e < E; ++e) d[e] = acc[e][q];
                out[(size_t)(l0 + q) * vstr + (size_t)k * rstr + p] = PK::make(d);
            }
    }
}

// u += x
template <typename C>
__global__ void __launch_bounds__(kGsThreads) k_axpy_c(long long n, const C *__restrict__ x, C *__restrict__ u) {
    pdl_wait();
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
        u[e] = u[e] + x[e];
}

// ----------------------------------------------------------------------------
// workspace
// ----------------------------------------------------------------------------
template <typename C> size_t GmresWork<C>::bytes() const {
    const size_t vec = sizeof(C) * (size_t)n * nrhs;
    return vec * (2 * (restart + 1) + 3) +
           sizeof(double2) * ((size_t)kGsBlocks * nrhs * (restart + 1) + 3 * (size_t)nrhs * (restart + 1) +
                              (size_t)nrhs * (restart + 1) * (deflate + 1 + kMaxAug)) +
           sizeof(double) * 2 * nrhs;
}

template <typename C> tdda_status GmresWork<C>::init(long long n3, int nrhs_, int restart_, int degree_, int deflate_) {
    release();
    n = n3; nrhs = nrhs_; restart = restart_; degree = degree_; deflate = deflate_;
    // the opt-in dynamic shared memory limit is a per-function attribute
    TDDA_CUDA_TRY(cudaFuncSetAttribute(k_multidot_bulk<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBdSmem));
    const size_t vec = (size_t)n * nrhs;
    C **bufs[] = {&W, &Y, &U};
    for (C **b : bufs) TDDA_CUDA_TRY(cudaMalloc(b, sizeof(C) * vec));
    TDDA_CUDA_TRY(cudaMalloc(&V, sizeof(C) * vec * (restart + 1)));
    if (deflate > 0) TDDA_CUDA_TRY(cudaMalloc(&V2, sizeof(C) * vec * (restart + 1)));
    // cells without a dipole must read as zero in every vector
    TDDA_CUDA_TRY(cudaMemset(V, 0, sizeof(C) * vec * (restart + 1)));
    if (V2) TDDA_CUDA_TRY(cudaMemset(V2, 0, sizeof(C) * vec * (restart + 1)));
    for (C **b : bufs) TDDA_CUDA_TRY(cudaMemset(*b, 0, sizeof(C) * vec));
    TDDA_CUDA_TRY(cudaMalloc(&part, sizeof(double2) * (size_t)kGsBlocks * nrhs * (restart + 1)));
    TDDA_CUDA_TRY(cudaMalloc(&h, sizeof(double2) * 2 * (size_t)nrhs * (restart + 1)));
    TDDA_CUDA_TRY(cudaMalloc(&coef, sizeof(double2) * (size_t)nrhs * (restart + 1)));
    TDDA_CUDA_TRY(cudaMalloc(&P, sizeof(double2) * (size_t)nrhs * (restart + 1) * (deflate + 1 + kMaxAug)));
    TDDA_CUDA_TRY(cudaMalloc(&nrm, sizeof(double) * 2 * nrhs));
    TDDA_CUDA_TRY(cudaMallocHost(&h_host, sizeof(double2) * (2 * (size_t)nrhs * (restart + 1) + nrhs)));
    TDDA_CUDA_TRY(cudaMallocHost(&c_host, sizeof(double2) * (size_t)nrhs * (restart + 1)));
    return TDDA_OK;
}

template <typename C> void GmresWork<C>::release() {
    cudaFree(V); cudaFree(V2); cudaFree(U); cudaFree(W); cudaFree(Y);
    cudaFree(part); cudaFree(h); cudaFree(coef); cudaFree(P); cudaFree(nrm);
    cudaFreeHost(h_host);
    cudaFreeHost(c_host);
    V = V2 = U = W = Y = nullptr;
    part = h = coef = P = nullptr;
    nrm = nullptr;
    h_host = c_host = nullptr;
    nrhs = 0;
}

// ----------------------------------------------------------------------------
// host linear algebra of the polynomial
// ----------------------------------------------------------------------------
bool hessenberg_eigenvalues(cplx *H, int n, int ld, std::vector<cplx> &ev) {
    auto h = [&](int i, int j) -> cplx & { return H[i + (size_t)j * ld]; };
    ev.assign(n, cplx(0.0, 0.0));
    int hi = n - 1, iter = 0;
    while (hi >= 0) {
        if (hi == 0) { ev[0] = h(0, 0); break; }
        int lo = hi;
        while (lo > 0) {
            double s = std::abs(h(lo - 1, lo - 1)) + std::abs(h(lo, lo));
            if (s == 0.0) s = 1.0;
            if (std::abs(h(lo, lo - 1)) <= 1e-15 * s) { h(lo, lo - 1) = 0.0; break; }
            --lo;
        }
        if (lo == hi) { ev[hi] = h(hi, hi); --hi; iter = 0; continue; }
        if (++iter > 60 * (hi - lo + 1)) return false;
        // Wilkinson shift: the eigenvalue of the trailing 2x2 block nearer h(hi, hi)
        const cplx a = h(hi - 1, hi - 1), b = h(hi - 1, hi), c = h(hi, hi - 1), d = h(hi, hi);
        const cplx tr = a + d, det = a * d - b * c;
        const cplx disc = std::sqrt(tr * tr / 4.0 - det);
        const cplx l1 = tr / 2.0 + disc, l2 = tr / 2.0 - disc;
        cplx mu = (std::abs(l1 - d) < std::abs(l2 - d)) ? l1 : l2;
        if (iter % 11 == 10) mu = d + cplx(std::abs(c), 0.0);  // exceptional shift
        // H - mu I = Q R by Givens rotations, then H <- R Q + mu I on the active block
        for (int k = lo; k <= hi; ++k) h(k, k) -= mu;
        std::vector<cplx> cs(hi - lo), sn(hi - lo);
        for (int k = lo; k < hi; ++k) {
            const cplx x = h(k, k), y = h(k + 1, k);
            const double r = std::sqrt(std::norm(x) + std::norm(y));
            const cplx cc = r == 0.0 ? cplx(1.0) : x / r, ss = r == 0.0 ? cplx(0.0) : y / r;
            cs[k - lo] = cc;
            sn[k - lo] = ss;
            for (int j = k; j < n; ++j) {
                const cplx u = h(k, j), v = h(k + 1, j);
                h(k, j) = std::conj(cc) * u + std::conj(ss) * v;
                h(k + 1, j) = -ss * u + cc * v;
            }
        }
        for (int k = lo; k < hi; ++k) {
            const cplx cc = cs[k - lo], ss = sn[k - lo];
            for (int i = 0; i <= std::min(k + 2, hi); ++i) {
                const cplx u = h(i, k), v = h(i, k + 1);
                h(i, k) = u * cc + v * ss;
                h(i, k + 1) = -u * std::conj(ss) + v * std::conj(cc);
            }
        }
        for (int k = lo; k <= hi; ++k) h(k, k) += mu;
    }
    return true;
}

// Dense n x n solve by Gaussian elimination with partial pivoting
// (column-major, ld; A and b destroyed).
static bool dense_solve(cplx *A, int n, int ld, cplx *b) {
    auto a = [&](int i, int j) -> cplx & { return A[i + (size_t)j * ld]; };
    for (int k = 0; k < n; ++k) {
        int p = k;
        for (int i = k + 1; i < n; ++i)
            if (std::abs(a(i, k)) > std::abs(a(p, k))) p = i;
        if (a(p, k) == cplx(0.0)) return false;
        if (p != k) {
            for (int j = 0; j < n; ++j) std::swap(a(k, j), a(p, j));
            std::swap(b[k], b[p]);
        }
        for (int i = k + 1; i < n; ++i) {
            const cplx f = a(i, k) / a(k, k);
            if (f == cplx(0.0)) continue;
            for (int j = k; j < n; ++j) a(i, j) -= f * a(k, j);
            b[i] -= f * b[k];
        }
    }
    for (int i = n - 1; i >= 0; --i) {
        cplx s = b[i];
        for (int j = i + 1; j < n; ++j) s -= a(i, j) * b[j];
        b[i] = s / a(i, i);
    }
    return true;
}

bool harmonic_ritz(const cplx *Hbar, int d, int ld, std::vector<cplx> &theta) {
    // eigenvalues of H_d + |h_{d+1,d}|^2 f e_d^T with H_d^H f = e_d (still
    // upper Hessenberg: only the last column changes)
    std::vector<cplx> Ht((size_t)d * d), f(d, cplx(0.0)), M((size_t)d * d);
    for (int i = 0; i < d; ++i)
        for (int j = 0; j < d; ++j) Ht[i + (size_t)j * d] = std::conj(Hbar[j + (size_t)i * ld]);
    f[d - 1] = 1.0;
    if (!dense_solve(Ht.data(), d, d, f.data())) return false;
    const double h2 = std::norm(Hbar[d + (size_t)(d - 1) * ld]);
    for (int i = 0; i < d; ++i)
        for (int j = 0; j < d; ++j) M[i + (size_t)j * d] = (i <= j + 1) ? Hbar[i + (size_t)j * ld] : cplx(0.0);
    for (int i = 0; i < d; ++i) M[i + (size_t)(d - 1) * d] += h2 * f[i];
    return hessenberg_eigenvalues(M.data(), d, d, theta);
}

void leja_order(std::vector<cplx> &th) {
    const int d = (int)th.size();
    if (d == 0) return;
    std::vector<cplx> out;
    std::vector<char> used(d, 0);
    int k0 = 0;
    for (int i = 1; i < d; ++i)
        if (std::abs(th[i]) > std::abs(th[k0])) k0 = i;
    out.push_back(th[k0]);
    used[k0] = 1;
    std::vector<double> lp(d, 0.0);  // log of the product of distances to the roots taken
    for (int step = 1; step < d; ++step) {
        int best = -1;
        for (int i = 0; i < d; ++i) {
            if (used[i]) continue;
            lp[i] += std::log(std::abs(th[i] - out.back()) + 1e-300);
            if (best < 0 || lp[i] > lp[best]) best = i;
        }
        out.push_back(th[best]);
        used[best] = 1;
    }
    // a root whose other factors multiply to more than 1e4 at it gets one
    // extra copy per 14 decades beyond (the product form stays stable)
    std::vector<cplx> extra;
    for (int i = 0; i < d; ++i) {
        double pof = 0.0;
        for (int j = 0; j < d; ++j)
            if (j != i) pof += std::log10(std::abs(1.0 - out[i] / out[j]));
        if (pof > 4.0) {
            const int copies = (int)std::ceil((pof - 4.0) / 14.0);
            for (int c = 0; c < copies; ++c) extra.push_back(out[i]);
        }
    }
    out.insert(out.end(), extra.begin(), extra.end());
    th.swap(out);
}

// ----------------------------------------------------------------------------
// the solver
// ----------------------------------------------------------------------------
namespace {

unsigned gs_blocks(long long n) {
    return (unsigned)std::max<long long>(1, std::min<long long>((n + kGsThreads - 1) / kGsThreads, kGsBlocks));
}

// whether the basis and w[k] can be read in 16-byte packs
template <typename C> bool packed(const GmresWork<C> &gw, const void *w) {
    constexpr int E = Pack<C>::E;
    return gw.n % E == 0 && ((uintptr_t)gw.V & 15) == 0 && ((uintptr_t)w & 15) == 0;
}

template <typename C> C *basis(GmresWork<C> &gw, int i) { return gw.V + (size_t)i * gw.n * gw.nrhs; }

// h[k * (nv + 1) + i] = V_i[k]^H w[k] for i < nv and ||w[k]||^2 at i = nv (device)
template <typename C> void multidot(GmresWork<C> &gw, int nv, const C *w, double2 *h, cudaStream_t s) {
    using PT = typename Pack<C>::T;
    constexpr int E = Pack<C>::E;
    const size_t rstr = gw.n, vstr = (size_t)gw.n * gw.nrhs;
    const unsigned nch = (unsigned)std::max(1, (nv + kGsChunk - 1) / kGsChunk);
    unsigned nb;
    count_launches(2);
    if (packed(gw, w)) {
        // two CTAs per SM over all chunks and right-hand sides
        const long long np = gw.n / E;
        const long long ntiles = (np + kBdTile - 1) / kBdTile;
        nb = (unsigned)std::max<long long>(
            1, std::min<long long>({(2LL * 148) / ((long long)nch * gw.nrhs), ntiles, (long long)kGsBlocks}));
        launch_dep(k_multidot_bulk<C>, dim3(nb, nch, gw.nrhs), dim3(kGsThreads), kBdSmem, s, np, nv, nv + 1,
                   (const PT *)gw.V, vstr / E, rstr / E, (const PT *)w, gw.part);
    } else {
        nb = gs_blocks(gw.n);
        launch_dep(k_multidot_e<C>, dim3(nb, nch, gw.nrhs), dim3(kGsThreads), 0, s, gw.n, nv, nv + 1,
                   (const C *)gw.V, vstr, rstr, w, gw.part);
    }
    const int nout = gw.nrhs * (nv + 1);
    launch_dep(k_sum_parts, dim3((nout + 7) / 8), dim3(256), 0, s, nout, (int)nb, (const double2 *)gw.part, h,
               (double *)nullptr, (double *)nullptr);
}

// w[k] = (w[k] - V[0..nv)[k] c[k]) * c[k][nv].x (c: device, rows of nv + 1)
template <typename C> void gs_update_scale(GmresWork<C> &gw, int nv, const double2 *c, C *w, cudaStream_t s) {
    using PT = typename Pack<C>::T;
    constexpr int E = Pack<C>::E;
    const size_t rstr = gw.n, vstr = (size_t)gw.n * gw.nrhs;
    const size_t smem = sizeof(double2) * (nv + 1);
    count_launches(1);
    if (packed(gw, w)) {
        const long long np = gw.n / E;
        const unsigned nb = (unsigned)std::max<long long>(1, std::min<long long>((np + kGsThreads - 1) / kGsThreads,
                                                                                 148 * 16));
        launch_dep(k_gs_update_scale<C>, dim3(nb, 1, gw.nrhs), dim3(kGsThreads), smem, s, np, nv, (const PT *)gw.V,
                   vstr / E, rstr / E, c, (PT *)w);
    } else {
        launch_dep(k_gs_update_scale_e<C>, dim3(gs_blocks(gw.n), 1, gw.nrhs), dim3(kGsThreads), smem, s, gw.n, nv,
                   (const C *)gw.V, vstr, rstr, c, w);
    }
}

// w[k] -= V[0..nv)[k] h[k]; with norms: nrm[k] = ||w[k]||, nrm[nrhs + k] = 1 / nrm[k]
template <typename C>
void gs_update(GmresWork<C> &gw, int nv, const double2 *h, int hstr, C *w, bool norms, cudaStream_t s) {
    const size_t rstr = gw.n, vstr = (size_t)gw.n * gw.nrhs;
    const unsigned nb = gs_blocks(gw.n);
    count_launches(1);
    launch_dep(k_gs_update<C>, dim3(nb, 1, gw.nrhs), dim3(kGsThreads), sizeof(double2) * std::max(nv, 1), s, gw.n,
               nv, (const C *)gw.V, vstr, rstr, h, hstr, w, norms ? gw.part : (double2 *)nullptr);
    if (norms) {
        count_launches(1);
        launch_dep(k_sum_parts, dim3((gw.nrhs + 7) / 8), dim3(256), 0, s, gw.nrhs, (int)nb, (const double2 *)gw.part,
                   (double2 *)nullptr, gw.nrm, gw.nrm + gw.nrhs);
    }
}

// out_l[k] = sum_{i < nin} P[k * pstr + i * ldp + l] V_i[k], l < nout (device
// coefficients; out has the basis layout: vector l of right-hand side k at
// l * vstr + k * n)
template <typename C>
void lincomb(GmresWork<C> &gw, int nin, int nout, const C *V, const double2 *P, int ldp, size_t pstr, C *out,
             cudaStream_t s) {
    using PT = typename Pack<C>::T;
    constexpr int E = Pack<C>::E;
    const size_t vstr = (size_t)gw.n * gw.nrhs;
    count_launches(1);
    const bool pk = gw.n % E == 0 && ((uintptr_t)V & 15) == 0 && ((uintptr_t)out & 15) == 0;
    if (pk && nout == 1 && (size_t)nin * sizeof(double2) <= 48 * 1024) {
        const long long np = gw.n / E;
        launch_dep(k_lincomb_pack<C, 1>, dim3(gs_blocks(np), 1, gw.nrhs), dim3(kGsThreads),
                   sizeof(double2) * nin, s, np, nin, 1, (const PT *)V, vstr / E, (size_t)gw.n / E, P, ldp, pstr,
                   (PT *)out);
    } else if (pk && (size_t)nin * kGsChunk * sizeof(double2) <= 48 * 1024) {
        const long long np = gw.n / E;
        launch_dep(k_lincomb_pack<C, kGsChunk>, dim3(gs_blocks(np), (nout + kGsChunk - 1) / kGsChunk, gw.nrhs),
                   dim3(kGsThreads), sizeof(double2) * nin * kGsChunk, s, np, nin, nout, (const PT *)V, vstr / E,
                   (size_t)gw.n / E, P, ldp, pstr, (PT *)out);
    } else {
        launch_dep(k_lincomb_multi<C>, dim3(gs_blocks(gw.n), (nout + kGsChunk - 1) / kGsChunk, gw.nrhs),
                   dim3(kGsThreads), 0, s, gw.n, nin, nout, V, vstr, (size_t)gw.n, P, ldp, pstr, out);
    }
}

template <typename C> void scale_vec(GmresWork<C> &gw, const double *f, const C *x, C *out, cudaStream_t s) {
    count_launches(1);
    launch_dep(k_scale_vec<C>, dim3(gs_blocks(gw.n), 1, gw.nrhs), dim3(kGsThreads), 0, s, gw.n, (size_t)gw.n, f, x,
               out);
}

// Orthonormalises w (basis slot nv) against V[0..nv) with classical
// Gram-Schmidt: one pass for the projections and the norm of w, one pass for
// the update and the normalisation (the new norm by Pythagoras); when the
// update leaves less than sqrt(kReorth) of ||w|| a second projection pass runs ("twice is
// enough").  The coefficients of every right-hand side land in
// Hcol[k][0..nv) and the remaining norm in Hcol[k][nv].
template <typename C>
tdda_status orthonormalise(GmresWork<C> &gw, int nv, C *w, std::vector<std::vector<cplx>> &Hcol, cudaStream_t s) {
    const int nr = gw.nrhs;
    double2 *hh = gw.h_host;
    double2 *coef = gw.c_host;
    for (int k = 0; k < nr; ++k) Hcol[k].assign(nv + 1, cplx(0.0));
    bool final = false;
    for (int pass = 0; pass < 2 && !final; ++pass) {
        multidot(gw, nv, w, gw.h, s);
        TDDA_CUDA_TRY(cudaMemcpyAsync(hh, gw.h, sizeof(double2) * (size_t)nr * (nv + 1), cudaMemcpyDeviceToHost, s));
        TDDA_CUDA_TRY(cudaStreamSynchronize(s));
        TDDA_CUDA_TRY(cudaGetLastError());
        bool cancel = false;
        std::vector<double> wp2(nr);
        for (int k = 0; k < nr; ++k) {
            const double2 *hk = hh + (size_t)k * (nv + 1);
            double proj = 0.0;
            for (int i = 0; i < nv; ++i) {
                proj += hk[i].x * hk[i].x + hk[i].y * hk[i].y;
                Hcol[k][i] += cplx(hk[i].x, hk[i].y);
                coef[(size_t)k * (nv + 1) + i] = hk[i];
            }
            const double wn2 = hk[nv].x;
            if (!std::isfinite(wn2) || !std::isfinite(proj)) {
                set_error("GMRES: non-finite Gram-Schmidt sums (a non-finite operator result, or a device wait "
                          "in the projection kernel that gave up)");
                return TDDA_ERR_BREAKDOWN;
            }
            wp2[k] = wn2 - proj;
            if (wn2 > 0.0 && wp2[k] < kReorth * wn2) cancel = true;
        }
        final = !cancel || pass == 1;
        for (int k = 0; k < nr; ++k) {
            const double nrm = final ? std::sqrt(std::max(wp2[k], 0.0)) : 1.0;
            coef[(size_t)k * (nv + 1) + nv] = make_double2(final ? (nrm > 0.0 ? 1.0 / nrm : 0.0) : 1.0, 0.0);
            if (final) Hcol[k][nv] = cplx(nrm, 0.0);
        }
        TDDA_CUDA_TRY(cudaMemcpyAsync(gw.coef, coef, sizeof(double2) * (size_t)nr * (nv + 1), cudaMemcpyHostToDevice, s));
        gs_update_scale(gw, nv, (const double2 *)gw.coef, w, s);
    }
    return TDDA_OK;
}

// One Arnoldi step on operator `op_fn`: w = op(V[j]) lands in V[j + 1 + aug]
// and is orthonormalised against V[0..j + 1 + aug).  aug = 1 in the first
// cycle of an inner solve that starts from a recycled space: there the new
// right-hand side's direction sits in slot kd + 1, one ahead of the Arnoldi
// sequence, so every column has two entries below its diagonal.  The column
// of every right-hand side lands in Hcol[k][0..j + 1 + aug].
template <typename C, class OpFn>
tdda_status arnoldi_step(GmresWork<C> &gw, int j, OpFn op_fn, std::vector<std::vector<cplx>> &Hcol, cudaStream_t s,
                         int aug = 0) {
    C *w = basis(gw, j + 1 + aug);
    tdda_status st = op_fn(basis(gw, j), w);
    if (st != TDDA_OK) return st;
    return orthonormalise(gw, j + 1 + aug, w, Hcol, s);
}

// Least-squares state of one right-hand side: the projected matrix Hbar
// ((m+1) x m, column-major; after a deflated restart its leading block is
// dense), its QR by Givens rotations between arbitrary row pairs, and the
// rotated right-hand side g.
struct LsqState {
    int m = 0;
    std::vector<cplx> H, R, g, c0;   // H, R: (m+1) x m; g, c0: m+1
    struct Rot { int i, l; cplx c, s; };
    std::vector<Rot> rots;
    void reset(int m_) {
        m = m_;
        H.assign((size_t)(m + 1) * m, cplx(0.0));
        R = H;
        g.assign(m + 1, cplx(0.0));
        c0 = g;
        rots.clear();
    }
    cplx &h(int i, int j) { return H[i + (size_t)j * (m + 1)]; }
    cplx &r(int i, int j) { return R[i + (size_t)j * (m + 1)]; }
    // starts from the coefficient vector c of the residual in the basis
    void start(const std::vector<cplx> &c) {
        std::fill(g.begin(), g.end(), cplx(0.0));
        for (size_t i = 0; i < c.size(); ++i) g[i] = c[i];
        c0 = g;
        rots.clear();
    }
    // column j of H is set (rows 0..m): rotate it into R; returns the
    // residual estimate ||g[j+1..m]||
    double add(int j) {
        cplx *col = &R[(size_t)j * (m + 1)];
        for (int i = 0; i <= m; ++i) col[i] = H[i + (size_t)j * (m + 1)];
        for (const Rot &q : rots) {
            const cplx a = col[q.i], b = col[q.l];
            col[q.i] = q.c * a + q.s * b;
            col[q.l] = -std::conj(q.s) * a + std::conj(q.c) * b;
        }
        for (int l = m; l > j; --l) {
            if (col[l] == cplx(0.0)) continue;
            const cplx a = col[j], b = col[l];
            const double den = std::sqrt(std::norm(a) + std::norm(b));
            Rot q{j, l, std::conj(a) / den, std::conj(b) / den};
            col[j] = den;
            col[l] = 0.0;
            const cplx ga = g[j], gb = g[l];
            g[j] = q.c * ga + q.s * gb;
            g[l] = -std::conj(q.s) * ga + std::conj(q.c) * gb;
            rots.push_back(q);
        }
        double e = 0.0;
        for (int i = j + 1; i <= m; ++i) e += std::norm(g[i]);
        return std::sqrt(e);
    }
    // least-squares solution over the first k columns
    void solve(int k, std::vector<cplx> &y) const {
        y.assign(k, cplx(0.0));
        for (int i = k - 1; i >= 0; --i) {
            cplx t = g[i];
            for (int l = i + 1; l < k; ++l) t -= R[i + (size_t)l * (m + 1)] * y[l];
            const cplx d = R[i + (size_t)i * (m + 1)];
            y[i] = d == cplx(0.0) ? cplx(0.0) : t / d;
        }
    }
};

// The deflated restart of GMRES-DR: from Hbar (jc columns used, rows jc + 1,
// or jc + 2 after a cycle that started from a recycled space; the rest of the
// (m+1) x m storage is zero), the least-squares solution y and the start
// coefficients c0, the orthonormal combination P ((m+1) x nc, column-major,
// ld m+1) whose first kept columns span the kept harmonic Ritz vectors of
// smallest magnitude and whose other rows - jc columns span the complement of
// range(Hbar), the residual's direction first; the new projected matrix
// P^H Hbar P[:m, :kept] (nc x kept) and the new start coefficients P^H rho.
// Returns kept (<= kd); with kept = 0 (no vector asked for, or the
// eigenproblem failed) P is the residual's direction alone: a plain restart.
int deflated_restart(LsqState &L, int kd, const std::vector<cplx> &y, std::vector<cplx> &P,
                     std::vector<cplx> &Hn, std::vector<cplx> &cn, int jc, int rows) {
    const int m = L.m, ld = m + 1;
    // residual coefficients rho = c0 - Hbar y
    std::vector<cplx> rho(L.c0);
    for (int j = 0; j < m; ++j)
        for (int i = 0; i <= m; ++i) rho[i] -= L.h(i, j) * y[j];
    std::vector<std::vector<cplx>> cols;
    if (kd > 0 && jc > 0) {
        // harmonic Ritz pairs of span(V_jc): Hbar^H Hbar g = theta T^H g with
        // T the top jc x jc block and B the rows below it, i.e.
        // (T + T^-H B^H B) g = theta g  (B = h e_jc^T after a plain Arnoldi
        // cycle: the usual rank-one update of the last column)
        DenseMat Ht(jc), M(jc);
        for (int i = 0; i < jc; ++i)
            for (int j = 0; j < jc; ++j) {
                Ht(i, j) = std::conj(L.h(j, i));
                M(i, j) = L.h(i, j);
            }
        bool ok = true;
        for (int b = jc; b < rows && ok; ++b) {
            // f = T^-H conj(B row b); M += f B row b
            std::vector<cplx> f(jc);
            for (int i = 0; i < jc; ++i) f[i] = std::conj(L.h(b, i));
            DenseMat Hw = Ht;
            ok = dense_solve(Hw.a.data(), jc, jc, f.data());
            if (ok)
                for (int j = 0; j < jc; ++j) {
                    const cplx bj = L.h(b, j);
                    if (bj == cplx(0.0)) continue;
                    for (int i = 0; i < jc; ++i) M(i, j) += f[i] * bj;
                }
        }
        if (ok) {
            std::vector<cplx> ev;
            ok = eigenpairs_few(M, ev, cols, [&](const std::vector<cplx> &e) {
                std::vector<int> id(e.size());
                for (size_t i = 0; i < e.size(); ++i) id[i] = (int)i;
                std::sort(id.begin(), id.end(), [&](int a, int b) { return std::abs(e[a]) < std::abs(e[b]); });
                id.resize(std::min<size_t>(kd, id.size()));
                return id;
            });
        }
        if (!ok) cols.clear();
    }
    // orthonormalise (twice), dropping dependent vectors; then the residual
    std::vector<std::vector<cplx>> Q;
    auto orth = [&](std::vector<cplx> v) -> bool {
        double n0 = 0.0;
        for (auto &e : v) n0 += std::norm(e);
        n0 = std::sqrt(n0);
        if (!(n0 > 0.0)) return false;
        for (int pass = 0; pass < 2; ++pass)
            for (auto &q : Q) {
                cplx d = 0.0;
                for (int i = 0; i <= m; ++i) d += std::conj(q[i]) * v[i];
                for (int i = 0; i <= m; ++i) v[i] -= d * q[i];
            }
        double n1 = 0.0;
        for (auto &e : v) n1 += std::norm(e);
        n1 = std::sqrt(n1);
        if (!(n1 > 1e-8 * n0)) return false;
        for (auto &e : v) e /= n1;
        Q.push_back(v);
        return true;
    };
    for (auto &c : cols) {
        std::vector<cplx> v(m + 1, cplx(0.0));
        for (int i = 0; i < jc; ++i) v[i] = c[i];
        orth(v);
    }
    const int kept = (int)Q.size();
    if (!orth(rho) || kept == 0) {
        // no deflation vector, or the residual lies in the deflation space:
        // a plain restart from the residual's direction
        Q.clear();
        Q.push_back(rho);
        double nr = 0.0;
        for (auto &e : Q[0]) nr += std::norm(e);
        nr = std::sqrt(nr);
        for (auto &e : Q[0]) e = nr > 0 ? e / nr : cplx(0.0);
        P.assign(ld, cplx(0.0));
        for (int i = 0; i <= m; ++i) P[i] = Q[0][i];
        Hn.clear();
        cn.assign(1, cplx(nr, 0.0));
        return 0;
    }
    // Hbar g - theta [g; 0] lies in the complement of range(Hbar), which has
    // rows - jc dimensions; the residual spans it after a plain Arnoldi cycle.
    // Otherwise the rest of the complement joins the new basis, so that
    // Ah V P[:, :kept] stays inside span(V P).
    const int ext = rows - jc;
    if (ext > 1) {
        std::vector<std::vector<cplx>> Rg;  // orthonormal basis of range(Hbar)
        for (int j = 0; j < jc; ++j) {
            std::vector<cplx> v(m + 1, cplx(0.0));
            for (int i = 0; i < rows; ++i) v[i] = L.h(i, j);
            for (int pass = 0; pass < 2; ++pass)
                for (auto &q : Rg) {
                    cplx d = 0.0;
                    for (int i = 0; i <= m; ++i) d += std::conj(q[i]) * v[i];
                    for (int i = 0; i <= m; ++i) v[i] -= d * q[i];
                }
            double nv = 0.0;
            for (auto &e : v) nv += std::norm(e);
            nv = std::sqrt(nv);
            if (!(nv > 0.0)) continue;
            for (auto &e : v) e /= nv;
            Rg.push_back(v);
        }
        // the unit vector whose complement part, with what P holds removed,
        // is largest, until the complement is covered
        for (int add = 1; add < ext; ++add) {
            std::vector<cplx> best;
            double bn = 0.0;
            for (int a = 0; a < rows; ++a) {
                std::vector<cplx> v(m + 1, cplx(0.0));
                v[a] = 1.0;
                for (int pass = 0; pass < 2; ++pass) {
                    for (auto &q : Rg) {
                        cplx d = std::conj(q[a]);
                        if (pass == 1) {
                            d = 0.0;
                            for (int i = 0; i <= m; ++i) d += std::conj(q[i]) * v[i];
                        }
                        for (int i = 0; i <= m; ++i) v[i] -= d * q[i];
                    }
                    for (auto &q : Q) {
                        cplx d = 0.0;
                        for (int i = 0; i <= m; ++i) d += std::conj(q[i]) * v[i];
                        for (int i = 0; i <= m; ++i) v[i] -= d * q[i];
                    }
                }
                double nv = 0.0;
                for (auto &e : v) nv += std::norm(e);
                if (nv > bn) { bn = nv; best = v; }
            }
            if (!(bn > 1e-12) || !orth(best)) {
                // the complement is not resolved: a plain restart
                return deflated_restart(L, 0, y, P, Hn, cn, jc, rows);
            }
        }
    }
    const int nc = (int)Q.size();
    P.assign((size_t)ld * nc, cplx(0.0));
    for (int c = 0; c < nc; ++c)
        for (int i = 0; i <= m; ++i) P[i + (size_t)c * ld] = Q[c][i];
    // Hn = P^H Hbar P[:m, :kept]  (nc x kept)
    std::vector<cplx> HP((size_t)ld * kept, cplx(0.0));
    for (int c = 0; c < kept; ++c)
        for (int j = 0; j < m; ++j) {
            const cplx pj = P[j + (size_t)c * ld];
            if (pj == cplx(0.0)) continue;
            for (int i = 0; i <= m; ++i) HP[i + (size_t)c * ld] += L.h(i, j) * pj;
        }
    Hn.assign((size_t)nc * kept, cplx(0.0));
    for (int c = 0; c < kept; ++c)
        for (int r = 0; r < nc; ++r) {
            cplx s = 0.0;
            for (int i = 0; i <= m; ++i) s += std::conj(P[i + (size_t)r * ld]) * HP[i + (size_t)c * ld];
            Hn[r + (size_t)c * nc] = s;
        }
    cn.assign(nc, cplx(0.0));
    for (int r = 0; r < nc; ++r) {
        cplx s = 0.0;
        for (int i = 0; i <= m; ++i) s += std::conj(P[i + (size_t)r * ld]) * rho[i];
        cn[r] = s;
    }
    return kept;
}

}  // namespace

template <typename C>
tdda_status pgmres_solve(const RefineWork<C> &w, GmresWork<C> &gw, const double2 *B, double2 *X, int nrhs,
                         bool x0_zero, int max_iter, double tol, const GmresOptions &o, tdda_solve_info *info) {
    const long long n = 3 * w.nbox;
    cudaStream_t s = w.s;
    if (gw.nrhs != nrhs || gw.n != n || gw.restart != o.restart || gw.degree != o.degree || gw.deflate != o.deflate) {
        set_error("GMRES workspace does not match the solve");
        return TDDA_ERR_STATE;
    }
    if (o.deflate >= o.restart) {
        set_error("GMRES: the deflation vectors must be fewer than the restart length");
        return TDDA_ERR_BAD_ARG;
    }
    if (x0_zero) TDDA_CUDA_TRY(cudaMemsetAsync(X, 0, sizeof(double2) * n * nrhs, s));
    const int m = o.restart, d = o.degree, ld = m + 1;
    std::vector<int> done(nrhs, 0), refines(nrhs, 0), steps(nrhs, 0), status(nrhs, TDDA_SOLVE_RUNNING), slow(nrhs, 0);
    std::vector<long long> mv(nrhs, 0);
    std::vector<double> err(nrhs, 0.0), prev(nrhs, 1e300);
    std::vector<cplx> roots;
    std::vector<std::vector<cplx>> Hcol(nrhs);
    std::vector<LsqState> L(nrhs);
    // the space carried from one inner solve to the next (o.recycle): slots
    // 0..kr + ar of V, with Ah V[:, :kr] = V[:, :kr + ar + 1] Hr[k]
    int kr = 0, ar = 0;
    std::vector<std::vector<cplx>> Hr(nrhs);
    double *h = w.h_part;
    // the inner operator, and the inner operator times the polynomial
    auto op_plain = [&](const C *x, C *y) { return apply_scaled<C>(*w.op, w.sc, w.al, x, y, nrhs, w.dstride, s); };
    auto op_poly = [&](const C *v, C *out) -> tdda_status {
        // out = v - prod(1 - Ah / theta_i) v  =  Ah p(Ah) v
        const int nr = (int)roots.size();
        for (int i = 0; i < nr; ++i) {
            const cplx c = 1.0 / roots[i];
            const C *rin = i == 0 ? v : gw.W;
            const bool last = i == nr - 1;
            tdda_status st = poly_factor<C>(*w.op, w.sc, w.al, rin, gw.W, nullptr, false, last ? v : nullptr,
                                            last ? out : nullptr, make_double2(c.real(), c.imag()), nrhs, w.dstride, s);
            if (st != TDDA_OK) return st;
        }
        return TDDA_OK;
    };
    const size_t vstr = (size_t)n * nrhs;
    const int max_refine = 60;
    for (int outer = 0; outer <= max_refine; ++outer) {
        tdda_status st = residual_c128(*w.op64, w.al64, B, X, w.Rm, w.st_res, nrhs, s, w.dstride,
                                        w.post.eres != nullptr ? &w.post : nullptr);
        if (st != TDDA_OK) return st;
        TDDA_CUDA_TRY(cudaMemcpyAsync(w.st_res_host, w.st_res, sizeof(SolverState) * nrhs, cudaMemcpyDeviceToHost, s));
        TDDA_CUDA_TRY(cudaStreamSynchronize(s));
        bool all = true;
        for (int k = 0; k < nrhs; ++k) {
            if (done[k]) continue;
            const SolverState &S = w.st_res_host[k];
            err[k] = S.err;
            if (S.enorm == 0.0) {
                TDDA_CUDA_TRY(cudaMemsetAsync(X + (size_t)k * n, 0, sizeof(double2) * n, s));
                done[k] = 1; status[k] = TDDA_SOLVE_ZERO_RHS; err[k] = 0.0;
            } else if (S.err <= tol) {
                done[k] = 1; status[k] = TDDA_SOLVE_CONVERGED;
            } else if (!std::isfinite(S.err)) {
                done[k] = 1; status[k] = TDDA_SOLVE_NONFINITE;
            } else if (mv[k] >= max_iter || outer == max_refine) {
                done[k] = 1; status[k] = TDDA_SOLVE_MAXITER;
            } else {
                // two refinements in a row that do not halve the true residual: stagnated
                slow[k] = (S.err > 0.5 * prev[k]) ? slow[k] + 1 : 0;
                if (slow[k] >= 2) { done[k] = 1; status[k] = TDDA_SOLVE_STAGNATED; }
            }
            prev[k] = S.err;
            all &= (done[k] != 0);
        }
        if (all) break;
        // inner right-hand sides R^ = S R / ||R|| (finished ones: zero)
        std::fill(h, h + 3 * (size_t)nrhs, 0.0);
        for (int k = 0; k < nrhs; ++k) {
            if (done[k]) continue;
            const SolverState &S = w.st_res_host[k];
            const double rn = S.err * S.enorm;
            h[k] = 1.0 / rn;
            h[nrhs + k] = rn;
            h[2 * nrhs + k] = std::max(0.5 * tol / S.err, o.floor);  // reduction this inner solve must reach
        }
        TDDA_CUDA_TRY(cudaMemcpyAsync(w.d_part, h, sizeof(double) * 3 * nrhs, cudaMemcpyHostToDevice, s));
        launch_to_inner<C>(n, w.nbox, nrhs, w.dstride, w.Rm, w.d_part, w.sc64, w.R, s);
        std::vector<double> beta(nrhs);
        // structure of the first cycle: aug extra directions below the
        // Arnoldi sequence (0: plain GMRES(-DR) from R^)
        int aug = 0;
        if (kr > 0) {
            // start from the recycled space: slots 0..kr + ar hold V_s with
            // Ah V_s[:, :kr] = V_s Hr; R^ joins as slot kr + ar + 1
            aug = ar + 1;
            C *w0 = basis(gw, kr + aug);
            TDDA_CUDA_TRY(cudaMemcpyAsync(w0, w.R, sizeof(C) * vstr, cudaMemcpyDeviceToDevice, s));
            st = orthonormalise(gw, kr + aug, w0, Hcol, s);
            if (st != TDDA_OK) return st;
            for (int k = 0; k < nrhs; ++k) {
                double b2 = 0.0;
                for (const cplx &c : Hcol[k]) b2 += std::norm(c);
                beta[k] = std::sqrt(b2);
            }
        } else {
            // V[0] = R^ / ||R^||
            gs_update(gw, 0, gw.h, 0, w.R, true, s);  // norms only
            scale_vec(gw, gw.nrm + nrhs, w.R, basis(gw, 0), s);
            TDDA_CUDA_TRY(cudaMemcpyAsync(gw.h_host, gw.nrm, sizeof(double) * nrhs, cudaMemcpyDeviceToHost, s));
            TDDA_CUDA_TRY(cudaStreamSynchronize(s));
            for (int k = 0; k < nrhs; ++k) beta[k] = reinterpret_cast<const double *>(gw.h_host)[k];
        }
        TDDA_CUDA_TRY(cudaMemsetAsync(gw.U, 0, sizeof(C) * vstr, s));
        if (roots.empty()) {
            // the polynomial: Arnoldi steps of the inner operator on the first
            // residual of the first unfinished right-hand side
            int k0 = 0;
            while (k0 < nrhs && done[k0]) ++k0;
            const int dd = std::min(d, m);
            std::vector<cplx> Hb((size_t)(dd + 1) * dd, cplx(0.0));
            int got = dd;
            for (int j = 0; j < dd; ++j) {
                st = arnoldi_step(gw, j, op_plain, Hcol, s);
                if (st != TDDA_OK) return st;
                for (int i = 0; i <= j + 1; ++i) Hb[i + (size_t)j * (dd + 1)] = Hcol[k0][i];
                for (int k = 0; k < nrhs; ++k) mv[k] += 1;
                if (std::abs(Hcol[k0][j + 1]) <= 1e-14 * std::abs(Hcol[k0][j])) { got = j + 1; break; }
            }
            std::vector<cplx> th, Hg((size_t)(got + 1) * got);
            for (int j = 0; j < got; ++j)
                for (int i = 0; i <= got; ++i) Hg[i + (size_t)j * (got + 1)] = Hb[i + (size_t)j * (dd + 1)];
            if (!harmonic_ritz(Hg.data(), got, got + 1, th)) {
                set_error("polynomial preconditioner: harmonic Ritz values did not converge");
                return TDDA_ERR_BREAKDOWN;
            }
            for (auto &t : th)
                if (std::abs(t) == 0.0 || !std::isfinite(t.real()) || !std::isfinite(t.imag())) {
                    set_error("polynomial preconditioner: a harmonic Ritz value is zero or not finite");
                    return TDDA_ERR_BREAKDOWN;
                }
            leja_order(th);
            roots = th;
            // V[0] is unchanged by those steps; the cycles overwrite V[1..]
        }
        // the inner solve: (deflated) restarted GMRES cycles on Ah p(Ah)
        int kd = 0;                      // deflation vectors at the start of this cycle
        for (int k = 0; k < nrhs; ++k) {
            L[k].reset(m);
            if (kr > 0) {
                const int nc = kr + aug;   // rows of Hr: the recycled slots
                for (int c = 0; c < kr; ++c)
                    for (int r = 0; r < nc; ++r) L[k].h(r, c) = Hr[k][r + (size_t)c * nc];
                L[k].start(Hcol[k]);
            } else {
                L[k].start({cplx(beta[k], 0.0)});
            }
        }
        if (kr > 0) kd = kr;
        kr = 0;                          // the recycled space is used up
        std::vector<double> cyc_prev(beta);
        std::vector<int> inner_slow(nrhs, 0), inner_done(nrhs, 0), last_cycle(nrhs, -1);
        for (int k = 0; k < nrhs; ++k) inner_done[k] = done[k];
        for (int cycle = 0;; ++cycle) {
            int jc = kd;                 // columns of Hbar filled
            for (int k = 0; k < nrhs; ++k)
                if (!inner_done[k])
                    for (int j = 0; j < kd; ++j) L[k].add(j);
            bool reached = false;
            for (int j = kd; j < m - aug; ++j) {
                st = arnoldi_step(gw, j, op_poly, Hcol, s, aug);
                if (st != TDDA_OK) return st;
                jc = j + 1;
                reached = true;
                for (int k = 0; k < nrhs; ++k) {
                    if (inner_done[k]) continue;
                    for (int i = 0; i <= j + 1 + aug; ++i) L[k].h(i, j) = Hcol[k][i];
                    const double est = L[k].add(j);
                    mv[k] += (long long)roots.size();
                    steps[k] += 1;
                    if (!(est <= h[2 * nrhs + k] * beta[k]) && mv[k] < max_iter) reached = false;
                }
                if (reached) break;
            }
            const int rows = jc + 1 + aug;
            // u += V y over the jc columns
            std::vector<double2> coef((size_t)nrhs * jc, make_double2(0.0, 0.0));
            std::vector<std::vector<cplx>> ys(nrhs);
            bool all_in = true;
            for (int k = 0; k < nrhs; ++k) {
                if (inner_done[k]) continue;
                L[k].solve(jc, ys[k]);
                for (int i = 0; i < jc; ++i) coef[(size_t)k * jc + i] = make_double2(ys[k][i].real(), ys[k][i].imag());
                double est = 0.0;
                for (int i = jc; i <= m; ++i) est += std::norm(L[k].g[i]);
                est = std::sqrt(est);
                // twelve cycles in a row that each gain less than 0.5%: the inner
                // solve has given what it can; the refinement takes over
                inner_slow[k] = (est > 0.995 * cyc_prev[k]) ? inner_slow[k] + 1 : 0;
                cyc_prev[k] = est;
                if (est <= h[2 * nrhs + k] * beta[k] || mv[k] >= max_iter || inner_slow[k] >= 12) {
                    inner_done[k] = 1;
                    last_cycle[k] = cycle;
                }
                all_in &= (inner_done[k] != 0);
            }
            TDDA_CUDA_TRY(cudaMemcpyAsync(gw.coef, coef.data(), sizeof(double2) * coef.size(), cudaMemcpyHostToDevice, s));
            lincomb(gw, jc, 1, (const C *)gw.V, (const double2 *)gw.coef, 1, (size_t)jc, gw.W, s);
            // U += W (the combination lands in W first: k_lincomb overwrites)
            count_launches(1);
            launch_dep(k_axpy_c<C>, dim3(gs_blocks(n * nrhs)), dim3(kGsThreads), 0, s, n * nrhs, (const C *)gw.W, gw.U);
            // the deflated restart, or (recycling, once the inner solve ends
            // with every right-hand side of this step finishing in this cycle)
            // the space the next refinement step starts from
            bool save = false;
            if (all_in) {
                // (room for the carried space plus two Arnoldi steps per cycle)
                save = o.recycle && o.deflate > 0 && aug < kMaxAug && o.deflate + kMaxAug + 2 <= m;
                for (int k = 0; k < nrhs; ++k)
                    if (!done[k] && last_cycle[k] != cycle) save = false;
                if (!save) break;
            } else if (cycle > 100000) {
                break;
            }
            std::vector<std::vector<cplx>> Ps(nrhs), Hns(nrhs), cns(nrhs);
            auto restart_k = [&](int k, int want) {
                std::vector<cplx> yfull(m, cplx(0.0));
                for (int i = 0; i < jc; ++i) yfull[i] = ys[k][i];
                return deflated_restart(L[k], want, yfull, Ps[k], Hns[k], cns[k], jc, rows);
            };
            auto active = [&](int k) { return save ? !done[k] : !inner_done[k]; };
            int kept = o.deflate;
            for (int k = 0; k < nrhs; ++k)
                if (active(k)) kept = std::min(kept, restart_k(k, o.deflate));
            // every right-hand side keeps the same number of vectors
            for (int k = 0; k < nrhs; ++k) {
                if (!active(k)) continue;
                const int have = Hns[k].empty() ? 0 : (int)(Hns[k].size() / (Ps[k].size() / ld));
                if (have != kept) {
                    restart_k(k, kept);
                    const int got = Hns[k].empty() ? 0 : (int)(Hns[k].size() / (Ps[k].size() / ld));
                    if (got != kept) kept = 0;
                }
            }
            if (kept == 0)
                for (int k = 0; k < nrhs; ++k)
                    if (active(k)) restart_k(k, 0);
            if (save && kept == 0) break;   // nothing worth carrying over
            const int nc = kept == 0 ? 1 : kept + rows - jc;
            std::vector<double2> Pd((size_t)nrhs * ld * nc, make_double2(0.0, 0.0));
            for (int k = 0; k < nrhs; ++k) {
                if (!active(k)) continue;
                for (int i = 0; i <= m; ++i)
                    for (int c = 0; c < nc; ++c) {
                        const cplx v = Ps[k][i + (size_t)c * ld];
                        Pd[(size_t)k * ld * nc + (size_t)i * nc + c] = make_double2(v.real(), v.imag());
                    }
            }
            TDDA_CUDA_TRY(cudaMemcpyAsync(gw.P, Pd.data(), sizeof(double2) * Pd.size(), cudaMemcpyHostToDevice, s));
            if (nc == 1) {
                // plain restart: V[0] = V P in place of a second basis
                lincomb(gw, m + 1, 1, (const C *)gw.V, (const double2 *)gw.P, 1, (size_t)ld, gw.W, s);
                TDDA_CUDA_TRY(cudaMemcpyAsync(gw.V, gw.W, sizeof(C) * vstr, cudaMemcpyDeviceToDevice, s));
            } else {
                lincomb(gw, m + 1, nc, (const C *)gw.V, (const double2 *)gw.P, nc, (size_t)ld * nc, gw.V2, s);
                std::swap(gw.V, gw.V2);
            }
            TDDA_CUDA_TRY(cudaGetLastError());
            if (save) {
                // slots 0..nc-1: Ah V[:, :kept] = V Hr (nc x kept)
                kr = kept;
                ar = nc - kept - 1;
                for (int k = 0; k < nrhs; ++k) Hr[k] = active(k) ? Hns[k] : std::vector<cplx>();
                break;
            }
            for (int k = 0; k < nrhs; ++k) {
                if (inner_done[k]) continue;
                L[k].reset(m);
                for (int c = 0; c < kept; ++c)
                    for (int r = 0; r < nc; ++r) L[k].h(r, c) = Hns[k][r + (size_t)c * nc];
                L[k].start(cns[k]);
            }
            kd = kept;
            aug = kept == 0 ? 0 : nc - kept - 1;
        }
        // correction D = p(Ah) U, X += ||R|| S D
        for (int i = 0; i < (int)roots.size(); ++i) {
            const cplx c = 1.0 / roots[i];
            st = poly_factor<C>(*w.op, w.sc, w.al, i == 0 ? gw.U : gw.W, gw.W, gw.Y, i == 0, nullptr, nullptr,
                                make_double2(c.real(), c.imag()), nrhs, w.dstride, s);
            if (st != TDDA_OK) return st;
        }
        for (int k = 0; k < nrhs; ++k)
            if (!done[k]) {
                mv[k] += (long long)roots.size();
                refines[k] += 1;
            }
        launch_axpy_inner<C>(n, w.nbox, nrhs, w.dstride, w.d_part + nrhs, w.sc64, gw.Y, X, s);
        TDDA_CUDA_TRY(cudaGetLastError());
    }
    if (info)
        for (int k = 0; k < nrhs; ++k) {
            info[k].iterations = steps[k];
            info[k].error = err[k];
            info[k].status = status[k];
            info[k].refinements = refines[k];
            info[k].inner_iterations = (int)std::min<long long>(mv[k], 2147483647LL);
            info[k].true_error = err[k];
        }
    return TDDA_OK;
}

// Timing of the two Gram-Schmidt kernels (CUDA events on stream s) on a
// scratch basis of nv + 1 vectors of n3 elements: ms[0] = projections and norm
// against nv vectors (k_multidot_bulk or its element-wise variant, without the
// host read-back), ms[1] = the update and normalisation.  The vectors hold a
// constant pattern; the time does not depend on the values.
template <typename C> tdda_status profile_gram_schmidt(long long n3, int nv, int iters, cudaStream_t s, double *ms) {
    GmresWork<C> gw;
    cudaEvent_t e[4] = {nullptr, nullptr, nullptr, nullptr};
    auto run = [&]() -> tdda_status {
        tdda_status st = gw.init(n3, 1, nv, 1, 0);
        if (st != TDDA_OK) return st;
        const size_t vec = sizeof(C) * (size_t)n3;
        TDDA_CUDA_TRY(cudaMemsetAsync(gw.V, 0x3c, vec * (nv + 1), s));   // finite floats and doubles
        TDDA_CUDA_TRY(cudaMemsetAsync(gw.coef, 0, sizeof(double2) * (nv + 1), s));
        C *w = basis(gw, nv);
        for (auto &x : e) TDDA_CUDA_TRY(cudaEventCreate(&x));
        multidot(gw, nv, w, gw.h, s);            // warm-up
        gs_update_scale(gw, nv, (const double2 *)gw.coef, w, s);
        TDDA_CUDA_TRY(cudaEventRecord(e[0], s));
        for (int i = 0; i < iters; ++i) multidot(gw, nv, w, gw.h, s);
        TDDA_CUDA_TRY(cudaEventRecord(e[1], s));
        TDDA_CUDA_TRY(cudaEventRecord(e[2], s));
        for (int i = 0; i < iters; ++i) gs_update_scale(gw, nv, (const double2 *)gw.coef, w, s);
        TDDA_CUDA_TRY(cudaEventRecord(e[3], s));
        TDDA_CUDA_TRY(cudaEventSynchronize(e[3]));
        float a = 0.f, b = 0.f;
        TDDA_CUDA_TRY(cudaEventElapsedTime(&a, e[0], e[1]));
        TDDA_CUDA_TRY(cudaEventElapsedTime(&b, e[2], e[3]));
        ms[0] = a / iters;
        ms[1] = b / iters;
        return TDDA_OK;
    };
    const tdda_status st = run();
    for (auto &x : e)
        if (x) cudaEventDestroy(x);
    cudaStreamSynchronize(s);   // the scratch basis is freed only after its kernels
    gw.release();
    return st;
}

template tdda_status profile_gram_schmidt<float2>(long long, int, int, cudaStream_t, double *);
template tdda_status profile_gram_schmidt<double2>(long long, int, int, cudaStream_t, double *);
template struct GmresWork<float2>;
template struct GmresWork<double2>;
template tdda_status pgmres_solve<float2>(const RefineWork<float2> &, GmresWork<float2> &, const double2 *, double2 *,
                                          int, bool, int, double, const GmresOptions &, tdda_solve_info *);
template tdda_status pgmres_solve<double2>(const RefineWork<double2> &, GmresWork<double2> &, const double2 *,
                                           double2 *, int, bool, int, double, const GmresOptions &,
                                           tdda_solve_info *);

}  // namespace tdda
