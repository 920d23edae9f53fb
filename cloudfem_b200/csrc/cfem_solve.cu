// Persistent batched Jacobi-PCG (replaces spla.spsolve / spla.factorized).
//
// All systems of a batch are solved by ONE cooperative launch. Rows of each
// system are cut into fixed chunks (aligned at the system's row 0) that the
// warps of the grid process; every step the grid runs one phase of every
// unfinished system and meets at a bounded grid barrier:
//
//   INIT  r = b - A x (FP64 matrix), ||b_lift||, Jacobi inverse, z = M r
//   A     p = z + beta p_old (computed on the fly for neighbours, so the
//         update needs no extra barrier), q = A p, p.q
//   B     x += alpha p (FP64), r -= alpha q, z = M r, r.z, r.r
//   R     true residual r = b - A x in FP64 replaces the recursive one
//         (reliable update: when the mixed-precision residual fell by 10x,
//         and always before convergence is declared)
//
// Each chunk reduces its part of the dot products warp-locally; the last
// chunk of a system to finish (atomic ticket) sums all chunk partials of
// that system in a fixed order and advances its state. Results therefore
// depend only on the system itself: bitwise identical alone or in a batch.
//
// CFEM_SOLVE_FP64 keeps all vectors and the matrix in FP64 (the plain
// path). CFEM_SOLVE_MIXED runs A, B in FP32 (FP32 matrix copy, FP32 r, z, p,
// q) and keeps FP64 only for the solution x, the true residual and the
// final convergence norm.
#include "cfem_common.cuh"

#include <math.h>
#include <vector>

namespace cfem {

enum { PH_INIT = 0, PH_A = 1, PH_B = 2, PH_R = 3, PH_ZERO = 4, PH_DONE = 5 };

constexpr int SOLVE_THREADS = 256;
constexpr int LANES = 8;                 // lanes per matrix row
constexpr int CHUNK_ROWS = 64;           // block rows per chunk
constexpr double RELIABLE_DELTA2 = 1e-2; // replace r when ||r|| < 0.1 ||r_ref||
constexpr int MAX_STALL = 8;
constexpr unsigned long long BARRIER_TIMEOUT_NS = 4000000000ull;  // 4 s

struct SysDev {
    int64_t n;
    int32_t bs, precond, mode, nchunks;
    int32_t chunk0, max_iter;
    const int32_t *rp;
    const int32_t *ci;
    const double *v64;
    const float *v32;
    const double *b;
    double *x;
    const uint8_t *fixed;
    void *r, *z, *p0, *p1, *q, *dinv;
    double *partial;
    double rtol2;
};

struct SysState {
    double rz, alpha, beta, bb, rmax2, best, relres;
    int32_t phase, iter, status, nres, stall, pbuf;
    unsigned int cnt;
    int32_t pad;
};

struct GridBar {
    unsigned int count;
    unsigned int gen;
    int err;
    int active;
};

__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded software grid barrier; all blocks are co-resident (cooperative
// launch). Returns false when a block gave up waiting (error flag set).
__device__ bool grid_sync(GridBar *bar, unsigned nblocks) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *vgen = &bar->gen;
        volatile int *verr = &bar->err;
        unsigned g = *vgen;
        __threadfence();
        unsigned arrived = atomicAdd(&bar->count, 1u);
        if (arrived == nblocks - 1) {
            atomicExch(&bar->count, 0u);
            __threadfence();
            atomicAdd(&bar->gen, 1u);
        } else {
            unsigned long long t0 = globaltimer();
            unsigned spins = 0;
            while (*vgen == g) {
                if (*verr) break;
                if ((++spins & 255u) == 0 && globaltimer() - t0 > BARRIER_TIMEOUT_NS) {
                    atomicExch(&bar->err, 1);
                    break;
                }
                __nanosleep(20);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *(volatile int *)&bar->err == 0;
}

template <typename T> __device__ __forceinline__ T ldcg(const T *p) { return __ldcg(p); }

__device__ __forceinline__ double vcg(const double *p) { return __ldcg(p); }
__device__ __forceinline__ int vcgi(const int32_t *p) { return __ldcg(p); }

template <int L, typename V>
__device__ __forceinline__ V group_sum(V v) {
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <typename T> struct MatVal;
template <> struct MatVal<double> {
    static __device__ __forceinline__ const double *get(const SysDev &S) { return S.v64; }
};
template <> struct MatVal<float> {
    static __device__ __forceinline__ const float *get(const SysDev &S) { return S.v32; }
};

// Inverse of the free part of a 3x3 block (fixed rows/cols -> 0).
__device__ __forceinline__ bool block_inverse(const double a[9], const bool fx[3],
                                              double out[9]) {
    double m[9];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int d = 0; d < 3; ++d)
            m[c * 3 + d] = (fx[c] || fx[d]) ? (c == d ? 1.0 : 0.0) : a[c * 3 + d];
    double c00 = m[4] * m[8] - m[5] * m[7];
    double c01 = m[5] * m[6] - m[3] * m[8];
    double c02 = m[3] * m[7] - m[4] * m[6];
    double det = m[0] * c00 + m[1] * c01 + m[2] * c02;
    if (!(det > 0.0) || !isfinite(det)) return false;
    double id = 1.0 / det;
    out[0] = c00 * id;
    out[1] = (m[2] * m[7] - m[1] * m[8]) * id;
    out[2] = (m[1] * m[5] - m[2] * m[4]) * id;
    out[3] = c01 * id;
    out[4] = (m[0] * m[8] - m[2] * m[6]) * id;
    out[5] = (m[2] * m[3] - m[0] * m[5]) * id;
    out[6] = c02 * id;
    out[7] = (m[1] * m[6] - m[0] * m[7]) * id;
    out[8] = (m[0] * m[4] - m[1] * m[3]) * id;
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int d = 0; d < 3; ++d)
            if (fx[c] || fx[d]) out[c * 3 + d] = 0.0;
    return true;
}

// z = M r for one block row (M = point or block Jacobi inverse).
template <typename T, int BS>
__device__ __forceinline__ void apply_prec(const SysDev &S, int64_t row,
                                           const T r[BS], T z[BS]) {
    const T *dinv = (const T *)S.dinv;
    if (BS == 3 && S.precond == CFEM_PRECOND_BLOCK) {
        const T *D = dinv + row * 9;
#pragma unroll
        for (int c = 0; c < 3; ++c)
            z[c] = ldcg(D + c * 3) * r[0] + ldcg(D + c * 3 + 1) * r[1] +
                   ldcg(D + c * 3 + 2) * r[2];
    } else {
#pragma unroll
        for (int c = 0; c < BS; ++c) z[c] = ldcg(dinv + row * BS + c) * r[c];
    }
}

// ---------------------------------------------------------------- phase A
template <typename T, int BS>
__device__ void phase_A(const SysDev &S, const SysState *st, int64_t r0,
                        int64_t r1, int lane, double part[4]) {
    constexpr int L = LANES, RPP = 32 / LANES;
    const T beta = (T)vcg(&st->beta);
    const int pbuf = vcgi(&st->pbuf);
    const T *pin = (const T *)(pbuf ? S.p1 : S.p0);
    T *pout = (T *)(pbuf ? S.p0 : S.p1);
    const T *z = (const T *)S.z;
    T *q = (T *)S.q;
    const T *v = MatVal<T>::get(S);
    const int sub = lane & (L - 1);
    T pq = 0;
    for (int64_t base = r0; base < r1; base += RPP) {
        const int64_t row = base + lane / L;
        const bool valid = row < r1;
        T acc[BS];
#pragma unroll
        for (int c = 0; c < BS; ++c) acc[c] = 0;
        if (valid) {
            const int32_t k1 = __ldg(S.rp + row + 1);
            for (int32_t k = __ldg(S.rp + row) + sub; k < k1; k += L) {
                const int64_t j = __ldg(S.ci + k);
                T pj[BS];
#pragma unroll
                for (int d = 0; d < BS; ++d)
                    pj[d] = ldcg(z + j * BS + d) + beta * ldcg(pin + j * BS + d);
                const T *vk = v + (int64_t)k * BS * BS;
#pragma unroll
                for (int c = 0; c < BS; ++c)
#pragma unroll
                    for (int d = 0; d < BS; ++d) acc[c] += __ldg(vk + c * BS + d) * pj[d];
            }
        }
#pragma unroll
        for (int c = 0; c < BS; ++c) acc[c] = group_sum<L>(acc[c]);
        if (valid && sub == 0) {
#pragma unroll
            for (int c = 0; c < BS; ++c) {
                const int64_t i = row * BS + c;
                const T pn = ldcg(z + i) + beta * ldcg(pin + i);
                pout[i] = pn;
                q[i] = acc[c];
                pq += pn * acc[c];
            }
        }
    }
    part[0] += (double)pq;
}

// ---------------------------------------------------------------- phase B
template <typename T, int BS>
__device__ void phase_B(const SysDev &S, const SysState *st, int64_t r0,
                        int64_t r1, int lane, double part[4]) {
    const T alpha = (T)vcg(&st->alpha);
    const double alpha64 = vcg(&st->alpha);
    const int pbuf = vcgi(&st->pbuf);
    const T *p = (const T *)(pbuf ? S.p1 : S.p0);
    T *r = (T *)S.r;
    T *z = (T *)S.z;
    const T *q = (const T *)S.q;
    T rz = 0, rr = 0;
    for (int64_t row = r0 + lane; row < r1; row += 32) {
        T rv[BS], zv[BS];
        bool fx[BS];
#pragma unroll
        for (int c = 0; c < BS; ++c) {
            const int64_t i = row * BS + c;
            fx[c] = S.fixed ? (__ldg(S.fixed + i) != 0) : false;
            const T pi = ldcg(p + i);
            rv[c] = ldcg(r + i);
            if (!fx[c]) {
                S.x[i] = ldcg(S.x + i) + alpha64 * (double)pi;
                rv[c] -= alpha * ldcg(q + i);
            }
        }
        apply_prec<T, BS>(S, row, rv, zv);
#pragma unroll
        for (int c = 0; c < BS; ++c) {
            const int64_t i = row * BS + c;
            if (fx[c]) zv[c] = 0;
            r[i] = rv[c];
            z[i] = zv[c];
            rz += rv[c] * zv[c];
            rr += rv[c] * rv[c];
        }
    }
    part[0] += (double)rz;
    part[1] += (double)rr;
}

// ------------------------------------------------------- phase R / INIT
// True residual in FP64. INIT also forms ||b_lift|| and the Jacobi inverse.
template <typename T, int BS, bool INIT>
__device__ void phase_R(const SysDev &S, int64_t r0, int64_t r1, int lane,
                        double part[4], int *bad) {
    constexpr int L = LANES, RPP = 32 / LANES;
    const int sub = lane & (L - 1);
    T *r = (T *)S.r;
    T *z = (T *)S.z;
    T *dinv = (T *)S.dinv;
    double rr = 0.0, bb = 0.0;
    T rz = 0;
    for (int64_t base = r0; base < r1; base += RPP) {
        const int64_t row = base + lane / L;
        const bool valid = row < r1;
        double acc[BS], accf[BS], dg[BS * BS];
#pragma unroll
        for (int c = 0; c < BS; ++c) acc[c] = accf[c] = 0.0;
#pragma unroll
        for (int c = 0; c < BS * BS; ++c) dg[c] = 0.0;
        if (valid) {
            const int32_t k1 = __ldg(S.rp + row + 1);
            for (int32_t k = __ldg(S.rp + row) + sub; k < k1; k += L) {
                const int64_t j = __ldg(S.ci + k);
                const double *vk = S.v64 + (int64_t)k * BS * BS;
                double xj[BS];
                bool fj[BS];
#pragma unroll
                for (int d = 0; d < BS; ++d) {
                    xj[d] = ldcg(S.x + j * BS + d);
                    fj[d] = INIT && S.fixed ? (__ldg(S.fixed + j * BS + d) != 0) : false;
                }
#pragma unroll
                for (int c = 0; c < BS; ++c)
#pragma unroll
                    for (int d = 0; d < BS; ++d) {
                        const double a = __ldg(vk + c * BS + d);
                        acc[c] += a * xj[d];
                        if (INIT && fj[d]) accf[c] += a * xj[d];
                        if (INIT && j == row) dg[c * BS + d] = a;
                    }
            }
        }
#pragma unroll
        for (int c = 0; c < BS; ++c) {
            acc[c] = group_sum<L>(acc[c]);
            if (INIT) accf[c] = group_sum<L>(accf[c]);
        }
        if (INIT) {
#pragma unroll
            for (int c = 0; c < BS * BS; ++c) dg[c] = group_sum<L>(dg[c]);
        }
        if (valid && sub == 0) {
            bool fx[BS];
            T rv[BS], zv[BS];
#pragma unroll
            for (int c = 0; c < BS; ++c) {
                const int64_t i = row * BS + c;
                fx[c] = S.fixed ? (__ldg(S.fixed + i) != 0) : false;
                const double bi = __ldg(S.b + i);
                const double rt = fx[c] ? 0.0 : bi - acc[c];
                if (INIT && !fx[c]) {
                    const double bl = bi - accf[c];
                    bb += bl * bl;
                }
                rr += rt * rt;
                rv[c] = (T)rt;
            }
            if (INIT) {
                if (BS == 3 && S.precond == CFEM_PRECOND_BLOCK) {
                    double inv[9];
                    if (!block_inverse(dg, fx, inv)) {
                        *bad = 1;
#pragma unroll
                        for (int c = 0; c < 9; ++c) inv[c] = 0.0;
                    }
#pragma unroll
                    for (int c = 0; c < 9; ++c) dinv[row * 9 + c] = (T)inv[c];
                } else {
#pragma unroll
                    for (int c = 0; c < BS; ++c) {
                        const double d = dg[c * BS + c];
                        double iv = 0.0;
                        if (!fx[c]) {
                            if (!(d > 0.0) || !isfinite(d)) *bad = 1;
                            else iv = 1.0 / d;
                        }
                        dinv[row * BS + c] = (T)iv;
                    }
                }
            }
            apply_prec<T, BS>(S, row, rv, zv);
#pragma unroll
            for (int c = 0; c < BS; ++c) {
                const int64_t i = row * BS + c;
                if (fx[c]) zv[c] = 0;
                r[i] = rv[c];
                z[i] = zv[c];
                rz += rv[c] * zv[c];
            }
        }
    }
    part[0] += rr;
    part[1] += bb;
    part[2] += (double)rz;
}

template <int BS>
__device__ void phase_zero(const SysDev &S, int64_t r0, int64_t r1, int lane) {
    for (int64_t i = r0 * BS + lane; i < r1 * BS; i += 32)
        if (!(S.fixed && __ldg(S.fixed + i))) S.x[i] = 0.0;
}

// Last-chunk bookkeeping: fixed-order sum of the system's chunk partials,
// then the state transition.
__device__ void finish_chunk(const SysDev &S, SysState *st, GridBar *bar,
                             int lc, int ph, double part[4], int lane,
                             int bad) {
#pragma unroll
    for (int v = 0; v < 4; ++v) part[v] = warp_sum(part[v]);
    int last = 0;
    if (lane == 0) {
#pragma unroll
        for (int v = 0; v < 4; ++v) S.partial[(int64_t)lc * 4 + v] = part[v];
        if (bad) atomicExch(&st->status, CFEM_ERR_BREAKDOWN);
        __threadfence();
        unsigned old = atomicAdd(&st->cnt, 1u);
        last = (old == (unsigned)S.nchunks - 1) ? 1 : 0;
    }
    last = __shfl_sync(0xffffffffu, last, 0);
    if (!last) return;
    __threadfence();
    double tot[4] = {0.0, 0.0, 0.0, 0.0};
    for (int c = lane; c < S.nchunks; c += 32)
#pragma unroll
        for (int v = 0; v < 4; ++v) tot[v] += vcg(S.partial + (int64_t)c * 4 + v);
#pragma unroll
    for (int v = 0; v < 4; ++v) tot[v] = warp_sum(tot[v]);
    if (lane != 0) return;
    st->cnt = 0;
    const double rtol2 = S.rtol2;
    int next = PH_DONE;
    const int status_now = *(volatile int32_t *)&st->status;
    if (status_now != CFEM_OK) {
        next = PH_DONE;   // a bad Jacobi block was found
    } else if (ph == PH_INIT) {
        const double rr = tot[0], bb = tot[1], rz = tot[2];
        st->bb = bb;
        if (!isfinite(rr) || !isfinite(bb) || !isfinite(rz)) {
            st->status = CFEM_ERR_BREAKDOWN;
        } else if (bb == 0.0) {
            st->relres = 0.0;
            next = PH_ZERO;
        } else if (rr <= rtol2 * bb) {
            st->relres = sqrt(rr / bb);
        } else {
            st->rz = rz;
            st->beta = 0.0;
            st->rmax2 = rr;
            st->best = rr;
            st->relres = sqrt(rr / bb);
            next = PH_A;
        }
    } else if (ph == PH_A) {
        const double pq = tot[0];
        if (!(pq > 0.0) || !isfinite(pq)) {
            st->status = CFEM_ERR_BREAKDOWN;
        } else {
            st->alpha = st->rz / pq;
            st->pbuf ^= 1;
            next = PH_B;
        }
    } else if (ph == PH_B) {
        const double rz = tot[0], rr = tot[1];
        const double bb = st->bb;
        st->iter += 1;
        if (!isfinite(rz) || !isfinite(rr)) {
            st->status = CFEM_ERR_BREAKDOWN;
        } else if (rr <= rtol2 * bb ||
                   (S.mode == CFEM_SOLVE_MIXED && rr < RELIABLE_DELTA2 * st->rmax2)) {
            next = PH_R;
        } else if (st->iter >= S.max_iter) {
            st->status = CFEM_ERR_NOT_CONVERGED;
            st->relres = sqrt(rr / bb);
        } else {
            st->beta = rz / st->rz;
            st->rz = rz;
            next = PH_A;
        }
    } else if (ph == PH_R) {
        const double rr = tot[0], rz = tot[2], bb = st->bb;
        st->nres += 1;
        st->relres = sqrt(rr / bb);
        if (!isfinite(rr) || !isfinite(rz)) {
            st->status = CFEM_ERR_BREAKDOWN;
        } else if (rr <= rtol2 * bb) {
            // converged on the FP64 true residual
        } else if (st->iter >= S.max_iter) {
            st->status = CFEM_ERR_NOT_CONVERGED;
        } else {
            if (rr < 0.25 * st->best) {
                st->best = rr;
                st->stall = 0;
            } else {
                st->stall += 1;
            }
            if (st->stall >= MAX_STALL) {
                st->status = CFEM_ERR_NOT_CONVERGED;
            } else {
                st->beta = rz / st->rz;
                st->rz = rz;
                st->rmax2 = rr;
                next = PH_A;
            }
        }
    } else if (ph == PH_ZERO) {
        next = PH_DONE;
    }
    st->phase = next;
    if (next == PH_DONE) atomicSub(&bar->active, 1);
}

template <typename T, int BS>
__device__ void run_chunk(const SysDev &S, SysState *st, GridBar *bar, int ph,
                          int lc, int lane) {
    const int64_t r0 = (int64_t)lc * CHUNK_ROWS;
    const int64_t r1 = min(S.n, r0 + CHUNK_ROWS);
    double part[4] = {0.0, 0.0, 0.0, 0.0};
    int bad = 0;
    switch (ph) {
        case PH_INIT: {
            int flag = 0;
            phase_R<T, BS, true>(S, r0, r1, lane, part, &flag);
            bad = __any_sync(0xffffffffu, flag != 0);
            break;
        }
        case PH_A: phase_A<T, BS>(S, st, r0, r1, lane, part); break;
        case PH_B: phase_B<T, BS>(S, st, r0, r1, lane, part); break;
        case PH_R: {
            int flag = 0;
            phase_R<T, BS, false>(S, r0, r1, lane, part, &flag);
            break;
        }
        default: phase_zero<BS>(S, r0, r1, lane); break;
    }
    finish_chunk(S, st, bar, lc, ph, part, lane, bad);
}

__global__ void __launch_bounds__(SOLVE_THREADS)
k_pcg_persistent(const SysDev *__restrict__ sys, SysState *st,
                 const int32_t *__restrict__ chunk_sys, int n_chunks,
                 GridBar *bar, int max_steps) {
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int step = 0; step < max_steps; ++step) {
        for (int c = gw; c < n_chunks; c += nw) {
            const int s = __ldg(chunk_sys + c);
            const SysDev &S = sys[s];
            const int ph = *(volatile int32_t *)&st[s].phase;
            if (ph == PH_DONE) continue;
            const int lc = c - S.chunk0;
            if (S.mode == CFEM_SOLVE_MIXED) {
                if (S.bs == 3) run_chunk<float, 3>(S, &st[s], bar, ph, lc, lane);
                else run_chunk<float, 1>(S, &st[s], bar, ph, lc, lane);
            } else {
                if (S.bs == 3) run_chunk<double, 3>(S, &st[s], bar, ph, lc, lane);
                else run_chunk<double, 1>(S, &st[s], bar, ph, lc, lane);
            }
        }
        if (!grid_sync(bar, gridDim.x)) return;
        if (*(volatile int *)&bar->active <= 0) return;
    }
}

}  // namespace cfem

using namespace cfem;

extern "C" int cfem_pcg_solve(cfem_ctx *ctx, const cfem_linsys *systems,
                              int32_t n_systems, cfem_solve_stats *stats,
                              void *stream) {
    CFEM_API_BEGIN
    CFEM_CHECK(ctx && systems && stats && n_systems > 0, CFEM_ERR_INVALID,
               "cfem_pcg_solve: bad args");
    CFEM_TRY(set_device(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;
    std::vector<SysDev> hs(n_systems);
    std::vector<int32_t> chunk_sys;
    size_t bytes = 0;
    auto align = [](size_t v) { return (v + 255) & ~(size_t)255; };
    int max_iter = 1;
    for (int i = 0; i < n_systems; ++i) {
        const cfem_linsys &L = systems[i];
        CFEM_CHECK(L.bs == 1 || L.bs == 3, CFEM_ERR_INVALID,
                   "system %d: block size %d (1 or 3)", i, L.bs);
        CFEM_CHECK(L.n_rows > 0 && L.d_row_ptr && L.d_col && L.d_vals64 &&
                       L.d_b && L.d_x,
                   CFEM_ERR_INVALID, "system %d: missing arrays", i);
        CFEM_CHECK(L.mode == CFEM_SOLVE_FP64 ||
                       (L.mode == CFEM_SOLVE_MIXED && L.d_vals32),
                   CFEM_ERR_INVALID, "system %d: mixed mode needs FP32 values", i);
        CFEM_CHECK(L.rtol > 0.0 && L.max_iter > 0, CFEM_ERR_INVALID,
                   "system %d: rtol and max_iter must be positive", i);
        CFEM_CHECK(L.n_rows < ((int64_t)1 << 31) / 9, CFEM_ERR_INVALID,
                   "system %d too large", i);
        SysDev &S = hs[i];
        S.n = L.n_rows;
        S.bs = L.bs;
        S.precond = (L.bs == 3) ? L.precond : CFEM_PRECOND_JACOBI;
        S.mode = L.mode;
        S.nchunks = (int32_t)((L.n_rows + CHUNK_ROWS - 1) / CHUNK_ROWS);
        S.chunk0 = (int32_t)chunk_sys.size();
        S.max_iter = L.max_iter;
        S.rp = L.d_row_ptr;
        S.ci = L.d_col;
        S.v64 = L.d_vals64;
        S.v32 = L.d_vals32;
        S.b = L.d_b;
        S.x = L.d_x;
        S.fixed = L.d_fixed;
        S.rtol2 = L.rtol * L.rtol;
        for (int c = 0; c < S.nchunks; ++c) chunk_sys.push_back(i);
        const size_t ts = (L.mode == CFEM_SOLVE_MIXED) ? 4 : 8;
        const size_t nd = (size_t)L.n_rows * L.bs;
        const size_t nprec = (S.precond == CFEM_PRECOND_BLOCK) ? (size_t)L.n_rows * 9 : nd;
        bytes += 5 * align(nd * ts) + align(nprec * ts) + align(S.nchunks * 4 * sizeof(double));
        if (L.max_iter > max_iter) max_iter = L.max_iter;
    }
    const int n_chunks = (int)chunk_sys.size();
    bytes += align(n_systems * sizeof(SysDev)) + align(n_systems * sizeof(SysState)) +
             align(n_chunks * sizeof(int32_t)) + align(sizeof(GridBar));
    char *ws = nullptr;
    CFEM_TRY(tmp_alloc(&ws, bytes, s));
    CFEM_CUDA(cudaMemsetAsync(ws, 0, bytes, s));
    size_t off = 0;
    auto take = [&](size_t b) { char *p = ws + off; off += align(b); return (void *)p; };
    for (int i = 0; i < n_systems; ++i) {
        SysDev &S = hs[i];
        const size_t ts = (S.mode == CFEM_SOLVE_MIXED) ? 4 : 8;
        const size_t nd = (size_t)S.n * S.bs;
        const size_t nprec = (S.precond == CFEM_PRECOND_BLOCK) ? (size_t)S.n * 9 : nd;
        S.r = take(nd * ts);
        S.z = take(nd * ts);
        S.p0 = take(nd * ts);
        S.p1 = take(nd * ts);
        S.q = take(nd * ts);
        S.dinv = take(nprec * ts);
        S.partial = (double *)take(S.nchunks * 4 * sizeof(double));
    }
    SysDev *d_sys = (SysDev *)take(n_systems * sizeof(SysDev));
    SysState *d_st = (SysState *)take(n_systems * sizeof(SysState));
    int32_t *d_chunks = (int32_t *)take(n_chunks * sizeof(int32_t));
    GridBar *d_bar = (GridBar *)take(sizeof(GridBar));
    GridBar hbar{0u, 0u, 0, n_systems};
    CFEM_CUDA(cudaMemcpyAsync(d_sys, hs.data(), n_systems * sizeof(SysDev),
                              cudaMemcpyHostToDevice, s));
    CFEM_CUDA(cudaMemcpyAsync(d_chunks, chunk_sys.data(),
                              n_chunks * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    CFEM_CUDA(cudaMemcpyAsync(d_bar, &hbar, sizeof(GridBar),
                              cudaMemcpyHostToDevice, s));

    int per_sm = 0;
    CFEM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, k_pcg_persistent, SOLVE_THREADS, 0));
    CFEM_CHECK(per_sm > 0, CFEM_ERR_CUDA, "solver kernel cannot be resident");
    if (per_sm > 4) per_sm = 4;
    int grid = ctx->num_sms * per_sm;
    const int warps_needed = (n_chunks + 0);
    const int max_blocks_useful = (warps_needed * 32 + SOLVE_THREADS - 1) / SOLVE_THREADS;
    if (grid > max_blocks_useful) grid = max_blocks_useful < 1 ? 1 : max_blocks_useful;
    int max_steps = 3 * max_iter + 16;
    void *args[] = {(void *)&d_sys, (void *)&d_st, (void *)&d_chunks,
                    (void *)&n_chunks, (void *)&d_bar, (void *)&max_steps};
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    CFEM_CUDA(cudaEventCreate(&ev0));
    CFEM_CUDA(cudaEventCreate(&ev1));
    CFEM_CUDA(cudaEventRecord(ev0, s));
    CFEM_CUDA(cudaLaunchCooperativeKernel((void *)k_pcg_persistent, dim3(grid),
                                          dim3(SOLVE_THREADS), args, 0, s));
    CFEM_CUDA(cudaEventRecord(ev1, s));
    g_launches.fetch_add(1, std::memory_order_relaxed);
    std::vector<SysState> hst(n_systems);
    CFEM_CUDA(cudaMemcpyAsync(hst.data(), d_st, n_systems * sizeof(SysState),
                              cudaMemcpyDeviceToHost, s));
    CFEM_CUDA(cudaMemcpyAsync(&hbar, d_bar, sizeof(GridBar),
                              cudaMemcpyDeviceToHost, s));
    tmp_free(ws, s);
    CFEM_CUDA(cudaStreamSynchronize(s));
    float kms = 0.0f;
    CFEM_CUDA(cudaEventElapsedTime(&kms, ev0, ev1));
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    for (int i = 0; i < n_systems; ++i) {
        stats[i].status = hst[i].status;
        if (hst[i].status == CFEM_OK && hst[i].phase != PH_DONE)
            stats[i].status = CFEM_ERR_NOT_CONVERGED;
        stats[i].iterations = hst[i].iter;
        stats[i].residual_updates = hst[i].nres;
        stats[i].pad_ = 0;
        stats[i].relres = hst[i].relres;
        stats[i].bnorm = sqrt(hst[i].bb);
        stats[i].kernel_ms = (double)kms;
    }
    CFEM_CHECK(hbar.err == 0, CFEM_ERR_TIMEOUT,
               "solver grid barrier timed out (device wait bound reached)");
    return CFEM_OK;
    CFEM_API_END
}
