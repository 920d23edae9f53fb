// Persistent batched Jacobi-PCG (replaces spla.spsolve / spla.factorized).
//
// All systems of a batch are solved by ONE cooperative launch (after one
// ordinary INIT launch). Rows of each system are cut into small chunks
// (8 block rows for 3x3 blocks, 16 rows for scalars, aligned at the
// system's row 0); the warps of the grid take chunks round-robin. Every
// step the grid runs one phase of every unfinished system and meets at a
// bounded two-level grid barrier:
//
//   INIT  r = b - A x (FP64 matrix), ||b_lift||, Jacobi inverse, z = M r
//   A     p = z + beta p_old (evaluated on the fly for neighbours, so the
//         update needs no extra barrier), q = A p, p.q
//   B     x += alpha p (FP64), r -= alpha q, z = M r, r.z, r.r
//   R     true residual r = b - A x in FP64 replaces the recursive one
//         (reliable update: when the mixed-precision residual fell by
//         `reliable_delta`, and always before convergence is declared)
//
// Dot products: each chunk reduces warp-locally; chunk partials are summed
// per tile of 32 chunks by the tile's last finisher, tile partials by the
// system's last tile (atomic tickets). The summation tree depends only on
// the system, so each result is bitwise the same alone or in any batch.
//
// CFEM_SOLVE_FP64 keeps all vectors and the matrix in FP64 (the plain
// path). CFEM_SOLVE_MIXED runs A and B in FP32 (FP32 matrix copy and FP32
// r, z, p, q) and keeps FP64 only for x, the true residual and the final
// convergence norm.
#include "cfem_common.cuh"

#include <cub/device/device_scan.cuh>
#include <cuda.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

namespace cfem {

enum { PH_INIT = 0, PH_A = 1, PH_B = 2, PH_R = 3, PH_ZERO = 4, PH_DONE = 5 };

constexpr int SOLVE_THREADS = 512;
constexpr int LANES = 8;                   // lanes per block row
constexpr int RPP = 32 / LANES;            // block rows per warp pass
constexpr int TILE = 32;                   // chunks per reduction tile
constexpr double RELIABLE_DELTA = 0.1;
constexpr int MAX_STALL = 8;
// The FP64 residual r_i = b_i - sum_j a_ij x_j carries a rounding error of
// a few eps * sum_j |a_ij x_j|; a residual at that level cannot be reduced
// or even measured further, so it counts as converged.
constexpr double FLOOR_C = 16.0 * 2.220446049250313e-16;
// A residual at or below FLOOR_TIGHT is converged at once; one between the
// two is accepted as the floor once a true-residual replacement fails to
// improve it 4x (it is then rounding noise, not progress). A direct solver's
// answer carries a residual of about eps * |A||x|, so stopping at the tight
// bound matches its accuracy even on ill-conditioned systems.
constexpr double FLOOR_TIGHT = 2.0 * 2.220446049250313e-16;
constexpr int BAR_GROUP = 16;              // blocks per first-level counter
constexpr int BAR_MAX_GROUPS = 64;

__host__ __device__ inline int chunk_rows(int bs) { return bs == 3 ? 8 : 16; }

struct SysDev {
    int64_t n;
    int32_t bs, precond, mode, max_iter;
    int32_t nchunks, ntiles, chunk0, crows;
    const int32_t *rp;
    const int32_t *ci;
    const double *v64;
    const float *v32;
    const double *b;
    double *x;
    const uint8_t *fixed;
    void *r, *z, *p0, *p1, *q, *dinv;
    double *partial;      // nchunks * 4
    double *tpartial;     // ntiles * 4
    unsigned int *tcnt;   // ntiles tickets
    double rtol2, delta2;
    int32_t max_stall, hist_cap;
    double *hist;
    // graph scheduler: update-phase chunks (whole block rows, <= 32 DOFs)
    int32_t nchunksB;
    int32_t vec4;         // bs 1, graph scheduler: ci4 / va4 present
    double *partialB;     // nchunksB * 4
    const void *vsoa;     // working-precision block values, entry-major
    int64_t nnzb;         // blocks of the matrix (stride of vsoa)
    // bs 1, graph scheduler: rows padded to whole units of 4 entries, row i
    // starting at unit (rp[i] + 3 i + 3) / 4 (padding: column i, value 0)
    const int32_t *ci4;
    const void *va4;
    const double *va4d;   // FP64 values in the same layout (== va4 in FP64 mode)
    // bs 3, graph scheduler with the staged SpMV: block rows padded to whole
    // units of 4 blocks, row i starting at unit (rp[i] + 3 i + 3) / 4
    // (padding: column i, zero block); working-precision values, 9 per slot
    const int32_t *c3;
    const void *v3;
    // graph scheduler: rows per SpMV-phase work entry, and entry count
    int32_t xrows, nxe;
    // bs 1, graph scheduler with the sliced-ELL SpMV (SpMV staging 3):
    // work entries of SELL_ROWS rows sorted by length into slices of 32 rows,
    // slot k of slice lane l at soff[slice] + 32 k + l (slot 0: the diagonal
    // entry, or the row sum of the FP32 difference form); sperm: the entry's
    // row (0..SELL_ROWS-1) at each sorted position
    const int32_t *scol;
    const void *sval;
    const int64_t *soff;
    const uint8_t *sperm;
    int32_t sell;
    int32_t lpr;          // bs 1, unit-padded residual phase: lanes per row (4 or 8;
                          // 0 means 8)
    int32_t rsell;        // bs 1, mixed, A phase staged: an FP64 sliced-ELL copy
                          // (scol / sval / soff / sperm) for the residual phase
};

struct SysState {
    double rz, alpha, beta, bb, rmax2, best, relres, zeta;
    int32_t phase, iter, status, nres, stall, pbuf;
    unsigned int cnt;
    int32_t pad;
};

// Counters live on separate 128-byte lines.
struct GridBar {
    unsigned int gen;
    int err;
    int active;
    unsigned int rounds;    // loop bodies run (graph scheduler)
    unsigned int pad0[28];
    unsigned int top;
    unsigned int pad1[31];
    unsigned int grp[BAR_MAX_GROUPS][32];
};

// Programmatic dependent launch: kernels of the graph scheduler are
// captured with programmatic stream serialisation, so the next kernel's
// launch is processed while the previous one drains; each waits here for
// its predecessor's completion and memory before reading anything it wrote.
// A no-op for ordinary launches.
__device__ __forceinline__ void pdl_wait() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
}
// Lets the next kernel of the graph launch before this one ends (it runs
// what precedes its own pdl_wait, which still waits for this kernel's
// completion and memory). Issued after this kernel's own wait, so every
// earlier kernel has completed by then.
__device__ __forceinline__ void pdl_trigger() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned atom_add_acqrel(unsigned *p, unsigned v) {
    unsigned old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;"
                 : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// Bounded two-level software grid barrier over co-resident blocks
// (cooperative launch). Returns false when a block gave up waiting.
// `timeout_ns` bounds each wait (CFEM_PARAM_BARRIER_TIMEOUT_US); `hold`
// phantom blocks are counted as still to arrive (CFEM_PARAM_BARRIER_HOLD,
// fault injection for the host's timeout path: with hold > 0 no wait can
// complete, so every block gives up at the limit and the launch returns).
__device__ bool grid_sync(GridBar *bar, unsigned long long timeout_ns, unsigned hold) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *vgen = &bar->gen;
        volatile int *verr = &bar->err;
        (void)vgen;
        const unsigned nb = gridDim.x;
        const unsigned grp = blockIdx.x / BAR_GROUP;
        const unsigned ngrp = (nb + BAR_GROUP - 1) / BAR_GROUP;
        const unsigned gsize = min((unsigned)BAR_GROUP, nb - grp * BAR_GROUP);
        unsigned g = *vgen;
        __threadfence();
        bool released = false;
        if (atomicAdd(&bar->grp[grp][0], 1u) == gsize - 1) {
            atomicExch(&bar->grp[grp][0], 0u);
            __threadfence();
            if (atomicAdd(&bar->top, 1u) == ngrp - 1 + hold) {
                atomicExch(&bar->top, 0u);
                __threadfence();
                atomicAdd(&bar->gen, 1u);
                released = true;
            }
        }
        if (!released) {
            unsigned long long t0 = globaltimer();
            unsigned spins = 0;
            while (ld_acquire(&bar->gen) == g) {
                if ((++spins & 1023u) == 0) {
                    if (*verr) break;
                    if (globaltimer() - t0 > timeout_ns) {
                        atomicExch(&bar->err, 1);
                        break;
                    }
                }
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

// ---------------------------------------------------------------- phase A
// q = A p with p = zeta z + beta p_old (zeta = 1 except right after a
// true-residual replacement, see advance()). Each lane group of LANES lanes works on
// two block rows at once and unrolls U column blocks per row, so every lane
// keeps 2U independent (index -> gather) load chains in flight.
//
// DIFF (mixed precision): the FP32 operator is stored in difference form
// (cfem_mixed_matrix): off-diagonal blocks A_ij and, in the diagonal slot,
// the FP64 row sum s_i = sum_j A_ij rounded once. Then
//     (A p)_i = s_i p_i + sum_{j != i} A_ij (p_j - p_i),
// which applies constant vectors (rigid translations, uniform fields)
// exactly whatever the rounding of A_ij, so the FP32 operator does not
// perturb the near-null space that governs the CG convergence.
template <typename T, int BS, bool DIFF, int U>
__device__ void phase_A(const SysDev &S, const SysState *st, int64_t r0,
                        int64_t r1, int lane, double part[4]) {
    constexpr int B2 = BS * BS;
    const T beta = (T)vcg(&st->beta);
    const T zeta = (T)vcg(&st->zeta);
    const int pbuf = vcgi(&st->pbuf);
    const T *pin = (const T *)(pbuf ? S.p1 : S.p0);
    T *pout = (T *)(pbuf ? S.p0 : S.p1);
    const T *z = (const T *)S.z;
    T *q = (T *)S.q;
    const T *v = MatVal<T>::get(S);
    const int32_t *ci = S.ci;
    const int sub = lane & (LANES - 1), grp = lane / LANES;
    T pq = 0;
    for (int64_t base = r0; base < r1; base += 2 * RPP) {
        int64_t row[2];
        bool valid[2];
        int32_t k0[2], k1[2];
        T pi[2][BS], acc[2][BS];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            row[h] = base + h * RPP + grp;
            valid[h] = row[h] < r1;
            const int64_t rr = valid[h] ? row[h] : r0;
            k0[h] = valid[h] ? __ldg(S.rp + rr) : 0;
            k1[h] = valid[h] ? __ldg(S.rp + rr + 1) : 0;
#pragma unroll
            for (int c = 0; c < BS; ++c) {
                pi[h][c] = zeta * ldcg(z + rr * BS + c) + beta * ldcg(pin + rr * BS + c);
                acc[h][c] = 0;
            }
        }
        const int32_t len = max(k1[0] - k0[0], k1[1] - k0[1]);
        for (int32_t off = sub; off < len; off += U * LANES) {
            int64_t j[2][U];
            T a[2][U][B2];
            bool on[2][U];
#pragma unroll
            for (int h = 0; h < 2; ++h)
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int32_t k = k0[h] + off + u * LANES;
                    on[h][u] = k < k1[h];
                    const int32_t kk = on[h][u] ? k : k0[0];
                    j[h][u] = __ldg(ci + kk);
#pragma unroll
                    for (int e = 0; e < B2; ++e) {
                        const T av = __ldg(v + (int64_t)kk * B2 + e);
                        a[h][u][e] = on[h][u] ? av : (T)0;
                    }
                }
#pragma unroll
            for (int h = 0; h < 2; ++h)
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    T pj[BS];
#pragma unroll
                    for (int d = 0; d < BS; ++d) {
                        pj[d] = zeta * ldcg(z + j[h][u] * BS + d) +
                                beta * ldcg(pin + j[h][u] * BS + d);
                        if (DIFF) pj[d] = (j[h][u] == row[h]) ? pi[h][d] : pj[d] - pi[h][d];
                    }
#pragma unroll
                    for (int c = 0; c < BS; ++c)
#pragma unroll
                        for (int d = 0; d < BS; ++d) acc[h][c] += a[h][u][c * BS + d] * pj[d];
                }
        }
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int c = 0; c < BS; ++c) acc[h][c] = group_sum<LANES>(acc[h][c]);
        if (sub == 0) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                if (!valid[h]) continue;
#pragma unroll
                for (int c = 0; c < BS; ++c) {
                    const int64_t i = row[h] * BS + c;
                    pout[i] = pi[h][c];
                    q[i] = acc[h][c];
                    pq += pi[h][c] * acc[h][c];
                }
            }
        }
    }
    part[0] += (double)pq;
}

// ---------------------------------------------------------------- phase B
// One lane per DOF of the chunk; every load (vectors, mask, the lane's row
// of the Jacobi inverse) is issued before any is used.
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
    const T *dinv = (const T *)S.dinv;
    const bool blockj = BS == 3 && S.precond == CFEM_PRECOND_BLOCK;
    const int64_t i = r0 * BS + lane;
    const bool valid = i < r1 * BS;
    const int64_t ii = valid ? i : r0 * BS;
    const int64_t row = ii / BS;
    const int c = (int)(ii - row * BS);
    const bool fx = S.fixed ? (__ldg(S.fixed + ii) != 0) : false;
    T rv = ldcg(r + ii);
    const T pi = ldcg(p + ii);
    const T qi = ldcg(q + ii);
    const double xi = ldcg(S.x + ii);
    T d0, d1 = 0, d2 = 0;
    if (blockj) {
        const T *D = dinv + row * 9 + c * 3;
        d0 = ldcg(D);
        d1 = ldcg(D + 1);
        d2 = ldcg(D + 2);
    } else {
        d0 = ldcg(dinv + ii);
    }
    if (valid && !fx) {
        S.x[i] = xi + alpha64 * (double)pi;
        rv -= alpha * qi;
    }
    T zv;
    if (blockj) {
        const int base = lane - c;
        const T ra = __shfl_sync(0xffffffffu, rv, base >= 0 ? base : 0);
        const T rb = __shfl_sync(0xffffffffu, rv, base + 1 < 32 ? base + 1 : 31);
        const T rc = __shfl_sync(0xffffffffu, rv, base + 2 < 32 ? base + 2 : 31);
        zv = d0 * ra + d1 * rb + d2 * rc;
    } else {
        zv = d0 * rv;
    }
    T rz = 0, rr = 0;
    if (valid) {
        if (fx) zv = 0;
        r[i] = rv;
        z[i] = zv;
        rz = rv * zv;
        rr = rv * rv;
    }
    part[0] += (double)rz;
    part[1] += (double)rr;
}

// ------------------------------------------------------- phase R / INIT
// True residual in FP64; INIT also forms ||b_lift|| and the Jacobi inverse.
// Compensated (double-double) sums for the FP64 true residual: hi + lo
// carries sum_j a_j x_j with the rounding error of every product (exact by
// FMA) and of every addition (TwoSum), so r = b - A x is accurate to about
// eps |r| rather than eps |A||x| and the solver can certify (and reach) a
// residual at the level a direct solver's answer has. The _rn intrinsics
// keep the compiler from contracting the error terms away.
__device__ __forceinline__ void dd_add(double &hi, double &lo, double h2, double l2) {
    const double s = __dadd_rn(hi, h2);
    const double bp = __dsub_rn(s, hi);
    const double e = __dadd_rn(__dsub_rn(hi, __dsub_rn(s, bp)), __dsub_rn(h2, bp));
    hi = s;
    lo = __dadd_rn(lo, __dadd_rn(e, l2));
}
__device__ __forceinline__ void dd_fma(double &hi, double &lo, double a, double x) {
    const double p = __dmul_rn(a, x);
    dd_add(hi, lo, p, fma(a, x, -p));
}
template <int L>
__device__ __forceinline__ void group_sum_dd(double &hi, double &lo) {
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) {
        const double h2 = __shfl_xor_sync(0xffffffffu, hi, o);
        const double l2 = __shfl_xor_sync(0xffffffffu, lo, o);
        dd_add(hi, lo, h2, l2);
    }
}
// b - (hi + lo), rounded once at the end
__device__ __forceinline__ double dd_residual(double b, double hi, double lo) {
    return __dsub_rn(__dsub_rn(b, hi), lo);
}

// NC: x is read-only for the whole launch (the per-phase kernels of the
// graph scheduler), so its gathers may go through L1; the persistent kernel,
// which also writes x, reads it through L2 (ldcg).
template <bool INIT, int BS, bool NC = false>
__device__ __forceinline__ void acc_R(const double *__restrict__ v,
                                      const int32_t *__restrict__ ci, int32_t k,
                                      int64_t row, const double *x,
                                      const uint8_t *fixed, double acc[BS],
                                      double alo[BS], double aab[BS], double accf[BS],
                                      double dg[BS * BS]) {
    const int64_t j = __ldg(ci + k);
    const double *vk = v + (int64_t)k * BS * BS;
    double xj[BS];
    bool fj[BS];
#pragma unroll
    for (int d = 0; d < BS; ++d) {
        xj[d] = NC ? __ldg(x + j * BS + d) : ldcg(x + j * BS + d);
        fj[d] = INIT && fixed ? (__ldg(fixed + j * BS + d) != 0) : false;
    }
#pragma unroll
    for (int c = 0; c < BS; ++c)
#pragma unroll
        for (int d = 0; d < BS; ++d) {
            const double a = __ldg(vk + c * BS + d);
            const double ax = a * xj[d];
            dd_fma(acc[c], alo[c], a, xj[d]);
            aab[c] += fabs(ax);
            if (INIT && fj[d]) accf[c] += ax;
            if (INIT && j == row) dg[c * BS + d] = a;
        }
}

template <typename T, int BS, bool INIT, bool NC = false>
__device__ void phase_R(const SysDev &S, const SysState *st, int64_t r0,
                        int64_t r1, int lane, double part[4], int *bad) {
    const int sub = lane & (LANES - 1), grp = lane / LANES;
    T *r = (T *)S.r;
    T *z = (T *)S.z;
    T *dinv = (T *)S.dinv;
    const T *pc = (const T *)((INIT || vcgi(&st->pbuf) == 0) ? S.p0 : S.p1);
    double rr = 0.0, bb = 0.0, aa = 0.0;
    T rz = 0, rp = 0;
    for (int64_t base = r0; base < r1; base += RPP) {
        const int64_t row = base + grp;
        const bool valid = row < r1;
        double acc[BS], alo[BS], accf[BS], aab[BS], dg[BS * BS];
#pragma unroll
        for (int c = 0; c < BS; ++c) acc[c] = alo[c] = accf[c] = aab[c] = 0.0;
#pragma unroll
        for (int c = 0; c < BS * BS; ++c) dg[c] = 0.0;
        if (valid) {
            const int32_t k1 = __ldg(S.rp + row + 1);
            for (int32_t k = __ldg(S.rp + row) + sub; k < k1; k += LANES)
                acc_R<INIT, BS, NC>(S.v64, S.ci, k, row, S.x, S.fixed, acc, alo, aab, accf, dg);
        }
#pragma unroll
        for (int c = 0; c < BS; ++c) {
            group_sum_dd<LANES>(acc[c], alo[c]);
            aab[c] = group_sum<LANES>(aab[c]);
            if (INIT) accf[c] = group_sum<LANES>(accf[c]);
        }
        if (INIT) {
#pragma unroll
            for (int c = 0; c < BS * BS; ++c) dg[c] = group_sum<LANES>(dg[c]);
        }
        if (valid && sub == 0) {
            bool fx[BS];
            T rv[BS];
#pragma unroll
            for (int c = 0; c < BS; ++c) {
                const int64_t i = row * BS + c;
                fx[c] = S.fixed ? (__ldg(S.fixed + i) != 0) : false;
                const double bi = __ldg(S.b + i);
                const double rt = fx[c] ? 0.0 : dd_residual(bi, acc[c], alo[c]);
                if (INIT && !fx[c]) {
                    const double bl = bi - accf[c];
                    bb += bl * bl;
                }
                rr += rt * rt;
                if (!fx[c]) aa += aab[c] * aab[c];
                rv[c] = (T)rt;
                r[i] = rv[c];
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
            // z = M r (row-local: this lane wrote or reads this row's dinv)
            const T *D = (const T *)S.dinv;
#pragma unroll
            for (int c = 0; c < BS; ++c) {
                T zv;
                if (BS == 3 && S.precond == CFEM_PRECOND_BLOCK)
                    zv = ldcg(D + row * 9 + c * 3) * rv[0] +
                         ldcg(D + row * 9 + c * 3 + 1) * rv[BS > 1 ? 1 : 0] +
                         ldcg(D + row * 9 + c * 3 + 2) * rv[BS > 2 ? 2 : 0];
                else
                    zv = ldcg(D + row * BS + c) * rv[c];
                if (fx[c]) zv = 0;
                z[row * BS + c] = zv;
                rz += rv[c] * zv;
                if (!INIT) rp += rv[c] * ldcg(pc + row * BS + c);
            }
        }
    }
    part[0] += rr;
    part[1] += INIT ? bb : (double)rp;
    part[2] += (double)rz;
    part[3] += aa;
}

// True residual (FP64) of scalar rows from the unit-padded copy, the same
// sums and epilogue as phase_R<T, 1, INIT>: each lane of a group of 8 reads
// whole units of four entries; padding entries (column = own row, value 0)
// add nothing and are told apart from the real diagonal by position.
template <typename T, bool INIT, bool NC = false, int LPR = 8>
__device__ void phase_R_vec1(const SysDev &S, const SysState *st, int64_t r0,
                             int64_t r1, int lane, double part[4], int *bad) {
    constexpr int H = 2, NG = 32 / LPR;
    const int sub = lane % LPR, grp = lane / LPR;
    T *r = (T *)S.r;
    T *z = (T *)S.z;
    T *dinv = (T *)S.dinv;
    const T *pc = (const T *)((INIT || vcgi(&st->pbuf) == 0) ? S.p0 : S.p1);
    const int32_t *ci = S.ci4;
    const double *va = S.va4d;
    double rr = 0.0, bb = 0.0, aa = 0.0;
    T rz = 0, rp = 0;
    for (int64_t base = r0; base < r1; base += NG * H) {
        int64_t row[H], u[H], u0[H], uend[H], len[H];
        bool valid[H];
        double acc[H], alo[H], aab[H], accf[H], dg[H];
#pragma unroll
        for (int h = 0; h < H; ++h) {
            row[h] = base + grp + NG * h;
            valid[h] = row[h] < r1;
            const int64_t rr_ = valid[h] ? row[h] : r0;
            const int64_t kb = valid[h] ? __ldg(S.rp + rr_) : 0;
            const int64_t k1 = valid[h] ? __ldg(S.rp + rr_ + 1) : 0;
            len[h] = k1 - kb;
            u0[h] = (kb + 3 * rr_ + 3) >> 2;
            u[h] = u0[h] + sub;
            uend[h] = u0[h] + ((len[h] + 3) >> 2);
            acc[h] = alo[h] = aab[h] = accf[h] = dg[h] = 0.0;
        }
        while (true) {
            bool more = false;
#pragma unroll
            for (int h = 0; h < H; ++h) more |= u[h] < uend[h];
            if (!more) break;
#pragma unroll
            for (int h = 0; h < H; ++h) {
                if (u[h] < uend[h]) {
                    const int4 cc = __ldg((const int4 *)ci + u[h]);
                    const double2 v0 = __ldg((const double2 *)va + 2 * u[h]);
                    const double2 v1 = __ldg((const double2 *)va + 2 * u[h] + 1);
                    const int32_t c[4] = {cc.x, cc.y, cc.z, cc.w};
                    const double a[4] = {v0.x, v0.y, v1.x, v1.y};
                    double xj[4];
                    bool fj[4];
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        xj[e] = NC ? __ldg(S.x + c[e]) : ldcg(S.x + c[e]);
                        fj[e] = INIT && S.fixed ? (__ldg(S.fixed + c[e]) != 0) : false;
                    }
                    const int64_t pos = (u[h] - u0[h]) * 4;
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const double ax = a[e] * xj[e];
                        dd_fma(acc[h], alo[h], a[e], xj[e]);
                        aab[h] += fabs(ax);
                        if (INIT && fj[e]) accf[h] += ax;
                        if (INIT && c[e] == row[h] && pos + e < len[h]) dg[h] = a[e];
                    }
                }
                u[h] += LPR;
            }
        }
#pragma unroll
        for (int h = 0; h < H; ++h) {
            group_sum_dd<LPR>(acc[h], alo[h]);
            aab[h] = group_sum<LPR>(aab[h]);
            if (INIT) {
                accf[h] = group_sum<LPR>(accf[h]);
                dg[h] = group_sum<LPR>(dg[h]);
            }
            if (valid[h] && sub == 0) {
                const int64_t i = row[h];
                const bool fx = S.fixed ? (__ldg(S.fixed + i) != 0) : false;
                const double bi = __ldg(S.b + i);
                const double rt = fx ? 0.0 : dd_residual(bi, acc[h], alo[h]);
                if (INIT && !fx) {
                    const double bl = bi - accf[h];
                    bb += bl * bl;
                }
                rr += rt * rt;
                if (!fx) aa += aab[h] * aab[h];
                const T rv = (T)rt;
                r[i] = rv;
                if (INIT) {
                    double iv = 0.0;
                    if (!fx) {
                        if (!(dg[h] > 0.0) || !isfinite(dg[h])) *bad = 1;
                        else iv = 1.0 / dg[h];
                    }
                    dinv[i] = (T)iv;
                }
                T zv = ldcg((const T *)S.dinv + i) * rv;   // this lane's row
                if (fx) zv = 0;
                z[i] = zv;
                rz += rv * zv;
                if (!INIT) rp += rv * ldcg(pc + i);
            }
        }
    }
    part[0] += rr;
    part[1] += INIT ? bb : (double)rp;
    part[2] += (double)rz;
    part[3] += aa;
}

template <int BS>
__device__ void phase_zero(const SysDev &S, int64_t r0, int64_t r1, int lane) {
    for (int64_t i = r0 * BS + lane; i < r1 * BS; i += 32)
        if (!(S.fixed && __ldg(S.fixed + i))) S.x[i] = 0.0;
}

// The true-residual phase of the graph scheduler's SpMV-phase kernels.
template <typename T, int BS>
__device__ __forceinline__ void run_R(const SysDev &S, const SysState *st, int64_t r0, int64_t r1,
                                   int lane, double part[4], int *bad) {
    if (BS == 1 && S.vec4)
        S.lpr == 4 ? phase_R_vec1<T, false, true, 4>(S, st, r0, r1, lane, part, bad)
                   : phase_R_vec1<T, false, true, 8>(S, st, r0, r1, lane, part, bad);
    else
        phase_R<T, BS, false, true>(S, st, r0, r1, lane, part, bad);
}

// State transition of a system once all its chunk sums are in.
__device__ void advance(const SysDev &S, SysState *st, GridBar *bar, int ph,
                        const double tot[4]) {
    const double rtol2 = S.rtol2;
    int next = PH_DONE;
    const int status_now = *(volatile int32_t *)&st->status;
    if (status_now != CFEM_OK) {
        next = PH_DONE;   // a bad Jacobi block was found
    } else if (ph == PH_INIT) {
        const double rr = tot[0], bb = tot[1], rz = tot[2];
        const double floor2 = FLOOR_TIGHT * FLOOR_TIGHT * tot[3];
        st->bb = bb;
        if (!isfinite(rr) || !isfinite(bb) || !isfinite(rz)) {
            st->status = CFEM_ERR_BREAKDOWN;
        } else if (bb == 0.0) {
            st->relres = 0.0;
            next = PH_ZERO;
        } else if (rr <= rtol2 * bb || rr <= floor2) {
            st->relres = sqrt(rr / bb);
        } else {
            st->rz = rz;
            st->beta = 0.0;
            st->zeta = 1.0;
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
            st->zeta = 1.0;
            next = PH_B;
        }
    } else if (ph == PH_B) {
        const double rz = tot[0], rr = tot[1];
        const double bb = st->bb;
        st->iter += 1;
        if (!isfinite(rz) || !isfinite(rr)) {
            st->status = CFEM_ERR_BREAKDOWN;
        } else if (rr <= rtol2 * bb || rr < S.delta2 * st->rmax2) {
            // target reached on the recursive residual, or a reliable update:
            // the recursive residual fell by delta since the last FP64 true
            // residual, which is recomputed before the two drift apart
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
        const double rr = tot[0], rp = tot[1], rz = tot[2], bb = st->bb;
        const double floor2 = FLOOR_TIGHT * FLOOR_TIGHT * tot[3];
        const double loose2 = FLOOR_C * FLOOR_C * tot[3];
        if (st->nres < S.hist_cap) {
            S.hist[2 * st->nres] = (double)st->iter;
            S.hist[2 * st->nres + 1] = sqrt(rr / bb);
        }
        st->nres += 1;
        st->relres = sqrt(rr / bb);
        if (!isfinite(rr) || !isfinite(rz)) {
            st->status = CFEM_ERR_BREAKDOWN;
        } else if (rr <= rtol2 * bb || rr <= floor2) {
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
            if (rr <= loose2 && st->stall >= 1) {
                // converged at the round-off floor
            } else if (st->stall >= S.max_stall) {
                st->status = CFEM_ERR_NOT_CONVERGED;
            } else {
                // The replaced residual is no longer orthogonal to the last
                // search direction; restore r.p' = 0 with p' = p - g z,
                // g = r.p / r.z, folded into the next p = z + beta p'.
                const double beta = rz / st->rz;
                st->beta = beta;
                st->zeta = (rz != 0.0) ? 1.0 - beta * (rp / rz) : 1.0;
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

// Chunk partial -> tile partial -> system total, each level summed in a
// fixed order by its last finisher.
__device__ void finish_chunk(const SysDev &S, SysState *st, GridBar *bar,
                             int lc, int ph, double part[4], int lane, int bad) {
#pragma unroll
    for (int v = 0; v < 4; ++v) part[v] = warp_sum(part[v]);
    const int tile = lc / TILE;
    const int tsize = min(TILE, S.nchunks - tile * TILE);
    int last = 0;
    if (lane == 0) {
#pragma unroll
        for (int v = 0; v < 4; ++v) S.partial[(int64_t)lc * 4 + v] = part[v];
        if (bad) atomicExch(&st->status, CFEM_ERR_BREAKDOWN);
        last = (atom_add_acqrel(&S.tcnt[tile], 1u) == (unsigned)tsize - 1) ? 1 : 0;
    }
    last = __shfl_sync(0xffffffffu, last, 0);
    if (!last) return;
    __threadfence();
    double t[4] = {0.0, 0.0, 0.0, 0.0};
    if (lane < tsize) {
        const int64_t c = (int64_t)tile * TILE + lane;
#pragma unroll
        for (int v = 0; v < 4; ++v) t[v] = vcg(S.partial + c * 4 + v);
    }
#pragma unroll
    for (int v = 0; v < 4; ++v) t[v] = warp_sum(t[v]);
    if (S.ntiles == 1) {            // the tile is the whole system
        if (lane == 0) {
            S.tcnt[0] = 0;
            advance(S, st, bar, ph, t);
        }
        return;
    }
    int last_sys = 0;
    if (lane == 0) {
        S.tcnt[tile] = 0;
#pragma unroll
        for (int v = 0; v < 4; ++v) S.tpartial[(int64_t)tile * 4 + v] = t[v];
        last_sys = (atom_add_acqrel(&st->cnt, 1u) == (unsigned)S.ntiles - 1) ? 1 : 0;
    }
    last_sys = __shfl_sync(0xffffffffu, last_sys, 0);
    if (!last_sys) return;
    __threadfence();
    double tot[4] = {0.0, 0.0, 0.0, 0.0};
    for (int c = lane; c < S.ntiles; c += 32)
#pragma unroll
        for (int v = 0; v < 4; ++v) tot[v] += vcg(S.tpartial + (int64_t)c * 4 + v);
#pragma unroll
    for (int v = 0; v < 4; ++v) tot[v] = warp_sum(tot[v]);
    if (lane != 0) return;
    st->cnt = 0;
    advance(S, st, bar, ph, tot);
}

// Which phases a kernel handles: INIT (k_pcg_init) or any (the persistent
// kernel; the graph scheduler's kernels run their phases themselves).
enum { RUN_INIT = 0, RUN_ALL = 1 };

// (defined with the sliced-ELL kernels below)
template <typename T>
__device__ void init_R_sell(const SysDev &S, int64_t lc, int lane, double part[4], int *bad);

template <typename T, int BS, int RUN>
__device__ void run_chunk(const SysDev &S, SysState *st, GridBar *bar, int ph,
                          int lc, int lane) {
    const int64_t r0 = (int64_t)lc * S.crows;
    const int64_t r1 = min(S.n, r0 + S.crows);
    double part[4] = {0.0, 0.0, 0.0, 0.0};
    int bad = 0;
    if (RUN == RUN_INIT) {
        int flag = 0;
        // (x is not written while the residual is initialised: L1 gathers)
        if (BS == 1 && S.rsell)
            init_R_sell<T>(S, lc, lane, part, &flag);
        else if (BS == 1 && S.vec4)
            S.lpr == 4 ? phase_R_vec1<T, true, true, 4>(S, st, r0, r1, lane, part, &flag)
                       : phase_R_vec1<T, true, true, 8>(S, st, r0, r1, lane, part, &flag);
        else
            phase_R<T, BS, true>(S, st, r0, r1, lane, part, &flag);
        bad = __any_sync(0xffffffffu, flag != 0);
    } else {
        switch (ph) {
            case PH_A:
                if (sizeof(T) == 4) phase_A<T, BS, true, 2>(S, st, r0, r1, lane, part);
                else phase_A<T, BS, false, 1>(S, st, r0, r1, lane, part);
                break;
            case PH_B: phase_B<T, BS>(S, st, r0, r1, lane, part); break;
            case PH_R: phase_R<T, BS, false>(S, st, r0, r1, lane, part, &bad); break;
            default: phase_zero<BS>(S, r0, r1, lane); break;
        }
    }
    finish_chunk(S, st, bar, lc, ph, part, lane, bad);
}

template <int RUN>
__device__ __forceinline__ void dispatch(const SysDev *__restrict__ sys,
                                         SysState *st, GridBar *bar,
                                         const int32_t *__restrict__ chunk_sys,
                                         int c, int lane) {
    const int s = __ldg(chunk_sys + c);
    const SysDev &S = sys[s];
    const int ph = RUN == RUN_INIT ? PH_INIT : *(volatile int32_t *)&st[s].phase;
    if (ph == PH_DONE) return;
    const int lc = c - S.chunk0;
    if (lc >= S.nchunks) return;   // a solve slot holding a smaller system
    if (S.mode == CFEM_SOLVE_MIXED) {
        if (S.bs == 3) run_chunk<float, 3, RUN>(S, &st[s], bar, ph, lc, lane);
        else run_chunk<float, 1, RUN>(S, &st[s], bar, ph, lc, lane);
    } else {
        if (S.bs == 3) run_chunk<double, 3, RUN>(S, &st[s], bar, ph, lc, lane);
        else run_chunk<double, 1, RUN>(S, &st[s], bar, ph, lc, lane);
    }
}

// INIT: one ordinary launch, one warp per chunk.
__global__ void __launch_bounds__(256)
k_pcg_init(const SysDev *__restrict__ sys, SysState *st,
           const int32_t *__restrict__ chunk_sys, int n_chunks, GridBar *bar) {
    const int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (c >= n_chunks) return;
    dispatch<RUN_INIT>(sys, st, bar, chunk_sys, c, threadIdx.x & 31);
}

__global__ void __launch_bounds__(SOLVE_THREADS, 1)
k_pcg_persistent(const SysDev *__restrict__ sys, SysState *st,
                 const int32_t *__restrict__ chunk_sys, int n_chunks,
                 GridBar *bar, int max_steps, unsigned long long timeout_ns,
                 unsigned hold) {
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    if (*(volatile int *)&bar->active <= 0) return;
    for (int step = 0; step < max_steps; ++step) {
        for (int c = gw; c < n_chunks; c += nw)
            dispatch<RUN_ALL>(sys, st, bar, chunk_sys, c, lane);
        if (!grid_sync(bar, timeout_ns, hold)) return;
        if (*(volatile int *)&bar->active <= 0) return;
    }
}

// FP32 difference-form operator: off-diagonal blocks rounded, the diagonal
// slot holding the rounded FP64 block row sum (see phase_A). A group of
// MX = 8 lanes per (block) row: lane s takes entries s, s + 8, ... (loads
// and stores coalesced along the row), the FP64 sums meet in a fixed
// shuffle tree, so every launch shape gives the same bits.
constexpr int MX = 8;

template <int BS>
__device__ __forceinline__ void mixed_row(const int32_t *__restrict__ rp,
                                          const int32_t *__restrict__ ci,
                                          const double *__restrict__ v64,
                                          float *__restrict__ v32, int64_t r, bool valid,
                                          int sub) {
    constexpr int B2 = BS * BS;
    double sum[B2];
#pragma unroll
    for (int e = 0; e < B2; ++e) sum[e] = 0.0;
    int32_t kd = -1;
    if (valid) {
        for (int32_t k = rp[r] + sub; k < rp[r + 1]; k += MX) {
            if (ci[k] == r) kd = k;
#pragma unroll
            for (int e = 0; e < B2; ++e) {
                const double a = v64[(int64_t)k * B2 + e];
                sum[e] += a;
                v32[(int64_t)k * B2 + e] = (float)a;
            }
        }
    }
#pragma unroll
    for (int o = MX / 2; o > 0; o >>= 1) {
        kd = max(kd, __shfl_xor_sync(0xffffffffu, kd, o));
#pragma unroll
        for (int e = 0; e < B2; ++e) sum[e] += __shfl_xor_sync(0xffffffffu, sum[e], o);
    }
    __syncwarp();   // the off-diagonal stores above before the diagonal's
    if (valid && kd >= 0)
#pragma unroll
        for (int e = 0; e < B2; ++e)
            if (e % MX == sub) v32[(int64_t)kd * B2 + e] = (float)sum[e];
}

template <int BS>
__global__ void k_mixed_matrix(int64_t n, const int32_t *__restrict__ rp,
                               const int32_t *__restrict__ ci,
                               const double *__restrict__ v64,
                               float *__restrict__ v32) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t r = t / MX;
    mixed_row<BS>(rp, ci, v64, v32, r, r < n, (int)(t % MX));
}

// k_mixed_matrix over many systems of one block size in one launch: job j
// covers global rows [row0_j, row0_j + n_j); a thread per row finds its
// job by binary search.
struct MixJob {
    int64_t row0, n;
    const int32_t *rp, *ci;
    const double *v64;
    float *v32;
};

template <int BS>
__global__ void k_mixed_matrix_batch(const MixJob *__restrict__ jobs, int nj, int64_t total) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t g = t / MX;
    const bool valid = g < total;
    int lo = 0;
    if (valid) {
        int hi = nj - 1;
        while (lo < hi) {   // last job with row0 <= g
            const int mid = (lo + hi + 1) >> 1;
            if (jobs[mid].row0 <= g) lo = mid; else hi = mid - 1;
        }
    }
    const MixJob &J = jobs[lo];
    mixed_row<BS>(J.rp, J.ci, J.v64, J.v32, valid ? g - J.row0 : 0, valid, (int)(t % MX));
}


// Lean SpMV phase for the graph scheduler: one block row per group of
// LANES lanes, one row in flight per group, few registers so that many
// warps are resident and hide the gather latency. Block values are read
// from an entry-major copy (vsoa[e * nnzb + k]) so that the lanes of a
// group read consecutive addresses for every entry e. The new direction
// p = zeta z + beta p_old is formed at every gathered entry (z and p_old are
// read-only for the whole launch, so their gathers go through the L1/texture
// path; neighbouring rows of a block share most of their columns) and
// written for the block's own rows.
template <typename T, int BS, bool DIFF>
__device__ void phase_A_lean(const SysDev &S, const SysState *st, int64_t r0,
                             int64_t r1, int lane, double part[4]) {
    const T beta = (T)vcg(&st->beta);
    const T zeta = (T)vcg(&st->zeta);
    const int pbuf = vcgi(&st->pbuf);
    const T *pin = (const T *)(pbuf ? S.p1 : S.p0);
    T *pout = (T *)(pbuf ? S.p0 : S.p1);
    const T *z = (const T *)S.z;
    T *q = (T *)S.q;
    const T *va = (const T *)S.vsoa;
    const int64_t ld = S.nnzb;
    const int sub = lane & (LANES - 1), grp = lane / LANES;
    T pq = 0;
    for (int64_t base = r0; base < r1; base += RPP) {
        const int64_t row = base + grp;
        const bool valid = row < r1;
        const int64_t rr = valid ? row : r0;
        T pi[BS], acc[BS];
#pragma unroll
        for (int c = 0; c < BS; ++c) {
            pi[c] = zeta * __ldg(z + rr * BS + c) + beta * __ldg(pin + rr * BS + c);
            acc[c] = 0;
        }
        const int32_t kb = valid ? __ldg(S.rp + rr) : 0;
        const int32_t k1 = valid ? __ldg(S.rp + rr + 1) : 0;
        // software pipeline: the next block's index and values are loaded
        // while the current block's gathers are in flight
        int32_t k = kb + sub;
        bool on = k < k1;
        int32_t kk = on ? k : 0;
        int64_t j = __ldg(S.ci + kk);
        T a[BS * BS];
#pragma unroll
        for (int e = 0; e < BS * BS; ++e) a[e] = __ldg(va + (int64_t)e * ld + kk);
        while (on) {
            T pj[BS];
#pragma unroll
            for (int d = 0; d < BS; ++d) {
                pj[d] = zeta * __ldg(z + j * BS + d) + beta * __ldg(pin + j * BS + d);
                if (DIFF) pj[d] = (j == rr) ? pi[d] : pj[d] - pi[d];
            }
            const int32_t k2 = k + LANES;
            const bool on2 = k2 < k1;
            const int32_t kk2 = on2 ? k2 : 0;
            const int64_t j2 = __ldg(S.ci + kk2);
            T a2[BS * BS];
#pragma unroll
            for (int e = 0; e < BS * BS; ++e) a2[e] = __ldg(va + (int64_t)e * ld + kk2);
#pragma unroll
            for (int c = 0; c < BS; ++c)
#pragma unroll
                for (int d = 0; d < BS; ++d) acc[c] += a[c * BS + d] * pj[d];
            j = j2;
#pragma unroll
            for (int e = 0; e < BS * BS; ++e) a[e] = a2[e];
            k = k2;
            on = on2;
        }
#pragma unroll
        for (int c = 0; c < BS; ++c) acc[c] = group_sum<LANES>(acc[c]);
        if (valid && sub == 0) {
#pragma unroll
            for (int c = 0; c < BS; ++c) {
                const int64_t i = row * BS + c;
                pout[i] = pi[c];
                q[i] = acc[c];
                pq += pi[c] * acc[c];
            }
        }
    }
    part[0] += (double)pq;
}

// Scalar rows (bs 1) from the unit-padded copy: each lane of a group of 8
// reads whole units of four entries (one 16-byte column load and one (FP32)
// or two (FP64) 16-byte value loads), so a row of up to 32 entries takes one
// step with no per-entry masking; each group keeps H rows in flight. Lanes
// without a unit use column = own row and coefficient 0.
template <typename T, bool DIFF, int H>
__device__ void phase_A_vec1(const SysDev &S, const SysState *st, int64_t r0,
                             int64_t r1, int lane, double part[4]) {
    const int pbuf = vcgi(&st->pbuf);
    const T *pv = (const T *)(pbuf ? S.p0 : S.p1);   // this iteration's p (k_gp)
    T *q = (T *)S.q;
    const T *va = (const T *)S.va4;
    const int32_t *ci = S.ci4;
    const int sub = lane & 7, grp = lane >> 3;
    T pq = 0;
    for (int64_t base = r0; base < r1; base += 4 * H) {
        int64_t row[H], rr[H], u[H], uend[H];
        bool valid[H];
        T pi[H], acc[H];
#pragma unroll
        for (int h = 0; h < H; ++h) {
            row[h] = base + grp + 4 * h;
            valid[h] = row[h] < r1;
            rr[h] = valid[h] ? row[h] : r0;
            pi[h] = __ldg(pv + rr[h]);
            acc[h] = 0;
            const int64_t kb = valid[h] ? __ldg(S.rp + rr[h]) : 0;
            const int64_t k1 = valid[h] ? __ldg(S.rp + rr[h] + 1) : 0;
            const int64_t u0 = (kb + 3 * rr[h] + 3) >> 2;
            u[h] = u0 + sub;
            uend[h] = u0 + ((k1 - kb + 3) >> 2);
        }
        while (true) {
            bool more = false;
#pragma unroll
            for (int h = 0; h < H; ++h) more |= u[h] < uend[h];
            if (!more) break;
            int32_t c[H][4];
            T a[H][4];
#pragma unroll
            for (int h = 0; h < H; ++h) {
                if (u[h] < uend[h]) {
                    const int4 cc = __ldg((const int4 *)ci + u[h]);
                    c[h][0] = cc.x; c[h][1] = cc.y; c[h][2] = cc.z; c[h][3] = cc.w;
                    if (sizeof(T) == 4) {
                        const float4 vv = __ldg((const float4 *)va + u[h]);
                        a[h][0] = (T)vv.x; a[h][1] = (T)vv.y; a[h][2] = (T)vv.z; a[h][3] = (T)vv.w;
                    } else {
                        const double2 v0 = __ldg((const double2 *)va + 2 * u[h]);
                        const double2 v1 = __ldg((const double2 *)va + 2 * u[h] + 1);
                        a[h][0] = (T)v0.x; a[h][1] = (T)v0.y; a[h][2] = (T)v1.x; a[h][3] = (T)v1.y;
                    }
                } else {
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        c[h][e] = (int32_t)rr[h];
                        a[h][e] = 0;
                    }
                }
            }
            T pj[H][4];
#pragma unroll
            for (int h = 0; h < H; ++h)
#pragma unroll
                for (int e = 0; e < 4; ++e) pj[h][e] = __ldg(pv + c[h][e]);
#pragma unroll
            for (int h = 0; h < H; ++h) {
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    T v = pj[h][e];
                    if (DIFF) v = (c[h][e] == rr[h]) ? pi[h] : v - pi[h];
                    acc[h] += a[h][e] * v;
                }
                u[h] += 8;
            }
        }
#pragma unroll
        for (int h = 0; h < H; ++h) {
            acc[h] = group_sum<8>(acc[h]);
            if (valid[h] && sub == 0) {
                q[row[h]] = acc[h];
                pq += pi[h] * acc[h];
            }
        }
    }
    part[0] += (double)pq;
}

// Unit-padded copy of a scalar CSR matrix for phase_A_vec1, phase_R_vec1
// and phase_A_staged: one warp per row, lanes writing consecutive entries.
// The diagonal entry, when the row has one, moves to the row's first slot
// (the others keep their order): the staged difference-form SpMV takes the
// row sum from there instead of testing every column against the row.
// All systems of a plan in one launch: job j covers global rows
// [row0_j, row0_j + n_j); one warp per row finds its job by binary search
// and writes the row's columns once and its FP32 and / or FP64 values
// (either may be absent).
struct PadJob {
    int64_t row0, n;
    const int32_t *rp, *ci;
    const float *v32;
    float *va4;
    const double *v64;
    double *va4d;
    int32_t *ci4;
};

__global__ void k_pad4_batch(const PadJob *__restrict__ jobs, int nj, int64_t total) {
    // 8 lanes per row, four rows per warp step (more rows' loads in flight)
    const int lane = threadIdx.x & 31, sub = lane & 7, grp = lane >> 3;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t g0 = ((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5) * 4; g0 < total;
         g0 += nw * 4) {
        const int64_t g = g0 + grp;
        const bool valid = g < total;
        int lo = 0;
        if (valid) {
            int hi = nj - 1;
            while (lo < hi) {   // last job with row0 <= g
                const int mid = (lo + hi + 1) >> 1;
                if (jobs[mid].row0 <= g) lo = mid; else hi = mid - 1;
            }
        }
        const PadJob &J = jobs[lo];
        const int64_t i = valid ? g - J.row0 : 0;
        const int64_t kb = valid ? J.rp[i] : 0, len = valid ? J.rp[i + 1] - kb : 0;
        // position of the diagonal entry (the first, should a row repeat it)
        int64_t dpos = INT64_MAX;
        for (int64_t t = sub; t < len; t += 8)
            if (J.ci[kb + t] == (int32_t)i && t < dpos) dpos = t;
#pragma unroll
        for (int o = 4; o > 0; o >>= 1) {
            const int64_t other = __shfl_xor_sync(0xffffffffu, dpos, o);
            dpos = other < dpos ? other : dpos;
        }
        if (dpos == INT64_MAX) dpos = -1;
        const int64_t o = ((kb + 3 * i + 3) >> 2) * 4;
        const int64_t m = valid ? ((len + 3) >> 2) * 4 : 0;
        for (int64_t t = sub; t < m; t += 8) {
            // slot t <- entry src: diagonal first, then the others in order
            const int64_t src = dpos < 0 ? t : (t == 0 ? dpos : (t <= dpos ? t - 1 : t));
            J.ci4[o + t] = t < len ? J.ci[kb + src] : (int32_t)i;
            if (J.va4) J.va4[o + t] = t < len ? J.v32[kb + src] : 0.0f;
            if (J.va4d) J.va4d[o + t] = t < len ? J.v64[kb + src] : 0.0;
        }
    }
}

// ---------------------------------------------------------------------------
// Bulk-staged scalar SpMV (graph scheduler, A phase of scalar systems).
// A warp owns one work entry of up to XR_MAX rows. Their units (16-byte
// groups of four entries) in the unit-padded copy (row i starting at unit
// (rp[i] + 3 i + 3) / 4, padding entries with column i and value 0) are one
// contiguous span, which the warp streams through two shared-memory windows
// of at most W units with 1-D bulk copies (cp.async.bulk, the TMA engine,
// completing on a transaction mbarrier): the copy of window k+1 is in
// flight while the rows of window k are multiplied, so the HBM stream no
// longer waits on the dependent gathers. Every row starts on a unit, so
// lanes read whole units with 128-bit shared-memory loads and need no
// per-entry bounds tests; LPR lanes share a row (4 for rows of up to 16
// entries, 8 above), lane s taking units s, s + LPR, .... Windows hold a
// whole number of row steps (32 / LPR groups x H rows) except at the end of
// the work entry. A row longer than a window is multiplied by the whole
// warp straight from global memory. Window bounds depend only on the
// system's row pointers, so sums are the same alone and in any batch. Every
// barrier wait is bounded (2 s); on expiry the warp records an error, waits
// (bounded) for its other copy and stops.
constexpr int XR_MAX = 128;    // rows of one staged work entry (X_CHUNKS_VEC * 16)

struct alignas(16) DUnit {     // four FP64 values
    double2 lo, hi;
};
template <typename TV> struct ValUnit;
template <> struct ValUnit<float> { using type = float4; };
template <> struct ValUnit<double> { using type = DUnit; };

template <typename TV, int W, int NB>
struct StageWarp {
    int2 row[XR_MAX + 4];                       // per row: first unit (from the
                                                // entry's first), unit count
    unsigned long long mbar[NB];                // one transaction barrier per buffer
    int4 c[NB][W];                              // column units
    typename ValUnit<TV>::type v[NB][W];        // value units
};

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long *m) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(m)) : "memory");
}
// Initialised barriers visible to the async (bulk-copy) proxy.
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect(unsigned long long *m, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(m)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_test(unsigned long long *m, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(m)), "r"(parity)
        : "memory");
    return done != 0;
}
// Wait for the phase of the given parity to complete; false after 2 s, or
// when another warp has already recorded an error in *err. The clock and
// the error word are read every 64 tests only, so that a completed phase is
// seen as soon as possible.
__device__ bool mbar_wait(unsigned long long *m, uint32_t parity, const int *err) {
    if (mbar_test(m, parity)) return true;
    const unsigned long long t0 = globaltimer();
    for (unsigned it = 1;; ++it) {
        if (mbar_test(m, parity)) return true;
        if ((it & 63) == 0 &&
            (globaltimer() - t0 > 2000000000ull || *(volatile const int *)err))
            return false;
    }
}
// 1-D bulk copy global -> this CTA's shared memory, completing on m.
// dst and src 16-byte aligned, bytes a non-zero multiple of 16.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes,
                                          unsigned long long *m) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(m))
        : "memory");
}

// The same bulk copy with an L2 evict-first policy: the matrix stream of an
// SpMV passes through L2 once, so it should not push out the vectors the
// gathers reread (p of a large batch is tens of MB).
#ifndef CFEM_L2_EVICT_FIRST
#define CFEM_L2_EVICT_FIRST 1
#endif
__device__ __forceinline__ void bulk_load_stream(void *dst, const void *src, uint32_t bytes,
                                                 unsigned long long *m) {
#if CFEM_L2_EVICT_FIRST
    unsigned long long pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
        " [%0], [%1], %2, [%3], %4;" ::"r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(m)), "l"(pol)
        : "memory");
#else
    bulk_load(dst, src, bytes, m);
#endif
}

// First unit of global row i whose entries start at kb (unit-padded copy).
__device__ __forceinline__ int64_t unit_start(int64_t kb, int64_t i) { return (kb + 3 * i + 3) >> 2; }

// One window: rows [a, b) of the work entry, staged in buffer buf (-1: the
// single long row a, read from global memory); unit ub (counted from the
// entry's first unit) sits at index 0 of the buffer.
struct StageWin {
    int a, b, buf, ub;
};

// Open the window starting at row a (warp-uniform; every lane calls): pick
// its rows and start the bulk copies of their units on the buffer's barrier.
// e0: the entry's first unit in the copy; SR: rows per processing step.
template <typename TV, int W, int NB, int SR>
__device__ __forceinline__ StageWin stage_open(StageWarp<TV, W, NB> &sm, const int32_t *ci4,
                                               const TV *va4, int64_t e0, int a, int nr,
                                               int lane, int &nbuf) {
    StageWin w;
    w.a = a;
    w.ub = sm.row[a].x;
    const int lim = w.ub + W;
    int b = a;
    for (int t0 = a + 1; t0 <= nr; t0 += 32) {
        const int t = t0 + lane;
        // unit starts do not decrease: the rows that fit are a prefix
        const unsigned m = __ballot_sync(0xffffffffu, t <= nr && sm.row[t].x <= lim);
        if (m) b = t0 + __popc(m) - 1;
        if (m != 0xffffffffu) break;
    }
    if (b == a) {   // row a alone is longer than a window
        w.b = a + 1;
        w.buf = -1;
        return w;
    }
    if (b < nr && b - a >= SR) b = a + (b - a) / SR * SR;   // whole steps
    w.b = b;
    w.buf = nbuf;
    nbuf = nbuf + 1 == NB ? 0 : nbuf + 1;   // buffers in turn: the oldest is free
    const uint32_t nu = (uint32_t)(sm.row[b].x - w.ub);
    if (lane == 0) {
        // earlier generic reads of this buffer before the async-proxy writes
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        const uint32_t bc = nu * 16u, bv = nu * 4u * (uint32_t)sizeof(TV);
        mbar_expect(&sm.mbar[w.buf], bc + bv);
        if (nu) {
            const int64_t u = e0 + w.ub;
            bulk_load_stream(&sm.c[w.buf][0], ci4 + 4 * u, bc, &sm.mbar[w.buf]);
            bulk_load_stream(&sm.v[w.buf][0], va4 + 4 * u, bv, &sm.mbar[w.buf]);
        }
    }
    return w;
}

__device__ __forceinline__ void unit_vals(const float4 &u, float a[4]) {
    a[0] = u.x; a[1] = u.y; a[2] = u.z; a[3] = u.w;
}
__device__ __forceinline__ void unit_vals(const DUnit &u, double a[4]) {
    a[0] = u.lo.x; a[1] = u.lo.y; a[2] = u.hi.x; a[3] = u.hi.y;
}

// q = A p and p.q over rows [r0, r1) of one scalar system (A phase), the
// unit-padded matrix streamed through the warp's staging windows. DIFF: the
// FP32 difference-form operator, q_i = s_i p_i + sum_j a_ij (p_j - p_i) with
// the row sum s_i in the diagonal slot, which the padded copy puts first in
// the row: every slot is applied as a (p_j - p_i) (the diagonal then adds
// nothing) and the lane holding the row's first unit adds s_i p_i. Padding
// slots (column i, value 0) add nothing either way.
template <typename T, bool DIFF, int W, int NB, int H, int LPR>
__device__ void phase_A_staged(const SysDev &S, const SysState *st, int64_t r0, int64_t r1,
                               int lane, double part[4], StageWarp<T, W, NB> &sm,
                               const int *err, int *fail) {
    constexpr int NG = 32 / LPR, SR = NG * H;
    using VU = typename ValUnit<T>::type;
    const int pbuf = vcgi(&st->pbuf);
    const T *pv = (const T *)(pbuf ? S.p0 : S.p1);   // this iteration's p (k_gp)
    T *q = (T *)S.q;
    const T *va4 = (const T *)S.va4;
    const int32_t *ci4 = S.ci4;
    const int nr = (int)(r1 - r0);
    const int sub = lane % LPR, grp = lane / LPR;
    const int64_t e0 = unit_start(__ldg(S.rp + r0), r0);   // the entry's first unit
    T pq = 0;
    for (int t = lane; t <= nr; t += 32) {
        const int64_t kb = __ldg(S.rp + r0 + t);
        const int len = t < nr ? __ldg(S.rp + r0 + t + 1) - (int)kb : 0;
        sm.row[t] = make_int2((int)(unit_start(kb, r0 + t) - e0), (len + 3) >> 2);
    }
    if (lane == 0) {
#pragma unroll
        for (int b = 0; b < NB; ++b) mbar_init(&sm.mbar[b]);
        mbar_init_fence();
    }
    __syncwarp();
    int nbuf = 0;
    uint32_t par = 0;   // bit b: parity of buffer b's next phase
    // windows in order: wq[0] is multiplied while the copies of wq[1..NB-1]
    // are in flight
    StageWin wq[NB];
#pragma unroll
    for (int k = 0; k < NB; ++k) {
        const int a = k == 0 ? 0 : wq[k - 1].b;
        if (a < nr) {
            wq[k] = stage_open<T, W, NB, SR>(sm, ci4, va4, e0, a, nr, lane, nbuf);
        } else {
            wq[k].a = wq[k].b = nr;
            wq[k].buf = -1;
            wq[k].ub = 0;
        }
    }
    while (wq[0].a < nr) {
        const StageWin w = wq[0];
        if (w.buf >= 0) {
            const bool ok = mbar_wait(&sm.mbar[w.buf], (par >> w.buf) & 1u, err);
            par ^= 1u << w.buf;
            if (!__all_sync(0xffffffffu, ok)) {
                // this window's copy and the later ones may still be in
                // flight: bounded waits (this window's parity bit has
                // already been advanced)
#pragma unroll
                for (int k = 0; k < NB; ++k)
                    if (wq[k].buf >= 0) {
                        const uint32_t ph = ((par >> wq[k].buf) & 1u) ^ (k == 0 ? 1u : 0u);
                        const unsigned long long t0 = globaltimer();
                        while (!mbar_test(&sm.mbar[wq[k].buf], ph) &&
                               globaltimer() - t0 < 2000000000ull) {
                        }
                    }
                *fail = 1;
                break;
            }
            const int4 *cs = sm.c[w.buf];
            const VU *vs = sm.v[w.buf];
            for (int base = w.a; base < w.b; base += SR) {
                int rl[H], u[H], ue[H];
                T pi[H], acc[H], dg[H];
#pragma unroll
                for (int h = 0; h < H; ++h) {
                    rl[h] = base + grp + NG * h;
                    const bool valid = rl[h] < w.b;
                    const int rr = valid ? rl[h] : w.a;
                    const int2 ri = sm.row[rr];
                    u[h] = ri.x - w.ub + sub;
                    ue[h] = valid ? ri.x - w.ub + ri.y : 0;
                    pi[h] = __ldg(pv + r0 + rr);
                    acc[h] = 0;
                    dg[h] = 0;
                }
                bool first = true;
                while (true) {
                    bool more = false;
#pragma unroll
                    for (int h = 0; h < H; ++h) more |= u[h] < ue[h];
                    if (!more) break;
                    // columns, then the gathers, then the values: fewer
                    // registers live across the gathers
                    int4 cc[H];
#pragma unroll
                    for (int h = 0; h < H; ++h)
                        if (u[h] < ue[h]) cc[h] = cs[u[h]];
                    T pj[H][4];
#pragma unroll
                    for (int h = 0; h < H; ++h) {
                        const bool on = u[h] < ue[h];
                        pj[h][0] = on ? __ldg(pv + cc[h].x) : (T)0;
                        pj[h][1] = on ? __ldg(pv + cc[h].y) : (T)0;
                        pj[h][2] = on ? __ldg(pv + cc[h].z) : (T)0;
                        pj[h][3] = on ? __ldg(pv + cc[h].w) : (T)0;
                    }
                    VU vv[H];
#pragma unroll
                    for (int h = 0; h < H; ++h)
                        if (u[h] < ue[h]) vv[h] = vs[u[h]];
#pragma unroll
                    for (int h = 0; h < H; ++h) {
                        if (u[h] < ue[h]) {
                            T a[4];
                            unit_vals(vv[h], a);
                            if (DIFF && first && sub == 0) dg[h] = a[0];
#pragma unroll
                            for (int e = 0; e < 4; ++e)
                                acc[h] += a[e] * (DIFF ? pj[h][e] - pi[h] : pj[h][e]);
                        }
                        u[h] += LPR;
                    }
                    first = false;
                }
#pragma unroll
                for (int h = 0; h < H; ++h) {
                    if (DIFF) acc[h] += dg[h] * pi[h];   // s_i p_i, lane sub == 0 only
                    acc[h] = group_sum<LPR>(acc[h]);
                    if (rl[h] < w.b && sub == 0) {
                        q[r0 + rl[h]] = acc[h];
                        pq += pi[h] * acc[h];
                    }
                }
            }
            __syncwarp();   // reads done before the buffer is refilled
        } else {
            const int64_t row = r0 + w.a;
            const int64_t u0 = e0 + sm.row[w.a].x, nu = sm.row[w.a].y;
            const T pi = __ldg(pv + row);
            T acc = 0;
            for (int64_t uu = lane; uu < nu; uu += 32) {
                const int4 cc = __ldg((const int4 *)ci4 + u0 + uu);
                T a[4];
                if (sizeof(T) == 4) {
                    const float4 f = __ldg((const float4 *)va4 + u0 + uu);
                    a[0] = (T)f.x; a[1] = (T)f.y; a[2] = (T)f.z; a[3] = (T)f.w;
                } else {
                    const double2 d0 = __ldg((const double2 *)va4 + 2 * (u0 + uu));
                    const double2 d1 = __ldg((const double2 *)va4 + 2 * (u0 + uu) + 1);
                    a[0] = (T)d0.x; a[1] = (T)d0.y; a[2] = (T)d1.x; a[3] = (T)d1.y;
                }
                const int c4[4] = {cc.x, cc.y, cc.z, cc.w};
#pragma unroll
                for (int e = 0; e < 4; ++e) acc += a[e] * (DIFF ? __ldg(pv + c4[e]) - pi : __ldg(pv + c4[e]));
                if (DIFF && uu == 0) acc += a[0] * pi;   // the diagonal slot, first
            }
            acc = group_sum<32>(acc);
            if (lane == 0) {
                q[row] = acc;
                pq += pi * acc;
            }
        }
#pragma unroll
        for (int k = 0; k + 1 < NB; ++k) wq[k] = wq[k + 1];
        if (wq[NB - 2].b < nr) {
            wq[NB - 1] = stage_open<T, W, NB, SR>(sm, ci4, va4, e0, wq[NB - 2].b, nr, lane, nbuf);
        } else {
            wq[NB - 1].a = wq[NB - 1].b = nr;
            wq[NB - 1].buf = -1;
            wq[NB - 1].ub = 0;
        }
    }
    part[0] += (double)pq;
}

// ---------------------------------------------------------------------------
// Bulk-staged 3x3-block SpMV (graph scheduler, A phase of 3x3 systems).
// Working copy: block rows padded to whole units of 4 blocks, row i starting
// at unit (rp[i] + 3 i + 3) / 4 (padding: column i, zero block), columns in
// one array and row-major block values (9 per slot) in another, so a work
// entry's rows are one contiguous span of units. Block rows of an elasticity
// pattern run from 10 to 65 blocks (76 B each in FP64), so windows cannot
// hold whole rows within the shared memory three blocks per SM leave;
// instead the span is cut into fixed windows of W units, streamed through
// two buffers with 1-D bulk copies (the next window in flight while the
// current one is used), and a row may straddle windows: the warp takes one
// block row at a time, lane l the row's blocks l, l+32, ... (two in flight
// in FP32, one in FP64 within 80 registers), and carries
// its three sums in registers from one window to the next. The new
// direction p = zeta z + beta p_old is formed at every gathered block (as
// the register path does) and written for the row's own DOFs. Waits are
// bounded as in the scalar staged SpMV.
constexpr int XR3 = 8;    // block rows of one 3x3 work entry (one chunk)

template <typename TV, int W>
struct Stage3Warp {
    int2 row[XR3 + 4];                // per row: first slot (from the entry's first), blocks
    unsigned long long mbar[2];       // one transaction barrier per buffer
    int4 c[2][W];                     // block columns, 4 per unit
    TV v[2][W * 36];                  // block values, 36 per unit
};

// Padded 3x3 working copy (one warp per block row, consecutive writes).
template <typename T>
__global__ void k_pad3(int64_t n, const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
                       const T *__restrict__ v, int32_t *__restrict__ c3, T *__restrict__ v3) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
        const int64_t kb = rp[i], len = rp[i + 1] - kb;
        const int64_t o = ((kb + 3 * i + 3) >> 2) * 4;
        const int64_t m = ((len + 3) >> 2) * 4;
        for (int64_t t = lane; t < m; t += 32) c3[o + t] = t < len ? ci[kb + t] : (int32_t)i;
        for (int64_t t = lane; t < 9 * m; t += 32) v3[9 * o + t] = t < 9 * len ? v[9 * kb + t] : (T)0;
    }
}

// Start the copy of window k (units [e0 + k W, min(e0 + (k+1) W, e1))) into
// buffer k & 1; lane 0 only.
template <typename TV, int W>
__device__ __forceinline__ void stage3_issue(Stage3Warp<TV, W> &sm, const int32_t *c3,
                                             const TV *v3, int64_t e0, int64_t e1, int k) {
    const int b = k & 1;
    const int64_t u0 = e0 + (int64_t)k * W;
    const int64_t u1 = min(e1, u0 + W);
    const uint32_t nu = (uint32_t)(u1 - u0);
    const uint32_t bc = nu * 16u, bv = nu * 36u * (uint32_t)sizeof(TV);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect(&sm.mbar[b], bc + bv);
    if (nu) {
        bulk_load_stream(&sm.c[b][0], c3 + 4 * u0, bc, &sm.mbar[b]);
        bulk_load_stream(&sm.v[b][0], v3 + 36 * u0, bv, &sm.mbar[b]);
    }
}

// q = A p, p = zeta z + beta p_old written for the rows, and p.q over block
// rows [r0, r1) (at most XR3) of one 3x3 system. DIFF: the FP32
// difference-form operator (off-diagonal blocks applied to p_j - p_i).
template <typename T, bool DIFF, int W>
__device__ void phase_A3_staged(const SysDev &S, const SysState *st, int64_t r0, int64_t r1,
                                int lane, double part[4], Stage3Warp<T, W> &sm,
                                const int *err, int *fail) {
    constexpr int HB = sizeof(T) == 8 ? 1 : 2;   // blocks per lane in flight
    const T beta = (T)vcg(&st->beta);
    const T zeta = (T)vcg(&st->zeta);
    const int pbuf = vcgi(&st->pbuf);
    const T *pin = (const T *)(pbuf ? S.p1 : S.p0);
    T *pout = (T *)(pbuf ? S.p0 : S.p1);
    const T *z = (const T *)S.z;
    T *q = (T *)S.q;
    const int32_t *c3 = S.c3;
    const T *v3 = (const T *)S.v3;
    const int nr = (int)(r1 - r0);
    const int64_t e0 = unit_start(__ldg(S.rp + r0), r0);   // the entry's first unit
    const int64_t e1 = unit_start(__ldg(S.rp + r1), r1);   // the next entry's first
    const int nwin = (int)((e1 - e0 + W - 1) / W);
    for (int t = lane; t < nr; t += 32) {
        const int64_t kb = __ldg(S.rp + r0 + t);
        const int len = __ldg(S.rp + r0 + t + 1) - (int)kb;
        sm.row[t] = make_int2((int)(4 * (unit_start(kb, r0 + t) - e0)), len);
    }
    if (lane == 0) {
        mbar_init(&sm.mbar[0]);
        mbar_init(&sm.mbar[1]);
        mbar_init_fence();
        if (nwin > 0) stage3_issue(sm, c3, v3, e0, e1, 0);
        if (nwin > 1) stage3_issue(sm, c3, v3, e0, e1, 1);
    }
    __syncwarp();
    // window k sits in buffer k & 1 and is that buffer's (k >> 1)-th use:
    // its barrier phase has parity (k >> 1) & 1
    int cur = 0;        // window in use
    bool ok = true;
    if (nwin > 0) ok = mbar_wait(&sm.mbar[0], 0u, err);
    ok = __all_sync(0xffffffffu, ok);
    T pq = 0;
    for (int t = 0; t < nr && ok; ++t) {
        const int64_t i = r0 + t;
        const int2 ri = sm.row[t];
        T pi[3], acc[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            pi[c] = zeta * __ldg(z + 3 * i + c) + beta * __ldg(pin + 3 * i + c);
            acc[c] = 0;
        }
        int done = 0;   // blocks of the row already multiplied
        while (true) {
            const int wlo = 4 * W * cur;
            const int tend = min(ri.y, wlo + 4 * W - ri.x);   // row blocks in this window
            const int32_t *cs = (const int32_t *)sm.c[cur & 1];
            const T *vs = sm.v[cur & 1];
            for (int b0 = lane; b0 < tend; b0 += 32 * HB) {
                // HB blocks per lane in flight: b0, b0 + 32, ...
                int col[HB], sl[HB];
                bool on[HB];
#pragma unroll
                for (int h = 0; h < HB; ++h) {
                    const int b = b0 + 32 * h;
                    on[h] = b >= done && b < tend;
                    sl[h] = ri.x + b - wlo;
                    col[h] = on[h] ? cs[sl[h]] : (int)i;
                }
                T pj[HB][3];
#pragma unroll
                for (int h = 0; h < HB; ++h)
#pragma unroll
                    for (int d = 0; d < 3; ++d)
                        pj[h][d] = on[h] ? zeta * __ldg(z + 3 * (int64_t)col[h] + d) +
                                               beta * __ldg(pin + 3 * (int64_t)col[h] + d)
                                         : (T)0;
#pragma unroll
                for (int h = 0; h < HB; ++h) {
                    if (!on[h]) continue;
                    if (DIFF) {
#pragma unroll
                        for (int d = 0; d < 3; ++d)
                            pj[h][d] = (col[h] == (int)i) ? pi[d] : pj[h][d] - pi[d];
                    }
                    const T *a = vs + 9 * sl[h];
#pragma unroll
                    for (int c = 0; c < 3; ++c)
#pragma unroll
                        for (int d = 0; d < 3; ++d) acc[c] += a[3 * c + d] * pj[h][d];
                }
            }
            done = max(done, tend);
            if (done >= ri.y) break;
            // the row goes on in the next window
            __syncwarp();   // reads of this buffer done before it is refilled
            if (lane == 0 && cur + 2 < nwin) stage3_issue(sm, c3, v3, e0, e1, cur + 2);
            ++cur;
            bool okw = false;
            if (cur < nwin) okw = mbar_wait(&sm.mbar[cur & 1], (uint32_t)(cur >> 1) & 1u, err);
            if (!__all_sync(0xffffffffu, okw)) {
                ok = false;
                break;
            }
        }
        if (!ok) break;
#pragma unroll
        for (int c = 0; c < 3; ++c) acc[c] = group_sum<32>(acc[c]);
        if (lane == 0) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                pout[3 * i + c] = pi[c];
                q[3 * i + c] = acc[c];
                pq += pi[c] * acc[c];
            }
        }
    }
    if (ok) {
        // window cur + 1 was issued and may hold only gap units: it must
        // have landed before the warp's shared memory is released
        if (cur + 1 < nwin) {
            const bool okw =
                mbar_wait(&sm.mbar[(cur + 1) & 1], (uint32_t)((cur + 1) >> 1) & 1u, err);
            if (!__all_sync(0xffffffffu, okw)) *fail = 1;
        }
    } else {
        // windows cur (whose wait gave up) and cur + 1 may still be in
        // flight: bounded waits, then report
        for (int k = cur; k < nwin && k <= cur + 1; ++k) {
            const unsigned long long t0 = globaltimer();
            while (!mbar_test(&sm.mbar[k & 1], (uint32_t)(k >> 1) & 1u) &&
                   globaltimer() - t0 < 2000000000ull) {
            }
        }
        *fail = 1;
    }
    part[0] += (double)pq;
}

// Entry-major working-precision copy of block values (AoS -> SoA).
template <typename TI, typename TO, int B2>
__global__ void k_to_soa(int64_t nnzb, const TI *__restrict__ in, TO *__restrict__ out) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnzb;
         k += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int e = 0; e < B2; ++e) out[(int64_t)e * nnzb + k] = (TO)in[k * B2 + e];
    }
}

// ---------------------------------------------------------------------------
// Graph scheduler kernels: lean, one template instance per precision and
// block size, so each keeps few registers and high occupancy. Chunk sums go
// to plain per-chunk slots; k_greduce then sums every system's slots in a
// fixed order (one block per system) and advances its state. An iteration
// is k_gx (A, R or ZERO), k_greduce, k_gb (B), k_greduce.
// Update-phase chunk: BPASS passes of one warp over whole block rows (10
// rows of 3 DOFs or 32 scalar rows per pass), all loads of a chunk issued
// before its arithmetic.
constexpr int BPASS = 4;
__host__ __device__ inline int brows(int bs) { return BPASS * (bs == 3 ? 10 : 32); }

template <typename T, int BS>
__device__ void phase_B_multi(const SysDev &S, const SysState *st, int64_t r0,
                              int64_t r1, int lane, double part[4]) {
    constexpr int RP = BS == 3 ? 10 : 32;      // rows per pass
    const T alpha = (T)vcg(&st->alpha);
    const double alpha64 = vcg(&st->alpha);
    const int pbuf = vcgi(&st->pbuf);
    const T *p = (const T *)(pbuf ? S.p1 : S.p0);
    T *r = (T *)S.r;
    T *z = (T *)S.z;
    const T *q = (const T *)S.q;
    const T *dinv = (const T *)S.dinv;
    const bool blockj = BS == 3 && S.precond == CFEM_PRECOND_BLOCK;
    int64_t iv[BPASS], ii[BPASS];
    bool valid[BPASS], fx[BPASS];
    int cc[BPASS];
    T rv[BPASS], pi[BPASS], qi[BPASS], d0[BPASS], d1[BPASS], d2[BPASS];
    double xi[BPASS];
#pragma unroll
    for (int k = 0; k < BPASS; ++k) {
        iv[k] = (r0 + (int64_t)k * RP) * BS + lane;
        valid[k] = lane < RP * BS && iv[k] < r1 * BS;
        ii[k] = valid[k] ? iv[k] : r0 * BS;
        const int64_t row = ii[k] / BS;
        cc[k] = (int)(ii[k] - row * BS);
        fx[k] = S.fixed ? (__ldg(S.fixed + ii[k]) != 0) : false;
        rv[k] = ldcg(r + ii[k]);
        pi[k] = ldcg(p + ii[k]);
        qi[k] = ldcg(q + ii[k]);
        xi[k] = ldcg(S.x + ii[k]);
        d1[k] = 0;
        d2[k] = 0;
        if (blockj) {
            const T *D = dinv + row * 9 + cc[k] * 3;
            d0[k] = ldcg(D);
            d1[k] = ldcg(D + 1);
            d2[k] = ldcg(D + 2);
        } else {
            d0[k] = ldcg(dinv + ii[k]);
        }
    }
    T rz = 0, rr = 0;
#pragma unroll
    for (int k = 0; k < BPASS; ++k) {
        if (valid[k] && !fx[k]) {
            S.x[iv[k]] = xi[k] + alpha64 * (double)pi[k];
            rv[k] -= alpha * qi[k];
        }
        T zv;
        if (blockj) {
            const int base = lane - cc[k];
            const T ra = __shfl_sync(0xffffffffu, rv[k], base >= 0 ? base : 0);
            const T rb = __shfl_sync(0xffffffffu, rv[k], base + 1 < 32 ? base + 1 : 31);
            const T rc = __shfl_sync(0xffffffffu, rv[k], base + 2 < 32 ? base + 2 : 31);
            zv = d0[k] * ra + d1[k] * rb + d2[k] * rc;
        } else {
            zv = d0[k] * rv[k];
        }
        if (valid[k]) {
            if (fx[k]) zv = 0;
            r[iv[k]] = rv[k];
            z[iv[k]] = zv;
            rz += rv[k] * zv;
            rr += rv[k] * rv[k];
        }
    }
    part[0] += (double)rz;
    part[1] += (double)rr;
}

// Work lists hold each system's chunks padded to whole groups of GROUP
// entries ({-1, -1} = padding), so every block of GROUP warps works on one
// group of one system and writes one group partial, summed in warp order.
constexpr int GROUP = 8;

// Resident blocks per SM asked of k_gx: four (64 registers) keeps the most
// warps in flight, except for FP64 3x3 blocks whose pipelined block values
// need more registers; there three blocks (80 registers, no spills) measured
// 12% faster per iteration than four with spills.
template <typename T, int BS> struct GxOcc {
    static constexpr int blocks = (sizeof(T) == 8 || BS == 1) ? 3 : 4;
};

__device__ __forceinline__ void group_store(double part[4], int nv, double *dst,
                                            int lane, int w) {
    __shared__ double red[GROUP][4];
#pragma unroll
    for (int v = 0; v < 4; ++v) part[v] = warp_sum(part[v]);
    if (lane == 0)
#pragma unroll
        for (int v = 0; v < 4; ++v) red[w][v] = part[v];
    __syncthreads();
    if (threadIdx.x == 0 && dst) {
        for (int v = 0; v < nv; ++v) {
            double t = 0.0;
#pragma unroll
            for (int g = 0; g < GROUP; ++g) t += red[g][v];
            dst[v] = t;
        }
    }
}

template <typename T, int BS>
__global__ void __launch_bounds__(32 * GROUP, (GxOcc<T, BS>::blocks))
k_gx(const SysDev *__restrict__ sys, SysState *st, const GridBar *bar,
     const int2 *__restrict__ list, int n) {
    pdl_wait();
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wid = blockIdx.x * GROUP + w;
    const int2 e = wid < n ? __ldg(list + wid) : make_int2(-1, -1);
    const int2 lead = __ldg(list + blockIdx.x * GROUP);
    if (*(volatile const int *)&bar->active <= 0) return;   // all finished
    const SysDev &S = sys[lead.x];
    const int ph = *(volatile int32_t *)&st[lead.x].phase;
    const bool x_phase = ph == PH_A || ph == PH_R || ph == PH_ZERO;
    if (!x_phase) return;                 // uniform over the block
    double part[4] = {0.0, 0.0, 0.0, 0.0};
    if (e.x >= 0 && (int64_t)e.y * S.xrows < S.n) {   // (slots: entries past a smaller system)
        const int64_t r0 = (int64_t)e.y * S.xrows;
        const int64_t r1 = min(S.n, r0 + S.xrows);
        if (ph == PH_A) {
            if (BS == 1 && S.vec4)
                phase_A_vec1<T, sizeof(T) == 4, sizeof(T) == 4 ? 2 : 1>(S, &st[e.x], r0, r1, lane, part);
            else
                phase_A_lean<T, BS, sizeof(T) == 4>(S, &st[e.x], r0, r1, lane, part);
        } else if (ph == PH_R) {
            int bad = 0;
            run_R<T, BS>(S, &st[e.x], r0, r1, lane, part, &bad);
        } else {
            phase_zero<BS>(S, r0, r1, lane);
        }
    }
    group_store(part, 4, S.partial + (int64_t)(lead.y / GROUP) * 4, lane, w);
}

// k_gx for scalar systems with the bulk-staged A phase (windows of W
// units, LPR lanes per row); R and ZERO phases as in k_gx. Dynamic shared
// memory: GROUP StageWarp<T, W> areas, about 70 KB, three blocks per SM.
// W units per window, NB windows per warp, H rows per lane group and step,
// BLOCKS resident blocks per SM.
template <typename T> struct StageUnits;
template <> struct StageUnits<float> {     // 2 x 4 KB windows per warp
    static constexpr int W = 128, NB = 2, H = 2, BLOCKS = 3;
};
template <> struct StageUnits<double> {    // 2 x 3.9 KB windows per warp
    static constexpr int W = 84, NB = 2, H = 1, BLOCKS = 3;
};
template <typename T>
using StageWarpOf = StageWarp<T, StageUnits<T>::W, StageUnits<T>::NB>;
template <typename T>
constexpr size_t gxs_smem() { return (size_t)GROUP * sizeof(StageWarpOf<T>); }

#ifndef CFEM_RESIDUAL_SELL
#define CFEM_RESIDUAL_SELL 1   // FP64 sliced-ELL residual copy for mixed P1 systems
#endif
// (defined with the sliced-ELL kernels below)
template <typename T>
__device__ __forceinline__ void phase_R_sell(const SysDev &S, const SysState *st, int64_t sl,
                                             int lane, double part[4]);

template <typename T, int LPR>
__global__ void __launch_bounds__(32 * GROUP, StageUnits<T>::BLOCKS)
k_gxs(const SysDev *__restrict__ sys, SysState *st, GridBar *bar,
      const int2 *__restrict__ list, int n) {
    extern __shared__ __align__(16) unsigned char gxs_area[];
    pdl_wait();
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wid = blockIdx.x * GROUP + w;
    const int2 e = wid < n ? __ldg(list + wid) : make_int2(-1, -1);
    const int2 lead = __ldg(list + blockIdx.x * GROUP);
    if (*(volatile const int *)&bar->active <= 0) return;   // all finished
    if (*(volatile const int *)&bar->err) return;           // a wait gave up
    const SysDev &S = sys[lead.x];
    const int ph = *(volatile int32_t *)&st[lead.x].phase;
    const bool x_phase = ph == PH_A || ph == PH_R || ph == PH_ZERO;
    if (!x_phase) return;                 // uniform over the block
    double part[4] = {0.0, 0.0, 0.0, 0.0};
    if (e.x >= 0 && (int64_t)e.y * S.xrows < S.n) {   // (slots: entries past a smaller system)
        const int64_t r0 = (int64_t)e.y * S.xrows;
        const int64_t r1 = min(S.n, r0 + S.xrows);
        if (ph == PH_A) {
            using SU = StageUnits<T>;
            StageWarpOf<T> &sm = reinterpret_cast<StageWarpOf<T> *>(gxs_area)[w];
            int fail = 0;
            phase_A_staged<T, sizeof(T) == 4, SU::W, SU::NB, SU::H, LPR>(
                S, &st[e.x], r0, r1, lane, part, sm, &bar->err, &fail);
            if (fail && lane == 0) atomicExch(&bar->err, 2);
        } else if (ph == PH_R && S.rsell) {
            // the entry's slices of 32 rows in the FP64 sliced-ELL copy
            // (entries are whole multiples of 32 rows, windows of 256 whole
            // multiples of entries)
            for (int64_t sl = r0 / 32; sl * 32 < r1; ++sl)
                phase_R_sell<T>(S, &st[e.x], sl, lane, part);
        } else if (ph == PH_R) {
            int bad = 0;
            run_R<T, 1>(S, &st[e.x], r0, r1, lane, part, &bad);
        } else {
            phase_zero<1>(S, r0, r1, lane);
        }
    }
    group_store(part, 4, S.partial + (int64_t)(lead.y / GROUP) * 4, lane, w);
}

// k_gx for 3x3 systems with the bulk-staged A phase; R and ZERO phases as
// in k_gx. Dynamic shared memory: GROUP Stage3Warp<T, W3> areas, about
// 68 KB, three blocks per SM.
template <typename T> struct Stage3Units;
template <> struct Stage3Units<float> { static constexpr int W = 26; };    // 2 x 3.9 KB per warp
template <> struct Stage3Units<double> { static constexpr int W = 14; };   // 2 x 4.1 KB per warp
template <typename T>
using Stage3WarpOf = Stage3Warp<T, Stage3Units<T>::W>;
template <typename T>
constexpr size_t gxs3_smem() { return (size_t)GROUP * sizeof(Stage3WarpOf<T>); }

template <typename T>
__global__ void __launch_bounds__(32 * GROUP, 3)
k_gxs3(const SysDev *__restrict__ sys, SysState *st, GridBar *bar,
       const int2 *__restrict__ list, int n) {
    extern __shared__ __align__(16) unsigned char gxs_area[];
    pdl_wait();
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wid = blockIdx.x * GROUP + w;
    const int2 e = wid < n ? __ldg(list + wid) : make_int2(-1, -1);
    const int2 lead = __ldg(list + blockIdx.x * GROUP);
    if (*(volatile const int *)&bar->active <= 0) return;   // all finished
    if (*(volatile const int *)&bar->err) return;           // a wait gave up
    const SysDev &S = sys[lead.x];
    const int ph = *(volatile int32_t *)&st[lead.x].phase;
    const bool x_phase = ph == PH_A || ph == PH_R || ph == PH_ZERO;
    if (!x_phase) return;                 // uniform over the block
    double part[4] = {0.0, 0.0, 0.0, 0.0};
    if (e.x >= 0 && (int64_t)e.y * S.xrows < S.n) {   // (slots: entries past a smaller system)
        const int64_t r0 = (int64_t)e.y * S.xrows;
        const int64_t r1 = min(S.n, r0 + S.xrows);
        if (ph == PH_A) {
            Stage3WarpOf<T> &sm = reinterpret_cast<Stage3WarpOf<T> *>(gxs_area)[w];
            int fail = 0;
            phase_A3_staged<T, sizeof(T) == 4, Stage3Units<T>::W>(S, &st[e.x], r0, r1, lane,
                                                                   part, sm, &bar->err, &fail);
            if (fail && lane == 0) atomicExch(&bar->err, 2);
        } else if (ph == PH_R) {
            int bad = 0;
            run_R<T, 3>(S, &st[e.x], r0, r1, lane, part, &bad);
        } else {
            phase_zero<3>(S, r0, r1, lane);
        }
    }
    group_store(part, 4, S.partial + (int64_t)(lead.y / GROUP) * 4, lane, w);
}

template <typename T, int BS>
__global__ void __launch_bounds__(32 * GROUP)
k_gb(const SysDev *__restrict__ sys, SysState *st, const GridBar *bar,
     const int2 *__restrict__ list, int n) {
    pdl_wait();
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wid = blockIdx.x * GROUP + w;
    const int2 e = wid < n ? __ldg(list + wid) : make_int2(-1, -1);
    const int2 lead = __ldg(list + blockIdx.x * GROUP);
    if (*(volatile const int *)&bar->active <= 0) return;   // all finished
    const SysDev &S = sys[lead.x];
    if (*(volatile int32_t *)&st[lead.x].phase != PH_B) return;
    double part[4] = {0.0, 0.0, 0.0, 0.0};
    if (e.x >= 0 && e.y < S.nchunksB) {
        const int64_t r0 = (int64_t)e.y * brows(BS);
        const int64_t r1 = min(S.n, r0 + brows(BS));
        phase_B_multi<T, BS>(S, &st[e.x], r0, r1, lane, part);
    }
    group_store(part, 4, S.partialB + (int64_t)(lead.y / GROUP) * 4, lane, w);
}

// Direction update of the A phase, p = zeta z + beta p_old, over the rows of
// the update-phase chunks of scalar systems. A separate streaming launch
// before k_gx so that the scalar SpMV gathers one precomputed vector instead
// of forming p from z and p_old at every gathered entry (half the gathers and
// their arithmetic). 3x3-block systems form p inside k_gx: there the extra
// launch costs more than it saves.
template <typename T, int BS>
__global__ void __launch_bounds__(32 * GROUP)
k_gp(const SysDev *__restrict__ sys, SysState *st, const GridBar *bar,
     const int2 *__restrict__ list, int n) {
    pdl_wait();
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wid = blockIdx.x * GROUP + w;
    const int2 e = wid < n ? __ldg(list + wid) : make_int2(-1, -1);
    if (*(volatile const int *)&bar->active <= 0) return;   // all finished
    if (e.x < 0) return;
    const SysDev &S = sys[e.x];
    const SysState *sst = &st[e.x];
    if (*(volatile const int32_t *)&sst->phase != PH_A) return;
    const T beta = (T)vcg(&sst->beta);
    const T zeta = (T)vcg(&sst->zeta);
    const int pbuf = vcgi(&sst->pbuf);
    const T *pin = (const T *)(pbuf ? S.p1 : S.p0);
    T *pout = (T *)(pbuf ? S.p0 : S.p1);
    const T *z = (const T *)S.z;
    const int64_t i0 = (int64_t)e.y * brows(BS) * BS;
    const int64_t i1 = min(S.n * BS, i0 + (int64_t)brows(BS) * BS);
    constexpr int NV = (BS == 3 ? 30 : 32) * BPASS / 32 + 1;
    T zz[NV], pp[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        const int64_t i = i0 + lane + 32 * k;
        zz[k] = i < i1 ? __ldcs(z + i) : (T)0;
        pp[k] = i < i1 ? __ldcs(pin + i) : (T)0;
    }
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        const int64_t i = i0 + lane + 32 * k;
        if (i < i1) pout[i] = zeta * zz[k] + beta * pp[k];
    }
}

// One block per system: fixed-order sum of its chunk slots, then advance.
constexpr int RED_THREADS = 1024;
__global__ void __launch_bounds__(RED_THREADS)
k_greduce(const SysDev *__restrict__ sys, SysState *st, GridBar *bar, int which) {
    pdl_wait();
    pdl_trigger();   // the next kernel's fixed-data prologue may start now
    __shared__ double red[4][RED_THREADS / 32];
    const int s = blockIdx.x, t = threadIdx.x, lane = t & 31, w = t >> 5;
    const SysDev &S = sys[s];
    const int ph = *(volatile int32_t *)&st[s].phase;
    const bool mine = which ? (ph == PH_B) : (ph == PH_A || ph == PH_R || ph == PH_ZERO);
    if (!mine) return;
    const int n = which ? (S.nchunksB + GROUP - 1) / GROUP : (S.nxe + GROUP - 1) / GROUP;
    const double *P = which ? S.partialB : S.partial;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    // four independent slots per round keep the loads in flight
    for (int c0 = t; c0 < n; c0 += 4 * RED_THREADS) {
        double v[4][4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int c = c0 + u * RED_THREADS;
#pragma unroll
            for (int e = 0; e < 4; ++e) v[u][e] = c < n ? __ldcg(P + (int64_t)c * 4 + e) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[e] += v[u][e];
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) acc[e] = warp_sum(acc[e]);
    if (lane == 0)
#pragma unroll
        for (int e = 0; e < 4; ++e) red[e][w] = acc[e];
    __syncthreads();
    if (w == 0) {
        double tot[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) tot[e] = warp_sum(lane < RED_THREADS / 32 ? red[e][lane] : 0.0);
        if (lane == 0) advance(S, &st[s], bar, ph, tot);
    }
}

// ---------------------------------------------------------------------------
// Sliced-ELL scalar SpMV (graph scheduler, A phase of scalar systems at SpMV
// staging 3). A work entry is SELL_ROWS consecutive rows of one system,
// sorted by length (longest first, ties in row order) and cut into slices
// of 32 rows; a slice stores its rows' entries slot-major (slot k of all 32
// rows, then slot k + 1), padded to its longest row with (own row, 0). One
// lane owns one row: the column and value loads of a warp are two coalesced
// 128-byte (FP32) lines per slot, read with no L1 allocation so that the
// gathered p stays in L1, and a row needs no cross-lane reduction. Slot 0
// holds the diagonal (FP64) or the FP32 difference form's row sum s_i, which
// is applied to p_i; the other slots a_ij (p_j - p_i) in the difference form,
// a_ij p_j otherwise (padding adds nothing either way). Sorting within
// SELL_ROWS rows keeps the padding of Tet10 patterns near 3 % (slices of
// unsorted rows: 14 %). The layout depends only on the system's pattern, so
// sums are the same alone and in any batch.
constexpr int SELL_ROWS = 256;
// Longest block row a 3x3 solve slot's sliced-ELL copy is sized for (Tet10
// vertex rows of box meshes hold up to 65 blocks).
constexpr int SLOT_SELL_ROW = 96;
constexpr int SELL_SLICES = SELL_ROWS / 32;
constexpr int SELL_BLOCKS = 4;     // resident blocks of k_gxl per SM
__host__ __device__ inline int64_t sell_windows(int64_t n) {
    return (n + SELL_ROWS - 1) / SELL_ROWS;
}

__device__ __forceinline__ int32_t ld_stream(const int32_t *p) {
    int32_t v;
    asm volatile("ld.global.nc.L1::no_allocate.b32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ float ld_stream(const float *p) {
    float v;
    asm volatile("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ double ld_stream(const double *p) {
    double v;
    asm volatile("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}

// Sort each window's rows by stored length (the diagonal counted once
// even when absent: it gets its own slot) and write the slice sizes. A
// slice holds RS rows, each over 32 / RS lanes, so its size is 32 x its
// longest row's slot count rounded up to whole steps of 32 / RS slots (0
// for slices of padding rows only). RS = 32: one row per lane.
template <int RS>
__global__ void __launch_bounds__(SELL_ROWS)
k_sell_rank(int64_t n, const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
            uint8_t *__restrict__ perm, int64_t *__restrict__ sizes, int sort) {
    constexpr int LPR = 32 / RS, NS = SELL_ROWS / RS;
    __shared__ int len[SELL_ROWS];
    const int t = threadIdx.x;
    const int64_t r0 = (int64_t)blockIdx.x * SELL_ROWS;
    const int64_t row = r0 + t;
    int L = 0;
    if (row < n) {
        const int32_t kb = __ldg(rp + row), ke = __ldg(rp + row + 1);
        bool diag = false;
        for (int32_t k = kb; k < ke; ++k) diag |= __ldg(ci + k) == (int32_t)row;
        L = ke - kb + (diag ? 0 : 1);
    }
    if (!sort) {   // rows in their own order: a slice is RS consecutive rows
        perm[r0 + t] = (uint8_t)t;
        int m = L;
#pragma unroll
        for (int o = RS / 2; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
        if ((t % RS) == 0)
            sizes[(int64_t)blockIdx.x * NS + t / RS] = 32 * (int64_t)((m + LPR - 1) / LPR);
        return;
    }
    len[t] = L;
    __syncthreads();
    int rank = 0;
    for (int u = 0; u < SELL_ROWS; ++u) {
        const int Lu = len[u];
        rank += (Lu > L || (Lu == L && u < t)) ? 1 : 0;
    }
    perm[r0 + rank] = (uint8_t)t;
    if ((rank % RS) == 0)
        sizes[(int64_t)blockIdx.x * NS + rank / RS] = 32 * (int64_t)((L + LPR - 1) / LPR);
}

// Fill the slices from the CSR: position t of entry blockIdx.x (slice t/32,
// lane t%32) holds row r0 + perm[t]: the diagonal first, then the other
// entries in column order, then padding.
template <typename T>
__global__ void __launch_bounds__(SELL_ROWS)
k_sell_fill(int64_t n, const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
            const T *__restrict__ v, const uint8_t *__restrict__ perm,
            const int64_t *__restrict__ soff, int32_t *__restrict__ scol, T *__restrict__ sval) {
    const int t = threadIdx.x;
    const int64_t r0 = (int64_t)blockIdx.x * SELL_ROWS;
    const int64_t sl = (int64_t)blockIdx.x * SELL_SLICES + (t >> 5);
    const int64_t base = soff[sl];
    const int w = (int)((soff[sl + 1] - base) >> 5);
    if (w == 0) return;
    const int64_t row = r0 + perm[r0 + t];
    const bool valid = row < n;
    const int32_t kb = valid ? __ldg(rp + row) : 0, len = valid ? __ldg(rp + row + 1) - kb : 0;
    int dpos = -1;
    for (int k = 0; k < len; ++k)
        if (__ldg(ci + kb + k) == (int32_t)row) { dpos = k; break; }
    const int32_t own = valid ? (int32_t)row : (int32_t)r0;
    int64_t o = base + (t & 31);
    // slot 0: the diagonal (value 0 if the pattern has none)
    scol[o] = own;
    sval[o] = dpos >= 0 ? v[kb + dpos] : (T)0;
    int k = 1;
    for (int e = 0; e < len; ++e) {
        if (e == dpos) continue;
        o += 32;
        scol[o] = __ldg(ci + kb + e);
        sval[o] = v[kb + e];
        ++k;
    }
    for (; k < w; ++k) {
        o += 32;
        scol[o] = own;
        sval[o] = (T)0;
    }
}

// 3x3 blocks: as k_sell_fill, with RS block rows per slice, each over
// L = 32 / RS lanes: slot k of the slice's row r sits at step k / L, lane
// r L + k % L, and the step's 9 values (row-major block) in 9 planes of 32
// lanes: column at soff[slice] + 32 step + lane, value e at
// 9 soff[slice] + (9 step + e) 32 + lane. Slot 0 is the diagonal block.
template <typename T, int RS>
__global__ void __launch_bounds__(SELL_ROWS)
k_sell_fill3(int64_t n, const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
             const T *__restrict__ v, const uint8_t *__restrict__ perm,
             const int64_t *__restrict__ soff, int32_t *__restrict__ scol, T *__restrict__ sval) {
    constexpr int L = 32 / RS, NS = SELL_ROWS / RS;
    const int t = threadIdx.x;
    const int64_t r0 = (int64_t)blockIdx.x * SELL_ROWS;
    const int64_t sl = (int64_t)blockIdx.x * NS + t / RS;
    const int64_t base = soff[sl];
    const int w = (int)((soff[sl + 1] - base) >> 5) * L;   // slots per row
    if (w == 0) return;
    const int64_t row = r0 + perm[r0 + t];
    const bool valid = row < n;
    const int32_t kb = valid ? __ldg(rp + row) : 0, len = valid ? __ldg(rp + row + 1) - kb : 0;
    int dpos = -1;
    for (int k = 0; k < len; ++k)
        if (__ldg(ci + kb + k) == (int32_t)row) { dpos = k; break; }
    const int32_t own = valid ? (int32_t)row : (int32_t)r0;
    const int r = t % RS;
    auto put = [&](int k, int32_t c, int64_t src) {
        const int64_t step = k / L;
        const int lane = r * L + k % L;
        scol[base + 32 * step + lane] = c;
        T *vb = sval + 9 * base + 9 * 32 * step + lane;
#pragma unroll
        for (int e = 0; e < 9; ++e) vb[32 * e] = src >= 0 ? v[src * 9 + e] : (T)0;
    };
    put(0, own, dpos >= 0 ? (int64_t)kb + dpos : -1);
    int k = 1;
    for (int e = 0; e < len; ++e) {
        if (e == dpos) continue;
        put(k++, __ldg(ci + kb + e), (int64_t)kb + e);
    }
    for (; k < w; ++k) put(k, own, -1);
}

// q = A p and p.q over the RS = 32 / L block rows of slice sl of a 3x3
// system (A phase), L lanes per block row, each over every L-th slot; the
// lanes' partial sums meet by shuffles. As the register path does, the new
// direction p = zeta z + beta p_old is formed at every gathered block and
// written for the row (3x3 systems have no separate direction launch).
// DIFF: slot 0 holds the FP32 block row sum S_i, applied to p_i, the other
// slots A_ij (p_j - p_i).
//
// Split in two: sell3_open reads only what is fixed for the whole solve
// (the slice's place, its row, its first columns and block values), so
// k_gxl3 runs it before waiting for its predecessor kernel; sell3_run
// then streams the slice: columns two steps ahead of their gathers, block
// values D steps ahead (D = 2 for FP32, 1 for FP64, whose registers allow
// one), the gathers of z and p_old one step ahead of their use.
template <typename T> struct Sell3Depth { static constexpr int D = sizeof(T) == 4 ? 2 : 1; };

template <typename T> struct Sell3Slice {
    const int32_t *cp;
    const T *vp;
    int w;            // steps
    int64_t row;      // the lane's block row (its window's first row if padding)
    bool valid, live;
    int64_t j0, j1;   // columns of steps 0 and 1
    T a0[9], a1[9];   // block values of steps 0 and 1 (a1: FP32 only)
};

template <typename T, int L>
__device__ __forceinline__ void sell3_open(const SysDev &S, int64_t sl, int lane,
                                           Sell3Slice<T> &q) {
    constexpr int RS = 32 / L, NS = SELL_ROWS / RS;
    const int64_t r0 = (sl / NS) * SELL_ROWS;
    const int s = (int)(sl % NS);
    const int nr = (int)min((int64_t)SELL_ROWS, S.n - r0);
    q.live = s * RS < nr;
    if (!q.live) return;
    const int64_t base = __ldg(S.soff + sl);
    q.w = (int)((__ldg(S.soff + sl + 1) - base) >> 5);
    const int rl = __ldg(S.sperm + r0 + s * RS + lane / L);
    q.valid = rl < nr;
    q.row = q.valid ? r0 + rl : r0;
    q.cp = S.scol + base + lane;
    q.vp = (const T *)S.sval + 9 * base + lane;
    q.j0 = ld_stream(q.cp);
    q.j1 = ld_stream(q.cp + 32 * (q.w > 1 ? 1 : 0));
#pragma unroll
    for (int e = 0; e < 9; ++e) q.a0[e] = ld_stream(q.vp + 32 * e);
    if (Sell3Depth<T>::D == 2) {
        const int t1 = q.w > 1 ? 1 : 0;
#pragma unroll
        for (int e = 0; e < 9; ++e) q.a1[e] = ld_stream(q.vp + 32 * (9 * t1 + e));
    }
}

template <typename T, bool DIFF, int L>
__device__ __forceinline__ void sell3_run(const SysDev &S, const SysState *st, Sell3Slice<T> &q,
                                          int lane, double part[4]) {
    constexpr int D = Sell3Depth<T>::D;
    if (!q.live) return;
    const T beta = (T)vcg(&st->beta);
    const T zeta = (T)vcg(&st->zeta);
    const int pbuf = vcgi(&st->pbuf);
    const T *pin = (const T *)(pbuf ? S.p1 : S.p0);
    T *pout = (T *)(pbuf ? S.p0 : S.p1);
    const T *z = (const T *)S.z;
    T *qv = (T *)S.q;
    const int u = lane % L;
    const int w = q.w;
    const int64_t row = q.row;
    T pi[3], acc[3], gz[3], gp[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        pi[c] = zeta * __ldg(z + row * 3 + c) + beta * __ldg(pin + row * 3 + c);
        acc[c] = 0;
        gz[c] = __ldg(z + q.j0 * 3 + c);
        gp[c] = __ldg(pin + q.j0 * 3 + c);
    }
    int64_t jn = q.j1;
    for (int t = 0; t < w; ++t) {
        const int tn = t + 1 < w ? t + 1 : t;
        const int tnn = t + 2 < w ? t + 2 : tn;
        const int64_t jnn = ld_stream(q.cp + 32 * tnn);
        T an[9], gz2[3], gp2[3];
        const int tl = D == 2 ? tnn : tn;   // the step whose values load now
#pragma unroll
        for (int e = 0; e < 9; ++e) an[e] = ld_stream(q.vp + 32 * (9 * tl + e));
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            gz2[d] = __ldg(z + jn * 3 + d);
            gp2[d] = __ldg(pin + jn * 3 + d);
        }
        T pj[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            pj[d] = zeta * gz[d] + beta * gp[d];
            if (DIFF) pj[d] = (t == 0 && u == 0) ? pi[d] : pj[d] - pi[d];
        }
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int d = 0; d < 3; ++d) acc[c] += q.a0[c * 3 + d] * pj[d];
#pragma unroll
        for (int e = 0; e < 9; ++e) {
            if (D == 2) {
                q.a0[e] = q.a1[e];
                q.a1[e] = an[e];
            } else {
                q.a0[e] = an[e];
            }
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            gz[d] = gz2[d];
            gp[d] = gp2[d];
        }
        jn = jnn;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int o = L / 2; o > 0; o >>= 1) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
    T pq = 0;
    if (q.valid && u == 0) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int64_t i = row * 3 + c;
            pout[i] = pi[c];
            qv[i] = acc[c];
            pq += pi[c] * acc[c];
        }
    }
    part[0] += (double)pq;
}

// q = A p and p.q over the 32 rows of slice sl (A phase).
template <typename T, bool DIFF>
__device__ __forceinline__ void phase_A_sell(const SysDev &S, const SysState *st, int64_t sl,
                                             int lane, double part[4]) {
    const int pbuf = vcgi(&st->pbuf);
    const T *pv = (const T *)(pbuf ? S.p0 : S.p1);   // this iteration's p (k_gp)
    T *q = (T *)S.q;
    const int32_t *scol = S.scol;
    const T *sval = (const T *)S.sval;
    const int64_t r0 = (sl / SELL_SLICES) * SELL_ROWS;   // the slice's window
    const int s = (int)(sl % SELL_SLICES);
    const int nr = (int)min((int64_t)SELL_ROWS, S.n - r0);
    T pq = 0;
    if (s * 32 < nr) {
        const int64_t base = __ldg(S.soff + sl);
        const int w = (int)((__ldg(S.soff + sl + 1) - base) >> 5);
        const int rl = __ldg(S.sperm + r0 + s * 32 + lane);
        const bool valid = rl < nr;
        const int64_t row = r0 + rl;
        const T pi = valid ? __ldg(pv + row) : (T)0;
        const int32_t *cp = scol + base + lane;
        const T *vp = sval + base + lane;
        T acc = ld_stream(vp) * pi;
        // U slots in flight per lane: their column and value loads first,
        // then the gathers
        constexpr int U = 8;
        int k = 1;
        for (; k + U <= w; k += U) {
            int32_t c[U];
            T a[U], g[U];
#pragma unroll
            for (int j = 0; j < U; ++j) c[j] = ld_stream(cp + 32 * (k + j));
#pragma unroll
            for (int j = 0; j < U; ++j) a[j] = ld_stream(vp + 32 * (k + j));
#pragma unroll
            for (int j = 0; j < U; ++j) g[j] = __ldg(pv + c[j]);
#pragma unroll
            for (int j = 0; j < U; ++j) acc += a[j] * (DIFF ? g[j] - pi : g[j]);
        }
        for (; k < w; ++k) {
            const int32_t c = ld_stream(cp + 32 * k);
            const T a = ld_stream(vp + 32 * k);
            const T g = __ldg(pv + c);
            acc += a * (DIFF ? g - pi : g);
        }
        if (valid) {
            q[row] = acc;
            pq += pi * acc;
        }
    }
    part[0] += (double)pq;
}

// FP64 true residual (R phase, not INIT) over the 32 rows of slice sl from
// the sliced-ELL copy itself, whose values are FP64 when the system is
// solved in FP64: one row per lane, compensated sums as in phase_R.
template <typename T>
__device__ __forceinline__ void phase_R_sell(const SysDev &S, const SysState *st, int64_t sl,
                                             int lane, double part[4]) {
    const int64_t r0 = (sl / SELL_SLICES) * SELL_ROWS;
    const int s = (int)(sl % SELL_SLICES);
    const int nr = (int)min((int64_t)SELL_ROWS, S.n - r0);
    if (s * 32 >= nr) return;
    const int64_t base = __ldg(S.soff + sl);
    const int w = (int)((__ldg(S.soff + sl + 1) - base) >> 5);
    const int rl = __ldg(S.sperm + r0 + s * 32 + lane);
    const int32_t *cp = S.scol + base + lane;
    const double *vp = (const double *)S.sval + base + lane;
    double hi = 0.0, lo = 0.0, aab = 0.0;
    // U slots in flight per lane (their column and value loads, then the
    // gathers of x, read-only in this launch), summed in slot order
    constexpr int U = 8;
    int k = 0;
    for (; k + U <= w; k += U) {
        int32_t c[U];
        double a[U], xj[U];
#pragma unroll
        for (int j = 0; j < U; ++j) c[j] = ld_stream(cp + 32 * (k + j));
#pragma unroll
        for (int j = 0; j < U; ++j) a[j] = ld_stream(vp + 32 * (k + j));
#pragma unroll
        for (int j = 0; j < U; ++j) xj[j] = __ldg(S.x + c[j]);
#pragma unroll
        for (int j = 0; j < U; ++j) {
            dd_fma(hi, lo, a[j], xj[j]);
            aab += fabs(a[j] * xj[j]);
        }
    }
    for (; k < w; ++k) {
        const double a = ld_stream(vp + 32 * k);
        const double xj = __ldg(S.x + ld_stream(cp + 32 * k));
        dd_fma(hi, lo, a, xj);
        aab += fabs(a * xj);
    }
    if (rl >= nr) return;
    const int64_t i = r0 + rl;
    const bool fx = S.fixed ? (__ldg(S.fixed + i) != 0) : false;
    const double rt = fx ? 0.0 : dd_residual(__ldg(S.b + i), hi, lo);
    const T rv = (T)rt;
    ((T *)S.r)[i] = rv;
    T zv = fx ? (T)0 : ldcg((const T *)S.dinv + i) * rv;
    ((T *)S.z)[i] = zv;
    const T *pc = (const T *)(vcgi(&st->pbuf) == 0 ? S.p0 : S.p1);
    part[0] += rt * rt;
    part[1] += (double)(rv * ldcg(pc + i));
    part[2] += (double)(rv * zv);
    if (!fx) part[3] += aab * aab;
}

// INIT from the sliced FP64 copy of a mixed P1 system (`rsell`). A window
// of SELL_ROWS rows holds SELL_ROWS / 16 chunks of 16 rows and SELL_SLICES
// slices of 32: the warp of the window's chunk 2s takes slice s (one row
// per lane) and reports its sums, the warp of chunk 2s + 1 reports none, so
// the chunk partials and their tickets are those of the other INIT paths.
// Writes what phase_R_vec1<INIT> writes: r = b - A x (compensated sums),
// the Jacobi inverse from the diagonal (slot 0; 0 there if the pattern has
// none: a bad row), z, and rr, |b'|^2 (b less the fixed columns' part),
// r.z and the floor sum.
template <typename T>
__device__ void init_R_sell(const SysDev &S, int64_t lc, int lane, double part[4], int *bad) {
    constexpr int CPW = SELL_ROWS / 16;   // chunks per window
    const int64_t win = lc / CPW;
    const int j = (int)(lc % CPW);
    if (j & 1) return;
    const int s = j >> 1;
    const int64_t sl = win * SELL_SLICES + s;
    const int64_t r0 = win * SELL_ROWS;
    const int nr = (int)min((int64_t)SELL_ROWS, S.n - r0);
    if (s * 32 >= nr) return;
    const int64_t base = __ldg(S.soff + sl);
    const int w = (int)((__ldg(S.soff + sl + 1) - base) >> 5);
    const int rl = __ldg(S.sperm + r0 + s * 32 + lane);
    const int32_t *cp = S.scol + base + lane;
    const double *vp = (const double *)S.sval + base + lane;
    const double dg = w > 0 ? ld_stream(vp) : 0.0;
    double hi = 0.0, lo = 0.0, aab = 0.0, accf = 0.0;
    for (int k = 0; k < w; ++k) {
        const int32_t c = ld_stream(cp + 32 * k);
        const double a = ld_stream(vp + 32 * k);
        const double xj = __ldg(S.x + c);   // x is not written in INIT
        const double ax = a * xj;
        dd_fma(hi, lo, a, xj);
        aab += fabs(ax);
        if (S.fixed && __ldg(S.fixed + c) != 0) accf += ax;
    }
    if (rl >= nr) return;
    const int64_t i = r0 + rl;
    const bool fx = S.fixed ? (__ldg(S.fixed + i) != 0) : false;
    const double bi = __ldg(S.b + i);
    const double rt = fx ? 0.0 : dd_residual(bi, hi, lo);
    double iv = 0.0;
    if (!fx) {
        if (!(dg > 0.0) || !isfinite(dg)) *bad = 1;
        else iv = 1.0 / dg;
        const double bl = bi - accf;
        part[1] += bl * bl;
        part[3] += aab * aab;
    }
    const T rv = (T)rt;
    const T dv = (T)iv;
    ((T *)S.r)[i] = rv;
    ((T *)S.dinv)[i] = dv;
    const T zv = fx ? (T)0 : dv * rv;
    ((T *)S.z)[i] = zv;
    part[0] += rt * rt;
    part[2] += (double)(rv * zv);
}

// k_gx for scalar systems with the sliced-ELL A phase: one slice of 32
// rows per warp (work entries of 32 rows, so the GROUP warps of a block
// cover one window of SELL_ROWS rows). R phase: from the sliced-ELL copy in
// FP64 (its values are FP64 then), else from the unit-padded copy as in
// k_gxs; ZERO phase on the entry's rows.
template <typename T>
__global__ void __launch_bounds__(32 * GROUP, SELL_BLOCKS)
k_gxl(const SysDev *__restrict__ sys, SysState *st, const GridBar *bar,
      const int2 *__restrict__ list, int n) {
    pdl_wait();
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wid = blockIdx.x * GROUP + w;
    const int2 e = wid < n ? __ldg(list + wid) : make_int2(-1, -1);
    const int2 lead = __ldg(list + blockIdx.x * GROUP);
    if (*(volatile const int *)&bar->active <= 0) return;   // all finished
    const SysDev &S = sys[lead.x];
    const int ph = *(volatile int32_t *)&st[lead.x].phase;
    const bool x_phase = ph == PH_A || ph == PH_R || ph == PH_ZERO;
    if (!x_phase) return;                 // uniform over the block
    double part[4] = {0.0, 0.0, 0.0, 0.0};
    if (e.x >= 0 && (int64_t)e.y * S.xrows < S.n) {   // (slots: entries past a smaller system)
        const int64_t r0 = (int64_t)e.y * S.xrows;
        const int64_t r1 = min(S.n, r0 + S.xrows);
        if (ph == PH_A) {
            phase_A_sell<T, sizeof(T) == 4>(S, &st[e.x], e.y, lane, part);
        } else if (ph == PH_R) {
            if (sizeof(T) == 8) {
                phase_R_sell<T>(S, &st[e.x], e.y, lane, part);
            } else {
                int bad = 0;
                run_R<T, 1>(S, &st[e.x], r0, r1, lane, part, &bad);
            }
        } else {
            phase_zero<1>(S, r0, r1, lane);
        }
    }
    group_store(part, 4, S.partial + (int64_t)(lead.y / GROUP) * 4, lane, w);
}

// k_gx for 3x3 systems with the sliced-ELL A phase (one slice of 32 / L
// block rows per warp, L lanes per block row); R and ZERO phases on the
// entry's block rows as in k_gx. The slice's fixed data is read before the
// wait for the predecessor kernel (dependent launches).
template <typename T> struct Sell3Occ {   // the pipelined blocks need 80 registers
    static constexpr int blocks = 3;
};
template <typename T, int L>
__global__ void __launch_bounds__(32 * GROUP, Sell3Occ<T>::blocks)
k_gxl3(const SysDev *__restrict__ sys, SysState *st, const GridBar *bar,
       const int2 *__restrict__ list, int n) {
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wid = blockIdx.x * GROUP + w;
    const int2 e = wid < n ? __ldg(list + wid) : make_int2(-1, -1);
    const int2 lead = __ldg(list + blockIdx.x * GROUP);   // a real entry (lists pad per system)
    const SysDev &S = sys[lead.x];
    const bool mine = e.x >= 0 && (int64_t)e.y * S.xrows < S.n;
    Sell3Slice<T> q;
    q.live = false;
    if (mine) sell3_open<T, L>(S, e.y, lane, q);
    pdl_wait();
    if (*(volatile const int *)&bar->active <= 0) return;   // all finished
    const int ph = *(volatile int32_t *)&st[lead.x].phase;
    const bool x_phase = ph == PH_A || ph == PH_R || ph == PH_ZERO;
    if (!x_phase) return;                 // uniform over the block
    double part[4] = {0.0, 0.0, 0.0, 0.0};
    if (mine) {
        const int64_t r0 = (int64_t)e.y * S.xrows;
        const int64_t r1 = min(S.n, r0 + S.xrows);
        if (ph == PH_A) {
            sell3_run<T, sizeof(T) == 4, L>(S, &st[e.x], q, lane, part);
        } else if (ph == PH_R) {
            int bad = 0;
            run_R<T, 3>(S, &st[e.x], r0, r1, lane, part, &bad);
        } else {
            phase_zero<3>(S, r0, r1, lane);
        }
    }
    group_store(part, 4, S.partial + (int64_t)(lead.y / GROUP) * 4, lane, w);
}

// k_gxl3 with the slice streamed through shared memory: a slice's step (a
// column plane and 9 value planes of 32 lanes) is contiguous in the
// sliced-ELL copy, so one lane issues two 1-D bulk copies per step into a
// ring of NS3 stages completing on transaction mbarriers, NS3 steps ahead
// of their use. The first NS3 steps are issued before the wait for the
// predecessor kernel (skipped when the system has already finished), so
// they travel while the previous kernel drains. Every issued copy is
// waited for before the warp leaves, also on the R / ZERO and early-exit
// paths; every wait is bounded (2 s) and a warp that gives up records the
// error and drains its other copies (bounded).
constexpr int NS3 = 3;
template <typename T> struct __align__(16) Sell3Ring {
    T val[NS3][9 * 32];
    int32_t col[NS3][32];
    unsigned long long mbar[NS3];
};
template <typename T>
constexpr size_t gxl3s_smem() { return (size_t)GROUP * sizeof(Sell3Ring<T>); }

template <typename T>
__device__ __forceinline__ void sell3_issue(Sell3Ring<T> &rg, const T *vb, const int32_t *cb,
                                            int t) {
    const int b = t % NS3;
    const uint32_t bv = 9 * 32 * (uint32_t)sizeof(T), bc = 32 * 4;
    mbar_expect(&rg.mbar[b], bv + bc);
    bulk_load_stream(&rg.val[b][0], vb + (int64_t)9 * 32 * t, bv, &rg.mbar[b]);
    bulk_load_stream(&rg.col[b][0], cb + (int64_t)32 * t, bc, &rg.mbar[b]);
}

// Waits (bounded) for the issued steps [from, to) that were not consumed.
template <typename T>
__device__ __forceinline__ void sell3_drain(Sell3Ring<T> &rg, int from, int to) {
    for (int t = from; t < to; ++t) {
        const unsigned long long t0 = globaltimer();
        while (!mbar_test(&rg.mbar[t % NS3], (uint32_t)(t / NS3) & 1u) &&
               globaltimer() - t0 < 2000000000ull) {
        }
    }
}

template <typename T, int L>
__global__ void __launch_bounds__(32 * GROUP, 3)
k_gxl3s(const SysDev *__restrict__ sys, SysState *st, GridBar *bar,
        const int2 *__restrict__ list, int n) {
    extern __shared__ __align__(16) unsigned char ring_area[];
    constexpr int RS = 32 / L, NSL = SELL_ROWS / RS;
    constexpr bool DIFF = sizeof(T) == 4;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wid = blockIdx.x * GROUP + w;
    const int2 e = wid < n ? __ldg(list + wid) : make_int2(-1, -1);
    const int2 lead = __ldg(list + blockIdx.x * GROUP);   // a real entry (lists pad per system)
    const SysDev &S = sys[lead.x];
    Sell3Ring<T> &rg = reinterpret_cast<Sell3Ring<T> *>(ring_area)[w];
    // the slice's place: fixed for the whole solve
    const bool mine = e.x >= 0 && (int64_t)e.y * S.xrows < S.n;
    bool live = false, valid = false;
    int wst = 0;
    int64_t row = 0;
    const T *vb = nullptr;
    const int32_t *cb = nullptr;
    if (mine) {
        const int64_t sl = e.y;
        const int64_t r0 = (sl / NSL) * SELL_ROWS;
        const int sidx = (int)(sl % NSL);
        const int nr = (int)min((int64_t)SELL_ROWS, S.n - r0);
        live = sidx * RS < nr;
        if (live) {
            const int64_t base = __ldg(S.soff + sl);
            wst = (int)((__ldg(S.soff + sl + 1) - base) >> 5);
            const int rl = __ldg(S.sperm + r0 + sidx * RS + lane / L);
            valid = rl < nr;
            row = valid ? r0 + rl : r0;
            vb = (const T *)S.sval + 9 * base;
            cb = S.scol + base;
        }
    }
    if (lane == 0) {
#pragma unroll
        for (int b = 0; b < NS3; ++b) mbar_init(&rg.mbar[b]);
        mbar_init_fence();
    }
    __syncwarp();
    // a finished system stays finished: no prefetch for it
    const bool done0 = *(volatile const int32_t *)&st[lead.x].phase == PH_DONE;
    int issued = 0;
    if (live && !done0) {
        issued = wst < NS3 ? wst : NS3;
        if (lane == 0)
            for (int t = 0; t < issued; ++t) sell3_issue(rg, vb, cb, t);
    }
    pdl_wait();
    const int ph = *(volatile int32_t *)&st[lead.x].phase;
    const bool go = *(volatile const int *)&bar->active > 0 &&
                    !*(volatile const int *)&bar->err &&
                    (ph == PH_A || ph == PH_R || ph == PH_ZERO);   // uniform over the block
    if (!go) {
        sell3_drain(rg, 0, issued);
        return;
    }
    double part[4] = {0.0, 0.0, 0.0, 0.0};
    if (mine && ph == PH_A && live && issued < wst && issued < NS3) {
        // (the prefetch was skipped: the phase changed since) issue now
        const int k = wst < NS3 ? wst : NS3;
        if (lane == 0)
            for (int t = issued; t < k; ++t) sell3_issue(rg, vb, cb, t);
        issued = k;
    }
    if (mine && ph == PH_A && live) {
        const SysState *sst = &st[e.x];
        const T beta = (T)vcg(&sst->beta);
        const T zeta = (T)vcg(&sst->zeta);
        const int pbuf = vcgi(&sst->pbuf);
        const T *pin = (const T *)(pbuf ? S.p1 : S.p0);
        T *pout = (T *)(pbuf ? S.p0 : S.p1);
        const T *z = (const T *)S.z;
        T *qv = (T *)S.q;
        const int u = lane % L;
        T pi[3], acc[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            pi[c] = zeta * __ldg(z + row * 3 + c) + beta * __ldg(pin + row * 3 + c);
            acc[c] = 0;
        }
        int t = 0;
        for (; t < wst; ++t) {
            const int b = t % NS3;
            const bool ok = mbar_wait(&rg.mbar[b], (uint32_t)(t / NS3) & 1u, &bar->err);
            if (!__all_sync(0xffffffffu, ok)) {
                sell3_drain(rg, t, issued);   // this step's copy may still be in flight
                if (lane == 0) atomicExch(&bar->err, 2);
                break;
            }
            const int64_t j = rg.col[b][lane];
            T a[9];
#pragma unroll
            for (int q = 0; q < 9; ++q) a[q] = rg.val[b][q * 32 + lane];
            T pj[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                pj[d] = zeta * __ldg(z + j * 3 + d) + beta * __ldg(pin + j * 3 + d);
                if (DIFF) pj[d] = (t == 0 && u == 0) ? pi[d] : pj[d] - pi[d];
            }
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int d = 0; d < 3; ++d) acc[c] += a[c * 3 + d] * pj[d];
            __syncwarp();   // every lane has read stage b
            if (issued < wst) {
                if (lane == 0) {
                    // the generic reads above before the async-proxy writes
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    sell3_issue(rg, vb, cb, issued);
                }
                ++issued;
            }
        }
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int o = L / 2; o > 0; o >>= 1) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
        T pq = 0;
        if (t == wst && valid && u == 0) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const int64_t i = row * 3 + c;
                pout[i] = pi[c];
                qv[i] = acc[c];
                pq += pi[c] * acc[c];
            }
        }
        part[0] += (double)pq;
    } else {
        sell3_drain(rg, 0, issued);
        if (mine) {
            const int64_t r0 = (int64_t)e.y * S.xrows;
            const int64_t r1 = min(S.n, r0 + S.xrows);
            if (ph == PH_R) {
                int bad = 0;
                run_R<T, 3>(S, &st[e.x], r0, r1, lane, part, &bad);
            } else if (ph == PH_ZERO) {
                phase_zero<3>(S, r0, r1, lane);
            }
        }
    }
    group_store(part, 4, S.partial + (int64_t)(lead.y / GROUP) * 4, lane, w);
}

template <typename T>
static void (*gxl3s_kernel(int L))(const SysDev *, SysState *, GridBar *, const int2 *, int) {
    return L == 1 ? k_gxl3s<T, 1> : L == 2 ? k_gxl3s<T, 2> : k_gxl3s<T, 4>;
}

template <typename T>
static int gxl3s_prepare(int L) {
    const size_t bytes = gxl3s_smem<T>();
    auto k = gxl3s_kernel<T>(L);
    CFEM_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    int pct = (int)((3 * (bytes + 1024) * 100 + 228 * 1024 - 1) / (228 * 1024));
    if (pct > 100) pct = 100;
    CFEM_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
    return CFEM_OK;
}

// The k_gxl3 instance for L lanes per block row (1, 2 or 4: slices of at
// least chunk_rows(3) block rows, so the work lists stay within their
// per-chunk allocation).
template <typename T>
static void (*gxl3_kernel(int L))(const SysDev *, SysState *, const GridBar *, const int2 *, int) {
    return L == 1 ? k_gxl3<T, 1> : L == 2 ? k_gxl3<T, 2> : k_gxl3<T, 4>;
}

// Rows per sliced-ELL slice: 32 scalar rows (one per lane), or 32 / L
// block rows of a 3x3 system.
__host__ __device__ inline int sell_slice_rows(int bs, int lanes3) {
    return bs == 3 ? 32 / lanes3 : 32;
}

constexpr int POLL_ITERS = 16;    // iterations per replay, host-polled graphs
constexpr int X_CHUNKS_VEC = 8;   // chunks per SpMV work entry, padded scalar rows
static_assert(X_CHUNKS_VEC * 16 <= XR_MAX, "staged work entries hold at most XR_MAX rows");
static_assert(SELL_SLICES == GROUP, "a block of k_gxl covers one sliced-ELL window");

// Start of a graph-scheduled solve: every system active, no barrier error.
__global__ void k_plan_start(GridBar *bar, int n_systems) {
    if (threadIdx.x == 0) {
        bar->active = n_systems;
        bar->err = 0;
        bar->rounds = 0;
    }
}

// Loop condition of a graph-scheduled solve: another body while a system is
// active and the round bound (from the largest max_iter) is not reached.
__global__ void k_loop_cond(cudaGraphConditionalHandle h, GridBar *bar, unsigned max_rounds) {
    pdl_wait();
    if (threadIdx.x == 0) {
        const unsigned r = bar->rounds + 1;
        bar->rounds = r;
        const int act = *(volatile int *)&bar->active;
        const int err = *(volatile int *)&bar->err;
        cudaGraphSetConditional(h, (act > 0 && r < max_rounds && err == 0) ? 1u : 0u);
    }
}
}  // namespace cfem

using namespace cfem;

extern "C" int cfem_mixed_matrix(cfem_ctx *ctx, int64_t n_rows, int32_t bs,
                                 const int32_t *d_row_ptr, const int32_t *d_col,
                                 const double *d_vals64, float *d_vals32,
                                 void *stream) {
    CFEM_API_BEGIN
    CFEM_CHECK(ctx && d_row_ptr && d_col && d_vals64 && d_vals32 && n_rows >= 0 &&
                   (bs == 1 || bs == 3),
               CFEM_ERR_INVALID, "cfem_mixed_matrix: bad args");
    if (n_rows == 0) return CFEM_OK;
    CFEM_TRY(set_device(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;
    if (bs == 1)
        CFEM_LAUNCH(k_mixed_matrix<1>, grid_for(n_rows * MX, 128), 128, 0, s, n_rows,
                    d_row_ptr, d_col, d_vals64, d_vals32);
    else
        CFEM_LAUNCH(k_mixed_matrix<3>, grid_for(n_rows * MX, 128), 128, 0, s, n_rows,
                    d_row_ptr, d_col, d_vals64, d_vals32);
    return CFEM_OK;
    CFEM_API_END
}

extern "C" int cfem_mixed_matrix_batch(cfem_ctx *ctx, const cfem_mixed_job *jobs,
                                       int32_t n_jobs, void *stream) {
    CFEM_API_BEGIN
    CFEM_CHECK(ctx && n_jobs >= 0 && (n_jobs == 0 || jobs), CFEM_ERR_INVALID,
               "cfem_mixed_matrix_batch: bad args");
    std::vector<MixJob> by_bs[2];
    int64_t rows[2] = {0, 0};
    for (int j = 0; j < n_jobs; ++j) {
        const cfem_mixed_job &J = jobs[j];
        CFEM_CHECK(J.n_rows >= 0 && (J.bs == 1 || J.bs == 3) &&
                       (J.n_rows == 0 || (J.d_row_ptr && J.d_col && J.d_vals64 && J.d_vals32)),
                   CFEM_ERR_INVALID, "cfem_mixed_matrix_batch: bad job %d", j);
        if (J.n_rows == 0) continue;
        const int t = J.bs == 3 ? 1 : 0;
        by_bs[t].push_back(MixJob{rows[t], J.n_rows, J.d_row_ptr, J.d_col, J.d_vals64, J.d_vals32});
        rows[t] += J.n_rows;
    }
    if (rows[0] + rows[1] == 0) return CFEM_OK;
    CFEM_TRY(set_device(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;
    for (int t = 0; t < 2; ++t) {
        if (by_bs[t].empty()) continue;
        MixJob *d = nullptr;
        CFEM_TRY(tmp_alloc(&d, by_bs[t].size(), s));
        CFEM_CUDA(cudaMemcpyAsync(d, by_bs[t].data(), by_bs[t].size() * sizeof(MixJob),
                                  cudaMemcpyHostToDevice, s));
        if (t == 0)
            CFEM_LAUNCH(k_mixed_matrix_batch<1>, grid_for(rows[t] * MX, 128), 128, 0, s,
                        (const MixJob *)d, (int)by_bs[t].size(), rows[t]);
        else
            CFEM_LAUNCH(k_mixed_matrix_batch<3>, grid_for(rows[t] * MX, 128), 128, 0, s,
                        (const MixJob *)d, (int)by_bs[t].size(), rows[t]);
        tmp_free(d, s);
    }
    return CFEM_OK;
    CFEM_API_END
}

// Launch for stream capture, with programmatic stream serialisation when
// pdl is set (the captured edge from the previous kernel node becomes a
// programmatic dependency; the kernel waits in pdl_wait()).
template <typename... KArgs, typename... Args>
static void glaunch(bool pdl, void (*kernel)(KArgs...), unsigned grid, unsigned block,
                    cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    (void)cudaLaunchKernelEx(&cfg, kernel, args...);
}

// glaunch with dynamic shared memory.
template <typename... KArgs, typename... Args>
static void glaunch_smem(bool pdl, void (*kernel)(KArgs...), unsigned grid, unsigned block,
                         size_t smem, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    (void)cudaLaunchKernelEx(&cfg, kernel, args...);
}

template <typename T>
static int gxs3_prepare() {
    const size_t bytes = gxs3_smem<T>();
    CFEM_CUDA(cudaFuncSetAttribute(k_gxs3<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)bytes));
    int pct = (int)((3 * (bytes + 1024) * 100 + 228 * 1024 - 1) / (228 * 1024));
    if (pct > 100) pct = 100;
    CFEM_CUDA(cudaFuncSetAttribute(k_gxs3<T>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                   pct));
    return CFEM_OK;
}

template <typename T, int LPR>
static int gxs_prepare() {
    const size_t bytes = gxs_smem<T>();
    CFEM_CUDA(cudaFuncSetAttribute(k_gxs<T, LPR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)bytes));
    // shared-memory share of the unified L1 for the resident blocks
    constexpr int nb = StageUnits<T>::BLOCKS;
    int pct = (int)((nb * (bytes + 1024) * 100 + 228 * 1024 - 1) / (228 * 1024));
    if (pct > 100) pct = 100;
    CFEM_CUDA(cudaFuncSetAttribute(k_gxs<T, LPR>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                   pct));
    return CFEM_OK;
}

// ---------------------------------------------------------------------------
// Solve plans. A plan holds everything a batch of systems needs on the
// device between solves: the system table, the work lists, the entry-major
// (3x3) or unit-padded (scalar) working copies of the matrix values, the
// solver vectors and the captured iteration graphs, plus its own stream,
// events and pinned polling words (plans of one context can run from
// different host threads and overlap on the device). A solve resets the
// solver state, runs k_pcg_init and then the persistent kernel or graph
// replays until every system has finished.
struct cfem_pcg_plan {
    cfem_ctx *ctx = nullptr;
    int device = 0;
    int n_systems = 0;
    int n_chunks = 0;
    int max_iter = 1;
    bool persistent = true;
    int grid = 1;
    unsigned long long bar_timeout_ns = 4000000000ull;   // grid-barrier wait limit
    unsigned bar_hold = 0;                               // phantom arrivals (tests)
    int per_iter = 0;
    std::vector<cfem::SysDev> hs;
    char *ws_copy = nullptr;      // system table, lists, working matrix copies
    char *ws_state = nullptr;     // vectors, partials, states, barrier
    char *ws_smeta = nullptr;     // sliced-ELL row orders and slice offsets
    char *ws_sdata = nullptr;     // sliced-ELL columns and values
    size_t state_bytes = 0;
    cfem::SysDev *d_sys = nullptr;
    cfem::SysState *d_st = nullptr;
    int32_t *d_chunks = nullptr;
    cfem::GridBar *d_bar = nullptr;
    cudaStream_t w = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t tev[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    int *h_flags = nullptr;       // pinned: [0..1] polled active counts, [2] active
                                  // count sent, [3] error word, [4] loop rounds
    cfem::SysState *h_st = nullptr;   // pinned: the systems' states after a solve
    cudaStream_t w2 = nullptr;    // captures the loop body
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    // host-polled variant (CFEM_SCHED_GRAPH_POLLED): two instantiations of
    // POLL_ITERS iterations replayed in turn
    bool polled = false;
    int giters = 2;               // iterations per body of the solve loop
    int lanes3 = 4;               // sliced ELL of 3x3 systems: lanes per block row
    int staged3 = 2;              // ... streamed through shared memory (k_gxl3s): 1 both
                                  // precisions, 2 FP32 only, 0 neither
    // solve slots (cfem_pcg_slots_*): each system of the plan is a slot of
    // fixed capacity whose system is replaced between rounds of iterations
    bool slots = false;
    std::vector<int64_t> cap_rows, cap_nnzb;
    // 3x3 slots in the sliced-ELL layout: entries each slot's copy holds,
    // two sets of row orders and slice offsets per slot (the system being
    // assigned ranks into the set the slot's last system did not use, on the
    // caller's stream, while rounds of the others may still read the other),
    // the set in use, the slice-size scan's scratch and a pinned word for
    // the layout's size
    struct SellMeta {
        uint8_t *perm;
        int64_t *sizes;
        int64_t *soff;
    };
    std::vector<int64_t> cap_sell;
    std::vector<SellMeta> smeta;      // slot i, set k at 2 i + k
    std::vector<int> mset;
    std::vector<cudaEvent_t> sev;     // per slot: its last assignment's table update ran
    char *scan_tmp = nullptr;
    size_t scan_bytes = 0;
    int64_t *h_total = nullptr;
    std::vector<cfem::SysDev> tmpl;   // slot templates: workspace pointers
    char *tmpl_mem = nullptr;         // the templates' placeholder CSR
    cudaGraph_t pgraph[2] = {nullptr, nullptr};
    cudaGraphExec_t pexec[2] = {nullptr, nullptr};
};

namespace cfem {

static size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

// (Re)build the working copies of the matrix values on stream s.
static int plan_copies(cfem_pcg_plan *P, cudaStream_t s, int first = 0, int last = -1) {
    if (last < 0) last = P->n_systems;
    std::vector<PadJob> pad_jobs;
    int64_t pad_rows = 0;
    for (int i = first; i < last; ++i) {
        SysDev &S = P->hs[i];
        if (S.bs == 3 && S.sell) {
            const unsigned nw = (unsigned)sell_windows(S.n);
            const int rs = sell_slice_rows(3, P->lanes3);
            auto fill = [&](auto kernel, const auto *v, auto *out) -> int {
                CFEM_LAUNCH(kernel, nw, SELL_ROWS, 0, s, S.n, S.rp, S.ci, v, S.sperm, S.soff,
                            (int32_t *)S.scol, out);
                return CFEM_OK;
            };
            if (S.mode == CFEM_SOLVE_MIXED) {
                float *o = (float *)S.sval;
                CFEM_TRY(rs == 32 ? fill(k_sell_fill3<float, 32>, S.v32, o)
                         : rs == 16 ? fill(k_sell_fill3<float, 16>, S.v32, o)
                                    : fill(k_sell_fill3<float, 8>, S.v32, o));
            } else {
                double *o = (double *)S.sval;
                CFEM_TRY(rs == 32 ? fill(k_sell_fill3<double, 32>, S.v64, o)
                         : rs == 16 ? fill(k_sell_fill3<double, 16>, S.v64, o)
                                    : fill(k_sell_fill3<double, 8>, S.v64, o));
            }
        } else if (S.bs == 3 && S.c3) {
            const unsigned g = std::min(grid_for(S.n * 32, 256), (unsigned)P->ctx->num_sms * 16);
            if (S.mode == CFEM_SOLVE_MIXED)
                CFEM_LAUNCH(k_pad3<float>, g, 256, 0, s, S.n, S.rp, S.ci, S.v32,
                            (int32_t *)S.c3, (float *)S.v3);
            else
                CFEM_LAUNCH(k_pad3<double>, g, 256, 0, s, S.n, S.rp, S.ci, S.v64,
                            (int32_t *)S.c3, (double *)S.v3);
        } else if (S.bs == 3 && S.vsoa) {
            if (S.mode == CFEM_SOLVE_MIXED)
                CFEM_LAUNCH((k_to_soa<float, float, 9>), grid_for(S.nnzb, 256), 256, 0,
                            s, S.nnzb, S.v32, (float *)S.vsoa);
            else
                CFEM_LAUNCH((k_to_soa<double, double, 9>), grid_for(S.nnzb, 256), 256, 0,
                            s, S.nnzb, S.v64, (double *)S.vsoa);
        } else if (S.vec4) {
            const unsigned g = std::min(grid_for(S.n * 32, 256), (unsigned)P->ctx->num_sms * 16);
            if (S.rsell)
                CFEM_LAUNCH(k_sell_fill<double>, (unsigned)sell_windows(S.n), SELL_ROWS, 0, s, S.n, S.rp,
                            S.ci, S.v64, S.sperm, S.soff, (int32_t *)S.scol, (double *)S.sval);
            if (S.sell) {
                if (S.mode == CFEM_SOLVE_MIXED)
                    CFEM_LAUNCH(k_sell_fill<float>, (unsigned)sell_windows(S.n), SELL_ROWS, 0, s, S.n, S.rp,
                                S.ci, S.v32, S.sperm, S.soff, (int32_t *)S.scol, (float *)S.sval);
                else
                    CFEM_LAUNCH(k_sell_fill<double>, (unsigned)sell_windows(S.n), SELL_ROWS, 0, s, S.n, S.rp,
                                S.ci, S.v64, S.sperm, S.soff, (int32_t *)S.scol, (double *)S.sval);
            }
            // unit-padded copies: one batched launch for all systems below
            PadJob J;
            J.row0 = pad_rows;
            J.n = S.n;
            J.rp = S.rp;
            J.ci = S.ci;
            const bool f32 = S.mode == CFEM_SOLVE_MIXED && !S.sell;
            J.v32 = f32 ? S.v32 : nullptr;
            J.va4 = f32 ? (float *)S.va4 : nullptr;
            J.v64 = S.v64;
            J.va4d = (double *)S.va4d;
            J.ci4 = (int32_t *)S.ci4;
            if (S.n > 0) {
                pad_jobs.push_back(J);
                pad_rows += S.n;
            }
            (void)g;
        }
    }
    if (!pad_jobs.empty()) {
        PadJob *d_jobs = nullptr;
        CFEM_TRY(tmp_alloc(&d_jobs, pad_jobs.size(), s));
        CFEM_CUDA(cudaMemcpyAsync(d_jobs, pad_jobs.data(), pad_jobs.size() * sizeof(PadJob),
                                  cudaMemcpyHostToDevice, s));
        const unsigned g = std::min(grid_for(pad_rows * 8, 256), (unsigned)P->ctx->num_sms * 16);
        CFEM_LAUNCH(k_pad4_batch, g, 256, 0, s, (const PadJob *)d_jobs, (int)pad_jobs.size(),
                    pad_rows);
        tmp_free(d_jobs, s);
    }
    return CFEM_OK;
}

// Sliced-ELL layout of every system flagged `sell` (or `rsell`: an FP64
// copy for the residual phases of a mixed scalar system): row orders and
// slice offsets (k_sell_rank, then an exclusive scan of the slice sizes),
// then room for the columns and values (filled by plan_copies). Slot plans
// keep two sets of row orders and offsets per slot (the placeholder
// template ranks into set 0; assignments alternate) and room for any
// system within the slot's capacity, bounded below.
static int sell_layout(cfem_pcg_plan *P, cudaStream_t s) {
    size_t meta = 0;
    int64_t max_sl = 0;
    const int sets = P->slots ? 2 : 1;
    for (const SysDev &S : P->hs)
        if (S.sell || S.rsell) {
            const int64_t nw = sell_windows(S.n);
            const int64_t nsl = nw * (SELL_ROWS / sell_slice_rows(S.bs, P->lanes3));
            meta += sets * (align256((size_t)nw * SELL_ROWS) + 2 * align256((nsl + 1) * 8));
            max_sl = std::max(max_sl, nsl + 1);
        }
    if (!meta) return CFEM_OK;
    size_t scan_bytes = 0;
    CFEM_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (const int64_t *)nullptr,
                                            (int64_t *)nullptr, max_sl, s));
    CFEM_TRY(tmp_alloc(&P->ws_smeta, meta, s));
    char *scan_tmp = nullptr;
    CFEM_TRY(tmp_alloc(&scan_tmp, scan_bytes, s));
    size_t o = 0;
    std::vector<int64_t> totals(P->hs.size(), 0);
    if (P->slots) {
        P->smeta.assign(2 * P->hs.size(), cfem_pcg_plan::SellMeta{nullptr, nullptr, nullptr});
        P->mset.assign(P->hs.size(), 0);
        P->cap_sell.assign(P->hs.size(), 0);
    }
    for (size_t i = 0; i < P->hs.size(); ++i) {
        SysDev &S = P->hs[i];
        if (!S.sell && !S.rsell) continue;
        const int rs = sell_slice_rows(S.bs, P->lanes3);
        const int64_t nw = sell_windows(S.n), nsl = nw * (SELL_ROWS / rs);
        uint8_t *perm = nullptr;
        int64_t *sizes = nullptr, *soff = nullptr;
        for (int k = 0; k < sets; ++k) {
            perm = (uint8_t *)(P->ws_smeta + o);
            o += align256((size_t)nw * SELL_ROWS);
            sizes = (int64_t *)(P->ws_smeta + o);
            o += align256((nsl + 1) * 8);
            soff = (int64_t *)(P->ws_smeta + o);
            o += align256((nsl + 1) * 8);
            if (P->slots) P->smeta[2 * i + (sets - 1 - k)] = {perm, sizes, soff};
        }   // the last set taken (set 0 of a slot) is ranked now
        CFEM_CUDA(cudaMemsetAsync(sizes + nsl, 0, sizeof(int64_t), s));
        const int srt = P->ctx->sell_sort;
        if (rs == 32)
            CFEM_LAUNCH(k_sell_rank<32>, (unsigned)nw, SELL_ROWS, 0, s, S.n, S.rp, S.ci, perm, sizes, srt);
        else if (rs == 16)
            CFEM_LAUNCH(k_sell_rank<16>, (unsigned)nw, SELL_ROWS, 0, s, S.n, S.rp, S.ci, perm, sizes, srt);
        else
            CFEM_LAUNCH(k_sell_rank<8>, (unsigned)nw, SELL_ROWS, 0, s, S.n, S.rp, S.ci, perm, sizes, srt);
        CFEM_CUDA(cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, sizes, soff, nsl + 1, s));
        CFEM_CUDA(cudaMemcpyAsync(&totals[i], soff + nsl, sizeof(int64_t),
                                  cudaMemcpyDeviceToHost, s));
        S.sperm = perm;
        S.soff = soff;
    }
    if (P->slots) {          // kept for the systems assigned later
        P->scan_tmp = scan_tmp;
        P->scan_bytes = scan_bytes;
    } else {
        tmp_free(scan_tmp, s);
    }
    CFEM_CUDA(cudaStreamSynchronize(s));
    // Slots: room for any system within the capacity whose longest block
    // row has at most SLOT_SELL_ROW blocks. Windows sorted by length make a
    // slice no longer than the shortest row of the slice before it, so a
    // window's slices hold at most its rows' blocks (+1 for an absent
    // diagonal), RS x its longest row, and L - 1 per row of rounding to
    // whole steps. A system beyond that is refused at assignment.
    for (size_t i = 0; P->slots && i < P->hs.size(); ++i) {
        const SysDev &S = P->hs[i];
        if (!S.sell) continue;
        const int rs = sell_slice_rows(S.bs, P->lanes3), l = 32 / rs;
        const int64_t nw = sell_windows(S.n);
        const int64_t bound = S.nnzb + S.n + nw * ((int64_t)rs * SLOT_SELL_ROW +
                                                   (int64_t)SELL_ROWS * (l - 1));
        totals[i] = std::max(totals[i], bound);
        P->cap_sell[i] = totals[i];
    }
    size_t data = 0;
    for (size_t i = 0; i < P->hs.size(); ++i) {
        const SysDev &S = P->hs[i];
        if (!S.sell && !S.rsell) continue;
        const size_t ts = (S.mode == CFEM_SOLVE_MIXED && S.sell) ? 4 : 8;   // rsell: FP64
        data += align256((size_t)totals[i] * 4) + align256((size_t)totals[i] * S.bs * S.bs * ts);
    }
    CFEM_TRY(tmp_alloc(&P->ws_sdata, data, s));
    o = 0;
    for (size_t i = 0; i < P->hs.size(); ++i) {
        SysDev &S = P->hs[i];
        if (!S.sell && !S.rsell) continue;
        const size_t ts = (S.mode == CFEM_SOLVE_MIXED && S.sell) ? 4 : 8;   // rsell: FP64
        S.scol = (const int32_t *)(P->ws_sdata + o);
        o += align256((size_t)totals[i] * 4);
        S.sval = P->ws_sdata + o;
        o += align256((size_t)totals[i] * S.bs * S.bs * ts);
    }
    return CFEM_OK;
}

static void plan_free(cfem_pcg_plan *P) {
    if (!P) return;
    cudaSetDevice(P->device);
    if (P->w) cudaStreamSynchronize(P->w);
    if (P->exec) cudaGraphExecDestroy(P->exec);
    if (P->graph) cudaGraphDestroy(P->graph);
    for (int gi = 0; gi < 2; ++gi) {
        if (P->pexec[gi]) cudaGraphExecDestroy(P->pexec[gi]);
        if (P->pgraph[gi]) cudaGraphDestroy(P->pgraph[gi]);
    }
    if (P->w) {
        if (P->ws_copy) cudaFreeAsync(P->ws_copy, P->w);
        if (P->ws_state) cudaFreeAsync(P->ws_state, P->w);
        if (P->ws_smeta) cudaFreeAsync(P->ws_smeta, P->w);
        if (P->tmpl_mem) cudaFreeAsync(P->tmpl_mem, P->w);
        if (P->ws_sdata) cudaFreeAsync(P->ws_sdata, P->w);
        if (P->scan_tmp) cudaFreeAsync(P->scan_tmp, P->w);
        cudaStreamSynchronize(P->w);
    }
    for (int i = 0; i < 4; ++i)
        if (P->ev[i]) cudaEventDestroy(P->ev[i]);
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j)
            if (P->tev[i][j]) cudaEventDestroy(P->tev[i][j]);
    if (P->h_flags) cudaFreeHost(P->h_flags);
    if (P->h_st) cudaFreeHost(P->h_st);
    if (P->h_total) cudaFreeHost(P->h_total);
    for (cudaEvent_t e : P->sev)
        if (e) cudaEventDestroy(e);
    if (P->w2) cudaStreamDestroy(P->w2);
    if (P->w) cudaStreamDestroy(P->w);
    (void)cudaGetLastError();
    delete P;
}

static int plan_build(cfem_ctx *ctx, const cfem_linsys *systems, int n_systems,
                      cudaStream_t s, cfem_pcg_plan *P) {
    P->ctx = ctx;
    P->device = ctx->device;
    P->lanes3 = ctx->sell3_lanes;
    P->staged3 = ctx->sell3_staged;
    P->n_systems = n_systems;
    CFEM_CUDA(cudaStreamCreateWithFlags(&P->w, cudaStreamNonBlocking));
    CFEM_CUDA(cudaStreamCreateWithFlags(&P->w2, cudaStreamNonBlocking));
    for (int i = 0; i < 4; ++i)
        CFEM_CUDA(cudaEventCreateWithFlags(&P->ev[i], i < 2 ? cudaEventDisableTiming
                                                            : cudaEventDefault));
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j) CFEM_CUDA(cudaEventCreate(&P->tev[i][j]));
    CFEM_CUDA(cudaMallocHost(&P->h_flags, 8 * sizeof(int)));
    CFEM_CUDA(cudaMallocHost(&P->h_st, (size_t)n_systems * sizeof(SysState)));
    std::vector<SysDev> &hs = P->hs;
    hs.assign(n_systems, SysDev{});
    std::vector<int32_t> chunk_sys;
    int max_iter = 1;
    int64_t n_chunks_b = 0;
    std::vector<int32_t> nnzbs(n_systems, 0);
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
        CFEM_CUDA(cudaMemcpyAsync(&nnzbs[i], L.d_row_ptr + L.n_rows, sizeof(int32_t),
                                  cudaMemcpyDeviceToHost, s));
    }
    CFEM_CUDA(cudaStreamSynchronize(s));
    size_t state_bytes = 0, copy_bytes = 0;
    for (int i = 0; i < n_systems; ++i) {
        const cfem_linsys &L = systems[i];
        SysDev &S = hs[i];
        S.n = L.n_rows;
        S.bs = L.bs;
        S.precond = (L.bs == 3) ? L.precond : CFEM_PRECOND_JACOBI;
        S.mode = L.mode;
        S.crows = chunk_rows(L.bs);
        S.nchunks = (int32_t)((L.n_rows + S.crows - 1) / S.crows);
        S.ntiles = (S.nchunks + TILE - 1) / TILE;
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
        const double dl = L.reliable_delta > 0.0 ? L.reliable_delta : RELIABLE_DELTA;
        S.delta2 = dl * dl;
        S.max_stall = L.max_stall > 0 ? L.max_stall : MAX_STALL;
        S.hist_cap = L.d_history ? L.history_cap : 0;
        S.hist = L.d_history;
        for (int c = 0; c < S.nchunks; ++c) chunk_sys.push_back(i);
        S.nchunksB = (int32_t)((L.n_rows + brows(L.bs) - 1) / brows(L.bs));
        S.nnzb = nnzbs[i];
        const size_t ts = (L.mode == CFEM_SOLVE_MIXED) ? 4 : 8;
        const size_t nd = (size_t)L.n_rows * L.bs;
        const size_t nprec = (S.precond == CFEM_PRECOND_BLOCK) ? (size_t)L.n_rows * 9 : nd;
        state_bytes += 5 * align256(nd * ts) + align256(nprec * ts) +
                       align256(S.nchunks * 4 * sizeof(double)) +
                       align256(S.ntiles * 4 * sizeof(double)) +
                       align256(S.ntiles * sizeof(unsigned)) +
                       align256(S.nchunksB * 4 * sizeof(double));
        n_chunks_b += S.nchunksB;
        if (L.max_iter > max_iter) max_iter = L.max_iter;
    }
    const int n_chunks = (int)chunk_sys.size();
    P->n_chunks = n_chunks;
    P->max_iter = max_iter;
    int per_sm = 0;
    CFEM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, k_pcg_persistent, SOLVE_THREADS, 0));
    CFEM_CHECK(per_sm > 0, CFEM_ERR_CUDA, "solver kernel cannot be resident");
    int grid = ctx->num_sms * per_sm;
    const int useful = (n_chunks * 32 + SOLVE_THREADS - 1) / SOLVE_THREADS;
    // One resident wave holds every chunk: the persistent kernel pays a grid
    // barrier per phase and no launches. Otherwise the graph scheduler keeps
    // the SMs fed with one warp per chunk per launch.
    const bool persistent = !P->slots &&
                            (ctx->scheduler == CFEM_SCHED_PERSISTENT ||
                             (ctx->scheduler == CFEM_SCHED_AUTO && useful <= grid));
    if (grid > useful) grid = useful < 1 ? 1 : useful;
    if (grid > BAR_GROUP * BAR_MAX_GROUPS) grid = BAR_GROUP * BAR_MAX_GROUPS;
    P->persistent = persistent;
    P->grid = grid;
    P->bar_timeout_ns = 1000ull * (unsigned long long)ctx->barrier_timeout_us;
    P->bar_hold = (unsigned)ctx->barrier_hold;
    // Scalar systems on the graph scheduler read a unit-padded copy; 3x3
    // systems a padded block copy (staged SpMV) or an entry-major copy.
    // SpMV staging per list type t = 2 (mixed) + (3x3): explicit, or AUTO
    // (4): sliced ELL for FP64 scalar rows and for 3x3 blocks in both
    // precisions (slices of 32 / L block rows, L lanes per block row), the
    // bulk-staged windows for FP32 scalar rows (the fastest measured for
    // each on the benchmark workloads)
    int tstage[4];
    for (int t = 0; t < 4; ++t)
        tstage[t] = ctx->spmv_stage != 4 ? ctx->spmv_stage : (t == 2 ? 1 : 3);
    // solve slots: scalar rows from the unit-padded copy (its size follows
    // the capacity alone); 3x3 blocks in the sliced ELL (SLOT_SELL3, room
    // for a bound on the padding, the layout built at assignment) or from
    // the entry-major copy
    if (P->slots)
        for (int t = 0; t < 4; ++t) tstage[t] = (t & 1) ? (ctx->slot_sell3 ? 3 : 0) : 1;
    auto stage_of = [&](const SysDev &S) {
        return tstage[(S.mode == CFEM_SOLVE_MIXED ? 2 : 0) + (S.bs == 3 ? 1 : 0)];
    };
    if (!persistent)
        for (int i = 0; i < n_systems; ++i) {
            const size_t ts = (hs[i].mode == CFEM_SOLVE_MIXED) ? 4 : 8;
            if (hs[i].bs == 1) {
                const size_t ne = (size_t)hs[i].nnzb + 3 * (size_t)hs[i].n + 8;
                copy_bytes += align256(ne * 4) + align256(ne * 8) +
                              (hs[i].mode == CFEM_SOLVE_MIXED && stage_of(hs[i]) != 3
                                   ? align256(ne * 4) : 0);
            } else if (stage_of(hs[i]) == 2) {
                const size_t ne = (size_t)hs[i].nnzb + 3 * (size_t)hs[i].n + 8;
                copy_bytes += align256(ne * 4) + align256(ne * 9 * ts);
            } else if (stage_of(hs[i]) == 3) {
                // sliced-ELL copy allocated by sell_layout
            } else {
                copy_bytes += align256((size_t)hs[i].nnzb * 9 * ts);
            }
        }
    const size_t list_a = n_chunks + (size_t)GROUP * n_systems;
    const size_t list_b = n_chunks_b + (size_t)GROUP * n_systems;
    copy_bytes += align256(n_systems * sizeof(SysDev)) + align256(n_chunks * sizeof(int32_t)) +
                  align256(list_a * sizeof(int2)) + align256(list_b * sizeof(int2));
    state_bytes += align256(n_systems * sizeof(SysState)) + align256(sizeof(GridBar));
    CFEM_TRY(tmp_alloc(&P->ws_copy, copy_bytes, s));
    CFEM_TRY(tmp_alloc(&P->ws_state, state_bytes, s));
    P->state_bytes = state_bytes;
    size_t oc = 0, os = 0;
    auto take_c = [&](size_t b) { char *p = P->ws_copy + oc; oc += align256(b); return (void *)p; };
    auto take_s = [&](size_t b) { char *p = P->ws_state + os; os += align256(b); return (void *)p; };
    for (int i = 0; i < n_systems; ++i) {
        SysDev &S = hs[i];
        const size_t ts = (S.mode == CFEM_SOLVE_MIXED) ? 4 : 8;
        const size_t nd = (size_t)S.n * S.bs;
        const size_t nprec = (S.precond == CFEM_PRECOND_BLOCK) ? (size_t)S.n * 9 : nd;
        S.r = take_s(nd * ts);
        S.z = take_s(nd * ts);
        S.p0 = take_s(nd * ts);
        S.p1 = take_s(nd * ts);
        S.q = take_s(nd * ts);
        S.dinv = take_s(nprec * ts);
        S.partial = (double *)take_s(S.nchunks * 4 * sizeof(double));
        S.tpartial = (double *)take_s(S.ntiles * 4 * sizeof(double));
        S.tcnt = (unsigned *)take_s(S.ntiles * sizeof(unsigned));
        S.partialB = (double *)take_s(S.nchunksB * 4 * sizeof(double));
        if (S.bs == 3) {
            if (!persistent && stage_of(S) == 2) {
                const size_t ne = (size_t)S.nnzb + 3 * (size_t)S.n + 8;
                S.c3 = (const int32_t *)take_c(ne * 4);
                S.v3 = take_c(ne * 9 * ts);
            } else if (!persistent && stage_of(S) == 3) {
                S.sell = 1;
            } else if (!persistent) {
                S.vsoa = take_c((size_t)S.nnzb * 9 * ts);
            }
        } else {
            S.vsoa = (S.mode == CFEM_SOLVE_MIXED) ? (const void *)S.v32 : (const void *)S.v64;
            if (!persistent) {
                const size_t ne = (size_t)S.nnzb + 3 * (size_t)S.n + 8;
                S.ci4 = (const int32_t *)take_c(ne * 4);
                S.va4d = (const double *)take_c(ne * 8);
                const bool sell = stage_of(S) == 3;
                S.va4 = (S.mode == CFEM_SOLVE_MIXED) ? (sell ? nullptr : take_c(ne * 4))
                                                     : (const void *)S.va4d;
                S.vec4 = 1;
                S.sell = sell ? 1 : 0;
                // short rows (P1: up to 16 entries, 4 units) on 4 lanes each
                S.lpr = S.nnzb <= 16 * S.n ? 4 : 8;
                // mixed P1 systems (a few iterations per solve, a residual
                // phase nearly every iteration: time marches) take their
                // FP64 residual from a sliced-ELL copy, one row per lane
                S.rsell = (CFEM_RESIDUAL_SELL && !sell && !P->slots &&
                           S.mode == CFEM_SOLVE_MIXED && S.lpr == 4) ? 1 : 0;
            }
        }
        // Scalar rows from the padded copy: eight chunks per SpMV work entry,
        // so a warp's set-up (work entry, system, state) is paid per 128 rows
        // (measured 1.8x faster than one chunk on the batched heat meshes; 3x3
        // systems keep one chunk: fewer, longer warps measured slower there).
        S.xrows = S.sell ? sell_slice_rows(S.bs, P->lanes3)               // one slice
                         : (S.vec4 ? X_CHUNKS_VEC : 1) * S.crows;
        CFEM_CHECK(!S.c3 || S.xrows <= XR3, CFEM_ERR_UNSUPPORTED,
                   "staged 3x3 work entries hold at most %d block rows", XR3);
        S.nxe = (int32_t)((S.n + S.xrows - 1) / S.xrows);
    }
    P->d_st = (SysState *)take_s(n_systems * sizeof(SysState));
    P->d_bar = (GridBar *)take_s(sizeof(GridBar));
    P->d_sys = (SysDev *)take_c(n_systems * sizeof(SysDev));
    P->d_chunks = (int32_t *)take_c(n_chunks * sizeof(int32_t));
    int2 *d_lista = (int2 *)take_c(list_a * sizeof(int2));
    int2 *d_listb = (int2 *)take_c(list_b * sizeof(int2));
    CFEM_TRY(sell_layout(P, s));
    CFEM_TRY(plan_copies(P, s));
    CFEM_CUDA(cudaMemcpyAsync(P->d_sys, hs.data(), n_systems * sizeof(SysDev),
                              cudaMemcpyHostToDevice, s));
    CFEM_CUDA(cudaMemcpyAsync(P->d_chunks, chunk_sys.data(),
                              n_chunks * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    if (persistent) {
        // host staging must stay valid until the copies ran
        CFEM_CUDA(cudaStreamSynchronize(s));
        return CFEM_OK;
    }
    // Work lists per (precision, block size): {system, chunk} pairs.
    std::vector<int2> la[4], lb[4];
    for (int i = 0; i < n_systems; ++i) {
        const int t = (hs[i].mode == CFEM_SOLVE_MIXED ? 2 : 0) + (hs[i].bs == 3 ? 1 : 0);
        for (int c = 0; c < hs[i].nxe; ++c) la[t].push_back(make_int2(i, c));
        while (la[t].size() % GROUP) la[t].push_back(make_int2(-1, -1));
        for (int c = 0; c < hs[i].nchunksB; ++c) lb[t].push_back(make_int2(i, c));
        while (lb[t].size() % GROUP) lb[t].push_back(make_int2(-1, -1));
    }
    {
        size_t na = 0, nb = 0;
        for (int t = 0; t < 4; ++t) {
            na += la[t].size();
            nb += lb[t].size();
        }
        CFEM_CHECK(na <= list_a && nb <= list_b, CFEM_ERR_INVALID,
                   "work lists (%zu, %zu entries) exceed their allocation (%zu, %zu)", na, nb,
                   list_a, list_b);
    }
    int2 *pa[4], *pb[4];
    size_t oa = 0, ob = 0;
    for (int t = 0; t < 4; ++t) {
        pa[t] = d_lista + oa;
        pb[t] = d_listb + ob;
        if (!la[t].empty())
            CFEM_CUDA(cudaMemcpyAsync(pa[t], la[t].data(), la[t].size() * sizeof(int2),
                                      cudaMemcpyHostToDevice, s));
        if (!lb[t].empty())
            CFEM_CUDA(cudaMemcpyAsync(pb[t], lb[t].data(), lb[t].size() * sizeof(int2),
                                      cudaMemcpyHostToDevice, s));
        oa += la[t].size();
        ob += lb[t].size();
    }
    CFEM_CUDA(cudaStreamSynchronize(s));
    cudaStream_t w = P->w;
    SysDev *d_sys = P->d_sys;
    SysState *d_st = P->d_st;
    GridBar *d_bar = P->d_bar;
    int per_iter = 2;
    // One iteration: direction (scalar systems), SpMV, reduction, update,
    // reduction. The SpMV of the first iteration is bracketed by the
    // timing events when tev is given.
    const bool use_pdl = ctx->pdl != 0;
    // scalar SpMV: bulk-staged windows (1, 2) or the register path (0); 3x3
    // SpMV: bulk-staged (2) or the register path (0, 1); lanes
    // per row from the mean row length of the list's systems (4 up to 16
    // entries, whole units of a P1 row; 8 above, Tet10 rows of ~27)
    int lpr[4] = {8, 8, 8, 8};
    for (int t = 0; t < 4; t += 2) {
        double nz = 0.0, rows = 0.0;
        for (int i = 0; i < n_systems; ++i)
            if (hs[i].bs == 1 && (hs[i].mode == CFEM_SOLVE_MIXED) == (t == 2)) {
                nz += (double)hs[i].nnzb;
                rows += (double)hs[i].n;
            }
        if (rows > 0 && nz <= 16.0 * rows) lpr[t] = 4;
    }
    if ((tstage[0] == 1 || tstage[0] == 2) && !la[0].empty())
        CFEM_TRY((lpr[0] == 4 ? gxs_prepare<double, 4>() : gxs_prepare<double, 8>()));
    if ((tstage[2] == 1 || tstage[2] == 2) && !la[2].empty())
        CFEM_TRY((lpr[2] == 4 ? gxs_prepare<float, 4>() : gxs_prepare<float, 8>()));
    if (tstage[1] == 2 && !la[1].empty()) CFEM_TRY(gxs3_prepare<double>());
    if (tstage[1] == 3 && P->staged3 == 1 && !la[1].empty()) CFEM_TRY(gxl3s_prepare<double>(P->lanes3));
    if (tstage[3] == 3 && P->staged3 && !la[3].empty()) CFEM_TRY(gxl3s_prepare<float>(P->lanes3));
    if (tstage[3] == 2 && !la[3].empty()) CFEM_TRY(gxs3_prepare<float>());
    auto iteration = [&](cudaStream_t cs, bool count, cudaEvent_t t0, cudaEvent_t t1) -> int {
        // dependent launches only between kernel nodes (not next to events)
        const bool pdl = use_pdl && !t0;
        bool first = true;
        auto L = [&](bool p) { const bool r = p && !first; first = false; return r; };
        for (int t = 0; t < 4; t += 2) {   // scalar types only
            const int n = (int)lb[t].size();
            if (!n) continue;
            const unsigned g = (unsigned)(n / GROUP);
            if (t == 0) glaunch(L(pdl), k_gp<double, 1>, g, 32 * GROUP, cs, (const SysDev *)d_sys, d_st, (const GridBar *)d_bar, (const int2 *)pb[t], n);
            if (t == 2) glaunch(L(pdl), k_gp<float, 1>, g, 32 * GROUP, cs, (const SysDev *)d_sys, d_st, (const GridBar *)d_bar, (const int2 *)pb[t], n);
            if (count) ++per_iter;
        }
        if (t0) CFEM_CUDA(cudaEventRecordWithFlags(t0, cs, cudaEventRecordExternal));
        first = first || t0 != nullptr;
        for (int t = 0; t < 4; ++t) {
            const int n = (int)la[t].size();
            if (!n) continue;
            const unsigned g = (unsigned)(n / GROUP);
            const bool p = L(pdl);
            const int stage = tstage[t];
            if (t == 0 && stage == 3) glaunch(p, k_gxl<double>, g, 32 * GROUP, cs, (const SysDev *)d_sys, d_st, (const GridBar *)d_bar, (const int2 *)pa[t], n);
            if (t == 2 && stage == 3) glaunch(p, k_gxl<float>, g, 32 * GROUP, cs, (const SysDev *)d_sys, d_st, (const GridBar *)d_bar, (const int2 *)pa[t], n);
            if (t == 0 && (stage == 1 || stage == 2))
                glaunch_smem(p, lpr[0] == 4 ? k_gxs<double, 4> : k_gxs<double, 8>, g, 32 * GROUP, gxs_smem<double>(), cs, (const SysDev *)d_sys, d_st, d_bar, (const int2 *)pa[t], n);
            if (t == 2 && (stage == 1 || stage == 2))
                glaunch_smem(p, lpr[2] == 4 ? k_gxs<float, 4> : k_gxs<float, 8>, g, 32 * GROUP, gxs_smem<float>(), cs, (const SysDev *)d_sys, d_st, d_bar, (const int2 *)pa[t], n);
            if (t == 0 && stage == 0) glaunch(p, k_gx<double, 1>, g, 32 * GROUP, cs, (const SysDev *)d_sys, d_st, (const GridBar *)d_bar, (const int2 *)pa[t], n);
            if (t == 1 && stage == 2)
                glaunch_smem(p, k_gxs3<double>, g, 32 * GROUP, gxs3_smem<double>(), cs, (const SysDev *)d_sys, d_st, d_bar, (const int2 *)pa[t], n);
            if (t == 1 && stage == 3 && P->staged3 == 1)
                glaunch_smem(p, gxl3s_kernel<double>(P->lanes3), g, 32 * GROUP, gxl3s_smem<double>(), cs, (const SysDev *)d_sys, d_st, d_bar, (const int2 *)pa[t], n);
            if (t == 1 && stage == 3 && P->staged3 != 1) glaunch(p, gxl3_kernel<double>(P->lanes3), g, 32 * GROUP, cs, (const SysDev *)d_sys, d_st, (const GridBar *)d_bar, (const int2 *)pa[t], n);
            if (t == 1 && stage < 2) glaunch(p, k_gx<double, 3>, g, 32 * GROUP, cs, (const SysDev *)d_sys, d_st, (const GridBar *)d_bar, (const int2 *)pa[t], n);
            if (t == 2 && stage == 0) glaunch(p, k_gx<float, 1>, g, 32 * GROUP, cs, (const SysDev *)d_sys, d_st, (const GridBar *)d_bar, (const int2 *)pa[t], n);
            if (t == 3 && stage == 2)
                glaunch_smem(p, k_gxs3<float>, g, 32 * GROUP, gxs3_smem<float>(), cs, (const SysDev *)d_sys, d_st, d_bar, (const int2 *)pa[t], n);
            if (t == 3 && stage == 3 && P->staged3)
                glaunch_smem(p, gxl3s_kernel<float>(P->lanes3), g, 32 * GROUP, gxl3s_smem<float>(), cs, (const SysDev *)d_sys, d_st, d_bar, (const int2 *)pa[t], n);
            if (t == 3 && stage == 3 && P->staged3 == 0) glaunch(p, gxl3_kernel<float>(P->lanes3), g, 32 * GROUP, cs, (const SysDev *)d_sys, d_st, (const GridBar *)d_bar, (const int2 *)pa[t], n);
            if (t == 3 && stage < 2) glaunch(p, k_gx<float, 3>, g, 32 * GROUP, cs, (const SysDev *)d_sys, d_st, (const GridBar *)d_bar, (const int2 *)pa[t], n);
            if (count) ++per_iter;
        }
        if (t1) CFEM_CUDA(cudaEventRecordWithFlags(t1, cs, cudaEventRecordExternal));
        first = first || t1 != nullptr;
        glaunch(L(use_pdl), k_greduce, n_systems, RED_THREADS, cs, (const SysDev *)d_sys, d_st, d_bar, 0);
        for (int t = 0; t < 4; ++t) {
            const int n = (int)lb[t].size();
            if (!n) continue;
            const unsigned g = (unsigned)(n / GROUP);
            const bool p = L(use_pdl);
            if (t == 0) glaunch(p, k_gb<double, 1>, g, 32 * GROUP, cs, (const SysDev *)d_sys, d_st, (const GridBar *)d_bar, (const int2 *)pb[t], n);
            if (t == 1) glaunch(p, k_gb<double, 3>, g, 32 * GROUP, cs, (const SysDev *)d_sys, d_st, (const GridBar *)d_bar, (const int2 *)pb[t], n);
            if (t == 2) glaunch(p, k_gb<float, 1>, g, 32 * GROUP, cs, (const SysDev *)d_sys, d_st, (const GridBar *)d_bar, (const int2 *)pb[t], n);
            if (t == 3) glaunch(p, k_gb<float, 3>, g, 32 * GROUP, cs, (const SysDev *)d_sys, d_st, (const GridBar *)d_bar, (const int2 *)pb[t], n);
            if (count) ++per_iter;
        }
        glaunch(L(use_pdl), k_greduce, n_systems, RED_THREADS, cs, (const SysDev *)d_sys, d_st, d_bar, 1);
        CFEM_CUDA(cudaGetLastError());
        return CFEM_OK;
    };
    // The whole solve is one graph: reset of the solver state, k_pcg_init,
    // a first (timed) iteration, then a device-side WHILE loop of bodies of
    // GRAPH_ITERS iterations that ends when no system is active. No host
    // polling; at most GRAPH_ITERS - 1 iterations run past convergence
    // (their kernels return at once for finished systems).
    if (ctx->scheduler == CFEM_SCHED_GRAPH_POLLED || P->slots) {
        // Plain graphs of POLL_ITERS iterations replayed by the host, which
        // polls the active count one replay behind (every kernel launch is
        // visible to per-launch profilers).
        P->polled = true;
        for (int gi = 0; gi < 2; ++gi) {
            CFEM_CUDA(cudaStreamBeginCapture(w, cudaStreamCaptureModeThreadLocal));
            for (int it = 0; it < POLL_ITERS; ++it)
                CFEM_TRY(iteration(w, it == 0 && gi == 0, it == 0 ? P->tev[gi][0] : nullptr,
                                   it == 0 ? P->tev[gi][1] : nullptr));
            cudaError_t ce = cudaStreamEndCapture(w, &P->pgraph[gi]);
            CFEM_CUDA(ce);
            CFEM_CUDA(cudaGetLastError());
            CFEM_CUDA(cudaGraphInstantiate(&P->pexec[gi], P->pgraph[gi], 0));
        }
        P->per_iter = per_iter;
        return CFEM_OK;
    }
    P->giters = ctx->graph_iters;
    const int GRAPH_ITERS = P->giters;
    const unsigned max_rounds = (unsigned)((2 * max_iter + 32) / GRAPH_ITERS + 2);
    CFEM_CUDA(cudaStreamBeginCapture(w, cudaStreamCaptureModeThreadLocal));
    CFEM_CUDA(cudaMemsetAsync(P->ws_state, 0, P->state_bytes, w));
    k_plan_start<<<1, 32, 0, w>>>(d_bar, n_systems);
    k_pcg_init<<<grid_for((int64_t)n_chunks * 32, 256), 256, 0, w>>>(
        d_sys, d_st, P->d_chunks, n_chunks, d_bar);
    CFEM_TRY(iteration(w, false, P->tev[0][0], P->tev[0][1]));
    cudaStreamCaptureStatus cst;
    cudaGraph_t cap = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    CFEM_CUDA(cudaStreamGetCaptureInfo(w, &cst, nullptr, &cap, &deps, &ndeps));
    cudaGraphConditionalHandle handle;
    CFEM_CUDA(cudaGraphConditionalHandleCreate(&handle, cap, 1, cudaGraphCondAssignDefault));
    k_loop_cond<<<1, 32, 0, w>>>(handle, d_bar, max_rounds);
    CFEM_CUDA(cudaStreamGetCaptureInfo(w, &cst, nullptr, &cap, &deps, &ndeps));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t loop;
    CFEM_CUDA(cudaGraphAddNode(&loop, cap, deps, ndeps, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    CFEM_CUDA(cudaStreamUpdateCaptureDependencies(w, &loop, 1, cudaStreamSetCaptureDependencies));
    CFEM_CUDA(cudaStreamBeginCaptureToGraph(P->w2, body, nullptr, nullptr, 0,
                                            cudaStreamCaptureModeThreadLocal));
    for (int it = 0; it < GRAPH_ITERS; ++it) CFEM_TRY(iteration(P->w2, it == 0, nullptr, nullptr));
    glaunch(use_pdl, k_loop_cond, 1, 32, P->w2, handle, d_bar, max_rounds);
    CFEM_CUDA(cudaGetLastError());
    cudaGraph_t body_out = nullptr;
    CFEM_CUDA(cudaStreamEndCapture(P->w2, &body_out));
    cudaError_t ce = cudaStreamEndCapture(w, &P->graph);
    CFEM_CUDA(ce);
    CFEM_CUDA(cudaGetLastError());
    CFEM_CUDA(cudaGraphInstantiate(&P->exec, P->graph, 0));
    P->per_iter = per_iter;
    return CFEM_OK;
}

static int plan_run(cfem_pcg_plan *P, cfem_solve_stats *stats, cudaStream_t s) {
    const int n_systems = P->n_systems;
    cudaStream_t w = P->w;
    SysDev *d_sys = P->d_sys;
    SysState *d_st = P->d_st;
    GridBar *d_bar = P->d_bar;
    int n_chunks = P->n_chunks;
    int max_steps = 3 * P->max_iter + 16;
    double spmv_ms = 0.0;
    int spmv_samples = 0;
    // The plan's stream runs after everything queued so far on s.
    CFEM_CUDA(cudaEventRecord(P->ev[0], s));
    CFEM_CUDA(cudaStreamWaitEvent(w, P->ev[0], 0));
    if (P->persistent || P->polled) {
        CFEM_CUDA(cudaMemsetAsync(P->ws_state, 0, P->state_bytes, w));
        P->h_flags[2] = n_systems;
        CFEM_CUDA(cudaMemcpyAsync(&d_bar->active, &P->h_flags[2], sizeof(int),
                                  cudaMemcpyHostToDevice, w));
        CFEM_CUDA(cudaEventRecord(P->ev[2], w));
        CFEM_LAUNCH(k_pcg_init, grid_for((int64_t)n_chunks * 32, 256), 256, 0, w,
                    d_sys, d_st, P->d_chunks, n_chunks, d_bar);
    }
    if (P->persistent) {
        void *args[] = {(void *)&d_sys, (void *)&d_st, (void *)&P->d_chunks,
                        (void *)&n_chunks, (void *)&d_bar, (void *)&max_steps,
                        (void *)&P->bar_timeout_ns, (void *)&P->bar_hold};
        CFEM_CUDA(cudaLaunchCooperativeKernel((void *)k_pcg_persistent, dim3(P->grid),
                                              dim3(SOLVE_THREADS), args, 0, w));
        g_launches.fetch_add(1, std::memory_order_relaxed);
    } else if (P->polled) {
        const int max_replays = (2 * P->max_iter + 32) / POLL_ITERS + 2;
        volatile int *flags = P->h_flags;
        flags[0] = flags[1] = 1;
        int active_before = n_systems;
        for (int rep = 0; rep < max_replays; ++rep) {
            CFEM_CUDA(cudaGraphLaunch(P->pexec[rep & 1], w));
            g_launches.fetch_add((int64_t)P->per_iter * POLL_ITERS, std::memory_order_relaxed);
            CFEM_CUDA(cudaMemcpyAsync((void *)&P->h_flags[rep & 1], &d_bar->active,
                                      sizeof(int), cudaMemcpyDeviceToHost, w));
            CFEM_CUDA(cudaEventRecord(P->ev[rep & 1], w));
            if (rep >= 1) {
                const int prev = (rep - 1) & 1;
                CFEM_CUDA(cudaEventSynchronize(P->ev[prev]));
                float sms = 0.0f;
                if (cudaEventElapsedTime(&sms, P->tev[prev][0], P->tev[prev][1]) ==
                        cudaSuccess) {
                    if (active_before > 0) {
                        spmv_ms += sms;
                        ++spmv_samples;
                    }
                } else {
                    (void)cudaGetLastError();   // timing is best effort
                }
                active_before = flags[prev];
                if (flags[prev] <= 0) break;
            }
        }
    } else {
        CFEM_CUDA(cudaEventRecord(P->ev[2], w));
        CFEM_CUDA(cudaGraphLaunch(P->exec, w));
    }
    CFEM_CUDA(cudaEventRecord(P->ev[3], w));
    // states, error word and loop rounds into pinned memory: one wait
    const bool graph_loop = !P->persistent && !P->polled;
    CFEM_CUDA(cudaMemcpyAsync(P->h_st, d_st, n_systems * sizeof(SysState),
                              cudaMemcpyDeviceToHost, w));
    CFEM_CUDA(cudaMemcpyAsync(&P->h_flags[3], &d_bar->err, sizeof(int),
                              cudaMemcpyDeviceToHost, w));
    if (graph_loop)
        CFEM_CUDA(cudaMemcpyAsync(&P->h_flags[4], &d_bar->rounds, sizeof(unsigned),
                                  cudaMemcpyDeviceToHost, w));
    CFEM_CUDA(cudaStreamSynchronize(w));
    const SysState *hst = P->h_st;
    const int h_err = P->h_flags[3];
    // later work on s sees the solution
    CFEM_CUDA(cudaEventRecord(P->ev[0], w));
    CFEM_CUDA(cudaStreamWaitEvent(s, P->ev[0], 0));
    float kms = 0.0f;
    CFEM_CUDA(cudaEventElapsedTime(&kms, P->ev[2], P->ev[3]));
    if (graph_loop) {
        const unsigned rounds = (unsigned)P->h_flags[4];
        const int64_t bodies = rounds > 0 ? (int64_t)rounds - 1 : 0;
        g_launches.fetch_add(3 + P->per_iter + bodies * (P->giters * P->per_iter + 1),
                             std::memory_order_relaxed);
        float sms = 0.0f;
        if (cudaEventElapsedTime(&sms, P->tev[0][0], P->tev[0][1]) == cudaSuccess) {
            spmv_ms += sms;
            ++spmv_samples;
        } else {
            (void)cudaGetLastError();   // timing is best effort
        }
    }
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
        stats[i].spmv_ms = spmv_samples ? spmv_ms / spmv_samples : 0.0;
        stats[i].spmv_samples = spmv_samples;
        stats[i].pad2_ = 0;
    }
    CFEM_CHECK(h_err != 2, CFEM_ERR_TIMEOUT,
               "solver SpMV bulk-copy wait timed out (device wait bound reached)");
    CFEM_CHECK(h_err == 0, CFEM_ERR_TIMEOUT,
               "solver grid barrier timed out (device wait bound reached)");
    return CFEM_OK;
}

}  // namespace cfem

extern "C" int cfem_pcg_plan_create(cfem_ctx *ctx, const cfem_linsys *systems,
                                    int32_t n_systems, void *stream,
                                    cfem_pcg_plan **out) {
    CFEM_API_BEGIN
    CFEM_CHECK(ctx && systems && out && n_systems > 0, CFEM_ERR_INVALID,
               "cfem_pcg_plan_create: bad args");
    *out = nullptr;
    CFEM_TRY(set_device(ctx->device));
    cfem_pcg_plan *P = new cfem_pcg_plan();
    const int st = plan_build(ctx, systems, n_systems, (cudaStream_t)stream, P);
    if (st != CFEM_OK) {
        plan_free(P);
        return st;
    }
    *out = P;
    return CFEM_OK;
    CFEM_API_END
}

extern "C" int cfem_pcg_plan_refresh(cfem_pcg_plan *plan, void *stream) {
    CFEM_API_BEGIN
    CFEM_CHECK(plan, CFEM_ERR_INVALID, "cfem_pcg_plan_refresh: plan is NULL");
    CFEM_TRY(set_device(plan->device));
    return plan_copies(plan, (cudaStream_t)stream);
    CFEM_API_END
}

extern "C" int cfem_pcg_plan_solve(cfem_pcg_plan *plan, cfem_solve_stats *stats,
                                   void *stream) {
    CFEM_API_BEGIN
    CFEM_CHECK(plan && stats, CFEM_ERR_INVALID, "cfem_pcg_plan_solve: bad args");
    CFEM_TRY(set_device(plan->device));
    return plan_run(plan, stats, (cudaStream_t)stream);
    CFEM_API_END
}

extern "C" int cfem_pcg_plan_destroy(cfem_pcg_plan *plan) {
    plan_free(plan);
    return CFEM_OK;
}

extern "C" int cfem_pcg_solve(cfem_ctx *ctx, const cfem_linsys *systems,
                              int32_t n_systems, cfem_solve_stats *stats,
                              void *stream) {
    CFEM_API_BEGIN
    CFEM_CHECK(ctx && systems && stats && n_systems > 0, CFEM_ERR_INVALID,
               "cfem_pcg_solve: bad args");
    CFEM_TRY(set_device(ctx->device));
    cfem_pcg_plan *P = new cfem_pcg_plan();
    int st = plan_build(ctx, systems, n_systems, (cudaStream_t)stream, P);
    if (st == CFEM_OK) st = plan_run(P, stats, (cudaStream_t)stream);
    plan_free(P);
    return st;
    CFEM_API_END
}

// ---------------------------------------------------------------------------
// Solve slots: continuous batching at iteration level. A slot plan is a
// plan of n_slots systems of fixed capacity (rows, nonzero blocks), built
// from placeholder systems of that size on the host-polled graph scheduler,
// so its work lists, workspace and captured iteration graphs never change.
// A system is put into a free slot between rounds (its SysDev entry
// replaced, its working copy built, its state reset and INIT run for its
// own chunks), every round replays the captured iterations over all slots
// (kernels skip idle slots and the list entries past a smaller system), and
// a finished system's slot is free for the next one at once: new systems
// join a running batch without waiting for the others to converge. Each
// system keeps its own scalars and fixed-order sums, so its answer does not
// depend on which other systems share the rounds.
namespace cfem {

__global__ void k_slots_idle(SysState *st, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) st[i].phase = PH_DONE;
}

__global__ void k_slot_open(GridBar *bar) {
    if (threadIdx.x == 0) atomicAdd(&bar->active, 1);
}

__global__ void k_slot_cancel(SysState *st, GridBar *bar) {
    if (threadIdx.x == 0 && st->phase != PH_DONE) {
        st->phase = PH_DONE;
        atomicSub(&bar->active, 1);
    }
}

// INIT (FP64 true residual, Jacobi inverse) over chunks [c0, c0 + n).
__global__ void __launch_bounds__(256)
k_pcg_init_range(const SysDev *__restrict__ sys, SysState *st,
                 const int32_t *__restrict__ chunk_sys, int c0, int n, GridBar *bar) {
    const int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (c >= n) return;
    dispatch<RUN_INIT>(sys, st, bar, chunk_sys, c0 + c, threadIdx.x & 31);
}

// Placeholder CSR of a slot template: rows of nnzb / rows entries, column 0.
__global__ void k_tmpl_rows(int64_t n, int64_t nnzb, int32_t *rp) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i <= n) rp[i] = (int32_t)((i * nnzb) / n);
}

}  // namespace cfem

extern "C" int cfem_pcg_slots_create(cfem_ctx *ctx, int32_t n_slots, int32_t bs,
                                     int32_t mode, int64_t max_rows, int64_t max_nnzb,
                                     void *stream, cfem_pcg_plan **out) {
    CFEM_API_BEGIN
    CFEM_CHECK(ctx && out && n_slots > 0 && (bs == 1 || bs == 3) &&
                   (mode == CFEM_SOLVE_FP64 || mode == CFEM_SOLVE_MIXED) && max_rows > 0 &&
                   max_nnzb > 0 && max_rows < ((int64_t)1 << 31) / 9 &&
                   max_nnzb < ((int64_t)1 << 31) / 9,
               CFEM_ERR_INVALID, "cfem_pcg_slots_create: bad arguments");
    *out = nullptr;
    CFEM_TRY(set_device(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;
    const size_t bb = (size_t)bs * bs;
    const size_t o_rp = 0, o_ci = align256((max_rows + 1) * 4);
    const size_t o_v64 = o_ci + align256(max_nnzb * 4);
    const size_t o_v32 = o_v64 + align256(max_nnzb * bb * 8);
    const size_t o_b = o_v32 + align256(max_nnzb * bb * 4);
    const size_t o_x = o_b + align256(max_rows * bs * 8);
    const size_t total = o_x + align256(max_rows * bs * 8);
    cfem_pcg_plan *P = new cfem_pcg_plan();
    P->slots = true;
    if (tmp_alloc(&P->tmpl_mem, total, s) != CFEM_OK ||
        cudaMemsetAsync(P->tmpl_mem, 0, total, s) != cudaSuccess) {
        const int st = fail(CFEM_ERR_NOMEM, "slot templates: %zu bytes", total);
        if (P->tmpl_mem) cudaFreeAsync(P->tmpl_mem, s);
        P->tmpl_mem = nullptr;
        delete P;
        return st;
    }
    int32_t *rp = (int32_t *)(P->tmpl_mem + o_rp);
    k_tmpl_rows<<<grid_for(max_rows + 1, 256), 256, 0, s>>>(max_rows, max_nnzb, rp);
    std::vector<cfem_linsys> L(n_slots);
    for (int i = 0; i < n_slots; ++i) {
        cfem_linsys &t = L[i];
        memset(&t, 0, sizeof(t));
        t.n_rows = max_rows;
        t.bs = bs;
        t.precond = CFEM_PRECOND_JACOBI;
        t.d_row_ptr = rp;
        t.d_col = (const int32_t *)(P->tmpl_mem + o_ci);
        t.d_vals64 = (const double *)(P->tmpl_mem + o_v64);
        t.d_vals32 = mode == CFEM_SOLVE_MIXED ? (const float *)(P->tmpl_mem + o_v32) : nullptr;
        t.d_b = (const double *)(P->tmpl_mem + o_b);
        t.d_x = (double *)(P->tmpl_mem + o_x);
        t.rtol = 1.0;
        t.max_iter = 1;
        t.mode = mode;
    }
    int st = plan_build(ctx, L.data(), n_slots, s, P);
    if (st == CFEM_OK && cudaMallocHost(&P->h_total, sizeof(int64_t)) != cudaSuccess) {
        P->h_total = nullptr;
        st = fail(CFEM_ERR_NOMEM, "slot plan: pinned host word");
    }
    if (st == CFEM_OK) {
        P->sev.assign(n_slots, nullptr);
        for (int i = 0; i < n_slots && st == CFEM_OK; ++i)
            if (cudaEventCreateWithFlags(&P->sev[i], cudaEventDisableTiming) != cudaSuccess)
                st = fail(CFEM_ERR_CUDA, "slot plan: events");
    }
    if (st == CFEM_OK) {
        P->tmpl = P->hs;
        P->cap_rows.assign(n_slots, max_rows);
        P->cap_nnzb.assign(n_slots, max_nnzb);
        // every slot idle, no system active
        if (cudaMemsetAsync(P->ws_state, 0, P->state_bytes, P->w) != cudaSuccess)
            st = fail(CFEM_ERR_CUDA, "slot state reset failed");
        else
            k_slots_idle<<<grid_for(n_slots, 128), 128, 0, P->w>>>(P->d_st, n_slots);
        if (st == CFEM_OK && cudaStreamSynchronize(P->w) != cudaSuccess)
            st = fail(CFEM_ERR_CUDA, "slot set-up failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    if (st != CFEM_OK) {
        plan_free(P);
        return st;
    }
    *out = P;
    return CFEM_OK;
    CFEM_API_END
}

extern "C" int cfem_pcg_slots_assign(cfem_pcg_plan *P, int32_t slot, const cfem_linsys *L,
                                     void *stream) {
    CFEM_API_BEGIN
    CFEM_CHECK(P && P->slots && L, CFEM_ERR_INVALID, "cfem_pcg_slots_assign: not a slot plan");
    CFEM_CHECK(slot >= 0 && slot < P->n_systems, CFEM_ERR_INVALID, "slot %d out of range", slot);
    CFEM_TRY(set_device(P->device));
    const SysDev &T = P->tmpl[slot];
    CFEM_CHECK(L->bs == T.bs && L->mode == T.mode, CFEM_ERR_INVALID,
               "slot %d holds bs %d mode %d systems", slot, T.bs, T.mode);
    CFEM_CHECK(L->bs == 1 || L->precond == CFEM_PRECOND_JACOBI, CFEM_ERR_INVALID,
               "solve slots use point Jacobi");
    CFEM_CHECK(L->n_rows > 0 && L->n_rows <= P->cap_rows[slot] && L->d_row_ptr && L->d_col &&
                   L->d_vals64 && L->d_b && L->d_x &&
                   (L->mode == CFEM_SOLVE_FP64 || L->d_vals32),
               CFEM_ERR_INVALID, "system does not fit slot %d (%lld rows, capacity %lld)",
               slot, (long long)L->n_rows, (long long)P->cap_rows[slot]);
    CFEM_CHECK(L->rtol > 0.0 && L->max_iter > 0, CFEM_ERR_INVALID,
               "rtol and max_iter must be positive");
    cudaStream_t s = (cudaStream_t)stream;
    // 3x3 slots in the sliced ELL: rank the new system's windows and scan
    // its slice sizes on the caller's stream (after its assembly), into the
    // row-order set the slot's previous system did not use
    const bool sell3 = T.bs == 3 && T.sell;
    int set = 0;
    if (sell3) {
        set = 1 - P->mset[slot];
        const cfem_pcg_plan::SellMeta &M = P->smeta[2 * slot + set];
        const int rs = sell_slice_rows(3, P->lanes3);
        const int64_t nw = sell_windows(L->n_rows), nsl = nw * (SELL_ROWS / rs);
        size_t need = 0;
        CFEM_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, need, (const int64_t *)nullptr,
                                                (int64_t *)nullptr, nsl + 1, s));
        CFEM_CHECK(need <= P->scan_bytes && P->h_total, CFEM_ERR_NOMEM,
                   "slot %d: slice-size scan scratch too small", slot);
        // rounds queued before the slot's last assignment may still read
        // this set (a slot freed by cfem_pcg_slots_poll has synchronised
        // them already; the wait then costs nothing)
        CFEM_CUDA(cudaStreamWaitEvent(s, P->sev[slot], 0));
        CFEM_CUDA(cudaMemsetAsync(M.sizes + nsl, 0, sizeof(int64_t), s));
        const int srt = P->ctx->sell_sort;
        if (rs == 32)
            CFEM_LAUNCH(k_sell_rank<32>, (unsigned)nw, SELL_ROWS, 0, s, L->n_rows, L->d_row_ptr,
                        L->d_col, M.perm, M.sizes, srt);
        else if (rs == 16)
            CFEM_LAUNCH(k_sell_rank<16>, (unsigned)nw, SELL_ROWS, 0, s, L->n_rows, L->d_row_ptr,
                        L->d_col, M.perm, M.sizes, srt);
        else
            CFEM_LAUNCH(k_sell_rank<8>, (unsigned)nw, SELL_ROWS, 0, s, L->n_rows, L->d_row_ptr,
                        L->d_col, M.perm, M.sizes, srt);
        CFEM_CUDA(cub::DeviceScan::ExclusiveSum(P->scan_tmp, need, M.sizes, M.soff, nsl + 1, s));
        CFEM_CUDA(cudaMemcpyAsync(P->h_total, M.soff + nsl, sizeof(int64_t),
                                  cudaMemcpyDeviceToHost, s));
    }
    int32_t nnzb = 0;
    CFEM_CUDA(cudaMemcpyAsync(&nnzb, L->d_row_ptr + L->n_rows, sizeof(int32_t),
                              cudaMemcpyDeviceToHost, s));
    CFEM_CUDA(cudaStreamSynchronize(s));
    CFEM_CHECK(nnzb >= 0 && nnzb <= P->cap_nnzb[slot], CFEM_ERR_INVALID,
               "system has %d blocks, slot %d holds %lld", nnzb, slot,
               (long long)P->cap_nnzb[slot]);
    CFEM_CHECK(!sell3 || *P->h_total <= P->cap_sell[slot], CFEM_ERR_INVALID,
               "system's sliced-ELL layout has %lld blocks, slot %d holds %lld",
               (long long)*P->h_total, slot, (long long)P->cap_sell[slot]);
    SysDev S = T;   // the slot's workspace, lists and copies
    if (sell3) {
        S.sperm = P->smeta[2 * slot + set].perm;
        S.soff = P->smeta[2 * slot + set].soff;
    }
    S.n = L->n_rows;
    S.nnzb = nnzb;
    if (S.vec4) S.lpr = S.nnzb <= 16 * S.n ? 4 : 8;
    S.nchunks = (int32_t)((S.n + S.crows - 1) / S.crows);
    S.ntiles = (S.nchunks + TILE - 1) / TILE;
    S.nchunksB = (int32_t)((S.n + brows(S.bs) - 1) / brows(S.bs));
    S.nxe = (int32_t)((S.n + S.xrows - 1) / S.xrows);
    S.max_iter = L->max_iter;
    S.rp = L->d_row_ptr;
    S.ci = L->d_col;
    S.v64 = L->d_vals64;
    S.v32 = L->d_vals32;
    S.b = L->d_b;
    S.x = L->d_x;
    S.fixed = L->d_fixed;
    S.rtol2 = L->rtol * L->rtol;
    const double dl = L->reliable_delta > 0.0 ? L->reliable_delta : RELIABLE_DELTA;
    S.delta2 = dl * dl;
    S.max_stall = L->max_stall > 0 ? L->max_stall : MAX_STALL;
    S.hist_cap = L->d_history ? L->history_cap : 0;
    S.hist = L->d_history;
    if (S.bs == 1) S.vsoa = (S.mode == CFEM_SOLVE_MIXED) ? (const void *)S.v32 : (const void *)S.v64;
    P->hs[slot] = S;
    cudaStream_t w = P->w;
    CFEM_CUDA(cudaEventRecord(P->ev[0], s));
    CFEM_CUDA(cudaStreamWaitEvent(w, P->ev[0], 0));
    CFEM_CUDA(cudaMemcpyAsync(P->d_sys + slot, &P->hs[slot], sizeof(SysDev),
                              cudaMemcpyHostToDevice, w));
    if (sell3) CFEM_CUDA(cudaEventRecord(P->sev[slot], w));
    CFEM_TRY(plan_copies(P, w, slot, slot + 1));
    if (sell3) P->mset[slot] = set;
    CFEM_CUDA(cudaMemsetAsync(P->d_st + slot, 0, sizeof(SysState), w));
    CFEM_CUDA(cudaMemsetAsync(S.tcnt, 0, (size_t)T.ntiles * sizeof(unsigned), w));
    CFEM_LAUNCH(k_slot_open, 1, 32, 0, w, P->d_bar);
    CFEM_LAUNCH(k_pcg_init_range, grid_for((int64_t)S.nchunks * 32, 256), 256, 0, w,
                (const SysDev *)P->d_sys, P->d_st, (const int32_t *)P->d_chunks, S.chunk0,
                S.nchunks, P->d_bar);
    // the pageable copy of hs[slot] is staged before cudaMemcpyAsync returns
    return CFEM_OK;
    CFEM_API_END
}

extern "C" int cfem_pcg_slots_run(cfem_pcg_plan *P, int32_t rounds, void *stream) {
    CFEM_API_BEGIN
    CFEM_CHECK(P && P->slots && rounds > 0, CFEM_ERR_INVALID, "cfem_pcg_slots_run: bad args");
    CFEM_TRY(set_device(P->device));
    cudaStream_t s = (cudaStream_t)stream, w = P->w;
    CFEM_CUDA(cudaEventRecord(P->ev[0], s));
    CFEM_CUDA(cudaStreamWaitEvent(w, P->ev[0], 0));
    for (int r = 0; r < rounds; ++r) {
        CFEM_CUDA(cudaGraphLaunch(P->pexec[r & 1], w));
        g_launches.fetch_add((int64_t)P->per_iter * POLL_ITERS, std::memory_order_relaxed);
    }
    // no wait on the caller's stream: new systems are assembled there while
    // the rounds run; poll orders the host after them
    CFEM_CUDA(cudaEventRecord(P->ev[1], w));
    return CFEM_OK;
    CFEM_API_END
}

extern "C" int cfem_pcg_slots_ready(cfem_pcg_plan *P) {
    CFEM_CHECK(P && P->slots, CFEM_ERR_INVALID, "cfem_pcg_slots_ready: not a slot plan");
    CFEM_TRY(set_device(P->device));
    const cudaError_t e = cudaEventQuery(P->ev[1]);
    if (e == cudaErrorNotReady) return CFEM_SLOT_RUNNING;
    CFEM_CUDA(e);
    return CFEM_OK;
}

extern "C" int cfem_pcg_slots_poll(cfem_pcg_plan *P, cfem_solve_stats *stats) {
    CFEM_API_BEGIN
    CFEM_CHECK(P && P->slots && stats, CFEM_ERR_INVALID, "cfem_pcg_slots_poll: bad args");
    CFEM_TRY(set_device(P->device));
    const int n = P->n_systems;
    CFEM_CUDA(cudaMemcpyAsync(P->h_st, P->d_st, n * sizeof(SysState),
                              cudaMemcpyDeviceToHost, P->w));
    CFEM_CUDA(cudaMemcpyAsync(&P->h_flags[3], &P->d_bar->err, sizeof(int),
                              cudaMemcpyDeviceToHost, P->w));
    CFEM_CUDA(cudaStreamSynchronize(P->w));
    const SysState *hst = P->h_st;
    const int h_err = P->h_flags[3];
    for (int i = 0; i < n; ++i) {
        cfem_solve_stats &o = stats[i];
        memset(&o, 0, sizeof(o));
        o.status = hst[i].phase == PH_DONE ? hst[i].status : CFEM_SLOT_RUNNING;
        o.iterations = hst[i].iter;
        o.residual_updates = hst[i].nres;
        o.relres = hst[i].relres;
        o.bnorm = sqrt(hst[i].bb);
    }
    CFEM_CHECK(h_err != 2, CFEM_ERR_TIMEOUT,
               "solver SpMV bulk-copy wait timed out (device wait bound reached)");
    return CFEM_OK;
    CFEM_API_END
}

extern "C" int cfem_pcg_slots_release(cfem_pcg_plan *P, int32_t slot, void *stream) {
    CFEM_API_BEGIN
    CFEM_CHECK(P && P->slots && slot >= 0 && slot < P->n_systems, CFEM_ERR_INVALID,
               "cfem_pcg_slots_release: bad args");
    CFEM_TRY(set_device(P->device));
    cudaStream_t s = (cudaStream_t)stream, w = P->w;
    CFEM_CUDA(cudaEventRecord(P->ev[0], s));
    CFEM_CUDA(cudaStreamWaitEvent(w, P->ev[0], 0));
    CFEM_LAUNCH(k_slot_cancel, 1, 32, 0, w, P->d_st + slot, P->d_bar);
    CFEM_CUDA(cudaEventRecord(P->ev[1], w));
    CFEM_CUDA(cudaStreamWaitEvent(s, P->ev[1], 0));
    return CFEM_OK;
    CFEM_API_END
}

// ---------------------------------------------------------------------------
// Allocation-free variant of cfem_pcg_solve for one system.
//
// Some callers cannot allocate device memory at solve time: an application
// that reserves the whole HBM budget for its own pools up front (so any
// library allocation mid-run can fail or fragment that budget), and
// latency-bound control loops that cannot afford the implicit
// synchronisation and unbounded latency of cudaMalloc. For them the solver
// workspace lives in one file-scope device array of fixed size, loaded with
// the library and held by every GPU that loads it until the process exits.
// The same kernels as cfem_pcg_solve run on it; nothing is allocated.
namespace cfem {

constexpr size_t NOALLOC_SCRATCH_BYTES = (size_t)32 << 20;   // 32 MiB

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// Device address of g_noalloc_scratch per CUDA context. In host code the
// array's name is only a host-side stand-in, so the address is looked up with
// the device (and its context) current the first time a context calls, and
// passed to the kernels. Keyed on the current driver context, so a caller
// that makes its own (non-primary) context current gets that context's copy
// of the array.
struct NoallocAddr {
    CUcontext cu;
    void *addr;
};
static std::vector<NoallocAddr> g_noalloc_addr;
static std::mutex g_noalloc_mu;
typedef CUresult (*CtxGetCurrentFn)(CUcontext *);

static int noalloc_scratch(void **out) {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    static CtxGetCurrentFn get_current = nullptr;
    if (!get_current) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        CFEM_CUDA(cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q));
        CFEM_CHECK(fn && q == cudaDriverEntryPointSuccess, CFEM_ERR_CUDA,
                   "driver entry point cuCtxGetCurrent not found");
        get_current = (CtxGetCurrentFn)fn;
    }
    CUcontext cu = nullptr;
    CFEM_CHECK(get_current(&cu) == CUDA_SUCCESS && cu, CFEM_ERR_CUDA,
               "no current CUDA context");
    for (const NoallocAddr &e : g_noalloc_addr)
        if (e.cu == cu) {
            *out = e.addr;
            return CFEM_OK;
        }
    void *p = nullptr;
    CFEM_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    CFEM_CHECK(p != nullptr, CFEM_ERR_CUDA, "scratch symbol has no address");
    g_noalloc_addr.push_back({cu, p});
    *out = p;
    return CFEM_OK;
}

}  // namespace cfem

extern "C" size_t cfem_pcg_noalloc_capacity(void) { return NOALLOC_SCRATCH_BYTES; }

extern "C" int cfem_pcg_solve_noalloc(cfem_ctx *ctx, const cfem_linsys *L,
                                      cfem_solve_stats *stats, void *stream) {
    CFEM_API_BEGIN
    CFEM_CHECK(ctx && L && stats, CFEM_ERR_INVALID,
               "cfem_pcg_solve_noalloc: NULL argument");
    CFEM_CHECK(L->bs == 1 || L->bs == 3, CFEM_ERR_INVALID,
               "block size %d (1 or 3)", L->bs);
    CFEM_CHECK(L->n_rows > 0 && L->d_row_ptr && L->d_col && L->d_vals64 &&
                   L->d_b && L->d_x,
               CFEM_ERR_INVALID, "missing arrays");
    CFEM_CHECK(L->mode == CFEM_SOLVE_FP64 ||
                   (L->mode == CFEM_SOLVE_MIXED && L->d_vals32),
               CFEM_ERR_INVALID, "mixed mode needs FP32 values");
    CFEM_CHECK(L->rtol > 0.0 && L->max_iter > 0, CFEM_ERR_INVALID,
               "rtol and max_iter must be positive");
    CFEM_CHECK(L->n_rows < ((int64_t)1 << 31) / 9, CFEM_ERR_INVALID,
               "system too large");
    CFEM_TRY(set_device(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;

    SysDev S;
    memset(&S, 0, sizeof(S));
    S.n = L->n_rows;
    S.bs = L->bs;
    S.precond = (L->bs == 3) ? L->precond : CFEM_PRECOND_JACOBI;
    S.mode = L->mode;
    S.crows = chunk_rows(L->bs);
    S.nchunks = (int32_t)((L->n_rows + S.crows - 1) / S.crows);
    S.ntiles = (S.nchunks + TILE - 1) / TILE;
    S.chunk0 = 0;
    S.max_iter = L->max_iter;
    S.rp = L->d_row_ptr;
    S.ci = L->d_col;
    S.v64 = L->d_vals64;
    S.v32 = L->d_vals32;
    S.b = L->d_b;
    S.x = L->d_x;
    S.fixed = L->d_fixed;
    S.rtol2 = L->rtol * L->rtol;
    const double dl = L->reliable_delta > 0.0 ? L->reliable_delta : RELIABLE_DELTA;
    S.delta2 = dl * dl;
    S.max_stall = L->max_stall > 0 ? L->max_stall : MAX_STALL;
    S.hist_cap = L->d_history ? L->history_cap : 0;
    S.hist = L->d_history;

    auto align = [](size_t v) { return (v + 255) & ~(size_t)255; };
    const size_t ts = (S.mode == CFEM_SOLVE_MIXED) ? 4 : 8;
    const size_t nd = (size_t)S.n * S.bs;
    const size_t nprec = (S.precond == CFEM_PRECOND_BLOCK) ? (size_t)S.n * 9 : nd;
    const size_t need = 5 * align(nd * ts) + align(nprec * ts) +
                        align(S.nchunks * 4 * sizeof(double)) +
                        align(S.ntiles * 4 * sizeof(double)) +
                        align(S.ntiles * sizeof(unsigned)) + align(sizeof(SysDev)) +
                        align(sizeof(SysState)) + align(S.nchunks * sizeof(int32_t)) +
                        align(sizeof(GridBar));
    CFEM_CHECK(need <= NOALLOC_SCRATCH_BYTES, CFEM_ERR_INVALID,
               "system needs %zu bytes of solver scratch; the allocation-free "
               "entry point has a fixed %zu (use cfem_pcg_solve)",
               need, NOALLOC_SCRATCH_BYTES);

    void *base = nullptr;
    CFEM_TRY(noalloc_scratch(&base));
    char *ws = (char *)base;
    // Every call reuses the array: clear all of it that this call uses
    // (state, tickets, chunk table, p buffers) before the launch.
    CFEM_CUDA(cudaMemsetAsync(ws, 0, need, s));
    size_t off = 0;
    auto take = [&](size_t b) { char *p = ws + off; off += align(b); return (void *)p; };
    S.r = take(nd * ts);
    S.z = take(nd * ts);
    S.p0 = take(nd * ts);
    S.p1 = take(nd * ts);
    S.q = take(nd * ts);
    S.dinv = take(nprec * ts);
    S.partial = (double *)take(S.nchunks * 4 * sizeof(double));
    S.tpartial = (double *)take(S.ntiles * 4 * sizeof(double));
    S.tcnt = (unsigned *)take(S.ntiles * sizeof(unsigned));
    SysDev *d_sys = (SysDev *)take(sizeof(SysDev));
    SysState *d_st = (SysState *)take(sizeof(SysState));
    int32_t *d_chunks = (int32_t *)take(S.nchunks * sizeof(int32_t));  // all 0
    GridBar *d_bar = (GridBar *)take(sizeof(GridBar));
    const int h_active = 1;
    CFEM_CUDA(cudaMemcpyAsync(d_sys, &S, sizeof(SysDev), cudaMemcpyHostToDevice, s));
    CFEM_CUDA(cudaMemcpyAsync(&d_bar->active, &h_active, sizeof(int),
                              cudaMemcpyHostToDevice, s));

    int per_sm = 0;
    CFEM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, k_pcg_persistent, SOLVE_THREADS, 0));
    CFEM_CHECK(per_sm > 0, CFEM_ERR_CUDA, "solver kernel cannot be resident");
    int n_chunks = S.nchunks;
    int grid = ctx->num_sms * per_sm;
    const int useful = (n_chunks * 32 + SOLVE_THREADS - 1) / SOLVE_THREADS;
    if (grid > useful) grid = useful < 1 ? 1 : useful;
    if (grid > BAR_GROUP * BAR_MAX_GROUPS) grid = BAR_GROUP * BAR_MAX_GROUPS;
    int max_steps = 3 * L->max_iter + 16;
    CFEM_LAUNCH(k_pcg_init, grid_for((int64_t)n_chunks * 32, 256), 256, 0, s,
                d_sys, d_st, d_chunks, n_chunks, d_bar);
    unsigned long long bar_timeout_ns = 1000ull * (unsigned long long)ctx->barrier_timeout_us;
    unsigned bar_hold = (unsigned)ctx->barrier_hold;
    void *args[] = {(void *)&d_sys, (void *)&d_st, (void *)&d_chunks,
                    (void *)&n_chunks, (void *)&d_bar, (void *)&max_steps,
                    (void *)&bar_timeout_ns, (void *)&bar_hold};
    CFEM_CUDA(cudaLaunchCooperativeKernel((void *)k_pcg_persistent, dim3(grid),
                                          dim3(SOLVE_THREADS), args, 0, s));
    g_launches.fetch_add(1, std::memory_order_relaxed);
    SysState hst;
    int h_err = 0;
    CFEM_CUDA(cudaMemcpyAsync(&hst, d_st, sizeof(SysState), cudaMemcpyDeviceToHost, s));
    CFEM_CUDA(cudaMemcpyAsync(&h_err, &d_bar->err, sizeof(int),
                              cudaMemcpyDeviceToHost, s));
    CFEM_CUDA(cudaStreamSynchronize(s));
    stats->status = hst.status;
    if (hst.status == CFEM_OK && hst.phase != PH_DONE)
        stats->status = CFEM_ERR_NOT_CONVERGED;
    stats->iterations = hst.iter;
    stats->residual_updates = hst.nres;
    stats->pad_ = 0;
    stats->relres = hst.relres;
    stats->bnorm = sqrt(hst.bb);
    stats->kernel_ms = 0.0;
    stats->spmv_ms = 0.0;
    stats->spmv_samples = 0;
    stats->pad2_ = 0;
    CFEM_CHECK(h_err == 0, CFEM_ERR_TIMEOUT,
               "solver grid barrier timed out (device wait bound reached)");
    return CFEM_OK;
    CFEM_API_END
}
