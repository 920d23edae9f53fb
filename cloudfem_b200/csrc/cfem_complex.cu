// Complex symmetric solver: Jacobi-preconditioned COCG (conjugate orthogonal
// CG: CG with the unconjugated bilinear form x^T y), for the phasor A-V
// eddy-current system of em3d_tet10.py:267-375 once its V rows are scaled
// by 1/(i omega), which makes the system complex symmetric (A^T = A).
//
// Complex values are interleaved (re, im) doubles. Every iteration is five
// launches (SpMV + p.q, alpha, update + r.z and |r|^2, beta and the
// convergence test, direction); block partial sums are reduced in block
// order by one block, so results are deterministic. A finished or broken
// down system turns every later launch into a no-op; the host checks the
// state once per batch of iterations.
#include "cfem_common.cuh"

#include <math.h>
#include <string.h>

#include <algorithm>

namespace cfem {
namespace {

constexpr int CT = 256;                 // threads per block
constexpr int CW = CT / 32;             // warps (rows) per block
constexpr int C_BATCH = 8;              // iterations between host checks

struct CState {
    double2 rho, alpha, beta;
    double rr, bb;
    int iter, status, done, pad;
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) {
    return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ double2 csub(double2 a, double2 b) {
    return make_double2(a.x - b.x, a.y - b.y);
}
__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
    const double d = b.x * b.x + b.y * b.y;
    return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}

// Fixed-order block sum of up to 4 doubles per thread into part[blockIdx].
__device__ __forceinline__ void block_sum4(double v[4], double *part) {
    __shared__ double red[4][CW];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = warp_sum(v[k]);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < 4; ++k) red[k][w] = v[k];
    __syncthreads();
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            double t = 0.0;
            for (int i = 0; i < CW; ++i) t += red[k][i];
            part[(int64_t)blockIdx.x * 4 + k] = t;
        }
}

// One block: sum the partials of nb blocks in block order.
__device__ __forceinline__ void sum_partials(const double *part, int nb, double out[4]) {
    __shared__ double red[4][CT / 32];
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < nb; b += CT)
#pragma unroll
        for (int k = 0; k < 4; ++k) acc[k] += part[(int64_t)b * 4 + k];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 4; ++k) acc[k] = warp_sum(acc[k]);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < 4; ++k) red[k][w] = acc[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        double t = 0.0;
        for (int i = 0; i < CT / 32; ++i) t += red[k][i];
        out[k] = t;
    }
}

// Row dot of A with v (warp per row), complex.
__device__ __forceinline__ double2 row_dot(const int32_t *__restrict__ ip,
                                          const int32_t *__restrict__ ix,
                                          const double2 *__restrict__ a,
                                          const double2 *v, int64_t row, int lane,
                                          double2 *diag) {
    double2 acc = make_double2(0.0, 0.0), dg = make_double2(0.0, 0.0);
    for (int32_t k = __ldg(ip + row) + lane; k < __ldg(ip + row + 1); k += 32) {
        const int32_t j = __ldg(ix + k);
        const double2 av = __ldg(a + k);
        acc = cadd(acc, cmul(av, v[j]));
        if (j == row) dg = av;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
        acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
        dg.x += __shfl_xor_sync(0xffffffffu, dg.x, o);
        dg.y += __shfl_xor_sync(0xffffffffu, dg.y, o);
    }
    if (diag) *diag = dg;
    return acc;
}

// r = b - A x, dinv = 1 / diag(A), z = dinv r, p = z; partial r.z, |r|^2, |b|^2.
__global__ void __launch_bounds__(CT)
k_c_init(int64_t n, const int32_t *__restrict__ ip, const int32_t *__restrict__ ix,
         const double2 *__restrict__ a, const double2 *__restrict__ b,
         const double2 *__restrict__ x, double2 *r, double2 *z, double2 *p,
         double2 *dinv, double *part, CState *st) {
    const int lane = threadIdx.x & 31;
    const int64_t row = (int64_t)blockIdx.x * CW + (threadIdx.x >> 5);
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    if (row < n) {
        double2 dg;
        const double2 ax = row_dot(ip, ix, a, x, row, lane, &dg);
        if (lane == 0) {
            const double2 bi = b[row];
            const double2 ri = csub(bi, ax);
            double2 di = make_double2(0.0, 0.0);
            if (dg.x != 0.0 || dg.y != 0.0) di = cdiv(make_double2(1.0, 0.0), dg);
            else atomicExch(&st->status, (int)CFEM_ERR_BREAKDOWN);
            const double2 zi = cmul(di, ri);
            r[row] = ri;
            z[row] = zi;
            p[row] = zi;
            dinv[row] = di;
            const double2 rz = cmul(ri, zi);
            v[0] = rz.x;
            v[1] = rz.y;
            v[2] = ri.x * ri.x + ri.y * ri.y;
            v[3] = bi.x * bi.x + bi.y * bi.y;
        }
    }
    block_sum4(v, part);
}

__global__ void __launch_bounds__(CT)
k_c_init_red(const double *part, int nb, CState *st, double rtol2) {
    double t[4];
    sum_partials(part, nb, t);
    if (threadIdx.x == 0) {
        st->rho = make_double2(t[0], t[1]);
        st->rr = t[2];
        st->bb = t[3];
        st->iter = 0;
        if (st->status != CFEM_OK || !isfinite(t[2])) {
            st->done = 1;
            if (st->status == CFEM_OK) st->status = CFEM_ERR_BREAKDOWN;
        } else if (t[2] <= rtol2 * t[3]) {
            st->done = 1;
        }
    }
}

// q = A p; partial p.q.
__global__ void __launch_bounds__(CT)
k_c_spmv(int64_t n, const int32_t *__restrict__ ip, const int32_t *__restrict__ ix,
         const double2 *__restrict__ a, const double2 *p, double2 *q, double *part,
         const CState *st) {
    if (*(volatile const int *)&st->done) return;
    const int lane = threadIdx.x & 31;
    const int64_t row = (int64_t)blockIdx.x * CW + (threadIdx.x >> 5);
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    if (row < n) {
        const double2 qi = row_dot(ip, ix, a, p, row, lane, nullptr);
        if (lane == 0) {
            q[row] = qi;
            const double2 pq = cmul(p[row], qi);
            v[0] = pq.x;
            v[1] = pq.y;
        }
    }
    block_sum4(v, part);
}

__global__ void __launch_bounds__(CT)
k_c_alpha(const double *part, int nb, CState *st) {
    if (*(volatile const int *)&st->done) return;
    double t[4];
    sum_partials(part, nb, t);
    if (threadIdx.x == 0) {
        const double2 mu = make_double2(t[0], t[1]);
        const double m2 = mu.x * mu.x + mu.y * mu.y;
        const double r2 = st->rho.x * st->rho.x + st->rho.y * st->rho.y;
        if (!(m2 > 1e-300 * (r2 + 1e-300)) || !isfinite(m2)) {
            st->status = CFEM_ERR_BREAKDOWN;
            st->done = 1;
        } else {
            st->alpha = cdiv(st->rho, mu);
        }
    }
}

// x += alpha p, r -= alpha q, z = dinv r; partial r.z, |r|^2.
__global__ void __launch_bounds__(CT)
k_c_update(int64_t n, double2 *x, double2 *r, double2 *z, const double2 *p,
           const double2 *q, const double2 *dinv, double *part, const CState *st) {
    if (*(volatile const int *)&st->done) return;
    const double2 al = st->alpha;
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    for (int64_t i = (int64_t)blockIdx.x * CT + threadIdx.x; i < n; i += (int64_t)gridDim.x * CT) {
        x[i] = cadd(x[i], cmul(al, p[i]));
        const double2 ri = csub(r[i], cmul(al, q[i]));
        const double2 zi = cmul(dinv[i], ri);
        r[i] = ri;
        z[i] = zi;
        const double2 rz = cmul(ri, zi);
        v[0] += rz.x;
        v[1] += rz.y;
        v[2] += ri.x * ri.x + ri.y * ri.y;
    }
    block_sum4(v, part);
}

__global__ void __launch_bounds__(CT)
k_c_beta(const double *part, int nb, CState *st, double rtol2, int max_iter) {
    if (*(volatile const int *)&st->done) return;
    double t[4];
    sum_partials(part, nb, t);
    if (threadIdx.x == 0) {
        const double2 rho_new = make_double2(t[0], t[1]);
        st->rr = t[2];
        st->iter += 1;
        if (!isfinite(t[2]) || !isfinite(t[0]) || !isfinite(t[1])) {
            st->status = CFEM_ERR_BREAKDOWN;
            st->done = 1;
        } else if (t[2] <= rtol2 * st->bb) {
            st->done = 1;
        } else if (st->iter >= max_iter) {
            st->status = CFEM_ERR_NOT_CONVERGED;
            st->done = 1;
        } else {
            st->beta = cdiv(rho_new, st->rho);
            st->rho = rho_new;
        }
    }
}

// p = z + beta p.
__global__ void __launch_bounds__(CT)
k_c_dir(int64_t n, const double2 *z, double2 *p, const CState *st) {
    if (*(volatile const int *)&st->done) return;
    const double2 be = st->beta;
    for (int64_t i = (int64_t)blockIdx.x * CT + threadIdx.x; i < n; i += (int64_t)gridDim.x * CT)
        p[i] = cadd(z[i], cmul(be, p[i]));
}

}  // namespace
}  // namespace cfem

using namespace cfem;

extern "C" int cfem_cocg_solve(cfem_ctx *ctx, int64_t n, const int32_t *d_indptr,
                               const int32_t *d_indices, const double *d_vals,
                               const double *d_b, double *d_x, double rtol,
                               int32_t max_iter, cfem_solve_stats *stats,
                               void *stream) {
    CFEM_API_BEGIN
    CFEM_CHECK(ctx && d_indptr && d_indices && d_vals && d_b && d_x && stats && n > 0 &&
                   rtol > 0.0 && max_iter > 0,
               CFEM_ERR_INVALID, "cfem_cocg_solve: bad args");
    CFEM_CHECK(((uintptr_t)d_vals & 15) == 0 && ((uintptr_t)d_b & 15) == 0 &&
                   ((uintptr_t)d_x & 15) == 0,
               CFEM_ERR_INVALID, "complex arrays must be 16-byte aligned");
    CFEM_TRY(set_device(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned nb_rows = grid_for(n, CW);                 // warp per row
    unsigned nb_vec = grid_for(n, CT);
    if (nb_vec > (unsigned)ctx->num_sms * 8) nb_vec = ctx->num_sms * 8;
    const int nb_part = (int)std::max(nb_rows, nb_vec);
    double2 *ws = nullptr;
    CFEM_TRY(tmp_alloc(&ws, 5 * (size_t)n + 2 * (size_t)nb_part + 8, s));
    double2 *r = ws, *z = ws + n, *p = ws + 2 * n, *q = ws + 3 * n, *dinv = ws + 4 * n;
    double *part = (double *)(ws + 5 * n);
    CState *st = (CState *)(ws + 5 * n + 2 * (size_t)nb_part);
    CFEM_CUDA(cudaMemsetAsync(st, 0, sizeof(CState), s));
    const auto *a = (const double2 *)d_vals;
    const auto *b = (const double2 *)d_b;
    auto *x = (double2 *)d_x;
    const double rtol2 = rtol * rtol;
    cudaEvent_t e0, e1;
    CFEM_CUDA(cudaEventCreate(&e0));
    CFEM_CUDA(cudaEventCreate(&e1));
    CFEM_CUDA(cudaEventRecord(e0, s));
    CFEM_LAUNCH(k_c_init, nb_rows, CT, 0, s, n, d_indptr, d_indices, a, b, x, r, z, p,
                dinv, part, st);
    CFEM_LAUNCH(k_c_init_red, 1, CT, 0, s, part, (int)nb_rows, st, rtol2);
    CState h{};
    int status = CFEM_OK;
    for (int done_iters = 0; ; done_iters += C_BATCH) {
        for (int k = 0; k < C_BATCH; ++k) {
            CFEM_LAUNCH(k_c_spmv, nb_rows, CT, 0, s, n, d_indptr, d_indices, a, p, q, part, st);
            CFEM_LAUNCH(k_c_alpha, 1, CT, 0, s, part, (int)nb_rows, st);
            CFEM_LAUNCH(k_c_update, nb_vec, CT, 0, s, n, x, r, z, p, q, dinv, part, st);
            CFEM_LAUNCH(k_c_beta, 1, CT, 0, s, part, (int)nb_vec, st, rtol2, max_iter);
            CFEM_LAUNCH(k_c_dir, nb_vec, CT, 0, s, n, z, p, st);
        }
        CFEM_CUDA(cudaMemcpyAsync(&h, st, sizeof(CState), cudaMemcpyDeviceToHost, s));
        CFEM_CUDA(cudaStreamSynchronize(s));
        if (h.done || done_iters + C_BATCH >= max_iter + C_BATCH) break;
    }
    CFEM_CUDA(cudaEventRecord(e1, s));
    tmp_free(ws, s);
    CFEM_CUDA(cudaStreamSynchronize(s));
    float ms = 0.0f;
    CFEM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    status = h.status;
    if (status == CFEM_OK && !h.done) status = CFEM_ERR_NOT_CONVERGED;
    memset(stats, 0, sizeof(*stats));
    stats->status = status;
    stats->iterations = h.iter;
    stats->relres = h.bb > 0.0 ? sqrt(h.rr / h.bb) : 0.0;
    stats->bnorm = sqrt(h.bb);
    stats->kernel_ms = ms;
    return CFEM_OK;
    CFEM_API_END
}
