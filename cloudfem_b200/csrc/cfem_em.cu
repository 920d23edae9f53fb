// Eddy-current post-processing on the device: the Joule power of one step
// of the transient Tet10 A-V march (em3d_tet10.py:665-692), so the march
// keeps its fields on the GPU between steps.
//
// One thread per element. The element's geometry is affine (straight-edged
// Tet10), so the gradient of the Tet10 shape functions at node p is
// dN_j/dxi(p) J^-T with J from the corners; the caller passes the reference
// element's table dN_j/dxi at its 10 nodes and its normalised mass matrix,
// so the node order and the quadrature are the caller's (the reference's).
// The power is summed in a fixed order (per-block tree, then the blocks in
// order by one block): bitwise the same on every run.
#include "cfem_common.cuh"

namespace cfem {
namespace {

constexpr int JT = 128;   // threads per block

__global__ void __launch_bounds__(JT)
k_t10_joule(int64_t n_elems, const int32_t *__restrict__ elems, const double *__restrict__ nodes,
            const double *__restrict__ sigma, const double *__restrict__ a_prev,
            const double *__restrict__ a_new, const int64_t *__restrict__ vcol,
            const double *__restrict__ v, double h, const double *__restrict__ dn,
            const double *__restrict__ mref, double *__restrict__ q_out,
            double *__restrict__ part) {
    __shared__ double s_dn[300], s_m[100], red[JT / 32];
    for (int i = threadIdx.x; i < 300; i += JT) s_dn[i] = dn[i];
    for (int i = threadIdx.x; i < 100; i += JT) s_m[i] = mref[i];
    __syncthreads();
    const int64_t e = (int64_t)blockIdx.x * JT + threadIdx.x;
    double pw = 0.0;
    if (e < n_elems) {
        const double sg = sigma[e];
        double Q = 0.0;
        if (sg > 0.0) {
            int32_t nd[10];
#pragma unroll
            for (int p = 0; p < 10; ++p) nd[p] = elems[e * 10 + p];
            double x0[3], J[3][3];
#pragma unroll
            for (int d = 0; d < 3; ++d) x0[d] = nodes[(int64_t)nd[0] * 3 + d];
#pragma unroll
            for (int c = 0; c < 3; ++c)       // column c: corner c+1 - corner 0
#pragma unroll
                for (int d = 0; d < 3; ++d) J[d][c] = nodes[(int64_t)nd[c + 1] * 3 + d] - x0[d];
            const double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                               J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                               J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
            // inverse of J (rows k: d xi_k / d x)
            double Ji[3][3];
            Ji[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det;
            Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
            Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
            Ji[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / det;
            Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
            Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
            Ji[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
            Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
            Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
            double vv[10];
#pragma unroll
            for (int j = 0; j < 10; ++j) {
                const int64_t c = vcol[nd[j]];
                vv[j] = c >= 0 ? v[c] : 0.0;
            }
            double E[10][3];
#pragma unroll
            for (int p = 0; p < 10; ++p) {
                double gx[3] = {0.0, 0.0, 0.0};   // sum_j v_j dN_j/dxi at node p
#pragma unroll
                for (int j = 0; j < 10; ++j)
#pragma unroll
                    for (int k = 0; k < 3; ++k) gx[k] += s_dn[(p * 10 + j) * 3 + k] * vv[j];
                const int64_t np = nd[p];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const double g = gx[0] * Ji[0][d] + gx[1] * Ji[1][d] + gx[2] * Ji[2][d];
                    E[p][d] = -(a_new[np * 3 + d] - a_prev[np * 3 + d]) / h - g;
                }
            }
#pragma unroll
            for (int p = 0; p < 10; ++p) {
                double row = 0.0;
#pragma unroll
                for (int qq = 0; qq < 10; ++qq)
                    row += s_m[p * 10 + qq] *
                           (E[p][0] * E[qq][0] + E[p][1] * E[qq][1] + E[p][2] * E[qq][2]);
                Q += row;
            }
            Q *= sg;
            pw = Q * fabs(det) / 6.0;
        }
        if (q_out) q_out[e] = Q;
    }
    pw = warp_sum(pw);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = pw;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
#pragma unroll
        for (int w = 0; w < JT / 32; ++w) t += red[w];
        part[blockIdx.x] = t;
    }
}

// One block: the block partials in a fixed order into *out.
__global__ void __launch_bounds__(256)
k_sum_parts(int64_t n, const double *__restrict__ part, double *__restrict__ out) {
    __shared__ double red[8];
    double t = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += 256) t += part[i];
    t = warp_sum(t);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < 8; ++w) s += red[w];
        *out = s;
    }
}

}  // namespace
}  // namespace cfem

using namespace cfem;

int cfem_t10_joule_power(cfem_ctx *ctx, int64_t n_elems, const int32_t *d_elems,
                         const double *d_nodes, const double *d_sigma, const double *d_a_prev,
                         const double *d_a_new, const int64_t *d_vcol, const double *d_v,
                         double h, const double *d_dn, const double *d_mref, double *d_power,
                         double *d_q, void *stream) {
    CFEM_API_BEGIN
    CFEM_CHECK(ctx && d_elems && d_nodes && d_sigma && d_a_prev && d_a_new && d_vcol && d_dn &&
                   d_mref && d_power && n_elems >= 0 && h > 0.0,
               CFEM_ERR_INVALID, "cfem_t10_joule_power: bad args");
    CFEM_TRY(set_device(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;
    if (n_elems == 0) {
        CFEM_CUDA(cudaMemsetAsync(d_power, 0, sizeof(double), s));
        return CFEM_OK;
    }
    const unsigned g = grid_for(n_elems, JT);
    double *part = nullptr;
    CFEM_TRY(tmp_alloc(&part, (size_t)g, s));
    CFEM_LAUNCH(k_t10_joule, g, JT, 0, s, n_elems, d_elems, d_nodes, d_sigma, d_a_prev, d_a_new,
                d_vcol, d_v, h, d_dn, d_mref, d_q, part);
    CFEM_LAUNCH(k_sum_parts, 1, 256, 0, s, (int64_t)g, (const double *)part, d_power);
    tmp_free(part, s);
    return CFEM_OK;
    CFEM_API_END
}
