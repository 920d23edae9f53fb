// Dirichlet elimination on a scalar CSR (cloudfem/fem/tet_poisson.py:72-110).
//
// The reference turns fixed rows into identity rows and zeroes fixed
// columns, keeping those zeros as explicit entries (a dense n x |fixed|
// block once the column assignment is done on CSR). Here the zeroed
// entries are dropped instead, which is the reference's matrix after
// eliminate_zeros() on the columns it cleared; the rhs is lifted exactly
// as rhs - A[:, fixed] v with rhs[fixed] = v.
#include "cfem_common.cuh"

#include <cub/device/device_scan.cuh>

namespace cfem {

__global__ void k_dir_count(int64_t n, const int32_t *__restrict__ indptr,
                            const int32_t *__restrict__ indices,
                            const double *__restrict__ vals,
                            const double *__restrict__ rhs,
                            const uint8_t *__restrict__ fixed,
                            const double *__restrict__ fval,
                            int32_t *__restrict__ counts,
                            double *__restrict__ rhs_out) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (fixed[i]) {
        counts[i] = 1;
        rhs_out[i] = fval[i];
        return;
    }
    int32_t cnt = 0;
    double lift = 0.0;
    for (int32_t k = indptr[i]; k < indptr[i + 1]; ++k) {
        int32_t j = indices[k];
        if (fixed[j]) lift += vals[k] * fval[j];
        else ++cnt;
    }
    counts[i] = cnt;
    rhs_out[i] = rhs[i] - lift;
}

__global__ void k_dir_fill(int64_t n, const int32_t *__restrict__ indptr,
                           const int32_t *__restrict__ indices,
                           const double *__restrict__ vals,
                           const uint8_t *__restrict__ fixed,
                           const int32_t *__restrict__ out_ptr,
                           int32_t *__restrict__ out_idx,
                           double *__restrict__ out_val) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int32_t o = out_ptr[i];
    if (fixed[i]) {
        out_idx[o] = (int32_t)i;
        out_val[o] = 1.0;
        return;
    }
    for (int32_t k = indptr[i]; k < indptr[i + 1]; ++k) {
        int32_t j = indices[k];
        if (fixed[j]) continue;
        out_idx[o] = j;
        out_val[o] = vals[k];
        ++o;
    }
}

}  // namespace cfem

using namespace cfem;

extern "C" int cfem_dirichlet_csr(cfem_ctx *ctx, int64_t n,
                                  const int32_t *d_indptr,
                                  const int32_t *d_indices,
                                  const double *d_vals, const double *d_rhs,
                                  const uint8_t *d_fixed,
                                  const double *d_fixed_val,
                                  int32_t *d_out_indptr,
                                  int32_t *d_out_indices, double *d_out_vals,
                                  double *d_rhs_out, int64_t *nnz_out,
                                  void *stream) {
    CFEM_API_BEGIN
    CFEM_CHECK(ctx && d_indptr && d_fixed && d_fixed_val && d_out_indptr &&
                   d_rhs && d_rhs_out && nnz_out && n > 0,
               CFEM_ERR_INVALID, "cfem_dirichlet_csr: bad args");
    CFEM_TRY(set_device(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;
    int32_t *counts = nullptr;
    CFEM_TRY(tmp_alloc(&counts, n + 1, s));
    CFEM_CUDA(cudaMemsetAsync(counts + n, 0, sizeof(int32_t), s));
    CFEM_LAUNCH(k_dir_count, grid_for(n, 128), 128, 0, s, n, d_indptr, d_indices,
                d_vals, d_rhs, d_fixed, d_fixed_val, counts, d_rhs_out);
    size_t tmp_bytes = 0;
    CFEM_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, counts,
                                            d_out_indptr, (int)(n + 1), s));
    void *tmp = nullptr;
    CFEM_TRY(tmp_alloc((char **)&tmp, tmp_bytes, s));
    CFEM_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, counts, d_out_indptr,
                                            (int)(n + 1), s));
    g_launches.fetch_add(1, std::memory_order_relaxed);
    CFEM_LAUNCH(k_dir_fill, grid_for(n, 128), 128, 0, s, n, d_indptr, d_indices,
                d_vals, d_fixed, d_out_indptr, d_out_indices, d_out_vals);
    int32_t nnz = 0;
    CFEM_CUDA(cudaMemcpyAsync(&nnz, d_out_indptr + n, sizeof(int32_t),
                              cudaMemcpyDeviceToHost, s));
    tmp_free(tmp, s);
    tmp_free(counts, s);
    CFEM_CUDA(cudaStreamSynchronize(s));
    *nnz_out = nnz;
    return CFEM_OK;
    CFEM_API_END
}
