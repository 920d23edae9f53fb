// Boundary-face integrals on the device: the Neumann, Robin and traction
// terms of tet_heat.py:123-172, tet10.py:354-464 and elastic3d.py /
// elastic_tet10.py over the exterior faces that cfem_face_exterior lists.
//
// cfem_face_geometry: one thread per face, the corner triangle's area and
// the quadrature points (barycentric weights on the corners, the caller's
// rule), so a coefficient given as a host function is evaluated at exactly
// these points. cfem_face_integrate: one thread per face forms
//   f_a   = area sum_q shape[q][a] (w_q load_q)       (per component)
//   K_ab  = area sum_q mt[q][a][b] (w_q h_q)
// and writes them with their keys (node, or position in the node pattern
// found by binary search); the keys are sorted stably (CUB radix sort) and
// each key's run is summed in face order, then added once into F / the
// pattern values: the same order as the reference's np.add.at / COO sum,
// and bitwise the same on every run.
#include "cfem_common.cuh"

#include <cub/device/device_radix_sort.cuh>

namespace cfem {
namespace {

constexpr int FT = 128;   // threads per block
constexpr int FQ = 8;     // most quadrature points per face
constexpr int FN = 6;     // most nodes per face

__global__ void __launch_bounds__(FT)
k_face_geom(int64_t nf, int npf, const int64_t *__restrict__ faces,
            const double *__restrict__ nodes, int nq, const double *__restrict__ bary,
            double *__restrict__ pts, double *__restrict__ area) {
    const int64_t f = (int64_t)blockIdx.x * FT + threadIdx.x;
    if (f >= nf) return;
    double p[3][3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const int64_t nd = faces[f * npf + c];
#pragma unroll
        for (int d = 0; d < 3; ++d) p[c][d] = nodes[nd * 3 + d];
    }
    double a[3], b[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        a[d] = p[1][d] - p[0][d];
        b[d] = p[2][d] - p[0][d];
    }
    const double cx = a[1] * b[2] - a[2] * b[1];
    const double cy = a[2] * b[0] - a[0] * b[2];
    const double cz = a[0] * b[1] - a[1] * b[0];
    area[f] = 0.5 * sqrt(cx * cx + cy * cy + cz * cz);
    if (!pts) return;
    for (int q = 0; q < nq; ++q) {
        const double *L = bary + 3 * q;
        const bool centroid = nq == 1;
#pragma unroll
        for (int d = 0; d < 3; ++d)
            pts[(f * nq + q) * 3 + d] =
                centroid ? (p[0][d] + p[1][d] + p[2][d]) / 3.0
                         : L[0] * p[0][d] + L[1] * p[1][d] + L[2] * p[2][d];
    }
}

// Position of column c in row r of a CSR with sorted columns, or -1.
__device__ __forceinline__ int64_t find_pos(const int32_t *__restrict__ rp,
                                            const int32_t *__restrict__ ci, int64_t r, int64_t c) {
    int32_t lo = rp[r], hi = rp[r + 1] - 1;
    while (lo <= hi) {
        const int32_t mid = (lo + hi) >> 1;
        const int32_t v = ci[mid];
        if (v == c) return mid;
        if (v < c) lo = mid + 1; else hi = mid - 1;
    }
    return -1;
}

__global__ void __launch_bounds__(FT)
k_face_terms(int64_t nf, int npf, const int64_t *__restrict__ faces,
             const double *__restrict__ area, int nq, const double *__restrict__ w,
             const double *__restrict__ shape, int ncomp, const double *__restrict__ load,
             double *__restrict__ lval, int64_t *__restrict__ lkey,
             const double *__restrict__ h, const double *__restrict__ mt,
             const int32_t *__restrict__ rp, const int32_t *__restrict__ ci,
             double *__restrict__ mval, int64_t *__restrict__ mkey, int *__restrict__ bad) {
    const int64_t f = (int64_t)blockIdx.x * FT + threadIdx.x;
    if (f >= nf) return;
    const double A = area[f];
    int64_t nd[FN];
    for (int a = 0; a < npf; ++a) nd[a] = faces[f * npf + a];
    if (load) {
        for (int a = 0; a < npf; ++a) {
            lkey[f * npf + a] = nd[a];
            for (int c = 0; c < ncomp; ++c) {
                double s = 0.0;
                for (int q = 0; q < nq; ++q)
                    s += shape[q * npf + a] * (w[q] * load[(f * nq + q) * ncomp + c]);
                lval[(f * npf + a) * ncomp + c] = A * s;
            }
        }
    }
    if (h) {
        double wh[FQ];
        for (int q = 0; q < nq; ++q) wh[q] = w[q] * h[f * nq + q];
        for (int a = 0; a < npf; ++a)
            for (int b = 0; b < npf; ++b) {
                double s = 0.0;
                for (int q = 0; q < nq; ++q) s += mt[(q * npf + a) * npf + b] * wh[q];
                const int64_t k = (f * npf + a) * npf + b;
                mval[k] = A * s;
                const int64_t pos = find_pos(rp, ci, nd[a], nd[b]);
                if (pos < 0) atomicExch(bad, 1);
                mkey[k] = pos < 0 ? 0 : pos;
            }
    }
}

// Runs of equal sorted keys summed in their (stable) order and added once:
// dst[key * ncomp + c] += sum over the run of val[idx * ncomp + c].
__global__ void __launch_bounds__(256)
k_run_add(int64_t n, int ncomp, const int64_t *__restrict__ key, const int32_t *__restrict__ idx,
          const double *__restrict__ val, double *__restrict__ dst) {
    const int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (i >= n) return;
    const int64_t k = key[i];
    if (i > 0 && key[i - 1] == k) return;   // not the first of its run
    for (int c = 0; c < ncomp; ++c) {
        double s = 0.0;
        for (int64_t j = i; j < n && key[j] == k; ++j) s += val[(int64_t)idx[j] * ncomp + c];
        dst[k * ncomp + c] += s;
    }
}

__global__ void k_iota(int64_t n, int32_t *__restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x;
    if (i < n) out[i] = (int32_t)i;
}

// Sort (key, index) pairs stably by key, then the run sums into dst.
int sorted_add(int64_t n, int ncomp, const int64_t *key, const double *val, double *dst,
               int64_t max_key, cudaStream_t s) {
    if (n == 0) return CFEM_OK;
    int64_t *key2 = nullptr;
    int32_t *idx = nullptr, *idx2 = nullptr;
    CFEM_TRY(tmp_alloc(&key2, (size_t)n, s));
    CFEM_TRY(tmp_alloc(&idx, (size_t)n, s));
    CFEM_TRY(tmp_alloc(&idx2, (size_t)n, s));
    CFEM_LAUNCH(k_iota, grid_for(n, 256), 256, 0, s, n, idx);
    int bits = 1;
    while (bits < 63 && (max_key >> bits) > 0) ++bits;
    // unsigned view of the (non-negative) keys
    const unsigned long long *uk = (const unsigned long long *)key;
    unsigned long long *uk2 = (unsigned long long *)key2;
    size_t tb = 0;
    CFEM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, uk, uk2, idx, idx2, (int)n, 0, bits, s));
    char *tmp = nullptr;
    CFEM_TRY(tmp_alloc(&tmp, tb, s));
    CFEM_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, uk, uk2, idx, idx2, (int)n, 0, bits, s));
    CFEM_LAUNCH(k_run_add, grid_for(n, 256), 256, 0, s, n, ncomp, (const int64_t *)key2,
                (const int32_t *)idx2, val, dst);
    tmp_free(tmp, s);
    tmp_free(idx2, s);
    tmp_free(idx, s);
    tmp_free(key2, s);
    return CFEM_OK;
}

}  // namespace
}  // namespace cfem

using namespace cfem;

int cfem_face_geometry(cfem_ctx *ctx, int32_t npf, int64_t n_faces, const int64_t *d_faces,
                       const double *d_nodes, int32_t nq, const double *d_bary, double *d_pts,
                       double *d_area, void *stream) {
    CFEM_API_BEGIN
    CFEM_CHECK(ctx && (npf == 3 || npf == 6) && n_faces >= 0 && nq >= 1 && nq <= FQ &&
                   d_area && (n_faces == 0 || (d_faces && d_nodes)) && (!d_pts || d_bary),
               CFEM_ERR_INVALID, "cfem_face_geometry: bad args");
    if (n_faces == 0) return CFEM_OK;
    CFEM_TRY(set_device(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;
    CFEM_LAUNCH(k_face_geom, grid_for(n_faces, FT), FT, 0, s, n_faces, (int)npf, d_faces,
                d_nodes, (int)nq, d_bary, d_pts, d_area);
    return CFEM_OK;
    CFEM_API_END
}

int cfem_face_integrate(cfem_ctx *ctx, int32_t npf, int64_t n_faces, const int64_t *d_faces,
                        const double *d_area, int32_t nq, const double *d_w,
                        const double *d_shape, int32_t ncomp, const double *d_load,
                        double *d_F, const double *d_h, const double *d_mt,
                        const int32_t *d_row_ptr, const int32_t *d_col, int64_t n_nodes,
                        double *d_vals, void *stream) {
    CFEM_API_BEGIN
    CFEM_CHECK(ctx && (npf == 3 || npf == 6) && n_faces >= 0 && nq >= 1 && nq <= FQ &&
                   (ncomp == 1 || ncomp == 3) && n_nodes > 0 && d_w &&
                   (!d_load || (d_shape && d_F)) &&
                   (!d_h || (d_mt && d_row_ptr && d_col && d_vals)),
               CFEM_ERR_INVALID, "cfem_face_integrate: bad args");
    if (n_faces == 0 || (!d_load && !d_h)) return CFEM_OK;
    CFEM_CHECK(d_faces && d_area, CFEM_ERR_INVALID, "cfem_face_integrate: no faces given");
    CFEM_TRY(set_device(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t nl = n_faces * npf, nm = d_h ? n_faces * npf * npf : 0;
    CFEM_CHECK(nl < ((int64_t)1 << 31) && nm < ((int64_t)1 << 31), CFEM_ERR_INVALID,
               "cfem_face_integrate: %lld faces exceed one sort", (long long)n_faces);
    double *lval = nullptr, *mval = nullptr;
    int64_t *lkey = nullptr, *mkey = nullptr;
    int *bad = nullptr;
    if (d_load) {
        CFEM_TRY(tmp_alloc(&lval, (size_t)(nl * ncomp), s));
        CFEM_TRY(tmp_alloc(&lkey, (size_t)nl, s));
    }
    if (d_h) {
        CFEM_TRY(tmp_alloc(&mval, (size_t)nm, s));
        CFEM_TRY(tmp_alloc(&mkey, (size_t)nm, s));
        CFEM_TRY(tmp_alloc(&bad, 1, s));
        CFEM_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), s));
    }
    CFEM_LAUNCH(k_face_terms, grid_for(n_faces, FT), FT, 0, s, n_faces, (int)npf, d_faces,
                d_area, (int)nq, d_w, d_shape, (int)ncomp, d_load, lval, lkey, d_h, d_mt,
                d_row_ptr, d_col, mval, mkey, bad);
    int h_bad = 0;
    if (d_h) {
        CFEM_CUDA(cudaMemcpyAsync(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
        CFEM_CUDA(cudaStreamSynchronize(s));
    }
    if (!h_bad) {
        if (d_load) CFEM_TRY(sorted_add(nl, ncomp, lkey, lval, d_F, n_nodes - 1, s));
        if (d_h) {
            int32_t nnz = 0;
            CFEM_CUDA(cudaMemcpyAsync(&nnz, d_row_ptr + n_nodes, sizeof(int32_t),
                                      cudaMemcpyDeviceToHost, s));
            CFEM_CUDA(cudaStreamSynchronize(s));
            CFEM_TRY(sorted_add(nm, 1, mkey, mval, d_vals, nnz > 0 ? nnz - 1 : 0, s));
        }
    }
    tmp_free(bad, s);
    tmp_free(mkey, s);
    tmp_free(mval, s);
    tmp_free(lkey, s);
    tmp_free(lval, s);
    CFEM_CHECK(!h_bad, CFEM_ERR_INVALID,
               "cfem_face_integrate: a face couples two nodes outside the node pattern");
    return CFEM_OK;
    CFEM_API_END
}
