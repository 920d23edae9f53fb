// Deterministic COO -> CSR structure build (replaces the structure half of
// scipy's coo_matrix(...).tocsr(), e.g. cloudfem/fem/tet_poisson.py:68).
//
// Every element contributes the npe*npe node pairs (el[i], el[j]). The
// pairs are encoded as 64-bit keys row*N + col and radix-sorted (stable),
// carrying the contribution id e*npe^2 + i*npe + j. Equal keys are then
// adjacent and ordered by element id; a head/scan pass yields the sorted,
// duplicate-free column list of every row (SciPy's canonical CSR) and the
// segment of contributions per entry that the assembly reduces in a fixed
// order.
#include "cfem_common.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>

namespace cfem {

__global__ void k_pair_keys(const int32_t *__restrict__ elems, int64_t n_elems,
                            int npe, int64_t n_nodes,
                            uint64_t *__restrict__ keys,
                            int32_t *__restrict__ ids, int *bad) {
    const int64_t per = (int64_t)npe * npe;
    const int64_t total = n_elems * per;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        int64_t e = t / per;
        int r = (int)(t - e * per);
        int i = r / npe, j = r - (r / npe) * npe;
        int64_t a = elems[e * npe + i];
        int64_t b = elems[e * npe + j];
        if (a < 0 || a >= n_nodes || b < 0 || b >= n_nodes) {
            atomicExch(bad, 1);
            a = 0;
            b = 0;
        }
        keys[t] = (uint64_t)a * (uint64_t)n_nodes + (uint64_t)b;
        ids[t] = (int32_t)t;
    }
}

__global__ void k_heads(const uint64_t *__restrict__ keys, int64_t total,
                        int32_t *__restrict__ head) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x)
        head[t] = (t == 0 || keys[t] != keys[t - 1]) ? 1 : 0;
}

__global__ void k_scatter_heads(const uint64_t *__restrict__ keys,
                                const int32_t *__restrict__ head,
                                const int32_t *__restrict__ pos, int64_t total,
                                int64_t n_nodes, int32_t *__restrict__ col,
                                int32_t *__restrict__ rowk,
                                int32_t *__restrict__ seg) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        if (!head[t]) continue;
        int32_t k = pos[t];
        uint64_t key = keys[t];
        rowk[k] = (int32_t)(key / (uint64_t)n_nodes);
        col[k] = (int32_t)(key % (uint64_t)n_nodes);
        seg[k] = (int32_t)t;
    }
}

// row_ptr[r] = first entry whose row >= r (rows of entries are sorted).
__global__ void k_row_ptr(const int32_t *__restrict__ rowk, int64_t nnz,
                          int64_t n_nodes, int64_t total,
                          int32_t *__restrict__ row_ptr,
                          int32_t *__restrict__ seg) {
    int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r > n_nodes) return;
    int64_t lo = 0, hi = nnz;
    while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if (rowk[mid] < r) lo = mid + 1; else hi = mid;
    }
    row_ptr[r] = (int32_t)lo;
    if (r == 0) seg[nnz] = (int32_t)total;
}

__global__ void k_diag(const int32_t *__restrict__ row_ptr,
                       const int32_t *__restrict__ col, int64_t n_nodes,
                       int32_t *__restrict__ diag) {
    int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= n_nodes) return;
    int32_t lo = row_ptr[r], hi = row_ptr[r + 1], end = hi;
    while (lo < hi) {
        int32_t mid = (lo + hi) >> 1;
        if (col[mid] < r) lo = mid + 1; else hi = mid;
    }
    diag[r] = (lo < end && col[lo] == r) ? lo : -1;
}

__device__ __forceinline__ int64_t row_of(const int32_t *row_ptr,
                                          int64_t n_rows, int64_t k) {
    int64_t lo = 0, hi = n_rows;   // last r with row_ptr[r] <= k
    while (hi - lo > 1) {
        int64_t mid = (lo + hi) >> 1;
        if (row_ptr[mid] <= k) lo = mid; else hi = mid;
    }
    return lo;
}

__global__ void k_expand(const int32_t *__restrict__ row_ptr,
                         const int32_t *__restrict__ col, int64_t n_nodes,
                         int64_t nnz, int bs, int32_t *__restrict__ indptr,
                         int32_t *__restrict__ indices) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz;
         k += (int64_t)gridDim.x * blockDim.x) {
        int64_t a = row_of(row_ptr, n_nodes, k);
        int64_t start = row_ptr[a], deg = row_ptr[a + 1] - start;
        int64_t off = k - start;
        int32_t b = col[k];
        for (int c = 0; c < bs; ++c) {
            int64_t base = (int64_t)bs * bs * start + (int64_t)c * bs * deg;
            for (int d = 0; d < bs; ++d)
                indices[base + off * bs + d] = b * bs + d;
        }
        if (k == start) {   // first entry of its row writes the row starts
            for (int c = 0; c < bs; ++c)
                indptr[a * bs + c] =
                    (int32_t)((int64_t)bs * bs * start + (int64_t)c * bs * deg);
        }
    }
}

__global__ void k_expand_tail(const int32_t *__restrict__ row_ptr,
                              int64_t n_nodes, int bs,
                              int32_t *__restrict__ indptr) {
    int64_t a = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (a > n_nodes) return;
    int64_t start = row_ptr[a];
    if (a == n_nodes) {
        indptr[n_nodes * bs] = (int32_t)((int64_t)bs * bs * start);
        return;
    }
    if (row_ptr[a + 1] == start) {   // empty row: the k-loop never saw it
        for (int c = 0; c < bs; ++c)
            indptr[a * bs + c] = (int32_t)((int64_t)bs * bs * start);
    }
}

__global__ void k_block_to_csr(const int32_t *__restrict__ row_ptr,
                               int64_t n_nodes, int64_t nnz, int bs,
                               const double *__restrict__ bvals,
                               double *__restrict__ vals) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz;
         k += (int64_t)gridDim.x * blockDim.x) {
        int64_t a = row_of(row_ptr, n_nodes, k);
        int64_t start = row_ptr[a], deg = row_ptr[a + 1] - start;
        int64_t off = k - start;
        for (int c = 0; c < bs; ++c) {
            int64_t base = (int64_t)bs * bs * start + (int64_t)c * bs * deg;
            for (int d = 0; d < bs; ++d)
                vals[base + off * bs + d] = bvals[k * bs * bs + c * bs + d];
        }
    }
}

// Exterior-face candidates: all three corners in the named node set.
__global__ void k_face_flags(const int32_t *__restrict__ elems,
                             int64_t n_elems, int npe, int faces10,
                             const uint8_t *__restrict__ in_set,
                             int64_t n_nodes, uint8_t *__restrict__ flags) {
    // tet_heat.py:112 (a,b,c),(a,b,d),(a,c,d),(b,c,d); tet10.py:287-292
    const int f4[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
    const int f10[4][3] = {{0, 1, 2}, {0, 3, 1}, {0, 2, 3}, {1, 3, 2}};
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
         t < n_elems * 4; t += (int64_t)gridDim.x * blockDim.x) {
        int64_t e = t >> 2;
        int f = (int)(t & 3);
        bool all = true;
        for (int v = 0; v < 3; ++v) {
            int lc = faces10 ? f10[f][v] : f4[f][v];
            int32_t nd = elems[e * npe + lc];
            all = all && nd >= 0 && nd < n_nodes && in_set[nd];
        }
        flags[t] = all ? 1 : 0;
    }
}

// Local face tables: corners (tet_heat.py:112, tet10.py:287-292) and, for
// Tet10, the midside nodes of the three face edges in corner order.
__device__ __forceinline__ int face_corner(int faces10, int f, int v) {
    const int f4[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
    const int f10[4][3] = {{0, 1, 2}, {0, 3, 1}, {0, 2, 3}, {1, 3, 2}};
    return faces10 ? f10[f][v] : f4[f][v];
}
__device__ __forceinline__ int face_mid(int f, int v) {
    const int m10[4][3] = {{4, 5, 6}, {7, 8, 4}, {6, 9, 7}, {8, 9, 5}};
    return m10[f][v];
}

// Sort keys of candidate faces: (min, mid) of the corner triple packed as
// min * n_nodes + mid, and max; value = the candidate's position.
__global__ void k_face_keys(const int32_t *__restrict__ elems, int npe, int faces10,
                            const int64_t *__restrict__ cand, int64_t n, int64_t n_nodes,
                            uint64_t *__restrict__ lo, uint32_t *__restrict__ hi,
                            int32_t *__restrict__ pos) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = cand[i] >> 2;
        const int f = (int)(cand[i] & 3);
        int64_t c[3];
        for (int v = 0; v < 3; ++v) c[v] = elems[e * npe + face_corner(faces10, f, v)];
        int64_t a = min(c[0], min(c[1], c[2])), z = max(c[0], max(c[1], c[2]));
        int64_t m = c[0] + c[1] + c[2] - a - z;
        lo[i] = (uint64_t)a * (uint64_t)n_nodes + (uint64_t)m;
        hi[i] = (uint32_t)z;
        pos[i] = (int32_t)i;
    }
}

template <typename K>
__global__ void k_gather_key(const K *__restrict__ in, const int32_t *__restrict__ pos,
                             int64_t n, K *__restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = in[pos[i]];
}

// In sorted order, a key that differs from both neighbours occurs once:
// flag its candidate position.
__global__ void k_face_once(const uint64_t *__restrict__ lo, const uint32_t *__restrict__ hi,
                            const int32_t *__restrict__ pos, int64_t n,
                            uint8_t *__restrict__ keep) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const bool prev = i > 0 && lo[i - 1] == lo[i] && hi[i - 1] == hi[i];
        const bool next = i + 1 < n && lo[i + 1] == lo[i] && hi[i + 1] == hi[i];
        keep[pos[i]] = (!prev && !next) ? 1 : 0;
    }
}

// Node lists of the kept faces: 3 corners (P1) or 3 corners + 3 midsides.
__global__ void k_face_nodes(const int32_t *__restrict__ elems, int npe, int faces10,
                             const int64_t *__restrict__ ids, int64_t n,
                             int64_t *__restrict__ out) {
    const int width = faces10 ? 6 : 3;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = ids[i] >> 2;
        const int f = (int)(ids[i] & 3);
        for (int v = 0; v < 3; ++v)
            out[i * width + v] = elems[e * npe + face_corner(faces10, f, v)];
        if (faces10)
            for (int v = 0; v < 3; ++v) out[i * width + 3 + v] = elems[e * npe + face_mid(f, v)];
    }
}

static int bits_for(uint64_t maxval) {
    int b = 1;
    while (b < 64 && (maxval >> b) != 0) ++b;
    return b;
}

}  // namespace cfem

using namespace cfem;

extern "C" {

// Pattern arrays and contribution lists of p (already sized fields set by
// the caller); on failure the caller destroys p.
static int build_pattern(cfem_ctx *ctx, const int32_t *d_elems, int64_t n_elems,
                         int32_t npe, int64_t n_nodes, int64_t total,
                         cudaStream_t s, cfem_pattern *p) {
    p->device = ctx->device;
    p->n_nodes = n_nodes;
    p->n_elems = n_elems;
    p->npe = npe;
    // pattern arrays come from the stream-ordered pool: building and
    // dropping patterns does not synchronise the device
    CFEM_TRY(tmp_alloc(&p->row_ptr, n_nodes + 1, s));
    CFEM_TRY(tmp_alloc(&p->diag, n_nodes, s));
    CFEM_TRY(tmp_alloc(&p->contrib, total, s));

    uint64_t *keys = nullptr, *keys_sorted = nullptr;
    int32_t *ids = nullptr, *head = nullptr, *pos = nullptr, *rowk = nullptr;
    int *d_bad = nullptr;
    int64_t nnz = 0;
    if (total > 0) {
        CFEM_TRY(tmp_alloc(&keys, total, s));
        CFEM_TRY(tmp_alloc(&keys_sorted, total, s));
        CFEM_TRY(tmp_alloc(&ids, total, s));
        CFEM_TRY(tmp_alloc(&d_bad, 1, s));
        CFEM_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(int), s));
        unsigned g = grid_for(total, 256);
        if (g > (unsigned)ctx->num_sms * 32) g = ctx->num_sms * 32;
        CFEM_LAUNCH(k_pair_keys, g, 256, 0, s, d_elems, n_elems, npe, n_nodes,
                    keys, ids, d_bad);
        int end_bit = bits_for((uint64_t)n_nodes * (uint64_t)n_nodes - 1);
        size_t tmp_bytes = 0;
        CFEM_CUDA(cub::DeviceRadixSort::SortPairs(
            nullptr, tmp_bytes, keys, keys_sorted, ids, p->contrib,
            (int)total, 0, end_bit, s));
        void *tmp = nullptr;
        CFEM_TRY(tmp_alloc((char **)&tmp, tmp_bytes, s));
        CFEM_CUDA(cub::DeviceRadixSort::SortPairs(
            tmp, tmp_bytes, keys, keys_sorted, ids, p->contrib, (int)total, 0,
            end_bit, s));
        g_launches.fetch_add(end_bit / 8 + 2, std::memory_order_relaxed);
        tmp_free(tmp, s);
        tmp_free(keys, s);
        keys = nullptr;
        tmp_free(ids, s);
        ids = nullptr;

        CFEM_TRY(tmp_alloc(&head, total, s));
        CFEM_TRY(tmp_alloc(&pos, total, s));
        CFEM_LAUNCH(k_heads, g, 256, 0, s, keys_sorted, total, head);
        tmp_bytes = 0;
        CFEM_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, head, pos,
                                                (int)total, s));
        CFEM_TRY(tmp_alloc((char **)&tmp, tmp_bytes, s));
        CFEM_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, head, pos,
                                                (int)total, s));
        g_launches.fetch_add(2, std::memory_order_relaxed);
        tmp_free(tmp, s);
        int32_t last_pos = 0, last_head = 0;
        CFEM_CUDA(cudaMemcpyAsync(&last_pos, pos + total - 1, sizeof(int32_t),
                                  cudaMemcpyDeviceToHost, s));
        CFEM_CUDA(cudaMemcpyAsync(&last_head, head + total - 1,
                                  sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        int bad = 0;
        CFEM_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof(int),
                                  cudaMemcpyDeviceToHost, s));
        CFEM_CUDA(cudaStreamSynchronize(s));
        if (bad) {
            tmp_free(keys_sorted, s);
            tmp_free(head, s);
            tmp_free(pos, s);
            tmp_free(d_bad, s);
            cudaStreamSynchronize(s);
            return fail(CFEM_ERR_INVALID,
                        "element connectivity references a node id outside "
                        "[0, %lld)", (long long)n_nodes);
        }
        nnz = (int64_t)last_pos + last_head;
        CFEM_TRY(tmp_alloc(&p->col, nnz, s));
        CFEM_TRY(tmp_alloc(&p->seg, nnz + 1, s));
        CFEM_TRY(tmp_alloc(&rowk, nnz, s));
        CFEM_LAUNCH(k_scatter_heads, g, 256, 0, s, keys_sorted, head, pos,
                    total, n_nodes, p->col, rowk, p->seg);
        CFEM_LAUNCH(k_row_ptr, grid_for(n_nodes + 1, 256), 256, 0, s, rowk, nnz,
                    n_nodes, total, p->row_ptr, p->seg);
        tmp_free(keys_sorted, s);
        tmp_free(head, s);
        tmp_free(pos, s);
        tmp_free(rowk, s);
        tmp_free(d_bad, s);
    } else {
        CFEM_TRY(tmp_alloc(&p->col, 1, s));
        CFEM_TRY(tmp_alloc(&p->seg, 1, s));
        CFEM_CUDA(cudaMemsetAsync(p->row_ptr, 0, (n_nodes + 1) * sizeof(int32_t), s));
        CFEM_CUDA(cudaMemsetAsync(p->seg, 0, sizeof(int32_t), s));
    }
    p->nnz = nnz;
    CFEM_LAUNCH(k_diag, grid_for(n_nodes, 256), 256, 0, s, p->row_ptr, p->col,
                n_nodes, p->diag);
    CFEM_CUDA(cudaStreamSynchronize(s));
    return CFEM_OK;
}

int cfem_pattern_create(cfem_ctx *ctx, const int32_t *d_elems,
                        int64_t n_elems, int32_t npe, int64_t n_nodes,
                        void *stream, cfem_pattern **out) {
    CFEM_API_BEGIN
    CFEM_CHECK(ctx && out && (d_elems || n_elems == 0), CFEM_ERR_INVALID,
               "cfem_pattern_create: NULL argument");
    CFEM_CHECK(npe == 4 || npe == 10, CFEM_ERR_INVALID,
               "nodes per element must be 4 or 10, got %d", npe);
    CFEM_CHECK(n_nodes > 0 && n_nodes < (int64_t)1 << 31 && n_elems >= 0,
               CFEM_ERR_INVALID, "bad mesh size (%lld nodes, %lld elements)",
               (long long)n_nodes, (long long)n_elems);
    const int64_t total = n_elems * npe * npe;
    CFEM_CHECK(total < ((int64_t)1 << 31), CFEM_ERR_INVALID,
               "mesh too large for one pattern (%lld element entries)",
               (long long)total);
    *out = nullptr;
    CFEM_TRY(set_device(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;

    cfem_pattern *p = new cfem_pattern();
    const int st = build_pattern(ctx, d_elems, n_elems, npe, n_nodes, total, s, p);
    if (st != CFEM_OK) {
        cudaStreamSynchronize(s);
        cfem_pattern_destroy(p);
        return st;
    }
    *out = p;
    return CFEM_OK;
    CFEM_API_END
}

int cfem_pattern_destroy(cfem_pattern *p) {
    if (!p) return CFEM_OK;
    cudaSetDevice(p->device);
    // ordered after all work queued on the legacy stream (which waits for
    // the blocking streams the library's callers use)
    for (void *ptr : {(void *)p->row_ptr, (void *)p->col, (void *)p->diag,
                      (void *)p->seg, (void *)p->contrib})
        if (ptr) cudaFreeAsync(ptr, 0);
    (void)cudaGetLastError();
    delete p;
    return CFEM_OK;
}

int cfem_pattern_info(const cfem_pattern *p, int64_t *n_nodes, int64_t *nnz) {
    CFEM_CHECK(p, CFEM_ERR_INVALID, "pattern is NULL");
    if (n_nodes) *n_nodes = p->n_nodes;
    if (nnz) *nnz = p->nnz;
    return CFEM_OK;
}

int cfem_pattern_node_csr(const cfem_pattern *p, const int32_t **d_row_ptr,
                          const int32_t **d_col) {
    CFEM_CHECK(p, CFEM_ERR_INVALID, "pattern is NULL");
    if (d_row_ptr) *d_row_ptr = p->row_ptr;
    if (d_col) *d_col = p->col;
    return CFEM_OK;
}

int cfem_pattern_expand(const cfem_pattern *p, int32_t bs, int32_t *d_indptr,
                        int32_t *d_indices, void *stream) {
    CFEM_API_BEGIN
    CFEM_CHECK(p && d_indptr && d_indices && (bs == 1 || bs == 3),
               CFEM_ERR_INVALID, "cfem_pattern_expand: bad args");
    CFEM_CHECK((int64_t)bs * bs * p->nnz < ((int64_t)1 << 31),
               CFEM_ERR_INVALID, "expanded CSR exceeds int32 indexing");
    CFEM_TRY(set_device(p->device));
    cudaStream_t s = (cudaStream_t)stream;
    if (p->nnz > 0)
        CFEM_LAUNCH(k_expand, grid_for(p->nnz, 256), 256, 0, s, p->row_ptr,
                    p->col, p->n_nodes, p->nnz, bs, d_indptr, d_indices);
    CFEM_LAUNCH(k_expand_tail, grid_for(p->n_nodes + 1, 256), 256, 0, s,
                p->row_ptr, p->n_nodes, bs, d_indptr);
    return CFEM_OK;
    CFEM_API_END
}

int cfem_block_to_csr(const cfem_pattern *p, int32_t bs, const double *d_bvals,
                      double *d_vals, void *stream) {
    CFEM_API_BEGIN
    CFEM_CHECK(p && d_bvals && d_vals && (bs == 1 || bs == 3),
               CFEM_ERR_INVALID, "cfem_block_to_csr: bad args");
    CFEM_TRY(set_device(p->device));
    if (p->nnz > 0)
        CFEM_LAUNCH(k_block_to_csr, grid_for(p->nnz, 256), 256, 0,
                    (cudaStream_t)stream, p->row_ptr, p->n_nodes, p->nnz, bs,
                    d_bvals, d_vals);
    return CFEM_OK;
    CFEM_API_END
}

int cfem_face_candidates(cfem_ctx *ctx, const int32_t *d_elems,
                         int64_t n_elems, int32_t npe, int32_t faces10,
                         const uint8_t *d_in_set, int64_t n_nodes,
                         int64_t *d_out, int64_t *n_out, void *stream) {
    CFEM_API_BEGIN
    CFEM_CHECK(ctx && d_in_set && d_out && n_out && (npe == 4 || npe == 10),
               CFEM_ERR_INVALID, "cfem_face_candidates: bad args");
    *n_out = 0;
    if (n_elems == 0) return CFEM_OK;
    CFEM_TRY(set_device(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t nf = n_elems * 4;
    uint8_t *flags = nullptr;
    int64_t *cnt = nullptr;
    CFEM_TRY(tmp_alloc(&flags, nf, s));
    CFEM_TRY(tmp_alloc(&cnt, 1, s));
    unsigned g = grid_for(nf, 256);
    if (g > (unsigned)ctx->num_sms * 32) g = ctx->num_sms * 32;
    CFEM_LAUNCH(k_face_flags, g, 256, 0, s, d_elems, n_elems, npe, faces10,
                d_in_set, n_nodes, flags);
    thrust::counting_iterator<int64_t> it(0);
    size_t tmp_bytes = 0;
    CFEM_CUDA(cub::DeviceSelect::Flagged(nullptr, tmp_bytes, it, flags, d_out,
                                         cnt, nf, s));
    void *tmp = nullptr;
    CFEM_TRY(tmp_alloc((char **)&tmp, tmp_bytes, s));
    CFEM_CUDA(cub::DeviceSelect::Flagged(tmp, tmp_bytes, it, flags, d_out, cnt,
                                         nf, s));
    g_launches.fetch_add(2, std::memory_order_relaxed);
    int64_t h_cnt = 0;
    CFEM_CUDA(cudaMemcpyAsync(&h_cnt, cnt, sizeof(int64_t),
                              cudaMemcpyDeviceToHost, s));
    tmp_free(tmp, s);
    tmp_free(flags, s);
    tmp_free(cnt, s);
    CFEM_CUDA(cudaStreamSynchronize(s));
    *n_out = h_cnt;
    return CFEM_OK;
    CFEM_API_END
}

int cfem_face_exterior(cfem_ctx *ctx, const int32_t *d_elems, int32_t npe, int32_t faces10,
                       const int64_t *d_cand, int64_t n_cand, int64_t n_nodes,
                       int64_t *d_ids, int64_t *d_nodes, int64_t *n_out, void *stream) {
    CFEM_API_BEGIN
    CFEM_CHECK(ctx && d_elems && d_ids && d_nodes && n_out && (npe == 4 || npe == 10) &&
                   (faces10 == 0 || npe == 10) && n_cand >= 0 && n_cand < ((int64_t)1 << 31) &&
                   n_nodes > 0 && n_nodes < ((int64_t)1 << 32),
               CFEM_ERR_INVALID, "cfem_face_exterior: bad args");
    *n_out = 0;
    if (n_cand == 0) return CFEM_OK;
    CFEM_CHECK(d_cand, CFEM_ERR_INVALID, "cfem_face_exterior: no candidates");
    CFEM_TRY(set_device(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t n = n_cand;
    uint64_t *lo = nullptr, *lo2 = nullptr;
    uint32_t *hi = nullptr, *hi2 = nullptr;
    int32_t *pos = nullptr, *pos2 = nullptr;
    uint8_t *keep = nullptr;
    int64_t *cnt = nullptr;
    CFEM_TRY(tmp_alloc(&lo, n, s));
    CFEM_TRY(tmp_alloc(&lo2, n, s));
    CFEM_TRY(tmp_alloc(&hi, n, s));
    CFEM_TRY(tmp_alloc(&hi2, n, s));
    CFEM_TRY(tmp_alloc(&pos, n, s));
    CFEM_TRY(tmp_alloc(&pos2, n, s));
    CFEM_TRY(tmp_alloc(&keep, n, s));
    CFEM_TRY(tmp_alloc(&cnt, 1, s));
    unsigned g = grid_for(n, 256);
    if (g > (unsigned)ctx->num_sms * 32) g = ctx->num_sms * 32;
    CFEM_LAUNCH(k_face_keys, g, 256, 0, s, d_elems, npe, faces10, d_cand, n, n_nodes, lo, hi,
                pos);
    // lexicographic (min, mid, max) with ties in candidate order: a stable
    // sort by max, then a stable sort by (min, mid)
    size_t b1 = 0, b2 = 0, b3 = 0;
    CFEM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, b1, hi, hi2, pos, pos2, (int)n, 0,
                                              bits_for(n_nodes), s));
    CFEM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, b2, lo2, lo, pos2, pos, (int)n, 0,
                                              bits_for((uint64_t)n_nodes * n_nodes), s));
    CFEM_CUDA(cub::DeviceSelect::Flagged(nullptr, b3, d_cand, keep, d_ids, cnt, n, s));
    char *tmp = nullptr;
    CFEM_TRY(tmp_alloc(&tmp, std::max(b1, std::max(b2, b3)), s));
    CFEM_CUDA(cub::DeviceRadixSort::SortPairs(tmp, b1, hi, hi2, pos, pos2, (int)n, 0,
                                              bits_for(n_nodes), s));
    CFEM_LAUNCH(k_gather_key<uint64_t>, g, 256, 0, s, lo, pos2, n, lo2);
    CFEM_CUDA(cub::DeviceRadixSort::SortPairs(tmp, b2, lo2, lo, pos2, pos, (int)n, 0,
                                              bits_for((uint64_t)n_nodes * n_nodes), s));
    // hi in the final order: hi2 is sorted by max with pos2; gather by pos
    CFEM_LAUNCH(k_gather_key<uint32_t>, g, 256, 0, s, hi, pos, n, hi2);
    CFEM_LAUNCH(k_face_once, g, 256, 0, s, lo, hi2, pos, n, keep);
    CFEM_CUDA(cub::DeviceSelect::Flagged(tmp, b3, d_cand, keep, d_ids, cnt, n, s));
    g_launches.fetch_add(4, std::memory_order_relaxed);
    int64_t h_cnt = 0;
    CFEM_CUDA(cudaMemcpyAsync(&h_cnt, cnt, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    CFEM_CUDA(cudaStreamSynchronize(s));
    if (h_cnt > 0)
        CFEM_LAUNCH(k_face_nodes, grid_for(h_cnt, 256), 256, 0, s, d_elems, npe, faces10, d_ids,
                    h_cnt, d_nodes);
    for (void *q : {(void *)lo, (void *)lo2, (void *)hi, (void *)hi2, (void *)pos, (void *)pos2,
                    (void *)keep, (void *)cnt, (void *)tmp})
        tmp_free(q, s);
    *n_out = h_cnt;
    return CFEM_OK;
    CFEM_API_END
}

}  // extern "C"
