// Shared internals of libcfem: error state, context, launch helpers,
// device utilities. Not part of the public C ABI (see include/cfem.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdarg.h>

#include <atomic>
#include <new>

#include "cfem.h"

namespace cfem {

// ---------------------------------------------------------------- errors
void set_error(const char *fmt, ...);
int fail(int code, const char *fmt, ...);

#define CFEM_CUDA(call)                                                     \
    do {                                                                    \
        cudaError_t e_ = (call);                                            \
        if (e_ != cudaSuccess) {                                            \
            return ::cfem::fail(e_ == cudaErrorMemoryAllocation             \
                                    ? CFEM_ERR_NOMEM : CFEM_ERR_CUDA,       \
                                "%s:%d %s: %s", __FILE__, __LINE__, #call,  \
                                cudaGetErrorString(e_));                    \
        }                                                                   \
    } while (0)

#define CFEM_CHECK(cond, code, ...)                                         \
    do {                                                                    \
        if (!(cond)) return ::cfem::fail((code), __VA_ARGS__);              \
    } while (0)

#define CFEM_TRY(expr)                                                      \
    do {                                                                    \
        int s_ = (expr);                                                    \
        if (s_ != CFEM_OK) return s_;                                       \
    } while (0)

#define CFEM_API_BEGIN try {
#define CFEM_API_END                                                        \
    }                                                                       \
    catch (const std::bad_alloc &) {                                        \
        return ::cfem::fail(CFEM_ERR_NOMEM, "host allocation failed");      \
    }                                                                       \
    catch (...) {                                                           \
        return ::cfem::fail(CFEM_ERR_CUDA, "unexpected C++ exception");     \
    }

// Kernel launches go through this counter so a caller can verify how many
// of this library's kernels ran (reported by bench.py as gpu_launches).
extern std::atomic<int64_t> g_launches;

#define CFEM_LAUNCH(kernel, grid, block, smem, stream, ...)                 \
    do {                                                                    \
        (void)cudaGetLastError(); /* drop stale non-sticky errors */        \
        kernel<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__);         \
        ::cfem::g_launches.fetch_add(1, std::memory_order_relaxed);         \
        CFEM_CUDA(cudaGetLastError());                                      \
    } while (0)

}  // namespace cfem

struct cfem_ctx {
    int device = 0;
    int num_sms = 0;
    int cc_major = 0, cc_minor = 0;
    int64_t launches_at_create = 0;
    int scheduler = 0;                 // CFEM_SCHED_*
    // launch parameters (cfem_ctx_set_param)
    int t10_warps = 4;                 // Tet10 elements per block (batched)
    int p1_threads = 128;              // P1 element kernels, threads per block
    int graph_iters = 2;               // iterations per solve-loop body
    int pdl = 1;                       // dependent launches in solve graphs
    int spmv_stage = 4;                // SpMV: 0 registers, 1 staged scalar rows, 2 also
                                       // 3x3, 3 sliced ELL, 4 auto (per precision and bs)
    int sell_sort = 1;                 // sliced ELL: sort rows by length per window
    int sell3_lanes = 4;               // sliced ELL of 3x3 blocks: lanes per block row
    int sell3_staged = 2;              // ... through a shared-memory ring: 1 always, 2 in
                                       // FP32 only (the faster choice measured), 0 never
    int slot_sell3 = 1;                // solve slots of 3x3 systems: sliced ELL (1) or the
                                       // entry-major copy (0)
    int barrier_timeout_us = 4000000;  // persistent grid-barrier wait limit
    int barrier_hold = 0;              // phantom barrier arrivals (fault injection)
    cudaStream_t work = nullptr;       // capture stream of the graph scheduler
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t tev[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // SpMV timing
    int *h_flags = nullptr;            // pinned host words (convergence polling)
};

struct cfem_pattern {
    int device = 0;
    int64_t n_nodes = 0;
    int64_t n_elems = 0;
    int64_t nnz = 0;          // node-level entries
    int32_t npe = 0;
    int32_t *row_ptr = nullptr;   // n_nodes + 1
    int32_t *col = nullptr;       // nnz
    int32_t *diag = nullptr;      // n_nodes, position of (a, a) or -1
    int32_t *seg = nullptr;       // nnz + 1, contribution segment starts
    int32_t *contrib = nullptr;   // n_elems*npe*npe, ids e*npe^2 + i*npe + j
};

namespace cfem {

// The library's stream-ordered memory pool on the current device. It keeps
// what it has mapped (release threshold: unlimited) so repeated assemblies
// and solves reuse the same physical pages instead of unmapping them at every
// synchronisation and mapping them again; cfem_ctx_trim hands them back.
cudaMemPool_t device_pool();

// Stream-ordered temporary allocation from device_pool().
template <typename T>
int tmp_alloc(T **ptr, size_t count, cudaStream_t s) {
    *ptr = nullptr;
    if (count == 0) count = 1;
    cudaMemPool_t pool = device_pool();
    if (!pool) return fail(CFEM_ERR_CUDA, "no memory pool on the current device");
    cudaError_t e = cudaMallocFromPoolAsync((void **)ptr, count * sizeof(T), pool, s);
    if (e != cudaSuccess) {
        return fail(e == cudaErrorMemoryAllocation ? CFEM_ERR_NOMEM
                                                   : CFEM_ERR_CUDA,
                    "cudaMallocAsync(%zu bytes): %s", count * sizeof(T),
                    cudaGetErrorString(e));
    }
    return CFEM_OK;
}

inline void tmp_free(void *ptr, cudaStream_t s) {
    if (ptr) cudaFreeAsync(ptr, s);
}

inline unsigned grid_for(int64_t n, int block) {
    int64_t g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > 0x7fffffff) g = 0x7fffffff;
    return (unsigned)g;
}

int set_device(int device);

// ---------------------------------------------------------------- device
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace cfem
