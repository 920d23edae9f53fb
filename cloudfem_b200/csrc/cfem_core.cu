// Context, error state and small sparse helpers of libcfem.
#include "cfem_common.cuh"
#include "cfem_tables.cuh"

#include <string.h>

#include <mutex>

namespace cfem {

static thread_local char g_err[1024] = "";
std::atomic<int64_t> g_launches{0};

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int fail(int code, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

int set_device(int device) {
    CFEM_CUDA(cudaSetDevice(device));
    return CFEM_OK;
}

static std::mutex g_pool_mu;
static cudaMemPool_t g_pools[64] = {};

cudaMemPool_t device_pool() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (!g_pools[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
            (void)cudaGetLastError();
            return nullptr;
        }
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        g_pools[dev] = pool;
    }
    return g_pools[dev];
}

// ---------------------------------------------------------------- kernels
__global__ void k_axpby(int64_t n, double a, const double *__restrict__ x,
                        double b, const double *__restrict__ y,
                        double *__restrict__ out) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    for (; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double xv = x ? a * x[i] : 0.0;
        double yv = y ? b * y[i] : 0.0;
        out[i] = xv + yv;
    }
}

// y = alpha A x + beta y over a (block) CSR: SL = 8 lanes per (block) row,
// lane s taking entries s, s + 8, ... (coalesced along the row), the lanes'
// sums meeting in a fixed shuffle tree.
constexpr int SL = 8;
template <int BS>
__global__ void k_spmv(int64_t n, const int32_t *__restrict__ rp,
                       const int32_t *__restrict__ ci,
                       const double *__restrict__ v, double alpha,
                       const double *__restrict__ x, double beta,
                       double *__restrict__ y) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t r = t / SL;
    const int sub = (int)(t % SL);
    double acc[BS];
#pragma unroll
    for (int c = 0; c < BS; ++c) acc[c] = 0.0;
    if (r < n) {
        for (int32_t k = rp[r] + sub; k < rp[r + 1]; k += SL) {
            const int64_t j = ci[k];
#pragma unroll
            for (int c = 0; c < BS; ++c)
#pragma unroll
                for (int d = 0; d < BS; ++d)
                    acc[c] += v[(int64_t)k * BS * BS + c * BS + d] * x[j * BS + d];
        }
    }
#pragma unroll
    for (int o = SL / 2; o > 0; o >>= 1)
#pragma unroll
        for (int c = 0; c < BS; ++c) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], o);
    if (r < n && sub < BS) {
#pragma unroll
        for (int c = 0; c < BS; ++c)
            if (c == sub) {
                const double yv = beta == 0.0 ? 0.0 : beta * y[r * BS + c];
                y[r * BS + c] = alpha * acc[c] + yv;
            }
    }
}

}  // namespace cfem

using namespace cfem;

extern "C" {

const char *cfem_last_error(void) { return g_err; }

int cfem_version(void) { return 10000; }

int cfem_ctx_create(int device, cfem_ctx **out) {
    CFEM_API_BEGIN
    CFEM_CHECK(out != nullptr, CFEM_ERR_INVALID, "out is NULL");
    *out = nullptr;
    int ndev = 0;
    CFEM_CUDA(cudaGetDeviceCount(&ndev));
    CFEM_CHECK(device >= 0 && device < ndev, CFEM_ERR_INVALID,
               "device %d out of range (%d devices)", device, ndev);
    CFEM_TRY(set_device(device));
    cudaDeviceProp prop;
    CFEM_CUDA(cudaGetDeviceProperties(&prop, device));
    CFEM_CHECK(prop.major == 10, CFEM_ERR_UNSUPPORTED,
               "libcfem is built for sm_100a; device %d is sm_%d%d (%s)",
               device, prop.major, prop.minor, prop.name);
    CFEM_TRY(upload_tables(device));
    CFEM_CHECK(device_pool() != nullptr, CFEM_ERR_CUDA,
               "cannot create the memory pool on device %d", device);
    cfem_ctx *c = new cfem_ctx();
    c->device = device;
    c->num_sms = prop.multiProcessorCount;
    c->cc_major = prop.major;
    c->cc_minor = prop.minor;
    c->launches_at_create = g_launches.load();
    CFEM_CUDA(cudaStreamCreateWithFlags(&c->work, cudaStreamNonBlocking));
    for (int i = 0; i < 4; ++i)
        CFEM_CUDA(cudaEventCreateWithFlags(&c->ev[i], i < 2 ? cudaEventDisableTiming
                                                            : cudaEventDefault));
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j) CFEM_CUDA(cudaEventCreate(&c->tev[i][j]));
    CFEM_CUDA(cudaMallocHost(&c->h_flags, 4 * sizeof(int)));
    *out = c;
    return CFEM_OK;
    CFEM_API_END
}

int cfem_ctx_destroy(cfem_ctx *ctx) {
    if (!ctx) return CFEM_OK;
    cudaSetDevice(ctx->device);
    if (ctx->work) cudaStreamSynchronize(ctx->work);
    for (int i = 0; i < 4; ++i)
        if (ctx->ev[i]) cudaEventDestroy(ctx->ev[i]);
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j)
            if (ctx->tev[i][j]) cudaEventDestroy(ctx->tev[i][j]);
    if (ctx->work) cudaStreamDestroy(ctx->work);
    if (ctx->h_flags) cudaFreeHost(ctx->h_flags);
    delete ctx;
    return CFEM_OK;
}

int cfem_ctx_set_scheduler(cfem_ctx *ctx, int scheduler) {
    CFEM_CHECK(ctx && scheduler >= CFEM_SCHED_AUTO && scheduler <= CFEM_SCHED_GRAPH_POLLED,
               CFEM_ERR_INVALID, "unknown scheduler %d", scheduler);
    ctx->scheduler = scheduler;
    return CFEM_OK;
}

int cfem_ctx_trim(cfem_ctx *ctx, uint64_t keep_bytes, uint64_t *reserved_bytes) {
    CFEM_API_BEGIN
    CFEM_CHECK(ctx, CFEM_ERR_INVALID, "cfem_ctx_trim: ctx is NULL");
    CFEM_TRY(set_device(ctx->device));
    cudaMemPool_t pool = device_pool();
    CFEM_CHECK(pool, CFEM_ERR_CUDA, "no memory pool on device %d", ctx->device);
    CFEM_CUDA(cudaDeviceSynchronize());
    CFEM_CUDA(cudaMemPoolTrimTo(pool, (size_t)keep_bytes));
    if (reserved_bytes) {
        uint64_t v = 0;
        CFEM_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &v));
        *reserved_bytes = v;
    }
    return CFEM_OK;
    CFEM_API_END
}

int cfem_ctx_set_param(cfem_ctx *ctx, int param, int value) {
    CFEM_CHECK(ctx, CFEM_ERR_INVALID, "cfem_ctx_set_param: ctx is NULL");
    switch (param) {
        case CFEM_PARAM_T10_WARPS:
            CFEM_CHECK(value == 2 || value == 4 || value == 8, CFEM_ERR_INVALID,
                       "Tet10 elements per block must be 2, 4 or 8 (got %d)", value);
            ctx->t10_warps = value;
            return CFEM_OK;
        case CFEM_PARAM_P1_THREADS:
            CFEM_CHECK(value == 32 || value == 64 || value == 128, CFEM_ERR_INVALID,
                       "P1 threads per block must be 32, 64 or 128 (got %d)", value);
            ctx->p1_threads = value;
            return CFEM_OK;
        case CFEM_PARAM_GRAPH_ITERS:
            CFEM_CHECK(value == 1 || value == 2 || value == 4 || value == 8 || value == 16,
                       CFEM_ERR_INVALID,
                       "iterations per solve-loop body must be 1, 2, 4, 8 or 16 (got %d)",
                       value);
            ctx->graph_iters = value;
            return CFEM_OK;
        case CFEM_PARAM_PDL:
            CFEM_CHECK(value == 0 || value == 1, CFEM_ERR_INVALID,
                       "dependent-launch switch must be 0 or 1 (got %d)", value);
            ctx->pdl = value;
            return CFEM_OK;
        case CFEM_PARAM_SPMV_STAGE:
            CFEM_CHECK(value >= 0 && value <= 4, CFEM_ERR_INVALID,
                       "SpMV staging must be 0, 1, 2, 3 or 4 (got %d)", value);
            ctx->spmv_stage = value;
            return CFEM_OK;
        case CFEM_PARAM_SELL_SORT:
            CFEM_CHECK(value == 0 || value == 1, CFEM_ERR_INVALID,
                       "sliced-ELL row sorting must be 0 or 1 (got %d)", value);
            ctx->sell_sort = value;
            return CFEM_OK;
        case CFEM_PARAM_SELL3_STAGED:
            CFEM_CHECK(value >= 0 && value <= 2, CFEM_ERR_INVALID,
                       "sliced-ELL 3x3 staging must be 0, 1 or 2 (got %d)", value);
            ctx->sell3_staged = value;
            return CFEM_OK;
        case CFEM_PARAM_SLOT_SELL3:
            CFEM_CHECK(value == 0 || value == 1, CFEM_ERR_INVALID,
                       "slot sliced-ELL switch must be 0 or 1 (got %d)", value);
            ctx->slot_sell3 = value;
            return CFEM_OK;
        case CFEM_PARAM_SELL3_LANES:
            CFEM_CHECK(value == 1 || value == 2 || value == 4, CFEM_ERR_INVALID,
                       "sliced-ELL lanes per 3x3 block row must be 1, 2 or 4 (got %d)", value);
            ctx->sell3_lanes = value;
            return CFEM_OK;
        case CFEM_PARAM_BARRIER_TIMEOUT_US:
            CFEM_CHECK(value >= 1 && value <= 60000000, CFEM_ERR_INVALID,
                       "grid-barrier wait limit must be 1 us .. 60 s (got %d us)", value);
            ctx->barrier_timeout_us = value;
            return CFEM_OK;
        case CFEM_PARAM_BARRIER_HOLD:
            CFEM_CHECK(value == 0 || value == 1, CFEM_ERR_INVALID,
                       "phantom barrier arrivals must be 0 or 1 (got %d)", value);
            ctx->barrier_hold = value;
            return CFEM_OK;
        default:
            return fail(CFEM_ERR_INVALID, "unknown parameter %d", param);
    }
}

int cfem_ctx_get_param(const cfem_ctx *ctx, int param) {
    if (!ctx) return -1;
    switch (param) {
        case CFEM_PARAM_T10_WARPS: return ctx->t10_warps;
        case CFEM_PARAM_P1_THREADS: return ctx->p1_threads;
        case CFEM_PARAM_GRAPH_ITERS: return ctx->graph_iters;
        case CFEM_PARAM_PDL: return ctx->pdl;
        case CFEM_PARAM_SPMV_STAGE: return ctx->spmv_stage;
        case CFEM_PARAM_SELL_SORT: return ctx->sell_sort;
        case CFEM_PARAM_SELL3_LANES: return ctx->sell3_lanes;
        case CFEM_PARAM_SELL3_STAGED: return ctx->sell3_staged;
        case CFEM_PARAM_SLOT_SELL3: return ctx->slot_sell3;
        case CFEM_PARAM_BARRIER_TIMEOUT_US: return ctx->barrier_timeout_us;
        case CFEM_PARAM_BARRIER_HOLD: return ctx->barrier_hold;
        default: return -1;
    }
}

int64_t cfem_ctx_launch_count(const cfem_ctx *ctx) {
    (void)ctx;
    return g_launches.load();
}

int cfem_axpby(cfem_ctx *ctx, int64_t n, double a, const double *d_x,
               double b, const double *d_y, double *d_out, void *stream) {
    CFEM_API_BEGIN
    CFEM_CHECK(ctx && d_out && n >= 0, CFEM_ERR_INVALID, "cfem_axpby: bad args");
    if (n == 0) return CFEM_OK;
    CFEM_TRY(set_device(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;
    unsigned g = grid_for(n, 256);
    if (g > (unsigned)ctx->num_sms * 16) g = ctx->num_sms * 16;
    CFEM_LAUNCH(k_axpby, g, 256, 0, s, n, a, d_x, b, d_y, d_out);
    return CFEM_OK;
    CFEM_API_END
}

int cfem_spmv(cfem_ctx *ctx, int64_t n_rows, int32_t bs,
              const int32_t *d_row_ptr, const int32_t *d_col,
              const double *d_vals, double alpha, const double *d_x,
              double beta, double *d_y, void *stream) {
    CFEM_API_BEGIN
    CFEM_CHECK(ctx && d_row_ptr && d_col && d_vals && d_x && d_y &&
                   n_rows >= 0 && (bs == 1 || bs == 3),
               CFEM_ERR_INVALID, "cfem_spmv: bad args");
    if (n_rows == 0) return CFEM_OK;
    CFEM_TRY(set_device(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;
    unsigned g = grid_for(n_rows * SL, 128);
    if (bs == 1)
        CFEM_LAUNCH(k_spmv<1>, g, 128, 0, s, n_rows, d_row_ptr, d_col, d_vals,
                    alpha, d_x, beta, d_y);
    else
        CFEM_LAUNCH(k_spmv<3>, g, 128, 0, s, n_rows, d_row_ptr, d_col, d_vals,
                    alpha, d_x, beta, d_y);
    return CFEM_OK;
    CFEM_API_END
}

}  // extern "C"
