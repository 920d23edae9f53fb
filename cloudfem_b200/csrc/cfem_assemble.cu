// Element kernels and the deterministic segmented reduction into CSR.
//
// Pass 1 computes every element matrix into a staging buffer laid out as
// contribution ids (e*npe^2 + i*npe + j, times bs*bs for vector problems):
//   * P1 (4 nodes): one thread per element, 3x3 inverse by cofactors.
//   * Tet10 (10 nodes): one warp per element; the Keast-5 physical shape
//     gradients G[q][a] (5 x 10 x 3) are staged in shared memory, then each
//     lane produces entries / 3x3 blocks of the element matrix.
// Pass 2 walks each CSR entry's contribution segment (sorted by element id
// when the pattern was built) and writes the sum once: no atomics, so the
// values are bitwise reproducible from run to run.
// Pass 3 does the same for load vectors through the diagonal entry's
// segment, which lists the node's (element, local index) pairs in element
// order - the order of the reference's rhs[el] += fe loop.
#include "cfem_common.cuh"
#include "cfem_tables.cuh"

#include <math.h>
#include <mutex>
#include <vector>

namespace cfem {

// --------------------------------------------------------- reference tables
// Keast 5-point rule (cloudfem/fem/tet10.py:84-100), quadratic shape values
// and barycentric derivatives (tet10.py:63-81), d/dxi = d/dL_{k+1} - d/dL_0
// (tet10.py:121-123), exact unit-volume mass (tet10.py:185-226).
__constant__ double c_wq[5];
__constant__ double c_Lq[5][4];
__constant__ double c_N[5][10];
__constant__ double c_dNdxi[5][10][3];
__constant__ double c_mass[10][10];

static const int kEdges[6][2] = {{0, 1}, {1, 2}, {2, 0}, {0, 3}, {1, 3}, {2, 3}};

static double factorial(int n) {
    double f = 1.0;
    for (int i = 2; i <= n; ++i) f *= i;
    return f;
}

int upload_tables(int device) {
    static std::mutex mu;
    static bool done[64] = {false};
    std::lock_guard<std::mutex> lock(mu);
    if (device >= 0 && device < 64 && done[device]) return CFEM_OK;
    double wq[5], Lq[5][4], N[5][10], dN[5][10][4], dxi[5][10][3], M[10][10];
    const double a = 0.5, b = 1.0 / 6.0;
    const double L[5][4] = {{0.25, 0.25, 0.25, 0.25}, {a, b, b, b},
                            {b, a, b, b}, {b, b, a, b}, {b, b, b, a}};
    wq[0] = -4.0 / 5.0;
    for (int q = 1; q < 5; ++q) wq[q] = 9.0 / 20.0;
    for (int q = 0; q < 5; ++q) {
        for (int i = 0; i < 4; ++i) Lq[q][i] = L[q][i];
        for (int s = 0; s < 10; ++s)
            for (int i = 0; i < 4; ++i) dN[q][s][i] = 0.0;
        for (int i = 0; i < 4; ++i) {
            N[q][i] = L[q][i] * (2.0 * L[q][i] - 1.0);
            dN[q][i][i] = 4.0 * L[q][i] - 1.0;
        }
        for (int k = 0; k < 6; ++k) {
            int i = kEdges[k][0], j = kEdges[k][1];
            N[q][4 + k] = 4.0 * L[q][i] * L[q][j];
            dN[q][4 + k][i] = 4.0 * L[q][j];
            dN[q][4 + k][j] = 4.0 * L[q][i];
        }
        for (int s = 0; s < 10; ++s)
            for (int k = 0; k < 3; ++k)
                dxi[q][s][k] = dN[q][s][k + 1] - dN[q][s][0];
    }
    // shape functions as sums of barycentric monomials c * L^alpha
    struct Term { double c; int al[4]; };
    Term poly[10][2];
    int nterm[10];
    for (int i = 0; i < 4; ++i) {
        poly[i][0] = {2.0, {0, 0, 0, 0}};
        poly[i][0].al[i] = 2;
        poly[i][1] = {-1.0, {0, 0, 0, 0}};
        poly[i][1].al[i] = 1;
        nterm[i] = 2;
    }
    for (int k = 0; k < 6; ++k) {
        poly[4 + k][0] = {4.0, {0, 0, 0, 0}};
        poly[4 + k][0].al[kEdges[k][0]] += 1;
        poly[4 + k][0].al[kEdges[k][1]] += 1;
        nterm[4 + k] = 1;
    }
    for (int r = 0; r < 10; ++r)
        for (int s = 0; s < 10; ++s) {
            double acc = 0.0;
            for (int t1 = 0; t1 < nterm[r]; ++t1)
                for (int t2 = 0; t2 < nterm[s]; ++t2) {
                    double num = 1.0;
                    int tot = 0;
                    for (int v = 0; v < 4; ++v) {
                        int e = poly[r][t1].al[v] + poly[s][t2].al[v];
                        num *= factorial(e);
                        tot += e;
                    }
                    acc += poly[r][t1].c * poly[s][t2].c * 6.0 * num /
                           factorial(tot + 3);
                }
            M[r][s] = acc;
        }
    CFEM_CUDA(cudaMemcpyToSymbol(c_wq, wq, sizeof(wq)));
    CFEM_CUDA(cudaMemcpyToSymbol(c_Lq, Lq, sizeof(Lq)));
    CFEM_CUDA(cudaMemcpyToSymbol(c_N, N, sizeof(N)));
    CFEM_CUDA(cudaMemcpyToSymbol(c_dNdxi, dxi, sizeof(dxi)));
    CFEM_CUDA(cudaMemcpyToSymbol(c_mass, M, sizeof(M)));
    if (device >= 0 && device < 64) done[device] = true;
    return CFEM_OK;
}

// ---------------------------------------------------------------- helpers
struct Coef {
    const double *v;
    double c;
    int mode;
};

static Coef to_coef(const cfem_coef *c) {
    Coef k{nullptr, 0.0, CFEM_COEF_CONST};
    if (c) {
        k.v = c->d_values;
        k.c = c->constant;
        k.mode = c->mode;
    }
    return k;
}

__device__ __forceinline__ double coef_at(const Coef &k, int64_t e, int q) {
    if (k.mode == CFEM_COEF_CONST) return k.c;
    if (k.mode == CFEM_COEF_ELEM) return k.v[e];
    return k.v[e * 5 + q];   // CFEM_COEF_QP
}

struct Geo {
    double inv[3][3];
    double vol;
};

// m[r][c] = (p_{c+1} - p_0)[r]  (tet_poisson.py:23, tet10.py:115)
__device__ __forceinline__ void tet_geo(const double *__restrict__ nodes,
                                        int32_t n0, int32_t n1, int32_t n2,
                                        int32_t n3, Geo &g) {
    const double *p0 = nodes + 3 * (int64_t)n0;
    const double *p1 = nodes + 3 * (int64_t)n1;
    const double *p2 = nodes + 3 * (int64_t)n2;
    const double *p3 = nodes + 3 * (int64_t)n3;
    double m[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        double o = __ldg(p0 + r);
        m[r][0] = __ldg(p1 + r) - o;
        m[r][1] = __ldg(p2 + r) - o;
        m[r][2] = __ldg(p3 + r) - o;
    }
    double c00 = m[1][1] * m[2][2] - m[1][2] * m[2][1];
    double c01 = m[1][2] * m[2][0] - m[1][0] * m[2][2];
    double c02 = m[1][0] * m[2][1] - m[1][1] * m[2][0];
    double det = m[0][0] * c00 + m[0][1] * c01 + m[0][2] * c02;
    double id = 1.0 / det;
    g.inv[0][0] = c00 * id;
    g.inv[0][1] = (m[0][2] * m[2][1] - m[0][1] * m[2][2]) * id;
    g.inv[0][2] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]) * id;
    g.inv[1][0] = c01 * id;
    g.inv[1][1] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]) * id;
    g.inv[1][2] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) * id;
    g.inv[2][0] = c02 * id;
    g.inv[2][1] = (m[0][1] * m[2][0] - m[0][0] * m[2][1]) * id;
    g.inv[2][2] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]) * id;
    g.vol = fabs(det) / 6.0;
}

// P1 gradients: G = g_ref * m^-1 (tet_poisson.py:26-31)
__device__ __forceinline__ void p1_grads(const Geo &g, double G[4][3]) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        G[1][c] = g.inv[0][c];
        G[2][c] = g.inv[1][c];
        G[3][c] = g.inv[2][c];
        G[0][c] = -(g.inv[0][c] + g.inv[1][c] + g.inv[2][c]);
    }
}

// ------------------------------------------------------------- P1 scalar
// OP = CFEM_OP_P1_STIFF: Ke = (k V) G G^T, fe = f V / 4 (tet_poisson.py:51-66)
// OP = CFEM_OP_P1_MASS : Ke = (rho V) (1 + d_ij)/20  (tet_heat.py:81-94)
template <int OP>
__device__ __forceinline__ void p1_scalar_elem(const double *__restrict__ nodes,
                                               const int32_t *__restrict__ elems,
                                               int64_t e, const Coef &coef,
                                               const Coef &load, double *ke,
                                               double *fe) {
    int4 el = __ldg(reinterpret_cast<const int4 *>(elems) + e);
    Geo g;
    tet_geo(nodes, el.x, el.y, el.z, el.w, g);
    double out[16];
    if (OP == CFEM_OP_P1_STIFF) {
        double G[4][3];
        p1_grads(g, G);
        double kv = coef_at(coef, e, 0) * g.vol;
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
                out[i * 4 + j] = kv * (G[i][0] * G[j][0] + G[i][1] * G[j][1] +
                                       G[i][2] * G[j][2]);
        if (fe) {
            double f = coef_at(load, e, 0) * g.vol / 4.0;
            *reinterpret_cast<double4 *>(fe) = make_double4(f, f, f, f);
        }
    } else {
        double rv = coef_at(coef, e, 0) * g.vol;
        double d = rv * (2.0 / 20.0), o = rv * (1.0 / 20.0);
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) out[i * 4 + j] = (i == j) ? d : o;
    }
    double4 *dst = reinterpret_cast<double4 *>(ke);
#pragma unroll
    for (int v = 0; v < 4; ++v)
        dst[v] = make_double4(out[4 * v], out[4 * v + 1], out[4 * v + 2],
                              out[4 * v + 3]);
}

template <int OP>
__global__ void __launch_bounds__(128)
k_p1_scalar(const double *__restrict__ nodes, const int32_t *__restrict__ elems,
            int64_t M, Coef coef, Coef load, double *__restrict__ ke,
            double *__restrict__ fe) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= M) return;
    p1_scalar_elem<OP>(nodes, elems, e, coef, load, ke + e * 16, fe ? fe + e * 4 : nullptr);
}

// ------------------------------------------------------------- P1 elastic
// Ke_ab = V (lam g_a g_b^T + mu g_b g_a^T + mu (g_a.g_b) I), the closed form
// of V B^T D B for isotropic D (elastic3d.py:145-149); body b V/4
// (elastic3d.py:157-162); thermal V B^T D eps_th (elastic3d.py:164-169).
__global__ void __launch_bounds__(128)
k_p1_elastic(const double *__restrict__ nodes, const int32_t *__restrict__ elems,
             int64_t M, double lam, double mu, Coef b0, Coef b1, Coef b2,
             Coef temp, const double *__restrict__ tnodal, int thermal,
             double alpha, double tref, double *__restrict__ ke,
             double *__restrict__ fe) {
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= M) return;
    int4 el = __ldg(reinterpret_cast<const int4 *>(elems) + e);
    Geo g;
    tet_geo(nodes, el.x, el.y, el.z, el.w, g);
    double G[4][3];
    p1_grads(g, G);
    const double V = g.vol;
    double *dst = ke + e * 144;
    for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 4; ++b) {
            double dot = G[a][0] * G[b][0] + G[a][1] * G[b][1] + G[a][2] * G[b][2];
            double blk[9];
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    blk[c * 3 + d] = V * (lam * G[a][c] * G[b][d] +
                                          mu * G[a][d] * G[b][c] +
                                          (c == d ? mu * dot : 0.0));
#pragma unroll
            for (int v = 0; v < 9; ++v) dst[(a * 4 + b) * 9 + v] = blk[v];
        }
    if (fe) {
        double bv[3] = {coef_at(b0, e, 0), coef_at(b1, e, 0), coef_at(b2, e, 0)};
        double th = 0.0;
        if (thermal) {
            double Tc;
            if (tnodal) {
                Tc = (((tnodal[el.x] + tnodal[el.y]) + tnodal[el.z]) + tnodal[el.w]) / 4.0;
            } else {
                Tc = coef_at(temp, e, 0);
            }
            th = (3.0 * lam + 2.0 * mu) * alpha * (Tc - tref);
        }
        for (int a = 0; a < 4; ++a)
            for (int c = 0; c < 3; ++c)
                fe[e * 12 + a * 3 + c] = bv[c] * V / 4.0 + G[a][c] * th * V;
    }
}

// ------------------------------------------------------------- Tet10
// One warp per element. Shared: physical gradients G[q][a][3].
constexpr int T10_WARPS = 4;

__device__ __forceinline__ void t10_stage_grads(const double *__restrict__ nodes,
                                                const int32_t *__restrict__ el,
                                                double (*Gs)[10][3], int lane,
                                                double &vol) {
    Geo g;
    tet_geo(nodes, __ldg(el + 0), __ldg(el + 1), __ldg(el + 2), __ldg(el + 3), g);
    vol = g.vol;
    for (int t = lane; t < 50; t += 32) {
        int q = t / 10, a = t - (t / 10) * 10;
#pragma unroll
        for (int j = 0; j < 3; ++j)
            Gs[q][a][j] = c_dNdxi[q][a][0] * g.inv[0][j] +
                          c_dNdxi[q][a][1] * g.inv[1][j] +
                          c_dNdxi[q][a][2] * g.inv[2][j];
    }
    __syncwarp();
}

// OP = CFEM_OP_T10_STIFF: Ke = V sum_q (w_q k_q) G_q G_q^T, fe = V sum_q N_q w_q f_q
//                        (tet10.py:150-161)
// OP = CFEM_OP_T10_MASS : Ke = (rho V) MASS_REF (tet10.py:241-246)
template <int OP>
__device__ __forceinline__ void t10_scalar_elem(const double *__restrict__ nodes,
                                                const int32_t *__restrict__ elems,
                                                int64_t e, const Coef &coef,
                                                const Coef &load, double *ke,
                                                double *fe, double (*sG)[10][3],
                                                int lane) {
    const int32_t *el = elems + e * 10;
    if (OP == CFEM_OP_T10_NGRAD_X || OP == CFEM_OP_T10_NGRAD_Y || OP == CFEM_OP_T10_NGRAD_Z) {
        // ke[p][j] = (sigma V) sum_q w_q N_qp dN_j/dx_m (em3d_tet10.py:225)
        constexpr int m = OP - CFEM_OP_T10_NGRAD_X;
        double vol;
        t10_stage_grads(nodes, el, sG, lane, vol);
        const double sv = coef_at(coef, e, 0) * vol;
        for (int t = lane; t < 100; t += 32) {
            int a = t / 10, b = t - (t / 10) * 10;
            double s = 0.0;
#pragma unroll
            for (int q = 0; q < 5; ++q) s += c_wq[q] * c_N[q][a] * sG[q][b][m];
            ke[t] = sv * s;
        }
        __syncwarp();
    } else if (OP == CFEM_OP_T10_STIFF) {
        double vol;
        t10_stage_grads(nodes, el, sG, lane, vol);
        double wk[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) wk[q] = c_wq[q] * coef_at(coef, e, q);
        // the 55 pairs a <= b, each written to (a, b) and (b, a): the dot
        // products are symmetric in floating point, so the matrix is the
        // same as entry by entry with half the shared-memory reads
        for (int t = lane; t < 55; t += 32) {
            // pair t in row-major order of the upper triangle
            int a = 0, r = t;
            while (r >= 10 - a) {
                r -= 10 - a;
                ++a;
            }
            const int b = a + r;
            double s = 0.0;
#pragma unroll
            for (int q = 0; q < 5; ++q)
                s += wk[q] * (sG[q][a][0] * sG[q][b][0] + sG[q][a][1] * sG[q][b][1] +
                              sG[q][a][2] * sG[q][b][2]);
            ke[a * 10 + b] = vol * s;
            ke[b * 10 + a] = vol * s;
        }
        if (fe && lane < 10) {
            double s = 0.0;
#pragma unroll
            for (int q = 0; q < 5; ++q) s += c_N[q][lane] * (c_wq[q] * coef_at(load, e, q));
            fe[lane] = vol * s;
        }
        __syncwarp();
    } else {
        Geo g;
        tet_geo(nodes, __ldg(el + 0), __ldg(el + 1), __ldg(el + 2), __ldg(el + 3), g);
        double rv = coef_at(coef, e, 0) * g.vol;
        for (int t = lane; t < 100; t += 32)
            ke[t] = rv * c_mass[t / 10][t - (t / 10) * 10];
    }
}

template <int OP>
__global__ void __launch_bounds__(32 * T10_WARPS)
k_t10_scalar(const double *__restrict__ nodes, const int32_t *__restrict__ elems,
             int64_t M, Coef coef, Coef load, double *__restrict__ ke,
             double *__restrict__ fe) {
    __shared__ double sG[T10_WARPS][5][10][3];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t e = (int64_t)blockIdx.x * T10_WARPS + w;
    if (e >= M) return;
    t10_scalar_elem<OP>(nodes, elems, e, coef, load, ke + e * 100,
                        fe ? fe + e * 10 : nullptr, sG[w], lane);
}

// Tet10 elasticity: block (a,b) = V sum_q w_q (lam g_a g_b^T + mu g_b g_a^T
// + mu (g_a.g_b) I) with g = G_q (elastic_tet10.py:166-172); body
// V sum_q w_q N_qa b_q (:177-181); thermal V sum_q w_q B_q^T D eps_th(q)
// (:183-192).
__global__ void __launch_bounds__(32 * T10_WARPS)
k_t10_elastic(const double *__restrict__ nodes, const int32_t *__restrict__ elems,
              int64_t M, double lam, double mu, Coef b0, Coef b1, Coef b2,
              Coef temp, const double *__restrict__ tnodal, int thermal,
              double alpha, double tref, double *__restrict__ ke,
              double *__restrict__ fe) {
    __shared__ double sG[T10_WARPS][5][10][3];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t e = (int64_t)blockIdx.x * T10_WARPS + w;
    if (e >= M) return;
    const int32_t *el = elems + e * 10;
    double vol;
    t10_stage_grads(nodes, el, sG[w], lane, vol);
    for (int t = lane; t < 100; t += 32) {
        int a = t / 10, b = t - (t / 10) * 10;
        double blk[9];
#pragma unroll
        for (int v = 0; v < 9; ++v) blk[v] = 0.0;
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            const double wq = c_wq[q];
            double ga[3], gb[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                ga[c] = sG[w][q][a][c];
                gb[c] = sG[w][q][b][c];
            }
            double dot = ga[0] * gb[0] + ga[1] * gb[1] + ga[2] * gb[2];
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    blk[c * 3 + d] += wq * (lam * ga[c] * gb[d] + mu * ga[d] * gb[c] +
                                            (c == d ? mu * dot : 0.0));
        }
        double *dst = ke + (e * 100 + t) * 9;
#pragma unroll
        for (int v = 0; v < 9; ++v) dst[v] = vol * blk[v];
    }
    if (fe && lane < 30) {
        const int a = lane / 3, c = lane - (lane / 3) * 3;
        const Coef &bc = (c == 0) ? b0 : (c == 1 ? b1 : b2);
        double sb = 0.0, st = 0.0;
        const double k3 = (3.0 * lam + 2.0 * mu) * alpha;
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            sb += c_wq[q] * c_N[q][a] * coef_at(bc, e, q);
            if (thermal) {
                double Tq;
                if (tnodal) {
                    Tq = 0.0;
#pragma unroll
                    for (int s = 0; s < 10; ++s) Tq += c_N[q][s] * tnodal[__ldg(el + s)];
                } else {
                    Tq = coef_at(temp, e, q);
                }
                st += c_wq[q] * sG[w][q][a][c] * (k3 * (Tq - tref));
            }
        }
        fe[e * 30 + lane] = vol * sb + vol * st;
    }
}

// Tet10 nodal curl-curl: block (a,b) = (nu V) sum_q w_q ((g_a.g_b) I - g_b g_a^T),
// the Levi-Civita contraction of em3d_tet10.py:205-208 in closed form.
__global__ void __launch_bounds__(32 * T10_WARPS)
k_t10_curlcurl(const double *__restrict__ nodes, const int32_t *__restrict__ elems,
               int64_t M, Coef nu, double *__restrict__ ke) {
    __shared__ double sG[T10_WARPS][5][10][3];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t e = (int64_t)blockIdx.x * T10_WARPS + w;
    if (e >= M) return;
    const int32_t *el = elems + e * 10;
    double vol;
    t10_stage_grads(nodes, el, sG[w], lane, vol);
    const double sv = coef_at(nu, e, 0) * vol;
    for (int t = lane; t < 100; t += 32) {
        int a = t / 10, b = t - (t / 10) * 10;
        double blk[9];
#pragma unroll
        for (int v = 0; v < 9; ++v) blk[v] = 0.0;
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            const double wq = c_wq[q];
            double ga[3], gb[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                ga[c] = sG[w][q][a][c];
                gb[c] = sG[w][q][b][c];
            }
            const double dot = ga[0] * gb[0] + ga[1] * gb[1] + ga[2] * gb[2];
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    blk[c * 3 + d] += wq * ((c == d ? dot : 0.0) - ga[d] * gb[c]);
        }
        double *dst = ke + (e * 100 + t) * 9;
#pragma unroll
        for (int v = 0; v < 9; ++v) dst[v] = sv * blk[v];
    }
}

// Centroid strain and stress per element (Voigt xx, yy, zz, yz, xz, xy,
// engineering shears), elastic3d.py:171-185 and elastic_tet10.py:232-262:
// eps = B(G_c) u_e with G_c the physical gradients at the centroid (Keast
// point 0 for Tet10), sig = D (eps - alpha (T_c - T_ref) [1,1,1,0,0,0]) with
// the isotropic D, T_c the centroid temperature (per-element value, or the
// nodal field interpolated: corner mean for P1, N(centroid) for Tet10).
template <int NPE>
__global__ void __launch_bounds__(128)
k_elem_stress(const double *__restrict__ nodes, const int32_t *__restrict__ elems,
              int64_t M, const double *__restrict__ u, double lam, double mu,
              Coef temp, int thermal, double alpha, double tref,
              double *__restrict__ sig, double *__restrict__ eps) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= M) return;
    const int32_t *el = elems + e * NPE;
    Geo g;
    tet_geo(nodes, __ldg(el + 0), __ldg(el + 1), __ldg(el + 2), __ldg(el + 3), g);
    double ev[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int a = 0; a < NPE; ++a) {
        double G[3];
        if (NPE == 4) {
#pragma unroll
            for (int c = 0; c < 3; ++c)
                G[c] = a == 0 ? -(g.inv[0][c] + g.inv[1][c] + g.inv[2][c]) : g.inv[a - 1][c];
        } else {
#pragma unroll
            for (int j = 0; j < 3; ++j)
                G[j] = c_dNdxi[0][a][0] * g.inv[0][j] + c_dNdxi[0][a][1] * g.inv[1][j] +
                       c_dNdxi[0][a][2] * g.inv[2][j];
        }
        const int64_t n = __ldg(el + a);
        const double ux = __ldg(u + 3 * n), uy = __ldg(u + 3 * n + 1), uz = __ldg(u + 3 * n + 2);
        ev[0] += G[0] * ux;
        ev[1] += G[1] * uy;
        ev[2] += G[2] * uz;
        ev[3] += G[2] * uy + G[1] * uz;
        ev[4] += G[2] * ux + G[0] * uz;
        ev[5] += G[1] * ux + G[0] * uy;
    }
    double th = 0.0;
    if (thermal) {
        double Tc;
        if (temp.mode == CFEM_COEF_NODAL) {
            if (NPE == 4) {
                Tc = (((temp.v[__ldg(el)] + temp.v[__ldg(el + 1)]) + temp.v[__ldg(el + 2)]) +
                      temp.v[__ldg(el + 3)]) / 4.0;
            } else {
                Tc = 0.0;
#pragma unroll
                for (int s2 = 0; s2 < 10; ++s2) Tc += temp.v[__ldg(el + s2)] * c_N[0][s2];
            }
        } else {
            Tc = coef_at(temp, e, 0);
        }
        th = alpha * (Tc - tref);
    }
    double em[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) em[i] = ev[i] - (i < 3 ? th : 0.0);
    const double d0 = lam + 2.0 * mu;
    sig[e * 6 + 0] = d0 * em[0] + lam * em[1] + lam * em[2];
    sig[e * 6 + 1] = lam * em[0] + d0 * em[1] + lam * em[2];
    sig[e * 6 + 2] = lam * em[0] + lam * em[1] + d0 * em[2];
    sig[e * 6 + 3] = mu * em[3];
    sig[e * 6 + 4] = mu * em[4];
    sig[e * 6 + 5] = mu * em[5];
#pragma unroll
    for (int i = 0; i < 6; ++i) eps[e * 6 + i] = ev[i];
}

// ------------------------------------------------------------- reductions
template <int BS>
__global__ void k_reduce_vals(const int32_t *__restrict__ seg,
                              const int32_t *__restrict__ contrib, int64_t nnz,
                              const double *__restrict__ ke,
                              double *__restrict__ vals, int accumulate) {
    constexpr int B2 = BS * BS;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz;
         k += (int64_t)gridDim.x * blockDim.x) {
        double s[B2];
#pragma unroll
        for (int v = 0; v < B2; ++v) s[v] = 0.0;
        const int32_t t1 = seg[k + 1];
        for (int32_t t = seg[k]; t < t1; ++t) {
            const int64_t id = __ldg(contrib + t);
#pragma unroll
            for (int v = 0; v < B2; ++v) s[v] += __ldg(ke + id * B2 + v);
        }
        double *dst = vals + k * B2;
#pragma unroll
        for (int v = 0; v < B2; ++v) dst[v] = accumulate ? dst[v] + s[v] : s[v];
    }
}

template <int BS>
__global__ void k_reduce_rhs(const int32_t *__restrict__ diag,
                             const int32_t *__restrict__ seg,
                             const int32_t *__restrict__ contrib,
                             int64_t n_nodes, int npe,
                             const double *__restrict__ fe,
                             double *__restrict__ rhs, int accumulate) {
    const int per = npe * npe;
    for (int64_t a = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; a < n_nodes;
         a += (int64_t)gridDim.x * blockDim.x) {
        double s[BS];
#pragma unroll
        for (int c = 0; c < BS; ++c) s[c] = 0.0;
        const int32_t k = diag[a];
        if (k >= 0) {
            for (int32_t t = seg[k]; t < seg[k + 1]; ++t) {
                const int32_t id = contrib[t];
                const int32_t ee = id / per;
                const int32_t r = id - ee * per;
                const int32_t i = r / npe, j = r - (r / npe) * npe;
                if (i != j) continue;
#pragma unroll
                for (int c = 0; c < BS; ++c)
                    s[c] += fe[((int64_t)ee * npe + i) * BS + c];
            }
        }
#pragma unroll
        for (int c = 0; c < BS; ++c)
            rhs[a * BS + c] = accumulate ? rhs[a * BS + c] + s[c] : s[c];
    }
}


// ------------------------------------------------------------- batches
// Many independent meshes in one launch per pass: a job table gives each
// mesh's arrays and its offsets in the concatenated element / CSR / node
// ranges; a thread (P1), warp (Tet10) or CSR entry finds its job by binary
// search over the offsets.
struct AsmJob {
    const double *nodes;
    const int32_t *elems;
    const int32_t *seg, *contrib, *diag;
    double *vals, *rhs;
    Coef coef, load;
    int64_t e0, k0, a0;          // element, CSR entry and node offsets
    int64_t m, nnz, n_nodes;
};

__device__ __forceinline__ int find_job(const AsmJob *jobs, int nj, int64_t g, int which) {
    int lo = 0, hi = nj - 1;     // last job with offset <= g
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        const int64_t off = which == 0 ? jobs[mid].e0 : (which == 1 ? jobs[mid].k0 : jobs[mid].a0);
        if (off <= g) lo = mid; else hi = mid - 1;
    }
    return lo;
}

template <int OP>
__global__ void __launch_bounds__(128)
k_p1_scalar_batch(const AsmJob *__restrict__ jobs, int nj, int64_t M,
                  double *__restrict__ ke, double *__restrict__ fe) {
    const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (g >= M) return;
    const AsmJob &J = jobs[find_job(jobs, nj, g, 0)];
    p1_scalar_elem<OP>(J.nodes, J.elems, g - J.e0, J.coef, J.load, ke + g * 16,
                       fe ? fe + g * 4 : nullptr);
}

template <int OP, int W>
__global__ void __launch_bounds__(32 * W)
k_t10_scalar_batch(const AsmJob *__restrict__ jobs, int nj, int64_t M,
                   double *__restrict__ ke, double *__restrict__ fe) {
    __shared__ double sG[W][5][10][3];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t g = (int64_t)blockIdx.x * W + w;
    if (g >= M) return;
    const AsmJob &J = jobs[find_job(jobs, nj, g, 0)];
    t10_scalar_elem<OP>(J.nodes, J.elems, g - J.e0, J.coef, J.load, ke + g * 100,
                        fe ? fe + g * 10 : nullptr, sG[w], lane);
}

// Elements per block of the batched Tet10 kernel (one warp per element), a
// launch parameter chosen per context (cfem_ctx_set_param, autotuned).
template <int OP>
static int launch_t10_batch(int warps, int64_t M, cudaStream_t s, const AsmJob *jobs,
                            int nj, double *ke, double *fe) {
    switch (warps) {
        case 2:
            CFEM_LAUNCH((k_t10_scalar_batch<OP, 2>), grid_for(M, 2), 64, 0, s, jobs, nj, M, ke, fe);
            break;
        case 8:
            CFEM_LAUNCH((k_t10_scalar_batch<OP, 8>), grid_for(M, 8), 256, 0, s, jobs, nj, M, ke, fe);
            break;
        default:
            CFEM_LAUNCH((k_t10_scalar_batch<OP, 4>), grid_for(M, 4), 128, 0, s, jobs, nj, M, ke, fe);
    }
    return CFEM_OK;
}

__global__ void k_reduce_vals_batch(const AsmJob *__restrict__ jobs, int nj,
                                    int64_t K, int npe, const double *__restrict__ ke) {
    const int64_t per = (int64_t)npe * npe;
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < K;
         g += (int64_t)gridDim.x * blockDim.x) {
        const AsmJob &J = jobs[find_job(jobs, nj, g, 1)];
        const int64_t k = g - J.k0;
        const double *kj = ke + J.e0 * per;
        double s = 0.0;
        for (int32_t t = J.seg[k]; t < J.seg[k + 1]; ++t) s += __ldg(kj + __ldg(J.contrib + t));
        J.vals[k] = s;
    }
}

__global__ void k_reduce_rhs_batch(const AsmJob *__restrict__ jobs, int nj,
                                   int64_t A, int npe, const double *__restrict__ fe) {
    const int per = npe * npe;
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < A;
         g += (int64_t)gridDim.x * blockDim.x) {
        const AsmJob &J = jobs[find_job(jobs, nj, g, 2)];
        const int64_t a = g - J.a0;
        const double *fj = fe + J.e0 * npe;
        double s = 0.0;
        const int32_t k = J.diag[a];
        if (k >= 0) {
            for (int32_t t = J.seg[k]; t < J.seg[k + 1]; ++t) {
                const int32_t id = J.contrib[t];
                const int32_t ee = id / per, r = id - ee * per;
                const int32_t i = r / npe, jj = r - (r / npe) * npe;
                if (i == jj) s += fj[(int64_t)ee * npe + i];
            }
        }
        J.rhs[a] = s;
    }
}

static int check_coef(const cfem_coef *c, bool allow_qp, const char *what) {
    if (!c) return CFEM_OK;
    CFEM_CHECK(c->mode >= CFEM_COEF_CONST && c->mode <= CFEM_COEF_NODAL,
               CFEM_ERR_INVALID, "%s: unknown coefficient mode %d", what, c->mode);
    CFEM_CHECK(c->mode == CFEM_COEF_CONST || c->d_values, CFEM_ERR_INVALID,
               "%s: coefficient array is NULL", what);
    CFEM_CHECK(allow_qp || c->mode != CFEM_COEF_QP, CFEM_ERR_INVALID,
               "%s: per-quadrature-point values need a Tet10 operator", what);
    return CFEM_OK;
}

static int reduce_all(const cfem_pattern *p, int bs, const double *ke,
                      const double *fe, double *d_vals, double *d_rhs,
                      int accumulate, int num_sms, cudaStream_t s) {
    if (p->nnz > 0) {
        unsigned g = grid_for(p->nnz, 256);
        if (g > (unsigned)num_sms * 32) g = num_sms * 32;
        if (bs == 1)
            CFEM_LAUNCH(k_reduce_vals<1>, g, 256, 0, s, p->seg, p->contrib,
                        p->nnz, ke, d_vals, accumulate);
        else
            CFEM_LAUNCH(k_reduce_vals<3>, g, 256, 0, s, p->seg, p->contrib,
                        p->nnz, ke, d_vals, accumulate);
    }
    if (d_rhs && fe) {
        unsigned g = grid_for(p->n_nodes, 256);
        if (bs == 1)
            CFEM_LAUNCH(k_reduce_rhs<1>, g, 256, 0, s, p->diag, p->seg,
                        p->contrib, p->n_nodes, p->npe, fe, d_rhs, accumulate);
        else
            CFEM_LAUNCH(k_reduce_rhs<3>, g, 256, 0, s, p->diag, p->seg,
                        p->contrib, p->n_nodes, p->npe, fe, d_rhs, accumulate);
    }
    return CFEM_OK;
}

}  // namespace cfem

using namespace cfem;

extern "C" {

int cfem_assemble(cfem_ctx *ctx, const cfem_pattern *p, int32_t op,
                  const double *d_nodes, const int32_t *d_elems,
                  const cfem_coef *coef, const cfem_coef *load, double *d_vals,
                  double *d_rhs, int32_t accumulate, void *stream) {
    CFEM_API_BEGIN
    CFEM_CHECK(ctx && p && d_nodes && d_elems && d_vals, CFEM_ERR_INVALID,
               "cfem_assemble: NULL argument");
    const bool p1 = (op == CFEM_OP_P1_STIFF || op == CFEM_OP_P1_MASS);
    const bool ngrad = (op >= CFEM_OP_T10_NGRAD_X && op <= CFEM_OP_T10_NGRAD_Z);
    const bool t10 = (op == CFEM_OP_T10_STIFF || op == CFEM_OP_T10_MASS || ngrad);
    CFEM_CHECK(p1 || t10, CFEM_ERR_INVALID, "cfem_assemble: unknown op %d", op);
    CFEM_CHECK(p->npe == (p1 ? 4 : 10), CFEM_ERR_INVALID,
               "operator %d needs %d-node elements, pattern has %d", op,
               p1 ? 4 : 10, p->npe);
    CFEM_CHECK(!ngrad || !coef || coef->mode == CFEM_COEF_CONST ||
                   coef->mode == CFEM_COEF_ELEM,
               CFEM_ERR_INVALID, "coupling operators take a constant or per-element coefficient");
    CFEM_TRY(check_coef(coef, op == CFEM_OP_T10_STIFF, "coef"));
    CFEM_TRY(check_coef(load, op == CFEM_OP_T10_STIFF, "load"));
    CFEM_CHECK(!coef || coef->mode != CFEM_COEF_NODAL, CFEM_ERR_INVALID,
               "nodal coefficients are only accepted for temperature");
    CFEM_CHECK(!load || load->mode != CFEM_COEF_NODAL, CFEM_ERR_INVALID,
               "nodal coefficients are only accepted for temperature");
    CFEM_CHECK(((uintptr_t)d_elems & 15) == 0, CFEM_ERR_INVALID,
               "element array must be 16-byte aligned");
    CFEM_TRY(set_device(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t M = p->n_elems, npe = p->npe;
    if (M == 0) {
        if (p->nnz && !accumulate)
            CFEM_CUDA(cudaMemsetAsync(d_vals, 0, p->nnz * sizeof(double), s));
        if (d_rhs && !accumulate)
            CFEM_CUDA(cudaMemsetAsync(d_rhs, 0, p->n_nodes * sizeof(double), s));
        return CFEM_OK;
    }
    const bool want_rhs = d_rhs && (op == CFEM_OP_P1_STIFF || op == CFEM_OP_T10_STIFF);
    double *ke = nullptr, *fe = nullptr;
    CFEM_TRY(tmp_alloc(&ke, M * npe * npe, s));
    if (want_rhs) CFEM_TRY(tmp_alloc(&fe, M * npe, s));
    Coef kc = to_coef(coef), lc = to_coef(load);
    if (!coef) kc.c = 1.0;
    switch (op) {
        case CFEM_OP_P1_STIFF:
            CFEM_LAUNCH(k_p1_scalar<CFEM_OP_P1_STIFF>, grid_for(M, ctx->p1_threads),
                        ctx->p1_threads, 0,
                        s, d_nodes, d_elems, M, kc, lc, ke, fe);
            break;
        case CFEM_OP_P1_MASS:
            CFEM_LAUNCH(k_p1_scalar<CFEM_OP_P1_MASS>, grid_for(M, ctx->p1_threads),
                        ctx->p1_threads, 0,
                        s, d_nodes, d_elems, M, kc, lc, ke, nullptr);
            break;
        case CFEM_OP_T10_STIFF:
            CFEM_LAUNCH(k_t10_scalar<CFEM_OP_T10_STIFF>, grid_for(M, T10_WARPS),
                        32 * T10_WARPS, 0, s, d_nodes, d_elems, M, kc, lc, ke, fe);
            break;
        case CFEM_OP_T10_NGRAD_X:
            CFEM_LAUNCH(k_t10_scalar<CFEM_OP_T10_NGRAD_X>, grid_for(M, T10_WARPS),
                        32 * T10_WARPS, 0, s, d_nodes, d_elems, M, kc, lc, ke, nullptr);
            break;
        case CFEM_OP_T10_NGRAD_Y:
            CFEM_LAUNCH(k_t10_scalar<CFEM_OP_T10_NGRAD_Y>, grid_for(M, T10_WARPS),
                        32 * T10_WARPS, 0, s, d_nodes, d_elems, M, kc, lc, ke, nullptr);
            break;
        case CFEM_OP_T10_NGRAD_Z:
            CFEM_LAUNCH(k_t10_scalar<CFEM_OP_T10_NGRAD_Z>, grid_for(M, T10_WARPS),
                        32 * T10_WARPS, 0, s, d_nodes, d_elems, M, kc, lc, ke, nullptr);
            break;
        default:
            CFEM_LAUNCH(k_t10_scalar<CFEM_OP_T10_MASS>, grid_for(M, T10_WARPS),
                        32 * T10_WARPS, 0, s, d_nodes, d_elems, M, kc, lc, ke,
                        nullptr);
    }
    // Mass operators carry no load: leave d_rhs alone unless overwriting.
    if (d_rhs && !want_rhs && !accumulate)
        CFEM_CUDA(cudaMemsetAsync(d_rhs, 0, p->n_nodes * sizeof(double), s));
    int st = reduce_all(p, 1, ke, want_rhs ? fe : nullptr, d_vals,
                        want_rhs ? d_rhs : nullptr, accumulate, ctx->num_sms, s);
    tmp_free(ke, s);
    tmp_free(fe, s);
    return st;
    CFEM_API_END
}


int cfem_assemble_batch(cfem_ctx *ctx, int32_t op, const cfem_assembly_job *jobs,
                        int32_t n_jobs, void *stream) {
    CFEM_API_BEGIN
    CFEM_CHECK(ctx && jobs && n_jobs > 0, CFEM_ERR_INVALID,
               "cfem_assemble_batch: bad args");
    const bool p1 = (op == CFEM_OP_P1_STIFF || op == CFEM_OP_P1_MASS);
    const bool t10 = (op == CFEM_OP_T10_STIFF || op == CFEM_OP_T10_MASS);
    CFEM_CHECK(p1 || t10, CFEM_ERR_INVALID, "cfem_assemble_batch: scalar operators only");
    const int npe = p1 ? 4 : 10;
    const bool stiff = (op == CFEM_OP_P1_STIFF || op == CFEM_OP_T10_STIFF);
    CFEM_TRY(set_device(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t per = (int64_t)npe * npe;
    // Staging is bounded: jobs are processed in groups of at most ~256 M
    // element-matrix entries (2 GiB).
    const int64_t stage_cap = (int64_t)256 << 20;
    int i0 = 0;
    while (i0 < n_jobs) {
        std::vector<AsmJob> hj;
        int64_t M = 0, K = 0, A = 0;
        int i1 = i0;
        bool rhs = false;
        while (i1 < n_jobs) {
            const cfem_assembly_job &J = jobs[i1];
            CFEM_CHECK(J.pattern && J.d_nodes && J.d_elems && J.d_vals, CFEM_ERR_INVALID,
                       "job %d: missing arrays", i1);
            CFEM_CHECK(J.pattern->npe == npe, CFEM_ERR_INVALID,
                       "job %d: pattern has %d nodes per element, operator needs %d",
                       i1, J.pattern->npe, npe);
            CFEM_CHECK(((uintptr_t)J.d_elems & 15) == 0, CFEM_ERR_INVALID,
                       "job %d: element array must be 16-byte aligned", i1);
            CFEM_TRY(check_coef(&J.coef, op == CFEM_OP_T10_STIFF, "coef"));
            CFEM_TRY(check_coef(&J.load, op == CFEM_OP_T10_STIFF, "load"));
            const int64_t m = J.pattern->n_elems;
            if (i1 > i0 && (M + m) * per > stage_cap) break;
            AsmJob a;
            a.nodes = J.d_nodes;
            a.elems = J.d_elems;
            a.seg = J.pattern->seg;
            a.contrib = J.pattern->contrib;
            a.diag = J.pattern->diag;
            a.vals = J.d_vals;
            a.rhs = J.d_rhs;
            a.coef = to_coef(&J.coef);
            a.load = to_coef(&J.load);
            a.e0 = M;
            a.k0 = K;
            a.a0 = A;
            a.m = m;
            a.nnz = J.pattern->nnz;
            a.n_nodes = J.pattern->n_nodes;
            rhs = rhs || (J.d_rhs != nullptr);
            CFEM_CHECK(!rhs || J.d_rhs, CFEM_ERR_INVALID,
                       "job %d: either every job of a batch has a load vector or none", i1);
            M += m;
            K += a.nnz;
            A += a.n_nodes;
            hj.push_back(a);
            ++i1;
        }
        const int nj = (int)hj.size();
        AsmJob *d_jobs = nullptr;
        double *ke = nullptr, *fe = nullptr;
        CFEM_TRY(tmp_alloc(&d_jobs, nj, s));
        CFEM_CUDA(cudaMemcpyAsync(d_jobs, hj.data(), nj * sizeof(AsmJob),
                                  cudaMemcpyHostToDevice, s));
        CFEM_TRY(tmp_alloc(&ke, M * per, s));
        const bool want_rhs = rhs && stiff;
        if (want_rhs) CFEM_TRY(tmp_alloc(&fe, M * npe, s));
        if (M > 0) {
            if (op == CFEM_OP_P1_STIFF)
                CFEM_LAUNCH(k_p1_scalar_batch<CFEM_OP_P1_STIFF>, grid_for(M, ctx->p1_threads),
                            ctx->p1_threads, 0, s,
                            d_jobs, nj, M, ke, fe);
            else if (op == CFEM_OP_P1_MASS)
                CFEM_LAUNCH(k_p1_scalar_batch<CFEM_OP_P1_MASS>, grid_for(M, ctx->p1_threads),
                            ctx->p1_threads, 0, s,
                            d_jobs, nj, M, ke, nullptr);
            else if (op == CFEM_OP_T10_STIFF)
                CFEM_TRY(launch_t10_batch<CFEM_OP_T10_STIFF>(ctx->t10_warps, M, s, d_jobs,
                                                             nj, ke, fe));
            else
                CFEM_TRY(launch_t10_batch<CFEM_OP_T10_MASS>(ctx->t10_warps, M, s, d_jobs,
                                                            nj, ke, nullptr));
        }
        unsigned g = grid_for(K, 256);
        if (g > (unsigned)ctx->num_sms * 32) g = ctx->num_sms * 32;
        if (K > 0) CFEM_LAUNCH(k_reduce_vals_batch, g, 256, 0, s, d_jobs, nj, K, npe, ke);
        if (rhs) {
            if (want_rhs) {
                g = grid_for(A, 256);
                if (g > (unsigned)ctx->num_sms * 32) g = ctx->num_sms * 32;
                CFEM_LAUNCH(k_reduce_rhs_batch, g, 256, 0, s, d_jobs, nj, A, npe, fe);
            } else {
                for (int j = 0; j < nj; ++j)
                    CFEM_CUDA(cudaMemsetAsync(hj[j].rhs, 0, hj[j].n_nodes * sizeof(double), s));
            }
        }
        tmp_free(ke, s);
        tmp_free(fe, s);
        tmp_free(d_jobs, s);
        i0 = i1;
    }
    return CFEM_OK;
    CFEM_API_END
}

int cfem_assemble_elastic(cfem_ctx *ctx, const cfem_pattern *p, int32_t op,
                          const double *d_nodes, const int32_t *d_elems,
                          double E, double nu, const cfem_coef *body3,
                          const cfem_coef *temp, double alpha, double T_ref,
                          double *d_vals, double *d_rhs, int32_t accumulate,
                          void *stream) {
    CFEM_API_BEGIN
    CFEM_CHECK(ctx && p && d_nodes && d_elems && d_vals, CFEM_ERR_INVALID,
               "cfem_assemble_elastic: NULL argument");
    CFEM_CHECK(op == CFEM_OP_P1_ELAST || op == CFEM_OP_T10_ELAST,
               CFEM_ERR_INVALID, "cfem_assemble_elastic: unknown op %d", op);
    const bool t10 = op == CFEM_OP_T10_ELAST;
    CFEM_CHECK(p->npe == (t10 ? 10 : 4), CFEM_ERR_INVALID,
               "operator %d needs %d-node elements, pattern has %d", op,
               t10 ? 10 : 4, p->npe);
    CFEM_CHECK(nu > -1.0 && nu < 0.5, CFEM_ERR_INVALID,
               "Poisson ratio %g outside (-1, 0.5)", nu);
    for (int c = 0; c < 3 && body3; ++c) {
        CFEM_TRY(check_coef(&body3[c], t10, "body"));
        CFEM_CHECK(body3[c].mode != CFEM_COEF_NODAL, CFEM_ERR_INVALID,
                   "body force cannot be nodal");
    }
    CFEM_TRY(check_coef(temp, t10, "temperature"));
    CFEM_CHECK(((uintptr_t)d_elems & 15) == 0, CFEM_ERR_INVALID,
               "element array must be 16-byte aligned");
    CFEM_TRY(set_device(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t M = p->n_elems, npe = p->npe;
    if (M == 0) {
        if (p->nnz && !accumulate)
            CFEM_CUDA(cudaMemsetAsync(d_vals, 0, p->nnz * 9 * sizeof(double), s));
        if (d_rhs && !accumulate)
            CFEM_CUDA(cudaMemsetAsync(d_rhs, 0, p->n_nodes * 3 * sizeof(double), s));
        return CFEM_OK;
    }
    // constitutive_3d (elastic3d.py:26-34)
    const double lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double mu = E / (2.0 * (1.0 + nu));
    Coef b[3];
    for (int c = 0; c < 3; ++c) b[c] = to_coef(body3 ? &body3[c] : nullptr);
    Coef tc = to_coef(temp);
    const double *tnodal = nullptr;
    if (temp && temp->mode == CFEM_COEF_NODAL) {
        tnodal = temp->d_values;
        tc = Coef{nullptr, 0.0, CFEM_COEF_CONST};
    }
    const int thermal = (temp != nullptr && alpha != 0.0) ? 1 : 0;
    double *ke = nullptr, *fe = nullptr;
    CFEM_TRY(tmp_alloc(&ke, M * npe * npe * 9, s));
    if (d_rhs) CFEM_TRY(tmp_alloc(&fe, M * npe * 3, s));
    if (t10)
        CFEM_LAUNCH(k_t10_elastic, grid_for(M, T10_WARPS), 32 * T10_WARPS, 0, s,
                    d_nodes, d_elems, M, lam, mu, b[0], b[1], b[2], tc, tnodal,
                    thermal, alpha, T_ref, ke, fe);
    else
        CFEM_LAUNCH(k_p1_elastic, grid_for(M, 128), 128, 0, s, d_nodes, d_elems,
                    M, lam, mu, b[0], b[1], b[2], tc, tnodal, thermal, alpha, T_ref,
                    ke, fe);
    int st = reduce_all(p, 3, ke, fe, d_vals, d_rhs, accumulate, ctx->num_sms, s);
    tmp_free(ke, s);
    tmp_free(fe, s);
    return st;
    CFEM_API_END
}

int cfem_element_stress(cfem_ctx *ctx, const double *d_nodes, const int32_t *d_elems,
                        int64_t n_elems, int32_t npe, const double *d_u, double E,
                        double nu, const cfem_coef *temp, double alpha, double T_ref,
                        double *d_sig, double *d_eps, void *stream) {
    CFEM_API_BEGIN
    CFEM_CHECK(ctx && d_nodes && d_elems && d_u && d_sig && d_eps && n_elems >= 0 &&
                   (npe == 4 || npe == 10),
               CFEM_ERR_INVALID, "cfem_element_stress: bad args");
    CFEM_CHECK(E > 0.0 && nu > -1.0 && nu < 0.5, CFEM_ERR_INVALID,
               "material constants out of range (E %g, nu %g)", E, nu);
    CFEM_TRY(check_coef(temp, false, "temperature"));
    if (n_elems == 0) return CFEM_OK;
    CFEM_TRY(set_device(ctx->device));
    const double lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double mu = E / (2.0 * (1.0 + nu));
    const int thermal = (temp != nullptr && alpha != 0.0) ? 1 : 0;
    Coef tc = to_coef(temp);
    cudaStream_t s = (cudaStream_t)stream;
    if (npe == 4)
        CFEM_LAUNCH(k_elem_stress<4>, grid_for(n_elems, 128), 128, 0, s, d_nodes, d_elems,
                    n_elems, d_u, lam, mu, tc, thermal, alpha, T_ref, d_sig, d_eps);
    else
        CFEM_LAUNCH(k_elem_stress<10>, grid_for(n_elems, 128), 128, 0, s, d_nodes, d_elems,
                    n_elems, d_u, lam, mu, tc, thermal, alpha, T_ref, d_sig, d_eps);
    return CFEM_OK;
    CFEM_API_END
}

int cfem_assemble_curlcurl(cfem_ctx *ctx, const cfem_pattern *p,
                           const double *d_nodes, const int32_t *d_elems,
                           cfem_coef nu, double *d_vals, int accumulate,
                           void *stream) {
    CFEM_API_BEGIN
    CFEM_CHECK(ctx && p && d_nodes && d_elems && d_vals, CFEM_ERR_INVALID,
               "cfem_assemble_curlcurl: NULL argument");
    CFEM_CHECK(p->npe == 10, CFEM_ERR_INVALID,
               "curl-curl needs 10-node elements, pattern has %d", p->npe);
    CFEM_CHECK(nu.mode == CFEM_COEF_CONST || (nu.mode == CFEM_COEF_ELEM && nu.d_values),
               CFEM_ERR_INVALID, "nu must be constant or per element");
    CFEM_CHECK(((uintptr_t)d_elems & 15) == 0, CFEM_ERR_INVALID,
               "element array must be 16-byte aligned");
    CFEM_TRY(set_device(ctx->device));
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t M = p->n_elems;
    if (M == 0) {
        if (p->nnz && !accumulate)
            CFEM_CUDA(cudaMemsetAsync(d_vals, 0, p->nnz * 9 * sizeof(double), s));
        return CFEM_OK;
    }
    double *ke = nullptr;
    CFEM_TRY(tmp_alloc(&ke, M * 100 * 9, s));
    CFEM_LAUNCH(k_t10_curlcurl, grid_for(M, T10_WARPS), 32 * T10_WARPS, 0, s,
                d_nodes, d_elems, M, to_coef(&nu), ke);
    int st = reduce_all(p, 3, ke, nullptr, d_vals, nullptr, accumulate, ctx->num_sms, s);
    tmp_free(ke, s);
    return st;
    CFEM_API_END
}

}  // extern "C"
