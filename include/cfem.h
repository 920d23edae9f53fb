/*
 * cfem.h - C ABI of libcfem, the B200 (sm_100a) implementation of
 * CloudFEM's tetrahedral assembly -> CSR -> sparse-solve hot path.
 *
 * The reference (zhangkalin627-svg/CloudFEM) is pure Python: every entry
 * point below replaces the per-element Python loop plus SciPy call that
 * the cited reference function runs. All pointers named d_* are device
 * pointers on the context's device; every other pointer is host memory.
 * Calls are asynchronous on the given stream (NULL = legacy default
 * stream) unless the comment says they synchronise.
 *
 * Index conventions follow the reference: node ids are 0-based, element
 * connectivity is row-major (n_elems, npe) with npe = 4 (Tet4,
 * cloudfem/mesh/tet_mesh.py:11) or 10 (Tet10, cloudfem/mesh/tet10_mesh.py:36,
 * local slots 4..9 on EDGES (0,1),(1,2),(2,0),(0,3),(1,3),(2,3)); vector
 * problems interleave DOFs as 3*node + component
 * (cloudfem/physics/elastic3d.py:80-85).
 *
 * Errors: every function returns a CFEM_* status; cfem_last_error()
 * returns the calling thread's message for the last failure.
 */
#ifndef CFEM_H
#define CFEM_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define CFEM_API __attribute__((visibility("default")))
#else
#define CFEM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum {
    CFEM_OK = 0,
    CFEM_ERR_INVALID = 1,       /* bad argument (the reference's ValueError) */
    CFEM_ERR_CUDA = 2,          /* CUDA runtime failure                      */
    CFEM_ERR_NOMEM = 3,         /* device allocation failed                  */
    CFEM_ERR_NOT_CONVERGED = 4, /* iteration cap or stagnation               */
    CFEM_ERR_BREAKDOWN = 5,     /* p'Ap <= 0, singular block, non-finite     */
    CFEM_ERR_TIMEOUT = 6,       /* a bounded device-side wait gave up        */
    CFEM_ERR_UNSUPPORTED = 7,   /* device is not sm_100 / feature missing    */
    CFEM_SLOT_RUNNING = -1      /* cfem_pcg_slots_poll: still iterating      */
};

/* Element operators of cfem_assemble (values are block bs x bs per node pair). */
enum {
    CFEM_OP_P1_STIFF = 1,   /* tet_poisson.py:35-69   k V G G^T, load f V/4     */
    CFEM_OP_P1_MASS = 2,    /* tet_heat.py:72-94      rho V/20 (1+d_ij)         */
    CFEM_OP_T10_STIFF = 3,  /* tet10.py:138-165       Keast-5 k G G^T, f N      */
    CFEM_OP_T10_MASS = 4,   /* tet10.py:229-249       rho V MASS_REF            */
    CFEM_OP_P1_ELAST = 5,   /* elastic3d.py:105-169   V B^T D B, body, thermal  */
    CFEM_OP_T10_ELAST = 6,  /* elastic_tet10.py:135-192 Keast-5 B^T D B, ...    */
    CFEM_OP_T10_CURLCURL = 7, /* em3d_tet10.py:205-210  nu V sum_q w_q curl.curl */
    CFEM_OP_T10_NGRAD_X = 8,  /* em3d_tet10.py:225-227  sigma V sum_q w_q N_p dN_j/dx */
    CFEM_OP_T10_NGRAD_Y = 9,  /*   same, d/dy (A-V coupling block G, one       */
    CFEM_OP_T10_NGRAD_Z = 10  /*   component of the A DOF per op)              */
};

/* How a coefficient array is sampled. */
enum {
    CFEM_COEF_CONST = 0,    /* one scalar (field `constant`)                */
    CFEM_COEF_ELEM = 1,     /* (n_elems,) at element centroids             */
    CFEM_COEF_QP = 2,       /* (n_elems, 5) at the Keast-5 points          */
    CFEM_COEF_NODAL = 3     /* (n_nodes,) nodal field, interpolated         */
};

typedef struct cfem_coef {
    const double *d_values; /* NULL for CFEM_COEF_CONST                   */
    double constant;
    int32_t mode;
    int32_t pad_;
} cfem_coef;

/* Solver precision modes. */
enum {
    CFEM_SOLVE_FP64 = 0,    /* plain FP64 Jacobi-PCG                        */
    CFEM_SOLVE_MIXED = 1    /* FP32 PCG + FP64 residual/update/final dot   */
};
enum {
    CFEM_PRECOND_JACOBI = 0, /* point Jacobi on the diagonal               */
    CFEM_PRECOND_BLOCK = 1   /* bs x bs nodal block Jacobi                 */
};

/* One sparse SPD system for cfem_pcg_solve. The matrix is block CSR with
 * bs x bs row-major blocks (bs = 1 is plain CSR). Dirichlet DOFs are given
 * by `d_fixed` (1 = fixed) and hold their value in `d_x` on entry; the
 * solve is then the reference's elimination (tet_poisson.py:72-110,
 * elastic3d.py:192-233): A_ff x_f = b_f - A_fD x_D. */
typedef struct cfem_linsys {
    int64_t n_rows;          /* block rows                                  */
    int32_t bs;              /* 1 or 3                                      */
    int32_t precond;         /* CFEM_PRECOND_*                              */
    const int32_t *d_row_ptr;
    const int32_t *d_col;
    const double *d_vals64;  /* FP64 values (required)                      */
    const float *d_vals32;   /* CFEM_SOLVE_MIXED: FP32 difference-form copy
                                from cfem_mixed_matrix; else NULL           */
    const double *d_b;       /* right-hand side, n_rows*bs                  */
    double *d_x;             /* in: guess + Dirichlet values; out: solution */
    const uint8_t *d_fixed;  /* n_rows*bs mask, or NULL                     */
    double rtol;             /* ||b - A x||_free <= rtol * ||b_lift||_free  */
    int32_t max_iter;
    int32_t mode;            /* CFEM_SOLVE_*                                */
    double reliable_delta;   /* mixed: replace r when it fell by this factor
                                since the last replacement (0 -> 0.1)       */
    int32_t max_stall;       /* true-residual replacements without a 4x
                                gain before giving up (0 -> 8)              */
    int32_t history_cap;     /* entries of d_history (0 = none)             */
    double *d_history;       /* (iteration, relres) at every FP64 residual  */
} cfem_linsys;

typedef struct cfem_solve_stats {
    int32_t status;          /* CFEM_OK / NOT_CONVERGED / BREAKDOWN        */
    int32_t iterations;
    int32_t residual_updates;/* FP64 true-residual replacements            */
    int32_t pad_;
    double relres;           /* final ||r||/||b_lift|| (FP64, true residual)*/
    double bnorm;
    double kernel_ms;        /* device time of the whole solve (the same
                                value in every record of a batch)          */
    double spmv_ms;          /* graph scheduler: mean device time of one
                                SpMV-phase launch (CUDA events inside the
                                replayed graphs), else 0                    */
    int32_t spmv_samples;    /* launches averaged into spmv_ms              */
    int32_t pad2_;
} cfem_solve_stats;

typedef struct cfem_ctx cfem_ctx;
typedef struct cfem_pattern cfem_pattern;

/* ---- library / context ------------------------------------------------- */
CFEM_API const char *cfem_last_error(void);
CFEM_API int cfem_version(void);
/* Creates a context on `device` (must be compute capability 10.x). */
CFEM_API int cfem_ctx_create(int device, cfem_ctx **out);
CFEM_API int cfem_ctx_destroy(cfem_ctx *ctx);
/* How cfem_pcg_solve runs its iterations:
 * PERSISTENT    - one cooperative launch, grid barrier between phases
 *                 (lowest latency when the whole batch fits in one wave);
 * GRAPH         - per-phase kernels with a warp per row chunk (direction,
 *                 SpMV, reduction, update, reduction per iteration); the
 *                 whole solve is ONE CUDA graph launch whose device-side
 *                 WHILE node repeats 2-iteration bodies until no system is
 *                 active (no host polling);
 * GRAPH_POLLED  - the same kernels replayed from plain graphs of 16
 *                 iterations, the host polling convergence once per replay
 *                 (every launch visible to per-launch profilers);
 * AUTO          - PERSISTENT when all row chunks fit in one resident wave,
 *                 else GRAPH (default). */
enum { CFEM_SCHED_AUTO = 0, CFEM_SCHED_PERSISTENT = 1, CFEM_SCHED_GRAPH = 2,
       CFEM_SCHED_GRAPH_POLLED = 3 };
CFEM_API int cfem_ctx_set_scheduler(cfem_ctx *ctx, int scheduler);
/* The library's device memory (patterns, solver workspaces, sort buffers)
 * comes from one stream-ordered pool per GPU that keeps what it has mapped,
 * so repeated assemblies and solves do not map and unmap pages. This waits
 * for the device, returns all but `keep_bytes` of the pool's unused memory
 * to the driver and reports the bytes still reserved (NULL: not wanted).
 * No counterpart in the reference (SciPy allocates host memory per call). */
CFEM_API int cfem_ctx_trim(cfem_ctx *ctx, uint64_t keep_bytes,
                           uint64_t *reserved_bytes);
/* Launch parameters of a context, chosen by the autotuner
 * (cloudfem_b200/autotune.py) or by hand; no counterpart in the reference.
 * T10_WARPS: Tet10 elements (one warp each) per block of the batched element
 * kernel, 2, 4 (default) or 8. P1_THREADS: threads (one element each) per
 * block of the P1 element kernels, 32, 64 or 128 (default). GRAPH_ITERS:
 * iterations per body of the graph scheduler's solve loop, 1, 2 (default),
 * 4, 8 or 16 (longer bodies: fewer loop-condition launches, more work past
 * convergence). PDL: 1 (default) captures the solve graphs' kernels as
 * programmatic dependent launches (launch processing overlaps the previous
 * kernel's drain), 0 as plain launches. SPMV_STAGE: how the graph
 * scheduler's SpMV reads its working copy of the matrix: 1 streams each
 * scalar work entry's span through two shared-memory windows of about 4 KB
 * per warp with 1-D bulk copies (TMA) and loads 3x3 blocks into registers,
 * 2 streams 3x3 blocks through shared memory too, 0 loads both into
 * registers, 3 stores scalar rows and 3x3 block rows in the sliced-ELL
 * layout (windows of 256 rows sorted by length and cut into slices: 32
 * scalar rows, one per lane, or 32 / SELL3_LANES block rows; coalesced
 * slot-major loads), 4 (default) picks per precision and block size what
 * measured fastest: sliced ELL for FP64 scalar rows and for 3x3 blocks, the
 * staged windows for FP32 scalar rows.
 * BARRIER_TIMEOUT_US: how long (microseconds, 1 .. 60e6; default 4e6) a
 * block of the persistent scheduler waits at its grid barrier before it
 * gives up; the solve then ends with CFEM_ERR_TIMEOUT and the context stays
 * usable. BARRIER_HOLD: fault injection for that path (0 default, or 1):
 * the barrier counts one phantom block that never arrives, so every wait
 * runs to the limit; no other waits of the library are affected. Both are
 * read when a solve plan is created. SELL_SORT (SpMV staging 3): 1
 * (default) sorts each window of 256 rows by length before cutting it into
 * slices of 32 (less padding), 0 keeps the rows in order (neighbouring
 * rows in a slice: gathers of p that share cache lines); 3x3 solve slots
 * read it again at each assignment, and their room assumes sorted windows
 * (an unsorted layout that does not fit is refused). SELL3_LANES
 * (SpMV staging 3, 3x3 blocks): lanes that share one block row, each over
 * every L-th block of it (1, 2 or 4 (default); a slice holds 32 / L block
 * rows). SELL3_STAGED: 1 streams each slice's steps through a ring of
 * three shared-memory stages filled by 1-D bulk copies (the first issued
 * before the kernel waits for its predecessor), 0 loads them into
 * registers, 2 (default) streams FP32 slices and loads FP64 ones (the
 * faster of the two measured for each). SLOT_SELL3: solve slots
 * (cfem_pcg_slots_*) of 3x3 systems store them in the sliced ELL (1,
 * default; room for rows of up to 96 blocks, the layout built when a
 * system is assigned, a system needing more refused) or in the entry-major
 * copy (0); read when the slots are created. get returns -1 for an unknown
 * parameter. */
enum { CFEM_PARAM_T10_WARPS = 1, CFEM_PARAM_P1_THREADS = 2, CFEM_PARAM_GRAPH_ITERS = 3,
       CFEM_PARAM_PDL = 4, CFEM_PARAM_SPMV_STAGE = 5, CFEM_PARAM_BARRIER_TIMEOUT_US = 6,
       CFEM_PARAM_BARRIER_HOLD = 7, CFEM_PARAM_SELL_SORT = 8, CFEM_PARAM_SELL3_LANES = 9,
       CFEM_PARAM_SELL3_STAGED = 10, CFEM_PARAM_SLOT_SELL3 = 11 };
CFEM_API int cfem_ctx_set_param(cfem_ctx *ctx, int param, int value);
CFEM_API int cfem_ctx_get_param(const cfem_ctx *ctx, int param);
/* Number of kernels this library launched through `ctx` so far. */
CFEM_API int64_t cfem_ctx_launch_count(const cfem_ctx *ctx);

/* ---- sparsity pattern (replaces sp.coo_matrix(...).tocsr() structure) ---
 * Builds the node-level CSR of all (el[i], el[j]) pairs by a stable radix
 * sort of (row, col) keys followed by a unique pass, so indices are sorted
 * and canonical like SciPy's (e.g. tet_poisson.py:68, tet10.py:162), plus
 * the per-entry contribution lists (sorted by element id) used by the
 * deterministic segmented reduction in cfem_assemble. Synchronises. */
CFEM_API int cfem_pattern_create(cfem_ctx *ctx, const int32_t *d_elems,
                        int64_t n_elems, int32_t npe, int64_t n_nodes,
                        void *stream, cfem_pattern **out);
CFEM_API int cfem_pattern_destroy(cfem_pattern *p);
CFEM_API int cfem_pattern_info(const cfem_pattern *p, int64_t *n_nodes,
                      int64_t *nnz);
/* Device pointers of the node-level CSR (owned by the pattern). */
CFEM_API int cfem_pattern_node_csr(const cfem_pattern *p, const int32_t **d_row_ptr,
                          const int32_t **d_col);
/* Expands the node pattern to the scalar DOF CSR of a bs-DOF problem:
 * d_indptr (n_nodes*bs+1), d_indices (nnz*bs*bs). */
CFEM_API int cfem_pattern_expand(const cfem_pattern *p, int32_t bs, int32_t *d_indptr,
                        int32_t *d_indices, void *stream);
/* Block values (nnz*bs*bs, block-major) -> scalar CSR value order: the
 * csr_matrix the reference's assemble_elasticity_* return
 * (elastic3d.py:188, elastic_tet10.py:208-210), built from device blocks. */
CFEM_API int cfem_block_to_csr(const cfem_pattern *p, int32_t bs,
                      const double *d_bvals, double *d_vals, void *stream);

/* ---- element assembly ---------------------------------------------------
 * Replaces the element loops of assemble (tet_poisson.py:35-69),
 * assemble_mass_tet (tet_heat.py:72-94), assemble_tet10 (tet10.py:138-165)
 * and assemble_mass_tet10 (tet10.py:229-249), and the scalar blocks of
 * assemble_tet10_av (em3d_tet10.py:172-264) through the NGRAD operators.
 * Computes every element matrix (one thread per P1 element, one warp per
 * Tet10 element with shape gradients staged in shared memory) and reduces
 * them into d_vals in element order per CSR entry (deterministic, no
 * atomics). d_vals has nnz*bs*bs entries (bs = 3 for the *_ELAST ops).
 * `coef` is k / rho_cp; `load` the scalar source f (STIFF ops). Loads go
 * into d_rhs (n_nodes*bs; NULL to skip). If `accumulate` is 1 the results
 * are added to d_vals / d_rhs, else they overwrite them. */
CFEM_API int cfem_assemble(cfem_ctx *ctx, const cfem_pattern *p, int32_t op,
                  const double *d_nodes, const int32_t *d_elems,
                  const cfem_coef *coef, const cfem_coef *load,
                  double *d_vals, double *d_rhs, int32_t accumulate,
                  void *stream);
/* One mesh of a batched scalar assembly (cfem_assemble_batch). */
typedef struct cfem_assembly_job {
    const cfem_pattern *pattern;   /* the mesh's pattern (cfem_pattern_create) */
    const double *d_nodes;
    const int32_t *d_elems;
    cfem_coef coef;                /* k or rho_cp                              */
    cfem_coef load;                /* f (stiffness operators)                  */
    double *d_vals;                /* nnz values, overwritten                  */
    double *d_rhs;                 /* n_nodes, overwritten; NULL in every job
                                      of the batch to skip                     */
} cfem_assembly_job;

/* Assembles many independent meshes with one launch per pass (elements of
 * all meshes, then CSR entries of all meshes, then loads), the batched
 * form of cfem_assemble for the scalar operators (tet_poisson.py:35-69,
 * tet10.py:138-165, tet_heat.py:72-94, tet10.py:229-249). Element-matrix
 * staging is bounded to about 2 GiB per pass group. */
CFEM_API int cfem_assemble_batch(cfem_ctx *ctx, int32_t op,
                                 const cfem_assembly_job *jobs, int32_t n_jobs,
                                 void *stream);

/* Tet10 nodal curl-curl operator (CFEM_OP_T10_CURLCURL), replacing the
 * element loop of em3d_tet10.py:196-210 and _assemble_curl_curl_tet10_nu
 * (:746-771): 3x3 block (a, b) = nu_e V sum_q w_q ((g_a . g_b) I - g_b g_a^T)
 * with g = G_q (grad N x e_m . grad N x e_n summed over curl components),
 * node-major DOF 3 p + m, into d_vals (nnz * 9) of a bs-3 view of the node
 * pattern. nu: CFEM_COEF_CONST or CFEM_COEF_ELEM. accumulate: add. */
CFEM_API int cfem_assemble_curlcurl(cfem_ctx *ctx, const cfem_pattern *p,
                                    const double *d_nodes, const int32_t *d_elems,
                                    cfem_coef nu, double *d_vals, int accumulate,
                                    void *stream);

/* Centroid strain and stress per element (elastic3d.py:171-185,
 * elastic_tet10.py:232-262): d_sig, d_eps (n_elems * 6, Voigt xx yy zz yz
 * xz xy with engineering shears) from the nodal displacement d_u (3 N,
 * node-major), isotropic E, nu, and an optional temperature (per-element
 * centroid values CFEM_COEF_ELEM, or a nodal field CFEM_COEF_NODAL
 * interpolated at the centroid; NULL or alpha 0: no thermal strain). */
CFEM_API int cfem_element_stress(cfem_ctx *ctx, const double *d_nodes,
                                 const int32_t *d_elems, int64_t n_elems, int32_t npe,
                                 const double *d_u, double E, double nu,
                                 const cfem_coef *temp, double alpha, double T_ref,
                                 double *d_sig, double *d_eps, void *stream);

/* Boundary-face geometry (tet_heat.py:123-134, tet10.py:354-360): for each
 * of n_faces faces (npf = 3 or 6 node ids, int64; the first three are the
 * corners) the corner triangle's area d_area[f] = |e1 x e2| / 2 and, if
 * d_pts is given, its nq (1..8) quadrature points d_pts[(f nq + q) 3 + d]
 * = sum_c d_bary[q][c] x_c (nq = 1: the centroid (x0 + x1 + x2) / 3). */
CFEM_API int cfem_face_geometry(cfem_ctx *ctx, int32_t npf, int64_t n_faces,
                                const int64_t *d_faces, const double *d_nodes, int32_t nq,
                                const double *d_bary, double *d_pts, double *d_area,
                                void *stream);
/* Boundary-face integrals (Neumann / traction loads, Robin terms;
 * tet_heat.py:136-172, tet10.py:362-464, elastic3d.py:171-186,
 * elastic_tet10.py:192-205). Per face, with the rule's weights d_w[q],
 * shape values d_shape[q][a] and mass tables d_mt[q][a][b]:
 *   d_F[node_a ncomp + c] += A sum_q d_shape[q][a] (w_q d_load[(f nq + q) ncomp + c])
 *   d_vals[pos(node_a, node_b)] += A sum_q d_mt[q][a][b] (w_q d_h[f nq + q])
 * where pos is the entry's position in the node pattern (d_row_ptr, d_col,
 * n_nodes rows, sorted columns). Either part may be skipped (d_load or d_h
 * NULL). Contributions to one node or entry are summed in face order and
 * added once (stable sort by key), so results are bitwise reproducible.
 * CFEM_ERR_INVALID if a face pair is outside the pattern (nothing added). */
CFEM_API int cfem_face_integrate(cfem_ctx *ctx, int32_t npf, int64_t n_faces,
                                 const int64_t *d_faces, const double *d_area, int32_t nq,
                                 const double *d_w, const double *d_shape, int32_t ncomp,
                                 const double *d_load, double *d_F, const double *d_h,
                                 const double *d_mt, const int32_t *d_row_ptr,
                                 const int32_t *d_col, int64_t n_nodes, double *d_vals,
                                 void *stream);

/* Joule power of one step of the transient Tet10 A-V march
 * (em3d_tet10.py:665-692, transient_joule_power_tet10): for every element
 * with d_sigma[e] > 0, the field at its 10 nodes
 *   E_p = -(a_new_p - a_prev_p) / h - sum_j grad N_j(x_p) v_j,
 * the density Q_e = sigma_e sum_pq mref_pq E_p . E_q (0 elsewhere), and the
 * power *d_power = sum_e Q_e V_e, summed in a fixed order. d_elems: 10
 * nodes per element (int32), d_nodes: 3 doubles per node; a_prev, a_new:
 * 3 per node (node-major); v on the V nodes: d_vcol[node] is the node's
 * index in d_v, or -1 (v = 0; d_v may be NULL if no node has one). d_dn:
 * the reference element's dN_j/dxi_k at its node p (10 x 10 x 3, p-major);
 * d_mref: its normalised mass matrix (10 x 10, the reference's _MASS_REF).
 * d_q (optional): Q per element. Geometry from the corners (straight-edged
 * elements). */
CFEM_API int cfem_t10_joule_power(cfem_ctx *ctx, int64_t n_elems, const int32_t *d_elems,
                                  const double *d_nodes, const double *d_sigma,
                                  const double *d_a_prev, const double *d_a_new,
                                  const int64_t *d_vcol, const double *d_v, double h,
                                  const double *d_dn, const double *d_mref, double *d_power,
                                  double *d_q, void *stream);

/* Isotropic elasticity (CFEM_OP_P1_ELAST / CFEM_OP_T10_ELAST): the
 * element loops of assemble_elasticity_3d (elastic3d.py:105-189) and
 * assemble_elasticity_tet10 (elastic_tet10.py:135-211) into 3x3 nodal
 * blocks. Voigt [xx,yy,zz,yz,xz,xy] (elastic3d.py:26-34), body force b (3
 * coefs), thermal strain alpha (T - T_ref) with T a coef (NODAL, ELEM or
 * QP). */
CFEM_API int cfem_assemble_elastic(cfem_ctx *ctx, const cfem_pattern *p, int32_t op,
                          const double *d_nodes, const int32_t *d_elems,
                          double E, double nu, const cfem_coef *body3,
                          const cfem_coef *temp, double alpha, double T_ref,
                          double *d_vals, double *d_rhs, int32_t accumulate,
                          void *stream);

/* ---- boundary faces -----------------------------------------------------
 * Exterior-face candidates of tet_heat.py:97-120 / tet10.py:329-352: the
 * local faces (element*4 + face, ascending) whose three corners are all in
 * the node mask d_in_set (n_nodes bytes). Faces are listed with the local
 * corner order (0,1,2),(0,1,3),(0,2,3),(1,2,3) when faces10 == 0 and the
 * Tet10 table ((0,1,2),(0,3,1),(0,2,3),(1,3,2)) when faces10 == 1. Writes
 * at most n_elems*4 ids to d_out and the count to *n_out. Synchronises. */
CFEM_API int cfem_face_candidates(cfem_ctx *ctx, const int32_t *d_elems,
                         int64_t n_elems, int32_t npe, int32_t faces10,
                         const uint8_t *d_in_set, int64_t n_nodes,
                         int64_t *d_out, int64_t *n_out, void *stream);

/* Exterior faces among the candidates of cfem_face_candidates
 * (tet_heat.py:97-120, tet10.py:329-352, elastic3d.py:37-59): the faces
 * whose sorted corner triple occurs once among the candidates - every face
 * sharing a key with one whose corners are all in the set is itself a
 * candidate, so this count equals the reference's count over all element
 * faces - in candidate order (the reference's first-occurrence order).
 * Writes their ids (element*4 + face) to d_ids and their nodes (3 corners,
 * or with faces10 3 corners + 3 midside nodes) to d_nodes (n_cand * 3 or 6
 * entries at most), and the count to *n_out. Sorting by the triple on the
 * device (two stable radix sorts). Synchronises. */
CFEM_API int cfem_face_exterior(cfem_ctx *ctx, const int32_t *d_elems, int32_t npe,
                                int32_t faces10, const int64_t *d_cand, int64_t n_cand,
                                int64_t n_nodes, int64_t *d_ids, int64_t *d_nodes,
                                int64_t *n_out, void *stream);

/* ---- sparse helpers -----------------------------------------------------
 * d_vals_out = a*d_x + b*d_y over n values (sums such as C + theta h K,
 * tet_heat.py:239-240). */
CFEM_API int cfem_axpby(cfem_ctx *ctx, int64_t n, double a, const double *d_x,
               double b, const double *d_y, double *d_out, void *stream);
/* y = alpha*A x + beta*y for block CSR (bs = 1 or 3), FP64: the
 * matrix-vector products of the time marches (tet_heat.py:264,
 * tet10.py:536-538, dynamics3d.py:177-186). */
CFEM_API int cfem_spmv(cfem_ctx *ctx, int64_t n_rows, int32_t bs,
              const int32_t *d_row_ptr, const int32_t *d_col,
              const double *d_vals, double alpha, const double *d_x,
              double beta, double *d_y, void *stream);

/* Dirichlet elimination of tet_poisson.py:72-110 on a scalar CSR:
 * fixed rows become identity rows, fixed columns are removed from free
 * rows (the reference stores them as explicit zeros), and
 * rhs_out = rhs - A[:, fixed] v with rhs_out[fixed] = v. Output CSR
 * buffers need n+1 and nnz_in + n_fixed entries; *nnz_out receives the
 * entry count. Synchronises. */
CFEM_API int cfem_dirichlet_csr(cfem_ctx *ctx, int64_t n, const int32_t *d_indptr,
                       const int32_t *d_indices, const double *d_vals,
                       const double *d_rhs, const uint8_t *d_fixed,
                       const double *d_fixed_val, int32_t *d_out_indptr,
                       int32_t *d_out_indices, double *d_out_vals,
                       double *d_rhs_out, int64_t *nnz_out, void *stream);

/* FP32 operator for CFEM_SOLVE_MIXED (a method change; the reference
 * solves in FP64 only) in difference form: off-diagonal
 * blocks rounded to FP32 and, in each diagonal slot, the FP64 block row
 * sum s_i = sum_j A_ij rounded once. The solver applies it as
 * s_i p_i + sum_{j!=i} A_ij (p_j - p_i), which keeps constant vectors
 * (rigid translations) exact under FP32 rounding. Same layout as d_vals64. */
CFEM_API int cfem_mixed_matrix(cfem_ctx *ctx, int64_t n_rows, int32_t bs,
                               const int32_t *d_row_ptr, const int32_t *d_col,
                               const double *d_vals64, float *d_vals32,
                               void *stream);
/* cfem_mixed_matrix for many systems in one launch per block size (a
 * batch of meshes: one launch instead of one per system). */
typedef struct cfem_mixed_job {
    int64_t n_rows;
    int32_t bs;                 /* 1 or 3 */
    int32_t reserved;
    const int32_t *d_row_ptr;
    const int32_t *d_col;
    const double *d_vals64;
    float *d_vals32;
} cfem_mixed_job;
CFEM_API int cfem_mixed_matrix_batch(cfem_ctx *ctx, const cfem_mixed_job *jobs,
                                     int32_t n_jobs, void *stream);

/* ---- solver -------------------------------------------------------------
 * Jacobi-preconditioned CG on a batch of independent systems. Batches whose
 * work fits one resident wave run in ONE persistent cooperative launch (two
 * grid barriers per iteration); larger ones replay captured CUDA graphs of
 * 16 iterations (direction update, SpMV, reduction, update, reduction per
 * iteration). Per-system scalars are reduced in a fixed order, so each
 * result is bitwise the same alone and in any batch on a given scheduler.
 * CFEM_SOLVE_MIXED runs the CG in FP32 and keeps FP64 for the true residual
 * r = b - A x, the solution update and the convergence test (reliable
 * updates). Replaces spla.spsolve / spla.factorized (tet_poisson.py:121,
 * tet10.py:177, elastic3d.py:230). Writes one stats record per system.
 * Synchronises. Returns CFEM_OK when the solve ran; per-system outcomes are
 * in stats[i].status. Equivalent to plan create + solve + destroy. */
CFEM_API int cfem_pcg_solve(cfem_ctx *ctx, const cfem_linsys *systems,
                   int32_t n_systems, cfem_solve_stats *stats, void *stream);

/* Solve plans: the set-up of cfem_pcg_solve kept for repeated solves of the
 * same systems (time steps, serving), as spla.factorized is kept by
 * tet_heat.py:254 and tet10.py:524. Create captures the systems' device
 * pointers, options and working copies of the matrix values and builds the
 * iteration graphs; each solve re-initialises the solver state from the
 * current contents of b, x (initial guess with Dirichlet values) and the
 * fixed mask. After changing matrix values in place, call refresh before
 * the next solve. A plan has its own stream, events and workspace: plans of
 * one context may be solved from different host threads at the same time.
 * Destroy waits for the plan's work. */
typedef struct cfem_pcg_plan cfem_pcg_plan;
CFEM_API int cfem_pcg_plan_create(cfem_ctx *ctx, const cfem_linsys *systems,
                                  int32_t n_systems, void *stream,
                                  cfem_pcg_plan **out);
CFEM_API int cfem_pcg_plan_refresh(cfem_pcg_plan *plan, void *stream);
CFEM_API int cfem_pcg_plan_solve(cfem_pcg_plan *plan, cfem_solve_stats *stats,
                                 void *stream);
CFEM_API int cfem_pcg_plan_destroy(cfem_pcg_plan *plan);

/* Solve slots: continuous batching at iteration level, for serving loops
 * where systems arrive while others are being solved (the reference solves
 * one call at a time and has no counterpart). A slot plan holds n_slots
 * systems of one block size (1 or 3) and precision mode, each of at most
 * max_rows block rows and max_nnzb stored blocks, with point Jacobi; its
 * work lists, workspace and iteration graphs are fixed at creation. Assign
 * puts a system into a free slot (its working copy built, its state reset,
 * INIT run: it joins whatever is running), run queues `rounds` replays of
 * 16 iterations over every slot on the plan's stream (idle slots cost an
 * early exit), poll waits for the plan's stream and reports every slot
 * (status CFEM_SLOT_RUNNING while a system iterates; a finished system keeps
 * its status until the slot is assigned again), ready returns CFEM_OK once
 * the queued rounds have run and CFEM_SLOT_RUNNING before (no wait), release
 * ends a running system or frees a finished one. 3x3 slots hold the
 * sliced-ELL layout by default (CFEM_PARAM_SLOT_SELL3): assign then also
 * refuses (CFEM_ERR_INVALID, nothing changed) a system whose layout exceeds
 * the slot's room, which a block row of more than 96 blocks can cause.
 * The caller keeps a system's arrays alive
 * while it is in a slot and reads x after poll reports it finished. Each
 * system's scalars and sums are its own, so its iterates do not depend on
 * the other slots. Calls on one slot plan must come from one thread at a
 * time; assign and poll synchronise (poll the plan's stream, assign the
 * given stream), create synchronises, run, ready and release do not; run
 * does not order the given stream after the rounds (poll does, for the
 * host). Destroy with
 * cfem_pcg_plan_destroy. */
CFEM_API int cfem_pcg_slots_create(cfem_ctx *ctx, int32_t n_slots, int32_t bs, int32_t mode,
                                   int64_t max_rows, int64_t max_nnzb, void *stream,
                                   cfem_pcg_plan **out);
CFEM_API int cfem_pcg_slots_assign(cfem_pcg_plan *plan, int32_t slot, const cfem_linsys *system,
                                   void *stream);
CFEM_API int cfem_pcg_slots_run(cfem_pcg_plan *plan, int32_t rounds, void *stream);
CFEM_API int cfem_pcg_slots_ready(cfem_pcg_plan *plan);
CFEM_API int cfem_pcg_slots_poll(cfem_pcg_plan *plan, cfem_solve_stats *stats);
CFEM_API int cfem_pcg_slots_release(cfem_pcg_plan *plan, int32_t slot, void *stream);

/* Jacobi-preconditioned COCG (CG with the unconjugated form x^T y) for one
 * complex symmetric CSR system (A^T = A), values and vectors interleaved
 * (re, im) FP64, 16-byte aligned. Replaces spla.spsolve in the phasor A-V
 * eddy-current solve (em3d_tet10.py:267-375) once its V rows are scaled by
 * 1/(i omega), which makes that system complex symmetric. d_x: initial
 * guess in, solution out. Stops at ||r|| <= rtol ||b||; stats: status,
 * iterations, relres, bnorm, kernel_ms. Synchronises. */
CFEM_API int cfem_cocg_solve(cfem_ctx *ctx, int64_t n, const int32_t *d_indptr,
                             const int32_t *d_indices, const double *d_vals,
                             const double *d_b, double *d_x, double rtol,
                             int32_t max_iter, cfem_solve_stats *stats, void *stream);

/* Allocation-free variant of cfem_pcg_solve for ONE system. It has no
 * counterpart in the reference, which only solves on the host with SciPy.
 * It is for callers that cannot allocate device memory while solving: an
 * application that reserves the whole HBM budget for its own pools up front
 * (a library allocation mid-run could fail or fragment that budget), or a
 * latency-bound control loop that cannot take cudaMalloc's implicit
 * synchronisation. The solver workspace is a fixed file-scope device array
 * of cfem_pcg_noalloc_capacity() bytes (32 MiB), held by every GPU that
 * loads the library until the process exits; systems that need more are
 * rejected with CFEM_ERR_INVALID. The first call in each CUDA context looks
 * up the array's device address (cudaGetSymbolAddress) and keeps it for
 * that context, so make that first call before any stream capture, and do
 * not reset the device (cudaDeviceReset) after it. Every call reuses the
 * same array and clears it first: calls that overlap on the GPU (other
 * streams, other threads) race and must be serialised by the caller.
 * It always runs the persistent scheduler (one cooperative launch, the
 * grid strided over the row chunks when they exceed one resident wave):
 * the context's scheduler, SpMV staging and tuned solve-loop parameters have
 * no effect (its grid-barrier wait limit does), and stats->kernel_ms and
 * stats->spmv_ms are 0 (no timing events are created). The arithmetic is
 * that of cfem_pcg_solve on the persistent scheduler. Synchronises. */
CFEM_API size_t cfem_pcg_noalloc_capacity(void);
CFEM_API int cfem_pcg_solve_noalloc(cfem_ctx *ctx, const cfem_linsys *system,
                                    cfem_solve_stats *stats, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* CFEM_H */
