/*
 * b200solve -- B200-native (sm_100a) Newton-step linear solve behind a C ABI.
 *
 * Drop-in for the linear-solve path of libuipc's CUDA backend:
 *   triplet -> block-sparse (3x3) Hessian assembly, symmetric block SpMV,
 *   MAS (multi-level additive Schwarz) preconditioner build and apply, and
 *   the PCG loop, plus a mixed-precision mode.
 *
 * Conventions (identical to libuipc's GlobalLinearSystem):
 *   - the matrix is given as raw 3x3 block triplets (row, col, value) in the
 *     global block numbering; only entries with 0 <= row <= col are kept
 *     (block-upper storage of a symmetric matrix); duplicates are summed;
 *   - block values are 9 doubles, column-major (Eigen::Matrix3d layout);
 *   - vectors are FP64 with 3 * n_block_rows entries;
 *   - every pointer argument named d_* is a device pointer on the solver's
 *     device; h_* is host memory; "any" accepts either (copied with
 *     cudaMemcpyDefault).
 *
 * Errors: every entry point returns B2S_OK (0) or a negative status; the
 * message is available from b2s_last_error(). No exception crosses the ABI.
 * A solver handle is used by one host thread at a time; all work runs on the
 * stream set by b2s_set_stream (default: the solver's own stream), and the
 * entry points return after that stream's work for the call has completed
 * unless stated otherwise.
 */
#ifndef B200SOLVE_H
#define B200SOLVE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define B2S_OK 0
#define B2S_ERR_ARGUMENT -1   /* invalid argument / size / index */
#define B2S_ERR_CUDA -2       /* CUDA runtime error */
#define B2S_ERR_STATE -3      /* call out of order (e.g. apply before assemble) */
#define B2S_ERR_NUMERIC -4    /* non-finite values / breakdown */
#define B2S_ERR_NOT_CONVERGED -5

typedef struct b2s_solver b2s_solver;

/* ---- lifetime ------------------------------------------------------------
 * Replaces the construction of GlobalLinearSystem::Impl's buffers and the
 * solver / preconditioner SimSystems
 * (src/backends/cuda/linear_system/global_linear_system.h:266-325). */
int         b2s_create(int device, b2s_solver** out);
int         b2s_destroy(b2s_solver* s);
const char* b2s_last_error(const b2s_solver* s); /* s may be NULL: last create error */
int         b2s_set_stream(b2s_solver* s, void* cuda_stream); /* cudaStream_t; NULL = own stream */
int         b2s_version(void);

/* ---- assembly --------------------------------------------------------------
 * Replaces MatrixConverter<Float,3>::convert_sym + convert(BCOO->BSR)
 * (src/backends/cuda/algorithm/details/matrix_converter.inl:1550-1701,
 * 1040-1097), called from GlobalLinearSystem::Impl::build_linear_system
 * (src/backends/cuda/linear_system/global_linear_system.cu:272-319).
 * Triplets with row < 0 (unwritten slots) or row > col are dropped, the rest
 * are sorted by (row, col, source index) and summed in source order. The
 * resulting pattern (block-upper BSR row pointers and column indices) is the
 * reference's exactly; the sums are deterministic. */
int b2s_assemble(b2s_solver* s, int32_t n_block_rows, int64_t n_triplets,
                 const int32_t* d_rows, const int32_t* d_cols, const double* d_vals);
/* Triplet arrays owned by the solver, for producers that write the raw
 * triplets in place (no staging copy): device pointers to room for
 * n_triplets (row, col, 9 values column-major), grown by ratio and kept
 * across calls; b2s_assemble_owned assembles the first n_triplets of them.
 * Replaces the staging of GlobalLinearSystem::Impl::_assemble_linear_system
 * (src/backends/cuda/linear_system/global_linear_system.cu:233-268, 407-497):
 * the subsystems' producers write their triplet sub-ranges here directly. */
int b2s_triplet_buffers(b2s_solver* s, int64_t n_triplets, int32_t** d_rows, int32_t** d_cols, double** d_vals);
int b2s_assemble_owned(b2s_solver* s, int32_t n_block_rows, int64_t n_triplets);
int b2s_matrix_info(const b2s_solver* s, int32_t* n_block_rows, int64_t* n_upper_blocks);
/* Copy the block-upper BSR out: rowptr [n_block_rows+1], colidx [nnz],
 * vals [nnz*9] column-major. Any pointer may be NULL; "any" memory. */
int b2s_get_upper_bsr(b2s_solver* s, int32_t* rowptr, int32_t* colidx, double* vals);

/* ---- SpMV --------------------------------------------------------------------
 * y = A x with A = U + U^T - diag(U) at block level, and optionally
 * d_dot = x . y. Replaces Spmv::rbk_sym_spmv / rbk_sym_spmv_dot
 * (src/backends/cuda/linear_system/spmv.cu:992-1160) as used by
 * IterativeSolver::spmv / spmv_dot (src/backends/cuda/linear_system/iterative_solver.h:30-40). */
int b2s_spmv(b2s_solver* s, const double* d_x, double* d_y, double* h_dot /* may be NULL */);
/* The same y = A x as the mixed-precision PCG computes it: FP32 copy of the
 * values, FP32 vectors [3 * n_block_rows], FP32 products and sums (y's
 * reductions in any order), x . y accumulated in FP64 (h_dot, host, may be
 * NULL). No counterpart in the reference (which runs the SpMV in FP64 only). */
int b2s_spmv_mixed(b2s_solver* s, const float* d_x, float* d_y, double* h_dot /* may be NULL */);
/* Measurement: the FP32 SpMV kernel (with its fused dot) launched `launches`
 * times back to back on the assembled matrix, CUDA events on the solver's
 * stream around the batch; *h_avg_ms = the average launch duration. */
int b2s_spmv_mixed_timing(b2s_solver* s, int32_t launches, double* h_avg_ms);

/* ---- MAS preconditioner ----------------------------------------------------------
 * Initialisation: replaces FEMMASPreconditioner::do_init ->
 * MASPreconditionerEngine::init_neighbor + init_matrix
 * (src/backends/cuda/finite_element/fem_mas_preconditioner.cu:157-404,
 *  src/backends/cuda/finite_element/mas_preconditioner_engine.h:67-80).
 * The MAS acts on block rows [block_offset, block_offset + vert_num);
 * h_adj_start/h_adj_list is the vertex adjacency (CSR, sorted), part_to_real
 * maps partition slots (parts padded to 16) to vertices (-1 = padding) and
 * real_to_part is its inverse (-1 = unpartitioned vertex, which then gets the
 * 3x3 block-Jacobi fallback). */
int b2s_mas_init(b2s_solver* s, int32_t block_offset, int32_t vert_num,
                 const int32_t* h_adj_start, const int32_t* h_adj_list,
                 int32_t part_map_size, const int32_t* h_part_to_real,
                 const int32_t* h_real_to_part);
/* MAS hierarchy introspection (for parity checks): level count, node slots
 * over all levels, per-level begin/count [L+1] and the per-vertex coarse
 * table [vert_num * (L-1)] (global node of vertex v at levels 1..L-1). */
int b2s_mas_info(const b2s_solver* s, int32_t* level_num, int32_t* total_nodes);
int b2s_mas_get_hierarchy(b2s_solver* s, int32_t* h_level_begin, int32_t* h_level_count,
                          int32_t* h_coarse_table);
/* Cluster matrices after b2s_precond_assemble: Galerkin matrices (FP64) and
 * inverses (FP32), 136 column-major 3x3 blocks per 16-node cluster. */
int b2s_mas_get_clusters(b2s_solver* s, double* h_hess, float* h_inv);
/* Stiff clusters of the last build: their count, and per cluster 1 when it
 * was inverted in FP64 (h_flags: total_nodes / 16 bytes, may be NULL). The
 * mixed-precision apply uses their FP32 inverse in place of BF16 tiles. */
int b2s_mas_stiff_info(b2s_solver* s, int32_t* n_stiff, uint8_t* h_flags);
/* Node buffers of the last MAS apply (FP32, 3 per node slot, total_nodes
 * slots): the restricted residual R of every coarse node and the local
 * solution Z of every node. */
int b2s_mas_get_nodes(b2s_solver* s, float* h_R, float* h_Z);

/* Partition utility (the caller-side step of FEMMASPreconditioner::do_init):
 * recursive coordinate bisection into parts of at most max_part vertices,
 * each part a multiple of max_part except the remainder, then the padded
 * part_to_real / real_to_part maps (fem_mas_preconditioner.cu:285-330).
 * b2s_partition_maps with h_part_to_real == NULL only returns the map size
 * in *part_map_size (call it first to size h_part_to_real). */
int b2s_partition_rcb(int32_t n, const double* h_positions, int32_t max_part,
                      int32_t* h_part_ids);
/* Graph partition from the vertex adjacency alone (CSR as b2s_mas_init takes
 * it), the drop-in for geometry::mesh_partition's METIS k-way call
 * (src/geometry/mesh_partition.cpp:77-231): ceil(n / max_part) parts of at
 * most max_part vertices, ids 0.. contiguous, no part empty; point clouds (no
 * edges) take sequential blocks; n <= max_part gives one part per connected
 * component. Recursive graph bisection, deterministic (no seed): the part
 * ids follow the bisection tree, so consecutive parts are neighbours. */
int b2s_partition_graph(int32_t n, const int32_t* h_adj_start, const int32_t* h_adj_list,
                        int32_t max_part, int32_t* h_part_ids);
int b2s_partition_maps(int32_t n, const int32_t* h_part_ids, int32_t max_part,
                       int32_t* h_part_to_real, int32_t* h_real_to_part,
                       int32_t* part_map_size);

#define B2S_PRECOND_NONE 0
#define B2S_PRECOND_JACOBI 1 /* 3x3 block Jacobi (fem_diag_preconditioner.cu:18-58) */
#define B2S_PRECOND_MAS 2    /* MAS on its range, 3x3 block Jacobi elsewhere */

/* Inversion of the MAS cluster matrices (the reference inverts every cluster
 * in FP32 without pivoting, mas_preconditioner_engine.cu:1077-1175). Here an
 * LDL^T factorisation per cluster; a cluster whose FP32 elimination cancels
 * more than 10 bits of a pivot (stiff contact couplings) is "stiff". */
#define B2S_INVERT_F32 0      /* FP32; stiff clusters again in FP64 (default) */
#define B2S_INVERT_F64 1      /* FP64 for every cluster */
#define B2S_INVERT_F32_ONLY 2 /* FP32 for every cluster, stiff ones too */

/* Affine bodies: block rows [block_offset, block_offset + 4 n_bodies) hold
 * n_bodies affine bodies of 12 DoF (4 block rows each). Every preconditioner
 * kind but NONE then applies, on that range, the inverse of each body's full
 * 12x12 diagonal Hessian block (FP64, built by b2s_precond_assemble): the
 * reference's ABDDiagPreconditioner, which has no configuration gate and acts
 * after any global preconditioner on the affine-body sub-range
 * (src/backends/cuda/affine_body/abd_diag_preconditioner.cu:15-125,185-191,
 *  src/backends/cuda/linear_system/global_linear_system.cu:555-576). The MAS
 * range (b2s_mas_init) must not overlap it. n_bodies = 0 removes the range. */
int b2s_abd_init(b2s_solver* s, int32_t block_offset, int32_t n_bodies);

/* Build the preconditioner from the current assembled matrix. Replaces
 * GlobalPreconditioner::do_assemble / LocalPreconditioner::do_assemble
 * (src/backends/cuda/linear_system/global_preconditioner.h:16,
 *  src/backends/cuda/finite_element/fem_mas_preconditioner.cu:406-439). */
int b2s_precond_assemble(b2s_solver* s, int kind, int invert_mode);
/* z = P r (FP64 vectors). Replaces GlobalPreconditioner::do_apply
 * (global_preconditioner.h:17; mas_preconditioner_engine.cu:2887-2960). */
int b2s_precond_apply(b2s_solver* s, const double* d_r, double* d_z);
/* The same z = P r as the mixed-precision PCG applies it: FP32 vectors
 * [3 * n_block_rows], MAS cluster inverses stored as BF16 of the
 * diagonal-scaled inverse S M S (S = diag(M)^-1/2 in FP32), FP32 accumulation.
 * No counterpart in the reference (which applies FP32 inverses only). */
int b2s_precond_apply_mixed(b2s_solver* s, const float* d_r, float* d_z);

/* ---- PCG ---------------------------------------------------------------------------
 * Replaces IterativeSolver::do_solve as implemented by LinearFusedPCG
 * (src/backends/cuda/linear_system/linear_fused_pcg.cu:851-943, 1782-2005) and
 * LinearPCG (src/backends/cuda/linear_system/linear_pcg.cu:395-438, 558-644). */
#define B2S_STOP_RZ 0     /* |r.z| <= tol |r0.z0| (the reference's rule) */
#define B2S_STOP_RELRES 1 /* ||b - A x||_2 <= tol ||b||_2, verified in FP64 */

#define B2S_PRECISION_FP64 0  /* FP64 matrix/vectors, FP32 MAS inverses */
#define B2S_PRECISION_MIXED 1 /* FP32 matrix/vectors, BF16 MAS inverses, FP64 dots + residual replacement */

typedef struct b2s_pcg_options
{
    double  tol;            /* stop tolerance (rule below) */
    int32_t stop_rule;      /* B2S_STOP_* */
    int32_t check_interval; /* iterations per host convergence check (graph block) */
    int64_t max_iter;       /* 0 = 2 * n_dof (the reference's max_iter_ratio = 2) */
    int32_t precision;      /* B2S_PRECISION_* */
    int32_t use_graph;      /* capture check_interval iterations in a CUDA graph */
    int32_t x0_given;       /* 1: d_x holds the initial guess; 0: start from 0 */
    int32_t replace_every;  /* mixed: FP64 residual replacement period (0 = off) */
} b2s_pcg_options;

typedef struct b2s_pcg_stats
{
    int64_t iterations;   /* as the reference reports them (multiple of check_interval when fused) */
    int64_t iterations_exact; /* iteration at which the stop rule fired */
    int32_t converged;
    int32_t bypassed;     /* preconditioner bypassed: rz0 < 0 or non-finite (PSD guard) */
    double  rz0;
    double  rel_res;      /* ||b - A x|| / ||b|| recomputed in FP64 at exit */
    int64_t replacements; /* residual replacements done */
} b2s_pcg_stats;

void b2s_pcg_default_options(b2s_pcg_options* o);
int  b2s_pcg(b2s_solver* s, const double* d_b, double* d_x, const b2s_pcg_options* opt,
             b2s_pcg_stats* stats);

/* ---- stage timers ------------------------------------------------------------------
 * Device-time counterparts of the reference's scoped timers "Convert To BCOO",
 * "Assemble Preconditioner", "FusedPCG", "SpMV" and "Apply Preconditioner"
 * (src/backends/cuda/linear_system/global_linear_system.cu:274-313,
 *  linear_fused_pcg.cu:1413,1438,1785): CUDA events on the solver's stream,
 * accumulated while timing is enabled. kernel_launches counts every kernel
 * this library launched (graph replays included) since the last reset. */
typedef struct b2s_timers
{
    double  assemble_ms;
    double  precond_build_ms;
    double  pcg_ms;
    double  spmv_ms;
    int64_t spmv_launches;
    double  precond_apply_ms;
    int64_t precond_apply_launches;
    int64_t kernel_launches;
} b2s_timers;

int b2s_set_timing(b2s_solver* s, int enable);
int b2s_get_timers(const b2s_solver* s, b2s_timers* out);
int b2s_reset_timers(b2s_solver* s);

/* ---- learned PCG warm start ------------------------------------------------------------
 * No counterpart in the reference (its PCG starts from x0 = 0,
 * linear_fused_pcg.cu:1782-2005). A small MLP on MAS level-1 aggregates
 * predicts the initial guess of the next Newton solve from the gradient b and
 * the solutions of earlier solves of the same run (history h1 = the latest,
 * h2, h3, ... older; at most B2S_WS_MAX_HISTORY device vectors of 3 n
 * doubles, of which the newest B2S_WS_HISTORY feed the network's fields).
 * Per aggregate, the network reads 22 features (mean of b, and of each field
 * f = {h1, h1 - h2, h1 - 2 h2 + h3, z = P b}: its mean and log RMS, plus the
 * mean products of consecutive fields) and outputs 4 coefficients c; the
 * predicted field is d_v = sum_i c_i f_i(v) on every vertex of the aggregate.
 * The start x0 is the A-optimal (Galerkin) combination of the candidate
 * vectors of `mode`, checked in FP64 by the PCG's own residual measure:
 * when r^T P r (r = b - A x0) is not below b^T P b, x0 = 0 (the plain start). Training uses Newton systems of the
 * same run (b2s_ws_add_sample with the solved x), a quadratic per-aggregate
 * loss sum_v |d_v - x_v|^2 / sum_v |x_v|^2 (fields scaled by RMS(z)), Adam,
 * FP32 weights; inference reads BF16 copies of the weights. Requires an
 * assembled matrix and the MAS preconditioner (b2s_precond_assemble). */
#define B2S_WS_HISTORY 3     /* history vectors the network's fields read */
#define B2S_WS_MAX_HISTORY 8 /* history vectors a start may combine */
#define B2S_WS_FEATURES 22
#define B2S_WS_OUTPUTS 4
#define B2S_WS_MODE_ZERO 0    /* x0 = 0 */
#define B2S_WS_MODE_PREV 1    /* Galerkin on {h1}: the scaled previous solution */
#define B2S_WS_MODE_HISTORY 2 /* Galerkin on the history {h1, ..., h_n}, no network */
#define B2S_WS_MODE_LEARNED 3 /* Galerkin on {network field, h1, ..., h_n} */

typedef struct b2s_ws_info
{
    int    mode;          /* mode used (ZERO when the residual check rejected the start) */
    int    n_candidates;  /* vectors in the Galerkin combination */
    double coeff[1 + B2S_WS_MAX_HISTORY]; /* their coefficients */
    double rel_res0;      /* ||b - A x0|| / ||b|| of the returned x0 (FP64) */
    double rel_res_tried; /* the same for the candidate before the check */
    double rz_ratio;      /* (r^T P r) / (b^T P b) of the candidate, r = b - A x0, P the preconditioner:
                             the check; the start is kept when it is below 1 */
    double predict_ms;    /* device time of the prediction (features, MLP, Galerkin, check) */
} b2s_ws_info;

/* allocate the network (hidden width `hidden`, 3 layers) with seeded random weights */
int b2s_ws_init(b2s_solver* s, int32_t hidden, uint64_t seed);
/* append one training sample: this system's aggregates with the solved x (device) */
int b2s_ws_add_sample(b2s_solver* s, const double* d_b, int32_t n_hist, const double* const* d_hist,
                      const double* d_x);
int b2s_ws_num_samples(const b2s_solver* s, int32_t* n_samples, int64_t* n_rows);
/* feature mean / std over the stored samples (inputs are standardised with them) */
int b2s_ws_fit_normalization(b2s_solver* s);
/* `epochs` passes over the stored samples (one Adam step per sample, order from `seed`) */
int b2s_ws_train(b2s_solver* s, int32_t epochs, double lr, uint64_t seed, double* h_mean_loss);
/* loss and gradient (n_params floats, host) of stored sample `index`, no update */
int b2s_ws_loss_grad(b2s_solver* s, int32_t index, double* h_loss, float* h_grad);
/* parameters: W0[F x H] b0[H] W1[H x H] b1[H] W2[H x O] b2[O] (row-major, x W + b), then
 * feature mean[F] and std[F]; h_params NULL = size query into *n */
int b2s_ws_get_params(const b2s_solver* s, float* h_params, int64_t* n);
int b2s_ws_set_params(b2s_solver* s, const float* h_params, int64_t n);
/* append a stored sample given as arrays ("any" memory: the layout
 * b2s_ws_get_sample returns), e.g. a training set read back from a checkpoint;
 * norm > 0 is the sample's loss normaliser */
int b2s_ws_put_sample(b2s_solver* s, int32_t rows, const float* feat, const float* H, const float* q,
                      const float* c0, double norm);
/* a stored sample for checking: raw features [rows x F], H [rows x 10] (upper
 * triangle of the 4x4 field Gram), q [rows x 4], c0 [rows], loss normaliser;
 * NULL pointers = size query of *rows */
int b2s_ws_get_sample(const b2s_solver* s, int32_t index, int32_t* rows, float* h_feat, float* h_H,
                      float* h_q, float* h_c0, double* h_norm);
/* the warm start x0 (device, 3 n doubles) for the current system */
int b2s_ws_predict(b2s_solver* s, int32_t mode, const double* d_b, int32_t n_hist,
                   const double* const* d_hist, double* d_x0, b2s_ws_info* info);

/* ---- SpMV for callers that cannot allocate -------------------------------------------
 * No counterpart in the reference. The same y = A x and x.(A x) as b2s_spmv,
 * for callers that must not (or cannot) call cudaMalloc: code running inside
 * a host callback or an allocator hook, a process whose device memory is
 * owned by another framework's caching allocator, or a loop that may not
 * touch the allocator after start-up. It takes no solver handle and
 * allocates nothing: the caller owns the block-upper BCOO (d_rows, d_cols,
 * d_vals: 9 doubles per block, column-major, row <= col, no duplicates, rows
 * non-decreasing -- the order b2s_get_upper_bsr returns), d_x, d_y
 * [3 * n_block_rows] and d_dot (one double, may be NULL). The kernel checks
 * every block: one whose row or column lies outside [0, n_block_rows), whose
 * row exceeds its column, or whose row is below the previous block's is
 * skipped (nothing is read or written through its indices) and *d_dot
 * becomes NaN, so pass d_dot to learn of bad input. Its scratch is a fixed device array in
 * the library (about 256 KB per device that loads it, held until exit), so
 * n_blocks is limited to 8,388,608; larger inputs are rejected with
 * B2S_ERR_ARGUMENT. Work is queued on `stream` (cudaStream_t, NULL = legacy
 * stream) and the call returns without waiting. The first call on a device
 * looks up the scratch array's device address; make that first call before
 * any stream capture. Every call shares the scratch array, so calls that
 * overlap on the GPU (concurrent streams) race: serialise them. Errors are
 * reported through b2s_last_error(NULL). */
int b2s_spmv_noalloc(int32_t n_block_rows, int64_t n_blocks, const int32_t* d_rows,
                     const int32_t* d_cols, const double* d_vals, const double* d_x,
                     double* d_y, double* d_dot, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* B200SOLVE_H */
