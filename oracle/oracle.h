// CPU oracle for the Newton-step linear solve -- TEST INFRASTRUCTURE ONLY.
//
// A plain C++ restatement of libuipc's algorithm on this path, used by the
// tests, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the
// checker. Nothing in the product links or calls it.
//
// Parity status: UNPINNED for the linear-solve math. libuipc's CUDA backend
// cannot be built here (Eigen 3.4 / fmt / spdlog are absent and the build
// needs cmake + vcpkg) and its tests ship no golden vectors for this path, so
// this restatement is checked against the reference's source semantics
// (file:line cited per function), against invariants (symmetry, SPD, exact
// integer patterns) and against an independent FP64 solve -- not against
// outputs of the reference itself. The MAS partition input can be pinned to
// the reference's own METIS (compiled from its sources into oracle/_ref).
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_matrix orc_matrix;
typedef struct orc_mas    orc_mas;

// ---- assembly: MatrixConverter<Float,3>::convert_sym + _calculate_block_offsets
// (src/backends/cuda/algorithm/details/matrix_converter.inl:1550-1701, 1058-1097)
orc_matrix* orc_assemble(int32_t n_block_rows, int64_t n_triplets, const int32_t* rows,
                         const int32_t* cols, const double* vals /* T x 9, column-major */);
void    orc_matrix_free(orc_matrix* m);
int64_t orc_matrix_nnz(const orc_matrix* m);       // unique upper blocks U
int32_t orc_matrix_rows(const orc_matrix* m);      // block rows nb
// rowptr [nb+1], rows/cols [U], vals [U*9] (column-major); any pointer may be NULL
void orc_matrix_copy(const orc_matrix* m, int32_t* rowptr, int32_t* rows, int32_t* cols, double* vals);

// ---- SpMV: y = a*A*x + b*y with A = U + U^T - diag(U) at block level
// (Spmv::cpu_sym_spmv, src/backends/cuda/linear_system/spmv.cu:1210-1297)
void orc_spmv(const orc_matrix* m, double a, const double* x, double b, double* y);

// ---- MAS (multi-level additive Schwarz), StiffGIPC hierarchy with BANKSIZE 16
// (src/backends/cuda/finite_element/mas_preconditioner_engine.cu)
orc_mas* orc_mas_create(int32_t vert_num, const int32_t* adj_start, const int32_t* adj_list,
                        int32_t part_map_size, const int32_t* part_to_real,
                        const int32_t* real_to_part);
void    orc_mas_free(orc_mas* s);
int32_t orc_mas_level_num(const orc_mas* s);
int32_t orc_mas_total_nodes(const orc_mas* s);  // node slots over all levels (= 16 * clusters)
// level_begin[L+1], level_count[L+1]
void orc_mas_levels(const orc_mas* s, int32_t* level_begin, int32_t* level_count);
// going_next [total_nodes] (level-0 part indexed by REAL vertex, as the reference),
// coarse_table [vert_num * (L-1)] (global node of vertex v at level l = 1..L-1)
void orc_mas_hierarchy(const orc_mas* s, int32_t* going_next, int32_t* coarse_table);
// Galerkin cluster matrices and inverses. dof_offset_blocks: block offset of
// the MAS vertex range inside A. invert_mode 0 = FP32 symmetric sweep exactly
// as the reference kernel; 1 = FP64 Gauss-Jordan rounded to FP32 storage.
int  orc_mas_assemble(orc_mas* s, const orc_matrix* A, int32_t dof_offset_blocks, int invert_mode);
// cluster_hess [clusters*136*9] FP64 and cluster_inv [clusters*136*9] FP32 (column-major blocks)
void orc_mas_clusters(const orc_mas* s, double* cluster_hess, float* cluster_inv);
// z = M^{-1} r on the MAS vertex range (r, z point at that range); FP32 inside.
void orc_mas_apply(const orc_mas* s, const double* r, double* z);
// overwrite the cluster inverses (clusters * 136 * 9 floats) after assemble
void orc_mas_set_inverses(orc_mas* s, const float* cluster_inv);
// Storage precision of the cluster inverses (applied to the current inverses
// in place): 0 = FP32 (as assembled), 1 = BF16 (round to nearest even),
// 2 = BF16 of the symmetrically diagonal-scaled inverse S M S with
// S = diag(M)^-1/2, the scale kept in FP32 (z = S (S M S)_bf16 S r).
void orc_mas_quantize(orc_mas* s, int mode);

// ---- PCG (LinearPCG::pcg, linear_pcg.cu:558-644; LinearFusedPCG::fused_pcg,
// linear_fused_pcg.cu:1782-2005)
enum
{
    ORC_PRECOND_NONE   = 0,
    ORC_PRECOND_JACOBI = 1,  // 3x3 block Jacobi (fem_diag_preconditioner.cu:18-58)
    ORC_PRECOND_MAS    = 2,  // MAS on [mas_offset, mas_offset + vert_num) blocks, 3x3 Jacobi elsewhere
};
enum
{
    ORC_STOP_RZ     = 0,  // |r.z| <= tol * |r0.z0| (the reference's rule)
    ORC_STOP_RELRES = 1,  // ||r||_2 <= tol * ||b||_2 on the recursive residual
};
typedef struct orc_pcg_result
{
    int64_t iterations;   // as the reference reports them
    int64_t converged;    // 1 if the stop rule fired
    double  rz0;
    double  rel_res_true; // ||b - A x|| / ||b|| recomputed in FP64 at exit
    int64_t bypassed;     // preconditioner bypassed (rz0 < 0 / non-finite)
} orc_pcg_result;

int orc_pcg(const orc_matrix* A, int precond, const orc_mas* mas, int32_t mas_offset_blocks,
            const double* b, double* x, double tol, int stop_rule, int check_interval,
            int64_t max_iter, int n_threads, orc_pcg_result* out);

// the same with the 12x12 block Jacobi of abd_n affine bodies on block rows
// [abd_off, abd_off + 4 abd_n) (applied after the other preconditioners)
int orc_pcg_abd(const orc_matrix* A, int precond, const orc_mas* mas, int32_t mas_offset_blocks,
                int32_t abd_off, int32_t abd_n, const double* b, double* x, double tol, int stop_rule,
                int check_interval, int64_t max_iter, int n_threads, orc_pcg_result* out);

// FP64 truth: block-Jacobi CG to ||r|| <= tol ||b|| (tol ~1e-13).
int orc_cg_truth(const orc_matrix* A, const double* b, double* x, double tol, int64_t max_iter,
                 int n_threads, int64_t* iterations);

#ifdef __cplusplus
}
#endif
