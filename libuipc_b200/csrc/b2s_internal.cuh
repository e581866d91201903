// Internal declarations of libb200solve (not part of the ABI).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/b200solve.h"

namespace b2s
{
constexpr int BANK = 16;                    // nodes per MAS cluster
constexpr int SYM  = BANK * (BANK + 1) / 2;  // 136 upper 3x3 blocks per cluster
constexpr int MAX_LEVELS = 6;
constexpr int NUM_SMS_HINT = 148;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
struct Error : std::runtime_error
{
    int code;
    Error(int c, const std::string& m)
        : std::runtime_error(m)
        , code(c)
    {
    }
};

#define B2S_CUDA(call)                                                                       \
    do                                                                                       \
    {                                                                                        \
        cudaError_t e__ = (call);                                                            \
        if(e__ != cudaSuccess)                                                               \
            throw ::b2s::Error(B2S_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e__) \
                                                 + " (" + __FILE__ + ":" + std::to_string(__LINE__) + ")"); \
    } while(0)

// kernels launched by this thread through the library (every launch site
// goes through B2S_CHECK_LAUNCH; graph replays add their node count)
extern thread_local long long g_kernel_launches;

#define B2S_CHECK_LAUNCH()                    \
    do                                        \
    {                                         \
        ++::b2s::g_kernel_launches;           \
        B2S_CUDA(cudaGetLastError());         \
    } while(0)

#define B2S_REQUIRE(cond, code, msg)          \
    do                                        \
    {                                         \
        if(!(cond))                           \
            throw ::b2s::Error((code), (msg)); \
    } while(0)

// device-side error bits (written by kernels with bounds checks)
enum DeviceError : int
{
    DERR_TRIPLET_INDEX = 1,  // triplet row/col outside [0, n_block_rows)
    DERR_ROW_OVERFLOW  = 2,  // a row's bucket exceeded its counted size
    DERR_MAS_INDEX     = 4,  // MAS hierarchy index out of range
    DERR_TMA_TIMEOUT   = 8,  // a bounded wait on a bulk-copy barrier ran out
};

// ---------------------------------------------------------------------------
// device buffer with capacity growth (no shrink)
// ---------------------------------------------------------------------------
template <typename T>
struct DBuf
{
    T*     ptr = nullptr;
    size_t n   = 0;  // size in elements
    size_t cap = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { release(); }
    void release()
    {
        if(ptr)
            cudaFree(ptr);
        ptr = nullptr;
        n = cap = 0;
    }
    // resize; contents are NOT preserved when capacity grows
    void resize(size_t count, double growth = 1.0)
    {
        if(count > cap)
        {
            release();
            size_t want = (size_t)((double)count * growth);
            if(want < count)
                want = count;
            if(want == 0)
                want = 1;
            B2S_CUDA(cudaMalloc(&ptr, want * sizeof(T)));
            cap = want;
        }
        n = count;
    }
    T*       data() { return ptr; }
    const T* data() const { return ptr; }
    size_t   size() const { return n; }
    size_t   bytes() const { return n * sizeof(T); }
};

// ---------------------------------------------------------------------------
// assembled matrix: block-upper BSR, values in 9 component planes
// ---------------------------------------------------------------------------
struct Matrix
{
    int32_t        nb  = 0;  // block rows
    int64_t        nnz = 0;  // unique upper blocks U
    int64_t        stride = 0;  // plane stride: U rounded up to 16 (16-byte aligned loads of 4 blocks)
    DBuf<int32_t>  rowptr;   // [nb+1]
    DBuf<int32_t>  rows;     // [stride] block row of each block (BCOO row index), -1 in the padding
    DBuf<int32_t>  cols;     // [stride]
    DBuf<double>   vals;     // [9][stride]: component q (column-major index) at vals[q*stride + k]
    DBuf<float>    vals32;   // FP32 copy of vals (mixed precision), same layout
    // rank of each block in (column, index) order inside its SPMV_TILE-block
    // tile: the SpMV places the transposed contributions of a tile by column
    // in shared memory and merges equal columns before its reductions
    DBuf<uint16_t> trank;    // [stride]
    bool           has_trank = false;
    DBuf<int32_t>  diag_index;  // [nb] position of block (i,i), -1 if absent
    // row starts of the FP32 SpMV, per group of 128 blocks: the first block's
    // row and a 128-bit mask of the blocks that start a row (no row ids read)
    DBuf<int32_t>  grp_row;
    DBuf<uint4>    grp_mask;
    bool           has_groups = false;
    bool           valid = false;
    long long      generation = 0;         // bumped by every assembly
    long long      vals32_generation = -1;  // assembly the FP32 planes were made from
};

// scratch of the assembly pipeline (reused across calls)
struct AssemblyScratch
{
    DBuf<int32_t> row_count, row_start, row_fill, uniq_count;
    DBuf<int2>    bucket;  // (column, source) of the kept triplets, bucketed by row
    DBuf<int32_t> sorted_col, sorted_src;
    DBuf<int32_t> run_start;  // [U+1] sorted position of each unique block's first source
    DBuf<int32_t> long_rows;  // [1 + nb]: count, then the rows too long for one warp
    DBuf<int32_t> scan_tmp;
    DBuf<int>     err;
};

// ---------------------------------------------------------------------------
// MAS
// ---------------------------------------------------------------------------
struct MasState
{
    bool    initialized = false;
    int32_t offset      = 0;  // block offset of the MAS vertex range
    int32_t vn          = 0;  // vertices in the range
    int32_t N           = 0;  // part map size (level-0 nodes)
    int32_t L           = 0;  // levels
    int32_t total       = 0;  // node slots over all levels
    int32_t clusters    = 0;  // total / 16
    std::vector<int32_t> level_begin, level_count;  // [L+1]
    // device hierarchy
    DBuf<int32_t> p2r, r2p;        // [N], [vn]
    DBuf<int32_t> ctable;          // [vn * (L-1)] global node at levels 1..L-1
    DBuf<int32_t> node1;           // [vn] global level-1 node of each vertex (-1: none)
    DBuf<int32_t> anc;             // [level_count[1] * (L-2)] global slots of each level-1 node's ancestors
    DBuf<int32_t> cst;             // [L * vn] local id of vertex v at level l+1
    DBuf<uint16_t> comp_mask[MAX_LEVELS];  // per level: component lane mask of each node
    DBuf<int32_t>  new_local[MAX_LEVELS];  // per level: local id of each node at the next level
    DBuf<int32_t>  level_begin_dev;        // [L+1]
    // per assembly
    DBuf<double>  hess;            // [clusters * 136 * 9]
    DBuf<float>   inv;             // [clusters * 136 * 9]
    DBuf<uint8_t> stiff;           // [clusters] 1: inverted in FP64, applied from the FP32 inverse
    DBuf<int32_t> stiff_list;      // [clusters] the stiff clusters (first stiff_count entries)
    DBuf<int32_t> stiff_count;     // [1]
    DBuf<unsigned char> inv16;     // [clusters * 3264]: FP32 factor D (48) + six BF16 16x16 tiles of D^-1 inv D^-1
    long long     inv16_generation = -1;  // assembly generation inv16 was packed from
    // coarse-level Galerkin matrices (upper BCOO per level, in level-local ids)
    Matrix        coarse[MAX_LEVELS];
    DBuf<int32_t> trip_rows, trip_cols;
    DBuf<double>  trip_vals;
    // apply buffers (FP32, 3 per node slot); after an apply the level-1 slots
    // of Z hold the folded prolongation Z_1 + Z_2[parent] + ...
    DBuf<float>   R, Z;
    // host copies for introspection
    std::vector<int32_t> h_ctable;
};

// ---------------------------------------------------------------------------
// PCG state
// ---------------------------------------------------------------------------
struct PcgScalars
{
    double rz;        // r.z of the current iterate
    double rz_new;
    double pAp;
    double rr;        // r.r (recursive residual)
    double rz_tol;    // tol * |rz0|
    double rr_tol;    // (tol * ||b||)^2
    double alpha;
    double beta;
    int    converged;
    int    stop_rule;
    long long iter;       // iterations executed
    long long iter_conv;  // iteration at which the rule fired
    long long max_iter;
};

struct Reduction
{
    DBuf<double>       partials;  // [2 * grid]
    DBuf<unsigned int> counter;
};

struct PcgState
{
    DBuf<double> r, z, p, Ap, tmp;
    DBuf<PcgScalars> sc;
    Reduction        red;
    PcgScalars*      h_sc = nullptr;  // pinned mirror
    cudaGraphExec_t  graph = nullptr;
    size_t           graph_key = 0;
    long long        graph_kernels = 0;  // kernel nodes per graph launch
    // mixed precision: FP32 recursion vectors and their own graph
    DBuf<float>      r32, z32, p32, Ap32;
    cudaGraphExec_t  graph_mixed = nullptr;
    size_t           graph_mixed_key = 0;
    long long        graph_mixed_kernels = 0;
};

struct LearnedState;  // learned warm start (b2s_learned.cu)
void ws_free(LearnedState* w);

}  // namespace b2s

// the opaque ABI handle
struct b2s_solver
{
    int          device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    std::string  last_error;
    b2s::Matrix          A;
    b2s::AssemblyScratch asmb;
    b2s::MasState        mas;
    b2s::PcgState        pcg;
    int                  precond_kind = -1;
    int                  invert_mode  = 0;
    long long            precond_generation = 0;  // bumped by every preconditioner build
    b2s::DBuf<double>    dinv;  // [nb*9] row-major inverses of diagonal blocks
    int32_t              abd_offset = 0, abd_n = 0;  // affine bodies: block rows abd_offset + [0, 4 abd_n)
    b2s::DBuf<double>    abd_inv;  // [abd_n * 144] row-major 12x12 inverses
    b2s::DBuf<double>    dot_out;
    b2s::Reduction       red;
    b2s::DBuf<int>       dev_err;  // DeviceError bits raised by kernels
    // the MAS apply's second stream: the coarse levels run on it beside the
    // fine level's products (forked from `stream` and joined back by events)
    cudaStream_t             mas_side = nullptr;
    cudaEvent_t              mas_fork = nullptr, mas_join = nullptr;
    // stage timers (CUDA events on `stream`)
    bool                     timing = false;
    b2s_timers               timers{};
    cudaEvent_t              ev_begin = nullptr, ev_end = nullptr;
    std::vector<cudaEvent_t> iter_events;  // 4 per iteration of a graph block
    b2s::LearnedState*       ws = nullptr;  // learned warm start, created on first use
    // triplet arrays owned by the solver (b2s_triplet_buffers): producers
    // write the raw triplets here, b2s_assemble_owned reads them in place
    b2s::DBuf<int32_t>       own_rows, own_cols;
    b2s::DBuf<double>        own_vals;
};

namespace b2s
{
// device-wide exclusive scan of int32 (n elements, out may alias in); returns
// the total (synchronises when want_total)
void exclusive_scan(b2s_solver* s, const int32_t* in, int32_t* out, int64_t n, DBuf<int32_t>& tmp);

// assembly of raw triplets into a block-upper matrix (shared by the global
// matrix and the MAS coarse levels); `spmv_tiles` also computes the per-tile
// column ranks the SpMV uses
void assemble_triplets(b2s_solver* s, Matrix& M, int32_t nb, int64_t T, const int32_t* rows,
                       const int32_t* cols, const double* vals, bool spmv_tiles);

constexpr int SPMV_TILE = 1024;  // blocks per SpMV tile (the span of the transposed-half ranks)

// y = A x (+ optional pAp into partial reduction slot)
void spmv_f64(b2s_solver* s, const Matrix& A, const double* x, double* y, double* d_dot);

// reductions
int  reduction_grid();
void launch_dot(b2s_solver* s, const double* a, const double* b, int64_t n, double* d_out);
// several dot products in one pass: d_out[k] = a[k] . b[k], k < m (FP64,
// deterministic)
constexpr int MAX_DOTS = 10;
struct DotPairs
{
    const double* a[MAX_DOTS];
    const double* b[MAX_DOTS];
};
void launch_dots(b2s_solver* s, int64_t n, const DotPairs& d, int m, double* d_out);
// partial-sum storage of the grid reductions for `grid` blocks x `nv` values
void ensure_reduction(Reduction& red, int grid, int nv);

// preconditioners
void precond_assemble(b2s_solver* s, int kind, int invert_mode);
void precond_apply(b2s_solver* s, const double* r, double* z);
void precond_launch(b2s_solver* s, const double* r, double* z);  // queued, no sync
void precond_apply_mixed(b2s_solver* s, const float* r, float* z);
void spmv_mixed(b2s_solver* s, const float* x, float* y, double* d_dot);
double spmv_mixed_timing(b2s_solver* s, int launches);
void check_device_errors(b2s_solver* s);

// message of the last failed call made without a solver handle (read back
// through b2s_last_error(NULL))
void set_handle_free_error(const std::string& msg);
void mas_init(b2s_solver* s, int32_t offset, int32_t vn, const int32_t* adj_start,
              const int32_t* adj_list, int32_t N, const int32_t* p2r, const int32_t* r2p);
void mas_assemble(b2s_solver* s, int invert_mode);
void mas_apply(b2s_solver* s, const double* r, double* z);
// host: recursive graph bisection into parts of at most max_part vertices
void partition_graph(int32_t n, const int32_t* xadj, const int32_t* adj, int32_t max_part, int32_t* part_ids);

// PCG
void pcg_solve(b2s_solver* s, const double* b, double* x, const b2s_pcg_options& o, b2s_pcg_stats& st);
void drop_graphs(b2s_solver* s);

// learned warm start
void    ws_init(b2s_solver* s, int hidden, uint64_t seed);
void    ws_add_sample(b2s_solver* s, const double* b, int n_hist, const double* const* hist, const double* x);
void    ws_num_samples(b2s_solver* s, int32_t* n, int64_t* rows);
void    ws_put_sample(b2s_solver* s, int32_t rows, const float* feat, const float* Hs, const float* q,
                      const float* c0, double norm);
void    ws_fit_normalization(b2s_solver* s);
double  ws_train(b2s_solver* s, int epochs, double lr, uint64_t seed);
double  ws_loss_grad(b2s_solver* s, int index, float* h_grad);
int64_t ws_get_params(b2s_solver* s, float* h);
void    ws_set_params(b2s_solver* s, const float* h, int64_t n);
int     ws_get_sample(b2s_solver* s, int index, float* feat, float* Hs, float* q, float* c0, double* norm);
void    ws_predict(b2s_solver* s, int mode, const double* b, int n_hist, const double* const* hist, double* x0,
                   b2s_ws_info* info);

inline int grid_for(int64_t n, int block) { return (int)((n + block - 1) / block); }
}  // namespace b2s
