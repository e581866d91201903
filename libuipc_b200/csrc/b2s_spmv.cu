// Symmetric block SpMV from block-upper storage, with the fused x.(A x).
//
// Semantics: y = (U + U^T - diag U) x at block level, as Spmv::cpu_sym_spmv
// (src/backends/cuda/linear_system/spmv.cu:1210-1297) and the default
// Spmv_rbk_sym_spmv_dot_chunked_kernel (:531-760): each stored block (i, j)
// adds B x_j to y_i and, off the diagonal, B^T x_i to y_j; the dot is
// sum (2 - delta_ij) x_i^T B x_j.
//
// Design, FP64 values (k_spmv_tile): persistent CTAs walk SPMV_TILE-block
// tiles of the row-sorted block stream. Each thread owns SPMV_BPT consecutive
// blocks and reads their row and column ids, tile ranks and the 9 value planes
// with 16-byte vector loads (the planes are padded to a multiple of 16
// blocks). The row halves B x_j of a thread's blocks are merged in registers
// (runs of equal rows) and each run goes to y with one fire-and-forget
// reduction per component (red.global, resolved in L2). The transposed halves
// B^T x_i are placed in shared memory at the block's precomputed rank in
// (column, index) order; after a barrier each thread merges its SPMV_BPT
// consecutive slots, so runs of equal columns also leave as one reduction
// each (~0.62 of the measured HBM bandwidth on 4.25 M blocks).
// FP32 values (k_spmv_direct, mixed precision): the same row runs, but every
// transposed half leaves as one vector reduction of the padded node and the
// kernel holds no shared memory and no barrier (~0.77).
#include "b2s_internal.cuh"
#include "b2s_reduce.cuh"

#include <algorithm>
#include <cstdlib>
#include <string>

namespace b2s
{
namespace
{
constexpr int SPMV_BPT     = 4;                     // blocks per thread
constexpr int SPMV_THREADS = SPMV_TILE / SPMV_BPT;  // threads per CTA

// fire-and-forget reductions in L2 (no value returned to the SM)
__device__ __forceinline__ void atomic_add_t(double* p, double v)
{
    asm volatile("red.global.add.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
__device__ __forceinline__ void atomic_add_t(float* p, float v)
{
    asm volatile("red.global.add.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}

// four consecutive elements from a 16-byte (8-byte for uint16) aligned address
__device__ __forceinline__ void ld4(const float* p, float v[4])
{
    const float4 q = __ldg(reinterpret_cast<const float4*>(p));
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
__device__ __forceinline__ void ld4(const double* p, double v[4])
{
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void ld4(const int32_t* p, int32_t v[4])
{
    const int4 q = __ldg(reinterpret_cast<const int4*>(p));
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
__device__ __forceinline__ void ld4(const uint16_t* p, int v[4])
{
    const uint2 q = __ldg(reinterpret_cast<const uint2*>(p));
    v[0] = (int)(q.x & 0xFFFFu); v[1] = (int)(q.x >> 16); v[2] = (int)(q.y & 0xFFFFu); v[3] = (int)(q.y >> 16);
}

// A node's three components. P4: the padded FP32 vectors of the mixed PCG
// (4 floats per node, the 4th zero): one 16-byte load, one vector reduction;
// otherwise 3 values per node (FP64 vectors).
template <typename XT, bool P4>
__device__ __forceinline__ void load_node(const XT* __restrict__ x, int32_t node, XT& a, XT& b, XT& c)
{
    if constexpr(P4)
    {
        const float4 q = __ldg(reinterpret_cast<const float4*>(x) + node);
        a = q.x;
        b = q.y;
        c = q.z;
    }
    else
    {
        a = __ldg(x + 3 * (int64_t)node);
        b = __ldg(x + 3 * (int64_t)node + 1);
        c = __ldg(x + 3 * (int64_t)node + 2);
    }
}

template <typename XT, bool P4>
__device__ __forceinline__ void red_node(XT* y, int32_t node, XT a0, XT a1, XT a2)
{
    if constexpr(P4)
        asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(y + 4 * (int64_t)node), "f"(a0), "f"(a1),
                     "f"(a2), "f"(0.0f)
                     : "memory");
    else
    {
        atomic_add_t(y + 3 * (int64_t)node, a0);
        atomic_add_t(y + 3 * (int64_t)node + 1, a1);
        atomic_add_t(y + 3 * (int64_t)node + 2, a2);
    }
}

// the streamed data of one thread's SPMV_BPT blocks
template <typename VT>
struct TileLoad
{
    int32_t r[4], c[4];
    int     rk[4];
    VT      b[9][4];
};

// S: plane stride (a multiple of 16, rows past the stored blocks are -1)
template <typename VT>
__device__ __forceinline__ void load_tile(TileLoad<VT>& t, int64_t e0, int64_t S, bool live,
                                          const int32_t* __restrict__ rows, const int32_t* __restrict__ cols,
                                          const uint16_t* __restrict__ trank, const VT* __restrict__ vals)
{
    if(!live)
    {
#pragma unroll
        for(int k = 0; k < 4; ++k)
            t.r[k] = -1;
        return;
    }
    ld4(rows + e0, t.r);
    ld4(cols + e0, t.c);
    ld4(trank + e0, t.rk);
#pragma unroll
    for(int q = 0; q < 9; ++q)
        ld4(vals + (int64_t)q * S + e0, t.b[q]);
}

// row halves of a thread's blocks to y (runs of equal rows merged), the
// transposed halves into shared memory at the blocks' ranks, and the dot
template <typename VT, typename XT, bool WITH_DOT>
__device__ __forceinline__ void tile_rows(const TileLoad<VT>& t, const XT* __restrict__ x, XT* y,
                                          XT (*s_t)[SPMV_TILE], int32_t* s_col, double& dot)
{
    int32_t cur = -1;
    XT      a0 = 0, a1 = 0, a2 = 0;
    XT      xi0 = 0, xi1 = 0, xi2 = 0;
#pragma unroll
    for(int k = 0; k < 4; ++k)
    {
        if(t.r[k] < 0)
            break;  // padding: only at the end of the stream
        const int32_t ck = t.c[k];
        XT            xj0, xj1, xj2;
        load_node<XT, false>(x, ck, xj0, xj1, xj2);
        if(t.r[k] != cur)
        {
            if(cur >= 0)
                red_node<XT, false>(y, cur, a0, a1, a2);
            cur = t.r[k];
            a0 = a1 = a2 = 0;
            load_node<XT, false>(x, cur, xi0, xi1, xi2);
        }
        // column-major: B(p,q) = b[q*3 + p]
        const XT y0 = (XT)t.b[0][k] * xj0 + (XT)t.b[3][k] * xj1 + (XT)t.b[6][k] * xj2;
        const XT y1 = (XT)t.b[1][k] * xj0 + (XT)t.b[4][k] * xj1 + (XT)t.b[7][k] * xj2;
        const XT y2 = (XT)t.b[2][k] * xj0 + (XT)t.b[5][k] * xj1 + (XT)t.b[8][k] * xj2;
        a0 += y0;
        a1 += y1;
        a2 += y2;
        const bool off = cur != ck;
        if(WITH_DOT)
        {
            const double d = (double)xi0 * (double)y0 + (double)xi1 * (double)y1 + (double)xi2 * (double)y2;
            dot += off ? 2.0 * d : d;
        }
        const int rk = t.rk[k];
        s_t[0][rk]   = off ? (XT)t.b[0][k] * xi0 + (XT)t.b[1][k] * xi1 + (XT)t.b[2][k] * xi2 : XT(0);
        s_t[1][rk]   = off ? (XT)t.b[3][k] * xi0 + (XT)t.b[4][k] * xi1 + (XT)t.b[5][k] * xi2 : XT(0);
        s_t[2][rk]   = off ? (XT)t.b[6][k] * xi0 + (XT)t.b[7][k] * xi1 + (XT)t.b[8][k] * xi2 : XT(0);
        s_col[rk]    = ck;
    }
    if(cur >= 0)
        red_node<XT, false>(y, cur, a0, a1, a2);
}

// transposed halves in (column, index) order: this thread's slots, runs of
// equal columns merged; n = blocks in the tile
template <typename XT>
__device__ __forceinline__ void tile_cols(int tid, int n, const XT (*s_t)[SPMV_TILE], const int32_t* s_col, XT* y)
{
    const int s0  = SPMV_BPT * tid;
    int32_t   cur = -1;
    XT        t0 = 0, t1 = 0, t2 = 0;
#pragma unroll
    for(int k = 0; k < SPMV_BPT; ++k)
    {
        const int sl = s0 + k;
        if(sl >= n)
            break;
        const int32_t cc = s_col[sl];
        if(cc != cur)
        {
            if(cur >= 0)
                red_node<XT, false>(y, cur, t0, t1, t2);
            cur = cc;
            t0 = t1 = t2 = 0;
        }
        t0 += s_t[0][sl];
        t1 += s_t[1][sl];
        t2 += s_t[2][sl];
    }
    if(cur >= 0)
        red_node<XT, false>(y, cur, t0, t1, t2);
}

// U: stored blocks; S: plane stride. FP64 values, loaded straight into
// registers (16-byte loads), one tile at a time.
template <typename VT, typename XT, bool WITH_DOT>
__global__ void __launch_bounds__(SPMV_THREADS)
    k_spmv_tile(int64_t U, int64_t S, const int32_t* __restrict__ rows, const int32_t* __restrict__ cols,
                const uint16_t* __restrict__ trank, const VT* __restrict__ vals, const XT* __restrict__ x, XT* y,
                double* partials, unsigned int* counter, double* dot_out, const int* stop)
{
    if(stop && *stop)
        return;
    __shared__ __align__(16) XT      s_t[3][SPMV_TILE];
    __shared__ __align__(16) int32_t s_col[SPMV_TILE];
    const int     tid     = threadIdx.x;
    const int64_t n_tiles = (U + SPMV_TILE - 1) / SPMV_TILE;
    double        dot     = 0.0;
    for(int64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x)
    {
        const int64_t rem = U - tile * SPMV_TILE;
        const int     n   = rem < SPMV_TILE ? (int)rem : SPMV_TILE;
        const int64_t e0  = tile * SPMV_TILE + SPMV_BPT * tid;
        TileLoad<VT>  cur;
        load_tile(cur, e0, S, e0 < S, rows, cols, trank, vals);
        tile_rows<VT, XT, WITH_DOT>(cur, x, y, s_t, s_col, dot);
        __syncthreads();
        tile_cols<XT>(tid, n, s_t, s_col, y);
        __syncthreads();
    }
    if(WITH_DOT)
    {
        double v[1] = {dot}, tot[1];
        if(grid_sum<1>(v, partials, counter, tot))
            *dot_out = tot[0];
    }
}

// FP32 values (mixed precision), streamed straight into registers: each
// thread takes SPMV_BPT consecutive blocks (16-byte streaming loads of the row
// and column ids and of the 9 value planes, marked evict-first so the stream
// does not push x and y out of L2), merges its row runs in registers as
// k_spmv_tile does, and sends each off-diagonal block's transposed half
// B^T x_i to y with its own red.global.add.v4.f32 -- no shared memory, no
// barriers, no tile ranks. x and y are the padded FP32 vectors of the mixed
// PCG (4 floats per node, the 4th zero): a gather is one 16-byte load, a
// reduction one vector red. 128-thread CTAs, six per SM (78 registers): with
// nothing to wait for but its own loads, each warp keeps 11 stream loads and
// its gathers in flight. Measured on the 8 x 40^3-cell stack (4.25 M blocks):
// 37.3 us (0.77 of the measured copy bandwidth) against 53.6 us (0.54) for a
// TMA-staged tile kernel with shared-memory-merged transposed halves, which
// saves reductions but serialises every tile behind its copy and two barriers.
// With FP64 values the per-component f64 reductions (no vector form) tip the
// balance the other way and k_spmv_tile stays.
constexpr int DIRECT_THREADS = 128;
constexpr int DIRECT_CTAS_SM = 6;

// Row ids without a per-block index (GROUPS): the stream is cut into groups
// of 128 blocks (one warp's 32 chunks); per group the row of its first block
// (grp_row) and a 128-bit mask whose bit k is set when block k starts a new
// row (grp_mask; rows without blocks do not occur, so every start is the
// next row). A thread's rows follow from the popcount of the mask bits up to
// its blocks: 20 bytes per 128 blocks instead of 4 bytes per block.
__device__ __forceinline__ void group_rows(const int32_t* __restrict__ grp_row, const uint4* __restrict__ grp_mask,
                                           int64_t c, int64_t U, int32_t r[4])
{
    const int64_t g  = c >> 5;
    const int     p  = (int)(c & 31) * SPMV_BPT;  // first block of the chunk in its group
    const uint4   m4 = __ldg(grp_mask + g);
    const int32_t r0 = __ldg(grp_row + g);
    const uint32_t w[4] = {m4.x, m4.y, m4.z, m4.w};
    const int      wi = p >> 5, bi = p & 31;
    int            cnt = 0;
#pragma unroll
    for(int j = 0; j < 3; ++j)
        cnt += j < wi ? __popc(w[j]) : 0;
    const uint32_t word = wi == 0 ? w[0] : wi == 1 ? w[1] : wi == 2 ? w[2] : w[3];
    cnt += __popc(word & ((2u << bi) - 1u));
    int32_t row = r0 + cnt;
#pragma unroll
    for(int k = 0; k < SPMV_BPT; ++k)
    {
        if(k > 0)
            row += (int32_t)((word >> (bi + k)) & 1u);
        r[k] = (c * SPMV_BPT + k < U) ? row : -1;
    }
}

template <bool WITH_DOT, bool GROUPS>
__global__ void __launch_bounds__(DIRECT_THREADS, DIRECT_CTAS_SM)
    k_spmv_direct(int64_t S, int64_t U, const int32_t* __restrict__ rows, const int32_t* __restrict__ grp_row,
                  const uint4* __restrict__ grp_mask, const int32_t* __restrict__ cols,
                  const float* __restrict__ vals, const float* __restrict__ x, float* y, double* partials,
                  unsigned int* counter, double* dot_out, const int* stop)
{
    if(stop && *stop)
        return;
    const int64_t n_chunks = S / SPMV_BPT;  // S is a multiple of 16
    double        dot      = 0.0;
    for(int64_t c = (int64_t)blockIdx.x * DIRECT_THREADS + threadIdx.x; c < n_chunks;
        c += (int64_t)gridDim.x * DIRECT_THREADS)
    {
        const int64_t e0 = c * SPMV_BPT;
        int32_t       r[4];
        if constexpr(GROUPS)
            group_rows(grp_row, grp_mask, c, U, r);
        else
        {
            const int4 r4 = __ldcs(reinterpret_cast<const int4*>(rows + e0));
            r[0] = r4.x, r[1] = r4.y, r[2] = r4.z, r[3] = r4.w;
        }
        const int4    c4 = __ldcs(reinterpret_cast<const int4*>(cols + e0));
        const int32_t cc[4] = {c4.x, c4.y, c4.z, c4.w};
        float         b[9][4];
#pragma unroll
        for(int q = 0; q < 9; ++q)
        {
            const float4 v = __ldcs(reinterpret_cast<const float4*>(vals + (int64_t)q * S + e0));
            b[q][0] = v.x; b[q][1] = v.y; b[q][2] = v.z; b[q][3] = v.w;
        }
        int32_t cur = -1;
        float   a0 = 0.f, a1 = 0.f, a2 = 0.f, xi0 = 0.f, xi1 = 0.f, xi2 = 0.f;
#pragma unroll
        for(int k = 0; k < SPMV_BPT; ++k)
        {
            if(r[k] < 0)
                break;  // padding: only at the end of the stream
            const int32_t ck = cc[k];
            float         xj0, xj1, xj2;
            load_node<float, true>(x, ck, xj0, xj1, xj2);
            if(r[k] != cur)
            {
                if(cur >= 0)
                    red_node<float, true>(y, cur, a0, a1, a2);
                cur = r[k];
                a0 = a1 = a2 = 0.f;
                load_node<float, true>(x, cur, xi0, xi1, xi2);
            }
            // column-major: B(p,q) = b[q*3 + p]
            const float y0 = b[0][k] * xj0 + b[3][k] * xj1 + b[6][k] * xj2;
            const float y1 = b[1][k] * xj0 + b[4][k] * xj1 + b[7][k] * xj2;
            const float y2 = b[2][k] * xj0 + b[5][k] * xj1 + b[8][k] * xj2;
            a0 += y0;
            a1 += y1;
            a2 += y2;
            const bool off = cur != ck;
            if(WITH_DOT)
            {
                const double d = (double)xi0 * (double)y0 + (double)xi1 * (double)y1 + (double)xi2 * (double)y2;
                dot += off ? 2.0 * d : d;
            }
            if(off)
                red_node<float, true>(y, ck, b[0][k] * xi0 + b[1][k] * xi1 + b[2][k] * xi2,
                                      b[3][k] * xi0 + b[4][k] * xi1 + b[5][k] * xi2,
                                      b[6][k] * xi0 + b[7][k] * xi1 + b[8][k] * xi2);
        }
        if(cur >= 0)
            red_node<float, true>(y, cur, a0, a1, a2);
    }
    if(WITH_DOT)
    {
        double v[1] = {dot}, tot[1];
        if(grid_sum<1>(v, partials, counter, tot))
            *dot_out = tot[0];
    }
}

// persistent grid: the CTAs that fit on the SMs at once, capped by the tiles
// (and by spmv_grid, which sizes the reduction partials)
template <typename K>
int tile_grid(K kernel, int64_t U)
{
    int occ = 0;
    if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, SPMV_THREADS, 0) != cudaSuccess || occ < 1)
        occ = 1;
    const int64_t t = (U + SPMV_TILE - 1) / SPMV_TILE;
    const int64_t g = std::min<int64_t>(t, (int64_t)NUM_SMS_HINT * std::min(occ, 8));
    return (int)std::max<int64_t>(1, g);
}

template <typename VT, typename XT, bool DOT>
void launch_stream(cudaStream_t st, int64_t U, int64_t S, const int32_t* rows, const int32_t* cols,
                   const uint16_t* trank, const VT* vals, const XT* x, XT* y, Reduction* red, double* d_dot,
                   const int* stop)
{
    auto k = k_spmv_tile<VT, XT, DOT>;
    k<<<tile_grid(k, U), SPMV_THREADS, 0, st>>>(U, S, rows, cols, trank, vals, x, y,
                                                red ? red->partials.data() : nullptr,
                                                red ? red->counter.data() : nullptr, d_dot, stop);
    B2S_CHECK_LAUNCH();
}
}  // namespace

// the largest grid any SpMV kernel launches for U blocks (sizes the dot partials)
int spmv_grid(int64_t U)
{
    const int64_t t = (U + SPMV_BPT * DIRECT_THREADS - 1) / (SPMV_BPT * DIRECT_THREADS);
    return (int)std::max<int64_t>(1, std::min<int64_t>(t, (int64_t)NUM_SMS_HINT * 8));
}

void ensure_reduction(Reduction& red, int grid, int nv)
{
    if(red.partials.size() < (size_t)grid * nv)
        red.partials.resize((size_t)grid * nv);
    if(red.counter.size() < 1)
    {
        red.counter.resize(1);
        B2S_CUDA(cudaMemset(red.counter.data(), 0, sizeof(unsigned int)));
    }
}

int* device_error_flag(b2s_solver* s)
{
    if(s->dev_err.size() < 1)
    {
        s->dev_err.resize(1);
        B2S_CUDA(cudaMemset(s->dev_err.data(), 0, sizeof(int)));
    }
    return s->dev_err.data();
}

// raise (and clear) the error bits kernels left in the device flag
void check_device_errors(b2s_solver* s)
{
    if(s->dev_err.size() < 1)
        return;
    int h = 0;
    B2S_CUDA(cudaMemcpyAsync(&h, s->dev_err.data(), sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    B2S_CUDA(cudaStreamSynchronize(s->stream));
    if(h != 0)
    {
        B2S_CUDA(cudaMemsetAsync(s->dev_err.data(), 0, sizeof(int), s->stream));
        B2S_CUDA(cudaStreamSynchronize(s->stream));
        throw Error(B2S_ERR_CUDA, std::string("device error flag ") + std::to_string(h)
                                      + ((h & DERR_TMA_TIMEOUT) ? ": a bulk-copy wait timed out" : ""));
    }
}

// y = A x; y is overwritten. d_dot (device) receives x.(A x) when non-null.
void spmv_f64(b2s_solver* s, const Matrix& A, const double* x, double* y, double* d_dot)
{
    cudaStream_t st = s->stream;
    B2S_CUDA(cudaMemsetAsync(y, 0, sizeof(double) * 3 * (size_t)A.nb, st));
    if(A.nnz == 0)
    {
        if(d_dot)
            B2S_CUDA(cudaMemsetAsync(d_dot, 0, sizeof(double), st));
        return;
    }
    B2S_REQUIRE(A.has_trank, B2S_ERR_STATE, "matrix lacks the SpMV tile ranks");
    ensure_reduction(s->red, spmv_grid(A.nnz), 1);
    if(d_dot)
        launch_stream<double, double, true>(st, A.nnz, A.stride, A.rows.data(), A.cols.data(), A.trank.data(), A.vals.data(), x, y,
                                            &s->red, d_dot, nullptr);
    else
        launch_stream<double, double, false>(st, A.nnz, A.stride, A.rows.data(), A.cols.data(), A.trank.data(), A.vals.data(), x,
                                             y, nullptr, nullptr, nullptr);
}

// launch shared with the PCG graph (y must be zero beforehand)
void spmv_f64_launch(b2s_solver* s, const Matrix& A, const double* x, double* y, Reduction& red, double* d_dot,
                     const int* stop)
{
    if(A.nnz == 0)
        return;
    launch_stream<double, double, true>(s->stream, A.nnz, A.stride, A.rows.data(), A.cols.data(), A.trank.data(), A.vals.data(), x,
                                        y, &red, d_dot, stop);
}

// FP32 values and padded FP32 vectors (mixed precision), FP64 dot
void spmv_f32_launch(b2s_solver* s, const Matrix& A, const float* x, float* y, Reduction& red, double* d_dot,
                     const int* stop)
{
    if(A.nnz == 0)
        return;
    const bool grp = A.has_groups;
    auto       k   = grp ? k_spmv_direct<true, true> : k_spmv_direct<true, false>;
    int        occ = 0;
    if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, DIRECT_THREADS, 0) != cudaSuccess || occ < 1)
        occ = 1;
    const int64_t ctas = (A.stride / SPMV_BPT + DIRECT_THREADS - 1) / DIRECT_THREADS;
    const int     grid = (int)std::max<int64_t>(
        1, std::min<int64_t>({ctas, (int64_t)NUM_SMS_HINT * std::min(occ, DIRECT_CTAS_SM), (int64_t)spmv_grid(A.nnz)}));
    k<<<grid, DIRECT_THREADS, 0, s->stream>>>(A.stride, A.nnz, A.rows.data(), grp ? A.grp_row.data() : nullptr,
                                              grp ? A.grp_mask.data() : nullptr, A.cols.data(), A.vals32.data(), x,
                                              y, red.partials.data(), red.counter.data(), d_dot, stop);
    B2S_CHECK_LAUNCH();
}

namespace
{
// per group of 128 blocks: the first block's row and the row-start mask
// (one warp per group); *gap is set when a row start skips a row (a row
// without blocks), and the FP32 SpMV then keeps reading the row ids
__global__ void k_row_groups(int64_t U, int64_t n_groups, const int32_t* __restrict__ rows,
                             int32_t* __restrict__ grp_row, uint4* __restrict__ grp_mask, int* gap)
{
    const int     lane = threadIdx.x & 31;
    const int64_t g    = (int64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    if(g >= n_groups)
        return;
    const int64_t e0 = g * 128 + 4 * lane;
    int32_t       r[4];
#pragma unroll
    for(int k = 0; k < 4; ++k)
        r[k] = e0 + k < U ? rows[e0 + k] : -1;
    const int32_t prev = __shfl_up_sync(0xffffffffu, r[3], 1);
    uint32_t      nib  = 0;
    bool          bad  = false;
#pragma unroll
    for(int k = 0; k < 4; ++k)
    {
        const int32_t before = k == 0 ? prev : r[k - 1];
        if(r[k] < 0 || (k == 0 && lane == 0))
            continue;
        if(r[k] != before)
        {
            nib |= 1u << k;
            bad |= r[k] != before + 1;
        }
    }
    uint32_t word = nib << (4 * (lane & 7));
#pragma unroll
    for(int o = 1; o < 8; o <<= 1)
        word |= __shfl_xor_sync(0xffffffffu, word, o);
    const uint32_t w0 = __shfl_sync(0xffffffffu, word, 0), w1 = __shfl_sync(0xffffffffu, word, 8);
    const uint32_t w2 = __shfl_sync(0xffffffffu, word, 16), w3 = __shfl_sync(0xffffffffu, word, 24);
    if(lane == 0)
    {
        grp_row[g]  = r[0];
        grp_mask[g] = make_uint4(w0, w1, w2, w3);
    }
    if(__any_sync(0xffffffffu, bad) && lane == 0)
        atomicOr(gap, 1);
}
}  // namespace

// the row-start groups of the FP32 SpMV (once per assembly, beside the FP32 planes)
void build_row_groups(b2s_solver* s, Matrix& A)
{
    A.has_groups = false;
    if(A.nnz == 0)
        return;
    const int64_t G = (A.nnz + 127) / 128;
    A.grp_row.resize(G, 1.2);
    A.grp_mask.resize(G, 1.2);
    s->asmb.err.resize(1);
    B2S_CUDA(cudaMemsetAsync(s->asmb.err.data(), 0, sizeof(int), s->stream));
    k_row_groups<<<(unsigned)((G + 7) / 8), 256, 0, s->stream>>>(A.nnz, G, A.rows.data(), A.grp_row.data(),
                                                                 A.grp_mask.data(), s->asmb.err.data());
    B2S_CHECK_LAUNCH();
    int h = 0;
    B2S_CUDA(cudaMemcpyAsync(&h, s->asmb.err.data(), sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    B2S_CUDA(cudaStreamSynchronize(s->stream));
    A.has_groups = h == 0;
}

// ---------------------------------------------------------------------------
// plain dot product (deterministic)
// ---------------------------------------------------------------------------
namespace
{
__global__ void __launch_bounds__(RED_BLOCK) k_dot(const double* __restrict__ a, const double* __restrict__ b,
                                                   int64_t n, double* partials, unsigned int* counter,
                                                   double* out)
{
    double acc = 0.0;
    for(int64_t i = (int64_t)blockIdx.x * RED_BLOCK + threadIdx.x; i < n; i += (int64_t)gridDim.x * RED_BLOCK)
        acc += a[i] * b[i];
    double v[1] = {acc}, tot[1];
    if(grid_sum<1>(v, partials, counter, tot))
        *out = tot[0];
}

// m <= MAX_DOTS dot products of n-vectors in one pass (repeated vectors are
// read once from DRAM, the rest from cache); out[k] = a_k . b_k
__global__ void __launch_bounds__(RED_BLOCK) k_multi_dot(int64_t n, int m, DotPairs d, double* partials,
                                                         unsigned int* counter, double* out)
{
    double acc[MAX_DOTS] = {};
    for(int64_t i = (int64_t)blockIdx.x * RED_BLOCK + threadIdx.x; i < n; i += (int64_t)gridDim.x * RED_BLOCK)
#pragma unroll
        for(int k = 0; k < MAX_DOTS; ++k)
            if(k < m)
                acc[k] += d.a[k][i] * d.b[k][i];
    double tot[MAX_DOTS];
    if(grid_sum<MAX_DOTS>(acc, partials, counter, tot))
        for(int k = 0; k < m; ++k)
            out[k] = tot[k];
}
}  // namespace

void launch_dots(b2s_solver* s, int64_t n, const DotPairs& d, int m, double* d_out)
{
    B2S_REQUIRE(m >= 1 && m <= MAX_DOTS, B2S_ERR_ARGUMENT, "launch_dots: 1 to MAX_DOTS products");
    const int grid = reduction_grid();
    ensure_reduction(s->red, grid, MAX_DOTS);
    k_multi_dot<<<grid, RED_BLOCK, 0, s->stream>>>(n, m, d, s->red.partials.data(), s->red.counter.data(), d_out);
    B2S_CHECK_LAUNCH();
}

// blocks of the grid-stride reductions and of the preconditioner collect (8
// per SM; 16 measured slower: the last block's in-order sum of the partials
// grows with the grid)
int reduction_grid() { return NUM_SMS_HINT * 8; }

void launch_dot(b2s_solver* s, const double* a, const double* b, int64_t n, double* d_out)
{
    const int grid = reduction_grid();
    ensure_reduction(s->red, grid, 1);
    k_dot<<<grid, RED_BLOCK, 0, s->stream>>>(a, b, n, s->red.partials.data(), s->red.counter.data(), d_out);
    B2S_CHECK_LAUNCH();
}
}  // namespace b2s
