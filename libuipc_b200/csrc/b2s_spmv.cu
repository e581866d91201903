// Symmetric block SpMV from block-upper storage, with the fused x.(A x).
//
// Semantics: y = (U + U^T - diag U) x at block level, as Spmv::cpu_sym_spmv
// (src/backends/cuda/linear_system/spmv.cu:1210-1297) and the default
// Spmv_rbk_sym_spmv_dot_chunked_kernel (:531-760): each stored block (i, j)
// adds B x_j to y_i and, off the diagonal, B^T x_i to y_j; the dot is
// sum (2 - delta_ij) x_i^T B x_j.
//
// Design: one persistent CTA per SM streams a contiguous range of the block
// stream through a 4-stage shared-memory ring filled by bulk asynchronous
// copies (cp.async.bulk, TMA) -- row ids, column ids and the 9 value planes
// of 512 blocks per stage -- so the DRAM stream runs ahead of the threads
// independently of their register-bound loads. Each thread takes one block
// of a stage: it gathers x_j and x_i (L2-resident), forms B x_j and B^T x_i,
// the warp merges runs of equal rows with an in-register segmented scan and
// writes one atomic per run, and the transposed contributions scatter with
// atomics that resolve in L2.
#include "b2s_internal.cuh"
#include "b2s_reduce.cuh"

#include <cstdlib>
#include <string>

namespace b2s
{
namespace
{
constexpr int SPMV_THREADS = SPMV_TILE;  // = blocks per tile

// fire-and-forget reductions in L2 (no value returned to the SM)
__device__ __forceinline__ void atomic_add_t(double* p, double v)
{
    asm volatile("red.global.add.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
__device__ __forceinline__ void atomic_add_t(float* p, float v)
{
    asm volatile("red.global.add.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}

// warp-level segmented inclusive scan of (a0,a1,a2) over equal keys; returns
// true in the last lane of each run
template <typename XT>
__device__ __forceinline__ bool seg_scan3(int32_t key, XT& a0, XT& a1, XT& a2, int lane)
{
#pragma unroll
    for(int o = 1; o < 32; o <<= 1)
    {
        const XT      t0 = __shfl_up_sync(0xffffffffu, a0, o);
        const XT      t1 = __shfl_up_sync(0xffffffffu, a1, o);
        const XT      t2 = __shfl_up_sync(0xffffffffu, a2, o);
        const int32_t tk = __shfl_up_sync(0xffffffffu, key, o);
        if(lane >= o && tk == key)
        {
            a0 += t0;
            a1 += t1;
            a2 += t2;
        }
    }
    const int32_t knext = __shfl_down_sync(0xffffffffu, key, 1);
    return lane == 31 || knext != key;
}

// Tile variant: a 512-thread CTA takes one 512-block tile at a time with
// plain coalesced loads. The row part is merged in-warp (runs of equal rows);
// the transposed contributions are placed in shared memory at the block's
// precomputed rank in (column, index) order, so runs of equal columns become
// contiguous and are merged by a second segmented scan before the reductions
// go to L2 -- about half the reduction traffic of a direct scatter.
template <typename VT, typename XT, bool WITH_DOT>
__global__ void __launch_bounds__(SPMV_THREADS, 3)
    k_spmv_tile(int64_t U, int64_t S, const int32_t* __restrict__ rows, const int32_t* __restrict__ cols,
                const uint16_t* __restrict__ trank, const VT* __restrict__ vals, const XT* __restrict__ x, XT* y,
                double* partials, unsigned int* counter, double* dot_out, const int* stop)
{
    if(stop && *stop)
        return;
    __shared__ XT      s_t[3][SPMV_THREADS];
    __shared__ int32_t s_col[SPMV_THREADS];
    const int     tid     = threadIdx.x;
    const int     lane    = tid & 31;
    const int64_t n_tiles = (U + SPMV_THREADS - 1) / SPMV_THREADS;
    double        dot     = 0.0;
    for(int64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x)
    {
        const int64_t base = tile * SPMV_THREADS;
        const int64_t rem  = U - base;
        const int     n    = rem < SPMV_THREADS ? (int)rem : SPMV_THREADS;
        const int64_t k    = base + tid;
        int32_t       r    = -1;
        XT            a0 = 0, a1 = 0, a2 = 0;
        if(tid < n)
        {
            r               = __ldg(rows + k);
            const int32_t c = __ldg(cols + k);
            const int     rk = __ldg(trank + k);
            XT b[9];
#pragma unroll
            for(int q = 0; q < 9; ++q)
                b[q] = (XT)__ldg(vals + (int64_t)q * S + k);
            const XT xj0 = __ldg(x + 3 * (int64_t)c), xj1 = __ldg(x + 3 * (int64_t)c + 1),
                     xj2 = __ldg(x + 3 * (int64_t)c + 2);
            const XT xi0 = __ldg(x + 3 * (int64_t)r), xi1 = __ldg(x + 3 * (int64_t)r + 1),
                     xi2 = __ldg(x + 3 * (int64_t)r + 2);
            // column-major: B(p,q) = b[q*3 + p]
            a0 = b[0] * xj0 + b[3] * xj1 + b[6] * xj2;
            a1 = b[1] * xj0 + b[4] * xj1 + b[7] * xj2;
            a2 = b[2] * xj0 + b[5] * xj1 + b[8] * xj2;
            const double d = (double)xi0 * (double)a0 + (double)xi1 * (double)a1 + (double)xi2 * (double)a2;
            const bool   off = r != c;
            s_t[0][rk] = off ? b[0] * xi0 + b[1] * xi1 + b[2] * xi2 : XT(0);
            s_t[1][rk] = off ? b[3] * xi0 + b[4] * xi1 + b[5] * xi2 : XT(0);
            s_t[2][rk] = off ? b[6] * xi0 + b[7] * xi1 + b[8] * xi2 : XT(0);
            s_col[rk]  = c;
            if(WITH_DOT)
                dot += off ? 2.0 * d : d;
        }
        if(seg_scan3<XT>(r, a0, a1, a2, lane) && r >= 0)
        {
            atomic_add_t(y + 3 * (int64_t)r, a0);
            atomic_add_t(y + 3 * (int64_t)r + 1, a1);
            atomic_add_t(y + 3 * (int64_t)r + 2, a2);
        }
        __syncthreads();
        int32_t tc = -1;
        XT      t0 = 0, t1 = 0, t2 = 0;
        if(tid < n)
        {
            tc = s_col[tid];
            t0 = s_t[0][tid];
            t1 = s_t[1][tid];
            t2 = s_t[2][tid];
        }
        if(seg_scan3<XT>(tc, t0, t1, t2, lane) && tc >= 0)
        {
            atomic_add_t(y + 3 * (int64_t)tc, t0);
            atomic_add_t(y + 3 * (int64_t)tc + 1, t1);
            atomic_add_t(y + 3 * (int64_t)tc + 2, t2);
        }
        __syncthreads();
    }
    if(WITH_DOT)
    {
        double v[1] = {dot}, tot[1];
        if(grid_sum<1>(v, partials, counter, tot))
            *dot_out = tot[0];
    }
}

// Many-warp variant: one thread per block, grid-stride, no staging; the
// warp merges runs of equal rows, the transposed half scatters directly.
constexpr int WARP_KERNEL_BLOCK = 256;

template <typename VT, typename XT, bool WITH_DOT>
__global__ void __launch_bounds__(WARP_KERNEL_BLOCK)
    k_spmv_warp(int64_t U, int64_t S, const int32_t* __restrict__ rows, const int32_t* __restrict__ cols,
                const VT* __restrict__ vals, const XT* __restrict__ x, XT* y, double* partials,
                unsigned int* counter, double* dot_out, const int* stop)
{
    if(stop && *stop)
        return;
    const int     lane   = threadIdx.x & 31;
    double        dot    = 0.0;
    const int64_t stride = (int64_t)gridDim.x * WARP_KERNEL_BLOCK;
    for(int64_t base = (int64_t)blockIdx.x * WARP_KERNEL_BLOCK; base < U; base += stride)
    {
        const int64_t k = base + threadIdx.x;
        int32_t       r = -1;
        XT            a0 = 0, a1 = 0, a2 = 0;
        if(k < U)
        {
            r               = __ldg(rows + k);
            const int32_t c = __ldg(cols + k);
            XT b[9];
#pragma unroll
            for(int q = 0; q < 9; ++q)
                b[q] = (XT)__ldg(vals + (int64_t)q * S + k);
            const XT xj0 = __ldg(x + 3 * (int64_t)c), xj1 = __ldg(x + 3 * (int64_t)c + 1),
                     xj2 = __ldg(x + 3 * (int64_t)c + 2);
            const XT xi0 = __ldg(x + 3 * (int64_t)r), xi1 = __ldg(x + 3 * (int64_t)r + 1),
                     xi2 = __ldg(x + 3 * (int64_t)r + 2);
            a0 = b[0] * xj0 + b[3] * xj1 + b[6] * xj2;
            a1 = b[1] * xj0 + b[4] * xj1 + b[7] * xj2;
            a2 = b[2] * xj0 + b[5] * xj1 + b[8] * xj2;
            const double d = (double)xi0 * (double)a0 + (double)xi1 * (double)a1 + (double)xi2 * (double)a2;
            if(r != c)
            {
                atomic_add_t(y + 3 * (int64_t)c, b[0] * xi0 + b[1] * xi1 + b[2] * xi2);
                atomic_add_t(y + 3 * (int64_t)c + 1, b[3] * xi0 + b[4] * xi1 + b[5] * xi2);
                atomic_add_t(y + 3 * (int64_t)c + 2, b[6] * xi0 + b[7] * xi1 + b[8] * xi2);
                if(WITH_DOT)
                    dot += 2.0 * d;
            }
            else if(WITH_DOT)
                dot += d;
        }
        if(seg_scan3<XT>(r, a0, a1, a2, lane) && r >= 0)
        {
            atomic_add_t(y + 3 * (int64_t)r, a0);
            atomic_add_t(y + 3 * (int64_t)r + 1, a1);
            atomic_add_t(y + 3 * (int64_t)r + 2, a2);
        }
    }
    if(WITH_DOT)
    {
        double v[1] = {dot}, tot[1];
        if(grid_sum<1>(v, partials, counter, tot))
            *dot_out = tot[0];
    }
}

// kernel selection: "tile" (default) or "warp", from B2S_SPMV_KERNEL, read once
int spmv_variant()
{
    static const int v = []
    {
        const char* e = std::getenv("B2S_SPMV_KERNEL");
        return (e && std::string(e) == "warp") ? 0 : 1;
    }();
    return v;
}

int tile_grid(int64_t U)
{
    const int64_t t = (U + SPMV_THREADS - 1) / SPMV_THREADS;
    return (int)std::max<int64_t>(1, std::min<int64_t>(t, (int64_t)NUM_SMS_HINT * 3));
}

int warp_grid(int64_t U)
{
    const int64_t g = (U + WARP_KERNEL_BLOCK - 1) / WARP_KERNEL_BLOCK;
    return (int)std::max<int64_t>(1, std::min<int64_t>(g, (int64_t)NUM_SMS_HINT * 8));
}

template <typename VT, typename XT, bool DOT>
void launch_stream(cudaStream_t st, int64_t U, int64_t S, const int32_t* rows, const int32_t* cols,
                   const uint16_t* trank, const VT* vals, const XT* x, XT* y, Reduction* red, double* d_dot,
                   const int* stop, int* err)
{
    if(spmv_variant() == 0)
    {
        k_spmv_warp<VT, XT, DOT><<<warp_grid(U), WARP_KERNEL_BLOCK, 0, st>>>(
            U, S, rows, cols, vals, x, y, red ? red->partials.data() : nullptr, red ? red->counter.data() : nullptr,
            d_dot, stop);
        B2S_CHECK_LAUNCH();
        return;
    }
    k_spmv_tile<VT, XT, DOT><<<tile_grid(U), SPMV_THREADS, 0, st>>>(
        U, S, rows, cols, trank, vals, x, y, red ? red->partials.data() : nullptr,
        red ? red->counter.data() : nullptr, d_dot, stop);
    B2S_CHECK_LAUNCH();
}
}  // namespace

int spmv_grid(int64_t U)
{
    return std::max(tile_grid(U), warp_grid(U));
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
    int* err = device_error_flag(s);
    B2S_REQUIRE(A.has_trank, B2S_ERR_STATE, "matrix lacks the SpMV tile ranks");
    ensure_reduction(s->red, spmv_grid(A.nnz), 1);
    if(d_dot)
        launch_stream<double, double, true>(st, A.nnz, A.stride, A.rows.data(), A.cols.data(), A.trank.data(), A.vals.data(), x, y,
                                            &s->red, d_dot, nullptr, err);
    else
        launch_stream<double, double, false>(st, A.nnz, A.stride, A.rows.data(), A.cols.data(), A.trank.data(), A.vals.data(), x,
                                             y, nullptr, nullptr, nullptr, err);
}

// launch shared with the PCG graph (y must be zero beforehand)
void spmv_f64_launch(b2s_solver* s, const Matrix& A, const double* x, double* y, Reduction& red, double* d_dot,
                     const int* stop)
{
    if(A.nnz == 0)
        return;
    launch_stream<double, double, true>(s->stream, A.nnz, A.stride, A.rows.data(), A.cols.data(), A.trank.data(), A.vals.data(), x,
                                        y, &red, d_dot, stop, device_error_flag(s));
}

// FP32 values and vectors (mixed precision), FP64 dot
void spmv_f32_launch(b2s_solver* s, const Matrix& A, const float* x, float* y, Reduction& red, double* d_dot,
                     const int* stop)
{
    if(A.nnz == 0)
        return;
    launch_stream<float, float, true>(s->stream, A.nnz, A.stride, A.rows.data(), A.cols.data(), A.trank.data(), A.vals32.data(), x,
                                      y, &red, d_dot, stop, device_error_flag(s));
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
}  // namespace

int reduction_grid() { return NUM_SMS_HINT * 4; }

void launch_dot(b2s_solver* s, const double* a, const double* b, int64_t n, double* d_out)
{
    const int grid = reduction_grid();
    ensure_reduction(s->red, grid, 1);
    k_dot<<<grid, RED_BLOCK, 0, s->stream>>>(a, b, n, s->red.partials.data(), s->red.counter.data(), d_out);
    B2S_CHECK_LAUNCH();
}
}  // namespace b2s
