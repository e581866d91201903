// Symmetric block SpMV from block-upper storage, with the fused x.(A x).
//
// Semantics: y = (U + U^T - diag U) x at block level, as Spmv::cpu_sym_spmv
// (src/backends/cuda/linear_system/spmv.cu:1210-1297) and the default
// Spmv_rbk_sym_spmv_dot_chunked_kernel (:531-760): each stored block (i, j)
// adds B x_j to y_i and, off the diagonal, B^T x_i to y_j; the dot is
// sum (2 - delta_ij) x_i^T B x_j.
//
// Layout: the 9 components of the blocks live in 9 planes (vals[q*U + k]), so
// every component load of a warp is one fully coalesced 256-byte request; the
// row indices are sorted, so a warp's row contributions are combined by an
// in-register segmented scan and written with one atomic per run; the
// transposed contributions scatter with FP64 atomics that resolve in L2 (the
// vectors of the largest systems fit in the 126 MB L2).
#include "b2s_internal.cuh"
#include "b2s_reduce.cuh"

namespace b2s
{
namespace
{
constexpr int SPMV_BLOCK = 256;

template <bool WITH_DOT>
__global__ void __launch_bounds__(SPMV_BLOCK) k_spmv_sym_f64(int64_t U, const int32_t* __restrict__ rows,
                                                             const int32_t* __restrict__ cols,
                                                             const double* __restrict__ vals,
                                                             const double* __restrict__ x, double* y,
                                                             double* partials, unsigned int* counter,
                                                             double* dot_out, const int* stop)
{
    if(stop && *stop)
        return;
    const int lane   = threadIdx.x & 31;
    double    dot    = 0.0;
    const int64_t stride = (int64_t)gridDim.x * SPMV_BLOCK;
    for(int64_t base = (int64_t)blockIdx.x * SPMV_BLOCK; base < U; base += stride)
    {
        const int64_t k = base + threadIdx.x;
        int32_t i = -1, j = 0;
        double  a0 = 0, a1 = 0, a2 = 0;  // B x_j
        if(k < U)
        {
            i = __ldg(rows + k);
            j = __ldg(cols + k);
            double b[9];
#pragma unroll
            for(int q = 0; q < 9; ++q)
                b[q] = __ldg(vals + (int64_t)q * U + k);
            const double xj0 = __ldg(x + 3 * (int64_t)j), xj1 = __ldg(x + 3 * (int64_t)j + 1),
                         xj2 = __ldg(x + 3 * (int64_t)j + 2);
            // column-major: B(p,q) = b[q*3 + p]
            a0 = b[0] * xj0 + b[3] * xj1 + b[6] * xj2;
            a1 = b[1] * xj0 + b[4] * xj1 + b[7] * xj2;
            a2 = b[2] * xj0 + b[5] * xj1 + b[8] * xj2;
            if(i != j)
            {
                const double xi0 = __ldg(x + 3 * (int64_t)i), xi1 = __ldg(x + 3 * (int64_t)i + 1),
                             xi2 = __ldg(x + 3 * (int64_t)i + 2);
                const double t0 = b[0] * xi0 + b[1] * xi1 + b[2] * xi2;
                const double t1 = b[3] * xi0 + b[4] * xi1 + b[5] * xi2;
                const double t2 = b[6] * xi0 + b[7] * xi1 + b[8] * xi2;
                atomicAdd(y + 3 * (int64_t)j, t0);
                atomicAdd(y + 3 * (int64_t)j + 1, t1);
                atomicAdd(y + 3 * (int64_t)j + 2, t2);
                if(WITH_DOT)
                    dot += 2.0 * (xi0 * a0 + xi1 * a1 + xi2 * a2);
            }
            else if(WITH_DOT)
            {
                dot += xj0 * a0 + xj1 * a1 + xj2 * a2;
            }
        }
        // segmented inclusive scan of (a0,a1,a2) over equal row ids
#pragma unroll
        for(int o = 1; o < 32; o <<= 1)
        {
            const double  t0 = __shfl_up_sync(0xffffffffu, a0, o);
            const double  t1 = __shfl_up_sync(0xffffffffu, a1, o);
            const double  t2 = __shfl_up_sync(0xffffffffu, a2, o);
            const int32_t ti = __shfl_up_sync(0xffffffffu, i, o);
            if(lane >= o && ti == i)
            {
                a0 += t0;
                a1 += t1;
                a2 += t2;
            }
        }
        const int32_t inext = __shfl_down_sync(0xffffffffu, i, 1);
        const bool    tail  = (lane == 31) || (inext != i);
        if(i >= 0 && tail)
        {
            atomicAdd(y + 3 * (int64_t)i, a0);
            atomicAdd(y + 3 * (int64_t)i + 1, a1);
            atomicAdd(y + 3 * (int64_t)i + 2, a2);
        }
    }
    if(WITH_DOT)
    {
        double v[1] = {dot}, tot[1];
        if(grid_sum<1>(v, partials, counter, tot))
            *dot_out = tot[0];
    }
}
}  // namespace

int spmv_grid(int64_t U)
{
    int64_t g = (U + SPMV_BLOCK - 1) / SPMV_BLOCK;
    const int64_t cap = (int64_t)NUM_SMS_HINT * 8;
    if(g > cap)
        g = cap;
    return (int)(g < 1 ? 1 : g);
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
    const int grid = spmv_grid(A.nnz);
    ensure_reduction(s->red, grid, 1);
    if(d_dot)
        k_spmv_sym_f64<true><<<grid, SPMV_BLOCK, 0, st>>>(A.nnz, A.rows.data(), A.cols.data(), A.vals.data(), x, y,
                                                          s->red.partials.data(), s->red.counter.data(), d_dot,
                                                          nullptr);
    else
        k_spmv_sym_f64<false><<<grid, SPMV_BLOCK, 0, st>>>(A.nnz, A.rows.data(), A.cols.data(), A.vals.data(), x,
                                                           y, nullptr, nullptr, nullptr, nullptr);
    B2S_CHECK_LAUNCH();
}

// launch parameters shared with the PCG graph (y must be zero beforehand)
void spmv_f64_launch(cudaStream_t st, const Matrix& A, const double* x, double* y, Reduction& red,
                     double* d_dot, const int* stop)
{
    if(A.nnz == 0)
        return;
    const int grid = spmv_grid(A.nnz);
    k_spmv_sym_f64<true><<<grid, SPMV_BLOCK, 0, st>>>(A.nnz, A.rows.data(), A.cols.data(), A.vals.data(), x, y,
                                                      red.partials.data(), red.counter.data(), d_dot, stop);
    B2S_CHECK_LAUNCH();
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
