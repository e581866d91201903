// b2s_spmv_noalloc: symmetric block SpMV + x.(A x) for callers that cannot
// allocate device memory.
//
// Who needs it: code that runs where cudaMalloc is not an option -- inside a
// host callback or a custom allocator hook, in a process whose device memory
// is fully carved up by another framework's caching allocator, or in a
// pre-sized real-time loop that must not touch the allocator after start-up.
// Such a caller owns every input and output buffer; this entry point then
// allocates nothing. Its only scratch -- one partial dot per 256-block tile
// and a completion counter -- lives in the file-scope device array below,
// which every device that loads this library holds until the process exits.
#include "b2s_internal.cuh"

#include <mutex>

namespace b2s
{
namespace
{
constexpr int NOALLOC_TILE      = 256;    // blocks per tile (one CTA pass)
constexpr int NOALLOC_MAX_TILES = 32768;  // => at most 8,388,608 blocks per call

struct NoallocScratch
{
    double       partials[NOALLOC_MAX_TILES];  // per-tile partial dots, summed in tile order
    unsigned int counter;                      // CTAs finished (reset by the last one)
    unsigned int bad_input;                    // a block failed the index / order checks
};

// Device-resident scratch shared by every call on a device (~256 KB). In host
// code this name is only a host-side stand-in: kernels get the real device
// address from cudaGetSymbolAddress.
static __device__ __align__(256) NoallocScratch g_noalloc_scratch;

std::mutex      g_setup_mutex;
NoallocScratch* g_scratch_ptr[256] = {};

// device address of the scratch array for the current device (set up once
// per device on the first call)
NoallocScratch* scratch_for_current_device()
{
    int dev = -1;
    B2S_CUDA(cudaGetDevice(&dev));
    B2S_REQUIRE(dev >= 0 && dev < 256, B2S_ERR_ARGUMENT, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if(!g_scratch_ptr[dev])
    {
        void*       ptr = nullptr;
        cudaError_t e   = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if(e != cudaSuccess || !ptr)
            throw Error(B2S_ERR_CUDA, std::string("cudaGetSymbolAddress(no-alloc scratch): ")
                                          + cudaGetErrorString(e));
        g_scratch_ptr[dev] = static_cast<NoallocScratch*>(ptr);
    }
    return g_scratch_ptr[dev];
}

__device__ __forceinline__ void red_add(double* p, double v)
{
    asm volatile("red.global.add.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}

// One CTA per tile pass (grid-stride over tiles); thread = block of the
// caller's BCOO (values 9 doubles, column-major, per block). Row parts are
// merged over equal rows in-warp (rows are non-decreasing, so equal rows are
// contiguous), transposed parts scatter as L2 reductions; the tile's dot goes
// to scratch->partials[tile] and the last CTA adds the partials in a fixed
// order (bit-reproducible for a given input). A block whose row or column is
// outside [0, nb), whose row exceeds its column, or whose row is below the
// previous block's is skipped (no access through its indices) and makes the
// dot NaN.
__global__ void __launch_bounds__(NOALLOC_TILE) k_spmv_noalloc(int32_t nb, int64_t U, const int32_t* __restrict__ rows,
                                                               const int32_t* __restrict__ cols,
                                                               const double* __restrict__ vals,
                                                               const double* __restrict__ x, double* y,
                                                               double* dot_out, NoallocScratch* scratch)
{
    __shared__ double red[NOALLOC_TILE];
    __shared__ bool   is_last;
    const int     lane    = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t n_tiles = (U + NOALLOC_TILE - 1) / NOALLOC_TILE;
    for(int64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x)
    {
        const int64_t k = tile * NOALLOC_TILE + threadIdx.x;
        int32_t       r = -1;
        double        a0 = 0, a1 = 0, a2 = 0, d = 0;
        if(k < U)
        {
            const int32_t rk = rows[k];
            const int32_t c  = cols[k];
            const bool    ok = rk >= 0 && rk < nb && c >= rk && c < nb && (k == 0 || rows[k - 1] <= rk);
            if(!ok)
                atomicOr(&scratch->bad_input, 1u);
            else
            {
                r = rk;
                double b[9];
#pragma unroll
                for(int q = 0; q < 9; ++q)
                    b[q] = vals[k * 9 + q];
                const double xj0 = x[3 * (int64_t)c], xj1 = x[3 * (int64_t)c + 1], xj2 = x[3 * (int64_t)c + 2];
                const double xi0 = x[3 * (int64_t)r], xi1 = x[3 * (int64_t)r + 1], xi2 = x[3 * (int64_t)r + 2];
                a0 = b[0] * xj0 + b[3] * xj1 + b[6] * xj2;
                a1 = b[1] * xj0 + b[4] * xj1 + b[7] * xj2;
                a2 = b[2] * xj0 + b[5] * xj1 + b[8] * xj2;
                d  = xi0 * a0 + xi1 * a1 + xi2 * a2;
                if(r != c)
                {
                    red_add(y + 3 * (int64_t)c, b[0] * xi0 + b[1] * xi1 + b[2] * xi2);
                    red_add(y + 3 * (int64_t)c + 1, b[3] * xi0 + b[4] * xi1 + b[5] * xi2);
                    red_add(y + 3 * (int64_t)c + 2, b[6] * xi0 + b[7] * xi1 + b[8] * xi2);
                    d += d;
                }
            }
        }
#pragma unroll
        for(int o = 1; o < 32; o <<= 1)
        {
            const double  t0 = __shfl_up_sync(0xffffffffu, a0, o);
            const double  t1 = __shfl_up_sync(0xffffffffu, a1, o);
            const double  t2 = __shfl_up_sync(0xffffffffu, a2, o);
            const int32_t tr = __shfl_up_sync(0xffffffffu, r, o);
            if(lane >= o && tr == r)
            {
                a0 += t0;
                a1 += t1;
                a2 += t2;
            }
        }
        const int32_t rnext = __shfl_down_sync(0xffffffffu, r, 1);
        if(r >= 0 && (lane == 31 || rnext != r))
        {
            red_add(y + 3 * (int64_t)r, a0);
            red_add(y + 3 * (int64_t)r + 1, a1);
            red_add(y + 3 * (int64_t)r + 2, a2);
        }
        // tile dot: warp butterfly then the 8 warp sums in order
#pragma unroll
        for(int o = 16; o > 0; o >>= 1)
            d += __shfl_xor_sync(0xffffffffu, d, o);
        if(lane == 0)
            red[warp] = d;
        __syncthreads();
        if(threadIdx.x == 0)
        {
            double t = 0.0;
            for(int w = 0; w < NOALLOC_TILE / 32; ++w)
                t += red[w];
            scratch->partials[tile] = t;
        }
        __syncthreads();
    }
    if(threadIdx.x == 0)
    {
        __threadfence();
        const unsigned int prev = atomicAdd(&scratch->counter, 1u);
        is_last                 = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if(!is_last)
        return;
    __threadfence();
    // the last CTA: thread t sums its contiguous chunk of the partials in
    // order, then a fixed pairwise tree over the threads
    const int64_t chunk = (n_tiles + NOALLOC_TILE - 1) / NOALLOC_TILE;
    const int64_t q0    = (int64_t)threadIdx.x * chunk;
    const int64_t q1    = q0 + chunk < n_tiles ? q0 + chunk : n_tiles;
    double        t     = 0.0;
    for(int64_t q = q0; q < q1; ++q)
        t += ((volatile double*)scratch->partials)[q];
    red[threadIdx.x] = t;
    __syncthreads();
    for(int h = NOALLOC_TILE / 2; h > 0; h >>= 1)
    {
        if(threadIdx.x < h)
            red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    if(threadIdx.x == 0)
    {
        const bool bad = ((volatile unsigned int*)&scratch->bad_input)[0] != 0u;
        if(dot_out)
            *dot_out = bad ? __longlong_as_double(0x7ff8000000000000ll) : red[0];
        scratch->counter   = 0u;
        scratch->bad_input = 0u;
    }
}
}  // namespace
}  // namespace b2s

extern "C" int b2s_spmv_noalloc(int32_t n_block_rows, int64_t n_blocks, const int32_t* d_rows,
                                const int32_t* d_cols, const double* d_vals, const double* d_x, double* d_y,
                                double* d_dot, void* stream)
{
    using namespace b2s;
    try
    {
        B2S_REQUIRE(n_block_rows >= 0 && n_blocks >= 0, B2S_ERR_ARGUMENT, "negative size");
        B2S_REQUIRE(n_blocks <= (int64_t)NOALLOC_MAX_TILES * NOALLOC_TILE, B2S_ERR_ARGUMENT,
                    "b2s_spmv_noalloc: n_blocks exceeds the no-alloc limit of "
                        + std::to_string((int64_t)NOALLOC_MAX_TILES * NOALLOC_TILE) + " blocks");
        B2S_REQUIRE(d_x && d_y && (n_blocks == 0 || (d_rows && d_cols && d_vals)), B2S_ERR_ARGUMENT,
                    "b2s_spmv_noalloc: null array");
        cudaStream_t   st      = static_cast<cudaStream_t>(stream);
        NoallocScratch* scratch = scratch_for_current_device();
        // y = A x overwrites y; the completion counter and the input-check
        // word must start at zero (the array keeps the last call's contents)
        B2S_CUDA(cudaMemsetAsync(d_y, 0, sizeof(double) * 3 * (size_t)n_block_rows, st));
        B2S_CUDA(cudaMemsetAsync(&scratch->counter, 0, 2 * sizeof(unsigned int), st));
        if(n_blocks == 0)
        {
            if(d_dot)
                B2S_CUDA(cudaMemsetAsync(d_dot, 0, sizeof(double), st));
            return B2S_OK;
        }
        const int64_t n_tiles = (n_blocks + NOALLOC_TILE - 1) / NOALLOC_TILE;
        const int     grid    = (int)std::min<int64_t>(n_tiles, (int64_t)NUM_SMS_HINT * 8);
        k_spmv_noalloc<<<grid, NOALLOC_TILE, 0, st>>>(n_block_rows, n_blocks, d_rows, d_cols, d_vals, d_x, d_y, d_dot, scratch);
        B2S_CUDA(cudaGetLastError());
        return B2S_OK;
    }
    catch(const Error& e)
    {
        set_handle_free_error(e.what());
        return e.code;
    }
    catch(const std::exception& e)
    {
        set_handle_free_error(e.what());
        return B2S_ERR_STATE;
    }
}
