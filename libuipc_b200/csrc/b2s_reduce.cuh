// Deterministic grid reductions: every block writes its partial sums, the
// last block to finish adds the partials in block order (fixed grid => fixed
// summation order => bit-reproducible results).
#pragma once
#include "b2s_internal.cuh"

namespace b2s
{
constexpr int RED_BLOCK = 256;

// block sum of NV doubles per thread; valid in thread 0
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double (*smem)[RED_BLOCK / 32])
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for(int k = 0; k < NV; ++k)
    {
#pragma unroll
        for(int o = 16; o > 0; o >>= 1)
            v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    }
    if(lane == 0)
    {
#pragma unroll
        for(int k = 0; k < NV; ++k)
            smem[k][warp] = v[k];
    }
    __syncthreads();
    if(warp == 0)
    {
#pragma unroll
        for(int k = 0; k < NV; ++k)
        {
            double t = (lane < (int)(blockDim.x >> 5)) ? smem[k][lane] : 0.0;
#pragma unroll
            for(int o = 16; o > 0; o >>= 1)
                t += __shfl_xor_sync(0xffffffffu, t, o);
            v[k] = t;
        }
    }
}

// Publish this block's NV partial sums; returns true in thread 0 of the last
// block, which then finds the totals in `total`.
template <int NV>
__device__ __forceinline__ bool grid_sum(double (&v)[NV], double* partials, unsigned int* counter,
                                         double (&total)[NV])
{
    __shared__ double smem[NV][RED_BLOCK / 32];
    __shared__ bool   is_last;
    block_sum<NV>(v, smem);
    if(threadIdx.x == 0)
    {
#pragma unroll
        for(int k = 0; k < NV; ++k)
            partials[(size_t)k * gridDim.x + blockIdx.x] = v[k];
        __threadfence();
        unsigned int prev = atomicAdd(counter, 1u);
        is_last           = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if(!is_last)
        return false;
    // last block: sum the partials in block order, NV values in parallel warps
    __threadfence();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __shared__ double res[NV];
    for(int k = warp; k < NV; k += blockDim.x >> 5)
    {
        // each lane sums a strided subset in order, then a fixed-shape tree;
        // the loads go out 8 at a time (independent), the adds keep the order
        const volatile double* pk  = (const volatile double*)partials + (size_t)k * gridDim.x;
        double                 acc = 0.0;
        for(unsigned int b = lane; b < gridDim.x; b += 32 * 8)
        {
            double t[8];
#pragma unroll
            for(int j = 0; j < 8; ++j)
                t[j] = b + 32u * j < gridDim.x ? pk[b + 32u * j] : 0.0;
#pragma unroll
            for(int j = 0; j < 8; ++j)
                if(b + 32u * j < gridDim.x)
                    acc += t[j];
        }
#pragma unroll
        for(int o = 16; o > 0; o >>= 1)
            acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if(lane == 0)
            res[k] = acc;
    }
    __syncthreads();
    if(threadIdx.x != 0)
        return false;
#pragma unroll
    for(int k = 0; k < NV; ++k)
        total[k] = res[k];
    *counter = 0u;  // ready for the next launch
    return true;
}
}  // namespace b2s
