// Deterministic reduction of a device array to one value: one CTA, each
// thread folds a fixed strided subset in index order, then a fixed
// shared-memory tree; the sum (or, with take_min, the minimum) comes out the
// same on every run and for every launch configuration of the producer.
#pragma once

#include <cmath>
#include <cstdint>

namespace b2s
{
constexpr int SUM_THREADS = 1024;

namespace
{
__global__ void __launch_bounds__(SUM_THREADS) k_fixed_reduce(int64_t n, const double* __restrict__ v, int take_min,
                                                              double* __restrict__ out)
{
    __shared__ double sh[SUM_THREADS];
    double            acc = take_min ? INFINITY : 0.0;
    for(int64_t i = threadIdx.x; i < n; i += SUM_THREADS)
        acc = take_min ? fmin(acc, v[i]) : acc + v[i];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for(int w = SUM_THREADS / 2; w > 0; w >>= 1)
    {
        if(threadIdx.x < w)
            sh[threadIdx.x] = take_min ? fmin(sh[threadIdx.x], sh[threadIdx.x + w]) : sh[threadIdx.x] + sh[threadIdx.x + w];
        __syncthreads();
    }
    if(threadIdx.x == 0)
        *out = sh[0];
}
}  // namespace
}  // namespace b2s
