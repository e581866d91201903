// Learned PCG warm start: a small MLP on MAS level-1 aggregates.
//
// No counterpart in libuipc (its PCG starts from zero). Per Newton system:
//  1. fields (FP64, length 3n): f0 = h1, f1 = h1 - h2, f2 = h1 - 2 h2 + h3
//     (the latest solutions of the run and their first and second
//     differences) and f3 = z = P b (one MAS application to the gradient);
//     missing history entries are zero.
//  2. per level-1 aggregate a (the MAS level-1 node of each vertex): sums over
//     its vertices, in units where b has unit RMS and the fields are divided
//     by s = RMS(z): count, sum b, sum f_i, sum |f_i|^2, sum f_i . f_{i+1},
//     and, for training, the Gram H_ij = sum f_i . f_j, q_i = sum f_i . x and
//     c0 = sum |x|^2 of the solved x. FP32 atomics (order not reproducible).
//  3. features (22): mean b; per field its mean and log RMS; the mean products
//     of consecutive fields. Standardised with the stored mean / std.
//  4. MLP 22 -> H -> H -> 4 (ReLU), FP32 weights; inference reads BF16 copies
//     held in shared memory, FP32 accumulation. Output: coefficients c_a.
//  5. field d_v = sum_i c_{a(v), i} f_i(v); the start x0 is the A-optimal
//     combination of the candidate vectors of the mode (Galerkin: solve
//     G alpha = g with G_kl = c_k . A c_l, g_k = c_k . b in FP64, pseudo-
//     inverse on the host), checked in FP64 by r^T P r < b^T P b (r = b - A x0),
//     the residual measure of the PCG itself; otherwise x0 = 0.
// Training minimises sum_a (c_a^T H_a c_a - 2 c_a^T q_a + c0_a) / sum_a c0_a,
// i.e. the squared error of the predicted field against the solved x, with
// one Adam step per stored system; the GEMMs of the forward and backward
// passes are the tiled FP32 kernel below.
#include "b2s_internal.cuh"
#include "b2s_reduce.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <type_traits>
#include <vector>

namespace b2s
{
void check_device_errors(b2s_solver* s);

constexpr int WS_FIELDS = 4;
constexpr int WS_F      = 3 + WS_FIELDS * 4 + (WS_FIELDS - 1);  // 22
constexpr int WS_O      = WS_FIELDS;
constexpr int WS_HSYM   = WS_FIELDS * (WS_FIELDS + 1) / 2;  // 10
// accumulator layout per aggregate
constexpr int ACC_CNT = 0, ACC_B = 1, ACC_F = 4, ACC_FF = ACC_F + 3 * WS_FIELDS, ACC_X = ACC_FF + WS_FIELDS,
              ACC_H = ACC_X + (WS_FIELDS - 1), ACC_Q = ACC_H + WS_HSYM, ACC_C0 = ACC_Q + WS_FIELDS,
              WS_ACC = ACC_C0 + 1;  // 38
static_assert(WS_F == B2S_WS_FEATURES && WS_O == B2S_WS_OUTPUTS, "header constants");

struct WsSample
{
    int64_t row0;   // first row in the sample store
    int32_t rows;   // aggregates
    double  norm;   // sum of c0 (loss normaliser)
};

struct LearnedState
{
    int     hidden   = 0;
    int64_t n_params = 0;
    DBuf<float> params, grad, adam_m, adam_v;
    std::vector<float> mean, stdv;  // feature standardisation (host copy)
    DBuf<float> norm_dev;           // [2F]: mean, 1/std
    long long   adam_t = 0;
    // sample store (device, grown by copy)
    std::vector<WsSample> samples;
    int64_t     store_rows = 0, store_cap = 0;
    DBuf<float> st_feat, st_H, st_q, st_c0;
    // per-system scratch
    DBuf<float>  acc, feat, X, Y, H1, H2, dY, dH, loss_dev;
    DBuf<double> fields, d_mlp, Ac, x0, dots;
    DBuf<__nv_bfloat16> w16;  // BF16 copy of the weights for inference
    long long    w16_version = -1, version = 0;
    cudaEvent_t  ev0 = nullptr, ev1 = nullptr;
};

void ws_free(LearnedState* w)
{
    if(!w)
        return;
    if(w->ev0)
        cudaEventDestroy(w->ev0);
    if(w->ev1)
        cudaEventDestroy(w->ev1);
    delete w;
}

namespace
{
constexpr int WS_BLOCK = 256;

int ws_grid(int64_t n)
{
    int64_t g = (n + WS_BLOCK - 1) / WS_BLOCK;
    const int64_t cap = (int64_t)NUM_SMS_HINT * 8;
    return (int)std::max<int64_t>(1, std::min(g, cap));
}

// parameter offsets: W0[F x H] b0[H] W1[H x H] b1[H] W2[H x O] b2[O]
struct PLayout
{
    int64_t W0, b0, W1, b1, W2, b2, n;
    __host__ __device__ explicit PLayout(int H)
    {
        W0 = 0;
        b0 = W0 + (int64_t)WS_F * H;
        W1 = b0 + H;
        b1 = W1 + (int64_t)H * H;
        W2 = b1 + H;
        b2 = W2 + (int64_t)H * WS_O;
        n  = b2 + WS_O;
    }
};

// f0 = h1, f1 = h1 - h2, f2 = h1 - 2 h2 + h3, f3 = z (fields laid out [4][n])
__global__ void k_ws_fields(int64_t n, const double* __restrict__ h1, const double* __restrict__ h2,
                            const double* __restrict__ h3, const double* __restrict__ z, double* __restrict__ f)
{
    for(int64_t i = (int64_t)blockIdx.x * WS_BLOCK + threadIdx.x; i < n; i += (int64_t)gridDim.x * WS_BLOCK)
    {
        const double a = h1 ? h1[i] : 0.0, b = h2 ? h2[i] : 0.0, c = h3 ? h3[i] : 0.0;
        f[i]         = a;
        f[n + i]     = a - b;
        f[2 * n + i] = a - 2.0 * b + c;
        f[3 * n + i] = z[i];
    }
}

// aggregate of MAS vertex v (level-1 local id) or -1
__device__ __forceinline__ int agg_of(const int32_t* ctable, int L, int level1_begin, int v)
{
    if(L < 2)
        return -1;
    const int g = ctable[(int64_t)v * (L - 1)];
    return g < 0 ? -1 : g - level1_begin;
}

// per-vertex sums into the aggregate accumulators (see the layout above)
__global__ void k_ws_accumulate(int vn, int off, int L, int level1_begin, int n_agg, const int32_t* __restrict__ ctable,
                                const double* __restrict__ b, const double* __restrict__ f, int64_t n,
                                const double* __restrict__ x, double inv_bs, double inv_s, float* __restrict__ acc)
{
    for(int v = blockIdx.x * WS_BLOCK + threadIdx.x; v < vn; v += gridDim.x * WS_BLOCK)
    {
        const int a = agg_of(ctable, L, level1_begin, v);
        if(a < 0 || a >= n_agg)
            continue;
        float*        A  = acc + (int64_t)a * WS_ACC;
        const int64_t i0 = 3 * ((int64_t)off + v);
        float         F[WS_FIELDS][3], X[3];
        for(int c = 0; c < 3; ++c)
        {
            for(int k = 0; k < WS_FIELDS; ++k)
                F[k][c] = (float)(f[k * n + i0 + c] * inv_s);
            X[c] = x ? (float)(x[i0 + c] * inv_s) : 0.f;
        }
        atomicAdd(A + ACC_CNT, 1.0f);
        for(int c = 0; c < 3; ++c)
            atomicAdd(A + ACC_B + c, (float)(b[i0 + c] * inv_bs));
        auto dot3 = [](const float* p, const float* q) { return p[0] * q[0] + p[1] * q[1] + p[2] * q[2]; };
        for(int k = 0; k < WS_FIELDS; ++k)
        {
            for(int c = 0; c < 3; ++c)
                atomicAdd(A + ACC_F + 3 * k + c, F[k][c]);
            atomicAdd(A + ACC_FF + k, dot3(F[k], F[k]));
        }
        for(int k = 0; k + 1 < WS_FIELDS; ++k)
            atomicAdd(A + ACC_X + k, dot3(F[k], F[k + 1]));
        if(x)
        {
            int e = 0;
            for(int i = 0; i < WS_FIELDS; ++i)
                for(int j = i; j < WS_FIELDS; ++j, ++e)
                    atomicAdd(A + ACC_H + e, dot3(F[i], F[j]));
            for(int i = 0; i < WS_FIELDS; ++i)
                atomicAdd(A + ACC_Q + i, dot3(F[i], X));
            atomicAdd(A + ACC_C0, dot3(X, X));
        }
    }
}

// raw features (and the training statistics) of every aggregate
__global__ void k_ws_features(int n_agg, const float* __restrict__ acc, float* __restrict__ feat,
                              float* __restrict__ Hs, float* __restrict__ q, float* __restrict__ c0)
{
    const int a = blockIdx.x * WS_BLOCK + threadIdx.x;
    if(a >= n_agg)
        return;
    const float* A   = acc + (int64_t)a * WS_ACC;
    const float  cnt = fmaxf(A[ACC_CNT], 1.0f), ic = 1.0f / cnt;
    float*       o   = feat + (int64_t)a * WS_F;
    int          e   = 0;
    for(int c = 0; c < 3; ++c)
        o[e++] = A[ACC_B + c] * ic;
    for(int k = 0; k < WS_FIELDS; ++k)
    {
        for(int c = 0; c < 3; ++c)
            o[e++] = A[ACC_F + 3 * k + c] * ic;
        o[e++] = logf(sqrtf(fmaxf(A[ACC_FF + k], 0.f) * ic) + 1e-6f);
    }
    for(int k = 0; k + 1 < WS_FIELDS; ++k)
        o[e++] = A[ACC_X + k] * ic;
    if(Hs)
    {
        for(int i = 0; i < WS_HSYM; ++i)
            Hs[(int64_t)a * WS_HSYM + i] = A[ACC_H + i];
        for(int i = 0; i < WS_FIELDS; ++i)
            q[(int64_t)a * WS_FIELDS + i] = A[ACC_Q + i];
        c0[a] = A[ACC_C0];
    }
}

// X = (feat - mean) / std
__global__ void k_ws_standardise(int64_t rows, const float* __restrict__ feat, const float* __restrict__ norm,
                                 float* __restrict__ X)
{
    const int64_t n = rows * WS_F;
    for(int64_t i = (int64_t)blockIdx.x * WS_BLOCK + threadIdx.x; i < n; i += (int64_t)gridDim.x * WS_BLOCK)
    {
        const int j = (int)(i % WS_F);
        X[i]        = (feat[i] - norm[j]) * norm[WS_F + j];
    }
}

__device__ __forceinline__ float hsym(const float* Hs, int i, int j)
{
    if(i > j)
    {
        const int t = i;
        i           = j;
        j           = t;
    }
    return Hs[i * WS_FIELDS - i * (i - 1) / 2 + (j - i)];
}

// per-row loss y^T H y - 2 y^T q + c0 (summed into *loss, divided by norm)
// and dY = 2 (H y - q) / norm
__global__ void k_ws_loss(int rows, const float* __restrict__ Y, const float* __restrict__ Hs,
                          const float* __restrict__ q, const float* __restrict__ c0, float inv_norm,
                          float* __restrict__ dY, float* __restrict__ loss)
{
    const int a = blockIdx.x * WS_BLOCK + threadIdx.x;
    float     l = 0.f;
    if(a < rows)
    {
        const float* y  = Y + (int64_t)a * WS_O;
        const float* H  = Hs + (int64_t)a * WS_HSYM;
        const float* qa = q + (int64_t)a * WS_O;
        float        Hy[WS_O];
        for(int i = 0; i < WS_O; ++i)
        {
            Hy[i] = 0.f;
            for(int j = 0; j < WS_O; ++j)
                Hy[i] += hsym(H, i, j) * y[j];
        }
        for(int i = 0; i < WS_O; ++i)
        {
            l += y[i] * Hy[i] - 2.f * y[i] * qa[i];
            dY[(int64_t)a * WS_O + i] = 2.f * (Hy[i] - qa[i]) * inv_norm;
        }
        l = (l + c0[a]) * inv_norm;
    }
    // block sum, one atomic per block
    __shared__ float s[WS_BLOCK / 32];
    for(int o = 16; o > 0; o >>= 1)
        l += __shfl_down_sync(0xffffffffu, l, o);
    if((threadIdx.x & 31) == 0)
        s[threadIdx.x >> 5] = l;
    __syncthreads();
    if(threadIdx.x == 0)
    {
        float t = 0.f;
        for(int w = 0; w < WS_BLOCK / 32; ++w)
            t += s[w];
        atomicAdd(loss, t);
    }
}

// C (M x N, row-major, ldc) = op(A) op(B), op(A): M x K, op(B): K x N.
// A is M x K (lda) or, with TA, K x M; B is K x N (ldb) or, with TB, N x K.
// 64 x 64 tiles, 16-deep K steps, 4 x 4 outputs per thread; blockIdx.z
// splits K into chunks of k_chunk and ATOMIC adds the partial products into C
// (which the caller zeroed).
template <bool TA, bool TB, bool ATOMIC>
__global__ void __launch_bounds__(256) k_gemm(int M, int N, int K, const float* __restrict__ A, int lda,
                                              const float* __restrict__ B, int ldb, float* __restrict__ C, int ldc,
                                              int k_chunk)
{
    __shared__ float As[16][64 + 4];
    __shared__ float Bs[16][64 + 4];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
    const int kb = blockIdx.z * k_chunk, ke = min(K, kb + k_chunk);
    float     acc[4][4];
#pragma unroll
    for(int i = 0; i < 4; ++i)
#pragma unroll
        for(int j = 0; j < 4; ++j)
            acc[i][j] = 0.f;
    for(int k0 = kb; k0 < ke; k0 += 16)
    {
        for(int e = threadIdx.x; e < 1024; e += 256)
        {
            int mm, kk;
            if(TA)
            {
                kk = e >> 6;
                mm = e & 63;
            }
            else
            {
                mm = e >> 4;
                kk = e & 15;
            }
            const int m = m0 + mm, k = k0 + kk;
            As[kk][mm] = (m < M && k < ke) ? (TA ? A[(int64_t)k * lda + m] : A[(int64_t)m * lda + k]) : 0.f;
            int nn, kk2;
            if(TB)
            {
                nn  = e >> 4;
                kk2 = e & 15;
            }
            else
            {
                kk2 = e >> 6;
                nn  = e & 63;
            }
            const int n = n0 + nn, k2 = k0 + kk2;
            Bs[kk2][nn] = (n < N && k2 < ke) ? (TB ? B[(int64_t)n * ldb + k2] : B[(int64_t)k2 * ldb + n]) : 0.f;
        }
        __syncthreads();
#pragma unroll
        for(int kk = 0; kk < 16; ++kk)
        {
            float a[4], b[4];
#pragma unroll
            for(int i = 0; i < 4; ++i)
                a[i] = As[kk][ty * 4 + i];
#pragma unroll
            for(int j = 0; j < 4; ++j)
                b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
            for(int i = 0; i < 4; ++i)
#pragma unroll
                for(int j = 0; j < 4; ++j)
                    acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for(int i = 0; i < 4; ++i)
#pragma unroll
        for(int j = 0; j < 4; ++j)
        {
            const int m = m0 + ty * 4 + i, n = n0 + tx * 4 + j;
            if(m < M && n < N)
            {
                if(ATOMIC)
                    atomicAdd(&C[(int64_t)m * ldc + n], acc[i][j]);
                else
                    C[(int64_t)m * ldc + n] = acc[i][j];
            }
        }
}

template <bool TA, bool TB>
void gemm(cudaStream_t st, int M, int N, int K, const float* A, int lda, const float* B, int ldb, float* C, int ldc,
          bool accumulate_split)
{
    dim3 grid((N + 63) / 64, (M + 63) / 64, 1);
    if(accumulate_split)
    {
        // split the long K (rows of a batch) so the small weight-gradient
        // products fill the GPU; C must be zero
        const int tiles  = (int)(grid.x * grid.y);
        int       splits = std::max(1, std::min((NUM_SMS_HINT * 4) / std::max(tiles, 1), (K + 255) / 256));
        int       chunk  = ((K + splits - 1) / splits + 15) / 16 * 16;
        splits           = (K + chunk - 1) / chunk;
        grid.z           = (unsigned)std::max(splits, 1);
        k_gemm<TA, TB, true><<<grid, 256, 0, st>>>(M, N, K, A, lda, B, ldb, C, ldc, chunk);
    }
    else
        k_gemm<TA, TB, false><<<grid, 256, 0, st>>>(M, N, K, A, lda, B, ldb, C, ldc, ((K + 15) / 16) * 16);
    B2S_CHECK_LAUNCH();
}

// C[m][n] += bias[n]; optional ReLU
__global__ void k_bias_act(int64_t M, int N, float* __restrict__ C, const float* __restrict__ bias, int relu)
{
    const int64_t total = M * N;
    for(int64_t i = (int64_t)blockIdx.x * WS_BLOCK + threadIdx.x; i < total; i += (int64_t)gridDim.x * WS_BLOCK)
    {
        float v = C[i] + bias[i % N];
        C[i]    = relu ? fmaxf(v, 0.f) : v;
    }
}

// D[m][n] *= (Hact[m][n] > 0): backward of ReLU through its output
__global__ void k_relu_mask(int64_t total, float* __restrict__ D, const float* __restrict__ Hact)
{
    for(int64_t i = (int64_t)blockIdx.x * WS_BLOCK + threadIdx.x; i < total; i += (int64_t)gridDim.x * WS_BLOCK)
        if(!(Hact[i] > 0.f))
            D[i] = 0.f;
}

// out[n] += sum_m D[m][n] (N <= 1024 threads per block, rows in chunks)
__global__ void k_colsum(int M, int N, const float* __restrict__ D, float* __restrict__ out, int rows_per_block)
{
    const int n = threadIdx.x;
    if(n >= N)
        return;
    const int m0 = blockIdx.x * rows_per_block, m1 = min(M, m0 + rows_per_block);
    float     s  = 0.f;
    for(int m = m0; m < m1; ++m)
        s += D[(int64_t)m * N + n];
    atomicAdd(&out[n], s);
}

__global__ void k_adam(int64_t n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2)
{
    for(int64_t i = (int64_t)blockIdx.x * WS_BLOCK + threadIdx.x; i < n; i += (int64_t)gridDim.x * WS_BLOCK)
    {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i]           = mi;
        v[i]           = vi;
        p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    }
}

__global__ void k_to_bf16(int64_t n, const float* __restrict__ a, __nv_bfloat16* __restrict__ o)
{
    for(int64_t i = (int64_t)blockIdx.x * WS_BLOCK + threadIdx.x; i < n; i += (int64_t)gridDim.x * WS_BLOCK)
        o[i] = __float2bfloat16_rn(a[i]);
}

// MLP inference, BF16 weights in shared memory, FP32 accumulation. One thread
// per hidden unit (blockDim = H); persistent over tiles of INF_TILE
// aggregates: h1 = relu(x W0 + b0), h2 = relu(h1 W1 + b1), y = h2 W2 + b2,
// x = (feat - mean) / std.
constexpr int INF_TILE = 16;

size_t inference_smem(int H)
{
    const size_t w = ((size_t)WS_F * H + (size_t)H * H + (size_t)H * WS_O) * sizeof(__nv_bfloat16);
    return ((w + 15) / 16) * 16 + sizeof(float) * ((size_t)2 * H + WS_O + INF_TILE * WS_F + (size_t)INF_TILE * H);
}

__global__ void k_ws_infer(int rows, int H, const __nv_bfloat16* __restrict__ w16, const float* __restrict__ params,
                           const float* __restrict__ feat, const float* __restrict__ norm, float* __restrict__ Y)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const PLayout P(H);
    __nv_bfloat16* W0 = reinterpret_cast<__nv_bfloat16*>(smem);
    __nv_bfloat16* W1 = W0 + (size_t)WS_F * H;
    __nv_bfloat16* W2 = W1 + (size_t)H * H;
    const size_t   wb = ((((size_t)WS_F * H + (size_t)H * H + (size_t)H * WS_O) * 2 + 15) / 16) * 16;
    float*         b0 = reinterpret_cast<float*>(smem + wb);
    float*         b1 = b0 + H;
    float*         b2 = b1 + H;
    float*         xs = b2 + WS_O;
    float*         hs = xs + INF_TILE * WS_F;
    const int      j  = threadIdx.x;
    // weights: the BF16 copy (W0, W1, W2 are contiguous there as well)
    const int64_t nw = (int64_t)WS_F * H + (int64_t)H * H + (int64_t)H * WS_O;
    for(int64_t i = j; i < nw; i += blockDim.x)
    {
        const int64_t src = i < (int64_t)WS_F * H ? P.W0 + i
                            : i < (int64_t)WS_F * H + (int64_t)H * H ? P.W1 + (i - (int64_t)WS_F * H)
                                                                     : P.W2 + (i - (int64_t)WS_F * H - (int64_t)H * H);
        W0[i] = w16[src];
    }
    b0[j] = params[P.b0 + j];
    b1[j] = params[P.b1 + j];
    if(j < WS_O)
        b2[j] = params[P.b2 + j];
    __syncthreads();
    const int n_tiles = (rows + INF_TILE - 1) / INF_TILE;
    for(int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x)
    {
        const int a0 = tile * INF_TILE;
        for(int e = j; e < INF_TILE * WS_F; e += blockDim.x)
        {
            const int a = a0 + e / WS_F, f = e % WS_F;
            xs[e]       = a < rows ? (feat[(int64_t)a * WS_F + f] - norm[f]) * norm[WS_F + f] : 0.f;
        }
        __syncthreads();
        float acc[INF_TILE];
#pragma unroll
        for(int a = 0; a < INF_TILE; ++a)
            acc[a] = b0[j];
        for(int f = 0; f < WS_F; ++f)
        {
            const float w = __bfloat162float(W0[f * H + j]);
#pragma unroll
            for(int a = 0; a < INF_TILE; ++a)
                acc[a] = fmaf(xs[a * WS_F + f], w, acc[a]);
        }
#pragma unroll
        for(int a = 0; a < INF_TILE; ++a)
            hs[a * H + j] = fmaxf(acc[a], 0.f);
        __syncthreads();
#pragma unroll
        for(int a = 0; a < INF_TILE; ++a)
            acc[a] = b1[j];
        for(int k = 0; k < H; ++k)
        {
            const float w = __bfloat162float(W1[k * H + j]);
#pragma unroll
            for(int a = 0; a < INF_TILE; ++a)
                acc[a] = fmaf(hs[a * H + k], w, acc[a]);
        }
        __syncthreads();
#pragma unroll
        for(int a = 0; a < INF_TILE; ++a)
            hs[a * H + j] = fmaxf(acc[a], 0.f);
        __syncthreads();
        if(j < INF_TILE * WS_O)
        {
            const int a = j / WS_O, o = j % WS_O;
            float     y = b2[o];
            for(int k = 0; k < H; ++k)
                y = fmaf(hs[a * H + k], __bfloat162float(W2[k * WS_O + o]), y);
            if(a0 + a < rows)
                Y[(int64_t)(a0 + a) * WS_O + o] = y;
        }
        __syncthreads();
    }
}

// The same inference on the tensor cores for width 128 (the width the bench
// and tests use): one warp per 16 aggregates, every layer as mma.m16n8k16
// with BF16 weights (as above) and activations split into BF16 high + low
// parts (two products into one FP32 accumulator: the activations keep ~16
// significant bits). Weights are stored transposed in shared memory, rows
// padded to 8 extra BF16 so the B-fragment loads of a warp hit 32 distinct
// banks. Layer l's accumulator fragments are layer l+1's A fragments (16 x 8
// C tiles 2k and 2k+1 form the 16 x 16 A tile k).
constexpr int MMA_H   = 128;
constexpr int MMA_K1  = 32;            // WS_F = 22 padded
constexpr int MMA_LD1 = MMA_K1 + 8;    // W0t row stride (BF16)
constexpr int MMA_LDH = MMA_H + 8;     // W1t / W2t row stride
constexpr int MMA_WARPS = 4;

size_t inference_mma_smem()
{
    return sizeof(__nv_bfloat16) * ((size_t)MMA_H * MMA_LD1 + (size_t)MMA_H * MMA_LDH + 8 * (size_t)MMA_LDH) +
           sizeof(float) * (2 * MMA_H + 8);
}

__device__ __forceinline__ void mma_16816_bf16(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// two floats as BF16 pairs: high parts and the remainders
__device__ __forceinline__ void split_bf16x2(float x0, float x1, uint32_t& hi, uint32_t& lo)
{
    const __nv_bfloat16 h0 = __float2bfloat16_rn(x0), h1 = __float2bfloat16_rn(x1);
    const __nv_bfloat16 l0 = __float2bfloat16_rn(x0 - __bfloat162float(h0));
    const __nv_bfloat16 l1 = __float2bfloat16_rn(x1 - __bfloat162float(h1));
    hi = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
    lo = (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
}

__device__ __forceinline__ uint32_t ld_b32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

__global__ void __launch_bounds__(MMA_WARPS * 32)
    k_ws_infer_mma(int rows, const __nv_bfloat16* __restrict__ w16, const float* __restrict__ params,
                   const float* __restrict__ feat, const float* __restrict__ norm, float* __restrict__ Y)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const PLayout  P(MMA_H);
    __nv_bfloat16* W0t = reinterpret_cast<__nv_bfloat16*>(smem);          // [H][LD1]: W0t[n][k] = W0[k][n]
    __nv_bfloat16* W1t = W0t + (size_t)MMA_H * MMA_LD1;                      // [H][LDH]
    __nv_bfloat16* W2t = W1t + (size_t)MMA_H * MMA_LDH;                      // [8][LDH] (rows 4..7 zero)
    float*         bs  = reinterpret_cast<float*>(W2t + 8 * MMA_LDH);        // b0[H] b1[H] b2[8]
    const __nv_bfloat16 zero = __float2bfloat16_rn(0.f);
    for(int i = threadIdx.x; i < MMA_H * MMA_LD1; i += blockDim.x)
    {
        const int n = i / MMA_LD1, k = i % MMA_LD1;
        W0t[i]      = k < WS_F ? w16[P.W0 + (int64_t)k * MMA_H + n] : zero;
    }
    for(int i = threadIdx.x; i < MMA_H * MMA_LDH; i += blockDim.x)
    {
        const int n = i / MMA_LDH, k = i % MMA_LDH;
        W1t[i]      = k < MMA_H ? w16[P.W1 + (int64_t)k * MMA_H + n] : zero;
    }
    for(int i = threadIdx.x; i < 8 * MMA_LDH; i += blockDim.x)
    {
        const int n = i / MMA_LDH, k = i % MMA_LDH;
        W2t[i]      = (n < WS_O && k < MMA_H) ? w16[P.W2 + (int64_t)k * WS_O + n] : zero;
    }
    for(int i = threadIdx.x; i < 2 * MMA_H + 8; i += blockDim.x)
        bs[i] = i < MMA_H ? params[P.b0 + i] : i < 2 * MMA_H ? params[P.b1 + i - MMA_H]
                                             : (i - 2 * MMA_H < WS_O ? params[P.b2 + i - 2 * MMA_H] : 0.f);
    __syncthreads();
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int n_tiles = (rows + 15) / 16;
    for(int tile = blockIdx.x * MMA_WARPS + (threadIdx.x >> 5); tile < n_tiles; tile += gridDim.x * MMA_WARPS)
    {
        const int r0 = tile * 16 + g, r1 = r0 + 8;
        // layer 1 A fragments (16 x 32): standardised features
        uint32_t ah[2][4], al[2][4];
#pragma unroll
        for(int kk = 0; kk < 2; ++kk)
#pragma unroll
            for(int q = 0; q < 4; ++q)
            {
                const int r = (q & 1) ? r1 : r0, k = 16 * kk + 2 * t + ((q & 2) ? 8 : 0);
                float     x[2];
#pragma unroll
                for(int e = 0; e < 2; ++e)
                    x[e] = (r < rows && k + e < WS_F) ? (feat[(int64_t)r * WS_F + k + e] - norm[k + e]) * norm[WS_F + k + e]
                                                      : 0.f;
                split_bf16x2(x[0], x[1], ah[kk][q], al[kk][q]);
            }
        float c[16][4];
#pragma unroll
        for(int j = 0; j < 16; ++j)
        {
            const float bb0 = bs[8 * j + 2 * t], bb1 = bs[8 * j + 2 * t + 1];
            c[j][0] = bb0;
            c[j][1] = bb1;
            c[j][2] = bb0;
            c[j][3] = bb1;
#pragma unroll
            for(int kk = 0; kk < 2; ++kk)
            {
                const __nv_bfloat16* wb = W0t + (size_t)(8 * j + g) * MMA_LD1 + 16 * kk + 2 * t;
                const uint32_t       b0 = ld_b32(wb), b1 = ld_b32(wb + 8);
                mma_16816_bf16(c[j], ah[kk], b0, b1);
                mma_16816_bf16(c[j], al[kk], b0, b1);
            }
        }
        // layers 2 and 3: ReLU of the previous layer as the A operand
#pragma unroll
        for(int layer = 0; layer < 2; ++layer)
        {
            uint32_t hh[8][4], hl[8][4];
#pragma unroll
            for(int kk = 0; kk < 8; ++kk)
            {
                split_bf16x2(fmaxf(c[2 * kk][0], 0.f), fmaxf(c[2 * kk][1], 0.f), hh[kk][0], hl[kk][0]);
                split_bf16x2(fmaxf(c[2 * kk][2], 0.f), fmaxf(c[2 * kk][3], 0.f), hh[kk][1], hl[kk][1]);
                split_bf16x2(fmaxf(c[2 * kk + 1][0], 0.f), fmaxf(c[2 * kk + 1][1], 0.f), hh[kk][2], hl[kk][2]);
                split_bf16x2(fmaxf(c[2 * kk + 1][2], 0.f), fmaxf(c[2 * kk + 1][3], 0.f), hh[kk][3], hl[kk][3]);
            }
            if(layer == 0)
            {
#pragma unroll
                for(int j = 0; j < 16; ++j)
                {
                    const float bb0 = bs[MMA_H + 8 * j + 2 * t], bb1 = bs[MMA_H + 8 * j + 2 * t + 1];
                    c[j][0] = bb0;
                    c[j][1] = bb1;
                    c[j][2] = bb0;
                    c[j][3] = bb1;
#pragma unroll
                    for(int kk = 0; kk < 8; ++kk)
                    {
                        const __nv_bfloat16* wb = W1t + (size_t)(8 * j + g) * MMA_LDH + 16 * kk + 2 * t;
                        const uint32_t       b0 = ld_b32(wb), b1 = ld_b32(wb + 8);
                        mma_16816_bf16(c[j], hh[kk], b0, b1);
                        mma_16816_bf16(c[j], hl[kk], b0, b1);
                    }
                }
            }
            else
            {
                float y[4] = {bs[2 * MMA_H + 2 * t], bs[2 * MMA_H + 2 * t + 1], bs[2 * MMA_H + 2 * t],
                              bs[2 * MMA_H + 2 * t + 1]};
#pragma unroll
                for(int kk = 0; kk < 8; ++kk)
                {
                    const __nv_bfloat16* wb = W2t + (size_t)g * MMA_LDH + 16 * kk + 2 * t;
                    const uint32_t       b0 = ld_b32(wb), b1 = ld_b32(wb + 8);
                    mma_16816_bf16(y, hh[kk], b0, b1);
                    mma_16816_bf16(y, hl[kk], b0, b1);
                }
                // y: rows g / g+8, output columns 2t, 2t+1 (the 4 outputs: t < 2)
                if(t < 2)
                {
                    if(r0 < rows)
                    {
                        Y[(int64_t)r0 * WS_O + 2 * t]     = y[0];
                        Y[(int64_t)r0 * WS_O + 2 * t + 1] = y[1];
                    }
                    if(r1 < rows)
                    {
                        Y[(int64_t)r1 * WS_O + 2 * t]     = y[2];
                        Y[(int64_t)r1 * WS_O + 2 * t + 1] = y[3];
                    }
                }
            }
        }
    }
}

// d(v) = sum_i Y[a(v)][i] f_i(v) on the MAS vertices, 0 elsewhere
__global__ void k_ws_combine(int64_t n, int vn, int off, int L, int level1_begin, int n_agg,
                             const int32_t* __restrict__ ctable, const float* __restrict__ Y,
                             const double* __restrict__ f, double* __restrict__ d)
{
    for(int64_t i = (int64_t)blockIdx.x * WS_BLOCK + threadIdx.x; i < n; i += (int64_t)gridDim.x * WS_BLOCK)
    {
        const int64_t v = i / 3 - off;
        double        o = 0.0;
        if(v >= 0 && v < vn)
        {
            const int a = agg_of(ctable, L, level1_begin, (int)v);
            if(a >= 0 && a < n_agg)
                for(int k = 0; k < WS_FIELDS; ++k)
                    o += (double)Y[(int64_t)a * WS_O + k] * f[k * n + i];
        }
        d[i] = o;
    }
}

// the candidate starts of one prediction: the network field and the history
constexpr int WS_MAXC = 1 + B2S_WS_MAX_HISTORY;
struct Cands
{
    const double* c[WS_MAXC];
    double        a[WS_MAXC];
};

// x = sum_k alpha_k c_k (k < nc)
__global__ void k_ws_lincomb(int64_t n, int nc, Cands cs, double* __restrict__ x)
{
    for(int64_t i = (int64_t)blockIdx.x * WS_BLOCK + threadIdx.x; i < n; i += (int64_t)gridDim.x * WS_BLOCK)
    {
        double v = cs.a[0] * cs.c[0][i];
        for(int k = 1; k < nc; ++k)
            v += cs.a[k] * cs.c[k][i];
        x[i] = v;
    }
}

// The Galerkin matrix of the candidate starts, G_ij = c_i . A c_j (i <= j,
// row-major upper triangle), in one pass over the stored upper blocks with no
// product vectors: with u_k = B c_k(col), a block B at (row, col) adds
// c_i(row) . u_j and, off the diagonal (the transposed block), u_i . c_j(row).
// FP64, fixed grid and order: deterministic.
template <int K>
__global__ void __launch_bounds__(RED_BLOCK) k_ws_gram(int64_t U, int64_t S, const int32_t* __restrict__ rows,
                                                       const int32_t* __restrict__ cols,
                                                       const double* __restrict__ vals, Cands cs, double* partials,
                                                       unsigned int* counter, double* out)
{
    constexpr int NP = K * (K + 1) / 2;
    double        g[NP] = {};
    for(int64_t o = (int64_t)blockIdx.x * RED_BLOCK + threadIdx.x; o < U; o += (int64_t)gridDim.x * RED_BLOCK)
    {
        const int64_t r = rows[o], c = cols[o];
        double        B[9];
#pragma unroll
        for(int q = 0; q < 9; ++q)
            B[q] = vals[(int64_t)q * S + o];
        double xr[K][3], u[K][3];
#pragma unroll
        for(int k = 0; k < K; ++k)
        {
            const double* ck = cs.c[k];
            xr[k][0]          = ck[3 * r];
            xr[k][1]          = ck[3 * r + 1];
            xr[k][2]          = ck[3 * r + 2];
            const double y0 = ck[3 * c], y1 = ck[3 * c + 1], y2 = ck[3 * c + 2];
            // column-major: B(p, q) = B[q * 3 + p]
            u[k][0] = B[0] * y0 + B[3] * y1 + B[6] * y2;
            u[k][1] = B[1] * y0 + B[4] * y1 + B[7] * y2;
            u[k][2] = B[2] * y0 + B[5] * y1 + B[8] * y2;
        }
        const bool off = r != c;
        int        p   = 0;
#pragma unroll
        for(int i = 0; i < K; ++i)
#pragma unroll
            for(int j = i; j < K; ++j, ++p)
            {
                double d = xr[i][0] * u[j][0] + xr[i][1] * u[j][1] + xr[i][2] * u[j][2];
                if(off)
                    d += u[i][0] * xr[j][0] + u[i][1] * xr[j][1] + u[i][2] * xr[j][2];
                g[p] += d;
            }
    }
    double tot[NP];
    if(grid_sum<NP>(g, partials, counter, tot))
        for(int q = 0; q < NP; ++q)
            out[q] = tot[q];
}

// r = b - sum_k alpha_k y_k (k < nc)
__global__ void k_ws_residual_comb(int64_t n, int nc, const double* __restrict__ b, const double* __restrict__ y0,
                                   const double* __restrict__ y1, const double* __restrict__ y2,
                                   const double* __restrict__ y3, double a0, double a1, double a2, double a3,
                                   double* __restrict__ r)
{
    for(int64_t i = (int64_t)blockIdx.x * WS_BLOCK + threadIdx.x; i < n; i += (int64_t)gridDim.x * WS_BLOCK)
    {
        double v = b[i] - a0 * y0[i];
        if(nc > 1)
            v -= a1 * y1[i];
        if(nc > 2)
            v -= a2 * y2[i];
        if(nc > 3)
            v -= a3 * y3[i];
        r[i] = v;
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
LearnedState& ws_of(b2s_solver* s)
{
    B2S_REQUIRE(s->ws != nullptr && s->ws->hidden > 0, B2S_ERR_STATE,
                "learned warm start not initialised (b2s_ws_init)");
    return *s->ws;
}

struct MasGeom
{
    int vn, off, L, level1_begin, n_agg;
    const int32_t* ctable;
};

MasGeom mas_geom(b2s_solver* s)
{
    const MasState& M = s->mas;
    B2S_REQUIRE(s->A.valid, B2S_ERR_STATE, "no assembled matrix");
    B2S_REQUIRE(M.initialized && s->precond_kind == B2S_PRECOND_MAS, B2S_ERR_STATE,
                "the learned warm start needs the MAS preconditioner (b2s_precond_assemble)");
    B2S_REQUIRE(M.L >= 2, B2S_ERR_STATE, "the MAS hierarchy has no level-1 aggregates");
    return MasGeom{M.vn, M.offset, M.L, M.level_begin[1], M.level_count[1], M.ctable.data()};
}


// fields, scales and the per-aggregate accumulators of the current system;
// x (nullable) adds the training statistics. Returns the aggregate count.
int system_aggregates(b2s_solver* s, const double* b, int n_hist, const double* const* hist, const double* x)
{
    LearnedState& W  = *s->ws;
    const MasGeom g  = mas_geom(s);
    cudaStream_t  st = s->stream;
    const int64_t n  = 3 * (int64_t)s->A.nb;
    B2S_REQUIRE(n_hist >= 0 && n_hist <= B2S_WS_MAX_HISTORY, B2S_ERR_ARGUMENT, "history length outside [0, 8]");
    for(int i = 0; i < n_hist; ++i)
        B2S_REQUIRE(hist && hist[i], B2S_ERR_ARGUMENT, "null history vector");
    W.fields.resize((size_t)WS_FIELDS * n);
    W.Ac.resize((size_t)5 * n);
    W.dots.resize(32);
    precond_launch(s, b, W.Ac.data());  // z = P b
    k_ws_fields<<<ws_grid(n), WS_BLOCK, 0, st>>>(n, n_hist > 0 ? hist[0] : nullptr, n_hist > 1 ? hist[1] : nullptr,
                                                  n_hist > 2 ? hist[2] : nullptr, W.Ac.data(), W.fields.data());
    B2S_CHECK_LAUNCH();
    DotPairs dp{};
    dp.a[0] = dp.b[0] = W.Ac.data();
    dp.a[1] = dp.b[1] = b;
    launch_dots(s, n, dp, 2, W.dots.data() + 28);
    double h2[2];
    B2S_CUDA(cudaMemcpyAsync(h2, W.dots.data() + 28, sizeof(h2), cudaMemcpyDeviceToHost, st));
    B2S_CUDA(cudaStreamSynchronize(st));
    const double zz = h2[0], bb = h2[1];
    const double sz = zz > 0 ? std::sqrt(zz / (double)n) : 1.0;
    const double sb = bb > 0 ? std::sqrt(bb / (double)n) : 1.0;
    W.acc.resize((size_t)g.n_agg * WS_ACC);
    B2S_CUDA(cudaMemsetAsync(W.acc.data(), 0, W.acc.bytes(), st));
    k_ws_accumulate<<<ws_grid(g.vn), WS_BLOCK, 0, st>>>(g.vn, g.off, g.L, g.level1_begin, g.n_agg, g.ctable, b,
                                                        W.fields.data(), n, x, 1.0 / sb, 1.0 / sz, W.acc.data());
    B2S_CHECK_LAUNCH();
    return g.n_agg;
}

void upload_norm(LearnedState& W)
{
    std::vector<float> h(2 * WS_F);
    for(int j = 0; j < WS_F; ++j)
    {
        h[j]        = W.mean[j];
        h[WS_F + j] = 1.0f / std::max(W.stdv[j], 1e-3f);
    }
    W.norm_dev.resize(2 * WS_F);
    B2S_CUDA(cudaMemcpy(W.norm_dev.data(), h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice));
}

// grow a device array to `cap` elements keeping its first `keep`
template <typename T>
void grow_keep(DBuf<T>& buf, size_t keep, size_t cap, cudaStream_t st)
{
    if(buf.cap >= cap)
    {
        buf.n = cap;
        return;
    }
    T* p = nullptr;
    B2S_CUDA(cudaMalloc(&p, cap * sizeof(T)));
    if(keep > 0)
        B2S_CUDA(cudaMemcpyAsync(p, buf.ptr, keep * sizeof(T), cudaMemcpyDeviceToDevice, st));
    B2S_CUDA(cudaStreamSynchronize(st));
    buf.release();
    buf.ptr = p;
    buf.n = buf.cap = cap;
}

// forward (and, with want_grad, backward into W.grad) of stored sample i;
// adds its normalised loss into W.loss_dev[0]
void forward_backward(b2s_solver* s, const WsSample& smp, bool want_grad)
{
    LearnedState& W  = *s->ws;
    cudaStream_t  st = s->stream;
    const int     H  = W.hidden, R = smp.rows;
    const PLayout P(H);
    float*        p  = W.params.data();
    float*        gr = W.grad.data();
    W.X.resize((size_t)R * WS_F);
    W.H1.resize((size_t)R * H);
    W.H2.resize((size_t)R * H);
    W.dH.resize((size_t)R * H);
    W.Y.resize((size_t)R * WS_O);
    W.dY.resize((size_t)R * WS_O);
    k_ws_standardise<<<ws_grid((int64_t)R * WS_F), WS_BLOCK, 0, st>>>(R, W.st_feat.data() + smp.row0 * WS_F,
                                                                       W.norm_dev.data(), W.X.data());
    B2S_CHECK_LAUNCH();
    gemm<false, false>(st, R, H, WS_F, W.X.data(), WS_F, p + P.W0, H, W.H1.data(), H, false);
    k_bias_act<<<ws_grid((int64_t)R * H), WS_BLOCK, 0, st>>>(R, H, W.H1.data(), p + P.b0, 1);
    B2S_CHECK_LAUNCH();
    gemm<false, false>(st, R, H, H, W.H1.data(), H, p + P.W1, H, W.H2.data(), H, false);
    k_bias_act<<<ws_grid((int64_t)R * H), WS_BLOCK, 0, st>>>(R, H, W.H2.data(), p + P.b1, 1);
    B2S_CHECK_LAUNCH();
    gemm<false, false>(st, R, WS_O, H, W.H2.data(), H, p + P.W2, WS_O, W.Y.data(), WS_O, false);
    k_bias_act<<<ws_grid((int64_t)R * WS_O), WS_BLOCK, 0, st>>>(R, WS_O, W.Y.data(), p + P.b2, 0);
    B2S_CHECK_LAUNCH();
    k_ws_loss<<<(R + WS_BLOCK - 1) / WS_BLOCK, WS_BLOCK, 0, st>>>(
        R, W.Y.data(), W.st_H.data() + smp.row0 * WS_HSYM, W.st_q.data() + smp.row0 * WS_O,
        W.st_c0.data() + smp.row0, (float)(1.0 / std::max(smp.norm, 1e-30)), W.dY.data(), W.loss_dev.data());
    B2S_CHECK_LAUNCH();
    if(!want_grad)
        return;
    B2S_CUDA(cudaMemsetAsync(gr, 0, sizeof(float) * W.n_params, st));
    const int rpb = 256;
    const int cs_grid = (R + rpb - 1) / rpb;
    // layer 3
    gemm<true, false>(st, H, WS_O, R, W.H2.data(), H, W.dY.data(), WS_O, gr + P.W2, WS_O, true);
    k_colsum<<<cs_grid, 32, 0, st>>>(R, WS_O, W.dY.data(), gr + P.b2, rpb);
    B2S_CHECK_LAUNCH();
    gemm<false, true>(st, R, H, WS_O, W.dY.data(), WS_O, p + P.W2, WS_O, W.dH.data(), H, false);
    k_relu_mask<<<ws_grid((int64_t)R * H), WS_BLOCK, 0, st>>>((int64_t)R * H, W.dH.data(), W.H2.data());
    B2S_CHECK_LAUNCH();
    // layer 2 (dZ2 in dH; dH1 goes into the H2 buffer)
    gemm<true, false>(st, H, H, R, W.H1.data(), H, W.dH.data(), H, gr + P.W1, H, true);
    k_colsum<<<cs_grid, H, 0, st>>>(R, H, W.dH.data(), gr + P.b1, rpb);
    B2S_CHECK_LAUNCH();
    gemm<false, true>(st, R, H, H, W.dH.data(), H, p + P.W1, H, W.H2.data(), H, false);
    k_relu_mask<<<ws_grid((int64_t)R * H), WS_BLOCK, 0, st>>>((int64_t)R * H, W.H2.data(), W.H1.data());
    B2S_CHECK_LAUNCH();
    // layer 1
    gemm<true, false>(st, WS_F, H, R, W.X.data(), WS_F, W.H2.data(), H, gr + P.W0, H, true);
    k_colsum<<<cs_grid, H, 0, st>>>(R, H, W.H2.data(), gr + P.b0, rpb);
    B2S_CHECK_LAUNCH();
}

// symmetric pseudo-inverse solve (k <= 4) by Jacobi rotations on the
// diagonally scaled matrix
void small_pinv_solve(int k, const double* G, const double* g, double* alpha)
{
    double a[WS_MAXC * WS_MAXC], v[WS_MAXC * WS_MAXC], d[WS_MAXC];
    for(int i = 0; i < k; ++i)
        d[i] = G[i * k + i] > 0 ? 1.0 / std::sqrt(G[i * k + i]) : 0.0;
    for(int i = 0; i < k; ++i)
        for(int j = 0; j < k; ++j)
        {
            a[i * k + j] = G[i * k + j] * d[i] * d[j];
            v[i * k + j] = i == j ? 1.0 : 0.0;
        }
    for(int sweep = 0; sweep < 60; ++sweep)
    {
        double off = 0.0;
        for(int i = 0; i < k; ++i)
            for(int j = i + 1; j < k; ++j)
                off += a[i * k + j] * a[i * k + j];
        if(off < 1e-30)
            break;
        for(int p = 0; p < k; ++p)
            for(int q = p + 1; q < k; ++q)
            {
                const double apq = a[p * k + q];
                if(std::fabs(apq) < 1e-300)
                    continue;
                const double th = 0.5 * (a[q * k + q] - a[p * k + p]) / apq;
                const double t  = (th >= 0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
                for(int r = 0; r < k; ++r)
                {
                    const double arp = a[r * k + p], arq = a[r * k + q];
                    a[r * k + p]     = c * arp - sn * arq;
                    a[r * k + q]     = sn * arp + c * arq;
                }
                for(int r = 0; r < k; ++r)
                {
                    const double apr = a[p * k + r], aqr = a[q * k + r];
                    a[p * k + r]     = c * apr - sn * aqr;
                    a[q * k + r]     = sn * apr + c * aqr;
                }
                for(int r = 0; r < k; ++r)
                {
                    const double vrp = v[r * k + p], vrq = v[r * k + q];
                    v[r * k + p]     = c * vrp - sn * vrq;
                    v[r * k + q]     = sn * vrp + c * vrq;
                }
            }
    }
    double lmax = 0.0;
    for(int i = 0; i < k; ++i)
        lmax = std::max(lmax, a[i * k + i]);
    double gs[WS_MAXC];
    for(int i = 0; i < k; ++i)
        gs[i] = g[i] * d[i];
    for(int i = 0; i < k; ++i)
        alpha[i] = 0.0;
    for(int e = 0; e < k; ++e)
    {
        const double lam = a[e * k + e];
        if(!(lam > 1e-13 * lmax))
            continue;
        double proj = 0.0;
        for(int i = 0; i < k; ++i)
            proj += v[i * k + e] * gs[i];
        for(int i = 0; i < k; ++i)
            alpha[i] += v[i * k + e] * proj / lam;
    }
    for(int i = 0; i < k; ++i)
        alpha[i] *= d[i];
}
}  // namespace

void ws_init(b2s_solver* s, int hidden, uint64_t seed)
{
    B2S_REQUIRE(hidden >= 64 && hidden <= 512 && hidden % 32 == 0, B2S_ERR_ARGUMENT,
                "hidden width must be a multiple of 32 in [64, 512]");
    if(!s->ws)
        s->ws = new LearnedState();
    LearnedState& W = *s->ws;
    W.hidden        = hidden;
    const PLayout P(hidden);
    W.n_params = P.n;
    std::vector<float> h(P.n, 0.0f);
    std::mt19937_64    rng(seed);
    std::normal_distribution<double> nd(0.0, 1.0);
    for(int64_t i = 0; i < (int64_t)WS_F * hidden; ++i)
        h[P.W0 + i] = (float)(nd(rng) * std::sqrt(2.0 / WS_F));
    for(int64_t i = 0; i < (int64_t)hidden * hidden; ++i)
        h[P.W1 + i] = (float)(nd(rng) * std::sqrt(2.0 / hidden));
    for(int64_t i = 0; i < (int64_t)hidden * WS_O; ++i)
        h[P.W2 + i] = (float)(nd(rng) * 0.01);
    W.params.resize(P.n);
    W.grad.resize(P.n);
    W.adam_m.resize(P.n);
    W.adam_v.resize(P.n);
    B2S_CUDA(cudaMemcpy(W.params.data(), h.data(), sizeof(float) * P.n, cudaMemcpyHostToDevice));
    B2S_CUDA(cudaMemset(W.adam_m.data(), 0, sizeof(float) * P.n));
    B2S_CUDA(cudaMemset(W.adam_v.data(), 0, sizeof(float) * P.n));
    W.adam_t = 0;
    W.mean.assign(WS_F, 0.0f);
    W.stdv.assign(WS_F, 1.0f);
    upload_norm(W);
    W.loss_dev.resize(1);
    W.version++;
    if(!W.ev0)
    {
        B2S_CUDA(cudaEventCreate(&W.ev0));
        B2S_CUDA(cudaEventCreate(&W.ev1));
    }
}

void ws_add_sample(b2s_solver* s, const double* b, int n_hist, const double* const* hist, const double* x)
{
    LearnedState& W = ws_of(s);
    B2S_REQUIRE(b && x, B2S_ERR_ARGUMENT, "null b or x");
    cudaStream_t st = s->stream;
    const int    na = system_aggregates(s, b, n_hist, hist, x);
    const int64_t r0 = W.store_rows, r1 = r0 + na;
    if(r1 > W.store_cap)
    {
        const int64_t cap = std::max<int64_t>(r1, W.store_cap * 2);
        grow_keep(W.st_feat, (size_t)r0 * WS_F, (size_t)cap * WS_F, st);
        grow_keep(W.st_H, (size_t)r0 * WS_HSYM, (size_t)cap * WS_HSYM, st);
        grow_keep(W.st_q, (size_t)r0 * WS_O, (size_t)cap * WS_O, st);
        grow_keep(W.st_c0, (size_t)r0, (size_t)cap, st);
        W.store_cap = cap;
    }
    k_ws_features<<<(na + WS_BLOCK - 1) / WS_BLOCK, WS_BLOCK, 0, st>>>(
        na, W.acc.data(), W.st_feat.data() + r0 * WS_F, W.st_H.data() + r0 * WS_HSYM, W.st_q.data() + r0 * WS_O,
        W.st_c0.data() + r0);
    B2S_CHECK_LAUNCH();
    std::vector<float> c0(na);
    B2S_CUDA(cudaMemcpyAsync(c0.data(), W.st_c0.data() + r0, sizeof(float) * na, cudaMemcpyDeviceToHost, st));
    B2S_CUDA(cudaStreamSynchronize(st));
    double norm = 0.0;
    for(float c : c0)
        norm += c;
    W.samples.push_back(WsSample{r0, na, norm});
    W.store_rows = r1;
}

// append a stored sample from host arrays (a training set read back from a
// checkpoint): rows aggregates of features, field Gram, q, |x|^2 and the
// sample's loss normaliser
void ws_put_sample(b2s_solver* s, int32_t rows, const float* feat, const float* Hs, const float* q, const float* c0,
                   double norm)
{
    LearnedState& W = ws_of(s);
    B2S_REQUIRE(rows > 0 && feat && Hs && q && c0, B2S_ERR_ARGUMENT, "empty or null sample");
    B2S_REQUIRE(std::isfinite(norm) && norm > 0.0, B2S_ERR_ARGUMENT, "sample normaliser must be positive");
    cudaStream_t  st = s->stream;
    const int64_t r0 = W.store_rows, r1 = r0 + rows;
    if(r1 > W.store_cap)
    {
        const int64_t cap = std::max<int64_t>(r1, W.store_cap * 2);
        grow_keep(W.st_feat, (size_t)r0 * WS_F, (size_t)cap * WS_F, st);
        grow_keep(W.st_H, (size_t)r0 * WS_HSYM, (size_t)cap * WS_HSYM, st);
        grow_keep(W.st_q, (size_t)r0 * WS_O, (size_t)cap * WS_O, st);
        grow_keep(W.st_c0, (size_t)r0, (size_t)cap, st);
        W.store_cap = cap;
    }
    B2S_CUDA(cudaMemcpyAsync(W.st_feat.data() + r0 * WS_F, feat, sizeof(float) * rows * WS_F, cudaMemcpyDefault, st));
    B2S_CUDA(cudaMemcpyAsync(W.st_H.data() + r0 * WS_HSYM, Hs, sizeof(float) * rows * WS_HSYM, cudaMemcpyDefault, st));
    B2S_CUDA(cudaMemcpyAsync(W.st_q.data() + r0 * WS_O, q, sizeof(float) * rows * WS_O, cudaMemcpyDefault, st));
    B2S_CUDA(cudaMemcpyAsync(W.st_c0.data() + r0, c0, sizeof(float) * rows, cudaMemcpyDefault, st));
    B2S_CUDA(cudaStreamSynchronize(st));
    W.samples.push_back(WsSample{r0, rows, norm});
    W.store_rows = r1;
}

void ws_num_samples(b2s_solver* s, int32_t* n, int64_t* rows)
{
    LearnedState& W = ws_of(s);
    if(n)
        *n = (int32_t)W.samples.size();
    if(rows)
        *rows = W.store_rows;
}

void ws_fit_normalization(b2s_solver* s)
{
    LearnedState& W = ws_of(s);
    B2S_REQUIRE(W.store_rows > 0, B2S_ERR_STATE, "no stored samples");
    std::vector<float> f((size_t)W.store_rows * WS_F);
    B2S_CUDA(cudaMemcpy(f.data(), W.st_feat.data(), sizeof(float) * f.size(), cudaMemcpyDeviceToHost));
    for(int j = 0; j < WS_F; ++j)
    {
        double m = 0.0, q = 0.0;
        for(int64_t r = 0; r < W.store_rows; ++r)
            m += f[(size_t)r * WS_F + j];
        m /= (double)W.store_rows;
        for(int64_t r = 0; r < W.store_rows; ++r)
        {
            const double d = f[(size_t)r * WS_F + j] - m;
            q += d * d;
        }
        W.mean[j] = (float)m;
        W.stdv[j] = (float)std::sqrt(q / (double)W.store_rows);
    }
    upload_norm(W);
}

double ws_train(b2s_solver* s, int epochs, double lr, uint64_t seed)
{
    LearnedState& W = ws_of(s);
    B2S_REQUIRE(!W.samples.empty(), B2S_ERR_STATE, "no stored samples");
    B2S_REQUIRE(epochs >= 1 && lr > 0, B2S_ERR_ARGUMENT, "epochs >= 1 and lr > 0");
    cudaStream_t      st = s->stream;
    std::mt19937_64   rng(seed);
    std::vector<int>  order(W.samples.size());
    double            last = 0.0;
    const float       b1 = 0.9f, b2 = 0.999f;
    for(int ep = 0; ep < epochs; ++ep)
    {
        std::iota(order.begin(), order.end(), 0);
        std::shuffle(order.begin(), order.end(), rng);
        B2S_CUDA(cudaMemsetAsync(W.loss_dev.data(), 0, sizeof(float), st));
        for(int i : order)
        {
            forward_backward(s, W.samples[i], true);
            W.adam_t++;
            const float c1 = 1.0f / (1.0f - std::pow(b1, (float)W.adam_t));
            const float c2 = 1.0f / (1.0f - std::pow(b2, (float)W.adam_t));
            k_adam<<<ws_grid(W.n_params), WS_BLOCK, 0, st>>>(W.n_params, W.params.data(), W.grad.data(),
                                                            W.adam_m.data(), W.adam_v.data(), (float)lr, b1, b2,
                                                            1e-8f, c1, c2);
            B2S_CHECK_LAUNCH();
        }
        float h = 0.f;
        B2S_CUDA(cudaMemcpyAsync(&h, W.loss_dev.data(), sizeof(float), cudaMemcpyDeviceToHost, st));
        B2S_CUDA(cudaStreamSynchronize(st));
        last = (double)h / (double)order.size();
    }
    W.version++;
    return last;
}

double ws_loss_grad(b2s_solver* s, int index, float* h_grad)
{
    LearnedState& W = ws_of(s);
    B2S_REQUIRE(index >= 0 && index < (int)W.samples.size(), B2S_ERR_ARGUMENT, "sample index out of range");
    cudaStream_t st = s->stream;
    B2S_CUDA(cudaMemsetAsync(W.loss_dev.data(), 0, sizeof(float), st));
    forward_backward(s, W.samples[index], true);
    float h = 0.f;
    B2S_CUDA(cudaMemcpyAsync(&h, W.loss_dev.data(), sizeof(float), cudaMemcpyDeviceToHost, st));
    if(h_grad)
        B2S_CUDA(cudaMemcpyAsync(h_grad, W.grad.data(), sizeof(float) * W.n_params, cudaMemcpyDeviceToHost, st));
    B2S_CUDA(cudaStreamSynchronize(st));
    return (double)h;
}

int64_t ws_get_params(b2s_solver* s, float* h)
{
    LearnedState& W = ws_of(s);
    if(h)
    {
        B2S_CUDA(cudaMemcpy(h, W.params.data(), sizeof(float) * W.n_params, cudaMemcpyDeviceToHost));
        std::memcpy(h + W.n_params, W.mean.data(), sizeof(float) * WS_F);
        std::memcpy(h + W.n_params + WS_F, W.stdv.data(), sizeof(float) * WS_F);
    }
    return W.n_params + 2 * WS_F;
}

void ws_set_params(b2s_solver* s, const float* h, int64_t n)
{
    LearnedState& W = ws_of(s);
    B2S_REQUIRE(h && n == W.n_params + 2 * WS_F, B2S_ERR_ARGUMENT, "parameter count does not match the network");
    B2S_CUDA(cudaMemcpy(W.params.data(), h, sizeof(float) * W.n_params, cudaMemcpyHostToDevice));
    std::memcpy(W.mean.data(), h + W.n_params, sizeof(float) * WS_F);
    std::memcpy(W.stdv.data(), h + W.n_params + WS_F, sizeof(float) * WS_F);
    upload_norm(W);
    W.version++;
}

int ws_get_sample(b2s_solver* s, int index, float* feat, float* Hs, float* q, float* c0, double* norm)
{
    LearnedState& W = ws_of(s);
    B2S_REQUIRE(index >= 0 && index < (int)W.samples.size(), B2S_ERR_ARGUMENT, "sample index out of range");
    const WsSample& m = W.samples[index];
    if(feat)
        B2S_CUDA(cudaMemcpy(feat, W.st_feat.data() + m.row0 * WS_F, sizeof(float) * m.rows * WS_F,
                            cudaMemcpyDeviceToHost));
    if(Hs)
        B2S_CUDA(cudaMemcpy(Hs, W.st_H.data() + m.row0 * WS_HSYM, sizeof(float) * m.rows * WS_HSYM,
                            cudaMemcpyDeviceToHost));
    if(q)
        B2S_CUDA(cudaMemcpy(q, W.st_q.data() + m.row0 * WS_O, sizeof(float) * m.rows * WS_O, cudaMemcpyDeviceToHost));
    if(c0)
        B2S_CUDA(cudaMemcpy(c0, W.st_c0.data() + m.row0, sizeof(float) * m.rows, cudaMemcpyDeviceToHost));
    if(norm)
        *norm = m.norm;
    return m.rows;
}

void ws_predict(b2s_solver* s, int mode, const double* b, int n_hist, const double* const* hist, double* x0,
                b2s_ws_info* info)
{
    B2S_REQUIRE(mode >= B2S_WS_MODE_ZERO && mode <= B2S_WS_MODE_LEARNED, B2S_ERR_ARGUMENT, "unknown warm-start mode");
    B2S_REQUIRE(b && x0, B2S_ERR_ARGUMENT, "null b or x0");
    B2S_REQUIRE(s->A.valid, B2S_ERR_STATE, "no assembled matrix");
    B2S_REQUIRE(n_hist >= 0 && n_hist <= B2S_WS_MAX_HISTORY, B2S_ERR_ARGUMENT, "history length outside [0, 8]");
    for(int i = 0; i < n_hist; ++i)
        B2S_REQUIRE(hist && hist[i], B2S_ERR_ARGUMENT, "null history vector");
    b2s_ws_info out{};
    out.mode          = B2S_WS_MODE_ZERO;
    out.rel_res0      = 1.0;
    out.rel_res_tried = 1.0;
    cudaStream_t  st = s->stream;
    const int64_t n  = 3 * (int64_t)s->A.nb;
    if(!s->ws)
        s->ws = new LearnedState();
    LearnedState& W = *s->ws;
    if(!W.ev0)
    {
        B2S_CUDA(cudaEventCreate(&W.ev0));
        B2S_CUDA(cudaEventCreate(&W.ev1));
    }
    B2S_CUDA(cudaEventRecord(W.ev0, st));
    // candidate vectors
    std::vector<const double*> cand;
    if(mode == B2S_WS_MODE_LEARNED)
    {
        B2S_REQUIRE(W.hidden > 0, B2S_ERR_STATE, "learned warm start not initialised (b2s_ws_init)");
        const MasGeom g  = mas_geom(s);
        const int     na = system_aggregates(s, b, n_hist, hist, nullptr);
        W.feat.resize((size_t)na * WS_F);
        W.Y.resize((size_t)na * WS_O);
        k_ws_features<<<(na + WS_BLOCK - 1) / WS_BLOCK, WS_BLOCK, 0, st>>>(na, W.acc.data(), W.feat.data(), nullptr,
                                                                           nullptr, nullptr);
        B2S_CHECK_LAUNCH();
        if(W.w16_version != W.version)
        {
            W.w16.resize(W.n_params);
            k_to_bf16<<<ws_grid(W.n_params), WS_BLOCK, 0, st>>>(W.n_params, W.params.data(), W.w16.data());
            B2S_CHECK_LAUNCH();
            W.w16_version = W.version;
        }
        if(W.hidden == MMA_H)
        {
            const size_t smem = inference_mma_smem();
            B2S_CUDA(cudaFuncSetAttribute(k_ws_infer_mma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            const int tiles = (na + 15) / 16;
            const int grid  = std::max(1, std::min((tiles + MMA_WARPS - 1) / MMA_WARPS, NUM_SMS_HINT * 2));
            k_ws_infer_mma<<<grid, MMA_WARPS * 32, smem, st>>>(na, W.w16.data(), W.params.data(), W.feat.data(),
                                                               W.norm_dev.data(), W.Y.data());
        }
        else
        {
            const size_t smem = inference_smem(W.hidden);
            B2S_CUDA(cudaFuncSetAttribute(k_ws_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            const int tiles = (na + INF_TILE - 1) / INF_TILE;
            k_ws_infer<<<std::max(1, std::min(tiles, NUM_SMS_HINT * 2)), W.hidden, smem, st>>>(
                na, W.hidden, W.w16.data(), W.params.data(), W.feat.data(), W.norm_dev.data(), W.Y.data());
        }
        B2S_CHECK_LAUNCH();
        W.d_mlp.resize(n);
        k_ws_combine<<<ws_grid(n), WS_BLOCK, 0, st>>>(n, g.vn, g.off, g.L, g.level1_begin, na, g.ctable, W.Y.data(),
                                                     W.fields.data(), W.d_mlp.data());
        B2S_CHECK_LAUNCH();
        cand.push_back(W.d_mlp.data());
    }
    if(mode == B2S_WS_MODE_PREV && n_hist > 0)
        cand.push_back(hist[0]);
    if(mode == B2S_WS_MODE_HISTORY || mode == B2S_WS_MODE_LEARNED)
        for(int i = 0; i < n_hist; ++i)
            cand.push_back(hist[i]);
    const int k = (int)cand.size();
    bool      have = false;
    if(k > 0)
    {
        // Galerkin: G alpha = g, G_kl = c_k . A c_l (one pass over the
        // matrix), g_k = c_k . b and b . b (one pass over the vectors), FP64.
        // dots: [0, 45) the Gram's upper triangle, [48, 48 + k] the right-hand
        // side and b . b, [60, 63) the acceptance check
        W.Ac.resize((size_t)4 * n);
        W.dots.resize(64);
        const Matrix& A    = s->A;
        const int     grid = reduction_grid();
        ensure_reduction(s->red, grid, WS_MAXC * (WS_MAXC + 1) / 2);
        Cands cs{};
        for(int i = 0; i < WS_MAXC; ++i)
            cs.c[i] = cand[i < k ? i : 0];
        double* gram = W.dots.data();
        auto    gram_launch = [&](auto K) {
            constexpr int KK = decltype(K)::value;
            k_ws_gram<KK><<<grid, RED_BLOCK, 0, st>>>(A.nnz, A.stride, A.rows.data(), A.cols.data(), A.vals.data(),
                                                      cs, s->red.partials.data(), s->red.counter.data(), gram);
        };
        switch(k)
        {
        case 1: gram_launch(std::integral_constant<int, 1>{}); break;
        case 2: gram_launch(std::integral_constant<int, 2>{}); break;
        case 3: gram_launch(std::integral_constant<int, 3>{}); break;
        case 4: gram_launch(std::integral_constant<int, 4>{}); break;
        case 5: gram_launch(std::integral_constant<int, 5>{}); break;
        case 6: gram_launch(std::integral_constant<int, 6>{}); break;
        case 7: gram_launch(std::integral_constant<int, 7>{}); break;
        case 8: gram_launch(std::integral_constant<int, 8>{}); break;
        default: gram_launch(std::integral_constant<int, WS_MAXC>{}); break;
        }
        B2S_CHECK_LAUNCH();
        DotPairs dp{};
        for(int i = 0; i < k; ++i)
        {
            dp.a[i] = cand[i];
            dp.b[i] = b;
        }
        dp.a[k] = dp.b[k] = b;
        launch_dots(s, n, dp, k + 1, W.dots.data() + 48);
        double hd[64];
        B2S_CUDA(cudaMemcpyAsync(hd, W.dots.data(), sizeof(hd), cudaMemcpyDeviceToHost, st));
        B2S_CUDA(cudaStreamSynchronize(st));
        double G[WS_MAXC * WS_MAXC], gv[WS_MAXC], alpha[WS_MAXC] = {};
        for(int i = 0, q = 0; i < k; ++i)
        {
            for(int j = i; j < k; ++j, ++q)
                G[i * k + j] = G[j * k + i] = hd[q];
            gv[i] = hd[48 + i];
        }
        small_pinv_solve(k, G, gv, alpha);
        const double bb = hd[48 + k];
        bool finite = std::isfinite(bb);
        for(int i = 0; i < k; ++i)
            finite = finite && std::isfinite(alpha[i]);
        if(finite && bb > 0)
        {
            for(int i = 0; i < k; ++i)
                cs.a[i] = alpha[i];
            k_ws_lincomb<<<ws_grid(n), WS_BLOCK, 0, st>>>(n, k, cs, x0);
            B2S_CHECK_LAUNCH();
            // FP64 residual of the candidate start, r = b - A x0
            double* Ax = W.Ac.data();
            double* y  = W.Ac.data() + (size_t)n;
            spmv_f64(s, A, x0, Ax, nullptr);
            k_ws_residual_comb<<<ws_grid(n), WS_BLOCK, 0, st>>>(n, 1, b, Ax, Ax, Ax, Ax, 1.0, 0.0, 0.0, 0.0, y);
            B2S_CHECK_LAUNCH();
            out.n_candidates = k;
            for(int i = 0; i < k; ++i)
                out.coeff[i] = alpha[i];
            // the judge is the PCG's own residual measure, r^T P r (the
            // quantity the reference's stop rule |r.z| <= tol |r0.z0| tracks):
            // accept the start when it is below b^T P b of the zero start
            double*       zr = W.Ac.data() + 2 * (size_t)n;
            const double* zb = W.fields.data() + 3 * (size_t)n;  // P b of the features
            precond_launch(s, y, zr);
            if(mode != B2S_WS_MODE_LEARNED)
            {
                precond_launch(s, b, W.Ac.data() + 3 * (size_t)n);
                zb = W.Ac.data() + 3 * (size_t)n;
            }
            DotPairs dc{};
            dc.a[0] = y;
            dc.b[0] = y;
            dc.a[1] = y;
            dc.b[1] = zr;
            dc.a[2] = b;
            dc.b[2] = zb;
            launch_dots(s, n, dc, 3, W.dots.data() + 60);
            double h3[3];
            B2S_CUDA(cudaMemcpyAsync(h3, W.dots.data() + 60, sizeof(h3), cudaMemcpyDeviceToHost, st));
            B2S_CUDA(cudaStreamSynchronize(st));
            const double rr = h3[0], rz = h3[1], bz = h3[2];
            out.rel_res_tried = std::sqrt(rr / bb);
            out.rz_ratio    = bz > 0 ? rz / bz : INFINITY;
            if(std::isfinite(rr) && std::isfinite(rz) && bz > 0 && rz < bz)
            {
                have         = true;
                out.mode     = mode;
                out.rel_res0 = out.rel_res_tried;
            }
        }
    }
    if(!have)
        B2S_CUDA(cudaMemsetAsync(x0, 0, sizeof(double) * n, st));
    B2S_CUDA(cudaEventRecord(W.ev1, st));
    B2S_CUDA(cudaEventSynchronize(W.ev1));
    float ms = 0.f;
    B2S_CUDA(cudaEventElapsedTime(&ms, W.ev0, W.ev1));
    out.predict_ms = ms;
    check_device_errors(s);
    if(info)
        *info = out;
}
}  // namespace b2s
