// Inversion of the MAS cluster matrices.
//
// What is computed is libuipc's (set_preconditioner ->
// invert_cluster_matrices, src/backends/cuda/finite_element/
// mas_preconditioner_engine.cu:1077-1182, 2281-2458): for every 16-node
// cluster the inverse of its 48x48 Galerkin matrix, no pivoting, a zero
// diagonal entry replaced by 1 (padding slots become identity rows), the
// inverse stored as the 136 upper 3x3 blocks in FP32.
//
// How it is computed here is this library's own: a blocked LDL^T
// factorisation followed by the inverse L^-T D^-1 L^-1, one warp per
// cluster with the whole matrix in shared memory, organised around the
// 3 x 3 grid of 16x16 tiles of the 48x48 matrix:
//   1. per panel P: unblocked LDL^T of the diagonal tile (16 lanes, one row
//      each, column broadcasts by shuffles), the panel below it solved row by
//      row (one lane per row), and the trailing tiles updated by 16x16x16
//      products in which every lane owns a 2x4 register tile;
//   2. Y = L^-1 by tiles: triangular inverses of the diagonal tiles, then the
//      off-diagonal tiles by 16x16 products;
//   3. A^-1 = Y^T D^-1 Y, its six upper tiles by 16x16 products;
//   4. the upper 3x3 blocks written out with coalesced stores.
// About n^3 multiply-adds per cluster as register-tiled products: the
// shared-memory traffic per multiply-add is a fraction of a broadcast load.
//
// Stiff clusters. Eliminating a cluster that holds a very stiff contact
// coupling cancels most of a pivot's digits: the pivot that remains is a
// small difference of large entries. Each FP32 factorisation records its
// smallest pivot ratio d_k / a_kk (a_kk the diagonal entry before
// elimination); below 2^-10 (more than 10 of FP32's 24 bits cancelled), or a
// pivot that is not positive, marks the cluster stiff. Stiff clusters are
// factorised and inverted again in FP64 (the same code in double) and stored
// in FP32; the mixed-precision apply reads their FP32 inverse instead of the
// BF16 tiles. A pivot that is not positive even in FP64 (an indefinite
// cluster) is replaced by the diagonal entry it started from.
#include "b2s_internal.cuh"
#include "b2s_tma.cuh"

#include <algorithm>

namespace b2s
{
int* device_error_flag(b2s_solver* s);

namespace
{
constexpr int    NI                = BANK * 3;  // 48 rows per cluster
constexpr double STIFF_PIVOT_RATIO = 1.0 / 1024.0;

// node pair (r, c), r <= c, of each of the 136 upper blocks in storage order
struct SymPairs
{
    unsigned char r[SYM], c[SYM];
};
constexpr SymPairs make_sym_pairs()
{
    SymPairs t{};
    int      k = 0;
    for(int a = 0; a < BANK; ++a)
        for(int b = a; b < BANK; ++b)
        {
            t.r[k] = (unsigned char)a;
            t.c[k] = (unsigned char)b;
            ++k;
        }
    return t;
}
__constant__ SymPairs c_sym_pairs = make_sym_pairs();

// shared-memory geometry per type: row stride of the 48x48 matrix and of the
// temporary tile (16-byte aligned rows, conflict-free 2x4 tile accesses),
// warps per CTA
template <typename T>
struct InvGeom;
template <>
struct InvGeom<float>
{
    static constexpr int LD = 52, TLD = 20, WARPS = 2;
};
template <>
struct InvGeom<double>
{
    static constexpr int LD = 50, TLD = 18, WARPS = 1;
};

template <typename T>
struct __align__(16) InvWarpSmem
{
    double stage[SYM * 9];     // the next cluster's FP64 Galerkin blocks (bulk copy)
    T S[NI * InvGeom<T>::LD];  // the cluster matrix, full symmetric storage
    T Tt[16 * InvGeom<T>::TLD];  // one temporary 16x16 tile
    T dinv[NI];                  // 1 / d_k of the factorisation
    T d0[NI];                    // diagonal before elimination
};

__device__ __forceinline__ float  fma_(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_(double a, double b, double c) { return __fma_rn(a, b, c); }

// 2x4 register tile of a 16x16 tile owned by `lane`: rows i0, i0 + 1, columns j0 .. j0 + 3
struct TileOwn
{
    int i0, j0;
    __device__ explicit TileOwn(int lane)
        : i0(2 * (lane >> 2))
        , j0(4 * (lane & 3))
    {
    }
};

template <typename T>
__device__ __forceinline__ void acc_zero(T acc[2][4])
{
#pragma unroll
    for(int a = 0; a < 2; ++a)
#pragma unroll
        for(int b = 0; b < 4; ++b)
            acc[a][b] = (T)0;
}

// acc += sign A B over k = 0..15, A and B 16x16 tiles in shared memory
// (row-major, leading dimensions lda / ldb). TA: read A transposed
// (acc += A^T B). With `dk`, row k of the product is scaled by dk[k]
// (A^T diag(dk) B).
template <typename T, bool TA>
__device__ __forceinline__ void tile_madd(T acc[2][4], const T* A, int lda, const T* B, int ldb, const T* dk,
                                          const TileOwn& o, T sign)
{
#pragma unroll 4
    for(int k = 0; k < 16; ++k)
    {
        T a0, a1;
        if constexpr(TA)
        {
            a0 = A[k * lda + o.i0];
            a1 = A[k * lda + o.i0 + 1];
        }
        else
        {
            a0 = A[o.i0 * lda + k];
            a1 = A[(o.i0 + 1) * lda + k];
        }
        const T sk = dk ? sign * dk[k] : sign;
        a0 *= sk;
        a1 *= sk;
        const T* b = B + k * ldb + o.j0;
        T        bv[4];
        if constexpr(sizeof(T) == 4)
        {
            const float4 q = *reinterpret_cast<const float4*>(b);
            bv[0] = q.x, bv[1] = q.y, bv[2] = q.z, bv[3] = q.w;
        }
        else
        {
            const double2 q0 = *reinterpret_cast<const double2*>(b);
            const double2 q1 = *reinterpret_cast<const double2*>(b + 2);
            bv[0] = q0.x, bv[1] = q0.y, bv[2] = q1.x, bv[3] = q1.y;
        }
#pragma unroll
        for(int c = 0; c < 4; ++c)
        {
            acc[0][c] = fma_(a0, bv[c], acc[0][c]);
            acc[1][c] = fma_(a1, bv[c], acc[1][c]);
        }
    }
}

template <typename T>
__device__ __forceinline__ void tile_store(const T acc[2][4], T* C, int ldc, T sign, const TileOwn& o)
{
#pragma unroll
    for(int a = 0; a < 2; ++a)
#pragma unroll
        for(int b = 0; b < 4; ++b)
            C[(o.i0 + a) * ldc + o.j0 + b] = sign * acc[a][b];
}

template <typename T>
__device__ __forceinline__ void tile_load(T acc[2][4], const T* C, int ldc, const TileOwn& o)
{
#pragma unroll
    for(int a = 0; a < 2; ++a)
#pragma unroll
        for(int b = 0; b < 4; ++b)
            acc[a][b] = C[(o.i0 + a) * ldc + o.j0 + b];
}

__device__ __forceinline__ bool pivot_ok(double d, double d0) { return d > STIFF_PIVOT_RATIO * d0; }

// Unblocked LDL^T of a 16x16 diagonal tile, lanes 0..15 (lane i holds row i
// in registers): step k broadcasts the pivot and the raw column k (a_jk,
// shuffles that do not wait for the pivot's reciprocal), then
// a_ij -= (a_ik / d_k) a_jk. The strict lower part becomes L, the diagonal
// D; dinv[i] = 1 / d_i. Returns true when a pivot ratio d_k / d0_k falls
// below STIFF_PIVOT_RATIO (or d_k is not positive).
template <typename T>
__device__ __forceinline__ bool factor_diag_tile(T* rowp, const T* d0, T* dinv, int lane)
{
    T    a[16];
    T    r_own = (T)1;  // 1 / this lane's pivot
    bool stiff = false;
#pragma unroll
    for(int j = 0; j < 16; ++j)
        a[j] = rowp[j];
#pragma unroll
    for(int k = 0; k < 16; ++k)
    {
        T col[16];
#pragma unroll
        for(int j = 0; j < 16; ++j)
            if(j >= k)
                col[j] = __shfl_sync(0x0000ffffu, a[k], j, 16);
        T       d   = col[k];
        const T dk0 = d0[k];
        if(!pivot_ok((double)d, (double)dk0))
            stiff = true;
        if(!(d > (T)0) || !isfinite((double)d))
            d = dk0;
        const T rd = (T)1 / d;
        const T l  = a[k] * rd;
        if(lane > k)
        {
#pragma unroll
            for(int j = 0; j < 16; ++j)
                if(j > k)
                    a[j] = fma_(-l, col[j], a[j]);
            a[k] = l;
        }
        else if(lane == k)
        {
            a[k]  = d;
            r_own = rd;
        }
    }
#pragma unroll
    for(int j = 0; j < 16; ++j)
        rowp[j] = a[j];
    dinv[lane] = r_own;
    return stiff;
}

// The tile products of steps 2 and 3 as data: dst (+/-)= sum of up to three
// A B terms (A read transposed and scaled by D^-1 in step 3). Tile ids: 3 I
// + J, 9 = the temporary tile.
struct TileTerm
{
    signed char a, b, k;  // A tile, B tile, D^-1 block (-1: none)
};
struct TileOp
{
    signed char dst, sign, n;
    TileTerm    t[3];
};
// Y = L^-1 below the diagonal: Y_10 = -Y_11 (L_10 Y_00),
// Y_20 = -Y_22 (L_20 Y_00 + L_21 Y_10), Y_21 = -Y_22 (L_21 Y_11)
__constant__ TileOp c_yops[6] = {
    {9, 1, 1, {{3, 0, -1}}},             {3, -1, 1, {{4, 9, -1}}},
    {9, 1, 2, {{6, 0, -1}, {7, 3, -1}}}, {6, -1, 1, {{8, 9, -1}}},
    {9, 1, 1, {{7, 4, -1}}},             {7, -1, 1, {{8, 9, -1}}},
};
// X = Y^T D^-1 Y, X_IJ = sum_{K >= max(I,J)} Y_KI^T D_K^-1 Y_KJ into the upper
// tiles (free once their W operands are spent); a diagonal tile is written
// after every product that reads it
__constant__ TileOp c_xops[6] = {
    {5, 1, 1, {{7, 8, 2}}},
    {2, 1, 1, {{6, 8, 2}}},
    {1, 1, 2, {{3, 4, 1}, {6, 7, 2}}},
    {4, 1, 2, {{4, 4, 1}, {7, 7, 2}}},
    {0, 1, 3, {{0, 0, 0}, {3, 3, 1}, {6, 6, 2}}},
    {8, 1, 1, {{8, 8, 2}}},
};

// Factorise and invert one cluster (the whole warp). Returns true when the
// cluster is stiff (a pivot ratio below STIFF_PIVOT_RATIO, or a pivot that
// is not positive).
template <typename T, typename AfterScatter>
__device__ bool invert_cluster(float* __restrict__ out, InvWarpSmem<T>& sm, const SymPairs& pairs, int lane,
                               AfterScatter after_scatter)
{
    constexpr int LD = InvGeom<T>::LD, TLD = InvGeom<T>::TLD;
    T*            S  = sm.S;
    auto          tile = [&](int I, int J) -> T* { return S + (16 * I) * LD + 16 * J; };
    const TileOwn own(lane);

    // 0. scatter the staged blocks: block (a, b), a <= b, column-major
    // component q = pb * 3 + pa is entry (3a + pa, 3b + pb); mirrored below
    // the diagonal for a < b
    const double* H = sm.stage;
    for(int e = lane; e < SYM * 9; e += 32)
    {
        const int    blk = e / 9, q = e - 9 * blk;
        const int    a = pairs.r[blk], b = pairs.c[blk];
        const int    row = 3 * a + q % 3, col = 3 * b + q / 3;
        const double v = H[e];
        S[row * LD + col] = (T)v;
        if(a != b)
            S[col * LD + row] = (T)v;
    }
    __syncwarp();
    after_scatter();  // the stage is free: the next cluster's copy may start
    for(int i = lane; i < NI; i += 32)
    {
        T d = S[i * LD + i];
        if(d == (T)0)
            d = (T)1;
        S[i * LD + i] = d;
        sm.d0[i]      = d;
    }
    __syncwarp();

    bool stiff = false;
    // 1. blocked LDL^T
#pragma unroll 1
    for(int P = 0; P < 3; ++P)
    {
        // 1a. diagonal tile
        if(lane < 16)
            stiff |= factor_diag_tile<T>(tile(P, P) + lane * LD, sm.d0 + 16 * P, sm.dinv + 16 * P, lane);
        __syncwarp();
        if(P == 2)
            break;
        // 1b. panel below the diagonal tile: one lane per row R, x = l D L_PP^T
        // solved forward column by column (w_k = l_k d_k), l stored in the
        // lower tile and w in the mirrored upper tile (the operand of the
        // trailing update)
        const int n_rows = 16 * (2 - P);
        if(lane < n_rows)
        {
            const int R    = 16 * (P + 1) + lane;
            T*        rowp = S + R * LD + 16 * P;
            const T*  Lpp  = tile(P, P);
            T         w[16];
#pragma unroll
            for(int k = 0; k < 16; ++k)
                w[k] = rowp[k];
#pragma unroll
            for(int m = 0; m < 16; ++m)
#pragma unroll
                for(int k = m + 1; k < 16; ++k)
                    w[k] = fma_(-w[m], Lpp[k * LD + m], w[k]);
#pragma unroll
            for(int k = 0; k < 16; ++k)
            {
                rowp[k]                  = w[k] * sm.dinv[16 * P + k];
                S[(16 * P + k) * LD + R] = w[k];
            }
        }
        __syncwarp();
        // 1c. trailing tiles (I, J), P < J <= I: A_IJ -= L_IP W_JP^T
#pragma unroll 1
        for(int J = P + 1; J < 3; ++J)
#pragma unroll 1
            for(int I = J; I < 3; ++I)
            {
                T acc[2][4];
                tile_load(acc, tile(I, J), LD, own);
                tile_madd<T, false>(acc, tile(I, P), LD, tile(P, J), LD, nullptr, own, (T)-1);
                tile_store(acc, tile(I, J), LD, (T)1, own);
            }
        __syncwarp();
    }
    stiff = __any_sync(0xffffffffu, stiff);

    // 2a. Y_PP = L_PP^-1 (unit lower): lane c of a half-warp solves column c
    // forward, column by column; tiles 0 and 1 side by side, then tile 2
#pragma unroll 1
    for(int round = 0; round < 2; ++round)
    {
        const int  P   = round == 0 ? (lane >> 4) : 2;
        const int  c   = lane & 15;
        const bool act = round == 0 || lane < 16;
        T          y[16];
#pragma unroll
        for(int i = 0; i < 16; ++i)
            y[i] = i == c ? (T)1 : (T)0;
        if(act)
        {
            const T* L = tile(P, P);
#pragma unroll
            for(int m = 0; m < 15; ++m)
#pragma unroll
                for(int i = m + 1; i < 16; ++i)
                    y[i] = fma_(-L[i * LD + m], y[m], y[i]);
        }
        __syncwarp();
        if(act)
        {
            T* Y = tile(P, P);
#pragma unroll
            for(int i = 0; i < 16; ++i)
                Y[i * LD + c] = y[i];
        }
        __syncwarp();
    }
    // 2b / 3. the off-diagonal tiles of Y = L^-1, then X = Y^T D^-1 Y
    auto tptr = [&](int id) -> T* { return id == 9 ? sm.Tt : tile(id / 3, id % 3); };
    auto tld  = [&](int id) -> int { return id == 9 ? TLD : LD; };
#pragma unroll 1
    for(int o = 0; o < 12; ++o)
    {
        const bool    xop = o >= 6;
        const TileOp& op  = xop ? c_xops[o - 6] : c_yops[o];
        T             acc[2][4];
        acc_zero(acc);
#pragma unroll 1
        for(int t = 0; t < op.n; ++t)
        {
            const TileTerm tt = op.t[t];
            if(xop)
                tile_madd<T, true>(acc, tptr(tt.a), LD, tptr(tt.b), LD, sm.dinv + 16 * tt.k, own, (T)1);
            else
                tile_madd<T, false>(acc, tptr(tt.a), tld(tt.a), tptr(tt.b), tld(tt.b), nullptr, own, (T)1);
        }
        __syncwarp();
        tile_store(acc, tptr(op.dst), tld(op.dst), (T)op.sign, own);
        __syncwarp();
    }
    // 4. upper 3x3 blocks out (entries read from the upper triangle of X)
    for(int e = lane; e < SYM * 9; e += 32)
    {
        const int blk = e / 9, q = e - 9 * blk;
        const int a = pairs.r[blk], b = pairs.c[blk];
        int       row = 3 * a + q % 3, col = 3 * b + q / 3;
        if(row > col)
        {
            const int t = row;
            row         = col;
            col         = t;
        }
        out[e] = (float)S[row * LD + col];
    }
    return stiff;
}

// One warp per cluster. list == nullptr: every cluster (grid-stride), the
// stiffness flag of each written and, with `queue`, the stiff ones appended
// to stiff_list for the FP64 pass. Otherwise the clusters list[0 ..
// *list_count) (the FP64 pass over the stiff clusters). Each warp brings its
// next cluster's Galerkin blocks (9,792 B) into shared memory by a bulk copy
// (TMA) while it factorises the current one; a copy wait that runs out sets
// DERR_TMA_TIMEOUT and the warp stops.
template <typename T>
__global__ void __launch_bounds__(InvGeom<T>::WARPS * 32)
    k_cluster_inverse(int clusters, const double* __restrict__ hess, float* __restrict__ inv,
                      const int32_t* __restrict__ list, const int32_t* __restrict__ list_count,
                      uint8_t* __restrict__ stiff, int32_t* __restrict__ stiff_list, int32_t* __restrict__ stiff_count,
                      int queue, int* err)
{
    constexpr uint32_t BYTES = SYM * 9 * sizeof(double);  // 9,792, a multiple of 16
    __shared__ InvWarpSmem<T> sm[InvGeom<T>::WARPS];
    __shared__ SymPairs       pairs;
    __shared__ uint64_t       bar[InvGeom<T>::WARPS];
    for(int i = threadIdx.x; i < SYM; i += blockDim.x)
    {
        pairs.r[i] = c_sym_pairs.r[i];
        pairs.c[i] = c_sym_pairs.c[i];
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if(lane == 0)
    {
        mbar_init(&bar[w], 1);
        mbar_fence_init();
    }
    __syncthreads();
    const int gw = blockIdx.x * InvGeom<T>::WARPS + w;
    const int W  = gridDim.x * InvGeom<T>::WARPS;
    const int n  = list ? *list_count : clusters;
    auto cluster_at = [&](int i) { return list ? list[i] : i; };
    if(gw < n && lane == 0)
    {
        mbar_arrive_expect_tx(&bar[w], BYTES);
        bulk_copy_g2s(sm[w].stage, hess + (size_t)cluster_at(gw) * SYM * 9, BYTES, &bar[w]);
    }
    uint32_t phase = 0;
    for(int i = gw; i < n; i += W)
    {
        const int  cl = cluster_at(i);
        const bool ok = mbar_wait(&bar[w], phase, err, DERR_TMA_TIMEOUT);
        phase ^= 1u;
        if(!__all_sync(0xffffffffu, ok))
        {
            if(lane == 0)  // drain the copy that may still be in flight (bounded)
                mbar_wait(&bar[w], phase ^ 1u, nullptr, 0);
            __syncwarp();
            return;
        }
        // invert_cluster reads the staged blocks first; the next copy goes
        // out once they are in S (ordered by its first __syncwarp)
        const bool st = invert_cluster<T>(inv + (size_t)cl * SYM * 9, sm[w], pairs, lane, [&]
                                          {
                                              if(lane == 0 && i + W < n)
                                              {
                                                  fence_proxy_async_smem();
                                                  mbar_arrive_expect_tx(&bar[w], BYTES);
                                                  bulk_copy_g2s(sm[w].stage,
                                                                hess + (size_t)cluster_at(i + W) * SYM * 9, BYTES,
                                                                &bar[w]);
                                              }
                                          });
        if(lane == 0 && !list)
        {
            stiff[cl] = st ? 1 : 0;
            if(st && queue)
                stiff_list[atomicAdd(stiff_count, 1)] = cl;
        }
        __syncwarp();
    }
}

template <typename T>
int inverse_grid(int clusters)
{
    int occ = 0;
    if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_cluster_inverse<T>, InvGeom<T>::WARPS * 32, 0) !=
           cudaSuccess ||
       occ < 1)
        occ = 1;
    const int want = (clusters + InvGeom<T>::WARPS - 1) / InvGeom<T>::WARPS;
    const int cap  = NUM_SMS_HINT * occ;
    return std::max(1, std::min(want, cap));
}
}  // namespace

// Inverses of all clusters of the current Galerkin matrices (M.hess) into
// M.inv, stiffness flags into M.stiff. mode: B2S_INVERT_F32 = FP32,
// stiff clusters again in FP64; B2S_INVERT_F64 = FP64 for every cluster;
// B2S_INVERT_F32_ONLY = FP32 for every cluster (stiff ones flagged, not redone).
void mas_invert_clusters(b2s_solver* s, int mode)
{
    MasState&    M   = s->mas;
    cudaStream_t st  = s->stream;
    const int    C   = M.clusters;
    int*         err = device_error_flag(s);
    M.stiff.resize(std::max(C, 1));
    M.stiff_list.resize(std::max(C, 1));
    M.stiff_count.resize(1);
    B2S_CUDA(cudaMemsetAsync(M.stiff_count.data(), 0, sizeof(int32_t), st));
    if(C <= 0)
        return;
    if(mode == B2S_INVERT_F64)
    {
        k_cluster_inverse<double><<<inverse_grid<double>(C), InvGeom<double>::WARPS * 32, 0, st>>>(
            C, M.hess.data(), M.inv.data(), nullptr, nullptr, M.stiff.data(), M.stiff_list.data(),
            M.stiff_count.data(), 1, err);
        B2S_CHECK_LAUNCH();
        return;
    }
    k_cluster_inverse<float><<<inverse_grid<float>(C), InvGeom<float>::WARPS * 32, 0, st>>>(
        C, M.hess.data(), M.inv.data(), nullptr, nullptr, M.stiff.data(), M.stiff_list.data(), M.stiff_count.data(),
        1, err);
    B2S_CHECK_LAUNCH();
    if(mode == B2S_INVERT_F32_ONLY)
        return;
    // the FP64 pass over the stiff clusters: its length is on the device, so
    // a small fixed grid walks the list (it returns at once when it is empty)
    const int grid = std::min(inverse_grid<double>(C), 2 * NUM_SMS_HINT);
    k_cluster_inverse<double><<<grid, InvGeom<double>::WARPS * 32, 0, st>>>(
        C, M.hess.data(), M.inv.data(), M.stiff_list.data(), M.stiff_count.data(), nullptr, nullptr, nullptr, 0, err);
    B2S_CHECK_LAUNCH();
}
}  // namespace b2s
