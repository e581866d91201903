// MAS (multi-level additive Schwarz) preconditioner: hierarchy, Galerkin
// cluster matrices, cluster inversion and apply.
//
// Algorithm of libuipc's MASPreconditionerEngine (StiffGIPC MAS, 16-node
// banks), src/backends/cuda/finite_element/mas_preconditioner_engine.cu:
//  * hierarchy (:57-460, host :1958-2280): partition slots form 16-lane banks;
//    connected components of the mesh graph inside a bank become one node of
//    the next level, numbered by bank then by lowest lane; coarser levels
//    repeat on the remaining cross-bank edges; levels capped at 6.
//  * Galerkin matrices (:530-953): the 48x48 matrix of every bank at every
//    level is R_l A R_l^T restricted to the bank, R_l summing the fine
//    vertices of each level-l node.
//  * inversion (:1077-1175): the inverse of every cluster matrix, no pivoting,
//    zero diagonal -> 1 (b2s_mas_invert.cu).
//  * apply (:1604-1955, :2887-2960): z = sum_l P_l^T A_l^{-1} P_l r with
//    summation restriction and injection prolongation, FP32 inside.
//
// Design here: the hierarchy is built by bank-parallel kernels; the coarse
// Galerkin matrices are built level by level as sparse matrices with the same
// deterministic triplet assembly as the global matrix (A_{l+1} from A_l), so
// no FP64 atomics pile onto the few clusters of the top levels; the apply
// runs one warp per bank and level with the restriction sums of the next
// level computed in the same pass (no atomics, bit-reproducible).
#include "b2s_internal.cuh"
#include "b2s_reduce.cuh"
#include "b2s_tma.cuh"

#include <cuda_bf16.h>

#include <algorithm>

namespace b2s
{
int* device_error_flag(b2s_solver* s);
void mas_invert_clusters(b2s_solver* s, int mode);

namespace
{
inline int bank_align(int n) { return (n + BANK - 1) / BANK * BANK; }
__host__ __device__ __forceinline__ int sym_index(int row, int col)
{
    return BANK * row - row * (row + 1) / 2 + col;
}

int compute_num_levels(int vert_num)
{
    int n_level = 1, sz = bank_align(vert_num);
    while(sz > BANK)
    {
        sz /= BANK;
        n_level++;
        sz = bank_align(sz);
    }
    n_level++;
    return std::min(n_level, MAX_LEVELS);
}

// ---------------------------------------------------------------------------
// hierarchy kernels
// ---------------------------------------------------------------------------

// level 0: direct in-bank adjacency mask of every partition slot; cross-bank
// neighbours stay in the (compacted) list, unpartitioned ones are dropped
__global__ void k_h_mask_l0(int N, const int32_t* p2r, const int32_t* r2p, const int32_t* nbr_start,
                            int32_t* nbr_num, int32_t* nbr_list, uint32_t* mask)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= N)
        return;
    const int v = p2r[p];
    if(v < 0)
    {
        mask[p] = 0;
        return;
    }
    uint32_t m = 1u << (p % BANK);
    const int s = nbr_start[v], n = nbr_num[v];
    int       keep = 0;
    for(int e = 0; e < n; ++e)
    {
        const int u  = nbr_list[s + e];
        const int pu = r2p[u];
        if(pu < 0)
            continue;
        if(pu / BANK == p / BANK)
            m |= 1u << (pu % BANK);
        else
            nbr_list[s + keep++] = u;
    }
    nbr_num[v] = keep;
    mask[p]    = m;
}

// level l >= 1: OR the in-bank adjacency of every level-l node from its fine
// vertices' remaining neighbours
__global__ void k_h_mask_lx(int N, int vn, const int32_t* p2r, const int32_t* cst_prev, const int32_t* nbr_start,
                            int32_t* nbr_num, int32_t* nbr_list, uint32_t* next_mask, int cnt)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= N)
        return;
    const int v = p2r[p];
    if(v < 0)
        return;
    const int c = cst_prev[v];
    if(c < 0 || c >= cnt)
        return;
    uint32_t  conn = 0;
    const int s = nbr_start[v], n = nbr_num[v];
    int       keep = 0;
    for(int e = 0; e < n; ++e)
    {
        const int u  = nbr_list[s + e];
        const int cu = cst_prev[u];
        if(cu < 0 || cu >= cnt)
        {
            nbr_list[s + keep++] = u;
            continue;
        }
        if(cu / BANK == c / BANK)
            conn |= 1u << (cu % BANK);
        else
            nbr_list[s + keep++] = u;
    }
    nbr_num[v] = keep;
    if(conn)
        atomicOr(&next_mask[c], conn);
}

// one thread per bank: components (transitive closure of the lane masks),
// numbered by lowest lane; writes the component count, each node's rank and
// each node's component mask
__global__ void k_h_components(int n_nodes, int n_banks, const uint32_t* mask, const int32_t* valid_p2r,
                               int level0, int32_t* comp_count, int32_t* rank, uint16_t* comp_mask)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if(b >= n_banks)
        return;
    uint32_t m[BANK];
    bool     valid[BANK];
    for(int l = 0; l < BANK; ++l)
    {
        const int node = b * BANK + l;
        valid[l]       = node < n_nodes && (!level0 || valid_p2r[node] >= 0);
        m[l]           = valid[l] ? (mask[node] | (1u << l)) : 0u;
    }
    uint32_t closure[BANK];
    uint32_t elected = 0;
    for(int l = 0; l < BANK; ++l)
    {
        if(!valid[l])
        {
            closure[l] = 0;
            continue;
        }
        uint32_t c = m[l], visited = 1u << l;
        for(int guard = 0; guard < BANK; ++guard)
        {
            const uint32_t todo = visited ^ c;
            if(!todo)
                break;
            const int nv = __ffs(todo) - 1;
            visited |= 1u << nv;
            c |= m[nv];
        }
        closure[l] = c;
        if((c & ((1u << l) - 1u)) == 0)
            elected |= 1u << l;
    }
    for(int l = 0; l < BANK; ++l)
    {
        const int node = b * BANK + l;
        if(node >= n_nodes)
            break;
        if(valid[l])
        {
            const int el = __ffs(closure[l]) - 1;
            rank[node]      = __popc(elected & ((1u << el) - 1u));
            comp_mask[node] = (uint16_t)closure[l];
        }
        else
        {
            rank[node]      = -1;
            comp_mask[node] = 0;
        }
    }
    comp_count[b] = __popc(elected);
}

// next-level local id of every node (bank offset + component rank)
__global__ void k_h_assign(int n_nodes, const int32_t* rank, const int32_t* bank_offset, int32_t* new_local)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if(c >= n_nodes)
        return;
    const int rk = rank[c];
    new_local[c] = rk >= 0 ? bank_offset[c / BANK] + rk : -1;
}

// per vertex: local id at level 1 from its partition slot
__global__ void k_h_cst_l1(int vn, const int32_t* r2p, const int32_t* new_local0, int32_t* cst0)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if(v >= vn)
        return;
    const int p = r2p[v];
    cst0[v]     = p >= 0 ? new_local0[p] : -1;
}

__global__ void k_h_cst_next(int vn, const int32_t* cst_prev, const int32_t* new_local, int cnt, int32_t* cst_next)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if(v >= vn)
        return;
    const int c = cst_prev[v];
    cst_next[v] = (c >= 0 && c < cnt) ? new_local[c] : -1;
}

__global__ void k_h_ctable(int vn, int L, const int32_t* cst, const int32_t* level_begin_dev, int32_t* ctable)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if(v >= vn)
        return;
    for(int l = 1; l < L; ++l)
    {
        const int c = cst[(size_t)(l - 1) * vn + v];
        ctable[(size_t)v * (L - 1) + (l - 1)] = c >= 0 ? level_begin_dev[l] + c : -1;
    }
}

__global__ void k_h_node1(int vn, int L, const int32_t* ctable, int32_t* node1)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if(v < vn)
        node1[v] = ctable[(size_t)v * (L - 1)];
}

// ---------------------------------------------------------------------------
// Galerkin matrices
// ---------------------------------------------------------------------------

// level 0: blocks of A inside one partition bank, stored oriented by slot
__global__ void k_g_level0(int64_t U, const int32_t* rows, const int32_t* cols, const double* vals, int64_t S, int off, int vn,
                           const int32_t* r2p, double* hess)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(k >= U)
        return;
    const int i = rows[k] - off, j = cols[k] - off;
    if(i < 0 || i >= vn || j < 0 || j >= vn)
        return;
    const int pi = r2p[i], pj = r2p[j];
    if(pi < 0 || pj < 0 || pi / BANK != pj / BANK)
        return;
    const bool swap = pj < pi;
    const int  a = swap ? pj : pi, b = swap ? pi : pj;
    double*    dst = hess + ((size_t)(a / BANK) * SYM + sym_index(a % BANK, b % BANK)) * 9;
#pragma unroll
    for(int p = 0; p < 3; ++p)
#pragma unroll
        for(int q = 0; q < 3; ++q)
        {
            // dst(p,q) column-major; source B(p,q) = vals[(q*3+p)*S + k]
            const double v = swap ? vals[(int64_t)(p * 3 + q) * S + k] : vals[(int64_t)(q * 3 + p) * S + k];
            dst[q * 3 + p] = v;
        }
}

// restriction of a block-upper matrix to the next level as raw triplets:
// (a, b, B) -> (P a, P b) with B, B^T or (a != b) B + B^T when both map to
// one node. Entries that leave the MAS range are written with row -1.
__global__ void k_g_restrict(int64_t U, const int32_t* rows, const int32_t* cols, const double* vals, int64_t S, int off,
                             int n_in, const int32_t* map, int32_t* out_rows, int32_t* out_cols, double* out_vals)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(k >= U)
        return;
    const int a = rows[k] - off, b = cols[k] - off;
    int       ca = -1, cb = -1;
    if(a >= 0 && a < n_in && b >= 0 && b < n_in)
    {
        ca = map[a];
        cb = map[b];
    }
    if(ca < 0 || cb < 0)
    {
        out_rows[k] = -1;
        out_cols[k] = -1;
#pragma unroll
        for(int q = 0; q < 9; ++q)
            out_vals[k * 9 + q] = 0.0;
        return;
    }
    double B[9];
#pragma unroll
    for(int q = 0; q < 9; ++q)
        B[q] = vals[(int64_t)q * S + k];
    double o[9];
    if(ca < cb)
    {
#pragma unroll
        for(int q = 0; q < 9; ++q)
            o[q] = B[q];
    }
    else if(ca > cb)
    {
#pragma unroll
        for(int p = 0; p < 3; ++p)
#pragma unroll
            for(int q = 0; q < 3; ++q)
                o[q * 3 + p] = B[p * 3 + q];
    }
    else if(a == b)
    {
#pragma unroll
        for(int q = 0; q < 9; ++q)
            o[q] = B[q];
    }
    else
    {
#pragma unroll
        for(int p = 0; p < 3; ++p)
#pragma unroll
            for(int q = 0; q < 3; ++q)
                o[q * 3 + p] = B[q * 3 + p] + B[p * 3 + q];
    }
    out_rows[k] = ca < cb ? ca : cb;
    out_cols[k] = ca < cb ? cb : ca;
#pragma unroll
    for(int q = 0; q < 9; ++q)
        out_vals[k * 9 + q] = o[q];
}

// level l >= 1: in-bank blocks of the level-l Galerkin matrix into clusters
__global__ void k_g_extract(int64_t U, const int32_t* rows, const int32_t* cols, const double* vals, int64_t S,
                            int level_begin, double* hess)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(k >= U)
        return;
    const int a = rows[k], b = cols[k];
    if(a / BANK != b / BANK)
        return;
    const int ga = level_begin + a, gb = level_begin + b;
    double*   dst = hess + ((size_t)(ga / BANK) * SYM + sym_index(ga % BANK, gb % BANK)) * 9;
#pragma unroll
    for(int q = 0; q < 9; ++q)
        dst[q] = vals[(int64_t)q * S + k];
}

// ---------------------------------------------------------------------------
// apply: one warp per bank, persistent over banks. The bank's inverse is
// brought into shared memory by bulk asynchronous copies (TMA), NST deep per
// warp, so later banks' copies are in flight while this one computes. The
// residual of the next bank (and, at level 0, the part_to_real index of the
// bank after it) is loaded into registers one bank ahead, so the dependent
// part_to_real -> r gather never stalls the product.
//
// FP32 inverses (4,896 B: the 136 upper 3x3 blocks, column-major) are applied
// on the CUDA cores: lanes 0-15 own the bank's nodes and the 48x48 product is
// split over the two half-warps (columns 0-7 / 8-15).
//
// BF16 inverses (mixed precision) are applied on the tensor cores. Per cluster:
// the FP32 factor D = diag(M)^1/2 (48 floats, 192 B), then the six upper 16x16
// tiles (I <= J) of the 48x48 matrix D^-1 M D^-1 in BF16 (6 x 512 B), 3,264 B
// in all. Tile rows are 32 B; the two 16-B halves of row R are swapped when
// bit 2 of R is set, so each 8-row ldmatrix phase touches all 32 banks once.
// z = D (M_s (D r)) by mma.m16n8k16 (BF16 operands, FP32 accumulation): A is
// tile (I, J), for J < I the stored tile (J, I) loaded transposed; B column 0
// is BF16(D r) and column 1 its BF16 rounding remainder, so the FP32 residual
// enters with ~16 significant bits and the stored inverse is the only 8-bit
// rounding. (A 48x48 matrix times one vector is an HBM-bound GEMV; the tensor
// cores are used to cut the instruction count per byte, not for FLOPs.)
// ---------------------------------------------------------------------------
constexpr int APPLY_WARPS = 4;
constexpr uint32_t INV_BYTES = SYM * 9 * sizeof(float);  // 4896, a multiple of 16
constexpr uint32_t INV16_SCALE_BYTES = BANK * 3 * sizeof(float);                    // 192
constexpr uint32_t INV16_TILE_BYTES  = 16 * 16 * 2;                                 // 512
constexpr uint32_t INV16_BYTES       = INV16_SCALE_BYTES + 6 * INV16_TILE_BYTES;  // 3264
constexpr int APPLY_STAGES_F32  = 2;
constexpr int APPLY_STAGES_BF16 = 2;

// index of the upper tile (I, J), I <= J: (0,0) (0,1) (0,2) (1,1) (1,2) (2,2)
__host__ __device__ __forceinline__ int tile_id(int I, int J) { return I * 3 - I * (I + 1) / 2 + J; }
// byte offset of 16-B half `half` of row `row` inside a tile
__host__ __device__ __forceinline__ uint32_t tile_off(int row, int half)
{
    return (uint32_t)row * 32u + ((uint32_t)(half ^ ((row >> 2) & 1)) << 4);
}

__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t& a0, uint32_t& a1, uint32_t& a2, uint32_t& a3)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];"
                 : "=r"(a0), "=r"(a1), "=r"(a2), "=r"(a3)
                 : "r"(addr));
}
__device__ __forceinline__ void ldsm_x4_trans(uint32_t addr, uint32_t& a0, uint32_t& a1, uint32_t& a2, uint32_t& a3)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0, %1, %2, %3}, [%4];"
                 : "=r"(a0), "=r"(a1), "=r"(a2), "=r"(a3)
                 : "r"(addr));
}
// c += A (16x16, row) * B (16x8, col), BF16 in, FP32 accumulate
__device__ __forceinline__ void mma_bf16_16816(float& c0, float& c1, float& c2, float& c3, uint32_t a0, uint32_t a1,
                                               uint32_t a2, uint32_t a3, uint32_t b0, uint32_t b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};"
        : "+f"(c0), "+f"(c1), "+f"(c2), "+f"(c3)
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}
__device__ __forceinline__ uint32_t pack_bf16x2(__nv_bfloat16 lo, __nv_bfloat16 hi)
{
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// Zb[0..48) = D M_s D r for one cluster; r48: the bank's residual (node-major)
__device__ __forceinline__ void cluster_product_mma(const unsigned char* slot, const float* r48, int lane,
                                                    float* __restrict__ Zb)
{
    const float*   D     = reinterpret_cast<const float*>(slot);
    const uint32_t tiles = smem_addr(slot + INV16_SCALE_BYTES);
    const int      g = lane >> 2, t = lane & 3;
    uint32_t       b[3][2];
#pragma unroll
    for(int J = 0; J < 3; ++J)
    {
#pragma unroll
        for(int h = 0; h < 2; ++h)
        {
            const int           k  = J * 16 + 2 * t + 8 * h;
            const float         x0 = r48[k] * D[k], x1 = r48[k + 1] * D[k + 1];
            const __nv_bfloat16 h0 = __float2bfloat16_rn(x0), h1 = __float2bfloat16_rn(x1);
            uint32_t            v  = 0;
            if(g == 0)
                v = pack_bf16x2(h0, h1);
            else if(g == 1)
                v = pack_bf16x2(__float2bfloat16_rn(x0 - __bfloat162float(h0)),
                                __float2bfloat16_rn(x1 - __bfloat162float(h1)));
            b[J][h] = v;
        }
    }
    // row address this lane gives ldmatrix: matrix q = lane / 8 of the four
    // 8x8 quarters, row lane % 8 of it
    const int      q = lane >> 3, rr = lane & 7;
    const uint32_t offN = tile_off(rr + ((q & 1) << 3), q >> 1);
    const uint32_t offT = tile_off(rr + ((q >> 1) << 3), q & 1);
#pragma unroll
    for(int I = 0; I < 3; ++I)
    {
        float c0 = 0.f, c1 = 0.f, c2 = 0.f, c3 = 0.f;
#pragma unroll
        for(int J = 0; J < 3; ++J)
        {
            uint32_t a0, a1, a2, a3;
            if(J >= I)
                ldsm_x4(tiles + tile_id(I, J) * INV16_TILE_BYTES + offN, a0, a1, a2, a3);
            else
                ldsm_x4_trans(tiles + tile_id(J, I) * INV16_TILE_BYTES + offT, a0, a1, a2, a3);
            mma_bf16_16816(c0, c1, c2, c3, a0, a1, a2, a3, b[J][0], b[J][1]);
        }
        if(t == 0)
        {
            const int k0 = I * 16 + g, k1 = k0 + 8;
            Zb[k0] = (c0 + c1) * D[k0];
            Zb[k1] = (c2 + c3) * D[k1];
        }
    }
}

// pack the FP32 inverse M of every cluster as D (FP32) + the BF16 tiles of
// D^-1 M D^-1, D = diag(M)^1/2: the stored matrix has a unit diagonal, so BF16
// rounds every entry relative to O(1), and M = D (D^-1 M D^-1) D is recovered
// in the apply. Entry (a, b) comes from the stored upper 3x3 block of nodes
// (min, max) and is scaled as stored row times stored column.
// One CTA per cluster: the FP32 inverse staged in shared memory by 16-byte
// loads, then each thread writes 8 consecutive BF16 entries of one tile row
// (one 16-byte store): 6 tiles x 16 rows x 2 halves = 192 threads.
constexpr int PACK_THREADS = 192;
__global__ void __launch_bounds__(PACK_THREADS) k_pack_inverse_bf16(int clusters, const float* __restrict__ inv,
                                                                    unsigned char* __restrict__ out)
{
    const int c = blockIdx.x;
    if(c >= clusters)
        return;
    __shared__ float4 Ms4[SYM * 9 / 4];
    __shared__ float  S[BANK * 3];  // 1 / D
    const float4*  src = reinterpret_cast<const float4*>(inv + (size_t)c * SYM * 9);
    unsigned char* o   = out + (size_t)c * INV16_BYTES;
    for(int i = threadIdx.x; i < SYM * 9 / 4; i += PACK_THREADS)
        Ms4[i] = src[i];
    __syncthreads();
    const float* M = reinterpret_cast<const float*>(Ms4);
    if(threadIdx.x < BANK * 3)
    {
        const int   nd = threadIdx.x / 3, a = threadIdx.x % 3;
        const float d  = M[sym_index(nd, nd) * 9 + a * 3 + a];
        const float Dv = d > 0.f ? sqrtf(d) : 1.0f;
        S[threadIdx.x] = 1.0f / Dv;
        reinterpret_cast<float*>(o)[threadIdx.x] = Dv;
    }
    __syncthreads();
    const int t = threadIdx.x >> 5, row = (threadIdx.x >> 1) & 15, half = threadIdx.x & 1;
    const int I = t < 3 ? 0 : (t < 5 ? 1 : 2);
    const int J = t - (I * 3 - I * (I + 1) / 2);
    const int a = I * 16 + row, na = a / 3, pa = a % 3;
    uint32_t  w[4];
#pragma unroll
    for(int k = 0; k < 8; k += 2)
    {
        float v2[2];
#pragma unroll
        for(int u = 0; u < 2; ++u)
        {
            const int b = J * 16 + half * 8 + k + u, nb = b / 3, pb = b % 3;
            v2[u] = na <= nb ? M[sym_index(na, nb) * 9 + pb * 3 + pa] * S[a] * S[b]
                             : M[sym_index(nb, na) * 9 + pa * 3 + pb] * S[b] * S[a];
        }
        const __nv_bfloat162 h = __floats2bfloat162_rn(v2[0], v2[1]);
        w[k >> 1]              = *reinterpret_cast<const uint32_t*>(&h);
    }
    *reinterpret_cast<uint4*>(o + INV16_SCALE_BYTES + t * INV16_TILE_BYTES + tile_off(row, half)) =
        make_uint4(w[0], w[1], w[2], w[3]);
}

__device__ __forceinline__ void cluster_product(const float* M, const float (*r)[3], int lane, float out[3])
{
    // lanes 0..15: row node `lane`, columns 0..7; lanes 16..31: row node lane-16, columns 8..15
    const int rn = lane & 15, c0 = (lane >> 4) * 8;
    float acc0 = 0.f, acc1 = 0.f, acc2 = 0.f;
#pragma unroll
    for(int cc = 0; cc < 8; ++cc)
    {
        const int cn = c0 + cc;
        const float x0 = r[cn][0], x1 = r[cn][1], x2 = r[cn][2];
        if(cn >= rn)
        {
            const float* B = M + sym_index(rn, cn) * 9;  // column-major
            acc0 = __fmaf_rn(B[0], x0, acc0); acc0 = __fmaf_rn(B[3], x1, acc0); acc0 = __fmaf_rn(B[6], x2, acc0);
            acc1 = __fmaf_rn(B[1], x0, acc1); acc1 = __fmaf_rn(B[4], x1, acc1); acc1 = __fmaf_rn(B[7], x2, acc1);
            acc2 = __fmaf_rn(B[2], x0, acc2); acc2 = __fmaf_rn(B[5], x1, acc2); acc2 = __fmaf_rn(B[8], x2, acc2);
        }
        else
        {
            const float* B = M + sym_index(cn, rn) * 9;  // use B^T
            acc0 = __fmaf_rn(B[0], x0, acc0); acc0 = __fmaf_rn(B[1], x1, acc0); acc0 = __fmaf_rn(B[2], x2, acc0);
            acc1 = __fmaf_rn(B[3], x0, acc1); acc1 = __fmaf_rn(B[4], x1, acc1); acc1 = __fmaf_rn(B[5], x2, acc1);
            acc2 = __fmaf_rn(B[6], x0, acc2); acc2 = __fmaf_rn(B[7], x1, acc2); acc2 = __fmaf_rn(B[8], x2, acc2);
        }
    }
    acc0 += __shfl_down_sync(0xffffffffu, acc0, 16);
    acc1 += __shfl_down_sync(0xffffffffu, acc1, 16);
    acc2 += __shfl_down_sync(0xffffffffu, acc2, 16);
    out[0] = acc0;
    out[1] = acc1;
    out[2] = acc2;
}

// The banks of one level handled by one warp (warp gw of W). Every bank's
// residual slice R_l (16 nodes x 3 floats, 192 B, contiguous: level 0's slots
// are written by k_restrict_fine) and its inverse come into shared memory by
// bulk copies (TMA) on one barrier, NST banks ahead per warp, so a warp never
// waits on a dependent gather. With `push`, the restriction sums of the next
// level (one per connected component of the bank, summed by its lowest lane
// in lane order) are written to R_{l+1}. Z_l = A_l^{-1} R_l for every node of
// the bank. BF: BF16 tiles on the tensor cores (INV16_BYTES per cluster),
// otherwise FP32 (INV_BYTES); a stiff cluster (inverted in FP64) is applied
// from its FP32 inverse in HBM in the BF16 path. `u` counts the banks this
// warp has run through its slots (slot and phase of the next copy). Returns
// false when a copy wait ran out (the error flag is set and the warp's copies
// in flight are drained).
constexpr uint32_t R_BYTES = BANK * 3 * sizeof(float);  // 192

template <bool BF>
__host__ __device__ constexpr uint32_t stage_bytes()
{
    return (BF ? INV16_BYTES : INV_BYTES) + R_BYTES;
}

// the bank's inverse and its residual slice, on one barrier
template <bool BF>
__device__ __forceinline__ void issue_bank_copy(unsigned char* stage, uint64_t* bar, const unsigned char* inv,
                                                const float* R, int64_t gbank)
{
    constexpr uint32_t CB = BF ? INV16_BYTES : INV_BYTES;
    mbar_arrive_expect_tx(bar, CB + R_BYTES);
    bulk_copy_g2s(stage, inv + (size_t)gbank * CB, CB, bar);
    bulk_copy_g2s(stage + CB, R + (size_t)gbank * (BANK * 3), R_BYTES, bar);
}

template <bool BF, int NST>
__device__ __forceinline__ bool apply_banks(int gw, int W, int lane, int& u, int n_banks, int cnt, int level_begin,
                                            const uint16_t* __restrict__ comp_mask,
                                            const int32_t* __restrict__ new_local, int next_begin, int push,
                                            const unsigned char* __restrict__ inv, float* R, float* __restrict__ Z,
                                            const uint8_t* __restrict__ stiff, const float* __restrict__ inv32,
                                            int* err, unsigned char* s_stage, uint64_t* s_bar)
{
    constexpr uint32_t CB = BF ? INV16_BYTES : INV_BYTES;
    constexpr uint32_t SB = stage_bytes<BF>();
    const int     sub    = lane & 15;
    const int     mine   = gw < n_banks ? (n_banks - 1 - gw) / W + 1 : 0;
    const int64_t gbank0 = level_begin / BANK;
    if(lane == 0)
    {
        fence_proxy_async_smem();
        for(int j = 0; j < mine && j < NST; ++j)
        {
            const int slot = (u + j) % NST;
            issue_bank_copy<BF>(s_stage + slot * SB, &s_bar[slot], inv, R, gbank0 + gw + (int64_t)j * W);
        }
    }
    __syncwarp();
    // component mask and next-level index of the next bank (lanes 0-15)
    uint32_t ncm = 0;
    int      nnl = 0;
    auto load_meta = [&](int jj) {
        ncm = 0;
        nnl = 0;
        if(!push || lane >= 16 || jj >= mine)
            return;
        const int node = (gw + jj * W) * BANK + sub;
        if(node < cnt)
        {
            ncm = comp_mask[node];
            nnl = new_local[node];
        }
    };
    load_meta(0);
    int j = 0;
    for(; j < mine; ++j)
    {
        const int      bank  = gw + j * W;
        const int      slot  = (u + j) % NST;
        const bool     use32 = BF && stiff != nullptr && stiff[gbank0 + bank] != 0;
        const uint32_t cm    = ncm;
        const int      nl    = nnl;
        const bool     live  = bank * BANK + sub < cnt;
        load_meta(j + 1);
        unsigned char* stage = s_stage + slot * SB;
        float(*s_r)[3]       = reinterpret_cast<float(*)[3]>(stage + CB);
        const bool ok = mbar_wait(&s_bar[slot], (uint32_t)(((u + j) / NST) & 1), err, DERR_TMA_TIMEOUT);
        if(!__all_sync(0xffffffffu, ok))
            break;
        if(push && lane < 16 && live && (cm & ((1u << lane) - 1u)) == 0)
        {
            float s0 = 0.f, s1 = 0.f, s2 = 0.f;
            for(uint32_t m = cm; m; m &= m - 1)
            {
                const int l = __ffs(m) - 1;
                s0 += s_r[l][0];
                s1 += s_r[l][1];
                s2 += s_r[l][2];
            }
            const int64_t g = (int64_t)next_begin + nl;
            R[3 * g]     = s0;
            R[3 * g + 1] = s1;
            R[3 * g + 2] = s2;
        }
        float* Zb = Z + 3 * ((int64_t)level_begin + (int64_t)bank * BANK);
        if(BF && !use32)
            cluster_product_mma(stage, &s_r[0][0], lane, Zb);
        else
        {
            float        out[3];
            const float* Mc = use32 ? inv32 + (size_t)(gbank0 + bank) * SYM * 9 : reinterpret_cast<const float*>(stage);
            cluster_product(Mc, s_r, lane, out);
            if(lane < 16)
            {
                Zb[3 * sub]     = out[0];
                Zb[3 * sub + 1] = out[1];
                Zb[3 * sub + 2] = out[2];
            }
        }
        __syncwarp();
        if(lane == 0 && j + NST < mine)
        {
            fence_proxy_async_smem();
            issue_bank_copy<BF>(stage, &s_bar[slot], inv, R, gbank0 + bank + (int64_t)NST * W);
        }
    }
    if(j < mine)
    {
        // a wait ran out: drain this warp's copies still in flight (bounded)
        if(lane == 0)
            for(int q = j; q < mine && q < j + NST; ++q)
                mbar_wait(&s_bar[(u + q) % NST], (uint32_t)(((u + q) / NST) & 1), nullptr, 0);
        __syncwarp();
        return false;
    }
    u += mine;
    return true;
}

// one level over a persistent grid of APPLY_WARPS-warp CTAs
template <bool BF, int NST>
__global__ void __launch_bounds__(APPLY_WARPS * 32)
    k_apply_level(int n_banks, int cnt, int level_begin, const uint16_t* __restrict__ comp_mask,
                  const int32_t* __restrict__ new_local, int next_begin, int push,
                  const unsigned char* __restrict__ inv, float* R, float* __restrict__ Z,
                  const uint8_t* __restrict__ stiff, const float* __restrict__ inv32, const int* converged, int* err)
{
    if(converged && *converged)
        return;
    constexpr uint32_t SB = stage_bytes<BF>();
    __shared__ __align__(128) unsigned char s_stage[APPLY_WARPS][NST][SB];
    __shared__ uint64_t s_bar[APPLY_WARPS][NST];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if(lane == 0)
    {
        for(int q = 0; q < NST; ++q)
            mbar_init(&s_bar[w][q], 1);
        mbar_fence_init();
    }
    __syncwarp();
    int u = 0;
    apply_banks<BF, NST>(blockIdx.x * APPLY_WARPS + w, gridDim.x * APPLY_WARPS, lane, u, n_banks, cnt,
                               level_begin, comp_mask, new_local, next_begin, push, inv, R, Z, stiff, inv32, err,
                               &s_stage[w][0][0], s_bar[w]);
}

// persistent grid: as many CTAs as fit on the SMs at once (less `spare` per
// SM, at least one), at most `cap` per SM when cap > 0, capped by the banks
template <typename K>
int apply_grid(K kernel, int n_banks, int spare = 0, int cap = 0)
{
    int occ = 0;
    if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, APPLY_WARPS * 32, 0) != cudaSuccess || occ < 1)
        occ = 1;
    occ = occ - spare >= 1 ? occ - spare : 1;
    if(cap > 0 && occ > cap)
        occ = cap;
    const int max_warps = NUM_SMS_HINT * occ * APPLY_WARPS;
    const int warps     = n_banks < max_warps ? n_banks : max_warps;
    return (warps + APPLY_WARPS - 1) / APPLY_WARPS;
}

// The fine residual in partition order and its level-1 restriction, one
// half-warp per bank over the whole grid: R_0 (the slots of level 0, FP32,
// zero in padding slots) is the only gather of r through part_to_real, so the
// fine level streams its banks' residuals with their inverses; with `push`,
// R_1 = per connected component of a bank the sum of its nodes by its lowest
// lane, in lane order, so the coarse levels can run beside the fine level.
template <typename VT>
__global__ void __launch_bounds__(APPLY_WARPS * 32)
    k_restrict_fine(int n_banks, const int32_t* __restrict__ p2r, const VT* __restrict__ r, int roff,
                    const uint16_t* __restrict__ comp_mask, const int32_t* __restrict__ new_local, int next_begin,
                    int push, float* __restrict__ R, const int* converged)
{
    if(converged && *converged)
        return;
    __shared__ float s_r[APPLY_WARPS][2][BANK][3];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, half = lane >> 4, sub = lane & 15;
    const int bank = (blockIdx.x * APPLY_WARPS + w) * 2 + half;
    float     n0 = 0.f, n1 = 0.f, n2 = 0.f;
    bool      live = false;
    uint32_t  cm   = 0;
    int       nl   = 0;
    if(bank < n_banks)
    {
        const int node = bank * BANK + sub;
        const int v    = p2r[node];
        live           = v >= 0;
        if(live)
        {
            if constexpr(sizeof(VT) == 4)
            {
                const float4 q = *reinterpret_cast<const float4*>(r + roff + 4 * (int64_t)v);
                n0 = q.x;
                n1 = q.y;
                n2 = q.z;
            }
            else
            {
                n0 = (float)r[roff + 3 * (int64_t)v];
                n1 = (float)r[roff + 3 * (int64_t)v + 1];
                n2 = (float)r[roff + 3 * (int64_t)v + 2];
            }
            if(push)
            {
                cm = comp_mask[node];
                nl = new_local[node];
            }
        }
        R[3 * (int64_t)node]     = n0;
        R[3 * (int64_t)node + 1] = n1;
        R[3 * (int64_t)node + 2] = n2;
    }
    s_r[w][half][sub][0] = n0;
    s_r[w][half][sub][1] = n1;
    s_r[w][half][sub][2] = n2;
    __syncwarp();
    if(push && live && (cm & ((1u << sub) - 1u)) == 0)
    {
        float s0 = 0.f, s1 = 0.f, s2 = 0.f;
        for(uint32_t m = cm; m; m &= m - 1)
        {
            const int l = __ffs(m) - 1;
            s0 += s_r[w][half][l][0];
            s1 += s_r[w][half][l][1];
            s2 += s_r[w][half][l][2];
        }
        const int64_t g = (int64_t)next_begin + nl;
        R[3 * g]     = s0;
        R[3 * g + 1] = s1;
        R[3 * g + 2] = s2;
    }
}

// The additive prolongation of the coarse levels folded top-down into the
// level-1 slots: Z_1[n] += Z_2[parent(n)] + Z_3[grandparent(n)] + ...
// (left to right from level 2), so the finish adds one coarse value per
// vertex (Z_0 of its slot + this sum of its level-1 node) instead of one per
// level. One thread per level-1 node; each reads its own slot and coarser
// levels only.
// anc[c * (L - 2) + (l - 2)]: global slot of level-1 node c's ancestor at
// level l (-1: none), from the hierarchy (mas_init)
__global__ void k_fold_prolongation(int cnt1, int begin1, int L, const int32_t* __restrict__ anc, float* __restrict__ Z,
                                    const int* converged)
{
    if(converged && *converged)
        return;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if(c >= cnt1)
        return;
    int32_t a[MAX_LEVELS - 2];
#pragma unroll
    for(int l = 0; l < MAX_LEVELS - 2; ++l)
        a[l] = l < L - 2 ? anc[(int64_t)c * (L - 2) + l] : -1;
    const int64_t g1 = (int64_t)begin1 + c;
    float         a0 = Z[3 * g1], a1 = Z[3 * g1 + 1], a2 = Z[3 * g1 + 2];
#pragma unroll
    for(int l = 0; l < MAX_LEVELS - 2; ++l)
        if(a[l] >= 0)
        {
            a0 += Z[3 * (int64_t)a[l]];
            a1 += Z[3 * (int64_t)a[l] + 1];
            a2 += Z[3 * (int64_t)a[l] + 2];
        }
    Z[3 * g1]     = a0;
    Z[3 * g1 + 1] = a1;
    Z[3 * g1 + 2] = a2;
}

// the ancestor table of the level-1 nodes (walks the next-level ids once)
struct LevelIds
{
    const int32_t* new_local[MAX_LEVELS];
    int32_t        begin[MAX_LEVELS + 1];
};
__global__ void k_h_ancestors(int cnt1, int L, LevelIds ids, int32_t* anc)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if(c >= cnt1)
        return;
    int loc = c;
    for(int l = 2; l < L; ++l)
    {
        loc = loc >= 0 ? ids.new_local[l - 1][loc] : -1;
        anc[(int64_t)c * (L - 2) + (l - 2)] = loc >= 0 ? ids.begin[l] + loc : -1;
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
void mas_init(b2s_solver* s, int32_t offset, int32_t vn, const int32_t* adj_start, const int32_t* adj_list, int32_t N,
              const int32_t* p2r, const int32_t* r2p)
{
    B2S_REQUIRE(vn > 0 && N > 0 && offset >= 0, B2S_ERR_ARGUMENT, "MAS range must be non-empty");
    B2S_REQUIRE(N % BANK == 0, B2S_ERR_ARGUMENT, "part_map_size must be a multiple of 16");
    if(!s->mas_side)
    {
        B2S_CUDA(cudaStreamCreateWithFlags(&s->mas_side, cudaStreamNonBlocking));
        B2S_CUDA(cudaEventCreateWithFlags(&s->mas_fork, cudaEventDisableTiming));
        B2S_CUDA(cudaEventCreateWithFlags(&s->mas_join, cudaEventDisableTiming));
    }
    // validate the maps on the host (the reference asserts the same, fem_mas_preconditioner.cu:331-360)
    for(int p = 0; p < N; ++p)
    {
        B2S_REQUIRE(p2r[p] >= -1 && p2r[p] < vn, B2S_ERR_ARGUMENT, "part_to_real entry out of range");
        if(p2r[p] >= 0)
            B2S_REQUIRE(r2p[p2r[p]] == p, B2S_ERR_ARGUMENT, "part_to_real / real_to_part are not inverse");
    }
    for(int v = 0; v < vn; ++v)
    {
        B2S_REQUIRE(r2p[v] >= -1 && r2p[v] < N, B2S_ERR_ARGUMENT, "real_to_part entry out of range");
        if(r2p[v] >= 0)
            B2S_REQUIRE(p2r[r2p[v]] == v, B2S_ERR_ARGUMENT, "part_to_real / real_to_part are not inverse");
        B2S_REQUIRE(adj_start[v + 1] >= adj_start[v], B2S_ERR_ARGUMENT, "adjacency start not monotone");
    }
    const int64_t nnz_adj = adj_start[vn];
    for(int64_t e = 0; e < nnz_adj; ++e)
        B2S_REQUIRE(adj_list[e] >= 0 && adj_list[e] < vn, B2S_ERR_ARGUMENT, "adjacency entry out of range");

    cudaStream_t st = s->stream;
    MasState&    M  = s->mas;
    MasState&    X  = s->mas;
    M.initialized   = false;
    M.offset        = offset;
    M.vn            = vn;
    M.N             = N;
    M.L             = compute_num_levels(std::max(N, vn));
    const int L     = M.L;
    M.level_begin.assign(L + 1, 0);
    M.level_count.assign(L + 1, 0);

    DBuf<int32_t> d_start, d_num, d_list;
    std::vector<int32_t> h_num(vn);
    for(int v = 0; v < vn; ++v)
        h_num[v] = adj_start[v + 1] - adj_start[v];
    d_start.resize(vn + 1);
    d_num.resize(vn);
    d_list.resize(std::max<int64_t>(nnz_adj, 1));
    M.p2r.resize(N);
    M.r2p.resize(vn);
    B2S_CUDA(cudaMemcpyAsync(d_start.data(), adj_start, sizeof(int32_t) * (vn + 1), cudaMemcpyHostToDevice, st));
    B2S_CUDA(cudaMemcpyAsync(d_num.data(), h_num.data(), sizeof(int32_t) * vn, cudaMemcpyHostToDevice, st));
    if(nnz_adj > 0)
        B2S_CUDA(cudaMemcpyAsync(d_list.data(), adj_list, sizeof(int32_t) * nnz_adj, cudaMemcpyHostToDevice, st));
    B2S_CUDA(cudaMemcpyAsync(M.p2r.data(), p2r, sizeof(int32_t) * N, cudaMemcpyHostToDevice, st));
    B2S_CUDA(cudaMemcpyAsync(M.r2p.data(), r2p, sizeof(int32_t) * vn, cudaMemcpyHostToDevice, st));

    // level-1 node slots start after every level-0 slot and every vertex id
    // (mas_preconditioner_engine.cu:2162-2184 numbers them the same way)
    const int level1_begin = bank_align(std::max(bank_align(N), vn));
    X.cst.resize((size_t)L * vn);
    B2S_CUDA(cudaMemsetAsync(X.cst.data(), 0xff, sizeof(int32_t) * (size_t)L * vn, st));

    DBuf<uint32_t> mask;
    DBuf<int32_t>  comp_count, bank_off, rank, scan_tmp;
    mask.resize(std::max(N, vn) + BANK);
    rank.resize(std::max(N, vn) + BANK);
    const int TB = 256;

    // level 0
    {
        const int n_banks = N / BANK;
        comp_count.resize(n_banks + 1);
        bank_off.resize(n_banks + 1);
        X.comp_mask[0].resize(N);
        X.new_local[0].resize(N);
        k_h_mask_l0<<<grid_for(N, TB), TB, 0, st>>>(N, M.p2r.data(), M.r2p.data(), d_start.data(), d_num.data(),
                                                    d_list.data(), mask.data());
        B2S_CHECK_LAUNCH();
        k_h_components<<<grid_for(n_banks, 128), 128, 0, st>>>(N, n_banks, mask.data(), M.p2r.data(), 1,
                                                                comp_count.data(), rank.data(),
                                                                X.comp_mask[0].data());
        B2S_CHECK_LAUNCH();
        exclusive_scan(s, comp_count.data(), bank_off.data(), n_banks, scan_tmp);
        k_h_assign<<<grid_for(N, TB), TB, 0, st>>>(N, rank.data(), bank_off.data(), X.new_local[0].data());
        B2S_CHECK_LAUNCH();
        k_h_cst_l1<<<grid_for(vn, TB), TB, 0, st>>>(vn, M.r2p.data(), X.new_local[0].data(), X.cst.data());
        B2S_CHECK_LAUNCH();
        int32_t cnt1 = 0;
        B2S_CUDA(cudaMemcpyAsync(&cnt1, bank_off.data() + n_banks, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        B2S_CUDA(cudaStreamSynchronize(st));
        M.level_begin[0] = 0;
        M.level_count[0] = N;
        M.level_begin[1] = level1_begin;
        M.level_count[1] = cnt1;
    }
    // levels 1 .. L-1
    for(int level = 1; level < L; ++level)
    {
        const int cnt = M.level_count[level], beg = M.level_begin[level];
        const int n_banks = (cnt + BANK - 1) / BANK;
        const int next_begin = beg + bank_align(cnt);
        B2S_CUDA(cudaMemsetAsync(mask.data(), 0, sizeof(uint32_t) * (cnt + BANK), st));
        const int32_t* cst_prev = X.cst.data() + (size_t)(level - 1) * vn;
        k_h_mask_lx<<<grid_for(N, TB), TB, 0, st>>>(N, vn, M.p2r.data(), cst_prev, d_start.data(), d_num.data(),
                                                    d_list.data(), mask.data(), cnt);
        B2S_CHECK_LAUNCH();
        comp_count.resize(n_banks + 1);
        bank_off.resize(n_banks + 1);
        X.comp_mask[level].resize(std::max(cnt, 1));
        X.new_local[level].resize(std::max(cnt, 1));
        k_h_components<<<grid_for(n_banks, 128), 128, 0, st>>>(cnt, n_banks, mask.data(), nullptr, 0,
                                                                comp_count.data(), rank.data(),
                                                                X.comp_mask[level].data());
        B2S_CHECK_LAUNCH();
        exclusive_scan(s, comp_count.data(), bank_off.data(), n_banks, scan_tmp);
        k_h_assign<<<grid_for(cnt, TB), TB, 0, st>>>(cnt, rank.data(), bank_off.data(), X.new_local[level].data());
        B2S_CHECK_LAUNCH();
        k_h_cst_next<<<grid_for(vn, TB), TB, 0, st>>>(vn, cst_prev, X.new_local[level].data(), cnt,
                                                      X.cst.data() + (size_t)level * vn);
        B2S_CHECK_LAUNCH();
        int32_t cnt_next = 0;
        B2S_CUDA(cudaMemcpyAsync(&cnt_next, bank_off.data() + n_banks, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        B2S_CUDA(cudaStreamSynchronize(st));
        if(level + 1 <= L)
        {
            if(level + 1 < (int)M.level_begin.size())
            {
                M.level_begin[level + 1] = next_begin;
                M.level_count[level + 1] = cnt_next;
            }
        }
    }
    M.total    = M.level_begin[L];
    M.clusters = M.total / BANK;
    // coarse table
    X.level_begin_dev.resize(L + 1);
    B2S_CUDA(cudaMemcpyAsync(X.level_begin_dev.data(), M.level_begin.data(), sizeof(int32_t) * (L + 1),
                             cudaMemcpyHostToDevice, st));
    M.ctable.resize((size_t)vn * std::max(L - 1, 1));
    if(L > 1)
    {
        k_h_ctable<<<grid_for(vn, TB), TB, 0, st>>>(vn, L, X.cst.data(), X.level_begin_dev.data(), M.ctable.data());
        B2S_CHECK_LAUNCH();
    }
    M.hess.resize((size_t)M.clusters * SYM * 9);
    M.inv.resize((size_t)M.clusters * SYM * 9);
    M.R.resize((size_t)M.total * 3 + 3);
    M.Z.resize((size_t)M.total * 3 + 3);
    B2S_CUDA(cudaMemsetAsync(M.R.data(), 0, M.R.bytes(), st));
    B2S_CUDA(cudaMemsetAsync(M.Z.data(), 0, M.Z.bytes(), st));
    // the coarse ancestors of every level-1 node (the prolongation fold)
    if(L > 2 && M.level_count[1] > 0)
    {
        LevelIds ids{};
        for(int l = 0; l < L; ++l)
        {
            ids.new_local[l] = X.new_local[l].data();
            ids.begin[l]     = M.level_begin[l];
        }
        M.anc.resize((size_t)M.level_count[1] * (L - 2));
        k_h_ancestors<<<grid_for(M.level_count[1], TB), TB, 0, st>>>(M.level_count[1], L, ids, M.anc.data());
        B2S_CHECK_LAUNCH();
    }
    // level-1 node of every vertex, contiguous (the finish reads it per vertex)
    M.node1.resize(std::max(vn, 1));
    if(L > 1)
    {
        k_h_node1<<<grid_for(vn, TB), TB, 0, st>>>(vn, L, M.ctable.data(), M.node1.data());
        B2S_CHECK_LAUNCH();
    }
    M.h_ctable.resize((size_t)vn * std::max(L - 1, 1));
    if(L > 1)
        B2S_CUDA(cudaMemcpyAsync(M.h_ctable.data(), M.ctable.data(), sizeof(int32_t) * M.h_ctable.size(),
                                 cudaMemcpyDeviceToHost, st));
    B2S_CUDA(cudaStreamSynchronize(st));
    M.initialized = true;
}

void mas_assemble(b2s_solver* s, int invert_mode)
{
    MasState& M = s->mas;
    MasState& X = s->mas;
    B2S_REQUIRE(M.initialized, B2S_ERR_STATE, "MAS not initialised");
    B2S_REQUIRE(s->A.valid, B2S_ERR_STATE, "no assembled matrix");
    B2S_REQUIRE(M.offset + M.vn <= s->A.nb, B2S_ERR_ARGUMENT, "MAS range exceeds the matrix");
    cudaStream_t st = s->stream;
    const int    TB = 256;
    const Matrix& A = s->A;
    B2S_CUDA(cudaMemsetAsync(M.hess.data(), 0, M.hess.bytes(), st));
    if(A.nnz > 0)
    {
        k_g_level0<<<grid_for(A.nnz, TB), TB, 0, st>>>(A.nnz, A.rows.data(), A.cols.data(), A.vals.data(), A.stride,
                                                       M.offset,
                                                       M.vn, M.r2p.data(), M.hess.data());
        B2S_CHECK_LAUNCH();
    }
    // coarse levels: A_1 from A (vertex ids -> level-1 ids), A_{l+1} from A_l
    const Matrix* prev     = &A;
    int           prev_off = M.offset;
    int           prev_n   = M.vn;
    const int32_t* map     = X.cst.data();  // vertex -> level-1 local id
    for(int level = 1; level < M.L; ++level)
    {
        const int64_t T = prev->nnz;
        Matrix&       C = M.coarse[level];
        M.trip_rows.resize(std::max<int64_t>(T, 1), 1.2);
        M.trip_cols.resize(std::max<int64_t>(T, 1), 1.2);
        M.trip_vals.resize((size_t)9 * std::max<int64_t>(T, 1), 1.2);
        if(T > 0)
        {
            k_g_restrict<<<grid_for(T, TB), TB, 0, st>>>(T, prev->rows.data(), prev->cols.data(), prev->vals.data(),
                                                         prev->stride, prev_off, prev_n, map, M.trip_rows.data(),
                                                         M.trip_cols.data(), M.trip_vals.data());
            B2S_CHECK_LAUNCH();
        }
        assemble_triplets(s, C, M.level_count[level], T, M.trip_rows.data(), M.trip_cols.data(), M.trip_vals.data(),
                          false);
        if(C.nnz > 0)
        {
            k_g_extract<<<grid_for(C.nnz, TB), TB, 0, st>>>(C.nnz, C.rows.data(), C.cols.data(), C.vals.data(),
                                                            C.stride, M.level_begin[level], M.hess.data());
            B2S_CHECK_LAUNCH();
        }
        prev     = &C;
        prev_off = 0;
        prev_n   = M.level_count[level];
        map      = X.new_local[level].data();
    }
    mas_invert_clusters(s, invert_mode);
}

// z[off..off+vn) gets the MAS part of z = P r; Jacobi/identity elsewhere is
// handled by the caller (collect kernel in the PCG, or precond_apply).
// bf16: use the packed D + BF16 tiles of D^-1 M D^-1 (mas_pack_bf16 first).
template <typename VT>
static void apply_levels_t(b2s_solver* s, const VT* r, const int* converged, bool bf16)
{
    MasState&    M   = s->mas;
    cudaStream_t st  = s->stream;
    int*         err = device_error_flag(s);
    const int    n_banks0 = M.N / BANK;
    const int    tb       = APPLY_WARPS * 32;
    const unsigned char* inv = bf16 ? M.inv16.data() : reinterpret_cast<const unsigned char*>(M.inv.data());
    const uint8_t*       stiff = bf16 ? M.stiff.data() : nullptr;
    // element offset of the range's first vertex in r (FP32: 4 per node)
    const int off = (sizeof(VT) == 4 ? 4 : 3) * M.offset;
    auto level_kernel = bf16 ? k_apply_level<true, APPLY_STAGES_BF16> : k_apply_level<false, APPLY_STAGES_F32>;
    auto launch_level = [&](int level, cudaStream_t cs, int spare, int cap)
    {
        const int cnt     = level == 0 ? M.N : M.level_count[level];
        const int n_banks = (cnt + BANK - 1) / BANK;
        const int push    = level > 0 && level + 1 < M.L ? 1 : 0;
        level_kernel<<<apply_grid(level_kernel, n_banks, spare, cap), tb, 0, cs>>>(
            n_banks, cnt, M.level_begin[level], M.comp_mask[level].data(), M.new_local[level].data(),
            push ? M.level_begin[level + 1] : 0, push, inv, M.R.data(), M.Z.data(), stiff, M.inv.data(), converged,
            err);
        B2S_CHECK_LAUNCH();
    };
    // 1. R_0 (the fine residual in partition order) and R_1, whole grid.
    // 2. Level 1 -- the largest coarse level, a few thousand banks -- on the
    //    whole GPU (it pushes R_2).
    // 3. The fine level's products on `st` with one CTA slot per SM left free,
    //    beside the rest of the coarse chain on the side stream (one launch per
    //    level in the free slots, then the prolongation fold); `st` waits for
    //    them before the finish. (One CTA running the small top levels with
    //    CTA barriers between them needs more shared memory than the fine
    //    level leaves on an SM, so it waited for the fine level: 1 ms per
    //    solve slower.)
    if(n_banks0 > 0)
    {
        const int pairs = (n_banks0 + 1) / 2;
        k_restrict_fine<VT><<<(pairs + APPLY_WARPS - 1) / APPLY_WARPS, tb, 0, st>>>(
            n_banks0, M.p2r.data(), r, off, M.comp_mask[0].data(), M.new_local[0].data(),
            M.L > 1 ? M.level_begin[1] : 0, M.L > 1 ? 1 : 0, M.R.data(), converged);
        B2S_CHECK_LAUNCH();
    }
    const bool coarse = M.L > 1 && M.level_count[1] > 0;
    if(coarse)
        launch_level(1, st, 0, 0);
    const bool fork = coarse && M.L > 2 && n_banks0 > 0 && s->mas_side != nullptr;
    if(fork)
    {
        B2S_CUDA(cudaEventRecord(s->mas_fork, st));
        B2S_CUDA(cudaStreamWaitEvent(s->mas_side, s->mas_fork, 0));
    }
    if(n_banks0 > 0)
        launch_level(0, st, fork ? 1 : 0, 0);
    cudaStream_t cs = fork ? s->mas_side : st;
    for(int level = 2; level < M.L; ++level)
    {
        if(M.level_count[level] <= 0)
            break;
        launch_level(level, cs, 0, fork ? 1 : 0);
    }
    if(M.L > 2 && M.level_count[1] > 0)
    {
        k_fold_prolongation<<<grid_for(M.level_count[1], 256), 256, 0, cs>>>(
            M.level_count[1], M.level_begin[1], M.L, M.anc.data(), M.Z.data(), converged);
        B2S_CHECK_LAUNCH();
    }
    if(fork)
    {
        B2S_CUDA(cudaEventRecord(s->mas_join, cs));
        B2S_CUDA(cudaStreamWaitEvent(st, s->mas_join, 0));
    }
}

void mas_apply_levels(b2s_solver* s, const double* r, const int* converged)
{
    apply_levels_t<double>(s, r, converged, false);
}

void mas_apply_levels_f32(b2s_solver* s, const float* r, const int* converged, bool bf16)
{
    apply_levels_t<float>(s, r, converged, bf16);
}

// BF16 diagonal-scaled copy of the current FP32 inverses
void mas_pack_bf16(b2s_solver* s)
{
    MasState& M = s->mas;
    M.inv16.resize((size_t)M.clusters * INV16_BYTES);
    if(M.clusters > 0)
    {
        k_pack_inverse_bf16<<<M.clusters, PACK_THREADS, 0, s->stream>>>(M.clusters, M.inv.data(), M.inv16.data());
        B2S_CHECK_LAUNCH();
    }
}
}  // namespace b2s
