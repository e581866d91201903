// Triplet -> block-upper BSR assembly (deterministic), and the device scan.
//
// Semantics follow MatrixConverter<Float,3>::convert_sym
// (src/backends/cuda/algorithm/details/matrix_converter.inl:1550-1701):
// keep row >= 0 && row <= col, order by (row, col) with ties in source
// order, sum each run. The reference sorts a 64-bit key with CUB and sums
// runs with cross-warp FP64 atomics (rounding-nondeterministic). Here the
// sort is a counting sort on the row followed by an in-warp rank sort of each
// row's (col, source) pairs, and every run is summed by one lane in source
// order -- the pattern is identical, the values are bit-reproducible.
#include "b2s_internal.cuh"

namespace b2s
{
namespace
{
constexpr int SCAN_BLOCK = 256;
constexpr int SCAN_ITEMS = 4;  // elements per thread
constexpr int SCAN_TILE  = SCAN_BLOCK * SCAN_ITEMS;

// block-wide inclusive scan of one int per thread (warp shuffles + smem)
__device__ __forceinline__ int block_inclusive_scan(int v, int* warp_sums)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for(int o = 1; o < 32; o <<= 1)
    {
        int t = __shfl_up_sync(0xffffffffu, v, o);
        if(lane >= o)
            v += t;
    }
    if(lane == 31)
        warp_sums[warp] = v;
    __syncthreads();
    if(warp == 0)
    {
        int w = (lane < (int)(blockDim.x >> 5)) ? warp_sums[lane] : 0;
#pragma unroll
        for(int o = 1; o < 32; o <<= 1)
        {
            int t = __shfl_up_sync(0xffffffffu, w, o);
            if(lane >= o)
                w += t;
        }
        if(lane < (int)(blockDim.x >> 5))
            warp_sums[lane] = w;
    }
    __syncthreads();
    if(warp > 0)
        v += warp_sums[warp - 1];
    return v;
}

// tile exclusive scan; writes out[i] (i < n) and the tile total into tile_sums
__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_tiles(const int32_t* in, int32_t* out, int64_t n,
                                                           int32_t* tile_sums)
{
    __shared__ int warp_sums[SCAN_BLOCK / 32];
    const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
    int           v[SCAN_ITEMS];
    int           local = 0;
#pragma unroll
    for(int k = 0; k < SCAN_ITEMS; ++k)
    {
        v[k] = (base + k < n) ? in[base + k] : 0;
        local += v[k];
    }
    int incl = block_inclusive_scan(local, warp_sums);
    int run  = incl - local;
#pragma unroll
    for(int k = 0; k < SCAN_ITEMS; ++k)
    {
        if(base + k < n)
            out[base + k] = run;
        run += v[k];
    }
    if(threadIdx.x == blockDim.x - 1)
        tile_sums[blockIdx.x] = incl;
}

__global__ void k_scan_add(int32_t* out, int64_t n, const int32_t* tile_offsets)
{
    const int64_t i = (int64_t)blockIdx.x * SCAN_TILE + threadIdx.x;
    const int32_t add = tile_offsets[blockIdx.x];
#pragma unroll
    for(int k = 0; k < SCAN_ITEMS; ++k)
    {
        int64_t j = i + (int64_t)k * SCAN_BLOCK;
        if(j < n)
            out[j] += add;
    }
}

__global__ void k_write_total(int32_t* out, int64_t n, const int32_t* in, const int32_t* tile_offsets,
                              int64_t last_tile)
{
    // out[n] = exclusive(out[n-1]) + in[n-1]; computed from the last element
    if(threadIdx.x == 0 && blockIdx.x == 0)
        out[n] = (n > 0) ? (out[n - 1] + in[n - 1]) : 0;
}
}  // namespace

// Exclusive scan of n int32 into out[0..n] (out[n] = total). `in` may alias
// `out` only when the caller keeps a copy of in[n-1]; here in != out always.
void exclusive_scan(b2s_solver* s, const int32_t* in, int32_t* out, int64_t n, DBuf<int32_t>& tmp)
{
    cudaStream_t st = s->stream;
    if(n <= 0)
    {
        B2S_CUDA(cudaMemsetAsync(out, 0, sizeof(int32_t), st));
        return;
    }
    const int64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    // recursion through a flat list of levels inside one scratch buffer
    std::vector<int64_t> level_n{n};
    while(level_n.back() > SCAN_TILE)
        level_n.push_back((level_n.back() + SCAN_TILE - 1) / SCAN_TILE);
    // scratch: for each level k >= 1 an array of level_n[k] sums + their scan (+1)
    int64_t need = 0;
    std::vector<int64_t> off_sums, off_scan;
    for(size_t k = 0; k < level_n.size(); ++k)
    {
        int64_t t = (level_n[k] + SCAN_TILE - 1) / SCAN_TILE;
        off_sums.push_back(need);
        need += t;
        off_scan.push_back(need);
        need += t + 1;
    }
    tmp.resize(need + 1, 1.5);
    // up-sweep: scan tiles at every level
    const int32_t* cur_in  = in;
    int32_t*       cur_out = out;
    for(size_t k = 0; k < level_n.size(); ++k)
    {
        int64_t nk = level_n[k];
        int64_t t  = (nk + SCAN_TILE - 1) / SCAN_TILE;
        k_scan_tiles<<<(unsigned)t, SCAN_BLOCK, 0, st>>>(cur_in, cur_out, nk, tmp.data() + off_sums[k]);
        B2S_CHECK_LAUNCH();
        cur_in  = tmp.data() + off_sums[k];
        cur_out = tmp.data() + off_scan[k];
        if(t == 1)
        {
            // single tile: its exclusive scan is zero
            B2S_CUDA(cudaMemsetAsync(cur_out, 0, sizeof(int32_t), st));
            break;
        }
    }
    // down-sweep: add scanned tile offsets
    for(int k = (int)level_n.size() - 1; k >= 0; --k)
    {
        int64_t nk = level_n[k];
        int64_t t  = (nk + SCAN_TILE - 1) / SCAN_TILE;
        if(t == 1)
            continue;
        int32_t* target = (k == 0) ? out : tmp.data() + off_scan[k - 1];
        k_scan_add<<<(unsigned)t, SCAN_BLOCK, 0, st>>>(target, nk, tmp.data() + off_scan[k]);
        B2S_CHECK_LAUNCH();
    }
    (void)tiles;
    k_write_total<<<1, 32, 0, st>>>(out, n, in, nullptr, 0);
    B2S_CHECK_LAUNCH();
}

namespace
{
constexpr int ASM_BLOCK = 256;
constexpr int ROW_CAP   = 256;  // (col, src) pairs per row held in shared memory

// The triplets of a warp mostly come from one or two elements, so few
// distinct rows: the lanes holding the same row (__match_any_sync) add their
// count with one atomic by the lowest of them. The loops step warp by warp so
// all lanes take part in every match.
__global__ void k_count_rows(const int32_t* __restrict__ rows, const int32_t* __restrict__ cols, int64_t T,
                             int32_t nb, int32_t* __restrict__ row_count, int* err)
{
    const int     lane   = threadIdx.x & 31;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for(int64_t base = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < T; base += stride)
    {
        const int64_t t = base + lane;
        int32_t       r = -1, c = 0;
        if(t < T)
        {
            r = rows[t];
            c = cols[t];
        }
        bool ok = t < T && r >= 0 && r <= c;
        if(ok && c >= nb)
        {
            atomicOr(err, DERR_TRIPLET_INDEX);
            ok = false;
        }
        const unsigned peers = __match_any_sync(0xffffffffu, ok ? r : -1 - lane);
        if(ok && lane == __ffs(peers) - 1)
            atomicAdd(&row_count[r], __popc(peers));
    }
}

// (column, source) of every kept triplet into its row's bucket; the lanes of
// a row take consecutive places from one atomic of the lowest of them
__global__ void k_scatter_rows(const int32_t* __restrict__ rows, const int32_t* __restrict__ cols, int64_t T,
                               int32_t nb, const int32_t* __restrict__ row_start, int32_t* __restrict__ row_fill,
                               int2* __restrict__ bucket, int* err)
{
    const int     lane   = threadIdx.x & 31;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for(int64_t base = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < T; base += stride)
    {
        const int64_t t = base + lane;
        int32_t       r = -1, c = 0;
        if(t < T)
        {
            r = rows[t];
            c = cols[t];
        }
        const bool ok  = t < T && r >= 0 && r <= c && c < nb;
        int32_t    beg = 0, len = 0;
        if(ok)
        {
            beg = row_start[r];
            len = row_start[r + 1] - beg;
        }
        const unsigned peers  = __match_any_sync(0xffffffffu, ok ? r : -1 - lane);
        const int      leader = __ffs(peers) - 1;
        int32_t        pos    = 0;
        if(ok && lane == leader)
            pos = atomicAdd(&row_fill[r], __popc(peers));
        pos = __shfl_sync(0xffffffffu, pos, leader);
        if(!ok)
            continue;
        const int32_t k = pos + __popc(peers & ((1u << lane) - 1u));
        if(k >= len)
        {
            atomicOr(err, DERR_ROW_OVERFLOW);
            continue;
        }
        bucket[beg + k] = make_int2(c, (int32_t)t);
    }
}

__device__ __forceinline__ bool key_less(int32_t ca, int32_t sa, int32_t cb, int32_t sb)
{
    return ca < cb || (ca == cb && sa < sb);
}

// One warp per row: rank every (col, src) pair of the row by counting the
// pairs that order before it, write the sorted row and its unique-column count.
__global__ void __launch_bounds__(ASM_BLOCK) k_sort_rows(int32_t nb, const int32_t* __restrict__ row_start,
                                                         const int2* __restrict__ bucket,
                                                         int32_t* __restrict__ sorted_col,
                                                         int32_t* __restrict__ sorted_src,
                                                         int32_t* __restrict__ uniq_count, int32_t* long_rows)
{
    __shared__ int32_t s_col[ASM_BLOCK / 32][ROW_CAP];
    __shared__ int32_t s_src[ASM_BLOCK / 32][ROW_CAP];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int warps_total = gridDim.x * (ASM_BLOCK / 32);
    for(int32_t r = blockIdx.x * (ASM_BLOCK / 32) + w; r < nb; r += warps_total)
    {
        const int32_t beg = row_start[r], L = row_start[r + 1] - beg;
        int           uniq = 0;
        if(L <= 32)
        {
            // one key per lane (column << 32 | source), bitonic sort across
            // the warp, padding = max key
            uint64_t key = ~0ull;
            if(lane < L)
            {
                const int2 q = bucket[beg + lane];
                key          = ((uint64_t)(uint32_t)q.x << 32) | (uint64_t)(uint32_t)q.y;
            }
#pragma unroll
            for(int k = 2; k <= 32; k <<= 1)
#pragma unroll
                for(int s = k >> 1; s > 0; s >>= 1)
                {
                    const uint64_t other    = __shfl_xor_sync(0xffffffffu, key, s);
                    const bool     keep_min = ((lane & s) == 0) == ((lane & k) == 0);
                    key = keep_min ? (key < other ? key : other) : (key < other ? other : key);
                }
            const uint64_t prev = __shfl_up_sync(0xffffffffu, key, 1);
            if(lane < L)
            {
                sorted_col[beg + lane] = (int32_t)(key >> 32);
                sorted_src[beg + lane] = (int32_t)(key & 0xFFFFFFFFull);
                uniq = (lane == 0 || (prev >> 32) != (key >> 32)) ? 1 : 0;
            }
        }
        else if(L <= 64)
        {
            // bitonic sort of the (column << 32 | source) keys in registers,
            // two per lane (positions lane and lane + 32), padding = max key
            uint64_t key[2];
#pragma unroll
            for(int j = 0; j < 2; ++j)
            {
                const int p = j * 32 + lane;
                if(p < L)
                {
                    const int2 q = bucket[beg + p];
                    key[j]       = ((uint64_t)(uint32_t)q.x << 32) | (uint64_t)(uint32_t)q.y;
                }
                else
                    key[j] = ~0ull;
            }
#pragma unroll
            for(int k = 2; k <= 64; k <<= 1)
#pragma unroll
                for(int s = k >> 1; s > 0; s >>= 1)
                {
                    if(s == 32)
                    {
                        // k = 64: ascending; the partner is this lane's other key
                        const uint64_t lo = key[0] < key[1] ? key[0] : key[1];
                        const uint64_t hi = key[0] < key[1] ? key[1] : key[0];
                        key[0]            = lo;
                        key[1]            = hi;
                    }
                    else
                    {
#pragma unroll
                        for(int j = 0; j < 2; ++j)
                        {
                            const int      p     = j * 32 + lane;
                            const uint64_t other = __shfl_xor_sync(0xffffffffu, key[j], s);
                            const bool     up    = (p & k) == 0;
                            const bool     keep_min = ((p & s) == 0) == up;
                            key[j] = keep_min ? (key[j] < other ? key[j] : other) : (key[j] < other ? other : key[j]);
                        }
                    }
                }
            const uint64_t last0 = __shfl_sync(0xffffffffu, key[0], 31);
#pragma unroll
            for(int j = 0; j < 2; ++j)
            {
                const int      p    = j * 32 + lane;
                const uint64_t up1  = __shfl_up_sync(0xffffffffu, key[j], 1);
                const uint64_t prev = lane > 0 ? up1 : (j == 1 ? last0 : ~0ull);
                if(p < L)
                {
                    sorted_col[beg + p] = (int32_t)(key[j] >> 32);
                    sorted_src[beg + p] = (int32_t)(key[j] & 0xFFFFFFFFull);
                    uniq += (p == 0 || (prev >> 32) != (key[j] >> 32)) ? 1 : 0;
                }
            }
        }
        else if(L <= ROW_CAP)
        {
            for(int k = lane; k < L; k += 32)
            {
                const int2 q = bucket[beg + k];
                s_col[w][k]  = q.x;
                s_src[w][k]  = q.y;
            }
            __syncwarp();
            for(int k = lane; k < L; k += 32)
            {
                const int32_t c = s_col[w][k], sr = s_src[w][k];
                int rank = 0, head = 1;
                for(int q = 0; q < L; ++q)
                {
                    const int32_t cq = s_col[w][q], sq = s_src[w][q];
                    rank += key_less(cq, sq, c, sr) ? 1 : 0;
                    if(cq == c && sq < sr)
                        head = 0;
                }
                sorted_col[beg + rank] = c;
                sorted_src[beg + rank] = sr;
                uniq += head;
            }
            __syncwarp();
        }
        else
        {
            // longer than a warp's shared memory: sorted by k_sort_long_rows
            if(lane == 0)
                long_rows[1 + atomicAdd(long_rows, 1)] = (int32_t)r;
            continue;
        }
#pragma unroll
        for(int o = 16; o > 0; o >>= 1)
            uniq += __shfl_xor_sync(0xffffffffu, uniq, o);
        if(lane == 0)
            uniq_count[r] = uniq;
    }
}

// Rows longer than ROW_CAP pairs (e.g. an affine body touched by thousands of
// cloth vertices), listed by k_sort_rows: one CTA per row (persistent over the
// list). Every key (column << 32 | source; unique) gets its rank by counting
// the smaller keys, tile by tile through shared memory; a key is the head of
// its column's run when no key has its column and a smaller source. O(L^2 / T)
// work per row with T threads.
constexpr int LONG_THREADS = 1024;
constexpr int LONG_TILE    = 4096;

__global__ void __launch_bounds__(LONG_THREADS) k_sort_long_rows(const int32_t* __restrict__ long_rows,
                                                                 const int32_t* __restrict__ row_start,
                                                                 const int2* __restrict__ bucket,
                                                                 int32_t* __restrict__ sorted_col,
                                                                 int32_t* __restrict__ sorted_src,
                                                                 int32_t* __restrict__ uniq_count)
{
    __shared__ uint64_t s_key[LONG_TILE];
    __shared__ int      s_heads[LONG_THREADS / 32];
    const int n_long = long_rows[0];
    for(int e = blockIdx.x; e < n_long; e += gridDim.x)
    {
        const int32_t r = long_rows[1 + e], beg = row_start[r], L = row_start[r + 1] - beg;
        int           heads = 0;
        for(int base = 0; base < L; base += LONG_THREADS)
        {
            const int      i    = base + (int)threadIdx.x;
            uint64_t       me   = ~0ull;
            if(i < L)
            {
                const int2 q = bucket[beg + i];
                me           = ((uint64_t)(uint32_t)q.x << 32) | (uint64_t)(uint32_t)q.y;
            }
            const uint32_t col  = (uint32_t)(me >> 32);
            int            rank = 0;
            bool           head = true;
            for(int t0 = 0; t0 < L; t0 += LONG_TILE)
            {
                const int n = min(LONG_TILE, L - t0);
                __syncthreads();  // the previous tile is read
                for(int k = threadIdx.x; k < n; k += LONG_THREADS)
                {
                    const int2 q = bucket[beg + t0 + k];
                    s_key[k]     = ((uint64_t)(uint32_t)q.x << 32) | (uint64_t)(uint32_t)q.y;
                }
                __syncthreads();
                if(i < L)
                    for(int k = 0; k < n; ++k)
                    {
                        const uint64_t o = s_key[k];
                        rank += o < me ? 1 : 0;
                        head = head && !((uint32_t)(o >> 32) == col && o < me);
                    }
            }
            if(i < L)
            {
                sorted_col[beg + rank] = (int32_t)col;
                sorted_src[beg + rank] = (int32_t)(me & 0xFFFFFFFFull);
                heads += head ? 1 : 0;
            }
        }
        // the row's number of distinct columns
#pragma unroll
        for(int o = 16; o > 0; o >>= 1)
            heads += __shfl_xor_sync(0xffffffffu, heads, o);
        if((threadIdx.x & 31) == 0)
            s_heads[threadIdx.x >> 5] = heads;
        __syncthreads();
        if(threadIdx.x < 32)
        {
            int h = s_heads[threadIdx.x];
#pragma unroll
            for(int o = 16; o > 0; o >>= 1)
                h += __shfl_xor_sync(0xffffffffu, h, o);
            if(threadIdx.x == 0)
                uniq_count[r] = h;
        }
        __syncthreads();  // s_heads and s_key are free for the next row
    }
}

// One warp per row: every run of equal columns becomes one slot of the
// block-upper BSR: its row, column and the position of its first source in
// the sorted order (run_start; run_start[U] = T written by the caller).
__global__ void __launch_bounds__(ASM_BLOCK) k_mark_runs(int32_t nb, const int32_t* __restrict__ row_start,
                                                         const int32_t* __restrict__ sorted_col,
                                                         const int32_t* __restrict__ rowptr,
                                                         int32_t* __restrict__ out_rows, int32_t* __restrict__ out_cols,
                                                         int32_t* __restrict__ run_start,
                                                         int32_t* __restrict__ diag_index)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int warps_total = gridDim.x * (ASM_BLOCK / 32);
    for(int32_t r = blockIdx.x * (ASM_BLOCK / 32) + w; r < nb; r += warps_total)
    {
        const int32_t beg = row_start[r], L = row_start[r + 1] - beg;
        const int32_t obeg = rowptr[r];
        int           heads_before = 0;
        for(int base = 0; base < L; base += 32)
        {
            const int k = base + lane;
            bool head = false;
            int32_t c = 0;
            if(k < L)
            {
                c    = sorted_col[beg + k];
                head = (k == 0) || (sorted_col[beg + k - 1] != c);
            }
            const unsigned hm   = __ballot_sync(0xffffffffu, head);
            const int      slot = heads_before + __popc(hm & ((1u << lane) - 1u));
            if(head)
            {
                const int64_t o = (int64_t)obeg + slot;
                out_rows[o]  = r;
                out_cols[o]  = c;
                run_start[o] = beg + k;
            }
            heads_before += __popc(hm);
        }
        if(lane == 0)
            diag_index[r] = (L > 0 && sorted_col[beg] == r) ? obeg : -1;
    }
}

// One thread per (unique block, column of its 3x3): the column's 3 values
// summed over the run's sources in source order (the sorted order). The
// three threads of a block read its sources' 72 contiguous bytes together;
// four sources are fetched ahead, the additions stay in order from the first.
__global__ void __launch_bounds__(ASM_BLOCK) k_sum_runs(int64_t U, const int32_t* __restrict__ run_start,
                                                         const int32_t* __restrict__ sorted_src,
                                                         const double* __restrict__ src_vals,
                                                         double* __restrict__ out_vals, int64_t S)
{
    for(int64_t t = (int64_t)blockIdx.x * ASM_BLOCK + threadIdx.x; t < 3 * U; t += (int64_t)gridDim.x * ASM_BLOCK)
    {
        const int64_t o = t / 3;
        const int     c = (int)(t - 3 * o);
        const int32_t b = run_start[o], e = run_start[o + 1];
        double        acc[3] = {};
        for(int32_t k = b; k < e; k += 4)
        {
            int64_t src[4];
#pragma unroll
            for(int u = 0; u < 4; ++u)
                src[u] = k + u < e ? (int64_t)sorted_src[k + u] : -1;
            double v[4][3];
#pragma unroll
            for(int u = 0; u < 4; ++u)
#pragma unroll
                for(int q = 0; q < 3; ++q)
                    v[u][q] = src[u] >= 0 ? src_vals[src[u] * 9 + 3 * c + q] : 0.0;
#pragma unroll
            for(int u = 0; u < 4; ++u)
                if(src[u] >= 0)
#pragma unroll
                    for(int q = 0; q < 3; ++q)
                        acc[q] = k + u == b ? v[u][q] : acc[q] + v[u][q];
        }
#pragma unroll
        for(int q = 0; q < 3; ++q)
            out_vals[(int64_t)(3 * c + q) * S + o] = acc[q];
    }
}

// rank of every block in (column, index) order within its SPMV_TILE-block
// tile: bitonic sort of the unique keys (column << 16 | index) in shared memory
constexpr int RANK_THREADS = 512;
__global__ void __launch_bounds__(RANK_THREADS) k_tile_rank(int64_t U, const int32_t* __restrict__ cols,
                                                            uint16_t* __restrict__ trank)
{
    static_assert(SPMV_TILE <= 65536 && (SPMV_TILE & (SPMV_TILE - 1)) == 0, "tile: power of two <= 2^16");
    __shared__ uint64_t key[SPMV_TILE];
    const int64_t base = (int64_t)blockIdx.x * SPMV_TILE;
    const int64_t rem  = U - base;
    const int     n    = rem < SPMV_TILE ? (int)rem : SPMV_TILE;
    for(int i = threadIdx.x; i < SPMV_TILE; i += RANK_THREADS)
        key[i] = i < n ? ((uint64_t)(uint32_t)cols[base + i] << 16) | (uint64_t)i : ~0ull;
    __syncthreads();
    for(int size = 2; size <= SPMV_TILE; size <<= 1)
        for(int stride = size >> 1; stride > 0; stride >>= 1)
        {
            for(int i = threadIdx.x; i < SPMV_TILE / 2; i += RANK_THREADS)
            {
                const int      lo = 2 * i - (i & (stride - 1));
                const int      hi = lo + stride;
                const bool     up = (lo & size) == 0;
                const uint64_t a = key[lo], b = key[hi];
                if((a > b) == up)
                {
                    key[lo] = b;
                    key[hi] = a;
                }
            }
            __syncthreads();
        }
    for(int i = threadIdx.x; i < n; i += RANK_THREADS)
        trank[base + (int64_t)(key[i] & 0xFFFFu)] = (uint16_t)i;
}

int asm_grid(int64_t work, int block)
{
    int64_t g = (work + block - 1) / block;
    const int64_t cap = (int64_t)NUM_SMS_HINT * 16;
    if(g > cap)
        g = cap;
    if(g < 1)
        g = 1;
    return (int)g;
}
}  // namespace

void assemble_triplets(b2s_solver* s, Matrix& M, int32_t nb, int64_t T, const int32_t* rows, const int32_t* cols,
                       const double* vals, bool spmv_tiles)
{
    B2S_REQUIRE(nb >= 0 && T >= 0, B2S_ERR_ARGUMENT, "negative matrix size");
    B2S_REQUIRE(T < (int64_t)INT32_MAX, B2S_ERR_ARGUMENT, "more than 2^31-1 triplets");
    cudaStream_t     st = s->stream;
    AssemblyScratch& w  = s->asmb;
    M.valid             = false;
    M.generation += 1;
    M.nb                = nb;
    w.err.resize(1);
    B2S_CUDA(cudaMemsetAsync(w.err.data(), 0, sizeof(int), st));
    w.row_count.resize((size_t)nb + 1, 1.25);
    w.row_start.resize((size_t)nb + 1, 1.25);
    w.row_fill.resize((size_t)nb + 1, 1.25);
    w.uniq_count.resize((size_t)nb + 1, 1.25);
    M.rowptr.resize((size_t)nb + 1, 1.25);
    M.diag_index.resize((size_t)std::max(nb, 1), 1.25);
    B2S_CUDA(cudaMemsetAsync(w.row_count.data(), 0, sizeof(int32_t) * ((size_t)nb + 1), st));
    B2S_CUDA(cudaMemsetAsync(w.row_fill.data(), 0, sizeof(int32_t) * ((size_t)nb + 1), st));
    if(T > 0)
    {
        w.bucket.resize(T, 1.25);
        w.sorted_col.resize(T, 1.25);
        w.sorted_src.resize(T, 1.25);
        k_count_rows<<<asm_grid(T, ASM_BLOCK), ASM_BLOCK, 0, st>>>(rows, cols, T, nb, w.row_count.data(),
                                                                   w.err.data());
        B2S_CHECK_LAUNCH();
    }
    exclusive_scan(s, w.row_count.data(), w.row_start.data(), nb, w.scan_tmp);
    if(T > 0)
    {
        k_scatter_rows<<<asm_grid(T, ASM_BLOCK), ASM_BLOCK, 0, st>>>(rows, cols, T, nb, w.row_start.data(),
                                                                     w.row_fill.data(), w.bucket.data(),
                                                                     w.err.data());
        B2S_CHECK_LAUNCH();
    }
    if(nb > 0)
    {
        w.long_rows.resize((size_t)nb + 1, 1.25);
        B2S_CUDA(cudaMemsetAsync(w.long_rows.data(), 0, sizeof(int32_t), st));
        k_sort_rows<<<asm_grid((int64_t)nb * 32, ASM_BLOCK), ASM_BLOCK, 0, st>>>(
            nb, w.row_start.data(), w.bucket.data(), w.sorted_col.data(),
            w.sorted_src.data(), w.uniq_count.data(), w.long_rows.data());
        B2S_CHECK_LAUNCH();
        // the long rows (count in long_rows[0], read on the device)
        k_sort_long_rows<<<NUM_SMS_HINT * 2, LONG_THREADS, 0, st>>>(w.long_rows.data(), w.row_start.data(),
                                                                    w.bucket.data(), w.sorted_col.data(),
                                                                    w.sorted_src.data(), w.uniq_count.data());
        B2S_CHECK_LAUNCH();
    }
    exclusive_scan(s, w.uniq_count.data(), M.rowptr.data(), nb, w.scan_tmp);
    int32_t U = 0;
    int     herr = 0;
    B2S_CUDA(cudaMemcpyAsync(&U, M.rowptr.data() + nb, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    B2S_CUDA(cudaMemcpyAsync(&herr, w.err.data(), sizeof(int), cudaMemcpyDeviceToHost, st));
    B2S_CUDA(cudaStreamSynchronize(st));
    B2S_REQUIRE(!(herr & DERR_TRIPLET_INDEX), B2S_ERR_ARGUMENT,
                "triplet column index outside [0, n_block_rows)");
    B2S_REQUIRE(!(herr & DERR_ROW_OVERFLOW), B2S_ERR_ARGUMENT,
                "triplet arrays changed during assembly (row bucket overflow)");
    M.nnz    = U;
    M.stride = ((std::max<int64_t>(U, 1) + 15) / 16) * 16;
    M.rows.resize(M.stride, 1.2);
    M.cols.resize(M.stride, 1.2);
    M.vals.resize((size_t)9 * M.stride, 1.2);
    // padding past U: row -1 / col 0 (never used: every reader checks k < U)
    B2S_CUDA(cudaMemsetAsync(M.rows.data() + U, 0xff, sizeof(int32_t) * (M.stride - U), st));
    B2S_CUDA(cudaMemsetAsync(M.cols.data() + U, 0, sizeof(int32_t) * (M.stride - U), st));
    if(nb > 0)
    {
        // slots of the runs, then their sums (values as planes with stride M.stride)
        w.run_start.resize((size_t)U + 1, 1.2);
        k_mark_runs<<<asm_grid((int64_t)nb * 32, ASM_BLOCK), ASM_BLOCK, 0, st>>>(
            nb, w.row_start.data(), w.sorted_col.data(), M.rowptr.data(), M.rows.data(), M.cols.data(),
            w.run_start.data(), M.diag_index.data());
        B2S_CHECK_LAUNCH();
        B2S_CUDA(cudaMemcpyAsync(w.run_start.data() + U, w.row_start.data() + nb, sizeof(int32_t),
                                 cudaMemcpyDeviceToDevice, st));
        if(U > 0)
        {
            // one pass in block order (no grid-stride loop): the CTAs in
            // flight cover neighbouring rows, whose sources share cache lines
            k_sum_runs<<<(unsigned)((3 * U + ASM_BLOCK - 1) / ASM_BLOCK), ASM_BLOCK, 0, st>>>(
                U, w.run_start.data(), w.sorted_src.data(), vals, M.vals.data(), M.stride);
            B2S_CHECK_LAUNCH();
        }
    }
    M.has_trank = false;
    if(spmv_tiles && U > 0)
    {
        M.trank.resize(M.stride, 1.2);
        k_tile_rank<<<(unsigned)((U + SPMV_TILE - 1) / SPMV_TILE), RANK_THREADS, 0, st>>>(U, M.cols.data(),
                                                                                     M.trank.data());
        B2S_CHECK_LAUNCH();
        M.has_trank = true;
    }
    M.valid = true;
}
}  // namespace b2s
