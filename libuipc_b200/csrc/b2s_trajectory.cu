// Candidate detection of the line search's trajectory filter on the GPU
// (include/b200gen.h: b2gen_trajectory_*): the point-triangle and edge-edge
// pairs of a surface whose swept boxes over the step come within dhat of each
// other -- what libuipc's simplex trajectory filter collects with its BVH
// before the narrow phase (collision_detection/filters/
// lbvh_simplex_trajectory_filter.cu:1100-1300 detect, :876-1010 filter_toi;
// the far test of utils/distance/details/ccd.inl: point_triangle_ccd_broadphase,
// edge_edge_ccd_broadphase) -- followed by the narrow phase (b2s_ccd.cuh) and
// the minimum time of impact.
//
// Design: a uniform grid hashed into a power-of-two bucket table instead of a
// BVH. Triangles (and, in their own table, edges) enter every cell their
// swept box covers; buckets are filled by a counting sort and each bucket is
// ordered by primitive id, so the output does not depend on the order atomics
// resolve in. A query walks the cells of its primitive's swept box grown by
// the far distance, tests every entry of each cell's bucket with the
// reference's far test, and emits a pair only from the first cell both
// primitives' cell ranges share (the lowest cell of their intersection, in
// integer cell coordinates), so a pair seen in several cells -- or through a
// hash collision -- comes out once. Two passes (count, scan, write) give every
// query a fixed output range: the pairs come out in query order, then cell
// order, then primitive id. Pairs that share a vertex are skipped.
#include "b2s_ccd.cuh"
#include "b2s_fixed_reduce.cuh"
#include "b2s_internal.cuh"

#include "../../include/b200gen.h"

#include <algorithm>
#include <cmath>
#include <string>

namespace
{
thread_local std::string g_traj_err;

constexpr int TRAJ_BLOCK = 128;
int           grid_of(int64_t n) { return (int)((n + TRAJ_BLOCK - 1) / TRAJ_BLOCK); }

struct Box
{
    double lo[3], hi[3];
};

// the swept box of NV vertices over x -> x + alpha dx
template <int NV>
__device__ __forceinline__ Box swept_box(const int32_t* v, const double* __restrict__ x, const double* __restrict__ dx,
                                         double alpha)
{
    Box b;
    for(int a = 0; a < 3; ++a)
    {
        b.lo[a] = 1e300;
        b.hi[a] = -1e300;
    }
    for(int k = 0; k < NV; ++k)
        for(int a = 0; a < 3; ++a)
        {
            const double p = x[3 * (int64_t)v[k] + a], q = p + alpha * dx[3 * (int64_t)v[k] + a];
            b.lo[a]        = fmin(b.lo[a], fmin(p, q));
            b.hi[a]        = fmax(b.hi[a], fmax(p, q));
        }
    return b;
}

// the reference's far test: apart by more than dist on some axis
__device__ __forceinline__ bool far_apart(const Box& a, const Box& b, double dist)
{
    for(int k = 0; k < 3; ++k)
        if(a.lo[k] - b.hi[k] > dist || b.lo[k] - a.hi[k] > dist)
            return true;
    return false;
}

__device__ __forceinline__ uint32_t bucket_of(int64_t ix, int64_t iy, int64_t iz, uint32_t mask)
{
    const uint64_t h = (uint64_t)(ix * 73856093ll) ^ (uint64_t)(iy * 19349663ll) ^ (uint64_t)(iz * 83492791ll);
    return (uint32_t)(h ^ (h >> 29)) & mask;
}

// cell ranges of a box (grown by g). A box that is not finite or spans more
// than CELL_CAP cells on an axis (a move of many cells in one step) gets an
// empty range and sets bit 0 of *err: the detection reports it instead of
// walking an unbounded range.
constexpr double CELL_CAP = 64.0;
__device__ __forceinline__ void cell_range(const Box& b, double g, double inv_cell, int64_t lo[3], int64_t hi[3],
                                           int* err)
{
    for(int a = 0; a < 3; ++a)
    {
        const double l = (b.lo[a] - g) * inv_cell, h = (b.hi[a] + g) * inv_cell;
        if(!(l > -1e15 && h < 1e15 && h - l < CELL_CAP))
        {
            for(int k = 0; k < 3; ++k)
            {
                lo[k] = 0;
                hi[k] = -1;
            }
            atomicOr(err, 1);
            return;
        }
        lo[a] = (int64_t)floor(l);
        hi[a] = (int64_t)floor(h);
    }
}

// swept boxes of the primitives (NV = 2 edges, 3 triangles) and their cell
// counts
template <int NV>
__global__ void k_prim_boxes(int32_t n, const int32_t* __restrict__ prim, const double* __restrict__ x,
                             const double* __restrict__ dx, double alpha, double inv_cell, Box* __restrict__ box,
                             int64_t* __restrict__ cnt, int* err)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n)
        return;
    const Box b = swept_box<NV>(prim + (int64_t)NV * i, x, dx, alpha);
    box[i]      = b;
    int64_t lo[3], hi[3];
    cell_range(b, 0.0, inv_cell, lo, hi, err);
    cnt[i] = (hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1);
}

// Exclusive scan of n int64 counts into off[0..n] (off[n] = the total), in
// three passes: per tile of SCAN_TILE elements its sum (coalesced loads, block
// reduction), the tile sums scanned by one CTA, each tile scanned in shared
// memory from its carry.
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_PER     = 8;
constexpr int SCAN_TILE    = SCAN_THREADS * SCAN_PER;

__device__ __forceinline__ int64_t block_exclusive(int64_t v, int64_t* sh, int64_t* total)
{
    // inclusive warp scan, then the warps' totals
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int64_t   inc  = v;
    for(int o = 1; o < 32; o <<= 1)
    {
        const int64_t u = __shfl_up_sync(0xffffffffu, inc, o);
        if(lane >= o)
            inc += u;
    }
    if(lane == 31)
        sh[w] = inc;
    __syncthreads();
    if(threadIdx.x == 0)
    {
        int64_t run = 0;
        for(int k = 0; k < SCAN_THREADS / 32; ++k)
        {
            const int64_t t = sh[k];
            sh[k]           = run;
            run += t;
        }
        sh[SCAN_THREADS / 32] = run;
    }
    __syncthreads();
    const int64_t ex = sh[w] + inc - v;
    *total           = sh[SCAN_THREADS / 32];
    __syncthreads();
    return ex;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_tile_sums(int64_t n, const int64_t* __restrict__ in,
                                                            int64_t* __restrict__ sums)
{
    __shared__ int64_t sh[SCAN_THREADS / 32 + 1];
    const int64_t      base = (int64_t)blockIdx.x * SCAN_TILE;
    int64_t            s    = 0;
    for(int k = 0; k < SCAN_PER; ++k)
    {
        const int64_t i = base + k * SCAN_THREADS + threadIdx.x;
        if(i < n)
            s += in[i];
    }
    int64_t total = 0;
    block_exclusive(s, sh, &total);
    if(threadIdx.x == 0)
        sums[blockIdx.x] = total;
}

// one CTA over the (few) tile sums: off[0..nt], off[nt] = total
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_sums(int64_t nt, const int64_t* __restrict__ sums,
                                                            int64_t* __restrict__ off)
{
    __shared__ int64_t sh[SCAN_THREADS / 32 + 1];
    int64_t            carry = 0;
    for(int64_t b = 0; b < nt; b += SCAN_THREADS)
    {
        const int64_t i = b + threadIdx.x;
        const int64_t v = i < nt ? sums[i] : 0;
        int64_t       total;
        const int64_t ex = block_exclusive(v, sh, &total);
        if(i < nt)
            off[i] = carry + ex;
        carry += total;
    }
    if(threadIdx.x == 0)
        off[nt] = carry;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_tile_scan(int64_t n, const int64_t* __restrict__ in,
                                                            const int64_t* __restrict__ tile_off,
                                                            int64_t* __restrict__ off)
{
    __shared__ int64_t tile[SCAN_TILE];
    __shared__ int64_t sh[SCAN_THREADS / 32 + 1];
    const int64_t      base = (int64_t)blockIdx.x * SCAN_TILE;
    for(int k = 0; k < SCAN_PER; ++k)
    {
        const int64_t i              = base + k * SCAN_THREADS + threadIdx.x;
        tile[k * SCAN_THREADS + threadIdx.x] = i < n ? in[i] : 0;
    }
    __syncthreads();
    // each thread its SCAN_PER consecutive elements, then across the threads
    int64_t s = 0;
    for(int k = 0; k < SCAN_PER; ++k)
        s += tile[threadIdx.x * SCAN_PER + k];
    int64_t       total;
    int64_t       run = tile_off[blockIdx.x] + block_exclusive(s, sh, &total);
    for(int k = 0; k < SCAN_PER; ++k)
    {
        const int64_t v                  = tile[threadIdx.x * SCAN_PER + k];
        tile[threadIdx.x * SCAN_PER + k] = run;
        run += v;
    }
    __syncthreads();
    for(int k = 0; k < SCAN_PER; ++k)
    {
        const int64_t i = base + k * SCAN_THREADS + threadIdx.x;
        if(i < n)
            off[i] = tile[k * SCAN_THREADS + threadIdx.x];
    }
    if(blockIdx.x == 0 && threadIdx.x == 0)
        off[n] = tile_off[gridDim.x];
}

// off[0..n] = exclusive scan of in[0..n), off[n] the total (tmp: scratch)
void scan_counts(int64_t n, const int64_t* in, int64_t* off, b2s::DBuf<int64_t>& tmp, cudaStream_t st)
{
    const int64_t nt = std::max<int64_t>((n + SCAN_TILE - 1) / SCAN_TILE, 1);
    tmp.resize(2 * (size_t)nt + 1);
    k_tile_sums<<<(unsigned)nt, SCAN_THREADS, 0, st>>>(n, in, tmp.data());
    B2S_CHECK_LAUNCH();
    k_scan_sums<<<1, SCAN_THREADS, 0, st>>>(nt, tmp.data(), tmp.data() + nt);
    B2S_CHECK_LAUNCH();
    k_tile_scan<<<(unsigned)nt, SCAN_THREADS, 0, st>>>(n, in, tmp.data() + nt, off);
    B2S_CHECK_LAUNCH();
}

// every (bucket, primitive) entry of the primitives' cells
__global__ void k_prim_fill(int32_t n, const Box* __restrict__ box, const int64_t* __restrict__ off, double inv_cell,
                            uint32_t mask, uint32_t* __restrict__ ent_bucket, int32_t* __restrict__ ent_id, int* err)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n)
        return;
    int64_t lo[3], hi[3];
    cell_range(box[i], 0.0, inv_cell, lo, hi, err);
    int64_t k = off[i];
    for(int64_t ix = lo[0]; ix <= hi[0]; ++ix)
        for(int64_t iy = lo[1]; iy <= hi[1]; ++iy)
            for(int64_t iz = lo[2]; iz <= hi[2]; ++iz)
            {
                ent_bucket[k] = bucket_of(ix, iy, iz, mask);
                ent_id[k]     = i;
                ++k;
            }
}

__global__ void k_bucket_count(int64_t E, const uint32_t* __restrict__ ent_bucket, int64_t* __restrict__ count)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(k < E)
        atomicAdd(reinterpret_cast<unsigned long long*>(count + ent_bucket[k]), 1ull);
}

__global__ void k_bucket_scatter(int64_t E, const uint32_t* __restrict__ ent_bucket, const int32_t* __restrict__ ent_id,
                                 int64_t* __restrict__ cursor, int32_t* __restrict__ sorted)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(k < E)
        sorted[atomicAdd(reinterpret_cast<unsigned long long*>(cursor + ent_bucket[k]), 1ull)] = ent_id[k];
}

// each bucket's primitives in id order (insertion sort; buckets are short),
// so queries see them in an order independent of the scatter's atomics
__global__ void k_bucket_order(int64_t H, const int64_t* __restrict__ start, int32_t* __restrict__ sorted)
{
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(b >= H)
        return;
    for(int64_t i = start[b] + 1; i < start[b + 1]; ++i)
    {
        const int32_t v = sorted[i];
        int64_t       j = i - 1;
        while(j >= start[b] && sorted[j] > v)
        {
            sorted[j + 1] = sorted[j];
            --j;
        }
        sorted[j + 1] = v;
    }
}

struct Grid
{
    const int64_t* start;   // [H + 1]
    const int32_t* sorted;  // primitive ids by bucket
    const Box*     box;     // per primitive
    uint32_t       mask;
    double         inv_cell;
    int*           err;
};

// One query primitive (NQ vertices qv) against the grid of NP-vertex
// primitives: every candidate not far apart (the reference's test at dist),
// not sharing a vertex, (edge-edge: only the larger id) found in the lowest
// cell of the two cell ranges' intersection. WRITE = false counts them,
// otherwise writes the 4 vertex ids (query's first) from out.
template <int NQ, int NP, bool WRITE>
__device__ int64_t query(int32_t self, const int32_t* qv, const Box& qb, const Grid& G, const int32_t* __restrict__ prim,
                         double dist, int64_t out, int32_t* __restrict__ pairs)
{
    // the query's cells, grown past the far distance by a margin well above
    // the rounding of a coordinate, so every pair the far test keeps shares a
    // cell range with its query
    int64_t qlo[3], qhi[3];
    cell_range(qb, dist * (1.0 + 1e-6) + 1e-9 / G.inv_cell, G.inv_cell, qlo, qhi, G.err);
    int64_t n = 0;
    for(int64_t ix = qlo[0]; ix <= qhi[0]; ++ix)
        for(int64_t iy = qlo[1]; iy <= qhi[1]; ++iy)
            for(int64_t iz = qlo[2]; iz <= qhi[2]; ++iz)
            {
                const uint32_t b = bucket_of(ix, iy, iz, G.mask);
                for(int64_t e = G.start[b]; e < G.start[b + 1]; ++e)
                {
                    const int32_t t = G.sorted[e];
                    // a primitive whose cells share this bucket appears once per
                    // such cell, next to itself (ids sorted): test it once
                    if(e > G.start[b] && G.sorted[e - 1] == t)
                        continue;
                    if(NQ == NP && t <= self)
                        continue;
                    const Box& pb = G.box[t];
                    int64_t    plo[3], phi[3];
                    cell_range(pb, 0.0, G.inv_cell, plo, phi, G.err);
                    // the pair's first shared cell must be this one
                    if(ix != max(qlo[0], plo[0]) || iy != max(qlo[1], plo[1]) || iz != max(qlo[2], plo[2]))
                        continue;
                    if(ix > phi[0] || iy > phi[1] || iz > phi[2])
                        continue;  // a hash collision: t is not in this cell
                    if(far_apart(qb, pb, dist))
                        continue;
                    const int32_t* pv     = prim + (int64_t)NP * t;
                    bool           shared = false;
                    for(int a = 0; a < NQ; ++a)
                        for(int c = 0; c < NP; ++c)
                            shared |= qv[a] == pv[c];
                    if(shared)
                        continue;
                    if(WRITE)
                    {
                        int32_t* o = pairs + 4 * (out + n);
                        for(int a = 0; a < NQ; ++a)
                            o[a] = qv[a];
                        for(int c = 0; c < NP; ++c)
                            o[NQ + c] = pv[c];
                    }
                    ++n;
                }
            }
    return n;
}

// point-triangle: one thread per surface vertex
template <bool WRITE>
__global__ void k_query_pt(int32_t nsv, const int32_t* __restrict__ sv, const double* __restrict__ x,
                           const double* __restrict__ dx, double alpha, double dist, Grid G,
                           const int32_t* __restrict__ tris, int64_t* __restrict__ cnt, const int64_t* __restrict__ off,
                           int32_t* __restrict__ pairs)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= nsv)
        return;
    const Box     qb = swept_box<1>(sv + i, x, dx, alpha);
    const int64_t n  = query<1, 3, WRITE>(-1, sv + i, qb, G, tris, dist, WRITE ? off[i] : 0, pairs);
    if(!WRITE)
        cnt[i] = n;
}

// edge-edge: one thread per surface edge, partners of larger id
template <bool WRITE>
__global__ void k_query_ee(int32_t nse, const int32_t* __restrict__ se, double dist, Grid G,
                           int64_t* __restrict__ cnt, const int64_t* __restrict__ off, int32_t* __restrict__ pairs)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= nse)
        return;
    const int64_t n = query<2, 2, WRITE>(i, se + 2 * (int64_t)i, G.box[i], G, se, dist, WRITE ? off[i] : 0, pairs);
    if(!WRITE)
        cnt[i] = n;
}

__global__ void k_fill_u8(int64_t n, uint8_t v, uint8_t* __restrict__ out)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(k < n)
        out[k] = v;
}

void fail(const char* msg) { throw b2s::Error(B2S_ERR_ARGUMENT, msg); }

template <typename F>
int guarded(F&& f)
{
    try
    {
        f();
        return 0;
    }
    catch(const b2s::Error& e)
    {
        g_traj_err = e.what();
        return e.code;
    }
    catch(const std::exception& e)
    {
        g_traj_err = e.what();
        return B2S_ERR_CUDA;
    }
}

uint32_t pow2_at_least(int64_t n)
{
    uint64_t h = 1024;
    while((int64_t)h < n && h < (1ull << 30))
        h <<= 1;
    return (uint32_t)h;
}
}  // namespace

struct b2gen_trajectory
{
    int32_t                  nsv = 0, nse = 0, nst = 0;
    b2s::DBuf<int32_t>       sv, se, st;
    double                   dhat = 0.0, cell = 0.0;
    int                      device = 0;
    // per detection
    b2s::DBuf<Box>           tbox, ebox;
    b2s::DBuf<int64_t>       cnt, off, off_pt, off_ee, bstart, cursor, scan_tmp;
    b2s::DBuf<uint32_t>      ent_bucket;
    b2s::DBuf<int32_t>       ent_id, tsorted, esorted;
    b2s::DBuf<int64_t>       tstart, estart;
    b2s::DBuf<int32_t>       pairs;  // [n_pt + n_ee][4]: point-triangle pairs, then edge-edge
    b2s::DBuf<uint8_t>       is_ee;
    b2s::DBuf<double>        terms, result;
    b2s::DBuf<int>           err;  // bit 0: a box beyond the grid's range (see cell_range)
    int64_t                  n_pt = 0, n_ee = 0;
};

namespace
{
// the grid of n primitives (boxes already in `box`): entries, bucket counting
// sort, buckets in id order; start [H + 1] and sorted ids out
void build_grid(b2gen_trajectory* T, int32_t n, b2s::DBuf<Box>& box, b2s::DBuf<int64_t>& start,
                b2s::DBuf<int32_t>& sorted, uint32_t& mask, cudaStream_t st)
{
    // cell counts were written by k_prim_boxes into T->cnt
    T->off.resize((size_t)n + 1);
    scan_counts(n, T->cnt.data(), T->off.data(), T->scan_tmp, st);
    int64_t E = 0;
    B2S_CUDA(cudaMemcpyAsync(&E, T->off.data() + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    B2S_CUDA(cudaStreamSynchronize(st));
    const uint32_t H = pow2_at_least(2 * std::max<int64_t>(E, 1));
    mask             = H - 1;
    T->ent_bucket.resize((size_t)std::max<int64_t>(E, 1));
    T->ent_id.resize((size_t)std::max<int64_t>(E, 1));
    sorted.resize((size_t)std::max<int64_t>(E, 1));
    start.resize((size_t)H + 1);
    T->cursor.resize((size_t)H + 1);
    T->bstart.resize((size_t)H);
    const double inv_cell = 1.0 / T->cell;
    if(n > 0)
    {
        k_prim_fill<<<grid_of(n), TRAJ_BLOCK, 0, st>>>(n, box.data(), T->off.data(), inv_cell, mask,
                                                       T->ent_bucket.data(), T->ent_id.data(), T->err.data());
        B2S_CHECK_LAUNCH();
    }
    B2S_CUDA(cudaMemsetAsync(T->bstart.data(), 0, sizeof(int64_t) * H, st));
    if(E > 0)
    {
        k_bucket_count<<<grid_of(E), TRAJ_BLOCK, 0, st>>>(E, T->ent_bucket.data(), T->bstart.data());
        B2S_CHECK_LAUNCH();
    }
    scan_counts(H, T->bstart.data(), start.data(), T->scan_tmp, st);
    B2S_CUDA(cudaMemcpyAsync(T->cursor.data(), start.data(), sizeof(int64_t) * H, cudaMemcpyDeviceToDevice, st));
    if(E > 0)
    {
        k_bucket_scatter<<<grid_of(E), TRAJ_BLOCK, 0, st>>>(E, T->ent_bucket.data(), T->ent_id.data(),
                                                            T->cursor.data(), sorted.data());
        B2S_CHECK_LAUNCH();
    }
    k_bucket_order<<<grid_of(H), TRAJ_BLOCK, 0, st>>>(H, start.data(), sorted.data());
    B2S_CHECK_LAUNCH();
}

// both candidate lists for the move alpha dx from x into T->pairs / T->is_ee
// (point-triangle pairs first): grids, counting passes, then writing passes
void detect(b2gen_trajectory* T, const double* d_x, const double* d_dx, double alpha, cudaStream_t st)
{
    const double inv_cell = 1.0 / T->cell;
    const double dist     = T->dhat;
    int64_t      tot[2]   = {0, 0};
    const bool   pt = T->nsv > 0 && T->nst > 0, ee = T->nse > 1;
    Grid         Gt{}, Ge{};
    T->cnt.resize((size_t)std::max({T->nst, T->nsv, T->nse}) + 1);
    T->err.resize(1);
    B2S_CUDA(cudaMemsetAsync(T->err.data(), 0, sizeof(int), st));
    if(pt)
    {
        T->tbox.resize(T->nst);
        k_prim_boxes<3><<<grid_of(T->nst), TRAJ_BLOCK, 0, st>>>(T->nst, T->st.data(), d_x, d_dx, alpha, inv_cell,
                                                                 T->tbox.data(), T->cnt.data(), T->err.data());
        B2S_CHECK_LAUNCH();
        uint32_t mask = 0;
        build_grid(T, T->nst, T->tbox, T->tstart, T->tsorted, mask, st);
        Gt = Grid{T->tstart.data(), T->tsorted.data(), T->tbox.data(), mask, inv_cell, T->err.data()};
        k_query_pt<false><<<grid_of(T->nsv), TRAJ_BLOCK, 0, st>>>(T->nsv, T->sv.data(), d_x, d_dx, alpha, dist, Gt,
                                                                   T->st.data(), T->cnt.data(), nullptr, nullptr);
        B2S_CHECK_LAUNCH();
        T->off_pt.resize((size_t)T->nsv + 1);
        scan_counts(T->nsv, T->cnt.data(), T->off_pt.data(), T->scan_tmp, st);
        B2S_CUDA(cudaMemcpyAsync(&tot[0], T->off_pt.data() + T->nsv, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    }
    if(ee)
    {
        T->ebox.resize(T->nse);
        k_prim_boxes<2><<<grid_of(T->nse), TRAJ_BLOCK, 0, st>>>(T->nse, T->se.data(), d_x, d_dx, alpha, inv_cell,
                                                                 T->ebox.data(), T->cnt.data(), T->err.data());
        B2S_CHECK_LAUNCH();
        uint32_t mask = 0;
        build_grid(T, T->nse, T->ebox, T->estart, T->esorted, mask, st);
        Ge = Grid{T->estart.data(), T->esorted.data(), T->ebox.data(), mask, inv_cell, T->err.data()};
        k_query_ee<false><<<grid_of(T->nse), TRAJ_BLOCK, 0, st>>>(T->nse, T->se.data(), dist, Ge, T->cnt.data(),
                                                                   nullptr, nullptr);
        B2S_CHECK_LAUNCH();
        T->off_ee.resize((size_t)T->nse + 1);
        scan_counts(T->nse, T->cnt.data(), T->off_ee.data(), T->scan_tmp, st);
        B2S_CUDA(cudaMemcpyAsync(&tot[1], T->off_ee.data() + T->nse, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    }
    int err = 0;
    B2S_CUDA(cudaMemcpyAsync(&err, T->err.data(), sizeof(int), cudaMemcpyDeviceToHost, st));
    B2S_CUDA(cudaStreamSynchronize(st));
    if(err)
        fail("trajectory detection: a swept box spans more than 64 grid cells on an axis or is not finite "
             "(positions, step or cell size)");
    T->n_pt         = tot[0];
    T->n_ee         = tot[1];
    const int64_t np = tot[0] + tot[1];
    T->pairs.resize(4 * (size_t)std::max<int64_t>(np, 1), 1.5);
    T->is_ee.resize((size_t)std::max<int64_t>(np, 1), 1.5);
    if(tot[0] > 0)
    {
        k_query_pt<true><<<grid_of(T->nsv), TRAJ_BLOCK, 0, st>>>(T->nsv, T->sv.data(), d_x, d_dx, alpha, dist, Gt,
                                                                  T->st.data(), nullptr, T->off_pt.data(),
                                                                  T->pairs.data());
        B2S_CHECK_LAUNCH();
        k_fill_u8<<<grid_of(tot[0]), TRAJ_BLOCK, 0, st>>>(tot[0], 0, T->is_ee.data());
        B2S_CHECK_LAUNCH();
    }
    if(tot[1] > 0)
    {
        k_query_ee<true><<<grid_of(T->nse), TRAJ_BLOCK, 0, st>>>(T->nse, T->se.data(), dist, Ge, nullptr,
                                                                  T->off_ee.data(), T->pairs.data() + 4 * tot[0]);
        B2S_CHECK_LAUNCH();
        k_fill_u8<<<grid_of(tot[1]), TRAJ_BLOCK, 0, st>>>(tot[1], 1, T->is_ee.data() + tot[0]);
        B2S_CHECK_LAUNCH();
    }
}
}  // namespace

extern "C" {

const char* b2gen_trajectory_last_error(void) { return g_traj_err.c_str(); }

int b2gen_trajectory_create(int device, int32_t n_verts, int32_t n_surf_verts, const int32_t* surf_verts,
                            int32_t n_surf_edges, const int32_t* surf_edges, int32_t n_surf_tris,
                            const int32_t* surf_tris, double dhat, double cell, b2gen_trajectory** out)
{
    return guarded(
        [&]
        {
            if(!out || n_verts <= 0 || n_surf_verts < 0 || n_surf_edges < 0 || n_surf_tris < 0 || !(dhat > 0.0) ||
               !(cell > 0.0))
                fail("b2gen_trajectory_create: bad arguments");
            if((n_surf_verts && !surf_verts) || (n_surf_edges && !surf_edges) || (n_surf_tris && !surf_tris))
                fail("b2gen_trajectory_create: null primitive list");
            auto check = [&](const int32_t* v, int64_t n)
            {
                for(int64_t i = 0; i < n; ++i)
                    if(v[i] < 0 || v[i] >= n_verts)
                        fail("b2gen_trajectory_create: vertex index out of range");
            };
            check(surf_verts, n_surf_verts);
            check(surf_edges, 2ll * n_surf_edges);
            check(surf_tris, 3ll * n_surf_tris);
            B2S_CUDA(cudaSetDevice(device));
            auto T    = new b2gen_trajectory();
            T->device = device;
            T->nsv    = n_surf_verts;
            T->nse    = n_surf_edges;
            T->nst    = n_surf_tris;
            T->dhat   = dhat;
            T->cell   = cell;
            T->sv.resize(std::max(n_surf_verts, 1));
            T->se.resize(2 * (size_t)std::max(n_surf_edges, 1));
            T->st.resize(3 * (size_t)std::max(n_surf_tris, 1));
            if(n_surf_verts)
                B2S_CUDA(cudaMemcpy(T->sv.data(), surf_verts, sizeof(int32_t) * n_surf_verts, cudaMemcpyHostToDevice));
            if(n_surf_edges)
                B2S_CUDA(cudaMemcpy(T->se.data(), surf_edges, sizeof(int32_t) * 2 * n_surf_edges,
                                    cudaMemcpyHostToDevice));
            if(n_surf_tris)
                B2S_CUDA(cudaMemcpy(T->st.data(), surf_tris, sizeof(int32_t) * 3 * n_surf_tris,
                                    cudaMemcpyHostToDevice));
            *out = T;
        });
}

int b2gen_trajectory_destroy(b2gen_trajectory* t)
{
    delete t;
    return 0;
}

int b2gen_trajectory_detect(b2gen_trajectory* t, const double* d_x, const double* d_dx, double alpha,
                            int64_t* h_counts, void* stream)
{
    return guarded(
        [&]
        {
            if(!t || !d_x || !d_dx || !h_counts || !(alpha >= 0.0))
                fail("b2gen_trajectory_detect: bad arguments");
            B2S_CUDA(cudaSetDevice(t->device));
            cudaStream_t st = static_cast<cudaStream_t>(stream);
            detect(t, d_x, d_dx, alpha, st);
            B2S_CUDA(cudaStreamSynchronize(st));
            h_counts[0] = t->n_pt;
            h_counts[1] = t->n_ee;
        });
}

int b2gen_trajectory_pairs(b2gen_trajectory* t, int32_t* h_pairs, uint8_t* h_is_ee)
{
    return guarded(
        [&]
        {
            if(!t || !h_pairs || !h_is_ee)
                fail("b2gen_trajectory_pairs: null argument");
            B2S_CUDA(cudaSetDevice(t->device));
            const int64_t np = t->n_pt + t->n_ee;
            if(np > 0)
            {
                B2S_CUDA(cudaMemcpy(h_pairs, t->pairs.data(), sizeof(int32_t) * 4 * np, cudaMemcpyDeviceToHost));
                B2S_CUDA(cudaMemcpy(h_is_ee, t->is_ee.data(), (size_t)np, cudaMemcpyDeviceToHost));
            }
        });
}

int b2gen_trajectory_toi(b2gen_trajectory* t, const double* d_x, const double* d_dx, double alpha, double* h_toi,
                         void* stream)
{
    return guarded(
        [&]
        {
            if(!t || !d_x || !d_dx || !h_toi || !(alpha > 0.0))
                fail("b2gen_trajectory_toi: bad arguments");
            B2S_CUDA(cudaSetDevice(t->device));
            cudaStream_t st = static_cast<cudaStream_t>(stream);
            detect(t, d_x, d_dx, alpha, st);
            const int64_t np = t->n_pt + t->n_ee;
            double        toi = b2s::TOI_NONE;
            if(np > 0)
            {
                t->terms.resize((size_t)np);
                t->result.resize(1);
                b2s::k_contact_toi<<<grid_of(np), TRAJ_BLOCK, 0, st>>>(np, t->pairs.data(), t->is_ee.data(), d_x, d_dx,
                                                                       alpha, t->dhat, 0.0, b2s::CCD_ETA,
                                                                       b2s::CCD_MAX_ITER, t->terms.data());
                B2S_CHECK_LAUNCH();
                b2s::k_fixed_reduce<<<1, b2s::SUM_THREADS, 0, st>>>(np, t->terms.data(), 1, t->result.data());
                B2S_CHECK_LAUNCH();
                B2S_CUDA(cudaMemcpyAsync(&toi, t->result.data(), sizeof(double), cudaMemcpyDeviceToHost, st));
            }
            B2S_CUDA(cudaStreamSynchronize(st));
            *h_toi = toi < 1.0 ? toi : 1.0;
        });
}

}  // extern "C"
