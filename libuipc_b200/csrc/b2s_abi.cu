// C ABI of libb200solve (include/b200solve.h): argument checks, error
// capture, and dispatch into the solver. No exception crosses the ABI.
#include "b2s_internal.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

namespace
{
thread_local std::string g_create_error;
}

namespace b2s
{
thread_local long long g_kernel_launches = 0;

void set_handle_free_error(const std::string& msg) { g_create_error = msg; }
}  // namespace b2s

namespace
{

template <typename F>
int guarded(b2s_solver* s, F&& f)
{
    if(!s)
        return B2S_ERR_ARGUMENT;
    const long long launches_before = b2s::g_kernel_launches;
    try
    {
        int dev = -1;
        if(cudaGetDevice(&dev) != cudaSuccess || dev != s->device)
            B2S_CUDA(cudaSetDevice(s->device));
        f();
        s->timers.kernel_launches += b2s::g_kernel_launches - launches_before;
        s->last_error.clear();
        return B2S_OK;
    }
    catch(const b2s::Error& e)
    {
        s->timers.kernel_launches += b2s::g_kernel_launches - launches_before;
        s->last_error = e.what();
        return e.code;
    }
    catch(const std::exception& e)
    {
        s->last_error = e.what();
        return B2S_ERR_STATE;
    }
}

// bracket a stage with CUDA events on the solver's stream when timing is on
template <typename F>
void timed_stage(b2s_solver* s, double b2s_timers::*field, F&& f)
{
    if(!s->timing)
    {
        f();
        return;
    }
    B2S_CUDA(cudaEventRecord(s->ev_begin, s->stream));
    f();
    B2S_CUDA(cudaEventRecord(s->ev_end, s->stream));
    B2S_CUDA(cudaEventSynchronize(s->ev_end));
    float ms = 0.f;
    B2S_CUDA(cudaEventElapsedTime(&ms, s->ev_begin, s->ev_end));
    s->timers.*field += ms;
}
}  // namespace

extern "C" {

int b2s_version(void) { return 1; }

int b2s_create(int device, b2s_solver** out)
{
    if(!out)
        return B2S_ERR_ARGUMENT;
    *out = nullptr;
    try
    {
        int count = 0;
        B2S_CUDA(cudaGetDeviceCount(&count));
        B2S_REQUIRE(device >= 0 && device < count, B2S_ERR_ARGUMENT, "no such CUDA device");
        cudaDeviceProp prop{};
        B2S_CUDA(cudaGetDeviceProperties(&prop, device));
        B2S_REQUIRE(prop.major >= 10, B2S_ERR_ARGUMENT,
                    "libb200solve is built for sm_100a (Blackwell B200); device is sm_" + std::to_string(prop.major)
                        + std::to_string(prop.minor));
        B2S_CUDA(cudaSetDevice(device));
        auto* s   = new b2s_solver;
        s->device = device;
        cudaError_t e = cudaStreamCreateWithFlags(&s->own_stream, cudaStreamNonBlocking);
        if(e != cudaSuccess)
        {
            delete s;
            throw b2s::Error(B2S_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
        }
        s->stream = s->own_stream;
        *out      = s;
        return B2S_OK;
    }
    catch(const b2s::Error& e)
    {
        g_create_error = e.what();
        return e.code;
    }
    catch(const std::exception& e)
    {
        g_create_error = e.what();
        return B2S_ERR_STATE;
    }
}

int b2s_destroy(b2s_solver* s)
{
    if(!s)
        return B2S_OK;
    cudaSetDevice(s->device);
    cudaStreamSynchronize(s->stream);
    b2s::drop_graphs(s);
    if(s->pcg.h_sc)
        cudaFreeHost(s->pcg.h_sc);
    if(s->ev_begin)
        cudaEventDestroy(s->ev_begin);
    if(s->ev_end)
        cudaEventDestroy(s->ev_end);
    for(cudaEvent_t e : s->iter_events)
        cudaEventDestroy(e);
    b2s::ws_free(s->ws);
    if(s->mas_fork)
        cudaEventDestroy(s->mas_fork);
    if(s->mas_join)
        cudaEventDestroy(s->mas_join);
    if(s->mas_side)
        cudaStreamDestroy(s->mas_side);
    if(s->own_stream)
        cudaStreamDestroy(s->own_stream);
    delete s;
    return B2S_OK;
}

const char* b2s_last_error(const b2s_solver* s) { return s ? s->last_error.c_str() : g_create_error.c_str(); }

int b2s_set_stream(b2s_solver* s, void* stream)
{
    return guarded(s,
                   [&]
                   {
                       B2S_CUDA(cudaStreamSynchronize(s->stream));
                       s->stream = stream ? (cudaStream_t)stream : s->own_stream;
                       b2s::drop_graphs(s);
                   });
}

int b2s_assemble(b2s_solver* s, int32_t nb, int64_t T, const int32_t* rows, const int32_t* cols, const double* vals)
{
    return guarded(s,
                   [&]
                   {
                       B2S_REQUIRE(nb >= 0 && T >= 0, B2S_ERR_ARGUMENT, "negative size");
                       B2S_REQUIRE(T == 0 || (rows && cols && vals), B2S_ERR_ARGUMENT, "null triplet array");
                       B2S_REQUIRE(nb <= INT32_MAX / 3, B2S_ERR_ARGUMENT, "too many block rows");
                       timed_stage(s, &b2s_timers::assemble_ms,
                                   [&] { b2s::assemble_triplets(s, s->A, nb, T, rows, cols, vals, true); });
                       s->precond_kind = -1;  // any preconditioner must be rebuilt
                       B2S_CUDA(cudaStreamSynchronize(s->stream));
                   });
}

int b2s_triplet_buffers(b2s_solver* s, int64_t T, int32_t** d_rows, int32_t** d_cols, double** d_vals)
{
    return guarded(s,
                   [&]
                   {
                       B2S_REQUIRE(T >= 0, B2S_ERR_ARGUMENT, "negative triplet count");
                       B2S_REQUIRE(d_rows && d_cols && d_vals, B2S_ERR_ARGUMENT, "null output pointer");
                       B2S_CUDA(cudaSetDevice(s->device));
                       const size_t n = (size_t)std::max<int64_t>(T, 1);
                       s->own_rows.resize(n, 1.1);
                       s->own_cols.resize(n, 1.1);
                       s->own_vals.resize(9 * n, 1.1);
                       *d_rows = s->own_rows.data();
                       *d_cols = s->own_cols.data();
                       *d_vals = s->own_vals.data();
                   });
}

int b2s_assemble_owned(b2s_solver* s, int32_t nb, int64_t T)
{
    if(!s)
        return B2S_ERR_ARGUMENT;
    if(T > (int64_t)s->own_rows.size() || (T > 0 && s->own_vals.size() < 9 * (size_t)T))
    {
        s->last_error = "b2s_assemble_owned: more triplets than b2s_triplet_buffers provided";
        return B2S_ERR_ARGUMENT;
    }
    return b2s_assemble(s, nb, T, s->own_rows.data(), s->own_cols.data(), s->own_vals.data());
}

int b2s_matrix_info(const b2s_solver* s, int32_t* nb, int64_t* nnz)
{
    if(!s)
        return B2S_ERR_ARGUMENT;
    if(nb)
        *nb = s->A.valid ? s->A.nb : 0;
    if(nnz)
        *nnz = s->A.valid ? s->A.nnz : 0;
    return B2S_OK;
}

int b2s_get_upper_bsr(b2s_solver* s, int32_t* rowptr, int32_t* colidx, double* vals)
{
    return guarded(s,
                   [&]
                   {
                       B2S_REQUIRE(s->A.valid, B2S_ERR_STATE, "no assembled matrix");
                       const b2s::Matrix& A = s->A;
                       cudaStream_t st = s->stream;
                       if(rowptr)
                           B2S_CUDA(cudaMemcpyAsync(rowptr, A.rowptr.data(), sizeof(int32_t) * (A.nb + 1),
                                                    cudaMemcpyDefault, st));
                       if(colidx && A.nnz)
                           B2S_CUDA(cudaMemcpyAsync(colidx, A.cols.data(), sizeof(int32_t) * A.nnz,
                                                    cudaMemcpyDefault, st));
                       if(vals && A.nnz)
                       {
                           // planes -> column-major blocks: one strided copy per component
                           for(int q = 0; q < 9; ++q)
                               B2S_CUDA(cudaMemcpy2DAsync(vals + q, 9 * sizeof(double), A.vals.data() + (size_t)q * A.stride,
                                                          sizeof(double), sizeof(double), A.nnz, cudaMemcpyDefault, st));
                       }
                       B2S_CUDA(cudaStreamSynchronize(st));
                   });
}

int b2s_spmv(b2s_solver* s, const double* x, double* y, double* h_dot)
{
    return guarded(s,
                   [&]
                   {
                       B2S_REQUIRE(s->A.valid, B2S_ERR_STATE, "no assembled matrix");
                       B2S_REQUIRE(x && y, B2S_ERR_ARGUMENT, "null vector");
                       s->dot_out.resize(4);
                       b2s::spmv_f64(s, s->A, x, y, h_dot ? s->dot_out.data() : nullptr);
                       b2s::check_device_errors(s);
                       if(h_dot)
                           B2S_CUDA(cudaMemcpyAsync(h_dot, s->dot_out.data(), sizeof(double), cudaMemcpyDeviceToHost,
                                                    s->stream));
                       B2S_CUDA(cudaStreamSynchronize(s->stream));
                   });
}

int b2s_spmv_mixed(b2s_solver* s, const float* x, float* y, double* h_dot)
{
    return guarded(s,
                   [&]
                   {
                       B2S_REQUIRE(s->A.valid, B2S_ERR_STATE, "no assembled matrix");
                       B2S_REQUIRE(x && y, B2S_ERR_ARGUMENT, "null vector");
                       s->dot_out.resize(4);
                       b2s::spmv_mixed(s, x, y, s->dot_out.data());
                       if(h_dot)
                           B2S_CUDA(cudaMemcpyAsync(h_dot, s->dot_out.data(), sizeof(double), cudaMemcpyDeviceToHost,
                                                    s->stream));
                       B2S_CUDA(cudaStreamSynchronize(s->stream));
                   });
}

int b2s_spmv_mixed_timing(b2s_solver* s, int32_t launches, double* h_avg_ms)
{
    return guarded(s,
                   [&]
                   {
                       B2S_REQUIRE(s->A.valid, B2S_ERR_STATE, "no assembled matrix");
                       B2S_REQUIRE(h_avg_ms, B2S_ERR_ARGUMENT, "null output");
                       *h_avg_ms = b2s::spmv_mixed_timing(s, launches);
                   });
}

int b2s_mas_init(b2s_solver* s, int32_t off, int32_t vn, const int32_t* adj_start, const int32_t* adj_list,
                 int32_t N, const int32_t* p2r, const int32_t* r2p)
{
    return guarded(s,
                   [&]
                   {
                       B2S_REQUIRE(adj_start && p2r && r2p, B2S_ERR_ARGUMENT, "null MAS input");
                       B2S_REQUIRE(adj_list || adj_start[vn] == 0, B2S_ERR_ARGUMENT, "null adjacency list");
                       b2s::mas_init(s, off, vn, adj_start, adj_list, N, p2r, r2p);
                       s->precond_kind = -1;
                   });
}

int b2s_mas_info(const b2s_solver* s, int32_t* L, int32_t* total)
{
    if(!s)
        return B2S_ERR_ARGUMENT;
    if(L)
        *L = s->mas.initialized ? s->mas.L : 0;
    if(total)
        *total = s->mas.initialized ? s->mas.total : 0;
    return B2S_OK;
}

int b2s_mas_get_hierarchy(b2s_solver* s, int32_t* level_begin, int32_t* level_count, int32_t* coarse_table)
{
    return guarded(s,
                   [&]
                   {
                       const b2s::MasState& M = s->mas;
                       B2S_REQUIRE(M.initialized, B2S_ERR_STATE, "MAS not initialised");
                       for(int l = 0; l <= M.L; ++l)
                       {
                           if(level_begin)
                               level_begin[l] = M.level_begin[l];
                           if(level_count)
                               level_count[l] = M.level_count[l];
                       }
                       if(coarse_table && !M.h_ctable.empty() && M.L > 1)
                           std::memcpy(coarse_table, M.h_ctable.data(), sizeof(int32_t) * (size_t)M.vn * (M.L - 1));
                   });
}

int b2s_mas_get_clusters(b2s_solver* s, double* hess, float* inv)
{
    return guarded(s,
                   [&]
                   {
                       const b2s::MasState& M = s->mas;
                       B2S_REQUIRE(M.initialized, B2S_ERR_STATE, "MAS not initialised");
                       if(hess)
                           B2S_CUDA(cudaMemcpy(hess, M.hess.data(), M.hess.bytes(), cudaMemcpyDeviceToHost));
                       if(inv)
                           B2S_CUDA(cudaMemcpy(inv, M.inv.data(), M.inv.bytes(), cudaMemcpyDeviceToHost));
                   });
}

int b2s_mas_stiff_info(b2s_solver* s, int32_t* n_stiff, uint8_t* h_flags)
{
    return guarded(s,
                   [&]
                   {
                       const b2s::MasState& M = s->mas;
                       B2S_REQUIRE(M.initialized, B2S_ERR_STATE, "MAS not initialised");
                       B2S_REQUIRE(M.stiff_count.size() == 1, B2S_ERR_STATE, "no MAS build yet");
                       B2S_CUDA(cudaStreamSynchronize(s->stream));
                       if(n_stiff)
                           B2S_CUDA(cudaMemcpy(n_stiff, M.stiff_count.data(), sizeof(int32_t),
                                               cudaMemcpyDeviceToHost));
                       if(h_flags && M.clusters > 0)
                           B2S_CUDA(cudaMemcpy(h_flags, M.stiff.data(), (size_t)M.clusters, cudaMemcpyDeviceToHost));
                   });
}

int b2s_mas_get_nodes(b2s_solver* s, float* R, float* Z)
{
    return guarded(s,
                   [&]
                   {
                       const b2s::MasState& M = s->mas;
                       B2S_REQUIRE(M.initialized, B2S_ERR_STATE, "MAS not initialised");
                       B2S_CUDA(cudaStreamSynchronize(s->stream));
                       if(R)
                           B2S_CUDA(cudaMemcpy(R, M.R.data(), sizeof(float) * 3 * (size_t)M.total,
                                               cudaMemcpyDeviceToHost));
                       if(Z)
                           B2S_CUDA(cudaMemcpy(Z, M.Z.data(), sizeof(float) * 3 * (size_t)M.total,
                                               cudaMemcpyDeviceToHost));
                   });
}

int b2s_abd_init(b2s_solver* s, int32_t block_offset, int32_t n_bodies)
{
    return guarded(s,
                   [&]
                   {
                       B2S_REQUIRE(block_offset >= 0 && n_bodies >= 0, B2S_ERR_ARGUMENT, "negative affine-body range");
                       B2S_REQUIRE((int64_t)block_offset + 4 * (int64_t)n_bodies <= INT32_MAX / 3, B2S_ERR_ARGUMENT,
                                   "affine-body range too large");
                       if(s->mas.initialized && n_bodies > 0)
                       {
                           const int64_t a0 = block_offset, a1 = a0 + 4 * (int64_t)n_bodies;
                           const int64_t m0 = s->mas.offset, m1 = m0 + s->mas.vn;
                           B2S_REQUIRE(a1 <= m0 || m1 <= a0, B2S_ERR_ARGUMENT,
                                       "affine-body range overlaps the MAS range");
                       }
                       s->abd_offset   = block_offset;
                       s->abd_n        = n_bodies;
                       s->precond_kind = -1;  // rebuild before the next apply
                       b2s::drop_graphs(s);
                   });
}

int b2s_precond_assemble(b2s_solver* s, int kind, int invert_mode)
{
    return guarded(s, [&]
                   { timed_stage(s, &b2s_timers::precond_build_ms, [&] { b2s::precond_assemble(s, kind, invert_mode); }); });
}

int b2s_precond_apply(b2s_solver* s, const double* r, double* z)
{
    return guarded(s,
                   [&]
                   {
                       B2S_REQUIRE(r && z, B2S_ERR_ARGUMENT, "null vector");
                       b2s::precond_apply(s, r, z);
                   });
}

int b2s_precond_apply_mixed(b2s_solver* s, const float* r, float* z)
{
    return guarded(s,
                   [&]
                   {
                       B2S_REQUIRE(r && z, B2S_ERR_ARGUMENT, "null vector");
                       b2s::precond_apply_mixed(s, r, z);
                   });
}

void b2s_pcg_default_options(b2s_pcg_options* o)
{
    if(!o)
        return;
    std::memset(o, 0, sizeof(*o));
    o->tol            = 1e-3;  // linear_system/tol_rate default (scene_default_config.cpp:146-175)
    o->stop_rule      = B2S_STOP_RZ;
    o->check_interval = 5;
    o->max_iter       = 0;
    o->precision      = B2S_PRECISION_FP64;
    o->use_graph      = 1;
    o->x0_given       = 0;
    o->replace_every  = 0;
}

int b2s_pcg(b2s_solver* s, const double* b, double* x, const b2s_pcg_options* opt, b2s_pcg_stats* stats)
{
    b2s_pcg_stats local{};
    int rc = guarded(s,
                     [&]
                     {
                         B2S_REQUIRE(b && x, B2S_ERR_ARGUMENT, "null vector");
                         b2s_pcg_options o;
                         if(opt)
                             o = *opt;
                         else
                             b2s_pcg_default_options(&o);
                         timed_stage(s, &b2s_timers::pcg_ms, [&] { b2s::pcg_solve(s, b, x, o, local); });
                     });
    if(stats)
        *stats = local;
    return rc;
}

int b2s_set_timing(b2s_solver* s, int enable)
{
    return guarded(s,
                   [&]
                   {
                       if(enable && !s->ev_begin)
                       {
                           B2S_CUDA(cudaEventCreate(&s->ev_begin));
                           B2S_CUDA(cudaEventCreate(&s->ev_end));
                       }
                       s->timing = enable != 0;
                       // the captured graphs carry (or lack) the event nodes
                       b2s::drop_graphs(s);
                   });
}

int b2s_get_timers(const b2s_solver* s, b2s_timers* out)
{
    if(!s || !out)
        return B2S_ERR_ARGUMENT;
    *out = s->timers;
    return B2S_OK;
}

int b2s_reset_timers(b2s_solver* s)
{
    if(!s)
        return B2S_ERR_ARGUMENT;
    s->timers = b2s_timers{};
    return B2S_OK;
}

// ---------------------------------------------------------------------------
// partition utilities (host)
// ---------------------------------------------------------------------------
int b2s_partition_rcb(int32_t n, const double* pos, int32_t max_part, int32_t* part_ids)
{
    if(n < 0 || (n > 0 && (!pos || !part_ids)) || max_part < 1)
        return B2S_ERR_ARGUMENT;
    if(n == 0)
        return B2S_OK;
    std::vector<int32_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    struct Range
    {
        int32_t lo, hi;
    };
    // depth-first with an explicit stack, left part first: part ids follow a
    // space-filling order so consecutive parts are neighbours
    std::vector<Range> stack{{0, n}};
    int32_t            next_part = 0;
    while(!stack.empty())
    {
        Range r = stack.back();
        stack.pop_back();
        const int32_t m = r.hi - r.lo;
        if(m <= max_part)
        {
            for(int32_t k = r.lo; k < r.hi; ++k)
                part_ids[idx[k]] = next_part;
            ++next_part;
            continue;
        }
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for(int32_t k = r.lo; k < r.hi; ++k)
            for(int a = 0; a < 3; ++a)
            {
                const double v = pos[(size_t)idx[k] * 3 + a];
                lo[a]          = std::min(lo[a], v);
                hi[a]          = std::max(hi[a], v);
            }
        int axis = 0;
        for(int a = 1; a < 3; ++a)
            if(hi[a] - lo[a] > hi[axis] - lo[axis])
                axis = a;
        // left part: half the vertices rounded to whole parts
        int32_t parts_total = (m + max_part - 1) / max_part;
        int32_t left        = ((parts_total + 1) / 2) * max_part;
        if(left >= m)
            left = m - 1;
        auto less = [&](int32_t a, int32_t b)
        {
            const double va = pos[(size_t)a * 3 + axis], vb = pos[(size_t)b * 3 + axis];
            return va < vb || (va == vb && a < b);
        };
        std::nth_element(idx.begin() + r.lo, idx.begin() + r.lo + left, idx.begin() + r.hi, less);
        stack.push_back({r.lo + left, r.hi});  // right processed after left
        stack.push_back({r.lo, r.lo + left});
    }
    return B2S_OK;
}

// geometry::mesh_partition (src/geometry/mesh_partition.cpp:77-231) from the
// vertex adjacency alone: point clouds (no edges) take sequential blocks of
// max_part; up to max_part vertices take one part per connected component
// (the reference's n_parts <= 1 branch); otherwise recursive graph bisection
// into ceil(n / max_part) parts.
int b2s_partition_graph(int32_t n, const int32_t* adj_start, const int32_t* adj_list, int32_t max_part,
                        int32_t* part_ids)
{
    if(n < 0 || max_part < 1 || (n > 0 && (!adj_start || !part_ids)))
        return B2S_ERR_ARGUMENT;
    if(n == 0)
        return B2S_OK;
    if(adj_start[0] != 0)
        return B2S_ERR_ARGUMENT;
    for(int32_t v = 0; v < n; ++v)
        if(adj_start[v + 1] < adj_start[v])
            return B2S_ERR_ARGUMENT;
    const int32_t E = adj_start[n];
    if(E > 0 && !adj_list)
        return B2S_ERR_ARGUMENT;
    for(int32_t e = 0; e < E; ++e)
        if(adj_list[e] < 0 || adj_list[e] >= n)
            return B2S_ERR_ARGUMENT;
    if(E == 0)
    {
        for(int32_t v = 0; v < n; ++v)
            part_ids[v] = v / max_part;
        return B2S_OK;
    }
    if(n <= max_part)
    {
        std::fill(part_ids, part_ids + n, -1);
        std::vector<int32_t> queue;
        int32_t              comp = 0;
        for(int32_t v0 = 0; v0 < n; ++v0)
        {
            if(part_ids[v0] >= 0)
                continue;
            queue.assign(1, v0);
            part_ids[v0] = comp;
            for(size_t h = 0; h < queue.size(); ++h)
                for(int32_t e = adj_start[queue[h]]; e < adj_start[queue[h] + 1]; ++e)
                    if(part_ids[adj_list[e]] < 0)
                    {
                        part_ids[adj_list[e]] = comp;
                        queue.push_back(adj_list[e]);
                    }
            ++comp;
        }
        return B2S_OK;
    }
    try
    {
        b2s::partition_graph(n, adj_start, adj_list, max_part, part_ids);
    }
    catch(const std::exception& e)
    {
        b2s::set_handle_free_error(e.what());
        return B2S_ERR_STATE;
    }
    return B2S_OK;
}

// FEMMASPreconditioner::do_init step 4 (fem_mas_preconditioner.cu:285-330):
// vertices grouped by part id (parts in id order, vertices ascending), each
// part padded to a multiple of 16 slots
int b2s_partition_maps(int32_t n, const int32_t* part_ids, int32_t max_part, int32_t* p2r, int32_t* r2p,
                       int32_t* map_size)
{
    if(n < 0 || !r2p || !map_size || (n > 0 && !part_ids) || max_part < 1 || max_part > b2s::BANK)
        return B2S_ERR_ARGUMENT;
    int32_t max_id = -1;
    for(int32_t v = 0; v < n; ++v)
        max_id = std::max(max_id, part_ids[v]);
    std::vector<int32_t> count(max_id + 2, 0);
    for(int32_t v = 0; v < n; ++v)
        if(part_ids[v] >= 0)
            if(++count[part_ids[v]] > max_part)
                return B2S_ERR_ARGUMENT;
    std::vector<int32_t> start(max_id + 2, 0);
    int32_t              total = 0;
    for(int32_t p = 0; p <= max_id; ++p)
    {
        start[p] = total;
        total += (count[p] + b2s::BANK - 1) / b2s::BANK * b2s::BANK;
    }
    *map_size = total;
    if(!p2r)
        return B2S_OK;  // size query
    std::fill(p2r, p2r + total, -1);
    std::vector<int32_t> fill(max_id + 2, 0);
    for(int32_t v = 0; v < n; ++v)
    {
        const int32_t p = part_ids[v];
        if(p < 0)
        {
            r2p[v] = -1;
            continue;
        }
        const int32_t slot = start[p] + fill[p]++;
        p2r[slot]          = v;
        r2p[v]             = slot;
    }
    return B2S_OK;
}

// ---- learned warm start -------------------------------------------------------------
int b2s_ws_init(b2s_solver* s, int32_t hidden, uint64_t seed)
{
    return guarded(s, [&] { b2s::ws_init(s, hidden, seed); });
}

int b2s_ws_add_sample(b2s_solver* s, const double* d_b, int32_t n_hist, const double* const* d_hist,
                      const double* d_x)
{
    return guarded(s, [&] { b2s::ws_add_sample(s, d_b, n_hist, d_hist, d_x); });
}

int b2s_ws_put_sample(b2s_solver* s, int32_t rows, const float* feat, const float* H, const float* q,
                      const float* c0, double norm)
{
    return guarded(s, [&] { b2s::ws_put_sample(s, rows, feat, H, q, c0, norm); });
}

int b2s_ws_num_samples(const b2s_solver* s, int32_t* n_samples, int64_t* n_rows)
{
    b2s_solver* m = const_cast<b2s_solver*>(s);
    return guarded(m, [&] { b2s::ws_num_samples(m, n_samples, n_rows); });
}

int b2s_ws_fit_normalization(b2s_solver* s)
{
    return guarded(s, [&] { b2s::ws_fit_normalization(s); });
}

int b2s_ws_train(b2s_solver* s, int32_t epochs, double lr, uint64_t seed, double* h_mean_loss)
{
    return guarded(s,
                   [&]
                   {
                       const double l = b2s::ws_train(s, epochs, lr, seed);
                       if(h_mean_loss)
                           *h_mean_loss = l;
                   });
}

int b2s_ws_loss_grad(b2s_solver* s, int32_t index, double* h_loss, float* h_grad)
{
    return guarded(s,
                   [&]
                   {
                       const double l = b2s::ws_loss_grad(s, index, h_grad);
                       if(h_loss)
                           *h_loss = l;
                   });
}

int b2s_ws_get_params(const b2s_solver* s, float* h_params, int64_t* n)
{
    b2s_solver* m = const_cast<b2s_solver*>(s);
    return guarded(m,
                   [&]
                   {
                       B2S_REQUIRE(n, B2S_ERR_ARGUMENT, "null size");
                       *n = b2s::ws_get_params(m, h_params);
                   });
}

int b2s_ws_set_params(b2s_solver* s, const float* h_params, int64_t n)
{
    return guarded(s, [&] { b2s::ws_set_params(s, h_params, n); });
}

int b2s_ws_get_sample(const b2s_solver* s, int32_t index, int32_t* rows, float* h_feat, float* h_H, float* h_q,
                      float* h_c0, double* h_norm)
{
    b2s_solver* m = const_cast<b2s_solver*>(s);
    return guarded(m,
                   [&]
                   {
                       const int r = b2s::ws_get_sample(m, index, h_feat, h_H, h_q, h_c0, h_norm);
                       if(rows)
                           *rows = r;
                   });
}

int b2s_ws_predict(b2s_solver* s, int32_t mode, const double* d_b, int32_t n_hist, const double* const* d_hist,
                   double* d_x0, b2s_ws_info* info)
{
    return guarded(s, [&] { b2s::ws_predict(s, mode, d_b, n_hist, d_hist, d_x0, info); });
}

}  // extern "C"
