// CPU oracle -- TEST INFRASTRUCTURE ONLY (see oracle.h for the parity status).
//
// Every function restates the libuipc CUDA backend's algorithm on the
// Newton-step linear-solve path, with the source lines it follows cited
// (paths relative to the libuipc source tree). Sums run in a fixed,
// documented order so that the product's deterministic kernels can be
// compared bit-exactly where they use the same order.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace
{
constexpr int BANK = 16;                    // MASPreconditionerEngine::BANKSIZE
constexpr int SYM  = BANK * (BANK + 1) / 2;  // 136 upper blocks per cluster
constexpr int MAX_LEVELS = 6;

inline int bank_align(int n) { return (n + BANK - 1) / BANK * BANK; }
// mas_preconditioner_engine.cu:36-39
inline int sym_index(int row, int col) { return BANK * row - row * (row + 1) / 2 + col; }
}  // namespace

struct orc_matrix
{
    int32_t              nb = 0;
    std::vector<int32_t> rowptr, rows, cols;
    std::vector<double>  vals;  // U x 9 column-major
    // full (both triangles) CSR for the threaded CPU baseline, built lazily
    mutable std::vector<int32_t> f_rowptr, f_cols;
    mutable std::vector<double>  f_vals;  // row-major 3x3 per block
    mutable bool                 full_ready = false;
};

extern "C" {

// matrix_converter.inl:1550-1701 (convert_sym): keep row >= 0 && row <= col
// (k1 :129-144), key = row * cols + col (k2 :146-176), stable radix sort of
// (key, source index) (:1610-1616), run-length unique (:1627), segmented sum
// of the blocks of each run in sorted = source order (:1660-1700). The sum is
// sequential left to right (v[s0] + v[s1] + ...).
orc_matrix* orc_assemble(int32_t nb, int64_t T, const int32_t* rows, const int32_t* cols, const double* vals)
{
    auto* m = new orc_matrix;
    m->nb   = nb;
    std::vector<int64_t> src;
    src.reserve(T);
    for(int64_t i = 0; i < T; ++i)
        if(rows[i] >= 0 && rows[i] <= cols[i])
            src.push_back(i);
    const uint64_t C = (uint64_t)(nb > 0 ? nb : 1);
    std::vector<uint64_t> key(src.size());
    for(size_t k = 0; k < src.size(); ++k)
        key[k] = (uint64_t)rows[src[k]] * C + (uint64_t)cols[src[k]];
    std::vector<int64_t> order(src.size());
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return key[a] < key[b]; });
    m->rowptr.assign(nb + 1, 0);
    size_t k = 0;
    while(k < order.size())
    {
        size_t e = k;
        while(e < order.size() && key[order[e]] == key[order[k]])
            ++e;
        const int64_t s0 = src[order[k]];
        m->rows.push_back(rows[s0]);
        m->cols.push_back(cols[s0]);
        double acc[9];
        for(int q = 0; q < 9; ++q)
            acc[q] = vals[s0 * 9 + q];
        for(size_t t = k + 1; t < e; ++t)
        {
            const int64_t s = src[order[t]];
            for(int q = 0; q < 9; ++q)
                acc[q] += vals[s * 9 + q];
        }
        for(int q = 0; q < 9; ++q)
            m->vals.push_back(acc[q]);
        k = e;
    }
    // _calculate_block_offsets (:1058-1097): rowptr = exclusive scan of per-row counts
    for(size_t u = 0; u < m->rows.size(); ++u)
        m->rowptr[m->rows[u] + 1]++;
    for(int32_t r = 0; r < nb; ++r)
        m->rowptr[r + 1] += m->rowptr[r];
    return m;
}

void    orc_matrix_free(orc_matrix* m) { delete m; }
int64_t orc_matrix_nnz(const orc_matrix* m) { return (int64_t)m->rows.size(); }
int32_t orc_matrix_rows(const orc_matrix* m) { return m->nb; }

void orc_matrix_copy(const orc_matrix* m, int32_t* rowptr, int32_t* rows, int32_t* cols, double* vals)
{
    if(rowptr)
        std::memcpy(rowptr, m->rowptr.data(), sizeof(int32_t) * m->rowptr.size());
    if(rows)
        std::memcpy(rows, m->rows.data(), sizeof(int32_t) * m->rows.size());
    if(cols)
        std::memcpy(cols, m->cols.data(), sizeof(int32_t) * m->cols.size());
    if(vals)
        std::memcpy(vals, m->vals.data(), sizeof(double) * m->vals.size());
}

}  // extern "C"

namespace
{
// block y_i += B x_j (B column-major)
inline void bmv(const double* B, const double* x, double* y)
{
    y[0] += B[0] * x[0] + B[3] * x[1] + B[6] * x[2];
    y[1] += B[1] * x[0] + B[4] * x[1] + B[7] * x[2];
    y[2] += B[2] * x[0] + B[5] * x[1] + B[8] * x[2];
}
inline void bmtv(const double* B, const double* x, double* y)
{
    y[0] += B[0] * x[0] + B[1] * x[1] + B[2] * x[2];
    y[1] += B[3] * x[0] + B[4] * x[1] + B[5] * x[2];
    y[2] += B[6] * x[0] + B[7] * x[1] + B[8] * x[2];
}

void build_full(const orc_matrix* m)
{
    if(m->full_ready)
        return;
    const int32_t nb = m->nb;
    std::vector<int32_t> cnt(nb + 1, 0);
    for(size_t u = 0; u < m->rows.size(); ++u)
    {
        cnt[m->rows[u] + 1]++;
        if(m->rows[u] != m->cols[u])
            cnt[m->cols[u] + 1]++;
    }
    for(int32_t r = 0; r < nb; ++r)
        cnt[r + 1] += cnt[r];
    m->f_rowptr = cnt;
    m->f_cols.resize(cnt[nb]);
    m->f_vals.resize((size_t)cnt[nb] * 9);
    std::vector<int32_t> fill(cnt.begin(), cnt.end() - 1);
    for(size_t u = 0; u < m->rows.size(); ++u)
    {
        const int32_t i = m->rows[u], j = m->cols[u];
        const double* B = &m->vals[u * 9];
        int32_t s = fill[i]++;
        m->f_cols[s] = j;
        for(int p = 0; p < 3; ++p)
            for(int q = 0; q < 3; ++q)
                m->f_vals[(size_t)s * 9 + p * 3 + q] = B[q * 3 + p];
        if(i != j)
        {
            s = fill[j]++;
            m->f_cols[s] = i;
            for(int p = 0; p < 3; ++p)
                for(int q = 0; q < 3; ++q)
                    m->f_vals[(size_t)s * 9 + p * 3 + q] = B[p * 3 + q];
        }
    }
    m->full_ready = true;
}

// y = A x, threaded over rows of the full matrix (CPU baseline path)
void spmv_full(const orc_matrix* m, const double* x, double* y)
{
    build_full(m);
    const int32_t nb = m->nb;
#pragma omp parallel for schedule(static)
    for(int32_t i = 0; i < nb; ++i)
    {
        double acc[3] = {0, 0, 0};
        for(int32_t s = m->f_rowptr[i]; s < m->f_rowptr[i + 1]; ++s)
        {
            const double* B  = &m->f_vals[(size_t)s * 9];
            const double* xj = &x[(size_t)m->f_cols[s] * 3];
            acc[0] += B[0] * xj[0] + B[1] * xj[1] + B[2] * xj[2];
            acc[1] += B[3] * xj[0] + B[4] * xj[1] + B[5] * xj[2];
            acc[2] += B[6] * xj[0] + B[7] * xj[1] + B[8] * xj[2];
        }
        y[(size_t)i * 3 + 0] = acc[0];
        y[(size_t)i * 3 + 1] = acc[1];
        y[(size_t)i * 3 + 2] = acc[2];
    }
}

// y = A x, sequential symmetric form (Spmv::cpu_sym_spmv semantics)
void spmv_sym(const orc_matrix* m, const double* x, double* y)
{
    const size_t n = (size_t)m->nb * 3;
    std::fill(y, y + n, 0.0);
    for(size_t u = 0; u < m->rows.size(); ++u)
    {
        const int32_t i = m->rows[u], j = m->cols[u];
        const double* B = &m->vals[u * 9];
        bmv(B, &x[(size_t)j * 3], &y[(size_t)i * 3]);
        if(i != j)
            bmtv(B, &x[(size_t)i * 3], &y[(size_t)j * 3]);
    }
}
}  // namespace

extern "C" void orc_spmv(const orc_matrix* m, double a, const double* x, double b, double* y)
{
    const size_t        n = (size_t)m->nb * 3;
    std::vector<double> t(n);
    spmv_sym(m, x, t.data());
    for(size_t i = 0; i < n; ++i)
        y[i] = a * t[i] + (b == 0.0 ? 0.0 : b * y[i]);
}

// ---------------------------------------------------------------------------
// MAS
// ---------------------------------------------------------------------------
struct orc_mas
{
    int32_t vn = 0, N = 0, L = 0, total = 0;
    std::vector<int32_t> p2r, r2p;
    std::vector<int32_t> level_begin, level_count;
    std::vector<int32_t> going_next;   // level-0 slots indexed by real vertex
    std::vector<int32_t> ctable;       // [vn * (L-1)] global node at levels 1..L-1
    std::vector<double>  hess;         // [clusters * 136 * 9]
    std::vector<float>   inv;          // [clusters * 136 * 9]
    int32_t              clusters = 0;
};

namespace
{
// compute_num_levels, mas_preconditioner_engine.cu:1958-1972
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

// connected components of a bank: mask[lane] = direct adjacency (incl. self);
// closure as in prepare_prefix_sum_L0 (:108-156) / next_level_cluster (:296-338);
// returns per-lane rank of its component, components ordered by lowest lane
// (build_level1 :158-212, prefix_sum_Lx :340-388). `valid` marks lanes that exist.
int bank_components(const unsigned* mask, const bool* valid, int* rank)
{
    unsigned closure[BANK];
    for(int l = 0; l < BANK; ++l)
    {
        if(!valid[l])
            continue;
        unsigned m = mask[l], visited = 1u << l;
        while(true)
        {
            unsigned todo = visited ^ m;
            if(!todo)
                break;
            int nv = __builtin_ctz(todo);
            visited |= 1u << nv;
            m |= mask[nv];
        }
        closure[l] = m;
    }
    unsigned elected = 0;
    for(int l = 0; l < BANK; ++l)
        if(valid[l] && (closure[l] & ((1u << l) - 1u)) == 0)
            elected |= 1u << l;
    for(int l = 0; l < BANK; ++l)
        if(valid[l])
        {
            int el  = __builtin_ctz(closure[l]);
            rank[l] = __builtin_popcount(elected & ((1u << el) - 1u));
        }
    return __builtin_popcount(elected);
}
}  // namespace

extern "C" {

// FEMMASPreconditioner::do_init -> MASPreconditionerEngine::init_neighbor /
// init_matrix / reorder_realtime (mas_preconditioner_engine.cu:1974-2117) and
// the hierarchy kernels (:57-494).
orc_mas* orc_mas_create(int32_t vn, const int32_t* adj_start, const int32_t* adj_list, int32_t N,
                        const int32_t* p2r, const int32_t* r2p)
{
    auto* s = new orc_mas;
    s->vn   = vn;
    s->N    = N;
    s->p2r.assign(p2r, p2r + N);
    s->r2p.assign(r2p, r2p + vn);
    const int max_nodes = std::max(N, vn);
    s->L                = compute_num_levels(max_nodes);
    const int L         = s->L;
    s->level_begin.assign(L + 2, 0);
    s->level_count.assign(L + 2, 0);
    // mutable neighbour lists
    std::vector<std::vector<int32_t>> nbr(vn);
    for(int v = 0; v < vn; ++v)
        nbr[v].assign(adj_list + adj_start[v], adj_list + adj_start[v + 1]);

    std::vector<int32_t> cst((size_t)vn * L, -1);  // coarse_space_tables: local id at level l+1
    s->going_next.assign(bank_align(max_nodes) * 2 + 64, -1);
    auto gn_set = [&](size_t idx, int32_t val)
    {
        if(idx >= s->going_next.size())
            s->going_next.resize(idx * 2 + 64, -1);
        s->going_next[idx] = val;
    };

    // ---- level 0 -> 1 (build_connect_mask_L0 :57-106, prepare_prefix_sum_L0, build_level1)
    const int n_banks0 = (N + BANK - 1) / BANK;
    std::vector<unsigned> mask0(vn, 0);
    for(int p = 0; p < N; ++p)
    {
        int v = p2r[p];
        if(v < 0)
            continue;
        unsigned m  = 1u << (p % BANK);
        auto&    nl = nbr[v];
        std::vector<int32_t> keep;
        for(int32_t u : nl)
        {
            int pu = r2p[u];
            if(pu < 0)
                continue;  // dropped from the list
            if(pu / BANK == p / BANK)
                m |= 1u << (pu % BANK);
            else
                keep.push_back(u);
        }
        nl.swap(keep);
        mask0[v] = m;
    }
    std::vector<int> comps0(n_banks0), rank0(N, 0);
    for(int b = 0; b < n_banks0; ++b)
    {
        unsigned msk[BANK] = {0};
        bool     valid[BANK] = {false};
        int      rk[BANK];
        for(int l = 0; l < BANK; ++l)
        {
            int p = b * BANK + l;
            if(p < N && p2r[p] >= 0)
            {
                valid[l] = true;
                msk[l]   = mask0[p2r[p]];
            }
        }
        comps0[b] = bank_components(msk, valid, rk);
        for(int l = 0; l < BANK; ++l)
            if(valid[l])
                rank0[b * BANK + l] = rk[l];
    }
    std::vector<int> pre0(n_banks0 + 1, 0);
    for(int b = 0; b < n_banks0; ++b)
        pre0[b + 1] = pre0[b] + comps0[b];
    const int level1_begin = bank_align(std::max(bank_align(N), vn));
    for(int p = 0; p < N; ++p)
    {
        int v = p2r[p];
        if(v < 0)
            continue;
        int local = pre0[p / BANK] + rank0[p];
        cst[(size_t)0 * vn + v] = local;
        gn_set(v, local + level1_begin);
    }
    s->level_begin[0] = 0;
    s->level_count[0] = N;
    s->level_begin[1] = level1_begin;
    s->level_count[1] = pre0[n_banks0];

    // ---- levels 1 .. L-1 (build_connect_mask_Lx :214-294, next_level_cluster,
    // prefix_sum_Lx, compute_next_level :390-409)
    for(int level = 1; level < L; ++level)
    {
        const int cnt = s->level_count[level], beg = s->level_begin[level];
        std::vector<unsigned> next_mask(std::max(cnt, 1), 0u);
        for(int p = 0; p < N; ++p)
        {
            int v = p2r[p];
            if(v < 0)
                continue;
            int c = cst[(size_t)(level - 1) * vn + v];
            if(c < 0 || c >= N)
                continue;
            unsigned conn = 0;
            auto&    nl   = nbr[v];
            std::vector<int32_t> keep;
            for(int32_t u : nl)
            {
                int cu = cst[(size_t)(level - 1) * vn + u];
                if(cu < 0 || cu >= N)
                {
                    keep.push_back(u);
                    continue;
                }
                if(c / BANK == cu / BANK)
                    conn |= 1u << (cu % BANK);
                else
                    keep.push_back(u);
            }
            nl.swap(keep);
            next_mask[c] |= conn;
        }
        const int n_banks = (cnt + BANK - 1) / BANK;
        std::vector<int> comps(n_banks), rank(std::max(cnt, 1), 0);
        for(int b = 0; b < n_banks; ++b)
        {
            unsigned msk[BANK] = {0};
            bool     valid[BANK] = {false};
            int      rk[BANK];
            for(int l = 0; l < BANK; ++l)
            {
                int c = b * BANK + l;
                if(c < cnt)
                {
                    valid[l] = true;
                    msk[l]   = (1u << l) | next_mask[c];
                }
            }
            comps[b] = bank_components(msk, valid, rk);
            for(int l = 0; l < BANK; ++l)
                if(valid[l])
                    rank[b * BANK + l] = rk[l];
        }
        std::vector<int> pre(n_banks + 1, 0);
        for(int b = 0; b < n_banks; ++b)
            pre[b + 1] = pre[b] + comps[b];
        const int next_begin = beg + bank_align(cnt);
        std::vector<int> newid(std::max(cnt, 1), -1);
        for(int c = 0; c < cnt; ++c)
        {
            newid[c] = pre[c / BANK] + rank[c];
            gn_set((size_t)beg + c, newid[c] + next_begin);
        }
        s->level_begin[level + 1] = next_begin;
        s->level_count[level + 1] = pre[n_banks];
        for(int v = 0; v < vn; ++v)
        {
            int prev = cst[(size_t)(level - 1) * vn + v];
            cst[(size_t)level * vn + v] = (prev < 0 || prev >= vn) ? -1 : newid[prev];
        }
    }
    s->total    = s->level_begin[L];
    s->clusters = s->total / BANK;
    // aggregation_kernel (:411-460)
    s->ctable.assign((size_t)vn * std::max(L - 1, 1), -1);
    for(int v = 0; v < vn; ++v)
    {
        int first = s->going_next[v];
        if(first < 0)
            continue;
        int cur = first;
        s->ctable[(size_t)v * (L - 1) + 0] = cur;
        for(int l = 1; l < L - 1; ++l)
        {
            cur = s->going_next[cur];
            s->ctable[(size_t)v * (L - 1) + l] = cur;
        }
    }
    s->going_next.resize(std::max<size_t>(s->going_next.size(), (size_t)s->total), -1);
    return s;
}

void    orc_mas_free(orc_mas* s) { delete s; }
int32_t orc_mas_level_num(const orc_mas* s) { return s->L; }
int32_t orc_mas_total_nodes(const orc_mas* s) { return s->total; }

void orc_mas_levels(const orc_mas* s, int32_t* level_begin, int32_t* level_count)
{
    for(int l = 0; l <= s->L; ++l)
    {
        if(level_begin)
            level_begin[l] = s->level_begin[l];
        if(level_count)
            level_count[l] = s->level_count[l];
    }
}

void orc_mas_hierarchy(const orc_mas* s, int32_t* going_next, int32_t* coarse_table)
{
    if(going_next)
        for(int i = 0; i < s->total; ++i)
            going_next[i] = i < (int)s->going_next.size() ? s->going_next[i] : -1;
    if(coarse_table)
        std::memcpy(coarse_table, s->ctable.data(), sizeof(int32_t) * s->ctable.size());
}

}  // extern "C"

namespace
{
// cluster-local 3x3 add: dst (column-major) += B or B^T or B + B^T
inline void add_block(double* dst, const double* B, int mode)
{
    for(int i = 0; i < 3; ++i)
        for(int j = 0; j < 3; ++j)
        {
            double v = mode == 0 ? B[j * 3 + i] : mode == 1 ? B[i * 3 + j] : B[j * 3 + i] + B[i * 3 + j];
            dst[j * 3 + i] += v;
        }
}

// invert_cluster_matrices_sweep_kernel (:1077-1175): FP32 symmetric sweep,
// no pivoting, zero diagonal -> 1, stores -(-A^{-1}) upper blocks.
void invert_sweep_f32(const double* H, float* out)
{
    constexpr int D = BANK * 3;
    static thread_local float c[D][D];  // c[col][row]
    for(int col = 0; col < D; ++col)
    {
        const int a = col % 3, nc = col / 3;
        for(int row = 0; row < D; ++row)
        {
            const int node_row = row / 3;
            float     v;
            if(nc >= node_row)
                v = (float)H[sym_index(node_row, nc) * 9 + a * 3 + (row % 3)];
            else
                v = (float)H[sym_index(nc, node_row) * 9 + (row % 3) * 3 + a];
            if(row == col && v == 0.0f)
                v = 1.0f;
            c[col][row] = v;
        }
    }
    float sr[D];
    for(int p = 0; p < D; ++p)
    {
        for(int col = 0; col < D; ++col)
            sr[col] = c[col][p];
        const float akk = sr[p];
        for(int col = 0; col < D; ++col)
        {
            const float f = sr[col];
            float       nv;
            if(col == p)
            {
                const float inv = 1.0f / akk;
                for(int i = 0; i < D; ++i)
                    c[col][i] *= inv;
                nv = -inv;
            }
            else
            {
                const float s = f / akk;
                for(int i = 0; i < D; ++i)
                    c[col][i] = std::fmaf(-sr[i], s, c[col][i]);
                nv = s;
            }
            c[col][p] = nv;
        }
    }
    for(int i = 0; i < SYM * 9; ++i)
        out[i] = 0.0f;
    for(int col = 0; col < D; ++col)
    {
        const int a = col % 3, nc = col / 3;
        for(int row = 0; row < D; ++row)
        {
            const int   node_row = row / 3, b = row % 3;
            const float v        = -c[col][row];
            if(node_row < nc)
                out[sym_index(node_row, nc) * 9 + a * 3 + b] = v;
            else if(node_row == nc)
            {
                const int si = sym_index(nc, nc);
                if(b <= a)
                    out[si * 9 + a * 3 + b] = v;
                if(b < a)
                    out[si * 9 + b * 3 + a] = v;
            }
        }
    }
}

// FP64 Gauss-Jordan (same sweep, double), stored as FP32
void invert_sweep_f64(const double* H, float* out)
{
    constexpr int D = BANK * 3;
    static thread_local double c[D][D];
    for(int col = 0; col < D; ++col)
    {
        const int a = col % 3, nc = col / 3;
        for(int row = 0; row < D; ++row)
        {
            const int node_row = row / 3;
            double    v = (nc >= node_row) ? H[sym_index(node_row, nc) * 9 + a * 3 + (row % 3)]
                                           : H[sym_index(nc, node_row) * 9 + (row % 3) * 3 + a];
            if(row == col && v == 0.0)
                v = 1.0;
            c[col][row] = v;
        }
    }
    double sr[D];
    for(int p = 0; p < D; ++p)
    {
        for(int col = 0; col < D; ++col)
            sr[col] = c[col][p];
        const double akk = sr[p];
        for(int col = 0; col < D; ++col)
        {
            const double f = sr[col];
            double       nv;
            if(col == p)
            {
                const double inv = 1.0 / akk;
                for(int i = 0; i < D; ++i)
                    c[col][i] *= inv;
                nv = -inv;
            }
            else
            {
                const double s = f / akk;
                for(int i = 0; i < D; ++i)
                    c[col][i] = std::fma(-sr[i], s, c[col][i]);
                nv = s;
            }
            c[col][p] = nv;
        }
    }
    for(int i = 0; i < SYM * 9; ++i)
        out[i] = 0.0f;
    for(int col = 0; col < D; ++col)
    {
        const int a = col % 3, nc = col / 3;
        for(int row = 0; row < D; ++row)
        {
            const int   node_row = row / 3, b = row % 3;
            const float v        = (float)(-c[col][row]);
            if(node_row < nc)
                out[sym_index(node_row, nc) * 9 + a * 3 + b] = v;
            else if(node_row == nc)
            {
                const int si = sym_index(nc, nc);
                if(b <= a)
                    out[si * 9 + a * 3 + b] = v;
                if(b < a)
                    out[si * 9 + b * 3 + a] = v;
            }
        }
    }
}
}  // namespace

extern "C" {

// set_preconditioner (:2281-2458): Galerkin cluster matrices at every level.
// Block (i, j) of the upper BCOO contributes, at every level l where the
// level-l nodes of i and j share a bank, B (or B^T when their order flips) at
// their (lane, lane) slot, and B + B^T when both map to one coarse node
// (scatter k1 :530-683 for cross-bank pairs, k2 :801-953 for pairs inside a
// level-0 bank). Blocks in the same level-0 bank land once at level 0.
int orc_mas_assemble(orc_mas* s, const orc_matrix* A, int32_t off, int invert_mode)
{
    const int L = s->L;
    s->hess.assign((size_t)s->clusters * SYM * 9, 0.0);
    auto node_at = [&](int v, int l) -> int
    { return l == 0 ? s->r2p[v] : s->ctable[(size_t)v * (L - 1) + (l - 1)]; };
    for(size_t u = 0; u < A->rows.size(); ++u)
    {
        const int i = A->rows[u] - off, j = A->cols[u] - off;
        if(i < 0 || i >= s->vn || j < 0 || j >= s->vn)
            continue;
        if(s->r2p[i] < 0 || s->r2p[j] < 0)
            continue;
        const double* B = &A->vals[u * 9];
        for(int l = 0; l < L; ++l)
        {
            const int ci = node_at(i, l), cj = node_at(j, l);
            if(ci < 0 || cj < 0)
                break;
            if(ci / BANK != cj / BANK)
                continue;
            double* dst;
            int     mode;
            if(ci == cj)
            {
                dst  = &s->hess[((size_t)(ci / BANK) * SYM + sym_index(ci % BANK, ci % BANK)) * 9];
                mode = (i == j) ? 0 : 2;
            }
            else if(ci < cj)
            {
                dst  = &s->hess[((size_t)(ci / BANK) * SYM + sym_index(ci % BANK, cj % BANK)) * 9];
                mode = 0;
            }
            else
            {
                dst  = &s->hess[((size_t)(cj / BANK) * SYM + sym_index(cj % BANK, ci % BANK)) * 9];
                mode = 1;
            }
            add_block(dst, B, mode);
        }
    }
    s->inv.assign((size_t)s->clusters * SYM * 9, 0.0f);
    // clusters are independent (each inversion uses its own thread's buffers)
#pragma omp parallel for schedule(dynamic, 64)
    for(int c = 0; c < s->clusters; ++c)
    {
        if(invert_mode == 0)
            invert_sweep_f32(&s->hess[(size_t)c * SYM * 9], &s->inv[(size_t)c * SYM * 9]);
        else
            invert_sweep_f64(&s->hess[(size_t)c * SYM * 9], &s->inv[(size_t)c * SYM * 9]);
    }
    return 0;
}

}  // extern "C"

namespace
{
// FP32 -> BF16 -> FP32, round to nearest even (finite inputs)
inline float bf16_round(float v)
{
    uint32_t u;
    std::memcpy(&u, &v, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    u &= 0xFFFF0000u;
    float o;
    std::memcpy(&o, &u, 4);
    return o;
}
}  // namespace

extern "C" {

void orc_mas_quantize(orc_mas* s, int mode)
{
    if(mode == 0)
        return;
    for(int c = 0; c < s->clusters; ++c)
    {
        float* M = &s->inv[(size_t)c * SYM * 9];
        float  sc[BANK * 3];
        for(int nd = 0; nd < BANK; ++nd)
        {
            const float* D = &M[sym_index(nd, nd) * 9];
            for(int a = 0; a < 3; ++a)
            {
                const float d  = D[a * 3 + a];
                sc[nd * 3 + a] = (mode == 2 && d > 0.f) ? 1.0f / std::sqrt(d) : 1.0f;
            }
        }
        for(int rn = 0; rn < BANK; ++rn)
            for(int cn = rn; cn < BANK; ++cn)
            {
                float* B = &M[sym_index(rn, cn) * 9];
                for(int q = 0; q < 3; ++q)      // column
                    for(int p = 0; p < 3; ++p)  // row
                    {
                        const float si = sc[rn * 3 + p], sj = sc[cn * 3 + q];
                        const float scaled = bf16_round(B[q * 3 + p] * si * sj);
                        B[q * 3 + p]       = scaled / (si * sj);
                    }
            }
    }
}

void orc_mas_clusters(const orc_mas* s, double* hess, float* inv)
{
    if(hess)
        std::memcpy(hess, s->hess.data(), sizeof(double) * s->hess.size());
    if(inv)
        std::memcpy(inv, s->inv.data(), sizeof(float) * s->inv.size());
}

// replace the cluster inverses (e.g. by the device's), so an apply can be
// compared with the same inverse entries
void orc_mas_set_inverses(orc_mas* s, const float* inv)
{
    std::memcpy(s->inv.data(), inv, sizeof(float) * s->inv.size());
}

// apply (:2887-2960): R_l = sum of float(r) over each level-l node's fine
// vertices (build_multi_level_R :1205-1321), Z = cluster inverse * R per
// cluster (schwarz_local_solve :1323-1414), z_v = double(sum_l Z_l[node_l(v)])
// (collect_final_Z :1895-1955). Float sums in partition order.
void orc_mas_apply(const orc_mas* s, const double* r, double* z)
{
    const int L = s->L;
    std::vector<float> R((size_t)s->total * 3, 0.0f), Z((size_t)s->total * 3, 0.0f);
    for(int p = 0; p < s->N; ++p)
    {
        const int v = s->p2r[p];
        if(v < 0)
            continue;
        const float rv[3] = {(float)r[(size_t)v * 3], (float)r[(size_t)v * 3 + 1], (float)r[(size_t)v * 3 + 2]};
        for(int a = 0; a < 3; ++a)
            R[(size_t)p * 3 + a] = rv[a];
        for(int l = 1; l < L; ++l)
        {
            const int node = s->ctable[(size_t)v * (L - 1) + (l - 1)];
            for(int a = 0; a < 3; ++a)
                R[(size_t)node * 3 + a] += rv[a];
        }
    }
    // local solves: clusters are independent
#pragma omp parallel for schedule(static)
    for(int c = 0; c < s->clusters; ++c)
    {
        const float* M = &s->inv[(size_t)c * SYM * 9];
        for(int rn = 0; rn < BANK; ++rn)
        {
            float acc[3] = {0.f, 0.f, 0.f};
            for(int cn = 0; cn < BANK; ++cn)
            {
                const float* x = &R[((size_t)c * BANK + cn) * 3];
                if(cn >= rn)
                {
                    const float* B = &M[sym_index(rn, cn) * 9];
                    for(int a = 0; a < 3; ++a)
                        for(int k = 0; k < 3; ++k)
                            acc[a] = std::fmaf(B[k * 3 + a], x[k], acc[a]);
                }
                else
                {
                    const float* B = &M[sym_index(cn, rn) * 9];
                    for(int a = 0; a < 3; ++a)
                        for(int k = 0; k < 3; ++k)
                            acc[a] = std::fmaf(B[a * 3 + k], x[k], acc[a]);
                }
            }
            for(int a = 0; a < 3; ++a)
                Z[((size_t)c * BANK + rn) * 3 + a] = acc[a];
        }
    }
#pragma omp parallel for schedule(static)
    for(int v = 0; v < s->vn; ++v)
    {
        const int p = s->r2p[v];
        if(p < 0)
            continue;
        float cz[3] = {Z[(size_t)p * 3], Z[(size_t)p * 3 + 1], Z[(size_t)p * 3 + 2]};
        for(int l = 1; l < L; ++l)
        {
            const int node = s->ctable[(size_t)v * (L - 1) + (l - 1)];
            for(int a = 0; a < 3; ++a)
                cz[a] += Z[(size_t)node * 3 + a];
        }
        for(int a = 0; a < 3; ++a)
            z[(size_t)v * 3 + a] = (double)cz[a];
    }
}

}  // extern "C"

// ---------------------------------------------------------------------------
// PCG
// ---------------------------------------------------------------------------
namespace
{
struct Precond
{
    int                 kind = 0;
    const orc_mas*      mas  = nullptr;
    int32_t             off  = 0;
    std::vector<double> dinv;  // 3x3 inverses (row-major) of the diagonal blocks
    std::vector<char>   in_mas;
    int32_t             abd_off = 0, abd_n = 0;  // affine bodies: 4 block rows each
    std::vector<double> abd_inv;                 // [abd_n][12][12] row-major

    // ABDDiagPreconditioner (affine_body/abd_diag_preconditioner.cu:15-125):
    // the inverse of each body's full 12x12 diagonal block (FP64; Eigen's
    // inverse there, Gauss-Jordan with partial pivoting here)
    void build_abd(const orc_matrix* A)
    {
        abd_inv.assign((size_t)abd_n * 144, 0.0);
        std::vector<double> H((size_t)abd_n * 144, 0.0);
        for(size_t u = 0; u < A->rows.size(); ++u)
        {
            const int i = A->rows[u] - abd_off, j = A->cols[u] - abd_off;
            if(i < 0 || j < 0 || i >= 4 * abd_n || j >= 4 * abd_n || i / 4 != j / 4)
                continue;
            double*       h  = &H[(size_t)(i / 4) * 144];
            const int     bi = i % 4, bj = j % 4;
            const double* B  = &A->vals[u * 9];  // column-major
            for(int p = 0; p < 3; ++p)
                for(int q = 0; q < 3; ++q)
                {
                    h[(3 * bi + p) * 12 + 3 * bj + q] = B[q * 3 + p];
                    if(bi != bj)
                        h[(3 * bj + q) * 12 + 3 * bi + p] = B[q * 3 + p];
                }
        }
        for(int b = 0; b < abd_n; ++b)
        {
            double M[12][24];
            for(int i = 0; i < 12; ++i)
                for(int j = 0; j < 24; ++j)
                    M[i][j] = j < 12 ? H[(size_t)b * 144 + i * 12 + j] : (j - 12 == i ? 1.0 : 0.0);
            bool ok = true;
            for(int c = 0; c < 12 && ok; ++c)
            {
                int piv = c;
                for(int r = c + 1; r < 12; ++r)
                    if(std::fabs(M[r][c]) > std::fabs(M[piv][c]))
                        piv = r;
                if(!(std::fabs(M[piv][c]) > 0.0))
                {
                    ok = false;
                    break;
                }
                for(int j = 0; j < 24; ++j)
                    std::swap(M[c][j], M[piv][j]);
                const double d = 1.0 / M[c][c];
                for(int j = 0; j < 24; ++j)
                    M[c][j] *= d;
                for(int r = 0; r < 12; ++r)
                    if(r != c && M[r][c] != 0.0)
                    {
                        const double f = M[r][c];
                        for(int j = 0; j < 24; ++j)
                            M[r][j] -= f * M[c][j];
                    }
            }
            for(int i = 0; i < 12; ++i)
                for(int j = 0; j < 12; ++j)
                    abd_inv[(size_t)b * 144 + i * 12 + j] = ok ? M[i][12 + j] : (i == j ? 1.0 : 0.0);
        }
    }

    void build(const orc_matrix* A)
    {
        const int32_t nb = A->nb;
        dinv.assign((size_t)nb * 9, 0.0);
        // FEMDiagPreconditioner_do_assemble (fem_diag_preconditioner.cu:18-44):
        // 3x3 inverse of each diagonal block
        for(size_t u = 0; u < A->rows.size(); ++u)
        {
            if(A->rows[u] != A->cols[u])
                continue;
            const double* B = &A->vals[u * 9];
            // row-major m
            double m[9] = {B[0], B[3], B[6], B[1], B[4], B[7], B[2], B[5], B[8]};
            double c0 = m[4] * m[8] - m[5] * m[7], c1 = m[5] * m[6] - m[3] * m[8], c2 = m[3] * m[7] - m[4] * m[6];
            double det = m[0] * c0 + m[1] * c1 + m[2] * c2;
            double id  = 1.0 / det;
            double* o  = &dinv[(size_t)A->rows[u] * 9];
            o[0] = c0 * id;
            o[1] = (m[2] * m[7] - m[1] * m[8]) * id;
            o[2] = (m[1] * m[5] - m[2] * m[4]) * id;
            o[3] = c1 * id;
            o[4] = (m[0] * m[8] - m[2] * m[6]) * id;
            o[5] = (m[2] * m[3] - m[0] * m[5]) * id;
            o[6] = c2 * id;
            o[7] = (m[1] * m[6] - m[0] * m[7]) * id;
            o[8] = (m[0] * m[4] - m[1] * m[3]) * id;
        }
        in_mas.assign(nb, 0);
        if(kind == ORC_PRECOND_MAS && mas)
            for(int v = 0; v < mas->vn; ++v)
                if(mas->r2p[v] >= 0 && v + off < nb)
                    in_mas[v + off] = 1;
    }
    void apply(const double* r, double* z, int32_t nb) const
    {
        const size_t n = (size_t)nb * 3;
        if(kind == ORC_PRECOND_NONE)
        {
            std::copy(r, r + n, z);
            return;
        }
#pragma omp parallel for schedule(static)
        for(int32_t i = 0; i < nb; ++i)
        {
            if(kind == ORC_PRECOND_MAS && in_mas[i])
                continue;
            const double* D = &dinv[(size_t)i * 9];
            const double* x = &r[(size_t)i * 3];
            for(int a = 0; a < 3; ++a)
                z[(size_t)i * 3 + a] = D[a * 3] * x[0] + D[a * 3 + 1] * x[1] + D[a * 3 + 2] * x[2];
        }
        if(kind == ORC_PRECOND_MAS && mas)
            orc_mas_apply(mas, r + (size_t)off * 3, z + (size_t)off * 3);
        // the affine-body range: the 12x12 block inverses (after the others,
        // global_linear_system.cu:555-576)
        for(int b = 0; b < abd_n; ++b)
        {
            const double* Hi = &abd_inv[(size_t)b * 144];
            const double* rb = &r[(size_t)(abd_off + 4 * b) * 3];
            double*       zb = &z[(size_t)(abd_off + 4 * b) * 3];
            for(int i = 0; i < 12; ++i)
            {
                double acc = 0.0;
                for(int j = 0; j < 12; ++j)
                    acc += Hi[i * 12 + j] * rb[j];
                zb[i] = acc;
            }
        }
    }
};

double dotp(const double* a, const double* b, size_t n)
{
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for(int64_t i = 0; i < (int64_t)n; ++i)
        s += a[i] * b[i];
    return s;
}
}  // namespace

extern "C" {

int orc_pcg(const orc_matrix* A, int precond, const orc_mas* mas, int32_t mas_off, const double* b,
            double* x, double tol, int stop_rule, int check_interval, int64_t max_iter, int n_threads,
            orc_pcg_result* out)
{
    return orc_pcg_abd(A, precond, mas, mas_off, 0, 0, b, x, tol, stop_rule, check_interval, max_iter, n_threads,
                       out);
}

int orc_pcg_abd(const orc_matrix* A, int precond, const orc_mas* mas, int32_t mas_off, int32_t abd_off,
                int32_t abd_n, const double* b, double* x, double tol, int stop_rule, int check_interval,
                int64_t max_iter, int n_threads, orc_pcg_result* out)
{
#ifdef _OPENMP
    const int saved = omp_get_max_threads();
    omp_set_num_threads(n_threads > 0 ? n_threads : 1);
#endif
    const int32_t nb = A->nb;
    const size_t  n  = (size_t)nb * 3;
    Precond       P;
    P.kind = precond;
    P.mas  = mas;
    P.off  = mas_off;
    P.build(A);
    if(precond != ORC_PRECOND_NONE && abd_n > 0)
    {
        P.abd_off = abd_off;
        P.abd_n   = abd_n;
        P.build_abd(A);
    }
    auto spmv = [&](const double* in, double* o)
    {
        if(n_threads > 1)
            spmv_full(A, in, o);
        else
            spmv_sym(A, in, o);
    };
    std::vector<double> r(b, b + n), z(n), p(n), Ap(n);
    std::fill(x, x + n, 0.0);
    P.apply(r.data(), z.data(), nb);
    double rz = dotp(r.data(), z.data(), n);
    orc_pcg_result res{};
    // PSD guard (linear_fused_pcg.cu:1819-1877): rz0 < 0 or non-finite -> plain CG
    bool bypass = false;
    if(rz < 0.0 || !std::isfinite(rz))
    {
        bypass = true;
        z      = r;
        rz     = dotp(r.data(), z.data(), n);
    }
    p                  = z;
    res.rz0            = rz;
    res.bypassed       = bypass;
    const double abs0  = std::fabs(rz);
    const double bnorm = std::sqrt(dotp(b, b, n));
    const int    ci    = check_interval > 0 ? check_interval : 1;
    int64_t      k     = 0;
    bool         conv  = false;
    if(abs0 == 0.0 || bnorm == 0.0)
    {
        conv = true;
    }
    else
    {
        const double rz_tol = tol * abs0;
        for(k = 1; k < max_iter; ++k)
        {
            spmv(p.data(), Ap.data());
            const double alpha = rz / dotp(p.data(), Ap.data(), n);
#pragma omp parallel for schedule(static)
            for(int64_t i = 0; i < (int64_t)n; ++i)
            {
                x[i] += alpha * p[i];
                r[i] -= alpha * Ap[i];
            }
            if(bypass)
                z = r;
            else
                P.apply(r.data(), z.data(), nb);
            const double rz_new = dotp(r.data(), z.data(), n);
            bool         hit;
            if(stop_rule == ORC_STOP_RZ)
                hit = std::fabs(rz_new) <= rz_tol;
            else
                hit = std::sqrt(dotp(r.data(), r.data(), n)) <= tol * bnorm;
            if(hit)
            {
                conv = true;
                break;
            }
            const double beta = rz_new / rz;
#pragma omp parallel for schedule(static)
            for(int64_t i = 0; i < (int64_t)n; ++i)
                p[i] = z[i] + beta * p[i];
            rz = rz_new;
        }
    }
    // the fused solver checks every `check_interval` iterations and reports
    // the iteration count of that check (linear_fused_pcg.cu:1923-1998)
    int64_t reported = k;
    if(ci > 1 && conv && k > 0)
        reported = std::min<int64_t>(((k + ci - 1) / ci) * ci, max_iter);
    if(!conv)
        reported = max_iter;
    res.iterations = reported;
    res.converged  = conv;
    std::vector<double> t(n);
    spmv(x, t.data());
    double rr = 0.0;
    for(size_t i = 0; i < n; ++i)
        rr += (b[i] - t[i]) * (b[i] - t[i]);
    res.rel_res_true = bnorm > 0 ? std::sqrt(rr) / bnorm : 0.0;
    if(out)
        *out = res;
#ifdef _OPENMP
    omp_set_num_threads(saved);
#endif
    return 0;
}

int orc_cg_truth(const orc_matrix* A, const double* b, double* x, double tol, int64_t max_iter, int n_threads,
                 int64_t* iterations)
{
    orc_pcg_result r{};
    int rc = orc_pcg(A, ORC_PRECOND_JACOBI, nullptr, 0, b, x, tol, ORC_STOP_RELRES, 1, max_iter, n_threads, &r);
    if(iterations)
        *iterations = r.iterations;
    return rc != 0 ? rc : (r.converged ? 0 : 2);
}

}  // extern "C"
