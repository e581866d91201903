// Matrix Market I/O of block-sparse Newton systems; format and semantics in
// include/b200io.h. The text is formatted by OpenMP threads into per-chunk
// buffers written in order, so a 4 M-block matrix (38 M lines) takes seconds.
#include "../../../include/b200io.h"

#include <omp.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

struct b2io_matrix
{
    int32_t              n_block_rows = 0;
    int64_t              n_entries    = 0;  // scalar entries kept (inside the stated size)
    std::vector<int32_t> rows, cols;
    std::vector<double>  vals;  // 9 per block, column-major
};

namespace
{
// the whole file in memory, NUL-terminated
bool slurp(const char* path, std::vector<char>& buf)
{
    FILE* f = std::fopen(path, "rb");
    if(!f)
        return false;
    std::fseek(f, 0, SEEK_END);
    const long size = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if(size < 0)
    {
        std::fclose(f);
        return false;
    }
    buf.resize((size_t)size + 1);
    const size_t got = size > 0 ? std::fread(buf.data(), 1, (size_t)size, f) : 0;
    std::fclose(f);
    buf[got] = '\0';
    buf.resize(got + 1);
    return got == (size_t)size;
}

// next line [p, end of line); returns the start of the following line
const char* next_line(const char* p, const char** line_end)
{
    const char* e = p;
    while(*e && *e != '\n')
        ++e;
    *line_end = e;
    return *e ? e + 1 : e;
}

// start of the next field of the line [p, e) (spaces and tabs skipped), or
// nullptr at the end of the line: numbers are never parsed across lines
const char* field(const char* p, const char* e)
{
    while(p < e && (*p == ' ' || *p == '\t'))
        ++p;
    return p < e && *p != '\r' ? p : nullptr;
}

bool is_blank_or_comment(const char* p, const char* e)
{
    while(p < e && (*p == ' ' || *p == '\t' || *p == '\r'))
        ++p;
    return p == e || *p == '%';
}

// write `count` items formatted by fmt(i, buf) -> length, in order, in chunks
template <typename F>
bool write_chunked(FILE* f, int64_t count, int max_len, F fmt)
{
    const int64_t chunk = 1 << 16;
    const int64_t n_chunks = (count + chunk - 1) / chunk;
    const int     threads = std::max(1, omp_get_max_threads());
    bool          ok = true;
    // groups of `threads` chunks: formatted in parallel, written in order
    for(int64_t g0 = 0; g0 < n_chunks && ok; g0 += threads)
    {
        const int64_t            g1 = std::min(n_chunks, g0 + threads);
        std::vector<std::string> out((size_t)(g1 - g0));
#pragma omp parallel for schedule(static)
        for(int64_t c = g0; c < g1; ++c)
        {
            std::string& s = out[(size_t)(c - g0)];
            const int64_t b = c * chunk, e = std::min(count, b + chunk);
            s.resize((size_t)((e - b) * max_len));
            size_t len = 0;
            for(int64_t i = b; i < e; ++i)
                len += (size_t)fmt(i, &s[len]);
            s.resize(len);
        }
        for(const std::string& s : out)
            ok = ok && std::fwrite(s.data(), 1, s.size(), f) == s.size();
    }
    return ok;
}
}  // namespace

extern "C" int b2io_write_block_matrix(const char* path, int32_t n_block_rows, int64_t n_blocks, const int32_t* rows,
                                       const int32_t* cols, const double* vals, int one_based)
{
    if(!path || n_block_rows < 0 || n_blocks < 0 || (n_blocks > 0 && (!rows || !cols || !vals)))
        return -3;
    FILE* f = std::fopen(path, "w");
    if(!f)
        return -1;
    const int64_t dim = (int64_t)n_block_rows * 3, entries = n_blocks * 9;
    std::fprintf(f, "%%MatrixMarket matrix coordinate real general\n");
    std::fprintf(f, "%% Exported from block-sparse triplet matrix\n");
    std::fprintf(f, "%% Block dimension: 3x3\n");
    std::fprintf(f, "%% Total rows: %lld, Total cols: %lld\n", (long long)dim, (long long)dim);
    std::fprintf(f, "%% Total entries (including zeros): %lld\n", (long long)entries);
    std::fprintf(f, "%lld %lld %lld\n", (long long)dim, (long long)dim, (long long)entries);
    const long long base = one_based ? 1 : 0;
    // entry e of block k: row bi = e / 3, column bj = e % 3, value B(bi, bj)
    const bool ok = write_chunked(f, entries, 64, [&](int64_t i, char* buf) {
        const int64_t k = i / 9;
        const int     e = (int)(i % 9), bi = e / 3, bj = e % 3;
        return std::snprintf(buf, 64, "%lld %lld %.17g\n", (long long)rows[k] * 3 + bi + base,
                             (long long)cols[k] * 3 + bj + base, vals[k * 9 + bj * 3 + bi]);
    });
    const bool closed = std::fclose(f) == 0;
    return ok && closed ? 0 : -1;
}

extern "C" int b2io_write_vector(const char* path, int64_t n, const double* x)
{
    if(!path || n < 0 || (n > 0 && !x))
        return -3;
    FILE* f = std::fopen(path, "w");
    if(!f)
        return -1;
    std::fprintf(f, "%%MatrixMarket matrix array real general\n");
    std::fprintf(f, "%% Exported from dense vector\n");
    std::fprintf(f, "%% Vector size: %lld\n", (long long)n);
    std::fprintf(f, "%lld 1\n", (long long)n);
    const bool ok = write_chunked(f, n, 40, [&](int64_t i, char* buf) {
        return std::snprintf(buf, 40, "%.17g\n", x[i]);
    });
    const bool closed = std::fclose(f) == 0;
    return ok && closed ? 0 : -1;
}

static int read_block_matrix(const char* path, int one_based, b2io_matrix** out)
{
    if(!path || !out)
        return -3;
    *out = nullptr;
    std::vector<char> buf;
    if(!slurp(path, buf))
        return -1;
    const char* p = buf.data();
    const char* e = nullptr;
    long long   R = 0, C = 0, NNZ = 0;
    bool        have_size = false;
    while(*p)
    {
        const char* line = p;
        p = next_line(p, &e);
        if(is_blank_or_comment(line, e))
            continue;
        if(std::sscanf(line, "%lld %lld %lld", &R, &C, &NNZ) != 3)
            return -2;
        have_size = true;
        break;
    }
    if(!have_size || R <= 0 || C <= 0 || NNZ <= 0 || R > (1ll << 31) - 3)
        return -2;
    const long long off = one_based ? 1 : 0;
    // entries in file order: block key, slot in the block, value
    std::vector<uint64_t> key;
    std::vector<uint8_t>  slot;
    std::vector<double>   val;
    // the stated count only sizes the arrays up front (an entry line has at
    // least 6 characters, so a larger claim cannot be true)
    const size_t expect = (size_t)std::min<long long>(NNZ, (long long)(buf.size() / 6 + 1));
    key.reserve(expect);
    slot.reserve(expect);
    val.reserve(expect);
    while(*p)
    {
        const char* line = p;
        p = next_line(p, &e);
        if(is_blank_or_comment(line, e))
            continue;
        const char* f0 = field(line, e);
        char*       q  = nullptr;
        if(!f0)
            continue;
        const long long i  = std::strtoll(f0, &q, 10);
        const char*     f1 = q != f0 ? field(q, e) : nullptr;
        if(!f1)
            continue;  // not an entry line
        const long long j  = std::strtoll(f1, &q, 10);
        const char*     f2 = q != f1 ? field(q, e) : nullptr;
        if(!f2)
            continue;
        const double v = std::strtod(f2, &q);
        if(q == f2)
            continue;
        const long long ii = i - off, jj = j - off;
        if(ii < 0 || ii >= R || jj < 0 || jj >= C)
            continue;
        key.push_back(((uint64_t)(ii / 3) << 32) | (uint64_t)(jj / 3));
        slot.push_back((uint8_t)((jj % 3) * 3 + ii % 3));
        val.push_back(v);
    }
    const size_t m = key.size();
    std::vector<uint32_t> order(m);
    std::iota(order.begin(), order.end(), 0u);
    if(!std::is_sorted(key.begin(), key.end()))
        std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return key[a] < key[b]; });
    auto* M          = new b2io_matrix();
    M->n_block_rows  = (int32_t)((R + 2) / 3);
    M->n_entries     = (int64_t)m;
    for(size_t t = 0; t < m; ++t)
    {
        const uint64_t k = key[order[t]];
        if(t == 0 || k != key[order[t - 1]])
        {
            M->rows.push_back((int32_t)(k >> 32));
            M->cols.push_back((int32_t)(k & 0xFFFFFFFFu));
            M->vals.resize(M->vals.size() + 9, 0.0);
        }
        M->vals[M->vals.size() - 9 + slot[order[t]]] = val[order[t]];  // the later entry wins
    }
    *out = M;
    return 0;
}

extern "C" int b2io_read_block_matrix(const char* path, int one_based, b2io_matrix** out)
{
    try
    {
        return read_block_matrix(path, one_based, out);
    }
    catch(...)  // allocation failure
    {
        return -1;
    }
}

extern "C" int b2io_matrix_size(const b2io_matrix* m, int32_t* n_block_rows, int64_t* n_blocks, int64_t* n_entries)
{
    if(!m)
        return -3;
    if(n_block_rows)
        *n_block_rows = m->n_block_rows;
    if(n_blocks)
        *n_blocks = (int64_t)m->rows.size();
    if(n_entries)
        *n_entries = m->n_entries;
    return 0;
}

extern "C" int b2io_matrix_copy(const b2io_matrix* m, int32_t* rows, int32_t* cols, double* vals)
{
    if(!m)
        return -3;
    if(rows)
        std::memcpy(rows, m->rows.data(), m->rows.size() * sizeof(int32_t));
    if(cols)
        std::memcpy(cols, m->cols.data(), m->cols.size() * sizeof(int32_t));
    if(vals)
        std::memcpy(vals, m->vals.data(), m->vals.size() * sizeof(double));
    return 0;
}

extern "C" void b2io_matrix_free(b2io_matrix* m) { delete m; }

extern "C" int b2io_read_vector(const char* path, int64_t capacity, double* x, int64_t* n)
{
    if(!path || !n)
        return -3;
    std::vector<char> buf;
    if(!slurp(path, buf))
        return -1;
    const char* p = buf.data();
    const char* e = nullptr;
    long long   R = 0, C = 0;
    bool        have_size = false;
    while(*p)
    {
        const char* line = p;
        p = next_line(p, &e);
        if(is_blank_or_comment(line, e))
            continue;
        if(std::sscanf(line, "%lld %lld", &R, &C) != 2)
            return -2;
        have_size = true;
        break;
    }
    if(!have_size || R <= 0 || C != 1)
        return -2;
    int64_t got = 0;
    while(*p)
    {
        const char* line = p;
        p = next_line(p, &e);
        if(is_blank_or_comment(line, e))
            continue;
        const char* f0 = field(line, e);
        char*       q  = nullptr;
        if(!f0)
            continue;
        const double v = std::strtod(f0, &q);
        if(q == f0)
            continue;
        if(x)
        {
            if(got >= capacity)
                return -3;
            x[got] = v;
        }
        ++got;
    }
    if(got != R)
        return -2;
    *n = got;
    return 0;
}
