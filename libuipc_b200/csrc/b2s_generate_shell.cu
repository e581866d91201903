// Newton systems of cloth (codim-2D) meshes and affine bodies generated on
// the GPU (include/b200gen.h): kinetic + Baraff-Witkin stretch/shear +
// discrete-shell bending for the cloth, kinetic + orthogonality potential for
// the bodies, straight into device triplet buffers. The element arithmetic is
// csrc/scene/elements.h, shared with the host generator (scene_gen.cpp:
// add_cloth_grid, add_affine_body), with the same triplet layout and the same
// per-vertex gradient sum order, so the two agree to rounding (FMA
// contraction on the device).
#include "b2s_ccd.cuh"
#include "b2s_fixed_reduce.cuh"
#include "b2s_internal.cuh"

#include "../../include/b200gen.h"
#include "scene/elements.h"

#include <algorithm>
#include <array>
#include <cstring>
#include <string>
#include <vector>

namespace
{
thread_local std::string g_shell_err;

constexpr int SHELL_BLOCK = 128;

int grid_of(int64_t n) { return (int)((n + SHELL_BLOCK - 1) / SHELL_BLOCK); }

// a row-major 3x3 block of the pair (ra, rb) into slot k, block-upper,
// column-major values (transposed when ra > rb)
__device__ __forceinline__ void put_block(int64_t k, int32_t ra, int32_t rb, const double* Hab, int32_t* rows,
                                          int32_t* cols, double* vals)
{
    const bool tp = ra > rb;
    rows[k]       = tp ? rb : ra;
    cols[k]       = tp ? ra : rb;
    double* V     = vals + k * 9;
    for(int q = 0; q < 3; ++q)
        for(int p = 0; p < 3; ++p)
            V[q * 3 + p] = tp ? Hab[q * 3 + p] : Hab[p * 3 + q];
}

// the upper 3x3 blocks of an NV-vertex element Hessian (row-major), in the
// order (0,0), (0,1), .., (0,NV-1), (1,1), ..
template <int NV>
__device__ void put_element(int64_t slot0, const int32_t* v, int32_t off, const double* H, int32_t* rows,
                            int32_t* cols, double* vals)
{
    int64_t k = slot0;
    for(int i = 0; i < NV; ++i)
        for(int j = i; j < NV; ++j, ++k)
        {
            double blk[9];
            for(int p = 0; p < 3; ++p)
                for(int q = 0; q < 3; ++q)
                    blk[p * 3 + q] = H[(3 * i + p) * (3 * NV) + 3 * j + q];
            put_block(k, v[i] + off, v[j] + off, blk, rows, cols, vals);
        }
}

__global__ void k_shell_rest(int nt, const double* __restrict__ X, const int32_t* __restrict__ tris,
                             double* __restrict__ IB, double* __restrict__ area)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if(t >= nt)
        return;
    const int32_t* T = tris + (int64_t)t * 3;
    b2el::bw_rest(X + 3 * T[0], X + 3 * T[1], X + 3 * T[2], IB + 4 * (int64_t)t);
    area[t] = b2el::tri_area(X + 3 * T[0], X + 3 * T[1], X + 3 * T[2]);
}

__global__ void k_hinge_rest(int nh, const double* __restrict__ X, const int32_t* __restrict__ hinges,
                             double* __restrict__ rest3)
{
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if(h >= nh)
        return;
    const int32_t* v = hinges + (int64_t)h * 4;
    double*        r = rest3 + (int64_t)h * 3;
    b2el::dsb_rest(X + 3 * v[0], X + 3 * v[1], X + 3 * v[2], X + 3 * v[3], r, r + 1, r + 2);
}

// Baraff-Witkin per triangle: 6 blocks from slot nv + 6 t, gradient to tri_g
__global__ void __launch_bounds__(SHELL_BLOCK) k_shell_bw(int nv, int nt, int32_t off, const int32_t* __restrict__ tris,
                                                          const double* __restrict__ IB,
                                                          const double* __restrict__ area,
                                                          const double* __restrict__ x, double stretch, double shear,
                                                          double rate, double dt2, int32_t* rows, int32_t* cols,
                                                          double* vals, double* __restrict__ tri_g)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if(t >= nt)
        return;
    const int32_t* T = tris + (int64_t)t * 3;
    double         xs[9];
    for(int i = 0; i < 3; ++i)
        for(int a = 0; a < 3; ++a)
            xs[3 * i + a] = x[3 * (int64_t)(T[i] + off) + a];
    double G[9], H[81];
    b2el::bw_grad_hess(xs, xs + 3, xs + 6, IB + 4 * (int64_t)t, stretch, shear, rate, area[t] * dt2, G, H);
    for(int i = 0; i < 9; ++i)
        tri_g[(int64_t)t * 9 + i] = G[i];
    put_element<3>((int64_t)nv + 6ll * t, T, off, H, rows, cols, vals);
}

// discrete-shell bending per hinge: 10 blocks from slot nv + 6 nt + 10 h
__global__ void __launch_bounds__(SHELL_BLOCK) k_shell_dsb(int nv, int nt, int nh, int32_t off,
                                                           const int32_t* __restrict__ hinges,
                                                           const double* __restrict__ rest3,
                                                           const double* __restrict__ x, double kappa, double dt2,
                                                           int32_t* rows, int32_t* cols, double* vals,
                                                           double* __restrict__ hinge_g)
{
    const int h = blockIdx.x * blockDim.x + threadIdx.x;
    if(h >= nh)
        return;
    const int32_t* V = hinges + (int64_t)h * 4;
    double         xs[12];
    for(int i = 0; i < 4; ++i)
        for(int a = 0; a < 3; ++a)
            xs[3 * i + a] = x[3 * (int64_t)(V[i] + off) + a];
    const double* r = rest3 + (int64_t)h * 3;
    double        G[12], H[144];
    b2el::dsb_grad_hess(xs, xs + 3, xs + 6, xs + 9, r[0], r[1], r[2], kappa, dt2, G, H);
    for(int i = 0; i < 12; ++i)
        hinge_g[(int64_t)h * 12 + i] = G[i];
    put_element<4>((int64_t)nv + 6ll * nt + 10ll * h, V, off, H, rows, cols, vals);
}

// kinetic block and the gradient per vertex: m (x - x_tilde), then the
// triangles' and the hinges' contributions in element order
__global__ void k_shell_vertex(int nv, int32_t off, const double* __restrict__ mass, const double* __restrict__ x,
                               const double* __restrict__ xt, const int32_t* __restrict__ inc_start,
                               const int32_t* __restrict__ inc_list, int nt, const double* __restrict__ tri_g,
                               const double* __restrict__ hinge_g, int32_t* rows, int32_t* cols, double* vals,
                               double* __restrict__ grad)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if(v >= nv)
        return;
    const double  m    = mass[v];
    const double  H[9] = {m, 0, 0, 0, m, 0, 0, 0, m};
    const int64_t g    = (int64_t)v + off;
    put_block(v, (int32_t)g, (int32_t)g, H, rows, cols, vals);
    double acc[3];
    for(int a = 0; a < 3; ++a)
        acc[a] = m * (x[g * 3 + a] - xt[g * 3 + a]);
    // incidences: triangle corners (4 t + c) then hinge corners (4 (nt + h) + c)
    for(int e = inc_start[v]; e < inc_start[v + 1]; ++e)
    {
        const int32_t code = inc_list[e], el = code >> 2, c = code & 3;
        const double* src  = el < nt ? tri_g + (int64_t)el * 9 + 3 * c : hinge_g + (int64_t)(el - nt) * 12 + 3 * c;
        for(int a = 0; a < 3; ++a)
            acc[a] += src[a];
    }
    for(int a = 0; a < 3; ++a)
        grad[g * 3 + a] = acc[a];
}

// Dirichlet vertices of the cloth: rows / columns zero, diagonal I, gradient 0
__global__ void k_shell_fixed(int64_t T, int nv, int32_t off, const uint8_t* __restrict__ fixed,
                              const int32_t* __restrict__ rows, const int32_t* __restrict__ cols, double* vals,
                              double* grad)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(s < T)
    {
        const int32_t i = rows[s] - off, j = cols[s] - off;
        if(fixed[i] || fixed[j])
        {
            double* V = vals + s * 9;
            for(int e = 0; e < 9; ++e)
                V[e] = 0.0;
            if(i == j)
                V[0] = V[4] = V[8] = 1.0;
        }
    }
    if(s < nv && fixed[s])
        grad[(s + off) * 3] = grad[(s + off) * 3 + 1] = grad[(s + off) * 3 + 2] = 0.0;
}

// affine bodies: M + ortho Hessian (PSD, V dt^2) as 16 blocks (lower ones
// zero), gradient M (q - q_tilde) + ortho gradient
__global__ void k_abd(int nb, int32_t off, const double* __restrict__ M, const double* __restrict__ kappa,
                      const double* __restrict__ volume, const double* __restrict__ q, const double* __restrict__ qt,
                      double dt2, int32_t* rows, int32_t* cols, double* vals, double* __restrict__ grad)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if(b >= nb)
        return;
    const int64_t base = (int64_t)off + 4ll * b;
    double        qb[12], H[144], G9[9], H9[81];
    for(int i = 0; i < 12; ++i)
        qb[i] = q[base * 3 + i];
    const double* Mb = M + (int64_t)b * 144;
    for(int i = 0; i < 144; ++i)
        H[i] = Mb[i];
    b2el::ortho_grad_hess(qb, kappa[b], volume[b] * dt2, G9, H9);
    for(int m = 0; m < 9; ++m)
        for(int n = 0; n < 9; ++n)
            H[(3 + m) * 12 + 3 + n] += H9[m * 9 + n];
    for(int i = 0; i < 12; ++i)
    {
        double g = 0.0;
        for(int j = 0; j < 12; ++j)
            g += Mb[i * 12 + j] * (q[base * 3 + j] - qt[base * 3 + j]);
        grad[base * 3 + i] = g + (i >= 3 ? G9[i - 3] : 0.0);
    }
    int64_t k = 16ll * b;
    for(int bi = 0; bi < 4; ++bi)
        for(int bj = 0; bj < 4; ++bj, ++k)
        {
            rows[k]   = (int32_t)(base + bi);
            cols[k]   = (int32_t)(base + bj);
            double* V = vals + k * 9;
            for(int c = 0; c < 3; ++c)
                for(int r = 0; r < 3; ++r)
                    V[c * 3 + r] = bi > bj ? 0.0 : H[(3 * bi + r) * 12 + 3 * bj + c];
        }
}

// contact pairs: 10 blocks per pair from slot 10 p, the pair's gradient to pair_g
constexpr int CONTACT_BLOCK = 64;

__global__ void __launch_bounds__(CONTACT_BLOCK)
    k_contacts(int np, const int32_t* __restrict__ pairs, const uint8_t* __restrict__ is_ee,
               const double* __restrict__ eps, const double* __restrict__ x, double dhat, double k, int32_t* rows,
               int32_t* cols, double* vals, double* __restrict__ pair_g, int8_t* __restrict__ pair_type)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= np)
        return;
    const int32_t* V = pairs + 4ll * p;
    double         X[12], G[12], H[144];
    for(int i = 0; i < 4; ++i)
        for(int a = 0; a < 3; ++a)
            X[3 * i + a] = x[3 * (int64_t)V[i] + a];
    pair_type[p] = (int8_t)b2el::contact_grad_hess(X, is_ee[p], eps[p], dhat, k, G, H);
    for(int i = 0; i < 12; ++i)
        pair_g[12ll * p + i] = G[i];
    put_element<4>(10ll * p, V, 0, H, rows, cols, vals);
}

// the pairs' gradients added per vertex, in pair order
__global__ void k_contacts_gather(int nlist, const int32_t* __restrict__ verts, const int32_t* __restrict__ start,
                                  const int32_t* __restrict__ list, const double* __restrict__ pair_g,
                                  double* __restrict__ grad)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= nlist)
        return;
    const int64_t v = verts[i];
    double        acc[3] = {grad[3 * v], grad[3 * v + 1], grad[3 * v + 2]};
    for(int e = start[i]; e < start[i + 1]; ++e)
        for(int a = 0; a < 3; ++a)
            acc[a] += pair_g[12ll * (list[e] >> 2) + 3 * (list[e] & 3) + a];
    for(int a = 0; a < 3; ++a)
        grad[3 * v + a] = acc[a];
}

// barrier energy of every pair at x (into e[p])
__global__ void k_contact_energy(int np, const int32_t* __restrict__ pairs, const uint8_t* __restrict__ is_ee,
                                 const double* __restrict__ eps, const double* __restrict__ x, double dhat, double k,
                                 double* __restrict__ e)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= np)
        return;
    const int32_t* V = pairs + 4ll * p;
    double         X[12];
    for(int i = 0; i < 4; ++i)
        for(int a = 0; a < 3; ++a)
            X[3 * i + a] = x[3 * (int64_t)V[i] + a];
    e[p] = b2el::contact_energy(X, is_ee[p], eps[p], dhat, k);
}

void fail(const char* msg) { throw b2s::Error(B2S_ERR_ARGUMENT, msg); }

template <typename F>
int guarded_gen(F&& f)
{
    try
    {
        f();
        return 0;
    }
    catch(const b2s::Error& e)
    {
        g_shell_err = e.what();
        return e.code;
    }
    catch(const std::exception& e)
    {
        g_shell_err = e.what();
        return B2S_ERR_CUDA;
    }
}
}  // namespace

struct b2gen_shell
{
    int32_t               nv = 0, nt = 0, nh = 0;
    b2s::DBuf<int32_t>    tris, hinges, inc_start, inc_list;
    b2s::DBuf<double>     IB, area, rest3, mass, tri_g, hinge_g;
    b2s::DBuf<uint8_t>    fixed;
    b2gen_shell_material  mat{};
    int                   device = 0;
};

struct b2gen_abd
{
    int32_t           nb = 0;
    b2s::DBuf<double> M, kappa, volume;
    double            dt     = 0.0;
    int               device = 0;
};

struct b2gen_contacts
{
    int32_t            np = 0, nvert = 0;
    b2s::DBuf<int32_t> pairs, verts, start, list;
    b2s::DBuf<uint8_t> is_ee;
    b2s::DBuf<int8_t>  pair_type;
    b2s::DBuf<double>  eps, pair_g;
    b2s::DBuf<double>  terms, result;  // per-pair energies or times of impact, and their reduction
    double             dhat = 0.0, kappa = 0.0, dt = 0.0;
    int                device = 0;
};

extern "C" {

const char* b2gen_shell_last_error(void) { return g_shell_err.c_str(); }

int b2gen_shell_create(int device, int32_t n_verts, int32_t n_tris, const double* rest, const int32_t* tris,
                       const double* mass, const uint8_t* fixed, const b2gen_shell_material* mat, b2gen_shell** out)
{
    return guarded_gen(
        [&]
        {
            if(!out || !rest || !tris || !mass || !mat || n_verts <= 0 || n_tris <= 0)
                fail("b2gen_shell_create: bad arguments");
            for(int64_t i = 0; i < 3ll * n_tris; ++i)
                if(tris[i] < 0 || tris[i] >= n_verts)
                    fail("b2gen_shell_create: triangle vertex out of range");
            // hinges: edges shared by exactly two triangles, in (min, max) edge
            // order, (opposite min, edge min, edge max, opposite max)
            std::vector<std::array<int32_t, 3>> opp;
            opp.reserve(3 * (size_t)n_tris);
            for(int32_t t = 0; t < n_tris; ++t)
            {
                int32_t T[3] = {tris[3 * t], tris[3 * t + 1], tris[3 * t + 2]};
                std::sort(T, T + 3);
                opp.push_back({T[0], T[1], T[2]});
                opp.push_back({T[0], T[2], T[1]});
                opp.push_back({T[1], T[2], T[0]});
            }
            std::sort(opp.begin(), opp.end());
            std::vector<int32_t> hinges;
            for(size_t e = 0; e < opp.size();)
            {
                size_t f = e + 1;
                while(f < opp.size() && opp[f][0] == opp[e][0] && opp[f][1] == opp[e][1])
                    ++f;
                if(f - e == 2)
                    hinges.insert(hinges.end(), {std::min(opp[e][2], opp[e + 1][2]), opp[e][0], opp[e][1],
                                                 std::max(opp[e][2], opp[e + 1][2])});
                e = f;
            }
            const int32_t nh = (int32_t)(hinges.size() / 4);
            if((int64_t)n_verts + 6ll * n_tris + 10ll * nh > (int64_t)INT32_MAX)
                fail("b2gen_shell_create: too many triplets for 32-bit slots");
            // vertex incidences: triangle corners by triangle, then hinge corners by hinge
            std::vector<int32_t> start(n_verts + 1, 0), list(3 * (size_t)n_tris + 4 * (size_t)nh);
            for(int64_t i = 0; i < 3ll * n_tris; ++i)
                ++start[tris[i] + 1];
            for(int32_t v : hinges)
                ++start[v + 1];
            for(int32_t v = 0; v < n_verts; ++v)
                start[v + 1] += start[v];
            std::vector<int32_t> fill(start.begin(), start.end() - 1);
            for(int32_t t = 0; t < n_tris; ++t)
                for(int c = 0; c < 3; ++c)
                    list[fill[tris[3 * t + c]]++] = 4 * t + c;
            for(int32_t h = 0; h < nh; ++h)
                for(int c = 0; c < 4; ++c)
                    list[fill[hinges[4 * h + c]]++] = 4 * (n_tris + h) + c;
            B2S_CUDA(cudaSetDevice(device));
            auto S    = new b2gen_shell();
            S->device = device;
            S->nv     = n_verts;
            S->nt     = n_tris;
            S->nh     = nh;
            S->mat    = *mat;
            b2s::DBuf<double> X;
            X.resize((size_t)n_verts * 3);
            S->tris.resize(3 * (size_t)n_tris);
            S->hinges.resize(std::max<size_t>(hinges.size(), 1));
            S->inc_start.resize(n_verts + 1);
            S->inc_list.resize(std::max<size_t>(list.size(), 1));
            S->IB.resize(4 * (size_t)n_tris);
            S->area.resize(n_tris);
            S->rest3.resize(3 * std::max<size_t>(nh, 1));
            S->mass.resize(n_verts);
            S->tri_g.resize(9 * (size_t)n_tris);
            S->hinge_g.resize(12 * std::max<size_t>(nh, 1));
            B2S_CUDA(cudaMemcpy(X.data(), rest, X.bytes(), cudaMemcpyHostToDevice));
            B2S_CUDA(cudaMemcpy(S->tris.data(), tris, sizeof(int32_t) * 3 * (size_t)n_tris, cudaMemcpyHostToDevice));
            if(nh > 0)
                B2S_CUDA(cudaMemcpy(S->hinges.data(), hinges.data(), sizeof(int32_t) * hinges.size(),
                                    cudaMemcpyHostToDevice));
            B2S_CUDA(cudaMemcpy(S->inc_start.data(), start.data(), sizeof(int32_t) * start.size(),
                                cudaMemcpyHostToDevice));
            B2S_CUDA(cudaMemcpy(S->inc_list.data(), list.data(), sizeof(int32_t) * list.size(),
                                cudaMemcpyHostToDevice));
            B2S_CUDA(cudaMemcpy(S->mass.data(), mass, sizeof(double) * n_verts, cudaMemcpyHostToDevice));
            if(fixed)
            {
                S->fixed.resize(n_verts);
                B2S_CUDA(cudaMemcpy(S->fixed.data(), fixed, n_verts, cudaMemcpyHostToDevice));
            }
            k_shell_rest<<<grid_of(n_tris), SHELL_BLOCK>>>(n_tris, X.data(), S->tris.data(), S->IB.data(),
                                                           S->area.data());
            B2S_CHECK_LAUNCH();
            if(nh > 0)
            {
                k_hinge_rest<<<grid_of(nh), SHELL_BLOCK>>>(nh, X.data(), S->hinges.data(), S->rest3.data());
                B2S_CHECK_LAUNCH();
            }
            B2S_CUDA(cudaDeviceSynchronize());
            *out = S;
        });
}

int b2gen_shell_destroy(b2gen_shell* s)
{
    delete s;
    return 0;
}

int64_t b2gen_shell_num_triplets(const b2gen_shell* s)
{
    return s ? (int64_t)s->nv + 6ll * s->nt + 10ll * s->nh : -1;
}

int32_t b2gen_shell_num_hinges(const b2gen_shell* s) { return s ? s->nh : -1; }

int b2gen_shell_system(b2gen_shell* s, const double* d_x, const double* d_xtilde, int32_t vertex_offset,
                       int32_t* d_rows, int32_t* d_cols, double* d_vals, double* d_grad, void* stream)
{
    return guarded_gen(
        [&]
        {
            if(!s || !d_x || !d_xtilde || !d_rows || !d_cols || !d_vals || !d_grad || vertex_offset < 0)
                fail("b2gen_shell_system: bad arguments");
            B2S_CUDA(cudaSetDevice(s->device));
            cudaStream_t                st  = static_cast<cudaStream_t>(stream);
            const b2gen_shell_material& c   = s->mat;
            const double                dt2 = c.dt * c.dt;
            k_shell_bw<<<grid_of(s->nt), SHELL_BLOCK, 0, st>>>(s->nv, s->nt, vertex_offset, s->tris.data(),
                                                               s->IB.data(), s->area.data(), d_x, c.stretch, c.shear,
                                                               c.strain_rate, dt2, d_rows, d_cols, d_vals,
                                                               s->tri_g.data());
            B2S_CHECK_LAUNCH();
            if(s->nh > 0)
            {
                k_shell_dsb<<<grid_of(s->nh), SHELL_BLOCK, 0, st>>>(s->nv, s->nt, s->nh, vertex_offset,
                                                                    s->hinges.data(), s->rest3.data(), d_x, c.bend,
                                                                    dt2, d_rows, d_cols, d_vals, s->hinge_g.data());
                B2S_CHECK_LAUNCH();
            }
            k_shell_vertex<<<grid_of(s->nv), SHELL_BLOCK, 0, st>>>(s->nv, vertex_offset, s->mass.data(), d_x,
                                                                   d_xtilde, s->inc_start.data(), s->inc_list.data(),
                                                                   s->nt, s->tri_g.data(), s->hinge_g.data(), d_rows,
                                                                   d_cols, d_vals, d_grad);
            B2S_CHECK_LAUNCH();
            if(s->fixed.size() > 0)
            {
                const int64_t T = b2gen_shell_num_triplets(s);
                k_shell_fixed<<<grid_of(std::max<int64_t>(T, s->nv)), SHELL_BLOCK, 0, st>>>(
                    T, s->nv, vertex_offset, s->fixed.data(), d_rows, d_cols, d_vals, d_grad);
                B2S_CHECK_LAUNCH();
            }
            B2S_CUDA(cudaStreamSynchronize(st));
        });
}

int b2gen_abd_create(int device, int32_t n_bodies, const double* mass12, const double* kappa, const double* volume,
                     double dt, b2gen_abd** out)
{
    return guarded_gen(
        [&]
        {
            if(!out || !mass12 || !kappa || !volume || n_bodies <= 0 || !(dt > 0.0))
                fail("b2gen_abd_create: bad arguments");
            B2S_CUDA(cudaSetDevice(device));
            auto A    = new b2gen_abd();
            A->device = device;
            A->nb     = n_bodies;
            A->dt     = dt;
            A->M.resize(144 * (size_t)n_bodies);
            A->kappa.resize(n_bodies);
            A->volume.resize(n_bodies);
            B2S_CUDA(cudaMemcpy(A->M.data(), mass12, A->M.bytes(), cudaMemcpyHostToDevice));
            B2S_CUDA(cudaMemcpy(A->kappa.data(), kappa, A->kappa.bytes(), cudaMemcpyHostToDevice));
            B2S_CUDA(cudaMemcpy(A->volume.data(), volume, A->volume.bytes(), cudaMemcpyHostToDevice));
            *out = A;
        });
}

int b2gen_abd_destroy(b2gen_abd* a)
{
    delete a;
    return 0;
}

int b2gen_abd_system(b2gen_abd* a, const double* d_q, const double* d_qtilde, int32_t block_offset,
                     int32_t* d_rows, int32_t* d_cols, double* d_vals, double* d_grad, void* stream)
{
    return guarded_gen(
        [&]
        {
            if(!a || !d_q || !d_qtilde || !d_rows || !d_cols || !d_vals || !d_grad || block_offset < 0)
                fail("b2gen_abd_system: bad arguments");
            B2S_CUDA(cudaSetDevice(a->device));
            cudaStream_t st = static_cast<cudaStream_t>(stream);
            k_abd<<<grid_of(a->nb), SHELL_BLOCK, 0, st>>>(a->nb, block_offset, a->M.data(), a->kappa.data(),
                                                          a->volume.data(), d_q, d_qtilde, a->dt * a->dt, d_rows,
                                                          d_cols, d_vals, d_grad);
            B2S_CHECK_LAUNCH();
            B2S_CUDA(cudaStreamSynchronize(st));
        });
}

int b2gen_contacts_create(int device, int32_t n_pairs, const int32_t* pairs, const uint8_t* is_ee,
                          const double* eps, double dhat, double kappa, double dt, b2gen_contacts** out)
{
    return guarded_gen(
        [&]
        {
            if(!out || n_pairs <= 0 || !pairs || !is_ee || !eps || !(dhat > 0.0) || !(dt > 0.0))
                fail("b2gen_contacts_create: bad arguments");
            int32_t vmax = -1;
            for(int64_t i = 0; i < 4ll * n_pairs; ++i)
            {
                if(pairs[i] < 0)
                    fail("b2gen_contacts_create: negative vertex index");
                vmax = std::max(vmax, pairs[i]);
            }
            // incidences of each touched vertex, in pair order
            std::vector<int32_t> count((size_t)vmax + 1, 0);
            for(int64_t i = 0; i < 4ll * n_pairs; ++i)
                ++count[pairs[i]];
            std::vector<int32_t> verts, start{0}, slot((size_t)vmax + 1, -1);
            for(int32_t v = 0; v <= vmax; ++v)
                if(count[v])
                {
                    slot[v] = (int32_t)verts.size();
                    verts.push_back(v);
                    start.push_back(start.back() + count[v]);
                }
            std::vector<int32_t> list(4 * (size_t)n_pairs), fill(start.begin(), start.end() - 1);
            for(int32_t p = 0; p < n_pairs; ++p)
                for(int c = 0; c < 4; ++c)
                    list[fill[slot[pairs[4 * p + c]]]++] = 4 * p + c;
            B2S_CUDA(cudaSetDevice(device));
            auto C    = new b2gen_contacts();
            C->device = device;
            C->np     = n_pairs;
            C->nvert  = (int32_t)verts.size();
            C->dhat   = dhat;
            C->kappa  = kappa;
            C->dt     = dt;
            C->pairs.resize(4 * (size_t)n_pairs);
            C->is_ee.resize(n_pairs);
            C->eps.resize(n_pairs);
            C->pair_g.resize(12 * (size_t)n_pairs);
            C->pair_type.resize(n_pairs);
            C->verts.resize(verts.size());
            C->start.resize(start.size());
            C->list.resize(list.size());
            B2S_CUDA(cudaMemcpy(C->pairs.data(), pairs, C->pairs.bytes(), cudaMemcpyHostToDevice));
            B2S_CUDA(cudaMemcpy(C->is_ee.data(), is_ee, C->is_ee.bytes(), cudaMemcpyHostToDevice));
            B2S_CUDA(cudaMemcpy(C->eps.data(), eps, C->eps.bytes(), cudaMemcpyHostToDevice));
            B2S_CUDA(cudaMemcpy(C->verts.data(), verts.data(), C->verts.bytes(), cudaMemcpyHostToDevice));
            B2S_CUDA(cudaMemcpy(C->start.data(), start.data(), C->start.bytes(), cudaMemcpyHostToDevice));
            B2S_CUDA(cudaMemcpy(C->list.data(), list.data(), C->list.bytes(), cudaMemcpyHostToDevice));
            *out = C;
        });
}

int b2gen_contacts_types(b2gen_contacts* c, int8_t* h_types)
{
    return guarded_gen(
        [&]
        {
            if(!c || !h_types)
                fail("b2gen_contacts_types: bad arguments");
            B2S_CUDA(cudaSetDevice(c->device));
            B2S_CUDA(cudaMemcpy(h_types, c->pair_type.data(), c->pair_type.bytes(), cudaMemcpyDeviceToHost));
        });
}

int b2gen_contacts_destroy(b2gen_contacts* c)
{
    delete c;
    return 0;
}

int b2gen_contacts_system(b2gen_contacts* c, const double* d_x, int32_t* d_rows, int32_t* d_cols, double* d_vals,
                          double* d_grad, void* stream)
{
    return guarded_gen(
        [&]
        {
            if(!c || !d_x || !d_rows || !d_cols || !d_vals || !d_grad)
                fail("b2gen_contacts_system: bad arguments");
            B2S_CUDA(cudaSetDevice(c->device));
            cudaStream_t st = static_cast<cudaStream_t>(stream);
            k_contacts<<<(c->np + CONTACT_BLOCK - 1) / CONTACT_BLOCK, CONTACT_BLOCK, 0, st>>>(
                c->np, c->pairs.data(), c->is_ee.data(), c->eps.data(), d_x, c->dhat, c->kappa * c->dt * c->dt, d_rows,
                d_cols, d_vals, c->pair_g.data(), c->pair_type.data());
            B2S_CHECK_LAUNCH();
            k_contacts_gather<<<grid_of(c->nvert), SHELL_BLOCK, 0, st>>>(c->nvert, c->verts.data(), c->start.data(),
                                                                         c->list.data(), c->pair_g.data(), d_grad);
            B2S_CHECK_LAUNCH();
            B2S_CUDA(cudaStreamSynchronize(st));
        });
}

int b2gen_contacts_energy(b2gen_contacts* c, const double* d_x, double* h_energy, void* stream)
{
    return guarded_gen(
        [&]
        {
            if(!c || !d_x || !h_energy)
                fail("b2gen_contacts_energy: null argument");
            B2S_CUDA(cudaSetDevice(c->device));
            cudaStream_t st = static_cast<cudaStream_t>(stream);
            c->terms.resize(c->np);
            c->result.resize(1);
            k_contact_energy<<<grid_of(c->np), SHELL_BLOCK, 0, st>>>(c->np, c->pairs.data(), c->is_ee.data(),
                                                                      c->eps.data(), d_x, c->dhat,
                                                                      c->kappa * c->dt * c->dt, c->terms.data());
            B2S_CHECK_LAUNCH();
            b2s::k_fixed_reduce<<<1, b2s::SUM_THREADS, 0, st>>>(c->np, c->terms.data(), 0, c->result.data());
            B2S_CHECK_LAUNCH();
            B2S_CUDA(cudaMemcpyAsync(h_energy, c->result.data(), sizeof(double), cudaMemcpyDeviceToHost, st));
            B2S_CUDA(cudaStreamSynchronize(st));
        });
}

int b2gen_contacts_toi(b2gen_contacts* c, const double* d_x, const double* d_dx, double alpha, double* h_toi,
                       void* stream)
{
    return guarded_gen(
        [&]
        {
            if(!c || !d_x || !d_dx || !h_toi || !(alpha > 0.0))
                fail("b2gen_contacts_toi: bad arguments");
            B2S_CUDA(cudaSetDevice(c->device));
            cudaStream_t st = static_cast<cudaStream_t>(stream);
            c->terms.resize(c->np);
            c->result.resize(1);
            b2s::k_contact_toi<<<grid_of(c->np), SHELL_BLOCK, 0, st>>>(c->np, c->pairs.data(), c->is_ee.data(), d_x,
                                                                   d_dx, alpha, c->dhat, 0.0, b2s::CCD_ETA, b2s::CCD_MAX_ITER,
                                                                   c->terms.data());
            B2S_CHECK_LAUNCH();
            b2s::k_fixed_reduce<<<1, b2s::SUM_THREADS, 0, st>>>(c->np, c->terms.data(), 1, c->result.data());
            B2S_CHECK_LAUNCH();
            double toi = b2s::TOI_NONE;
            B2S_CUDA(cudaMemcpyAsync(&toi, c->result.data(), sizeof(double), cudaMemcpyDeviceToHost, st));
            B2S_CUDA(cudaStreamSynchronize(st));
            *h_toi = toi < 1.0 ? toi : 1.0;
        });
}

}  // extern "C"
