// Newton systems of tet meshes generated on the GPU (include/b200gen.h):
// kinetic + stable Neo-Hookean (PSD-projected) + ground barrier + Dirichlet
// vertices, straight into device triplet buffers. The arithmetic restates the
// host generator (csrc/scene/scene_gen.cpp: snh_derivatives, jacobi_eigen,
// the kinetic / elastic / ground / fixed passes) per element; results agree
// with it to rounding (FMA contraction on the device).
#include "b2s_fixed_reduce.cuh"
#include "b2s_internal.cuh"

#include "../../include/b200gen.h"

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

namespace
{
thread_local std::string g_gen_err;

constexpr int GEN_BLOCK = 128;

struct DevMesh
{
    int32_t nv = 0, nt = 0, ng = 0;
    b2s::DBuf<int32_t> tets;      // [nt*4]
    b2s::DBuf<double>  vol;       // [nt]
    b2s::DBuf<double>  grad;      // [nt*12] shape gradients g_q[b]
    b2s::DBuf<double>  mass;      // [nv]
    b2s::DBuf<uint8_t> fixed;     // [nv] (empty: none)
    b2s::DBuf<int32_t> vt_start;  // [nv+1] incident (tet, corner) pairs by tet index
    b2s::DBuf<int32_t> vt_list;   // [4 nt]: t * 4 + q
    b2s::DBuf<int32_t> ground;    // [ng]
    b2s::DBuf<double>  tet_g;     // [nt*12] per-tet gradient scratch
    b2gen_material     mat{};
    int                device = 0;
};

// ---- stable Neo-Hookean: dPsi/dF and the PSD-projected d2Psi/dF2 -----------
__device__ void jacobi_eigen9(double* a, double* w, double* v)
{
    for(int i = 0; i < 81; ++i)
        v[i] = 0.0;
    for(int i = 0; i < 9; ++i)
        v[i * 9 + i] = 1.0;
    for(int sweep = 0; sweep < 60; ++sweep)
    {
        double off = 0.0, diag = 0.0;
        for(int p = 0; p < 9; ++p)
        {
            diag += a[p * 9 + p] * a[p * 9 + p];
            for(int q = p + 1; q < 9; ++q)
                off += a[p * 9 + q] * a[p * 9 + q];
        }
        if(off <= 1e-30 * (diag + 1e-300))
            break;
        for(int p = 0; p < 9; ++p)
            for(int q = p + 1; q < 9; ++q)
            {
                const double apq = a[p * 9 + q];
                if(fabs(apq) < 1e-300)
                    continue;
                const double app = a[p * 9 + p], aqq = a[q * 9 + q];
                const double theta = (aqq - app) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for(int k = 0; k < 9; ++k)
                {
                    const double akp = a[k * 9 + p], akq = a[k * 9 + q];
                    a[k * 9 + p] = c * akp - s * akq;
                    a[k * 9 + q] = s * akp + c * akq;
                }
                for(int k = 0; k < 9; ++k)
                {
                    const double apk = a[p * 9 + k], aqk = a[q * 9 + k];
                    a[p * 9 + k] = c * apk - s * aqk;
                    a[q * 9 + k] = s * apk + c * aqk;
                }
                for(int k = 0; k < 9; ++k)
                {
                    const double vkp = v[k * 9 + p], vkq = v[k * 9 + q];
                    v[k * 9 + p] = c * vkp - s * vkq;
                    v[k * 9 + q] = s * vkp + c * vkq;
                }
            }
    }
    for(int i = 0; i < 9; ++i)
        w[i] = a[i * 9 + i];
}

// F column-major; P = dPsi/dF, H = d2Psi/dF2 (vec(F) column-major), PSD
__device__ void snh_derivatives(const double F[9], double mu, double lambda, double P[9], double H[81])
{
    const double f0[3] = {F[0], F[1], F[2]}, f1[3] = {F[3], F[4], F[5]}, f2[3] = {F[6], F[7], F[8]};
    auto cross = [](const double* a, const double* b, double* c) {
        c[0] = a[1] * b[2] - a[2] * b[1];
        c[1] = a[2] * b[0] - a[0] * b[2];
        c[2] = a[0] * b[1] - a[1] * b[0];
    };
    double g[9];
    cross(f1, f2, g);
    cross(f2, f0, g + 3);
    cross(f0, f1, g + 6);
    const double J = f0[0] * g[0] + f0[1] * g[1] + f0[2] * g[2];
    const double s = lambda * (J - 1.0) - mu;
    for(int i = 0; i < 9; ++i)
        P[i] = mu * F[i] + s * g[i];
    for(int i = 0; i < 9; ++i)
        for(int j = 0; j < 9; ++j)
            H[i * 9 + j] = (i == j ? mu : 0.0) + lambda * g[i] * g[j];
    // d2J/df_a df_b: (0,1) = -[f2]x, (0,2) = [f1]x, (1,2) = -[f0]x (and transposes)
    auto put_cross = [&](int bi, int bj, const double* a, double sign) {
        const double m[9] = {0, -a[2], a[1], a[2], 0, -a[0], -a[1], a[0], 0};  // row-major [a]x
        for(int r = 0; r < 3; ++r)
            for(int c = 0; c < 3; ++c)
            {
                const double v = sign * s * m[r * 3 + c];
                H[(bi * 3 + r) * 9 + (bj * 3 + c)] += v;
                H[(bj * 3 + c) * 9 + (bi * 3 + r)] += v;
            }
    };
    put_cross(0, 1, f2, -1.0);
    put_cross(0, 2, f1, +1.0);
    put_cross(1, 2, f0, -1.0);
    double a[81], w[9], v[81];
    for(int i = 0; i < 81; ++i)
        a[i] = H[i];
    jacobi_eigen9(a, w, v);
    bool neg = false;
    for(int i = 0; i < 9; ++i)
        neg |= (w[i] < 0.0);
    if(!neg)
        return;
    for(int i = 0; i < 9; ++i)
        for(int j = 0; j < 9; ++j)
        {
            double acc = 0.0;
            for(int k = 0; k < 9; ++k)
                if(w[k] > 0.0)
                    acc += v[i * 9 + k] * w[k] * v[j * 9 + k];
            H[i * 9 + j] = acc;
        }
}

// a row-major 3x3 block of the pair (ra, rb) into slot k, upper orientation
__device__ __forceinline__ void write_block(int64_t k, int32_t ra, int32_t rb, const double* Hab, int32_t* rows,
                                            int32_t* cols, double* vals)
{
    const bool tp = ra > rb;
    rows[k]       = tp ? rb : ra;
    cols[k]       = tp ? ra : rb;
    double* V     = vals + k * 9;
    for(int p = 0; p < 3; ++p)
        for(int q = 0; q < 3; ++q)
            V[q * 3 + p] = tp ? Hab[q * 3 + p] : Hab[p * 3 + q];  // column-major
}

// ---- kernels -----------------------------------------------------------------
__global__ void k_rest(int nt, const double* __restrict__ X, const int32_t* __restrict__ tets, double rho,
                       double* __restrict__ vol, double* __restrict__ G)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if(t >= nt)
        return;
    const int32_t* T = tets + (int64_t)t * 4;
    double         e[3][3];
    for(int q = 0; q < 3; ++q)
        for(int a = 0; a < 3; ++a)
            e[q][a] = X[T[q + 1] * 3 + a] - X[T[0] * 3 + a];
    auto cross = [](const double* a, const double* b, double* c) {
        c[0] = a[1] * b[2] - a[2] * b[1];
        c[1] = a[2] * b[0] - a[0] * b[2];
        c[2] = a[0] * b[1] - a[1] * b[0];
    };
    double c12[3], c20[3], c01[3];
    cross(e[1], e[2], c12);
    cross(e[2], e[0], c20);
    cross(e[0], e[1], c01);
    const double det = e[0][0] * c12[0] + e[0][1] * c12[1] + e[0][2] * c12[2];
    vol[t]           = det / 6.0;
    double* g        = G + (int64_t)t * 12;
    for(int b = 0; b < 3; ++b)
    {
        const double r0 = c12[b] / det, r1 = c20[b] / det, r2 = c01[b] / det;
        g[3 + b] = r0;
        g[6 + b] = r1;
        g[9 + b] = r2;
        g[b]     = -(r0 + r1 + r2);
    }
}

// lumped masses, in tet order per vertex (the host generator's sum order)
__global__ void k_mass(int nv, const int32_t* __restrict__ vt_start, const int32_t* __restrict__ vt_list,
                       const double* __restrict__ vol, double rho, double* __restrict__ mass)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if(v >= nv)
        return;
    double m = 0.0;
    for(int e = vt_start[v]; e < vt_start[v + 1]; ++e)
        m += rho * vol[vt_list[e] >> 2] * 0.25;
    mass[v] = m;
}

__global__ void __launch_bounds__(GEN_BLOCK) k_elastic(int nv, int nt, const int32_t* __restrict__ tets,
                                                       const double* __restrict__ vol,
                                                       const double* __restrict__ G, const double* __restrict__ x,
                                                       double mu, double lambda, double dt2, int32_t* rows,
                                                       int32_t* cols, double* vals, double* __restrict__ tet_g)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if(t >= nt)
        return;
    const int32_t* T  = tets + (int64_t)t * 4;
    const double*  Gs = G + (int64_t)t * 12;
    double         F[9] = {0};
    for(int q = 0; q < 4; ++q)
        for(int a = 0; a < 3; ++a)
            for(int b = 0; b < 3; ++b)
                F[a + 3 * b] += x[T[q] * 3 + a] * Gs[q * 3 + b];
    double P[9], H[81];
    snh_derivatives(F, mu, lambda, P, H);
    const double s = vol[t] * dt2;
    for(int q = 0; q < 4; ++q)
        for(int a = 0; a < 3; ++a)
        {
            double acc = 0.0;
            for(int b = 0; b < 3; ++b)
                acc += P[a + 3 * b] * Gs[q * 3 + b];
            tet_g[(int64_t)t * 12 + q * 3 + a] = s * acc;
        }
    int slot = 0;
    for(int q = 0; q < 4; ++q)
        for(int r = q; r < 4; ++r, ++slot)
        {
            double Hb[9];
            for(int a = 0; a < 3; ++a)
                for(int c = 0; c < 3; ++c)
                {
                    double acc = 0.0;
                    for(int b = 0; b < 3; ++b)
                    {
                        const double gq = Gs[q * 3 + b];
                        for(int d = 0; d < 3; ++d)
                            acc += gq * H[(a + 3 * b) * 9 + (c + 3 * d)] * Gs[r * 3 + d];
                    }
                    Hb[a * 3 + c] = s * acc;
                }
            if(q == r)  // exact symmetry of diagonal blocks
                for(int a = 0; a < 3; ++a)
                    for(int c = a + 1; c < 3; ++c)
                    {
                        const double m = 0.5 * (Hb[a * 3 + c] + Hb[c * 3 + a]);
                        Hb[a * 3 + c] = Hb[c * 3 + a] = m;
                    }
            write_block((int64_t)nv + (int64_t)t * 10 + slot, T[q], T[r], Hb, rows, cols, vals);
        }
}

// kinetic block and the gradient (kinetic, tets by index, ground) per vertex
__global__ void k_vertex(int nv, int nt, const double* __restrict__ mass, const double* __restrict__ x,
                         const double* __restrict__ xt, const int32_t* __restrict__ vt_start,
                         const int32_t* __restrict__ vt_list, const double* __restrict__ tet_g, int32_t* rows,
                         int32_t* cols, double* vals, double* __restrict__ grad)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if(v >= nv)
        return;
    const double m    = mass[v];
    const double H[9] = {m, 0, 0, 0, m, 0, 0, 0, m};
    write_block(v, v, v, H, rows, cols, vals);
    double g[3];
    for(int a = 0; a < 3; ++a)
        g[a] = m * (x[(int64_t)v * 3 + a] - xt[(int64_t)v * 3 + a]);
    for(int e = vt_start[v]; e < vt_start[v + 1]; ++e)
    {
        const int tq = vt_list[e];  // t * 4 + q
        for(int a = 0; a < 3; ++a)
            g[a] += tet_g[(int64_t)(tq >> 2) * 12 + (tq & 3) * 3 + a];
    }
    for(int a = 0; a < 3; ++a)
        grad[(int64_t)v * 3 + a] = g[a];
}

// ground barrier (normal +y) on the candidates: one diagonal block each
__global__ void k_ground(int nv, int nt, int ng, const int32_t* __restrict__ ground, const double* __restrict__ x,
                         double ground_y, double dhat, double kappa, double dt2, int32_t* rows, int32_t* cols,
                         double* vals, double* __restrict__ grad)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= ng)
        return;
    const int32_t g   = ground[i];
    const double  d   = x[(int64_t)g * 3 + 1] - ground_y;
    double        k   = 0.0, gy = 0.0;
    if(d < dhat)
    {
        const double D = d * d, Dh = dhat * dhat, tt = D - Dh, l = log(D / Dh);
        const double b1 = -2.0 * tt * l - tt * tt / D;
        const double b2 = -2.0 * l - 4.0 * tt / D + tt * tt / (D * D);
        k               = fmax(0.0, dt2 * kappa * (b2 * 4.0 * D + 2.0 * b1));
        gy              = dt2 * kappa * b1 * 2.0 * d;
    }
    const double H[9] = {0, 0, 0, 0, k, 0, 0, 0, 0};
    write_block((int64_t)nv + (int64_t)nt * 10 + i, g, g, H, rows, cols, vals);
    // one candidate per vertex: the add keeps the order kinetic, tets, ground
    grad[(int64_t)g * 3 + 1] += gy;
}

// Dirichlet vertices: their rows / columns zero, diagonal I, gradient 0
__global__ void k_fixed(int64_t T, int nv, const uint8_t* __restrict__ fixed, const int32_t* __restrict__ rows,
                        const int32_t* __restrict__ cols, double* vals, double* grad)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(s < T)
    {
        const int32_t i = rows[s], j = cols[s];
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
        grad[s * 3] = grad[s * 3 + 1] = grad[s * 3 + 2] = 0.0;
}

int grid_of(int64_t n) { return (int)((n + GEN_BLOCK - 1) / GEN_BLOCK); }

// ---- energy and the ground's time of impact (the line search after the solve) ----
// per-term energies: kinetic 1/2 m |x - x_tilde|^2 per vertex, dt^2 vol Psi(F)
// per tet with Psi = mu/2 (|F|^2 - 3) - mu (J - 1) + lambda/2 (J - 1)^2 (the
// potential whose derivatives k_elastic writes), dt^2 kappa b(d^2) per ground
// candidate (infinite at or below the plane)
__global__ void k_energy_terms(int nv, int nt, int ng, const int32_t* __restrict__ tets, const double* __restrict__ vol,
                               const double* __restrict__ G, const double* __restrict__ mass,
                               const int32_t* __restrict__ ground, const double* __restrict__ x,
                               const double* __restrict__ xt, double mu, double lambda, double dt2, double ground_y,
                               double dhat, double kappa, double* __restrict__ e)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(i < nv)
    {
        double d2 = 0.0;
        for(int a = 0; a < 3; ++a)
        {
            const double d = x[i * 3 + a] - xt[i * 3 + a];
            d2 += d * d;
        }
        e[i] = 0.5 * mass[i] * d2;
    }
    else if(i < (int64_t)nv + nt)
    {
        const int64_t  t  = i - nv;
        const int32_t* T  = tets + t * 4;
        const double*  Gs = G + t * 12;
        double         F[9] = {0};
        for(int q = 0; q < 4; ++q)
            for(int a = 0; a < 3; ++a)
                for(int b = 0; b < 3; ++b)
                    F[a + 3 * b] += x[T[q] * 3 + a] * Gs[q * 3 + b];
        const double J = F[0] * (F[4] * F[8] - F[7] * F[5]) - F[3] * (F[1] * F[8] - F[7] * F[2]) +
                         F[6] * (F[1] * F[5] - F[4] * F[2]);
        double f2 = 0.0;
        for(int k = 0; k < 9; ++k)
            f2 += F[k] * F[k];
        const double psi = 0.5 * mu * (f2 - 3.0) - mu * (J - 1.0) + 0.5 * lambda * (J - 1.0) * (J - 1.0);
        e[i]             = dt2 * vol[t] * psi;
    }
    else if(i < (int64_t)nv + nt + ng)
    {
        const int32_t g = ground[i - nv - nt];
        const double  d = x[(int64_t)g * 3 + 1] - ground_y;
        double        v = 0.0;
        if(!(d > 0.0))
            v = INFINITY;
        else if(d < dhat)
        {
            const double D = d * d, Dh = dhat * dhat, tt = D - Dh;
            v              = -dt2 * kappa * tt * tt * log(D / Dh);
        }
        e[i] = v;
    }
}

// time of impact with the ground plane (normal +y) of every candidate moving
// along d: (1 - eta) (y - ground_y) / (-d_y) when it moves down, else 1.1
__global__ void k_ground_toi(int ng, const int32_t* __restrict__ ground, const double* __restrict__ x,
                             const double* __restrict__ dx, double ground_y, double eta, double* __restrict__ toi)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= ng)
        return;
    const int32_t g = ground[i];
    const double  t = -dx[(int64_t)g * 3 + 1];  // approach speed along -normal
    double        v = 1.1;
    if(t > 0.0)
        v = (x[(int64_t)g * 3 + 1] - ground_y) / t * (1.0 - eta);
    toi[i] = v;
}
}  // namespace

struct b2gen_mesh : DevMesh
{
    b2s::DBuf<double> terms;  // per-term energies / times of impact
    b2s::DBuf<double> result;
};

extern "C" {

const char* b2gen_last_error(void) { return g_gen_err.c_str(); }

int b2gen_mesh_create(int device, int32_t n_verts, int32_t n_tets, const double* rest, const int32_t* tets,
                      const uint8_t* fixed, int32_t n_ground, const int32_t* ground, const b2gen_material* mat,
                      b2gen_mesh** out)
{
    try
    {
        if(!out || !rest || !tets || !mat || n_verts <= 0 || n_tets <= 0 || n_ground < 0 ||
           (n_ground > 0 && !ground))
            throw b2s::Error(B2S_ERR_ARGUMENT, "b2gen_mesh_create: bad arguments");
        if((int64_t)n_verts + 10ll * n_tets + n_ground > (int64_t)INT32_MAX)
            throw b2s::Error(B2S_ERR_ARGUMENT, "b2gen_mesh_create: too many triplets for 32-bit slots");
        for(int64_t i = 0; i < 4ll * n_tets; ++i)
            if(tets[i] < 0 || tets[i] >= n_verts)
                throw b2s::Error(B2S_ERR_ARGUMENT, "b2gen_mesh_create: tet vertex out of range");
        for(int32_t i = 0; i < n_ground; ++i)
            if(ground[i] < 0 || ground[i] >= n_verts)
                throw b2s::Error(B2S_ERR_ARGUMENT, "b2gen_mesh_create: ground vertex out of range");
        B2S_CUDA(cudaSetDevice(device));
        auto M    = new b2gen_mesh();
        M->device = device;
        M->nv     = n_verts;
        M->nt     = n_tets;
        M->ng     = n_ground;
        M->mat    = *mat;
        // vertex -> (tet, corner) incidence, by tet index
        std::vector<int32_t> start(n_verts + 1, 0), list(4 * (size_t)n_tets);
        for(int64_t i = 0; i < 4ll * n_tets; ++i)
            ++start[tets[i] + 1];
        for(int32_t v = 0; v < n_verts; ++v)
            start[v + 1] += start[v];
        std::vector<int32_t> fill(start.begin(), start.end() - 1);
        for(int32_t t = 0; t < n_tets; ++t)
            for(int q = 0; q < 4; ++q)
                list[fill[tets[4 * t + q]]++] = 4 * t + q;
        b2s::DBuf<double> X;
        X.resize((size_t)n_verts * 3);
        M->tets.resize(4 * (size_t)n_tets);
        M->vol.resize(n_tets);
        M->grad.resize(12 * (size_t)n_tets);
        M->mass.resize(n_verts);
        M->vt_start.resize(n_verts + 1);
        M->vt_list.resize(list.size());
        M->tet_g.resize(12 * (size_t)n_tets);
        B2S_CUDA(cudaMemcpy(X.data(), rest, X.bytes(), cudaMemcpyHostToDevice));
        B2S_CUDA(cudaMemcpy(M->tets.data(), tets, M->tets.bytes(), cudaMemcpyHostToDevice));
        B2S_CUDA(cudaMemcpy(M->vt_start.data(), start.data(), M->vt_start.bytes(), cudaMemcpyHostToDevice));
        B2S_CUDA(cudaMemcpy(M->vt_list.data(), list.data(), M->vt_list.bytes(), cudaMemcpyHostToDevice));
        if(fixed)
        {
            M->fixed.resize(n_verts);
            B2S_CUDA(cudaMemcpy(M->fixed.data(), fixed, n_verts, cudaMemcpyHostToDevice));
        }
        if(n_ground > 0)
        {
            M->ground.resize(n_ground);
            B2S_CUDA(cudaMemcpy(M->ground.data(), ground, sizeof(int32_t) * n_ground, cudaMemcpyHostToDevice));
        }
        k_rest<<<grid_of(n_tets), GEN_BLOCK>>>(n_tets, X.data(), M->tets.data(), mat->rho, M->vol.data(),
                                               M->grad.data());
        B2S_CHECK_LAUNCH();
        k_mass<<<grid_of(n_verts), GEN_BLOCK>>>(n_verts, M->vt_start.data(), M->vt_list.data(), M->vol.data(),
                                                mat->rho, M->mass.data());
        B2S_CHECK_LAUNCH();
        B2S_CUDA(cudaDeviceSynchronize());
        *out = M;
        return 0;
    }
    catch(const b2s::Error& e)
    {
        g_gen_err = e.what();
        return e.code;
    }
    catch(const std::exception& e)
    {
        g_gen_err = e.what();
        return B2S_ERR_CUDA;
    }
}

int b2gen_mesh_destroy(b2gen_mesh* m)
{
    delete m;
    return 0;
}

int64_t b2gen_num_triplets(const b2gen_mesh* m)
{
    return m ? (int64_t)m->nv + 10ll * m->nt + m->ng : -1;
}

int b2gen_system(b2gen_mesh* m, const double* d_x, const double* d_xtilde, int32_t* d_rows, int32_t* d_cols,
                 double* d_vals, double* d_grad, void* stream)
{
    try
    {
        if(!m || !d_x || !d_xtilde || !d_rows || !d_cols || !d_vals || !d_grad)
            throw b2s::Error(B2S_ERR_ARGUMENT, "b2gen_system: null argument");
        B2S_CUDA(cudaSetDevice(m->device));
        cudaStream_t      st  = static_cast<cudaStream_t>(stream);
        const b2gen_material& c = m->mat;
        const double      dt2 = c.dt * c.dt;
        k_elastic<<<grid_of(m->nt), GEN_BLOCK, 0, st>>>(m->nv, m->nt, m->tets.data(), m->vol.data(), m->grad.data(),
                                                        d_x, c.mu, c.lambda, dt2, d_rows, d_cols, d_vals,
                                                        m->tet_g.data());
        B2S_CHECK_LAUNCH();
        k_vertex<<<grid_of(m->nv), GEN_BLOCK, 0, st>>>(m->nv, m->nt, m->mass.data(), d_x, d_xtilde,
                                                       m->vt_start.data(), m->vt_list.data(), m->tet_g.data(), d_rows,
                                                       d_cols, d_vals, d_grad);
        B2S_CHECK_LAUNCH();
        if(m->ng > 0)
        {
            k_ground<<<grid_of(m->ng), GEN_BLOCK, 0, st>>>(m->nv, m->nt, m->ng, m->ground.data(), d_x, c.ground_y,
                                                           c.dhat, c.kappa, dt2, d_rows, d_cols, d_vals, d_grad);
            B2S_CHECK_LAUNCH();
        }
        if(m->fixed.size() > 0)
        {
            const int64_t T = b2gen_num_triplets(m);
            k_fixed<<<grid_of(std::max<int64_t>(T, m->nv)), GEN_BLOCK, 0, st>>>(T, m->nv, m->fixed.data(), d_rows,
                                                                                 d_cols, d_vals, d_grad);
            B2S_CHECK_LAUNCH();
        }
        B2S_CUDA(cudaStreamSynchronize(st));
        return 0;
    }
    catch(const b2s::Error& e)
    {
        g_gen_err = e.what();
        return e.code;
    }
    catch(const std::exception& e)
    {
        g_gen_err = e.what();
        return B2S_ERR_CUDA;
    }
}

int b2gen_energy(b2gen_mesh* m, const double* d_x, const double* d_xtilde, double* h_energy, void* stream)
{
    try
    {
        if(!m || !d_x || !d_xtilde || !h_energy)
            throw b2s::Error(B2S_ERR_ARGUMENT, "b2gen_energy: null argument");
        B2S_CUDA(cudaSetDevice(m->device));
        cudaStream_t          st = static_cast<cudaStream_t>(stream);
        const b2gen_material& c  = m->mat;
        const int64_t         n  = (int64_t)m->nv + m->nt + m->ng;
        m->terms.resize(n);
        m->result.resize(1);
        k_energy_terms<<<grid_of(n), GEN_BLOCK, 0, st>>>(m->nv, m->nt, m->ng, m->tets.data(), m->vol.data(),
                                                         m->grad.data(), m->mass.data(),
                                                         m->ng ? m->ground.data() : nullptr, d_x, d_xtilde, c.mu,
                                                         c.lambda, c.dt * c.dt, c.ground_y, c.dhat, c.kappa,
                                                         m->terms.data());
        B2S_CHECK_LAUNCH();
        b2s::k_fixed_reduce<<<1, b2s::SUM_THREADS, 0, st>>>(n, m->terms.data(), 0, m->result.data());
        B2S_CHECK_LAUNCH();
        B2S_CUDA(cudaMemcpyAsync(h_energy, m->result.data(), sizeof(double), cudaMemcpyDeviceToHost, st));
        B2S_CUDA(cudaStreamSynchronize(st));
        return 0;
    }
    catch(const b2s::Error& e)
    {
        g_gen_err = e.what();
        return e.code;
    }
    catch(const std::exception& e)
    {
        g_gen_err = e.what();
        return B2S_ERR_CUDA;
    }
}

int b2gen_ground_toi(b2gen_mesh* m, const double* d_x, const double* d_dx, double* h_alpha, void* stream)
{
    try
    {
        if(!m || !d_x || !d_dx || !h_alpha)
            throw b2s::Error(B2S_ERR_ARGUMENT, "b2gen_ground_toi: null argument");
        *h_alpha = 1.0;
        if(m->ng == 0)
            return 0;
        B2S_CUDA(cudaSetDevice(m->device));
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        m->terms.resize(m->ng);
        m->result.resize(1);
        k_ground_toi<<<grid_of(m->ng), GEN_BLOCK, 0, st>>>(m->ng, m->ground.data(), d_x, d_dx, m->mat.ground_y, 0.1,
                                                           m->terms.data());
        B2S_CHECK_LAUNCH();
        b2s::k_fixed_reduce<<<1, b2s::SUM_THREADS, 0, st>>>(m->ng, m->terms.data(), 1, m->result.data());
        B2S_CHECK_LAUNCH();
        double toi = 1.1;
        B2S_CUDA(cudaMemcpyAsync(&toi, m->result.data(), sizeof(double), cudaMemcpyDeviceToHost, st));
        B2S_CUDA(cudaStreamSynchronize(st));
        *h_alpha = toi < 1.0 ? toi : 1.0;
        return 0;
    }
    catch(const b2s::Error& e)
    {
        g_gen_err = e.what();
        return e.code;
    }
    catch(const std::exception& e)
    {
        g_gen_err = e.what();
        return B2S_ERR_CUDA;
    }
}

}  // extern "C"
