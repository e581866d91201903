// Synthetic Newton-system generator (host C++, OpenMP). See scene_gen.h.
//
// Physics restated from the formulations libuipc uses (own code):
//  * Stable Neo-Hookean  Psi = lambda/2 (J-1)^2 - mu (J-1) + mu/2 (|F|^2 - 3)
//    (src/backends/cuda/finite_element/constitutions/sym/simplified_stable_neo_hookean_3d.inl),
//    element Hessian projected to PSD through the eigen-decomposition of
//    d2Psi/dF2, scaled by rest volume and dt^2.
//  * BDF1 kinetic term 1/2 m |x - x_tilde|^2, x_tilde = x + dt v + dt^2 g,
//    lumped mass rho V / 4 per tet corner
//    (src/backends/cuda/finite_element/bdf/finite_element_bdf1_kinetic.cu).
//  * Cloth: Baraff-Witkin strain-limiting stretch + shear and discrete-shell
//    bending (Gauss-Newton hinge Hessian), elements.h;
//    affine bodies: the orthogonality potential (elements.h) and the
//    kinetic term of their 12 DoF.
//  * IPC log barrier on squared distance D < dhat^2:
//        b(D) = -(D - Dhat)^2 log(D / Dhat), energy dt^2 kappa b(D).
//    Contact Hessians use the barrier curvature along the fixed contact
//    normal (rank-1 Gauss-Newton form, PSD by construction).
//  * Fixed vertices: every block touching one is written as 0 (off-diagonal)
//    or I (diagonal) and its gradient is zeroed
//    (src/backends/cuda/finite_element/fem_linear_subsystem.cu:23-52).
#include "scene_gen.h"
#include "elements.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace
{
thread_local std::string g_err;

using Vec3 = std::array<double, 3>;
using Mat3 = std::array<double, 9>;  // column-major

inline Vec3 sub(const Vec3& a, const Vec3& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
inline Vec3 add(const Vec3& a, const Vec3& b) { return {a[0] + b[0], a[1] + b[1], a[2] + b[2]}; }
inline Vec3 scale(const Vec3& a, double s) { return {a[0] * s, a[1] * s, a[2] * s}; }
inline double dot(const Vec3& a, const Vec3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline Vec3 cross(const Vec3& a, const Vec3& b)
{
    return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
inline double norm(const Vec3& a) { return std::sqrt(dot(a, a)); }

inline uint64_t splitmix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
// uniform in [-1, 1) from (seed, stream, index)
inline double urand(uint64_t seed, uint64_t stream, uint64_t idx)
{
    uint64_t r = splitmix64(seed * 0x632BE59BD9B4E019ull + stream * 0x9E3779B97F4A7C15ull + idx);
    r          = splitmix64(r);
    return (double)(r >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

// Cyclic Jacobi eigen-decomposition of a symmetric n x n matrix (row-major a),
// eigenvectors in the columns of v (row-major).
template <int N>
void jacobi_eigen(double* a, double* w, double* v)
{
    for(int i = 0; i < N * N; ++i)
        v[i] = 0.0;
    for(int i = 0; i < N; ++i)
        v[i * N + i] = 1.0;
    for(int sweep = 0; sweep < 60; ++sweep)
    {
        double off = 0.0, diag = 0.0;
        for(int p = 0; p < N; ++p)
        {
            diag += a[p * N + p] * a[p * N + p];
            for(int q = p + 1; q < N; ++q)
                off += a[p * N + q] * a[p * N + q];
        }
        if(off <= 1e-30 * (diag + 1e-300))
            break;
        for(int p = 0; p < N; ++p)
            for(int q = p + 1; q < N; ++q)
            {
                double apq = a[p * N + q];
                if(std::fabs(apq) < 1e-300)
                    continue;
                double app = a[p * N + p], aqq = a[q * N + q];
                double theta = (aqq - app) / (2.0 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for(int k = 0; k < N; ++k)
                {
                    double akp = a[k * N + p], akq = a[k * N + q];
                    a[k * N + p] = c * akp - s * akq;
                    a[k * N + q] = s * akp + c * akq;
                }
                for(int k = 0; k < N; ++k)
                {
                    double apk = a[p * N + k], aqk = a[q * N + k];
                    a[p * N + k] = c * apk - s * aqk;
                    a[q * N + k] = s * apk + c * aqk;
                }
                for(int k = 0; k < N; ++k)
                {
                    double vkp = v[k * N + p], vkq = v[k * N + q];
                    v[k * N + p] = c * vkp - s * vkq;
                    v[k * N + q] = s * vkp + c * vkq;
                }
            }
    }
    for(int i = 0; i < N; ++i)
        w[i] = a[i * N + i];
}

// d2Psi/dF2 (9x9, vec(F) column-major) of the stable Neo-Hookean energy,
// projected to PSD; also dPsi/dF. F column-major.
void snh_derivatives(const double F[9], double mu, double lambda, double P[9], double H[81])
{
    const Vec3 f0{F[0], F[1], F[2]}, f1{F[3], F[4], F[5]}, f2{F[6], F[7], F[8]};
    const double J = dot(f0, cross(f1, f2));
    Vec3 g0 = cross(f1, f2), g1 = cross(f2, f0), g2 = cross(f0, f1);
    double g[9] = {g0[0], g0[1], g0[2], g1[0], g1[1], g1[2], g2[0], g2[1], g2[2]};
    const double s = lambda * (J - 1.0) - mu;
    for(int i = 0; i < 9; ++i)
        P[i] = mu * F[i] + s * g[i];
    // H = mu I + lambda g g^T + s * d2J/dF2
    for(int i = 0; i < 9; ++i)
        for(int j = 0; j < 9; ++j)
            H[i * 9 + j] = (i == j ? mu : 0.0) + lambda * g[i] * g[j];
    // d2J/df_a df_b blocks: (0,1) = -[f2]x, (0,2) = [f1]x, (1,2) = -[f0]x (and transposes)
    auto put_cross = [&](int bi, int bj, const Vec3& a, double sign)
    {
        // [a]x = [[0,-a2,a1],[a2,0,-a0],[-a1,a0,0]]
        const double m[9] = {0, -a[2], a[1], a[2], 0, -a[0], -a[1], a[0], 0};  // row-major
        for(int r = 0; r < 3; ++r)
            for(int c = 0; c < 3; ++c)
            {
                double v = sign * s * m[r * 3 + c];
                H[(bi * 3 + r) * 9 + (bj * 3 + c)] += v;
                H[(bj * 3 + c) * 9 + (bi * 3 + r)] += v;
            }
    };
    put_cross(0, 1, f2, -1.0);
    put_cross(0, 2, f1, +1.0);
    put_cross(1, 2, f0, -1.0);
    // PSD projection
    double a[81], w[9], v[81];
    std::memcpy(a, H, sizeof(a));
    jacobi_eigen<9>(a, w, v);
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

// barrier b(D) = -(D - Dh)^2 log(D / Dh), derivatives in D
inline void barrier_d(double D, double Dh, double& b1, double& b2)
{
    const double t = D - Dh;
    const double l = std::log(D / Dh);
    b1 = -2.0 * t * l - t * t / D;
    b2 = -2.0 * l - 4.0 * t / D + t * t / (D * D);
}

struct Triplet
{
    int32_t r, c;
    double  v[9];
};

struct Builder
{
    std::vector<int32_t> rows, cols;
    std::vector<double>  vals;
    void reserve(size_t n)
    {
        rows.reserve(n);
        cols.reserve(n);
        vals.reserve(n * 9);
    }
    // block (r, c) of a row-major element matrix, stored block-upper and
    // column-major (transposed when r > c)
    void put(int32_t r, int32_t c, const double* Hrc)
    {
        const bool tp = r > c;
        rows.push_back(tp ? c : r);
        cols.push_back(tp ? r : c);
        for(int q = 0; q < 3; ++q)
            for(int p = 0; p < 3; ++p)
                vals.push_back(tp ? Hrc[q * 3 + p] : Hrc[p * 3 + q]);
    }
    // the upper blocks of an n-vertex element Hessian (row-major, 3n x 3n)
    template <int NV>
    void put_element(const int32_t* v, const double* H)
    {
        for(int i = 0; i < NV; ++i)
            for(int j = i; j < NV; ++j)
            {
                double blk[9];
                for(int p = 0; p < 3; ++p)
                    for(int q = 0; q < 3; ++q)
                        blk[p * 3 + q] = H[(3 * i + p) * (3 * NV) + 3 * j + q];
                put(v[i], v[j], blk);
            }
    }
};

// Cloth of N x N grid vertices (global block rows off + i + N k), cells
// split along the (i, k)-(i+1, k+1) diagonal; at state x with rest x_rest:
//  * Baraff-Witkin stretch (stiffness `stretch`) and shear (0.1 x stretch),
//    strain rate 100 (the reference's default): 6 triplets per triangle;
//  * discrete-shell bending (stiffness `bend`) on every interior edge, hinge
//    (opposite min, edge min, edge max, opposite max) as the reference orders
//    its stencils: 10 triplets per hinge;
// energies scaled by rest area x dt^2 (stretch) and dt^2 (bending); the
// gradient is added to grad. Returns the triangle count.
int64_t add_cloth_grid(Builder& B, std::vector<double>& grad, const std::vector<double>& x,
                       const std::vector<double>& x_rest, int64_t off, int N, double stretch, double bend, double dt2,
                       std::vector<int32_t>* tris_out = nullptr, std::vector<int32_t>* hinges_out = nullptr)
{
    auto vid = [&](int64_t i, int64_t k) { return (int32_t)(off + i + (int64_t)N * k); };
    std::vector<int32_t> tris;
    tris.reserve((size_t)6 * (N - 1) * (N - 1));
    for(int64_t k = 0; k + 1 < N; ++k)
        for(int64_t i = 0; i + 1 < N; ++i)
        {
            const int32_t a = vid(i, k), b = vid(i + 1, k), c = vid(i + 1, k + 1), d = vid(i, k + 1);
            tris.insert(tris.end(), {a, b, c, a, c, d});
        }
    const int64_t nt = (int64_t)tris.size() / 3;
    const double  shear = 0.1 * stretch, rate = 100.0;
    for(int64_t t = 0; t < nt; ++t)
    {
        const int32_t* v = &tris[3 * t];
        double         IB[4], G[9], H[81];
        b2el::bw_rest(&x_rest[3 * v[0]], &x_rest[3 * v[1]], &x_rest[3 * v[2]], IB);
        const double area = b2el::tri_area(&x_rest[3 * v[0]], &x_rest[3 * v[1]], &x_rest[3 * v[2]]);
        b2el::bw_grad_hess(&x[3 * v[0]], &x[3 * v[1]], &x[3 * v[2]], IB, stretch, shear, rate, area * dt2, G, H);
        B.put_element<3>(v, H);
        for(int i = 0; i < 3; ++i)
            for(int a = 0; a < 3; ++a)
                grad[3 * (size_t)v[i] + a] += G[3 * i + a];
    }
    // hinges: edges with two triangles, in (min, max) edge order
    std::vector<std::array<int32_t, 4>> opp;  // edge min, edge max, opposite, opposite
    opp.reserve((size_t)3 * nt);
    for(int64_t t = 0; t < nt; ++t)
    {
        int32_t T[3] = {tris[3 * t], tris[3 * t + 1], tris[3 * t + 2]};
        std::sort(T, T + 3);
        opp.push_back({T[0], T[1], T[2], 0});
        opp.push_back({T[0], T[2], T[1], 0});
        opp.push_back({T[1], T[2], T[0], 0});
    }
    std::sort(opp.begin(), opp.end());
    std::vector<int32_t> hinges;
    for(size_t e = 0; e + 1 < opp.size();)
    {
        size_t f = e + 1;
        while(f < opp.size() && opp[f][0] == opp[e][0] && opp[f][1] == opp[e][1])
            ++f;
        if(f - e == 2)
            hinges.insert(hinges.end(), {std::min(opp[e][2], opp[e + 1][2]), opp[e][0], opp[e][1],
                                         std::max(opp[e][2], opp[e + 1][2])});
        e = f;
    }
    const int64_t nh = (int64_t)hinges.size() / 4;
    for(int64_t h = 0; h < nh; ++h)
    {
        const int32_t* v = &hinges[4 * h];
        double         L0, hb, thb, G[12], H[144];
        b2el::dsb_rest(&x_rest[3 * v[0]], &x_rest[3 * v[1]], &x_rest[3 * v[2]], &x_rest[3 * v[3]], &L0, &hb, &thb);
        b2el::dsb_grad_hess(&x[3 * v[0]], &x[3 * v[1]], &x[3 * v[2]], &x[3 * v[3]], L0, hb, thb, bend, dt2, G, H);
        B.put_element<4>(v, H);
        for(int i = 0; i < 4; ++i)
            for(int a = 0; a < 3; ++a)
                grad[3 * (size_t)v[i] + a] += G[3 * i + a];
    }
    if(tris_out)
        *tris_out = std::move(tris);
    if(hinges_out)
        *hinges_out = std::move(hinges);
    return nt;
}

// Point-triangle contact of vertex g (position xv) with the triangle of an
// affine body's square face (body frame: y = fy, |x|, |z| <= h, split along
// (-h,-h)-(h,h)) under its projection (ux, uz): the triangle corners are
// x_i = p + A xbar_i, so the 12-coordinate contact gradient G and Hessian H
// (elements.h: contact_grad_hess) map to the vertex and the body's 12 DoF by
// the constant Jacobian T (x_v -> x_v; x_i -> p + sum_k xbar_i[k] a_k):
// 15 blocks over the block rows (g, 4b, .., 4b + 3), gradient T^T G.
// Returns false when the pair is beyond dhat.
bool add_vertex_body_contact(Builder& B, std::vector<double>& grad, int32_t g, const double* xv, int64_t b,
                             const double* p, const double A[3][3], double ux, double uz, double fy, double h,
                             double dhat, double k)
{
    const double c[4][3] = {{-h, fy, -h}, {h, fy, -h}, {h, fy, h}, {-h, fy, h}};
    const int    t0 = 0, t1 = uz <= ux ? 1 : 2, t2 = uz <= ux ? 2 : 3;
    const int    tri[3] = {t0, t1, t2};
    double       X[12], G[12], H[144];
    for(int a = 0; a < 3; ++a)
        X[a] = xv[a];
    for(int i = 0; i < 3; ++i)
        for(int r = 0; r < 3; ++r)
        {
            double v = p[r];
            for(int kk = 0; kk < 3; ++kk)
                v += A[r][kk] * c[tri[i]][kk];
            X[3 + 3 * i + r] = v;
        }
    if(b2el::contact_grad_hess(X, 0, 0.0, dhat, k, G, H) < 0)
        return false;
    // t[I][J]: coefficient of DoF block J (0 vertex, 1 p, 2 + k a_k) in coordinate block I
    double t[4][5] = {};
    t[0][0] = 1.0;
    for(int i = 0; i < 3; ++i)
    {
        t[1 + i][1] = 1.0;
        for(int kk = 0; kk < 3; ++kk)
            t[1 + i][2 + kk] = c[tri[i]][kk];
    }
    const int32_t rws[5] = {g, (int32_t)(4 * b), (int32_t)(4 * b + 1), (int32_t)(4 * b + 2), (int32_t)(4 * b + 3)};
    for(int J = 0; J < 5; ++J)
        for(int K = J; K < 5; ++K)
        {
            double Hb[9] = {};
            for(int I = 0; I < 4; ++I)
                for(int L = 0; L < 4; ++L)
                {
                    const double w = t[I][J] * t[L][K];
                    if(w == 0.0)
                        continue;
                    for(int r = 0; r < 3; ++r)
                        for(int cc = 0; cc < 3; ++cc)
                            Hb[r * 3 + cc] += w * H[(3 * I + r) * 12 + 3 * L + cc];
                }
            B.put(rws[J], rws[K], Hb);
        }
    for(int J = 0; J < 5; ++J)
        for(int r = 0; r < 3; ++r)
        {
            double v = 0.0;
            for(int I = 0; I < 4; ++I)
                v += t[I][J] * G[3 * I + r];
            grad[(size_t)rws[J] * 3 + r] += v;
        }
    return true;
}
}  // namespace

struct b2g_system
{
    std::vector<double>  x, x_rest;
    std::vector<int32_t> tets;
    std::vector<int32_t> rows, cols;
    std::vector<double>  vals;
    std::vector<double>  grad;
    std::vector<int32_t> adj_start, adj_list;
    int64_t              n_contacts = 0;
    int64_t              n_bodies   = 0;
};

extern "C" {

void b2g_default_config(b2g_config* c)
{
    std::memset(c, 0, sizeof(*c));
    c->scene         = 1;
    c->cells_x       = 10;
    c->cells_y       = 10;
    c->cells_z       = 10;
    c->n_cubes       = 1;
    c->h             = 0.01;
    c->jitter        = 0.1;
    c->normal_jitter = 0.45e-3;
    c->gap           = 1e-3;
    c->seed          = 0;
    c->E             = 1e5;
    c->nu            = 0.45;
    c->rho           = 1e3;
    c->dt            = 0.01;
    c->gravity       = 9.8;
    c->dhat          = 1e-3;
    c->kappa         = 1e9;
    c->ground_offset = 0.1e-3;
    c->twist_deg     = 2.0;
    c->n_threads     = 0;
    c->body_kappa    = 1e8;
    c->bend_k        = 1e-2;
    c->cloth_size    = 2.0;
    c->wall_gap      = 0.02;
    c->cloth_n       = 64;
    c->bodies_x      = 4;
    c->bodies_z      = 8;
    c->cloth_k       = 1e3;
}

const char* b2g_last_error(void) { return g_err.c_str(); }

}  // extern "C"

namespace
{
// Scene 3: a square cloth (N x N vertices, two triangles per cell) resting
// on an nbs x nbs grid of affine bodies (cubes rotated about +y by seeded
// angles), first Newton step from rest. Bodies first in the DoF order.
//  * affine body b: q = (p, A[:,0], A[:,1], A[:,2]), x = p + A xbar; the
//    kinetic Hessian is the body mass matrix (m I; m s^2/12 I per column, the
//    cube's second moments), plus the orthogonality potential (elements.h)
//    at A = R, scaled by V dt^2; 16 triplets per body (4 x 4 grid of 3x3
//    blocks), the lower ones written as zero blocks, as the reference's
//    affine-body subsystem writes them;
//  * cloth: lumped mass (1 mm sheet), Baraff-Witkin stretch (stiffness E) and
//    shear, discrete-shell bending (stiffness bend_k) (add_cloth_grid);
//  * contact: cloth vertex above a body's top face at distance d < dhat,
//    barrier b(d^2) along +y, coupling the vertex with the body's 12 DoF
//    (rank-1 Hessian over 5 block rows: 15 triplets, 4 vertex-body blocks);
//  * potentials scaled by dt^2, gravity -y.
// The 16 blocks of affine body b (block rows 4b .. 4b+3; lower blocks as
// zero blocks): mass matrix m_b I on p, I_b I on each column of A, plus the
// orthogonality potential's PSD Hessian at A = R (R a rotation about +y by
// theta), scaled by V dt^2; and its gravity gradient.
void add_affine_body(Builder& B, std::vector<double>& grad, int64_t b, const double* q, const double* qt,
                     double m_b, double I_b, double V, const b2g_config& C)
{
    const double dt2 = C.dt * C.dt;
    double       H[12][12] = {};
    for(int a = 0; a < 3; ++a)
    {
        H[a][a] = m_b;
        for(int k = 0; k < 3; ++k)
            H[3 + 3 * k + a][3 + 3 * k + a] = I_b;
    }
    // orthogonality potential at the body's affine matrix (q index 3 + 3 k + r
    // <-> A[r][k]): PSD Hessian, gradient (zero up to rounding at a rotation)
    double G9[9], H9[81];
    b2el::ortho_grad_hess(q, C.body_kappa, V * dt2, G9, H9);
    for(int m = 0; m < 9; ++m)
        for(int n = 0; n < 9; ++n)
            H[3 + m][3 + n] += H9[m * 9 + n];
    // kinetic gradient M (q - q_tilde), M diagonal
    for(int i = 0; i < 12; ++i)
        grad[(4 * b) * 3 + i] += (i < 3 ? m_b : I_b) * (q[i] - qt[i]) + (i >= 3 ? G9[i - 3] : 0.0);
    for(int bi = 0; bi < 4; ++bi)
        for(int bj = 0; bj < 4; ++bj)
        {
            const int32_t r = (int32_t)(4 * b + bi), c = (int32_t)(4 * b + bj);
            B.rows.push_back(r);
            B.cols.push_back(c);
            for(int qq = 0; qq < 3; ++qq)
                for(int p = 0; p < 3; ++p)
                    B.vals.push_back(bi > bj ? 0.0 : H[3 * bi + p][3 * bj + qq]);
        }
}

// q of a body at rest: centre c, the columns of R, a rotation about +y by theta
void body_rest_q(const double* c, double theta, double* q)
{
    const double cs = std::cos(theta), sn = std::sin(theta);
    const double R[3][3] = {{cs, 0, sn}, {0, 1, 0}, {-sn, 0, cs}};
    for(int a = 0; a < 3; ++a)
        q[a] = c[a];
    for(int k = 0; k < 3; ++k)
        for(int r = 0; r < 3; ++r)
            q[3 + 3 * k + r] = R[r][k];
}

// x = A^-1 (y - p) of a body with q = (p, A[:,0], A[:,1], A[:,2])
void body_frame(const double* q, const double* y, double* x)
{
    double A[3][3];
    for(int k = 0; k < 3; ++k)
        for(int r = 0; r < 3; ++r)
            A[r][k] = q[3 + 3 * k + r];
    const double d[3] = {y[0] - q[0], y[1] - q[1], y[2] - q[2]};
    const double det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) -
                       A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
                       A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
    double inv[3][3];
    inv[0][0] = (A[1][1] * A[2][2] - A[1][2] * A[2][1]) / det;
    inv[0][1] = (A[0][2] * A[2][1] - A[0][1] * A[2][2]) / det;
    inv[0][2] = (A[0][1] * A[1][2] - A[0][2] * A[1][1]) / det;
    inv[1][0] = (A[1][2] * A[2][0] - A[1][0] * A[2][2]) / det;
    inv[1][1] = (A[0][0] * A[2][2] - A[0][2] * A[2][0]) / det;
    inv[1][2] = (A[0][2] * A[1][0] - A[0][0] * A[1][2]) / det;
    inv[2][0] = (A[1][0] * A[2][1] - A[1][1] * A[2][0]) / det;
    inv[2][1] = (A[0][1] * A[2][0] - A[0][0] * A[2][1]) / det;
    inv[2][2] = (A[0][0] * A[1][1] - A[0][1] * A[1][0]) / det;
    for(int r = 0; r < 3; ++r)
        x[r] = inv[r][0] * d[0] + inv[r][1] * d[1] + inv[r][2] * d[2];
}

void generate_cloth_abd(const b2g_config& C, b2g_system* sys)
{
    const int N = C.cells_x, nbs = C.n_cubes;
    if(N < 2 || nbs < 1)
        throw std::runtime_error("scene 3 needs cells_x >= 2 and n_cubes >= 1");
    const int64_t nbod = (int64_t)nbs * nbs, ncv = (int64_t)N * N, rows = 4 * nbod + ncv;
    if(rows > (int64_t)INT32_MAX / 3)
        throw std::runtime_error("system too large for 32-bit DoF indices");
    const double Lc = C.cloth_size > 0 ? C.cloth_size : 2.0, hc = Lc / (N - 1);
    const double pitch = Lc / nbs, s = 0.6 * pitch, dt2 = C.dt * C.dt, Dh = C.dhat * C.dhat;
    const double rho_b = C.rho, m_b = rho_b * s * s * s, I_b = m_b * s * s / 12.0, V = s * s * s;
    const double m_v = C.rho * 1e-3 * hc * hc;
    const double y_cloth = 0.5 * C.dhat;  // tops at y = 0
    sys->n_bodies = nbod;
    sys->x.assign(rows * 3, 0.0);
    std::vector<double> theta(nbod);
    for(int64_t b = 0; b < nbod; ++b)
    {
        const int64_t i = b % nbs, k = b / nbs;
        const double c[3] = {(i + 0.5) * pitch - 0.5 * Lc, -0.5 * s, (k + 0.5) * pitch - 0.5 * Lc};
        theta[b]           = urand(C.seed, 4, b) * (M_PI / 4);
        // the body's 12 DoF on its 4 block rows: centre, then the columns of A = R
        body_rest_q(c, theta[b], &sys->x[(4 * b) * 3]);
    }
    for(int64_t v = 0; v < ncv; ++v)
    {
        const int64_t i = v % N, k = v / N, g = 4 * nbod + v;
        sys->x[g * 3 + 0] = i * hc - 0.5 * Lc;
        sys->x[g * 3 + 1] = y_cloth;
        sys->x[g * 3 + 2] = k * hc - 0.5 * Lc;
    }
    sys->x_rest = sys->x;
    sys->grad.assign(rows * 3, 0.0);
    Builder B;
    B.reserve((size_t)nbod * 16 + ncv * 8);
    auto put = [&](int32_t r, int32_t c, const double* Hrc /*row-major 3x3 of block (r,c)*/)
    {
        const bool tp = r > c;
        B.rows.push_back(tp ? c : r);
        B.cols.push_back(tp ? r : c);
        for(int q = 0; q < 3; ++q)
            for(int p = 0; p < 3; ++p)
                B.vals.push_back(tp ? Hrc[q * 3 + p] : Hrc[p * 3 + q]);  // column-major
    };
    // ---- affine bodies (first step from rest: q_tilde = q - dt^2 g on p) ----
    for(int64_t b = 0; b < nbod; ++b)
    {
        const double* q = &sys->x[(4 * b) * 3];
        double        qt[12];
        std::copy(q, q + 12, qt);
        qt[1] -= dt2 * C.gravity;
        add_affine_body(B, sys->grad, b, q, qt, m_b, I_b, V, C);
    }
    // ---- cloth ----
    const int32_t c0 = (int32_t)(4 * nbod);
    for(int64_t v = 0; v < ncv; ++v)
    {
        const double Hm[9] = {m_v, 0, 0, 0, m_v, 0, 0, 0, m_v};
        put(c0 + (int32_t)v, c0 + (int32_t)v, Hm);
        sys->grad[(c0 + v) * 3 + 1] += m_v * dt2 * C.gravity;
    }
    add_cloth_grid(B, sys->grad, sys->x, sys->x_rest, c0, N, C.E, C.bend_k, dt2);
    auto vid = [&](int64_t i, int64_t k) { return i + (int64_t)N * k; };
    std::vector<std::vector<int32_t>> nb(rows);
    auto link = [&](int64_t va, int64_t vb)
    {
        nb[c0 + va].push_back(c0 + (int32_t)vb);
        nb[c0 + vb].push_back(c0 + (int32_t)va);
    };
    for(int64_t k = 0; k < N; ++k)
        for(int64_t i = 0; i < N; ++i)
        {
            if(i + 1 < N)
                link(vid(i, k), vid(i + 1, k));
            if(k + 1 < N)
                link(vid(i, k), vid(i, k + 1));
            if(i + 1 < N && k + 1 < N)
                link(vid(i, k), vid(i + 1, k + 1));
        }
    // ---- cloth-body contacts ----
    int64_t n_contacts = 0;
    for(int64_t v = 0; v < ncv; ++v)
    {
        const int32_t g  = c0 + (int32_t)v;
        const double  xv = sys->x[g * 3], yv = sys->x[g * 3 + 1], zv = sys->x[g * 3 + 2];
        const int64_t bi = (int64_t)std::floor((xv + 0.5 * Lc) / pitch), bk = (int64_t)std::floor((zv + 0.5 * Lc) / pitch);
        if(bi < 0 || bi >= nbs || bk < 0 || bk >= nbs)
            continue;
        const int64_t b  = bi + nbs * bk;
        const double  px = sys->x[(4 * b) * 3], py = sys->x[(4 * b) * 3 + 1], pz = sys->x[(4 * b) * 3 + 2];
        const double  cs = std::cos(theta[b]), sn = std::sin(theta[b]);
        // body-frame position of the vertex (R^T (x - p), R about +y)
        const double ux = cs * (xv - px) - sn * (zv - pz), uz = sn * (xv - px) + cs * (zv - pz);
        if(std::fabs(ux) > 0.5 * s || std::fabs(uz) > 0.5 * s)
            continue;
        const double d = yv - (py + 0.5 * s);
        if(d <= 0.0 || d >= C.dhat)
            continue;
        const double R[3][3] = {{cs, 0, sn}, {0, 1, 0}, {-sn, 0, cs}};
        const double pb[3]   = {px, py, pz}, xvv[3] = {xv, yv, zv};
        if(add_vertex_body_contact(B, sys->grad, g, xvv, b, pb, R, ux, uz, 0.5 * s, 0.5 * s, C.dhat,
                                   dt2 * C.kappa))
            ++n_contacts;
    }
    sys->n_contacts = n_contacts;
    sys->rows       = std::move(B.rows);
    sys->cols       = std::move(B.cols);
    sys->vals       = std::move(B.vals);
    // neighbour graph: cloth triangle edges (bodies have none)
    sys->adj_start.assign(rows + 1, 0);
    for(int64_t r = 0; r < rows; ++r)
    {
        auto& L = nb[r];
        std::sort(L.begin(), L.end());
        L.erase(std::unique(L.begin(), L.end()), L.end());
        sys->adj_start[r + 1] = sys->adj_start[r] + (int32_t)L.size();
    }
    sys->adj_list.resize(sys->adj_start[rows]);
    for(int64_t r = 0; r < rows; ++r)
        std::copy(nb[r].begin(), nb[r].end(), sys->adj_list.begin() + sys->adj_start[r]);
}

// x_in / xt_in (optional, [n_verts*3]): current positions and kinetic target
// x_tilde; null = the scene's default first Newton step from rest
// Tet cubes (scene 1: stacked along +y; scene 2: one twisted bar; scene 4:
// a W x W grid in the x-z plane on the ground, W = n_cubes, cubes wall_gap
// apart so they do not touch each other), the first Newton step from rest or
// the step at a given state.
void generate_tets(const b2g_config& C, const double* x_in, const double* xt_in, b2g_system* sys)
{
    {
        if(C.cells_x < 1 || C.cells_y < 1 || C.cells_z < 1 || C.n_cubes < 1 || C.h <= 0 || C.dt <= 0)
            throw std::runtime_error("invalid configuration sizes");
        if(C.scene != 1 && C.scene != 2 && C.scene != 4)
            throw std::runtime_error("unknown scene id");
#ifdef _OPENMP
        if(C.n_threads > 0)
            omp_set_num_threads(C.n_threads);
#endif
        const bool grid = C.scene == 4;
        const int nx = C.cells_x, ny = C.cells_y, nz = C.cells_z;
        const int64_t vx = nx + 1, vy = ny + 1, vz = nz + 1;
        const int64_t verts_per = vx * vy * vz;
        const int64_t tets_per  = 6ll * nx * ny * nz;
        const int n_cubes       = (C.scene == 1) ? C.n_cubes : grid ? C.n_cubes * C.n_cubes : 1;
        const int64_t nv        = verts_per * n_cubes;
        const int64_t nt        = tets_per * n_cubes;
        if(nv > (int64_t)INT32_MAX / 3)
            throw std::runtime_error("system too large for 32-bit DoF indices");

        auto vid = [&](int c, int64_t i, int64_t j, int64_t k) -> int64_t
        { return c * verts_per + i + vx * (j + vy * k); };

        // ---- vertices (rest shape = jittered grid) ----
        sys->x_rest.resize(nv * 3);
        const double cube_pitch = ny * C.h + C.gap;
        const double grid_pitch_x = nx * C.h + C.wall_gap, grid_pitch_z = nz * C.h + C.wall_gap;
#pragma omp parallel for schedule(static)
        for(int64_t g = 0; g < nv; ++g)
        {
            int64_t c = g / verts_per, l = g % verts_per;
            int64_t i = l % vx, j = (l / vx) % vy, k = l / (vx * vy);
            double  px = i * C.h, py = j * C.h + c * cube_pitch, pz = k * C.h;
            if(grid)
            {
                px += (c % C.n_cubes) * grid_pitch_x;
                py = j * C.h;
                pz += (c / C.n_cubes) * grid_pitch_z;
            }
            double  jx = urand(C.seed, 0, g) * C.jitter * C.h;
            double  jy = urand(C.seed, 1, g) * C.jitter * C.h;
            double  jz = urand(C.seed, 2, g) * C.jitter * C.h;
            bool    x_face = (i == 0 || i == nx), z_face = (k == 0 || k == nz);
            bool    y_face = (j == 0 || j == ny);
            if(C.scene == 1 || grid)
            {
                // keep the outer faces planar in their normal direction; the
                // contact faces (y) get a bounded normal jitter instead (the
                // grid's top faces, under the cloth, stay planar)
                if(x_face)
                    jx = 0.0;
                if(z_face)
                    jz = 0.0;
                if(y_face)
                    jy = (grid && j == ny) ? 0.0 : urand(C.seed, 3, g) * C.normal_jitter;
            }
            else
            {
                if(i == 0 || i == nx)
                    jx = 0.0;
            }
            sys->x_rest[g * 3 + 0] = px + jx;
            sys->x_rest[g * 3 + 1] = py + jy;
            sys->x_rest[g * 3 + 2] = pz + jz;
        }

        // ---- tets: Kuhn 6-tet split of every cell ----
        sys->tets.resize(nt * 4);
        static const int perms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
#pragma omp parallel for schedule(static)
        for(int64_t cell = 0; cell < (int64_t)n_cubes * nx * ny * nz; ++cell)
        {
            int64_t c = cell / ((int64_t)nx * ny * nz), l = cell % ((int64_t)nx * ny * nz);
            int64_t i = l % nx, j = (l / nx) % ny, k = l / ((int64_t)nx * ny);
            for(int p = 0; p < 6; ++p)
            {
                int64_t d[3] = {0, 0, 0};
                int32_t t[4];
                t[0] = (int32_t)vid((int)c, i, j, k);
                for(int s = 0; s < 3; ++s)
                {
                    d[perms[p][s]] += 1;
                    t[s + 1] = (int32_t)vid((int)c, i + d[0], j + d[1], k + d[2]);
                }
                // positive orientation in the rest shape
                Vec3 a{sys->x_rest[t[0] * 3], sys->x_rest[t[0] * 3 + 1], sys->x_rest[t[0] * 3 + 2]};
                Vec3 b{sys->x_rest[t[1] * 3], sys->x_rest[t[1] * 3 + 1], sys->x_rest[t[1] * 3 + 2]};
                Vec3 cc{sys->x_rest[t[2] * 3], sys->x_rest[t[2] * 3 + 1], sys->x_rest[t[2] * 3 + 2]};
                Vec3 dd{sys->x_rest[t[3] * 3], sys->x_rest[t[3] * 3 + 1], sys->x_rest[t[3] * 3 + 2]};
                if(dot(sub(b, a), cross(sub(cc, a), sub(dd, a))) < 0)
                    std::swap(t[2], t[3]);
                int64_t base = (cell * 6 + p) * 4;
                for(int q = 0; q < 4; ++q)
                    sys->tets[base + q] = t[q];
            }
        }

        // ---- current positions ----
        sys->x = sys->x_rest;
        std::vector<uint8_t> fixed(nv, 0);
        if(x_in)
        {
            std::memcpy(sys->x.data(), x_in, sizeof(double) * nv * 3);
            if(C.scene == 2)
                for(int64_t g = 0; g < nv; ++g)
                {
                    const int64_t i = (g % verts_per) % vx;
                    fixed[g]        = (i == 0 || i == nx) ? 1 : 0;
                }
        }
        else if(C.scene == 2)
        {
            // bar along x, ends rotated by +-twist about the x axis through the
            // cross-section centre; the twist is linear along the bar and both
            // end layers are fixed (Dirichlet)
            const double L = nx * C.h, cy = 0.5 * ny * C.h, cz = 0.5 * nz * C.h;
            const double tw = C.twist_deg * M_PI / 180.0;
#pragma omp parallel for schedule(static)
            for(int64_t g = 0; g < nv; ++g)
            {
                double px = sys->x_rest[g * 3], py = sys->x_rest[g * 3 + 1] - cy,
                       pz = sys->x_rest[g * 3 + 2] - cz;
                double th = tw * (2.0 * px / L - 1.0);
                double cs = std::cos(th), sn = std::sin(th);
                sys->x[g * 3 + 1] = cy + cs * py - sn * pz;
                sys->x[g * 3 + 2] = cz + sn * py + cs * pz;
                int64_t i = (g % verts_per) % vx;
                fixed[g] = (i == 0 || i == nx) ? 1 : 0;
            }
        }

        const double mu = C.E / (2.0 * (1.0 + C.nu));
        const double lambda = C.E * C.nu / ((1.0 + C.nu) * (1.0 - 2.0 * C.nu));
        const double dt2 = C.dt * C.dt;

        // ---- per-tet rest data: volume, shape gradients ----
        std::vector<double> tet_vol(nt);
        std::vector<double> tet_grad(nt * 12);  // g_k[b], k = 0..3
#pragma omp parallel for schedule(static)
        for(int64_t t = 0; t < nt; ++t)
        {
            const int32_t* T = &sys->tets[t * 4];
            Vec3 X[4];
            for(int q = 0; q < 4; ++q)
                X[q] = {sys->x_rest[T[q] * 3], sys->x_rest[T[q] * 3 + 1], sys->x_rest[T[q] * 3 + 2]};
            Vec3 e1 = sub(X[1], X[0]), e2 = sub(X[2], X[0]), e3 = sub(X[3], X[0]);
            // Dm column-major: columns e1 e2 e3 ; B = Dm^{-1}
            double det = dot(e1, cross(e2, e3));
            tet_vol[t] = det / 6.0;
            Vec3 r0 = scale(cross(e2, e3), 1.0 / det);  // row 0 of Dm^{-1}
            Vec3 r1 = scale(cross(e3, e1), 1.0 / det);
            Vec3 r2 = scale(cross(e1, e2), 1.0 / det);
            double* G = &tet_grad[t * 12];
            for(int b = 0; b < 3; ++b)
            {
                G[3 + b] = r0[b];
                G[6 + b] = r1[b];
                G[9 + b] = r2[b];
                G[b]     = -(r0[b] + r1[b] + r2[b]);
            }
        }

        // ---- lumped masses ----
        std::vector<double> mass(nv, 0.0);
        for(int64_t t = 0; t < nt; ++t)
            for(int q = 0; q < 4; ++q)
                mass[sys->tets[t * 4 + q]] += C.rho * tet_vol[t] * 0.25;

        // ---- contacts ----
        struct Pair
        {
            int32_t v[4];  // (p, t0, t1, t2) or (a0, a1, b0, b1)
            int     is_ee;
        };
        std::vector<Pair> pairs;
        std::vector<std::pair<int32_t, double>> ground;  // vertex, distance
        double ground_y = 0.0;
        if(grid)
        {
            // every cube's bottom layer on the ground
            double miny = 1e300;
            for(int64_t g = 0; g < nv; ++g)
                if(((g % verts_per) / vx) % vy == 0)
                    miny = std::min(miny, sys->x_rest[g * 3 + 1]);
            ground_y = miny - C.ground_offset;
            for(int64_t g = 0; g < nv; ++g)
                if(((g % verts_per) / vx) % vy == 0)
                {
                    const double d = sys->x[g * 3 + 1] - ground_y;
                    if(d < C.dhat)
                        ground.push_back({(int32_t)g, d});
                }
        }
        if(C.scene == 1)
        {
            double miny = 1e300;
            for(int64_t k = 0; k < vz; ++k)
                for(int64_t i = 0; i < vx; ++i)
                    miny = std::min(miny, sys->x_rest[vid(0, i, 0, k) * 3 + 1]);
            ground_y = miny - C.ground_offset;
            for(int64_t k = 0; k < vz; ++k)
                for(int64_t i = 0; i < vx; ++i)
                {
                    int64_t g = vid(0, i, 0, k);
                    double  d = sys->x[g * 3 + 1] - ground_y;
                    if(d < C.dhat)
                        ground.push_back({(int32_t)g, d});
                }
            // stacked cube interfaces: top layer of cube c vs bottom layer of c+1.
            // Each layer is an aligned (nx+1) x (nz+1) grid; cell (i,k) of a
            // layer holds the two Kuhn face triangles split along (i,k)-(i+1,k+1).
            for(int c = 0; c + 1 < n_cubes; ++c)
            {
                auto P = [&](int cube, int64_t i, int64_t j, int64_t k) -> Vec3
                {
                    int64_t g = vid(cube, i, j, k);
                    return {sys->x[g * 3], sys->x[g * 3 + 1], sys->x[g * 3 + 2]};
                };
                // triangles of a layer cell
                auto cell_tris = [&](int cube, int64_t j, int64_t i, int64_t k, int32_t tri[2][3])
                {
                    int32_t v00 = (int32_t)vid(cube, i, j, k), v10 = (int32_t)vid(cube, i + 1, j, k);
                    int32_t v01 = (int32_t)vid(cube, i, j, k + 1), v11 = (int32_t)vid(cube, i + 1, j, k + 1);
                    tri[0][0] = v00; tri[0][1] = v10; tri[0][2] = v11;
                    tri[1][0] = v00; tri[1][1] = v11; tri[1][2] = v01;
                };
                auto vpos = [&](int32_t g) -> Vec3 { return {sys->x[g * 3], sys->x[g * 3 + 1], sys->x[g * 3 + 2]}; };
                // point-triangle: vertices of one layer against triangles of the other
                for(int side = 0; side < 2; ++side)
                {
                    int     pc = side == 0 ? c + 1 : c, tc = side == 0 ? c : c + 1;
                    int64_t pj = side == 0 ? 0 : ny, tj = side == 0 ? ny : 0;
                    for(int64_t k = 0; k < vz; ++k)
                        for(int64_t i = 0; i < vx; ++i)
                        {
                            Vec3    p  = P(pc, i, pj, k);
                            int32_t pv = (int32_t)vid(pc, i, pj, k);
                            bool    done = false;
                            for(int64_t ci = i - 1; ci <= i && !done; ++ci)
                                for(int64_t ck = k - 1; ck <= k && !done; ++ck)
                                {
                                    if(ci < 0 || ck < 0 || ci >= nx || ck >= nz)
                                        continue;
                                    int32_t tri[2][3];
                                    cell_tris(tc, tj, ci, ck, tri);
                                    for(int tt = 0; tt < 2 && !done; ++tt)
                                    {
                                        Vec3 t0 = vpos(tri[tt][0]), t1 = vpos(tri[tt][1]), t2 = vpos(tri[tt][2]);
                                        Vec3 n = cross(sub(t1, t0), sub(t2, t0));
                                        double nn = norm(n);
                                        n = scale(n, 1.0 / nn);
                                        Vec3 q = sub(p, t0);
                                        double d = dot(q, n);
                                        Vec3 proj = sub(p, scale(n, d));
                                        // barycentric of proj
                                        Vec3 v0 = sub(t1, t0), v1 = sub(t2, t0), v2 = sub(proj, t0);
                                        double d00 = dot(v0, v0), d01 = dot(v0, v1), d11 = dot(v1, v1);
                                        double d20 = dot(v2, v0), d21 = dot(v2, v1);
                                        double den = d00 * d11 - d01 * d01;
                                        double wb = (d11 * d20 - d01 * d21) / den;
                                        double wc = (d00 * d21 - d01 * d20) / den;
                                        double wa = 1.0 - wb - wc;
                                        if(wa < 0 || wb < 0 || wc < 0)
                                            continue;
                                        done = true;
                                        if(std::fabs(d) >= C.dhat)
                                            continue;
                                        Pair pr;
                                        pr.is_ee = 0;
                                        pr.v[0] = pv; pr.v[1] = tri[tt][0]; pr.v[2] = tri[tt][1]; pr.v[3] = tri[tt][2];
                                        pairs.push_back(pr);
                                    }
                                }
                        }
                }
                // edge-edge: axis-aligned layer edges of the upper layer against
                // face diagonals of the lower layer and vice versa
                auto layer_edges = [&](int cube, int64_t j, std::vector<std::array<int32_t, 2>>& E)
                {
                    for(int64_t k = 0; k < vz; ++k)
                        for(int64_t i = 0; i < vx; ++i)
                        {
                            if(i < nx)
                                E.push_back({(int32_t)vid(cube, i, j, k), (int32_t)vid(cube, i + 1, j, k)});
                            if(k < nz)
                                E.push_back({(int32_t)vid(cube, i, j, k), (int32_t)vid(cube, i, j, k + 1)});
                            if(i < nx && k < nz)
                                E.push_back({(int32_t)vid(cube, i, j, k), (int32_t)vid(cube, i + 1, j, k + 1)});
                        }
                };
                std::vector<std::array<int32_t, 2>> Eu, El;
                layer_edges(c + 1, 0, Eu);
                layer_edges(c, ny, El);
                // bucket the lower edges by their first vertex's (i,k)
                auto ik_of = [&](int32_t g) -> std::pair<int64_t, int64_t>
                {
                    int64_t l = g % verts_per;
                    return {l % vx, l / (vx * vy)};
                };
                std::vector<std::vector<int32_t>> bucket(vx * vz);
                for(size_t e = 0; e < El.size(); ++e)
                {
                    auto [i, k] = ik_of(El[e][0]);
                    bucket[i + vx * k].push_back((int32_t)e);
                }
                for(size_t e = 0; e < Eu.size(); ++e)
                {
                    auto [i0, k0] = ik_of(Eu[e][0]);
                    for(int64_t ci = i0 - 1; ci <= i0 + 1; ++ci)
                        for(int64_t ck = k0 - 1; ck <= k0 + 1; ++ck)
                        {
                            if(ci < 0 || ck < 0 || ci >= vx || ck >= vz)
                                continue;
                            for(int32_t f : bucket[ci + vx * ck])
                            {
                                Vec3 a0 = vpos(Eu[e][0]), a1 = vpos(Eu[e][1]);
                                Vec3 b0 = vpos(El[f][0]), b1 = vpos(El[f][1]);
                                Vec3 u = sub(a1, a0), v = sub(b1, b0), w0 = sub(a0, b0);
                                double A = dot(u, u), B = dot(u, v), Cc = dot(v, v), D = dot(u, w0), Ee = dot(v, w0);
                                double den = A * Cc - B * B;
                                if(den < 1e-12 * A * Cc)
                                    continue;  // (nearly) parallel: covered by point-triangle pairs
                                double s = (B * Ee - Cc * D) / den, t = (A * Ee - B * D) / den;
                                if(s <= 0.0 || s >= 1.0 || t <= 0.0 || t >= 1.0)
                                    continue;
                                Vec3 pa = add(a0, scale(u, s)), pb = add(b0, scale(v, t));
                                Vec3 dv = sub(pa, pb);
                                double d = norm(dv);
                                if(d >= C.dhat || d <= 0.0)
                                    continue;
                                Pair pr;
                                pr.is_ee = 1;
                                pr.v[0] = Eu[e][0]; pr.v[1] = Eu[e][1]; pr.v[2] = El[f][0]; pr.v[3] = El[f][1];
                                pairs.push_back(pr);
                            }
                        }
                }
            }
        }
        sys->n_contacts = (int64_t)pairs.size() + (int64_t)ground.size();

        // ---- triplet layout: kinetic | SNH | ground | pairs ----
        const int64_t n_kin = nv, n_snh = nt * 10, n_gnd = (int64_t)ground.size(),
                      n_pair = (int64_t)pairs.size() * 10;
        const int64_t n_trip = n_kin + n_snh + n_gnd + n_pair;
        sys->rows.assign(n_trip, 0);
        sys->cols.assign(n_trip, 0);
        sys->vals.assign(n_trip * 9, 0.0);
        sys->grad.assign(nv * 3, 0.0);

        auto write_block = [&](int64_t slot, int32_t ra, int32_t rb, const double* Hab /*row-major 3x3 of block (a,b)*/)
        {
            bool tp = ra > rb;
            sys->rows[slot] = tp ? rb : ra;
            sys->cols[slot] = tp ? ra : rb;
            double* V = &sys->vals[slot * 9];
            for(int p = 0; p < 3; ++p)
                for(int q = 0; q < 3; ++q)
                {
                    double v = tp ? Hab[q * 3 + p] : Hab[p * 3 + q];  // value at (p,q) of the written block
                    V[q * 3 + p] = v;                                  // column-major
                }
        };

        // kinetic: x_tilde = x_prev + dt v + dt^2 g (default: x_prev = rest, v = 0)
#pragma omp parallel for schedule(static)
        for(int64_t g = 0; g < nv; ++g)
        {
            double H[9] = {mass[g], 0, 0, 0, mass[g], 0, 0, 0, mass[g]};
            write_block(g, (int32_t)g, (int32_t)g, H);
            double xt[3] = {sys->x_rest[g * 3], sys->x_rest[g * 3 + 1] - dt2 * C.gravity, sys->x_rest[g * 3 + 2]};
            if(xt_in)
                for(int a = 0; a < 3; ++a)
                    xt[a] = xt_in[g * 3 + a];
            for(int a = 0; a < 3; ++a)
                sys->grad[g * 3 + a] += mass[g] * (sys->x[g * 3 + a] - xt[a]);
        }

        // SNH: the F = I Hessian is shared by every undeformed tet
        double P_I[9], H_I[81];
        {
            const double Fi[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
            snh_derivatives(Fi, mu, lambda, P_I, H_I);
        }
        std::vector<double> tet_grad_out(nt * 12);
#pragma omp parallel for schedule(static)
        for(int64_t t = 0; t < nt; ++t)
        {
            const int32_t* T  = &sys->tets[t * 4];
            const double*  Gs = &tet_grad[t * 12];
            double F[9] = {0};
            for(int q = 0; q < 4; ++q)
                for(int a = 0; a < 3; ++a)
                    for(int b = 0; b < 3; ++b)
                        F[a + 3 * b] += sys->x[T[q] * 3 + a] * Gs[q * 3 + b];
            double P[9], H[81];
            bool   ident = true;
            for(int a = 0; a < 3; ++a)
                for(int b = 0; b < 3; ++b)
                    ident &= std::fabs(F[a + 3 * b] - (a == b ? 1.0 : 0.0)) < 1e-12;
            if(ident)
            {
                std::memcpy(H, H_I, sizeof(H));
                for(int i = 0; i < 9; ++i)
                    P[i] = 0.0;  // zero stress at rest
            }
            else
                snh_derivatives(F, mu, lambda, P, H);
            const double s = tet_vol[t] * dt2;
            // gradient: dE/dx_{q,a} = s * sum_b P[a+3b] g_q[b]
            for(int q = 0; q < 4; ++q)
                for(int a = 0; a < 3; ++a)
                {
                    double acc = 0.0;
                    for(int b = 0; b < 3; ++b)
                        acc += P[a + 3 * b] * Gs[q * 3 + b];
                    tet_grad_out[t * 12 + q * 3 + a] = s * acc;
                }
            // Hessian blocks (q, r), q <= r in local order
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
                                double gq = Gs[q * 3 + b];
                                for(int d = 0; d < 3; ++d)
                                    acc += gq * H[(a + 3 * b) * 9 + (c + 3 * d)] * Gs[r * 3 + d];
                            }
                            Hb[a * 3 + c] = s * acc;
                        }
                    if(q == r)  // exact symmetry of diagonal blocks
                        for(int a = 0; a < 3; ++a)
                            for(int c = a + 1; c < 3; ++c)
                            {
                                double m = 0.5 * (Hb[a * 3 + c] + Hb[c * 3 + a]);
                                Hb[a * 3 + c] = Hb[c * 3 + a] = m;
                            }
                    write_block(n_kin + t * 10 + slot, T[q], T[r], Hb);
                }
        }
        for(int64_t t = 0; t < nt; ++t)
            for(int q = 0; q < 4; ++q)
                for(int a = 0; a < 3; ++a)
                    sys->grad[sys->tets[t * 4 + q] * 3 + a] += tet_grad_out[t * 12 + q * 3 + a];

        const double Dh = C.dhat * C.dhat;
        // ground barrier (normal +y)
        for(int64_t gi = 0; gi < n_gnd; ++gi)
        {
            int32_t g = ground[gi].first;
            double  d = ground[gi].second, D = d * d, b1, b2;
            barrier_d(D, Dh, b1, b2);
            double k = dt2 * C.kappa * (b2 * 4.0 * D + 2.0 * b1);
            if(k < 0.0)
                k = 0.0;
            double H[9] = {0, 0, 0, 0, k, 0, 0, 0, 0};
            write_block(n_kin + n_snh + gi, g, g, H);
            sys->grad[g * 3 + 1] += dt2 * C.kappa * b1 * 2.0 * d;
        }
        // pair barriers: the point-triangle / edge-edge contact energy of the
        // pair's closest-feature type (elements.h: contact_grad_hess)
        std::vector<double> pair_g(pairs.size() * 12);
#pragma omp parallel for schedule(static)
        for(int64_t pi = 0; pi < (int64_t)pairs.size(); ++pi)
        {
            const Pair& pr = pairs[pi];
            double      X[12], H[144], eps = 0.0;
            for(int q = 0; q < 4; ++q)
                for(int a = 0; a < 3; ++a)
                    X[q * 3 + a] = sys->x[pr.v[q] * 3 + a];
            if(pr.is_ee)
            {
                double ea[3], eb[3];
                for(int a = 0; a < 3; ++a)
                {
                    ea[a] = sys->x_rest[pr.v[1] * 3 + a] - sys->x_rest[pr.v[0] * 3 + a];
                    eb[a] = sys->x_rest[pr.v[3] * 3 + a] - sys->x_rest[pr.v[2] * 3 + a];
                }
                eps = 1e-3 * b2el::dot3(ea, ea) * b2el::dot3(eb, eb);
            }
            b2el::contact_grad_hess(X, pr.is_ee, eps, C.dhat, dt2 * C.kappa, &pair_g[pi * 12], H);
            int slot = 0;
            for(int q = 0; q < 4; ++q)
                for(int r = q; r < 4; ++r, ++slot)
                {
                    double Hb[9];
                    for(int a = 0; a < 3; ++a)
                        for(int c = 0; c < 3; ++c)
                            Hb[a * 3 + c] = H[(3 * q + a) * 12 + 3 * r + c];
                    write_block(n_kin + n_snh + n_gnd + pi * 10 + slot, pr.v[q], pr.v[r], Hb);
                }
        }
        for(int64_t pi = 0; pi < (int64_t)pairs.size(); ++pi)
            for(int q = 0; q < 4; ++q)
                for(int a = 0; a < 3; ++a)
                    sys->grad[pairs[pi].v[q] * 3 + a] += pair_g[pi * 12 + q * 3 + a];

        // fixed vertices (Dirichlet)
        bool any_fixed = false;
        for(auto f : fixed)
            any_fixed |= (f != 0);
        if(any_fixed)
        {
#pragma omp parallel for schedule(static)
            for(int64_t s = 0; s < n_trip; ++s)
            {
                int32_t i = sys->rows[s], j = sys->cols[s];
                if(fixed[i] || fixed[j])
                {
                    double* V = &sys->vals[s * 9];
                    for(int e = 0; e < 9; ++e)
                        V[e] = 0.0;
                    if(i == j)
                        V[0] = V[4] = V[8] = 1.0;
                }
            }
            for(int64_t g = 0; g < nv; ++g)
                if(fixed[g])
                    sys->grad[g * 3] = sys->grad[g * 3 + 1] = sys->grad[g * 3 + 2] = 0.0;
        }

        // ---- MAS neighbour graph (tet edges, sorted unique) ----
        {
            std::vector<std::vector<int32_t>> nb(nv);
            for(int64_t t = 0; t < nt; ++t)
                for(int q = 0; q < 4; ++q)
                    for(int r = q + 1; r < 4; ++r)
                    {
                        int32_t a = sys->tets[t * 4 + q], b = sys->tets[t * 4 + r];
                        nb[a].push_back(b);
                        nb[b].push_back(a);
                    }
            sys->adj_start.assign(nv + 1, 0);
            for(int64_t v = 0; v < nv; ++v)
            {
                auto& L = nb[v];
                std::sort(L.begin(), L.end());
                L.erase(std::unique(L.begin(), L.end()), L.end());
                sys->adj_start[v + 1] = sys->adj_start[v] + (int32_t)L.size();
            }
            sys->adj_list.resize(sys->adj_start[nv]);
            for(int64_t v = 0; v < nv; ++v)
                std::copy(nb[v].begin(), nb[v].end(), sys->adj_list.begin() + sys->adj_start[v]);
        }

    }
}

// Scene 4 (the full-scale case): a W x W grid of tet cubes on the ground
// (generate_tets, W = n_cubes), an N x N cloth (N = cloth_n) resting on their
// top faces, and bodies_x x bodies_z affine bodies resting on the cloth;
// first Newton step from rest.
//  * cloth: as scene 3 (lumped mass, Baraff-Witkin, bending), covering
//    the grid, 0.5 dhat above the (planar) top faces;
//  * cloth-cube contact: each cloth vertex over a top-face triangle at
//    distance 0 < d < dhat: point-triangle barrier b(d^2), D = (a . x)^2 with
//    a = (n, -w0 n, -w1 n, -w2 n) over the vertex and the triangle's corners
//    (10 triplets);
//  * cloth-body contact: each cloth vertex under a body's bottom face at
//    0 < d < dhat: barrier along -y coupling the vertex with the body's 12 DoF
//    (15 triplets);
//  * DoF order: bodies (4 block rows each), cube vertices, cloth vertices; the
//    neighbour graph holds the tet edges and the cloth triangle edges.
void generate_wall(const b2g_config& C, const double* x_in, const double* xt_in, b2g_system* sys)
{
    const int W = C.n_cubes, N = C.cloth_n, nbx = C.bodies_x, nbz = C.bodies_z;
    if(N < 2 || nbx < 0 || nbz < 0 || W < 1)
        throw std::runtime_error("scene 4 needs n_cubes >= 1, cloth_n >= 2, bodies_x/z >= 0");
    if((x_in == nullptr) != (xt_in == nullptr))
        throw std::runtime_error("scene 4 state input needs both x and x_tilde");
    b2g_config Cc = C;
    Cc.scene      = 4;
    b2g_system    cubes;
    const int64_t nbod = (int64_t)nbx * nbz, off_c = 4 * nbod;
    generate_tets(Cc, x_in ? x_in + off_c * 3 : nullptr, xt_in ? xt_in + off_c * 3 : nullptr, &cubes);
    const int     nx = C.cells_x, ny = C.cells_y, nz = C.cells_z;
    const int64_t vx = nx + 1, vy = ny + 1, vz = nz + 1, verts_per = vx * vy * vz;
    const int64_t ncube_v = (int64_t)cubes.x.size() / 3, ncv = (int64_t)N * N;
    const int64_t off_cl = off_c + ncube_v, rows = off_cl + ncv;
    if(rows > (int64_t)INT32_MAX / 3)
        throw std::runtime_error("system too large for 32-bit DoF indices");
    const double px_pitch = nx * C.h + C.wall_gap, pz_pitch = nz * C.h + C.wall_gap;
    const double Lx = W * px_pitch - C.wall_gap, Lz = W * pz_pitch - C.wall_gap;
    const double top = ny * C.h, hc = Lx / (N - 1), hcz = Lz / (N - 1);
    const double y_cloth = top + 0.5 * C.dhat, dt2 = C.dt * C.dt, Dh = C.dhat * C.dhat;
    const double m_v = C.rho * 1e-3 * hc * hcz;
    const double bpx = nbx > 0 ? Lx / nbx : 1.0, bpz = nbz > 0 ? Lz / nbz : 1.0;
    const double s = 0.6 * std::min(bpx, bpz), m_b = C.rho * s * s * s, I_b = m_b * s * s / 12.0, V = s * s * s;
    sys->n_bodies = nbod;
    sys->x.assign(rows * 3, 0.0);
    sys->grad.assign(rows * 3, 0.0);
    std::vector<double> theta(nbod);
    for(int64_t b = 0; b < nbod; ++b)
    {
        const int64_t i = b % nbx, k = b / nbx;
        const double  c[3] = {(i + 0.5) * bpx, y_cloth + 0.5 * C.dhat + 0.5 * s, (k + 0.5) * bpz};
        theta[b]           = urand(C.seed, 4, b) * (M_PI / 4);
        // the body's 12 DoF on its 4 block rows: centre, then the columns of A
        body_rest_q(c, theta[b], &sys->x[(4 * b) * 3]);
    }
    std::copy(cubes.x_rest.begin(), cubes.x_rest.end(), sys->x.begin() + off_c * 3);
    for(int64_t v = 0; v < ncv; ++v)
    {
        const int64_t g = off_cl + v;
        sys->x[g * 3 + 0] = (v % N) * hc;
        sys->x[g * 3 + 1] = y_cloth;
        sys->x[g * 3 + 2] = (v / N) * hcz;
    }
    sys->x_rest = sys->x;
    // the state: given, or the first step from rest (x_tilde = x - dt^2 g on
    // every translation DoF: cube and cloth vertices and the bodies' centres)
    std::vector<double> xt(sys->x);
    if(x_in)
    {
        std::copy(x_in, x_in + rows * 3, sys->x.begin());
        std::copy(xt_in, xt_in + rows * 3, xt.begin());
    }
    else
        for(int64_t r = 0; r < rows; ++r)
            if(r >= off_c || r % 4 == 0)
                xt[r * 3 + 1] -= dt2 * C.gravity;
    std::copy(cubes.x.begin(), cubes.x.end(), sys->x.begin() + off_c * 3);
    std::copy(cubes.grad.begin(), cubes.grad.end(), sys->grad.begin() + off_c * 3);

    Builder B;
    B.reserve((size_t)nbod * 16 + cubes.rows.size() + (size_t)ncv * 30);
    auto put = [&](int32_t r, int32_t c, const double* Hrc /*row-major 3x3 of block (r,c)*/)
    {
        const bool tp = r > c;
        B.rows.push_back(tp ? c : r);
        B.cols.push_back(tp ? r : c);
        for(int q = 0; q < 3; ++q)
            for(int p = 0; p < 3; ++p)
                B.vals.push_back(tp ? Hrc[q * 3 + p] : Hrc[p * 3 + q]);  // column-major
    };
    // ---- bodies, cubes ----
    for(int64_t b = 0; b < nbod; ++b)
        add_affine_body(B, sys->grad, b, &sys->x[(4 * b) * 3], &xt[(4 * b) * 3], m_b, I_b, V, C);
    for(size_t t = 0; t < cubes.rows.size(); ++t)
    {
        B.rows.push_back(cubes.rows[t] + (int32_t)off_c);
        B.cols.push_back(cubes.cols[t] + (int32_t)off_c);
    }
    B.vals.insert(B.vals.end(), cubes.vals.begin(), cubes.vals.end());
    // ---- cloth ----
    std::vector<std::vector<int32_t>> nb(ncv);
    auto cg = [&](int64_t i, int64_t k) { return (int32_t)(off_cl + i + (int64_t)N * k); };
    for(int64_t v = 0; v < ncv; ++v)
    {
        const double Hm[9] = {m_v, 0, 0, 0, m_v, 0, 0, 0, m_v};
        put((int32_t)(off_cl + v), (int32_t)(off_cl + v), Hm);
        for(int a = 0; a < 3; ++a)
            sys->grad[(off_cl + v) * 3 + a] += m_v * (sys->x[(off_cl + v) * 3 + a] - xt[(off_cl + v) * 3 + a]);
    }
    add_cloth_grid(B, sys->grad, sys->x, sys->x_rest, off_cl, N, C.cloth_k, C.bend_k, dt2);
    auto link = [&](int32_t ga, int32_t gb)
    {
        nb[ga - off_cl].push_back(gb);
        nb[gb - off_cl].push_back(ga);
    };
    for(int64_t k = 0; k < N; ++k)
        for(int64_t i = 0; i < N; ++i)
        {
            if(i + 1 < N)
                link(cg(i, k), cg(i + 1, k));
            if(k + 1 < N)
                link(cg(i, k), cg(i, k + 1));
            if(i + 1 < N && k + 1 < N)
                link(cg(i, k), cg(i + 1, k + 1));
        }
    // ---- cloth-cube contacts (point-triangle on the top faces) ----
    auto pos = [&](int64_t g) -> Vec3 { return {sys->x[g * 3], sys->x[g * 3 + 1], sys->x[g * 3 + 2]}; };
    auto cube_v = [&](int64_t c, int64_t i, int64_t k) { return off_c + c * verts_per + i + vx * (ny + vy * k); };
    int64_t n_contacts = (int64_t)cubes.n_contacts;
    for(int64_t v = 0; v < ncv; ++v)
    {
        const int64_t g = off_cl + v;
        const Vec3    p = pos(g);
        const int64_t ci = (int64_t)std::floor(p[0] / px_pitch), ck = (int64_t)std::floor(p[2] / pz_pitch);
        if(ci < 0 || ci >= W || ck < 0 || ck >= W)
            continue;
        const double ux = p[0] - ci * px_pitch, uz = p[2] - ck * pz_pitch;
        if(ux > nx * C.h || uz > nz * C.h)
            continue;  // over a gap between cubes
        const int64_t c  = ci + (int64_t)W * ck;
        const int64_t i0 = std::min<int64_t>((int64_t)(ux / C.h), nx - 1), k0 = std::min<int64_t>((int64_t)(uz / C.h), nz - 1);
        bool          done = false;
        for(int64_t i = i0 - 1; i <= i0 + 1 && !done; ++i)
            for(int64_t k = k0 - 1; k <= k0 + 1 && !done; ++k)
            {
                if(i < 0 || k < 0 || i >= nx || k >= nz)
                    continue;
                const int64_t v00 = cube_v(c, i, k), v10 = cube_v(c, i + 1, k), v01 = cube_v(c, i, k + 1),
                              v11 = cube_v(c, i + 1, k + 1);
                const int64_t tri[2][3] = {{v00, v10, v11}, {v00, v11, v01}};
                for(int tt = 0; tt < 2 && !done; ++tt)
                {
                    const Vec3 t0 = pos(tri[tt][0]), t1 = pos(tri[tt][1]), t2 = pos(tri[tt][2]);
                    Vec3       n  = cross(sub(t1, t0), sub(t2, t0));
                    n             = scale(n, (n[1] < 0 ? -1.0 : 1.0) / norm(n));
                    const double d = dot(sub(p, t0), n);
                    const Vec3   q = sub(p, scale(n, d));
                    const Vec3   e0 = sub(t1, t0), e1 = sub(t2, t0), e2 = sub(q, t0);
                    const double d00 = dot(e0, e0), d01 = dot(e0, e1), d11 = dot(e1, e1), d20 = dot(e2, e0),
                                 d21 = dot(e2, e1), den = d00 * d11 - d01 * d01;
                    const double wb = (d11 * d20 - d01 * d21) / den, wc = (d00 * d21 - d01 * d20) / den,
                                 wa = 1.0 - wb - wc;
                    if(wa < 0 || wb < 0 || wc < 0)
                        continue;
                    done = true;
                    if(d <= 0.0 || d >= C.dhat)
                        continue;
                    ++n_contacts;
                    const int32_t vs[4] = {(int32_t)g, (int32_t)tri[tt][0], (int32_t)tri[tt][1], (int32_t)tri[tt][2]};
                    double        X[12], G[12], H[144];
                    for(int q2 = 0; q2 < 4; ++q2)
                        for(int a2 = 0; a2 < 3; ++a2)
                            X[q2 * 3 + a2] = sys->x[(int64_t)vs[q2] * 3 + a2];
                    b2el::contact_grad_hess(X, 0, 0.0, C.dhat, dt2 * C.kappa, G, H);
                    B.put_element<4>(vs, H);
                    for(int q2 = 0; q2 < 4; ++q2)
                        for(int a2 = 0; a2 < 3; ++a2)
                            sys->grad[vs[q2] * 3 + a2] += G[q2 * 3 + a2];
                }
            }
    }
    // ---- cloth-body contacts (the bodies' bottom faces) ----
    for(int64_t v = 0; v < ncv && nbod > 0; ++v)
    {
        const int64_t g  = off_cl + v;
        const double  xv = sys->x[g * 3], yv = sys->x[g * 3 + 1], zv = sys->x[g * 3 + 2];
        const int64_t bi = (int64_t)std::floor(xv / bpx), bk = (int64_t)std::floor(zv / bpz);
        if(bi < 0 || bi >= nbx || bk < 0 || bk >= nbz)
            continue;
        const int64_t b  = bi + (int64_t)nbx * bk;
        const double* q  = &sys->x[(4 * b) * 3];
        const double  xvv[3] = {xv, yv, zv};
        double        u[3];
        body_frame(q, xvv, u);  // the vertex in the body's frame
        if(std::fabs(u[0]) > 0.5 * s || std::fabs(u[2]) > 0.5 * s)
            continue;
        const double d = -0.5 * s - u[1];  // below the bottom face (A near a rotation)
        if(d <= 0.0 || d >= C.dhat)
            continue;
        double A[3][3];
        for(int k = 0; k < 3; ++k)
            for(int r = 0; r < 3; ++r)
                A[r][k] = q[3 + 3 * k + r];
        if(add_vertex_body_contact(B, sys->grad, (int32_t)g, xvv, b, q, A, u[0], u[2], -0.5 * s, 0.5 * s, C.dhat,
                                   dt2 * C.kappa))
            ++n_contacts;
    }
    sys->n_contacts = n_contacts;
    sys->rows       = std::move(B.rows);
    sys->cols       = std::move(B.cols);
    sys->vals       = std::move(B.vals);
    // neighbour graph: bodies none, the cubes' tet edges, the cloth's edges
    sys->adj_start.assign(rows + 1, 0);
    for(int64_t r = 0; r < rows; ++r)
    {
        int32_t cnt = 0;
        if(r >= off_c && r < off_cl)
            cnt = cubes.adj_start[r - off_c + 1] - cubes.adj_start[r - off_c];
        else if(r >= off_cl)
        {
            auto& L = nb[r - off_cl];
            std::sort(L.begin(), L.end());
            L.erase(std::unique(L.begin(), L.end()), L.end());
            cnt = (int32_t)L.size();
        }
        sys->adj_start[r + 1] = sys->adj_start[r] + cnt;
    }
    sys->adj_list.resize(sys->adj_start[rows]);
    for(int64_t r = off_c; r < rows; ++r)
    {
        int32_t* dst = sys->adj_list.data() + sys->adj_start[r];
        if(r < off_cl)
            for(int32_t e = cubes.adj_start[r - off_c]; e < cubes.adj_start[r - off_c + 1]; ++e)
                *dst++ = cubes.adj_list[e] + (int32_t)off_c;
        else
            std::copy(nb[r - off_cl].begin(), nb[r - off_cl].end(), dst);
    }
}

int generate_impl(const b2g_config* cfg, const double* x_in, const double* xt_in, b2g_system** out)
{
    try
    {
        if(!cfg || !out)
            throw std::runtime_error("null argument");
        const b2g_config C = *cfg;
        auto sys = std::make_unique<b2g_system>();
        if(C.scene == 3)
        {
            if(x_in || xt_in)
                throw std::runtime_error("scene 3 has no state input");
            generate_cloth_abd(C, sys.get());
        }
        else if(C.scene == 4)
            generate_wall(C, x_in, xt_in, sys.get());
        else
            generate_tets(C, x_in, xt_in, sys.get());
        *out = sys.release();
        return 0;
    }
    catch(const std::exception& e)
    {
        g_err = e.what();
        return 1;
    }
}
}  // namespace

extern "C" {

int b2g_generate(const b2g_config* cfg, b2g_system** out) { return generate_impl(cfg, nullptr, nullptr, out); }

int b2g_generate_state(const b2g_config* cfg, const double* x, const double* x_tilde, b2g_system** out)
{
    if(!x || !x_tilde)
    {
        g_err = "b2g_generate_state: null state";
        return 1;
    }
    return generate_impl(cfg, x, x_tilde, out);
}

void b2g_free(b2g_system* s) { delete s; }

int64_t b2g_num_verts(const b2g_system* s) { return (int64_t)s->x.size() / 3; }
int64_t b2g_num_tets(const b2g_system* s) { return (int64_t)s->tets.size() / 4; }
int64_t b2g_num_triplets(const b2g_system* s) { return (int64_t)s->rows.size(); }
int64_t b2g_num_contacts(const b2g_system* s) { return s->n_contacts; }
int64_t b2g_num_bodies(const b2g_system* s) { return s->n_bodies; }
const double* b2g_positions(const b2g_system* s) { return s->x.data(); }
const double* b2g_rest_positions(const b2g_system* s) { return s->x_rest.data(); }
const int32_t* b2g_tets(const b2g_system* s) { return s->tets.data(); }
const int32_t* b2g_triplet_rows(const b2g_system* s) { return s->rows.data(); }
const int32_t* b2g_triplet_cols(const b2g_system* s) { return s->cols.data(); }
const double* b2g_triplet_vals(const b2g_system* s) { return s->vals.data(); }
const double* b2g_gradient(const b2g_system* s) { return s->grad.data(); }
int64_t b2g_num_adjacency(const b2g_system* s) { return (int64_t)s->adj_list.size(); }
const int32_t* b2g_adjacency_start(const b2g_system* s) { return s->adj_start.data(); }
const int32_t* b2g_adjacency_list(const b2g_system* s) { return s->adj_list.data(); }

double b2g_element_bw(const double* x, const double* rest, double stretch, double shear, double rate, double w,
                      double* G9, double* H81)
{
    double IB[4], fu[3], fv[3];
    b2el::bw_rest(rest, rest + 3, rest + 6, IB);
    b2el::bw_grad_hess(x, x + 3, x + 6, IB, stretch, shear, rate, w, G9, H81);
    b2el::bw_F(x, x + 3, x + 6, IB, fu, fv);
    return b2el::bw_energy(fu, fv, stretch, shear, rate);
}

double b2g_element_dsb(const double* x, const double* rest, double kappa, double w, double* G12, double* H144)
{
    double L0, hb, thb;
    b2el::dsb_rest(rest, rest + 3, rest + 6, rest + 9, &L0, &hb, &thb);
    b2el::dsb_grad_hess(x, x + 3, x + 6, x + 9, L0, hb, thb, kappa, w, G12, H144);
    return b2el::dsb_energy(x, x + 3, x + 6, x + 9, L0, hb, thb, kappa);
}

int b2g_element_contact(const double* X, int is_ee, double eps, double dhat, double k, double* G12, double* H144)
{
    return b2el::contact_grad_hess(X, is_ee, eps, dhat, k, G12, H144);
}

double b2g_element_ortho(const double* q, double kappa, double w, double* G9, double* H81)
{
    b2el::ortho_grad_hess(q, kappa, w, G9, H81);
    return b2el::ortho_energy(q, kappa);
}

double b2g_contact_energy(const double* X, int is_ee, double eps, double dhat, double k)
{
    return b2el::contact_energy(X, is_ee, eps, dhat, k);
}

int b2g_accd(const double* X, const double* dX, int is_ee, double eta, double xi, int max_iter, double toi_max,
             double* toi)
{
    return b2el::accd_pair(X, dX, is_ee, eta, xi, max_iter, toi_max, toi) ? 1 : 0;
}

}  // extern "C"
