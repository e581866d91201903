// Element energies of the cloth / affine-body scenes, shared by the host
// generator (scene_gen.cpp) and the device generator (b2s_generate.cu).
// Plain arrays, FP64; matrices row-major unless stated.
//
//  * Baraff-Witkin shell, strain-limiting stretch + shear
//    (libuipc src/backends/cuda/finite_element/constitutions/
//     strain_limiting_baraff_witkin_shell_2d.h:33-280,
//     strain_limiting_baraff_witkin_shell_2d.cu:75-150): F = Ds Dm^-1 (3x2)
//    in the rest triangle's own uv frame, warp a = (1,0), weft b = (0,1);
//    stretch per direction (r-1)^2 + c s (r-1)^3 (c = 1 when r > 1) of
//    r = |F a|, shear (a^T F^T F b)^2; the 6x6 d2E/dF2 in the reference's
//    closed form (exact for the stretch where r > 1, its positive part below;
//    the shear in its analytic PSD form); weight rest area x dt^2.
//  * Discrete-shell bending, Gauss-Newton Hessian (the reference's default)
//    (finite_element/constitutions/discrete_shell_bending_function.h:33-135,
//     discrete_shell_bending_reference.h:8-28, utils/dihedral_angle.h:14-60):
//    E = L0 kappa (theta - theta_bar)^2 / h_bar with h_bar = A / (3 L0), over
//    the hinge (x0, x1, x2, x3), edge x1-x2; H = (2 L0 kappa / h_bar) dt^2
//    grad(theta) grad(theta)^T.
//  * Affine-body orthogonality potential
//    (affine_body/constitutions/ortho_potential.cu:37-70, sym/ortho_potential.inl):
//    E = kappa sum_ij (a_i . a_j - delta_ij)^2 over the three 3-vectors
//    a_1..a_3 = q[3..11] of the body's 12 DoF; gradient and Hessian derived
//    here by hand, the 9x9 Hessian projected to PSD (eigenvalues clamped at 0),
//    weight volume x dt^2.
//  * IPC normal contact of a point-triangle or edge-edge pair
//    (contact_system/contact_models/ipc_simplex_normal_contact.cu:358-680 with
//    its default Hessian mode, codim_ipc_simplex_normal_contact_function.h,
//    utils/distance/distance_flagged.h:258-520, edge_edge_mollifier.inl):
//    barrier B(D) = -kappa dt^2 (D - dhat^2)^2 log(D / dhat^2) of the squared
//    distance D of the pair's closest-feature type (point-triangle /
//    point-edge / point-point, edge-edge / point-edge / point-point); edge-edge
//    energies times the mollifier m(c) = (2 - c/eps) c/eps of c = |ea x eb|^2
//    below eps = 1e-3 |ea_rest|^2 |eb_rest|^2. PT and EE types (and every
//    mollified pair): the exact Hessian, projected to PSD; PE and PP types:
//    the closed form (B'' + B' / (2D)) grad(D) grad(D)^T. The exact second
//    derivatives come from a second-order forward differentiation of the
//    distance formulas (Jet12 below), not from hand-expanded expressions.
#pragma once

#include <cmath>

#if defined(__CUDACC__)
#define B2_HD __host__ __device__ inline
// contact_grad_hess is compiled as a device function of its own: inlined into
// the contact kernel (CUDA 12.9, NVVM at -O3), its point-edge, point-point
// and edge-edge branches came out wrong (correct at NVVM -O1, or not
// inlined); the GPU test compares every type with the host build (static:
// one copy per translation unit that includes this header)
#define B2_HD_NOINLINE static __host__ __device__ __noinline__
#else
#define B2_HD inline
#define B2_HD_NOINLINE inline
#endif

namespace b2el
{
B2_HD double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
B2_HD void   cross3(const double* a, const double* b, double* c)
{
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}
B2_HD void sub3(const double* a, const double* b, double* c)
{
    c[0] = a[0] - b[0];
    c[1] = a[1] - b[1];
    c[2] = a[2] - b[2];
}

// cyclic Jacobi eigen-decomposition of a symmetric n x n matrix (n <= 12):
// a is destroyed (its diagonal ends as the eigenvalues w), v[i*n+k] is
// component i of eigenvector k
template <int N>
B2_HD void jacobi_eigen(double* a, double* w, double* v)
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
                const double apq = a[p * N + q];
                if(fabs(apq) < 1e-300)
                    continue;
                const double app = a[p * N + p], aqq = a[q * N + q];
                const double theta = (aqq - app) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for(int k = 0; k < N; ++k)
                {
                    const double akp = a[k * N + p], akq = a[k * N + q];
                    a[k * N + p] = c * akp - s * akq;
                    a[k * N + q] = s * akp + c * akq;
                }
                for(int k = 0; k < N; ++k)
                {
                    const double apk = a[p * N + k], aqk = a[q * N + k];
                    a[p * N + k] = c * apk - s * aqk;
                    a[q * N + k] = s * apk + c * aqk;
                }
                for(int k = 0; k < N; ++k)
                {
                    const double vkp = v[k * N + p], vkq = v[k * N + q];
                    v[k * N + p] = c * vkp - s * vkq;
                    v[k * N + q] = s * vkp + c * vkq;
                }
            }
    }
    for(int i = 0; i < N; ++i)
        w[i] = a[i * N + i];
}

// symmetric H (N x N, row-major) -> its positive part (negative eigenvalues
// set to zero); returns with H exactly symmetric
template <int N>
B2_HD void project_psd(double* H)
{
    double a[N * N], w[N], v[N * N];
    for(int i = 0; i < N * N; ++i)
        a[i] = H[i];
    jacobi_eigen<N>(a, w, v);
    bool neg = false;
    for(int k = 0; k < N; ++k)
        neg = neg || w[k] < 0.0;
    if(!neg)
        return;
    for(int i = 0; i < N; ++i)
        for(int j = i; j < N; ++j)
        {
            double s = 0.0;
            for(int k = 0; k < N; ++k)
                if(w[k] > 0.0)
                    s += v[i * N + k] * w[k] * v[j * N + k];
            H[i * N + j] = s;
            H[j * N + i] = s;
        }
}

// ---- Baraff-Witkin shell --------------------------------------------------------
// rest frame: the triangle rotated so its normal is +z (Rodrigues form of the
// rotation taking n to z; n = -z flips x and y), Dm = [uv1 - uv0, uv2 - uv0];
// IB = Dm^-1 as {IB00, IB10, IB01, IB11} (column-major 2x2)
B2_HD void bw_rest(const double* x0, const double* x1, const double* x2, double* IB)
{
    double e1[3], e2[3], n[3];
    sub3(x1, x0, e1);
    sub3(x2, x0, e2);
    cross3(e1, e2, n);
    const double nn = sqrt(dot3(n, n));
    for(int k = 0; k < 3; ++k)
        n[k] /= nn;
    const double z[3] = {0.0, 0.0, 1.0};
    double       vv[3];
    cross3(n, z, vv);
    const double c = dot3(n, z);
    double       R[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    if(c + 1.0 == 0.0)
    {
        R[0] = -1.0;
        R[4] = -1.0;
    }
    else
    {
        const double K[9] = {0.0, -vv[2], vv[1], vv[2], 0.0, -vv[0], -vv[1], vv[0], 0.0};
        for(int i = 0; i < 3; ++i)
            for(int j = 0; j < 3; ++j)
            {
                double kk = 0.0;
                for(int m = 0; m < 3; ++m)
                    kk += K[i * 3 + m] * K[m * 3 + j];
                R[i * 3 + j] += K[i * 3 + j] + kk / (1.0 + c);
            }
    }
    double uv[3][2];
    const double* xs[3] = {x0, x1, x2};
    for(int p = 0; p < 3; ++p)
        for(int r = 0; r < 2; ++r)
            uv[p][r] = R[r * 3 + 0] * xs[p][0] + R[r * 3 + 1] * xs[p][1] + R[r * 3 + 2] * xs[p][2];
    const double m00 = uv[1][0] - uv[0][0], m10 = uv[1][1] - uv[0][1];  // column 0
    const double m01 = uv[2][0] - uv[0][0], m11 = uv[2][1] - uv[0][1];  // column 1
    const double det = m00 * m11 - m01 * m10;
    IB[0] = m11 / det;   // (0,0)
    IB[1] = -m10 / det;  // (1,0)
    IB[2] = -m01 / det;  // (0,1)
    IB[3] = m00 / det;   // (1,1)
}

B2_HD double tri_area(const double* x0, const double* x1, const double* x2)
{
    double e1[3], e2[3], n[3];
    sub3(x1, x0, e1);
    sub3(x2, x0, e2);
    cross3(e1, e2, n);
    return 0.5 * sqrt(dot3(n, n));
}

// F columns fu = F a, fv = F b
B2_HD void bw_F(const double* x0, const double* x1, const double* x2, const double* IB, double* fu, double* fv)
{
    for(int k = 0; k < 3; ++k)
    {
        const double d1 = x1[k] - x0[k], d2 = x2[k] - x0[k];
        fu[k]           = d1 * IB[0] + d2 * IB[1];
        fv[k]           = d1 * IB[2] + d2 * IB[3];
    }
}

B2_HD double bw_energy(const double* fu, const double* fv, double stretch, double shear, double rate)
{
    const double I6 = dot3(fu, fv);
    const double ru = sqrt(dot3(fu, fu)), rv = sqrt(dot3(fv, fv));
    const double cu = ru <= 1.0 ? 0.0 : 1.0, cv = rv <= 1.0 ? 0.0 : 1.0;
    const double st = (ru - 1) * (ru - 1) + cu * rate * (ru - 1) * (ru - 1) * (ru - 1) + (rv - 1) * (rv - 1)
                      + cv * rate * (rv - 1) * (rv - 1) * (rv - 1);
    return stretch * st + shear * I6 * I6;
}

// dE/dF as P[6] = [dE/dfu, dE/dfv] and the 6x6 d2E/dF2 (row-major) in the
// reference's closed form
B2_HD void bw_dF(const double* fu, const double* fv, double stretch, double shear, double rate, double* P, double* HF)
{
    const double I6 = dot3(fu, fv);
    // stretch (the 1/sqrt(I5) singularity guarded as the reference does)
    double I5u = dot3(fu, fu), I5v = dot3(fv, fv);
    I5u        = I5u > 1e-12 ? I5u : 1e-12;
    I5v        = I5v > 1e-12 ? I5v : 1e-12;
    const double su = sqrt(I5u), sv = sqrt(I5v);
    double       cu = 1.0 - 1.0 / su, cv = 1.0 - 1.0 / sv;
    if(I5u > 1.0)
        cu += 1.5 * rate * (su + 1.0 / su - 2.0);
    if(I5v > 1.0)
        cv += 1.5 * rate * (sv + 1.0 / sv - 2.0);
    for(int k = 0; k < 3; ++k)
    {
        P[k]     = stretch * 2.0 * cu * fu[k] + shear * 2.0 * I6 * fv[k];
        P[3 + k] = stretch * 2.0 * cv * fv[k] + shear * 2.0 * I6 * fu[k];
    }
    for(int i = 0; i < 36; ++i)
        HF[i] = 0.0;
    // stretch block of each direction: D I + c fhat fhat^T
    const double* f[2]  = {fu, fv};
    const double  sq[2] = {su, sv};
    const double  I5[2] = {I5u, I5v};
    for(int d = 0; d < 2; ++d)
    {
        const double s = sq[d];
        const double D = s > 1.0 ? (s - 1.0) * (3.0 * s * rate - 3.0 * rate + 2.0) / s : 0.0;
        const double c = s > 1.0 ? (3.0 * I5[d] * rate - 3.0 * rate + 2.0) / s : 2.0;
        double       fh[3];
        const double fn = sqrt(dot3(f[d], f[d]));
        for(int k = 0; k < 3; ++k)
            fh[k] = f[d][k] / fn;
        for(int i = 0; i < 3; ++i)
            for(int j = 0; j < 3; ++j)
                HF[(3 * d + i) * 6 + 3 * d + j] = stretch * ((i == j ? D : 0.0) + c * fh[i] * fh[j]);
    }
    // shear: 2 (|I6| (T - Tq Tq^T / |Tq|^2) + lambda0 q0 q0^T), T = (I + sign(I6) S) / 2
    // with S the swap of the two columns, g = [fv, fu], q0 = unit(I6 S g + lambda0 g)
    double g[6];
    for(int k = 0; k < 3; ++k)
    {
        g[k]     = fv[k];
        g[3 + k] = fu[k];
    }
    const double I2      = dot3(fu, fu) + dot3(fv, fv);
    const double lambda0 = 0.5 * (I2 + sqrt(I2 * I2 + 12.0 * I6 * I6));
    const double sgn     = I6 >= 0.0 ? 1.0 : -1.0;
    double       q0[6];
    double       qn = 0.0;
    for(int i = 0; i < 6; ++i)
    {
        const double Sg = g[i < 3 ? i + 3 : i - 3];
        q0[i]           = I6 * Sg + lambda0 * g[i];
        qn += q0[i] * q0[i];
    }
    qn = sqrt(qn);
    for(int i = 0; i < 6; ++i)
        q0[i] /= qn;
    double Tq[6], tn = 0.0;
    for(int i = 0; i < 6; ++i)
    {
        Tq[i] = 0.5 * (q0[i] + sgn * q0[i < 3 ? i + 3 : i - 3]);
        tn += Tq[i] * Tq[i];
    }
    const double aI6 = fabs(I6);
    for(int i = 0; i < 6; ++i)
        for(int j = 0; j < 6; ++j)
        {
            const double T = 0.5 * ((i == j ? 1.0 : 0.0) + sgn * ((i < 3 ? i + 3 : i - 3) == j ? 1.0 : 0.0));
            HF[i * 6 + j] += shear * 2.0 * (aI6 * (T - Tq[i] * Tq[j] / tn) + lambda0 * q0[i] * q0[j]);
        }
}

// element gradient G[9] and Hessian H[81] (row-major, vertex-major 3-blocks)
// over (x0, x1, x2), scaled by w (rest area x dt^2)
B2_HD void bw_grad_hess(const double* x0, const double* x1, const double* x2, const double* IB, double stretch,
                        double shear, double rate, double w, double* G, double* H)
{
    double fu[3], fv[3], P[6], HF[36];
    bw_F(x0, x1, x2, IB, fu, fv);
    bw_dF(fu, fv, stretch, shear, rate, P, HF);
    // dfu/dx_i = cu[i] I, dfv/dx_i = cv[i] I
    const double cu[3] = {-(IB[0] + IB[1]), IB[0], IB[1]};
    const double cv[3] = {-(IB[2] + IB[3]), IB[2], IB[3]};
    for(int i = 0; i < 3; ++i)
        for(int k = 0; k < 3; ++k)
            G[3 * i + k] = w * (cu[i] * P[k] + cv[i] * P[3 + k]);
    for(int i = 0; i < 3; ++i)
        for(int j = 0; j < 3; ++j)
            for(int p = 0; p < 3; ++p)
                for(int q = 0; q < 3; ++q)
                    H[(3 * i + p) * 9 + 3 * j + q] =
                        w * (cu[i] * cu[j] * HF[p * 6 + q] + cu[i] * cv[j] * HF[p * 6 + 3 + q]
                             + cv[i] * cu[j] * HF[(3 + p) * 6 + q] + cv[i] * cv[j] * HF[(3 + p) * 6 + 3 + q]);
}

// ---- discrete-shell bending -------------------------------------------------------
// signed dihedral angle of the hinge (x0, x1, x2, x3), edge x1-x2
B2_HD double dihedral(const double* x0, const double* x1, const double* x2, const double* x3)
{
    double a[3], b[3], c[3], d[3], n1[3], n2[3], m[3], e[3];
    sub3(x1, x0, a);
    sub3(x2, x0, b);
    cross3(a, b, n1);
    sub3(x2, x3, c);
    sub3(x1, x3, d);
    cross3(c, d, n2);
    double cs = dot3(n1, n2) / sqrt(dot3(n1, n1) * dot3(n2, n2));
    cs        = cs < -1.0 ? -1.0 : (cs > 1.0 ? 1.0 : cs);
    double th = acos(cs);
    cross3(n2, n1, m);
    sub3(x1, x2, e);
    return dot3(m, e) < 0.0 ? -th : th;
}

// d theta / d(x0, x1, x2, x3)
B2_HD void dihedral_grad(const double* x0, const double* x1, const double* x2, const double* x3, double* g)
{
    double e0[3], e1[3], e2[3], e3[3], e4[3], n1[3], n2[3];
    sub3(x2, x1, e0);  // the hinge edge
    sub3(x0, x1, e1);
    sub3(x3, x1, e2);
    sub3(x0, x2, e3);
    sub3(x3, x2, e4);
    cross3(e0, e1, n1);
    cross3(e2, e0, n2);
    const double n1s = dot3(n1, n1), n2s = dot3(n2, n2), el = sqrt(dot3(e0, e0));
    for(int k = 0; k < 3; ++k)
    {
        g[k]     = -el / n1s * n1[k];
        g[3 + k] = -dot3(e0, e3) / (el * n1s) * n1[k] - dot3(e0, e4) / (el * n2s) * n2[k];
        g[6 + k] = dot3(e0, e1) / (el * n1s) * n1[k] + dot3(e0, e2) / (el * n2s) * n2[k];
        g[9 + k] = -el / n2s * n2[k];
    }
}

// rest quantities of a hinge: L0, h_bar, theta_bar
B2_HD void dsb_rest(const double* x0, const double* x1, const double* x2, const double* x3, double* L0,
                    double* h_bar, double* theta_bar)
{
    double e[3], a[3], b[3], c[3], d[3], n1[3], n2[3];
    sub3(x2, x1, e);
    *L0 = sqrt(dot3(e, e));
    sub3(x1, x0, a);
    sub3(x2, x0, b);
    cross3(a, b, n1);
    sub3(x2, x3, c);
    sub3(x1, x3, d);
    cross3(c, d, n2);
    const double A = (sqrt(dot3(n1, n1)) + sqrt(dot3(n2, n2))) / 2.0;
    *h_bar         = A / 3.0 / *L0;
    *theta_bar     = dihedral(x0, x1, x2, x3);
}

B2_HD double dsb_energy(const double* x0, const double* x1, const double* x2, const double* x3, double L0,
                        double h_bar, double theta_bar, double kappa)
{
    const double d = dihedral(x0, x1, x2, x3) - theta_bar;
    return L0 * kappa * d * d / h_bar;
}

// gradient G[12] and Gauss-Newton Hessian H[144] scaled by w (dt^2)
B2_HD void dsb_grad_hess(const double* x0, const double* x1, const double* x2, const double* x3, double L0,
                         double h_bar, double theta_bar, double kappa, double w, double* G, double* H)
{
    const double th = dihedral(x0, x1, x2, x3);
    double       g[12];
    dihedral_grad(x0, x1, x2, x3, g);
    const double dE  = 2.0 * L0 * kappa * (th - theta_bar) / h_bar;
    const double ddE = 2.0 * L0 * kappa / h_bar;
    for(int i = 0; i < 12; ++i)
        G[i] = w * dE * g[i];
    const double c = ddE * w;
    for(int i = 0; i < 12; ++i)
    {
        const double ci = c * g[i];
        H[i * 12 + i]   = ci * g[i];
        for(int j = i + 1; j < 12; ++j)
        {
            const double v = ci * g[j];
            H[i * 12 + j]  = v;
            H[j * 12 + i]  = v;
        }
    }
}

// ---- affine-body orthogonality potential -------------------------------------------
B2_HD double ortho_energy(const double* q, double kappa)
{
    double e = 0.0;
    for(int i = 0; i < 3; ++i)
        for(int j = 0; j < 3; ++j)
        {
            const double d = dot3(q + 3 + 3 * i, q + 3 + 3 * j) - (i == j ? 1.0 : 0.0);
            e += d * d;
        }
    return kappa * e;
}

// gradient over q[3..11] (G9) and the PSD-projected Hessian H9 (81), scaled by w
B2_HD void ortho_grad_hess(const double* q, double kappa, double w, double* G9, double* H9)
{
    const double* a[3] = {q + 3, q + 6, q + 9};
    double        Gm[3][3];
    for(int i = 0; i < 3; ++i)
        for(int j = 0; j < 3; ++j)
            Gm[i][j] = dot3(a[i], a[j]) - (i == j ? 1.0 : 0.0);
    // g_k = 4 kappa sum_j (a_k . a_j - delta_kj) a_j
    for(int k = 0; k < 3; ++k)
        for(int c = 0; c < 3; ++c)
        {
            double s = 0.0;
            for(int j = 0; j < 3; ++j)
                s += Gm[k][j] * a[j][c];
            G9[3 * k + c] = w * 4.0 * kappa * s;
        }
    // H_kl = 4 kappa (delta_kl sum_j a_j a_j^T + a_l a_k^T + (a_k . a_l - delta_kl) I)
    double S[3][3];
    for(int r = 0; r < 3; ++r)
        for(int c = 0; c < 3; ++c)
            S[r][c] = a[0][r] * a[0][c] + a[1][r] * a[1][c] + a[2][r] * a[2][c];
    for(int k = 0; k < 3; ++k)
        for(int l = 0; l < 3; ++l)
            for(int r = 0; r < 3; ++r)
                for(int c = 0; c < 3; ++c)
                    H9[(3 * k + r) * 9 + 3 * l + c] =
                        4.0 * kappa
                        * ((k == l ? S[r][c] : 0.0) + a[l][r] * a[k][c] + (r == c ? Gm[k][l] : 0.0));
    project_psd<9>(H9);
    for(int i = 0; i < 81; ++i)
        H9[i] *= w;
}

// ---- second-order forward differentiation over 12 variables ------------------------
// value, gradient and the upper triangle of the Hessian (packed row by row)
struct Jet12
{
    double v;
    double g[12];
    double h[78];
};
B2_HD int hidx(int i, int j) { return i * 12 - i * (i - 1) / 2 + (j - i); }  // i <= j
B2_HD void jet_const(Jet12& a, double v)
{
    a.v = v;
    for(int i = 0; i < 12; ++i)
        a.g[i] = 0.0;
    for(int i = 0; i < 78; ++i)
        a.h[i] = 0.0;
}
B2_HD void jet_var(Jet12& a, double v, int k)
{
    jet_const(a, v);
    a.g[k] = 1.0;
}
B2_HD void jet_add(const Jet12& a, const Jet12& b, Jet12& r, double sb = 1.0)
{
    r.v = a.v + sb * b.v;
    for(int i = 0; i < 12; ++i)
        r.g[i] = a.g[i] + sb * b.g[i];
    for(int i = 0; i < 78; ++i)
        r.h[i] = a.h[i] + sb * b.h[i];
}
B2_HD void jet_mul(const Jet12& a, const Jet12& b, Jet12& r)
{
    Jet12 t;
    t.v = a.v * b.v;
    for(int i = 0; i < 12; ++i)
        t.g[i] = a.v * b.g[i] + b.v * a.g[i];
    for(int i = 0; i < 12; ++i)
        for(int j = i; j < 12; ++j)
        {
            const int k = hidx(i, j);
            t.h[k]      = a.v * b.h[k] + b.v * a.h[k] + a.g[i] * b.g[j] + a.g[j] * b.g[i];
        }
    r = t;
}
// r = f(a) for a scalar function with f, f', f'' at a.v
B2_HD void jet_compose(const Jet12& a, double f, double f1, double f2, Jet12& r)
{
    Jet12 t;
    t.v = f;
    for(int i = 0; i < 12; ++i)
        t.g[i] = f1 * a.g[i];
    for(int i = 0; i < 12; ++i)
        for(int j = i; j < 12; ++j)
        {
            const int k = hidx(i, j);
            t.h[k]      = f1 * a.h[k] + f2 * a.g[i] * a.g[j];
        }
    r = t;
}
B2_HD void jet_div(const Jet12& a, const Jet12& b, Jet12& r)
{
    Jet12        ib;
    const double iv = 1.0 / b.v;
    jet_compose(b, iv, -iv * iv, 2.0 * iv * iv * iv, ib);
    jet_mul(a, ib, r);
}
B2_HD void jet_dot3(const Jet12* a, const Jet12* b, Jet12& r)
{
    Jet12 t;
    jet_mul(a[0], b[0], r);
    jet_mul(a[1], b[1], t);
    jet_add(r, t, r);
    jet_mul(a[2], b[2], t);
    jet_add(r, t, r);
}
B2_HD void jet_cross3(const Jet12* a, const Jet12* b, Jet12* r)
{
    Jet12 t, u;
    for(int c = 0; c < 3; ++c)
    {
        const int c1 = (c + 1) % 3, c2 = (c + 2) % 3;
        jet_mul(a[c1], b[c2], t);
        jet_mul(a[c2], b[c1], u);
        jet_add(t, u, r[c], -1.0);
    }
}

// squared distances as Jets of the 12 pair coordinates X (vertex k at 3k)
enum PairType
{
    PAIR_PP = 0,
    PAIR_PE = 1,
    PAIR_PT = 2,
    PAIR_EE = 3
};
// vertex i of the pair as three Jets
B2_HD void jet_point(const double* X, int i, Jet12* p)
{
    for(int c = 0; c < 3; ++c)
        jet_var(p[c], X[3 * i + c], 3 * i + c);
}
B2_HD void jet_d2_pp(const double* X, int a, int b, Jet12& D)
{
    Jet12 pa[3], pb[3], d[3];
    jet_point(X, a, pa);
    jet_point(X, b, pb);
    for(int c = 0; c < 3; ++c)
        jet_add(pa[c], pb[c], d[c], -1.0);
    jet_dot3(d, d, D);
}
// |(p - e0) x (e1 - e0)|^2 / |e1 - e0|^2
B2_HD void jet_d2_pe(const double* X, int p, int e0, int e1, Jet12& D)
{
    Jet12 P[3], A[3], B[3], w[3], e[3], n[3], nn, ee;
    jet_point(X, p, P);
    jet_point(X, e0, A);
    jet_point(X, e1, B);
    for(int c = 0; c < 3; ++c)
    {
        jet_add(P[c], A[c], w[c], -1.0);
        jet_add(B[c], A[c], e[c], -1.0);
    }
    jet_cross3(w, e, n);
    jet_dot3(n, n, nn);
    jet_dot3(e, e, ee);
    jet_div(nn, ee, D);
}
// ((q - a0) . n)^2 / |n|^2, n = u x v: point-plane (u, v the triangle edges) and
// line-line (u, v the two edges)
B2_HD void jet_d2_plane(const Jet12* q, const Jet12* a0, const Jet12* u, const Jet12* v, Jet12& D)
{
    Jet12 n[3], w[3], wn, nn;
    jet_cross3(u, v, n);
    for(int c = 0; c < 3; ++c)
        jet_add(q[c], a0[c], w[c], -1.0);
    jet_dot3(w, n, wn);
    jet_dot3(n, n, nn);
    jet_mul(wn, wn, wn);
    jet_div(wn, nn, D);
}
B2_HD void jet_d2_pt(const double* X, Jet12& D)
{
    Jet12 P[3], T0[3], T1[3], T2[3], u[3], v[3];
    jet_point(X, 0, P);
    jet_point(X, 1, T0);
    jet_point(X, 2, T1);
    jet_point(X, 3, T2);
    for(int c = 0; c < 3; ++c)
    {
        jet_add(T1[c], T0[c], u[c], -1.0);
        jet_add(T2[c], T0[c], v[c], -1.0);
    }
    jet_d2_plane(P, T0, u, v, D);
}
B2_HD void jet_d2_ee(const double* X, Jet12& D)
{
    Jet12 A0[3], A1[3], B0[3], B1[3], u[3], v[3];
    jet_point(X, 0, A0);
    jet_point(X, 1, A1);
    jet_point(X, 2, B0);
    jet_point(X, 3, B1);
    for(int c = 0; c < 3; ++c)
    {
        jet_add(A1[c], A0[c], u[c], -1.0);
        jet_add(B1[c], B0[c], v[c], -1.0);
    }
    jet_d2_plane(B0, A0, u, v, D);
}

// closest-feature type of a point-triangle pair (p, t0, t1, t2): the outside
// regions of the edges t0t1, t1t2, t2t0 (point-edge), then of the corners
// (point-point), else the face; returns the type and the participating
// pair-local vertices in v[]
B2_HD int pt_type(const double* X, int* v, int* nv)
{
    const double *p = X, *t[3] = {X + 3, X + 6, X + 9};
    double        e1[3], e2[3], n[3];
    sub3(t[1], t[0], e1);
    sub3(t[2], t[0], e2);
    cross3(e1, e2, n);
    double s[3];  // parameter along each edge (t0t1, t1t2, t2t0)
    bool   out[3];
    for(int k = 0; k < 3; ++k)
    {
        const double* a = t[k];
        const double* b = t[(k + 1) % 3];
        double        e[3], o[3], w[3];
        sub3(b, a, e);
        cross3(e, n, o);  // outward normal of the edge in the plane
        sub3(p, a, w);
        // coordinates of w in the (e, o) basis (e . o = 0)
        s[k]   = dot3(w, e) / dot3(e, e);
        out[k] = dot3(w, o) / dot3(o, o) >= 0.0;
    }
    for(int k = 0; k < 3; ++k)
        if(s[k] > 0.0 && s[k] < 1.0 && out[k])
        {
            v[0] = 0;
            v[1] = 1 + k;
            v[2] = 1 + (k + 1) % 3;
            *nv  = 3;
            return PAIR_PE;
        }
    // corners: t_k is closest when p is before edge k and past edge k-1
    for(int k = 0; k < 3; ++k)
        if(s[k] <= 0.0 && s[(k + 2) % 3] >= 1.0)
        {
            v[0] = 0;
            v[1] = 1 + k;
            *nv  = 2;
            return PAIR_PP;
        }
    v[0] = 0;
    v[1] = 1;
    v[2] = 2;
    v[3] = 3;
    *nv  = 4;
    return PAIR_PT;
}

// closest-feature type of an edge-edge pair (a0, a1, b0, b1): the segments'
// closest points by the clamped line parameters; an interior pair is EE, one
// clamped end gives point-edge, two give point-point; (near-)parallel edges
// take the closest of the four endpoint-to-segment candidates
B2_HD int ee_type(const double* X, int* v, int* nv)
{
    const double *a0 = X, *a1 = X + 3, *b0 = X + 6, *b1 = X + 9;
    double        u[3], w[3], z[3], ux[3];
    sub3(a1, a0, u);
    sub3(b1, b0, w);
    sub3(a0, b0, z);
    const double a = dot3(u, u), b = dot3(u, w), c = dot3(w, w), d = dot3(u, z), e = dot3(w, z);
    const double den = a * c - b * b;
    cross3(u, w, ux);
    // endpoint-to-segment candidates (point index, segment start, segment end)
    auto pseg = [&](int pi, int s0, int s1, double* dist, int* vv, int* n)
    {
        const double *P = X + 3 * pi, *S0 = X + 3 * s0, *S1 = X + 3 * s1;
        double        sv[3], pw[3];
        sub3(S1, S0, sv);
        sub3(P, S0, pw);
        const double t = dot3(pw, sv) / dot3(sv, sv);
        if(t <= 0.0 || t >= 1.0)
        {
            const double* Q = t <= 0.0 ? S0 : S1;
            double        q[3];
            sub3(P, Q, q);
            *dist = dot3(q, q);
            vv[0] = pi;
            vv[1] = t <= 0.0 ? s0 : s1;
            *n    = 2;
        }
        else
        {
            double q[3];
            for(int k = 0; k < 3; ++k)
                q[k] = pw[k] - t * sv[k];
            *dist = dot3(q, q);
            vv[0] = pi;
            vv[1] = s0;
            vv[2] = s1;
            *n    = 3;
        }
    };
    const bool parallel = dot3(ux, ux) <= 1e-12 * a * c;
    if(!parallel)
    {
        const double sN = b * e - c * d, tN = a * e - b * d;
        const bool   s_in = sN > 0.0 && sN < den, t_in = tN > 0.0 && tN < den;
        if(s_in && t_in)
        {
            v[0] = 0;
            v[1] = 1;
            v[2] = 2;
            v[3] = 3;
            *nv  = 4;
            return PAIR_EE;
        }
    }
    double best = 1e300;
    int    bv[3], bn = 0;
    const int cand[4][3] = {{0, 2, 3}, {1, 2, 3}, {2, 0, 1}, {3, 0, 1}};
    for(int k = 0; k < 4; ++k)
    {
        double dist;
        int    vv[3], n;
        pseg(cand[k][0], cand[k][1], cand[k][2], &dist, vv, &n);
        if(dist < best)
        {
            best = dist;
            bn   = n;
            for(int i = 0; i < n; ++i)
                bv[i] = vv[i];
        }
    }
    for(int i = 0; i < bn; ++i)
        v[i] = bv[i];
    *nv = bn;
    return bn == 2 ? PAIR_PP : PAIR_PE;
}

// B(D) = -k (D - Dh)^2 log(D / Dh) and its first two derivatives
B2_HD void barrier_B(double D, double Dh, double k, double* B0, double* B1, double* B2)
{
    const double t = D - Dh, l = log(D / Dh);
    *B0            = -k * t * t * l;
    *B1            = -k * (2.0 * t * l + t * t / D);
    *B2            = -k * (2.0 * l + 4.0 * t / D - t * t / (D * D));
}

// one contact pair: X[12] its 4 vertices ((p, t0, t1, t2) when is_ee is 0,
// (a0, a1, b0, b1) otherwise), eps the edge-edge mollifier threshold (unused
// for point-triangle), k = kappa dt^2; G[12], H[144] over the 4 vertices (zero
// rows for vertices outside the type's stencil). Returns the type, or -1 when
// the pair is at or beyond dhat (G, H zero).
B2_HD_NOINLINE int contact_grad_hess(const double* X, int is_ee, double eps, double dhat, double k, double* G,
                                     double* H)
{
    for(int i = 0; i < 12; ++i)
        G[i] = 0.0;
    for(int i = 0; i < 144; ++i)
        H[i] = 0.0;
    int       v[4], nv = 0;
    const int type = is_ee ? ee_type(X, v, &nv) : pt_type(X, v, &nv);
    Jet12     D;
    if(type == PAIR_PT)
        jet_d2_pt(X, D);
    else if(type == PAIR_EE)
        jet_d2_ee(X, D);
    else if(type == PAIR_PE)
        jet_d2_pe(X, v[0], v[1], v[2], D);
    else
        jet_d2_pp(X, v[0], v[1], D);
    const double Dh = dhat * dhat;
    if(!(D.v < Dh) || !(D.v > 0.0))
        return -1;
    double B0, B1, B2;
    barrier_B(D.v, Dh, k, &B0, &B1, &B2);
    // edge-edge mollifier
    bool  moll = false;
    Jet12 E;
    if(is_ee)
    {
        double u[3], w[3], ux[3];
        sub3(X + 3, X, u);
        sub3(X + 9, X + 6, w);
        cross3(u, w, ux);
        moll = dot3(ux, ux) < eps;
    }
    if(moll)
    {
        Jet12 A0[3], A1[3], B0j[3], B1j[3], u[3], w[3], n[3], c, m, Bj;
        jet_point(X, 0, A0);
        jet_point(X, 1, A1);
        jet_point(X, 2, B0j);
        jet_point(X, 3, B1j);
        for(int q = 0; q < 3; ++q)
        {
            jet_add(A1[q], A0[q], u[q], -1.0);
            jet_add(B1j[q], B0j[q], w[q], -1.0);
        }
        jet_cross3(u, w, n);
        jet_dot3(n, n, c);
        const double x = c.v / eps;
        jet_compose(c, (2.0 - x) * x, 2.0 / eps * (1.0 - x), -2.0 / (eps * eps), m);
        jet_compose(D, B0, B1, B2, Bj);
        jet_mul(m, Bj, E);
    }
    if(moll || type == PAIR_PT || type == PAIR_EE)
    {
        if(!moll)
            jet_compose(D, B0, B1, B2, E);
        for(int i = 0; i < 12; ++i)
            G[i] = E.g[i];
        for(int i = 0; i < 12; ++i)
            for(int j = i; j < 12; ++j)
                H[i * 12 + j] = H[j * 12 + i] = E.h[hidx(i, j)];
        project_psd<12>(H);
        return type;
    }
    // point-edge / point-point: the closed rank-1 form
    const double c = B2 + B1 / (2.0 * D.v);
    for(int i = 0; i < 12; ++i)
        G[i] = B1 * D.g[i];
    for(int i = 0; i < 12; ++i)
        for(int j = 0; j < 12; ++j)
            H[i * 12 + j] = c * D.g[i] * D.g[j];
    return type;
}
// ---- value-only distances, energy and continuous collision detection ------------
B2_HD double d2_pp(const double* a, const double* b)
{
    double d[3];
    sub3(a, b, d);
    return dot3(d, d);
}
// |(p - e0) x (e1 - e0)|^2 / |e1 - e0|^2
B2_HD double d2_pe(const double* p, const double* e0, const double* e1)
{
    double e[3], w[3], c[3];
    sub3(e1, e0, e);
    sub3(p, e0, w);
    cross3(w, e, c);
    return dot3(c, c) / dot3(e, e);
}
// ((q - a0) . n)^2 / |n|^2, n = u x v
B2_HD double d2_plane(const double* q, const double* a0, const double* u, const double* v)
{
    double n[3], w[3];
    cross3(u, v, n);
    sub3(q, a0, w);
    const double wn = dot3(w, n);
    return wn * wn / dot3(n, n);
}
// squared distance of a pair by its closest-feature type (the value the
// contact Jets carry)
B2_HD double pair_d2(const double* X, int is_ee)
{
    int       v[4], nv = 0;
    const int type = is_ee ? ee_type(X, v, &nv) : pt_type(X, v, &nv);
    if(type == PAIR_PP)
        return d2_pp(X + 3 * v[0], X + 3 * v[1]);
    if(type == PAIR_PE)
        return d2_pe(X + 3 * v[0], X + 3 * v[1], X + 3 * v[2]);
    double u[3], w[3];
    if(type == PAIR_PT)
    {
        sub3(X + 6, X + 3, u);
        sub3(X + 9, X + 3, w);
        return d2_plane(X, X + 3, u, w);
    }
    sub3(X + 3, X, u);
    sub3(X + 9, X + 6, w);
    return d2_plane(X + 6, X, u, w);
}

// barrier energy of one pair (k = kappa dt^2): B(D), times the edge-edge
// mollifier (2 - c/eps) c/eps (c = |ea x eb|^2) below eps; 0 at or beyond dhat
// (the energy whose gradient and Hessian contact_grad_hess returns)
B2_HD double contact_energy(const double* X, int is_ee, double eps, double dhat, double k)
{
    const double D = pair_d2(X, is_ee), Dh = dhat * dhat;
    if(!(D < Dh) || !(D > 0.0))
        return 0.0;
    double B0, B1, B2;
    barrier_B(D, Dh, k, &B0, &B1, &B2);
    if(is_ee)
    {
        double u[3], w[3], c[3];
        sub3(X + 3, X, u);
        sub3(X + 9, X + 6, w);
        cross3(u, w, c);
        const double cc = dot3(c, c);
        if(cc < eps)
        {
            const double x = cc / eps;
            return (2.0 - x) * x * B0;
        }
    }
    return B0;
}

// the distance the CCD advances on: an edge-edge pair whose distance is not
// above the thickness is a (nearly) parallel pair far apart, measured by its
// closest endpoints instead
B2_HD double ccd_d2(const double* X, int is_ee, double xi)
{
    double d2 = pair_d2(X, is_ee);
    if(is_ee && d2 - xi * xi <= 0.0)
    {
        const double a = d2_pp(X, X + 6), b = d2_pp(X, X + 9), c = d2_pp(X + 3, X + 6), d = d2_pp(X + 3, X + 9);
        d2 = fmin(fmin(a, b), fmin(c, d));
    }
    return d2;
}

// swept AABBs of the pair's two sides (point | triangle, edge | edge) over the
// step X -> X + dX: true when they come within dist on every axis
B2_HD bool ccd_broadphase(const double* X, const double* dX, int is_ee, double dist)
{
    const int na = is_ee ? 2 : 1;
    for(int c = 0; c < 3; ++c)
    {
        double amin = 1e300, amax = -1e300, bmin = 1e300, bmax = -1e300;
        for(int i = 0; i < 4; ++i)
        {
            const double p = X[3 * i + c], q = p + dX[3 * i + c];
            double&      lo = i < na ? amin : bmin;
            double&      hi = i < na ? amax : bmax;
            lo              = fmin(lo, fmin(p, q));
            hi              = fmax(hi, fmax(p, q));
        }
        if(amin - bmax > dist || bmin - amax > dist)
            return false;
    }
    return true;
}

// Additive CCD of one pair (X0 the positions, dX0 its displacement over the
// step): conservative advancement on the pair's distance (Li et al.,
// Codimensional Incremental Potential Contact, 2021). The pair's mean
// displacement is removed; l = the largest displacement of each side,
// summed; each step advances by (1 - eta) (d^2 - xi^2) / ((d + xi) l), which no
// motion bounded by l can cross; the loop ends with a hit when the distance
// function falls below eta times its start (after the first step: the time
// reached is the time of impact, the last step not taken) and without one
// when the time passes toi_max. max_iter steps end it with a hit at the time
// reached.
B2_HD bool accd_pair(const double* X0, const double* dX0, int is_ee, double eta, double xi, int max_iter,
                     double toi_max, double* toi)
{
    double X[12], dX[12], mov[3], n2[4];
    for(int c = 0; c < 3; ++c)
        mov[c] = (((dX0[c] + dX0[3 + c]) + dX0[6 + c]) + dX0[9 + c]) / 4.0;
    for(int i = 0; i < 4; ++i)
    {
        for(int c = 0; c < 3; ++c)
        {
            X[3 * i + c]  = X0[3 * i + c];
            dX[3 * i + c] = dX0[3 * i + c] - mov[c];
        }
        n2[i] = dot3(dX + 3 * i, dX + 3 * i);
    }
    const double l = is_ee ? sqrt(fmax(n2[0], n2[1])) + sqrt(fmax(n2[2], n2[3]))
                           : sqrt(n2[0]) + sqrt(fmax(fmax(n2[1], n2[2]), n2[3]));
    *toi = toi_max;
    if(!(l > 0.0))
        return false;
    const double xi2 = xi * xi;
    double       d2  = ccd_d2(X, is_ee, xi);
    double       f   = d2 - xi2;
    double       d   = sqrt(d2);
    const double gap = eta * f / (d + xi);
    double       t   = 0.0;
    for(;;)
    {
        if(max_iter-- <= 0)
        {
            *toi = t;
            return true;
        }
        const double tl = (1.0 - eta) * f / ((d + xi) * l);
        for(int i = 0; i < 12; ++i)
            X[i] += tl * dX[i];
        d2 = ccd_d2(X, is_ee, xi);
        f  = d2 - xi2;
        d  = sqrt(d2);
        if(t > 0.0 && f / (d + xi) < gap)
            break;
        t += tl;
        if(t > toi_max)
            return false;
    }
    *toi = t;
    return true;
}

}  // namespace b2el
