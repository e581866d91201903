// Preconditioner build/apply dispatch and the PCG loop (FP64 path).
//
// PCG semantics follow LinearFusedPCG::fused_pcg
// (src/backends/cuda/linear_system/linear_fused_pcg.cu:1782-2005) and
// LinearPCG::pcg (src/backends/cuda/linear_system/linear_pcg.cu:558-644):
// x0 = 0 (or the given guess), r = b - A x0, z = P r, p = z; per iteration
// alpha = rz / pAp, x += alpha p, r -= alpha Ap, z = P r, rz' = r.z,
// converged when |rz'| <= tol |rz0| (or, with the relative-residual rule,
// ||r|| <= tol ||b||), beta = rz'/rz, p = z + beta p; max_iter = 2 n; the
// PSD guard re-runs with the preconditioner bypassed when rz0 < 0 or is not
// finite (:1819-1877). The scalars live on the device; the convergence flag
// freezes every kernel once set, so `check_interval` iterations can be
// replayed from one CUDA graph and checked once by the host, as the
// reference's graph block replay does (:1923-1998).
#include "b2s_internal.cuh"
#include "b2s_reduce.cuh"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>

namespace b2s
{
void spmv_f64_launch(b2s_solver* s, const Matrix& A, const double* x, double* y, Reduction& red, double* d_dot,
                     const int* stop);
int* device_error_flag(b2s_solver* s);
void check_device_errors(b2s_solver* s);
int  spmv_grid(int64_t U);
void ensure_reduction(Reduction& red, int grid, int nv);
void mas_apply_levels(b2s_solver* s, const double* r, const int* converged);
void mas_apply_levels_f32(b2s_solver* s, const float* r, const int* converged, bool bf16);
void mas_pack_bf16(b2s_solver* s);
void spmv_f32_launch(b2s_solver* s, const Matrix& A, const float* x, float* y, Reduction& red, double* d_dot,
                     const int* stop);
void pcg_solve_mixed(b2s_solver* s, const double* b, double* x, const b2s_pcg_options& o, b2s_pcg_stats& st_out);
void build_row_groups(b2s_solver* s, Matrix& A);

namespace
{
constexpr int VEC_BLOCK = 256;

int vec_grid(int64_t n)
{
    int64_t g = (n + VEC_BLOCK - 1) / VEC_BLOCK;
    const int64_t cap = (int64_t)NUM_SMS_HINT * 8;
    if(g > cap)
        g = cap;
    return (int)(g < 1 ? 1 : g);
}

__device__ __forceinline__ bool frozen(const PcgScalars* sc) { return sc && sc->converged != 0; }

// 3x3 block Jacobi inverses (row-major), identity where the diagonal block is
// missing or singular
__global__ void k_diag_inverse(int32_t nb, const int32_t* diag_index, const double* vals, int64_t U, double* dinv)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= nb)
        return;
    const int k = diag_index[i];
    double*   o = dinv + (size_t)i * 9;
    if(k < 0)
    {
        for(int q = 0; q < 9; ++q)
            o[q] = (q % 4 == 0) ? 1.0 : 0.0;
        return;
    }
    double m[9];  // row-major
#pragma unroll
    for(int p = 0; p < 3; ++p)
#pragma unroll
        for(int q = 0; q < 3; ++q)
            m[p * 3 + q] = vals[(int64_t)(q * 3 + p) * U + k];
    const double c0 = m[4] * m[8] - m[5] * m[7], c1 = m[5] * m[6] - m[3] * m[8], c2 = m[3] * m[7] - m[4] * m[6];
    const double det = m[0] * c0 + m[1] * c1 + m[2] * c2;
    if(!(det != 0.0) || !isfinite(det))
    {
        for(int q = 0; q < 9; ++q)
            o[q] = (q % 4 == 0) ? 1.0 : 0.0;
        return;
    }
    const double id = 1.0 / det;
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

// 12x12 block-Jacobi inverses of the affine bodies (ABDDiagPreconditioner,
// src/backends/cuda/affine_body/abd_diag_preconditioner.cu:15-125: the inverse
// of each body's full 12x12 diagonal Hessian block): body b owns block rows
// off + 4b .. off + 4b + 3; its 10 stored upper 3x3 blocks are gathered from
// the BSR (binary search of the sorted columns), mirrored, and inverted in FP64
// by Gauss-Jordan with partial pivoting (identity when singular). One thread
// per body; out: 144 doubles per body, row-major.
__global__ void k_abd_inverse(int n_bodies, int off, const int32_t* __restrict__ rowptr,
                              const int32_t* __restrict__ cols, const double* __restrict__ vals, int64_t S,
                              double* __restrict__ out)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if(b >= n_bodies)
        return;
    double H[12][24];
    for(int i = 0; i < 12; ++i)
        for(int j = 0; j < 24; ++j)
            H[i][j] = (j == 12 + i) ? 1.0 : 0.0;
    for(int bi = 0; bi < 4; ++bi)
    {
        const int row = off + 4 * b + bi;
        int       lo = rowptr[row], hi = rowptr[row + 1];
        for(int bj = bi; bj < 4; ++bj)
        {
            const int col = off + 4 * b + bj;
            int       l = lo, h = hi;
            while(l < h)
            {
                const int m = (l + h) >> 1;
                if(cols[m] < col)
                    l = m + 1;
                else
                    h = m;
            }
            if(l >= hi || cols[l] != col)
                continue;
            for(int p = 0; p < 3; ++p)
                for(int q = 0; q < 3; ++q)
                {
                    const double v = vals[(int64_t)(q * 3 + p) * S + l];
                    H[3 * bi + p][3 * bj + q] = v;
                    if(bi != bj)
                        H[3 * bj + q][3 * bi + p] = v;
                }
        }
    }
    bool ok = true;
    for(int c = 0; c < 12 && ok; ++c)
    {
        int piv = c;
        for(int r = c + 1; r < 12; ++r)
            if(fabs(H[r][c]) > fabs(H[piv][c]))
                piv = r;
        if(!(fabs(H[piv][c]) > 0.0) || !isfinite(H[piv][c]))
        {
            ok = false;
            break;
        }
        if(piv != c)
            for(int j = 0; j < 24; ++j)
            {
                const double t = H[c][j];
                H[c][j]        = H[piv][j];
                H[piv][j]      = t;
            }
        const double inv = 1.0 / H[c][c];
        for(int j = 0; j < 24; ++j)
            H[c][j] *= inv;
        for(int r = 0; r < 12; ++r)
            if(r != c)
            {
                const double f = H[r][c];
                if(f != 0.0)
                    for(int j = 0; j < 24; ++j)
                        H[r][j] -= f * H[c][j];
            }
    }
    double* o = out + (size_t)b * 144;
    for(int i = 0; i < 12; ++i)
        for(int j = 0; j < 12; ++j)
            o[i * 12 + j] = ok ? H[i][12 + j] : (i == j ? 1.0 : 0.0);
}

struct MasView
{
    int            active;  // MAS present
    int            off, vn, L;
    int            abd_off, abd_n;  // affine-body range: block rows abd_off .. abd_off + 4 abd_n
    const double*  abd_inv;         // [abd_n * 144]
    const int32_t* r2p;
    const int32_t* node1;  // [vn] level-1 node of each vertex (its Z slot holds the folded coarse sum)
    int            T;      // coarse levels (L-1)
    const float*   Z;      // node values by slot
};

// node i's three entries of r: NS = 3 values per node (FP64 vectors), or 4
// (the padded FP32 vectors of the mixed PCG: one 16-byte load)
template <typename VT, int NS>
__device__ __forceinline__ void load_r(const VT* r, int64_t i, double& a, double& b, double& c)
{
    if constexpr(NS == 4)
    {
        const float4 q = *reinterpret_cast<const float4*>(r + 4 * i);
        a = q.x;
        b = q.y;
        c = q.z;
    }
    else
    {
        a = r[3 * i];
        b = r[3 * i + 1];
        c = r[3 * i + 2];
    }
}

// z_i for block row i: MAS (partitioned vertices of its range), else 3x3
// block Jacobi (kind 1 / 2), else identity (kind 0); r_i is returned in rr
template <typename VT, int NS>
__device__ __forceinline__ void precond_row(int kind, const MasView& mv, const double* dinv, const VT* r, int i,
                                            double z[3], double rr[3])
{
    load_r<VT, NS>(r, i, rr[0], rr[1], rr[2]);
    const double r0 = rr[0], r1 = rr[1], r2 = rr[2];
    if(kind == B2S_PRECOND_MAS && mv.active)
    {
        const int v = i - mv.off;
        if(v >= 0 && v < mv.vn)
        {
            const int p = mv.r2p[v];
            if(p >= 0)
            {
                // the fine level's Z of the vertex's slot plus the coarse
                // levels' sum folded into its level-1 node
                const int n1 = mv.T > 0 ? mv.node1[v] : -1;
                float     c0 = mv.Z[3 * (int64_t)p], c1 = mv.Z[3 * (int64_t)p + 1], c2 = mv.Z[3 * (int64_t)p + 2];
                if(n1 >= 0)
                {
                    c0 += mv.Z[3 * (int64_t)n1];
                    c1 += mv.Z[3 * (int64_t)n1 + 1];
                    c2 += mv.Z[3 * (int64_t)n1 + 2];
                }
                z[0] = (double)c0;
                z[1] = (double)c1;
                z[2] = (double)c2;
                return;
            }
        }
    }
    if(kind == B2S_PRECOND_NONE)
    {
        z[0] = r0;
        z[1] = r1;
        z[2] = r2;
        return;
    }
    if(mv.abd_n > 0 && i >= mv.abd_off && i < mv.abd_off + 4 * mv.abd_n)
    {
        // row l of body b: z = (H_b^-1)[3l .. 3l+2][0 .. 11] r_b
        const int     b = (i - mv.abd_off) >> 2, l = (i - mv.abd_off) & 3;
        const double* Hi = mv.abd_inv + (size_t)b * 144 + 36 * l;
        const int64_t n0 = (int64_t)mv.abd_off + 4 * b;  // the body's first node
        double        a0 = 0.0, a1 = 0.0, a2 = 0.0;
        for(int j = 0; j < 12; ++j)
        {
            const double rj = r[NS * (n0 + j / 3) + j % 3];
            a0 += Hi[j] * rj;
            a1 += Hi[12 + j] * rj;
            a2 += Hi[24 + j] * rj;
        }
        z[0] = a0;
        z[1] = a1;
        z[2] = a2;
        return;
    }
    const double* D = dinv + (size_t)i * 9;
    z[0] = D[0] * r0 + D[1] * r1 + D[2] * r2;
    z[1] = D[3] * r0 + D[4] * r1 + D[5] * r2;
    z[2] = D[6] * r0 + D[7] * r1 + D[8] * r2;
}

// z = P r for every block row; with `sc`, also r.z and r.r (FP64 sums) and
// the scalar update of the iteration (last block). VT: vector storage type.
// 32 registers, so the whole reduction grid (8 CTAs per SM) is resident at
// once (with 40 the last quarter of the grid ran as a second wave: the MAS
// apply with this finish measured 77.4 -> 73.8 us on 551 k vertices).
template <typename VT, int NS>
__global__ void __launch_bounds__(RED_BLOCK, 8) k_precond_finish(int32_t nb, int kind, MasView mv,
                                                              const double* __restrict__ dinv,
                                                              const VT* __restrict__ r, VT* __restrict__ z,
                                                              PcgScalars* sc, double* partials,
                                                              unsigned int* counter)
{
    if(frozen(sc))
        return;
    double rz = 0.0, rr = 0.0;
    for(int i = blockIdx.x * RED_BLOCK + threadIdx.x; i < nb; i += gridDim.x * RED_BLOCK)
    {
        double zi[3], ri[3];
        precond_row<VT, NS>(kind, mv, dinv, r, i, zi, ri);
        const VT z0 = (VT)zi[0], z1 = (VT)zi[1], z2 = (VT)zi[2];
        if constexpr(NS == 4)
            *reinterpret_cast<float4*>(z + 4 * (int64_t)i) = make_float4(z0, z1, z2, 0.0f);
        else
        {
            z[3 * (int64_t)i]     = z0;
            z[3 * (int64_t)i + 1] = z1;
            z[3 * (int64_t)i + 2] = z2;
        }
        if(sc)
        {
            rz += ri[0] * (double)z0 + ri[1] * (double)z1 + ri[2] * (double)z2;
            rr += ri[0] * ri[0] + ri[1] * ri[1] + ri[2] * ri[2];
        }
    }
    if(!sc)
        return;
    double v[2] = {rz, rr}, tot[2];
    if(!grid_sum<2>(v, partials, counter, tot))
        return;
    // scalar update of the iteration (one thread)
    const double rz_new = tot[0];
    sc->rz_new          = rz_new;
    sc->rr              = tot[1];
    sc->iter += 1;
    const bool hit = (sc->stop_rule == B2S_STOP_RZ) ? (fabs(rz_new) <= sc->rz_tol) : (tot[1] <= sc->rr_tol);
    if(!isfinite(rz_new))
        sc->converged = 3;
    else if(hit)
    {
        sc->converged = 1;
        sc->iter_conv = sc->iter;
    }
    else if(sc->iter >= sc->max_iter - 1)
        sc->converged = 2;
    else
    {
        sc->beta = rz_new / sc->rz;
        sc->rz   = rz_new;
    }
}

__global__ void k_update_xr(int64_t n, PcgScalars* sc, double* __restrict__ x, const double* __restrict__ p,
                            double* __restrict__ r, double* __restrict__ Ap)
{
    if(frozen(sc))
        return;
    const double alpha = sc->rz / sc->pAp;
    if(blockIdx.x == 0 && threadIdx.x == 0)
        sc->alpha = alpha;
    for(int64_t i = (int64_t)blockIdx.x * VEC_BLOCK + threadIdx.x; i < n; i += (int64_t)gridDim.x * VEC_BLOCK)
    {
        const double api = Ap[i];
        x[i] += alpha * p[i];
        r[i] -= alpha * api;
        Ap[i] = 0.0;
    }
}

__global__ void k_update_p(int64_t n, const PcgScalars* sc, const double* __restrict__ z, double* __restrict__ p)
{
    if(frozen(sc))
        return;
    const double beta = sc->beta;
    for(int64_t i = (int64_t)blockIdx.x * VEC_BLOCK + threadIdx.x; i < n; i += (int64_t)gridDim.x * VEC_BLOCK)
        p[i] = z[i] + beta * p[i];
}

// ---- mixed precision (FP32 vectors, FP64 solution and scalars) ----------------
// The FP32 vectors (r, z, p, Ap) hold 4 floats per node, the 4th zero
// (16-byte gathers and vector reductions in the SpMV and the MAS apply); the
// FP64 solution x holds 3. x += alpha p, r -= alpha Ap, Ap = 0, one node per
// thread and step.
__global__ void k_update_xr_mixed4(int32_t nb, PcgScalars* sc, double* __restrict__ x, const float* __restrict__ p,
                                   float* __restrict__ r, const float* __restrict__ Ap)
{
    if(frozen(sc))
        return;
    const double alpha = sc->rz / sc->pAp;
    if(blockIdx.x == 0 && threadIdx.x == 0)
        sc->alpha = alpha;
    const float af = (float)alpha;
    for(int64_t i = (int64_t)blockIdx.x * VEC_BLOCK + threadIdx.x; i < nb; i += (int64_t)gridDim.x * VEC_BLOCK)
    {
        const float4 ap = reinterpret_cast<const float4*>(Ap)[i];
        const float4 pp = reinterpret_cast<const float4*>(p)[i];
        float4       rr = reinterpret_cast<float4*>(r)[i];
        x[3 * i] += alpha * (double)pp.x;
        x[3 * i + 1] += alpha * (double)pp.y;
        x[3 * i + 2] += alpha * (double)pp.z;
        rr.x = __fmaf_rn(-af, ap.x, rr.x);
        rr.y = __fmaf_rn(-af, ap.y, rr.y);
        rr.z = __fmaf_rn(-af, ap.z, rr.z);
        reinterpret_cast<float4*>(r)[i] = rr;
    }
}

// p = z + beta p over the padded vectors (n = 4 nb; pads stay zero)
// p = z + beta p over the padded vectors (nb nodes), and Ap = 0 for the
// SpMV that follows: zeroed here rather than after its last reader, so the
// zero lines are still in L2 when the SpMV's reductions reach them
__global__ void k_update_p_mixed4(int32_t nb, const PcgScalars* sc, const float* __restrict__ z, float* __restrict__ p,
                                  float* __restrict__ Ap)
{
    if(frozen(sc))
        return;
    const float beta = (float)sc->beta;
    for(int64_t i = (int64_t)blockIdx.x * VEC_BLOCK + threadIdx.x; i < nb; i += (int64_t)gridDim.x * VEC_BLOCK)
    {
        const float4 zz = reinterpret_cast<const float4*>(z)[i];
        float4       pp = reinterpret_cast<float4*>(p)[i];
        pp.x = __fmaf_rn(beta, pp.x, zz.x);
        pp.y = __fmaf_rn(beta, pp.y, zz.y);
        pp.z = __fmaf_rn(beta, pp.z, zz.z);
        pp.w = __fmaf_rn(beta, pp.w, zz.w);
        reinterpret_cast<float4*>(p)[i]  = pp;
        reinterpret_cast<float4*>(Ap)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

// r32 = b - Ax computed in FP64, stored FP32 (padded: 4 floats per node)
__global__ void k_residual_f32(int32_t nb, const double* __restrict__ b, const double* __restrict__ Ax,
                               float* __restrict__ r)
{
    for(int64_t i = (int64_t)blockIdx.x * VEC_BLOCK + threadIdx.x; i < nb; i += (int64_t)gridDim.x * VEC_BLOCK)
        reinterpret_cast<float4*>(r)[i] = make_float4((float)(b[3 * i] - Ax[3 * i]), (float)(b[3 * i + 1] - Ax[3 * i + 1]),
                                                      (float)(b[3 * i + 2] - Ax[3 * i + 2]), 0.0f);
}

// between the 3-per-node FP32 vectors of the ABI and the padded ones
__global__ void k_pad4(int32_t nb, const float* __restrict__ a, float* __restrict__ b)
{
    for(int64_t i = (int64_t)blockIdx.x * VEC_BLOCK + threadIdx.x; i < nb; i += (int64_t)gridDim.x * VEC_BLOCK)
        reinterpret_cast<float4*>(b)[i] = make_float4(a[3 * i], a[3 * i + 1], a[3 * i + 2], 0.0f);
}
__global__ void k_unpad4(int32_t nb, const float* __restrict__ a, float* __restrict__ b)
{
    for(int64_t i = (int64_t)blockIdx.x * VEC_BLOCK + threadIdx.x; i < nb; i += (int64_t)gridDim.x * VEC_BLOCK)
    {
        const float4 q = reinterpret_cast<const float4*>(a)[i];
        b[3 * i]       = q.x;
        b[3 * i + 1]   = q.y;
        b[3 * i + 2]   = q.z;
    }
}

// FP32 vectors, FP64 sums: out[0] = a.b, out[1] = a.a
__global__ void __launch_bounds__(RED_BLOCK) k_dot2_f32(int64_t n, const float* __restrict__ a,
                                                        const float* __restrict__ b, double* partials,
                                                        unsigned int* counter, double* out)
{
    double ab = 0.0, aa = 0.0;
    for(int64_t i = (int64_t)blockIdx.x * RED_BLOCK + threadIdx.x; i < n; i += (int64_t)gridDim.x * RED_BLOCK)
    {
        const double ai = a[i];
        ab += ai * (double)b[i];
        aa += ai * ai;
    }
    double v[2] = {ab, aa}, tot[2];
    if(grid_sum<2>(v, partials, counter, tot))
    {
        out[0] = tot[0];
        out[1] = tot[1];
    }
}

// FP32 copy of the value planes (mixed-precision SpMV)
__global__ void k_planes_f32(int64_t count, const double* __restrict__ src, float* __restrict__ dst)
{
    for(int64_t i = (int64_t)blockIdx.x * VEC_BLOCK + threadIdx.x; i < count; i += (int64_t)gridDim.x * VEC_BLOCK)
        dst[i] = (float)src[i];
}

__global__ void k_residual(int64_t n, const double* __restrict__ b, const double* __restrict__ Ax,
                           double* __restrict__ r)
{
    for(int64_t i = (int64_t)blockIdx.x * VEC_BLOCK + threadIdx.x; i < n; i += (int64_t)gridDim.x * VEC_BLOCK)
        r[i] = b[i] - Ax[i];
}

// sum (b - Ax)^2 and b.b
__global__ void __launch_bounds__(RED_BLOCK) k_res_norms(int64_t n, const double* __restrict__ b,
                                                         const double* __restrict__ Ax, double* partials,
                                                         unsigned int* counter, double* out)
{
    double rr = 0.0, bb = 0.0;
    for(int64_t i = (int64_t)blockIdx.x * RED_BLOCK + threadIdx.x; i < n; i += (int64_t)gridDim.x * RED_BLOCK)
    {
        const double d = b[i] - Ax[i];
        rr += d * d;
        bb += b[i] * b[i];
    }
    double v[2] = {rr, bb}, tot[2];
    if(grid_sum<2>(v, partials, counter, tot))
    {
        out[0] = tot[0];
        out[1] = tot[1];
    }
}

}  // namespace

// ---------------------------------------------------------------------------
void precond_assemble(b2s_solver* s, int kind, int invert_mode)
{
    B2S_REQUIRE(s->A.valid, B2S_ERR_STATE, "precond_assemble before b2s_assemble");
    B2S_REQUIRE(kind >= B2S_PRECOND_NONE && kind <= B2S_PRECOND_MAS, B2S_ERR_ARGUMENT, "unknown preconditioner");
    B2S_REQUIRE(invert_mode == B2S_INVERT_F32 || invert_mode == B2S_INVERT_F64 || invert_mode == B2S_INVERT_F32_ONLY,
                B2S_ERR_ARGUMENT,
                "unknown inversion mode");
    cudaStream_t st = s->stream;
    const Matrix& A = s->A;
    s->dinv.resize((size_t)std::max(A.nb, 1) * 9);
    if(A.nb > 0)
    {
        k_diag_inverse<<<grid_for(A.nb, 256), 256, 0, st>>>(A.nb, A.diag_index.data(), A.vals.data(), A.stride,
                                                            s->dinv.data());
        B2S_CHECK_LAUNCH();
    }
    if(kind == B2S_PRECOND_MAS)
    {
        B2S_REQUIRE(s->mas.initialized, B2S_ERR_STATE, "MAS preconditioner requested before b2s_mas_init");
        mas_assemble(s, invert_mode);
    }
    if(s->abd_n > 0)
    {
        B2S_REQUIRE(s->abd_offset + 4 * (int64_t)s->abd_n <= A.nb, B2S_ERR_ARGUMENT,
                    "affine-body range exceeds the matrix");
        s->abd_inv.resize((size_t)s->abd_n * 144);
        k_abd_inverse<<<grid_for(s->abd_n, 128), 128, 0, st>>>(s->abd_n, s->abd_offset, A.rowptr.data(),
                                                               A.cols.data(), A.vals.data(), A.stride,
                                                               s->abd_inv.data());
        B2S_CHECK_LAUNCH();
    }
    s->precond_kind = kind;
    s->precond_generation += 1;
    s->invert_mode  = invert_mode;
    B2S_CUDA(cudaStreamSynchronize(st));
}

static MasView mas_view(b2s_solver* s)
{
    MasView mv{};
    const MasState& M = s->mas;
    mv.active = (s->precond_kind == B2S_PRECOND_MAS && M.initialized) ? 1 : 0;
    mv.abd_n   = s->abd_n;
    mv.abd_off = s->abd_offset;
    mv.abd_inv = s->abd_inv.data();
    mv.off    = M.offset;
    mv.vn     = M.vn;
    mv.L      = M.L;
    mv.r2p    = M.r2p.data();
    mv.node1  = M.node1.data();
    mv.T      = M.L <= 1 ? 0 : M.L - 1;
    mv.Z      = M.Z.data();
    return mv;
}

// z = P r, optionally fused with the dots + scalar update of a PCG iteration
static void precond_launch(b2s_solver* s, int kind, const double* r, double* z, PcgScalars* sc, Reduction& red)
{
    cudaStream_t st = s->stream;
    const int32_t nb = s->A.nb;
    if(nb == 0)
        return;
    if(kind == B2S_PRECOND_MAS)
        mas_apply_levels(s, r, sc ? &sc->converged : nullptr);
    const int grid = reduction_grid();
    ensure_reduction(red, grid, 2);
    k_precond_finish<double, 3><<<grid, RED_BLOCK, 0, st>>>(nb, kind, mas_view(s), s->dinv.data(), r, z, sc,
                                                 red.partials.data(), red.counter.data());
    B2S_CHECK_LAUNCH();
}

void precond_apply(b2s_solver* s, const double* r, double* z)
{
    B2S_REQUIRE(s->precond_kind >= 0, B2S_ERR_STATE, "precond_apply before b2s_precond_assemble");
    precond_launch(s, s->precond_kind, r, z, nullptr, s->red);
    check_device_errors(s);
    B2S_CUDA(cudaStreamSynchronize(s->stream));
}

// z = P r queued on the solver's stream (no synchronisation, no error check)
void precond_launch(b2s_solver* s, const double* r, double* z)
{
    B2S_REQUIRE(s->precond_kind >= 0, B2S_ERR_STATE, "precond_apply before b2s_precond_assemble");
    precond_launch(s, s->precond_kind, r, z, nullptr, s->red);
}

// ---------------------------------------------------------------------------
// PCG
// ---------------------------------------------------------------------------
namespace
{
struct GraphKey
{
    const void* ptrs[10];
    int64_t     ints[6];
    bool operator==(const GraphKey& o) const { return std::memcmp(this, &o, sizeof(GraphKey)) == 0; }
};
}  // namespace

// a stage-timing event: an external event node when the stream is being
// captured into the PCG graph, a plain stream event otherwise
static cudaError_t record_timing_event(cudaEvent_t ev, cudaStream_t st)
{
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t             e  = cudaStreamIsCapturing(st, &cs);
    if(e != cudaSuccess)
        return e;
    return cs == cudaStreamCaptureStatusActive ? cudaEventRecordWithFlags(ev, st, cudaEventRecordExternal)
                                               : cudaEventRecord(ev, st);
}

// one PCG iteration; with timing on, `slot` selects the 4 events that
// bracket its SpMV and its preconditioner apply
static void pcg_iteration(b2s_solver* s, int kind, double* x, int slot)
{
    PcgState&     P  = s->pcg;
    const Matrix& A  = s->A;
    cudaStream_t  st = s->stream;
    const int64_t n  = 3 * (int64_t)A.nb;
    cudaEvent_t*  ev = s->timing ? &s->iter_events[(size_t)slot * 4] : nullptr;
    if(ev)
        B2S_CUDA(record_timing_event(ev[0], st));
    spmv_f64_launch(s, A, P.p.data(), P.Ap.data(), P.red, &P.sc.data()->pAp, &P.sc.data()->converged);
    if(ev)
        B2S_CUDA(record_timing_event(ev[1], st));
    k_update_xr<<<vec_grid(n), VEC_BLOCK, 0, st>>>(n, P.sc.data(), x, P.p.data(), P.r.data(), P.Ap.data());
    B2S_CHECK_LAUNCH();
    if(ev)
        B2S_CUDA(record_timing_event(ev[2], st));
    precond_launch(s, kind, P.r.data(), P.z.data(), P.sc.data(), P.red);
    if(ev)
        B2S_CUDA(record_timing_event(ev[3], st));
    k_update_p<<<vec_grid(n), VEC_BLOCK, 0, st>>>(n, P.sc.data(), P.z.data(), P.p.data());
    B2S_CHECK_LAUNCH();
}

static void ensure_iter_events(b2s_solver* s, int ci)
{
    while((int)s->iter_events.size() < 4 * ci)
    {
        cudaEvent_t e;
        B2S_CUDA(cudaEventCreate(&e));
        s->iter_events.push_back(e);
    }
}

void pcg_solve(b2s_solver* s, const double* b, double* x, const b2s_pcg_options& o, b2s_pcg_stats& st_out)
{
    B2S_REQUIRE(s->A.valid, B2S_ERR_STATE, "b2s_pcg before b2s_assemble");
    B2S_REQUIRE(s->precond_kind >= 0, B2S_ERR_STATE, "b2s_pcg before b2s_precond_assemble");
    B2S_REQUIRE(o.precision == B2S_PRECISION_FP64 || o.precision == B2S_PRECISION_MIXED, B2S_ERR_ARGUMENT,
                "unknown precision");
    if(o.precision == B2S_PRECISION_MIXED)
    {
        pcg_solve_mixed(s, b, x, o, st_out);
        return;
    }
    B2S_REQUIRE(o.tol > 0.0 && std::isfinite(o.tol), B2S_ERR_ARGUMENT, "tolerance must be positive");
    B2S_REQUIRE(o.stop_rule == B2S_STOP_RZ || o.stop_rule == B2S_STOP_RELRES, B2S_ERR_ARGUMENT, "unknown stop rule");
    cudaStream_t  st = s->stream;
    const Matrix& A  = s->A;
    PcgState&     P  = s->pcg;
    const int64_t n  = 3 * (int64_t)A.nb;
    std::memset(&st_out, 0, sizeof(st_out));
    if(n == 0)
    {
        st_out.converged = 1;
        return;
    }
    P.r.resize(n, 1.1);
    P.z.resize(n, 1.1);
    P.p.resize(n, 1.1);
    P.Ap.resize(n, 1.1);
    P.tmp.resize(n, 1.1);
    P.sc.resize(1);
    if(!P.h_sc)
        B2S_CUDA(cudaMallocHost(&P.h_sc, sizeof(PcgScalars)));
    ensure_reduction(P.red, std::max(spmv_grid(A.nnz), reduction_grid()), 2);
    device_error_flag(s);  // allocated before any graph capture
    B2S_REQUIRE(A.nnz == 0 || A.has_trank, B2S_ERR_STATE, "matrix lacks the SpMV tile ranks");
    s->dot_out.resize(4);
    const int ci = o.check_interval > 0 ? o.check_interval : 1;
    const int64_t max_iter = o.max_iter > 0 ? o.max_iter : std::max<int64_t>(2 * n, 1);

    // r = b - A x0
    if(o.x0_given)
    {
        spmv_f64(s, A, x, P.tmp.data(), nullptr);
        k_residual<<<vec_grid(n), VEC_BLOCK, 0, st>>>(n, b, P.tmp.data(), P.r.data());
        B2S_CHECK_LAUNCH();
    }
    else
    {
        B2S_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, st));
        B2S_CUDA(cudaMemcpyAsync(P.r.data(), b, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    }
    int kind = s->precond_kind;
    precond_launch(s, kind, P.r.data(), P.z.data(), nullptr, s->red);
    launch_dot(s, P.r.data(), P.z.data(), n, s->dot_out.data());
    launch_dot(s, P.r.data(), P.r.data(), n, s->dot_out.data() + 1);
    launch_dot(s, b, b, n, s->dot_out.data() + 2);
    double h3[3];
    B2S_CUDA(cudaMemcpyAsync(h3, s->dot_out.data(), sizeof(h3), cudaMemcpyDeviceToHost, st));
    B2S_CUDA(cudaStreamSynchronize(st));
    double rz0 = h3[0];
    const double rr0 = h3[1], bb = h3[2];
    B2S_REQUIRE(std::isfinite(rr0) && std::isfinite(bb), B2S_ERR_NUMERIC,
                "non-finite right-hand side or initial residual");
    bool bypass = false;
    if(kind != B2S_PRECOND_NONE && (rz0 < 0.0 || !std::isfinite(rz0)))
    {
        // PSD guard: the preconditioner's action is not SPD/finite -> plain CG
        bypass = true;
        kind   = B2S_PRECOND_NONE;
        B2S_CUDA(cudaMemcpyAsync(P.z.data(), P.r.data(), sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        rz0 = rr0;
    }
    st_out.rz0      = rz0;
    st_out.bypassed = bypass ? 1 : 0;
    const double bnorm = std::sqrt(bb);

    auto true_residual = [&]() -> double
    {
        spmv_f64(s, A, x, P.tmp.data(), nullptr);
        k_res_norms<<<reduction_grid(), RED_BLOCK, 0, st>>>(n, b, P.tmp.data(), s->red.partials.data(),
                                                            s->red.counter.data(), s->dot_out.data());
        B2S_CHECK_LAUNCH();
        double h2[2];
        B2S_CUDA(cudaMemcpyAsync(h2, s->dot_out.data(), sizeof(h2), cudaMemcpyDeviceToHost, st));
        B2S_CUDA(cudaStreamSynchronize(st));
        return h2[1] > 0 ? std::sqrt(h2[0] / h2[1]) : 0.0;
    };

    if(rz0 == 0.0 || bb == 0.0)
    {
        st_out.converged = 1;
        st_out.rel_res   = true_residual();
        return;
    }
    ensure_reduction(s->red, reduction_grid(), 2);

    // device scalars
    PcgScalars h{};
    h.rz        = rz0;
    h.rz_tol    = o.tol * std::fabs(rz0);
    h.rr_tol    = (o.tol * bnorm) * (o.tol * bnorm);
    h.stop_rule = o.stop_rule;
    h.max_iter  = max_iter;
    int64_t iter_total = 0, replacements = 0;
    bool    done = false;
    while(!done)
    {
        h.converged = 0;
        h.iter      = iter_total;
        h.iter_conv = 0;
        B2S_CUDA(cudaMemcpyAsync(P.sc.data(), &h, sizeof(h), cudaMemcpyHostToDevice, st));
        B2S_CUDA(cudaMemcpyAsync(P.p.data(), P.z.data(), sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        B2S_CUDA(cudaMemsetAsync(P.Ap.data(), 0, sizeof(double) * n, st));

        // CUDA graph of `ci` iterations (re-captured when anything it bakes in changes)
        bool use_graph = o.use_graph && st != nullptr;
        if(s->timing)
            ensure_iter_events(s, ci);
        if(use_graph)
        {
            GraphKey key{};
            key.ptrs[0] = x;
            key.ptrs[1] = A.vals.data();
            key.ptrs[2] = A.rows.data();
            key.ptrs[3] = P.r.data();
            key.ptrs[4] = s->mas.inv.data();
            key.ptrs[5] = s->dinv.data();
            key.ptrs[6] = P.red.partials.data();
            key.ptrs[7] = s->mas.Z.data();
            key.ptrs[8] = A.cols.data();
            key.ptrs[9] = b;
            key.ints[0] = A.nnz;
            key.ints[1] = A.nb;
            key.ints[2] = kind;
            key.ints[3] = ci;
            key.ints[4] = s->mas.initialized ? s->mas.total : -1;
            key.ints[5] = s->mas.L + (s->timing ? 1000 : 0);
            size_t hk = 1469598103934665603ull;
            const unsigned char* kb = reinterpret_cast<const unsigned char*>(&key);
            for(size_t q = 0; q < sizeof(key); ++q)
                hk = (hk ^ kb[q]) * 1099511628211ull;
            if(!P.graph || P.graph_key != hk)
            {
                if(P.graph)
                {
                    cudaGraphExecDestroy(P.graph);
                    P.graph = nullptr;
                }
                cudaGraph_t g = nullptr;
                const long long before = g_kernel_launches;
                B2S_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
                for(int it = 0; it < ci; ++it)
                    pcg_iteration(s, kind, x, it);
                B2S_CUDA(cudaStreamEndCapture(st, &g));
                P.graph_kernels = g_kernel_launches - before;
                g_kernel_launches = before;
                cudaError_t e = cudaGraphInstantiate(&P.graph, g, 0);
                cudaGraphDestroy(g);
                if(e != cudaSuccess)
                {
                    P.graph   = nullptr;
                    use_graph = false;
                    cudaGetLastError();
                }
                else
                    P.graph_key = hk;
            }
        }
        long long iter_before = h.iter;
        while(true)
        {
            if(use_graph)
            {
                B2S_CUDA(cudaGraphLaunch(P.graph, st));
                g_kernel_launches += P.graph_kernels;
            }
            else
                for(int it = 0; it < ci; ++it)
                    pcg_iteration(s, kind, x, it);
            B2S_CUDA(cudaMemcpyAsync(P.h_sc, P.sc.data(), sizeof(PcgScalars), cudaMemcpyDeviceToHost, st));
            B2S_CUDA(cudaStreamSynchronize(st));
            if(s->timing)
            {
                // the iterations of this block that did work (the rest were frozen)
                const long long live = std::min<long long>(P.h_sc->iter - iter_before, ci);
                for(long long it = 0; it < live; ++it)
                {
                    float a = 0.f, c = 0.f;
                    B2S_CUDA(cudaEventElapsedTime(&a, s->iter_events[it * 4 + 0], s->iter_events[it * 4 + 1]));
                    B2S_CUDA(cudaEventElapsedTime(&c, s->iter_events[it * 4 + 2], s->iter_events[it * 4 + 3]));
                    s->timers.spmv_ms += a;
                    s->timers.spmv_launches += 1;
                    s->timers.precond_apply_ms += c;
                    s->timers.precond_apply_launches += 1;
                }
            }
            iter_before = P.h_sc->iter;
            if(P.h_sc->converged != 0)
                break;
        }
        const PcgScalars r = *P.h_sc;
        iter_total         = r.iter;
        if(r.converged == 3)
            throw Error(B2S_ERR_NUMERIC, "PCG breakdown: r.z became non-finite at iteration " + std::to_string(r.iter));
        st_out.iterations_exact = r.converged == 1 ? r.iter_conv : r.iter;
        st_out.converged        = r.converged == 1 ? 1 : 0;
        st_out.rel_res          = true_residual();
        done = true;
        if(r.converged == 1 && o.stop_rule == B2S_STOP_RELRES && st_out.rel_res > o.tol && replacements < 8
           && iter_total < max_iter - 1)
        {
            // the recursive residual drifted from b - A x: replace it and continue
            ++replacements;
            spmv_f64(s, A, x, P.tmp.data(), nullptr);
            k_residual<<<vec_grid(n), VEC_BLOCK, 0, st>>>(n, b, P.tmp.data(), P.r.data());
            B2S_CHECK_LAUNCH();
            precond_launch(s, kind, P.r.data(), P.z.data(), nullptr, s->red);
            launch_dot(s, P.r.data(), P.z.data(), n, s->dot_out.data());
            double rz;
            B2S_CUDA(cudaMemcpyAsync(&rz, s->dot_out.data(), sizeof(double), cudaMemcpyDeviceToHost, st));
            B2S_CUDA(cudaStreamSynchronize(st));
            h.rz = rz;
            done = false;
        }
    }
    st_out.replacements = replacements;
    check_device_errors(s);
    if(st_out.converged)
        st_out.iterations = ci > 1 ? std::min<int64_t>(((st_out.iterations_exact + ci - 1) / ci) * ci, max_iter)
                                   : st_out.iterations_exact;
    else
        st_out.iterations = max_iter;
}

// ---------------------------------------------------------------------------
// mixed precision PCG
// ---------------------------------------------------------------------------
void drop_graphs(b2s_solver* s)
{
    if(s->pcg.graph)
        cudaGraphExecDestroy(s->pcg.graph);
    if(s->pcg.graph_mixed)
        cudaGraphExecDestroy(s->pcg.graph_mixed);
    s->pcg.graph       = nullptr;
    s->pcg.graph_mixed = nullptr;
}

// storage of the MAS inverses in the mixed path: BF16 diagonal-scaled
// (default) or FP32, from B2S_MIXED_MAS_INVERSE=bf16|fp32, read once
static bool mixed_inverse_bf16()
{
    static const bool v = []
    {
        const char* e = std::getenv("B2S_MIXED_MAS_INVERSE");
        return !(e && std::string(e) == "fp32");
    }();
    return v;
}

// z = P r on FP32 vectors (MAS with BF16 inverses), optionally fused with the
// iteration's dots and scalar update
static void precond_launch_f32(b2s_solver* s, int kind, const float* r, float* z, PcgScalars* sc, Reduction& red)
{
    const int32_t nb = s->A.nb;
    if(nb == 0)
        return;
    if(kind == B2S_PRECOND_MAS)
        mas_apply_levels_f32(s, r, sc ? &sc->converged : nullptr, mixed_inverse_bf16());
    const int grid = reduction_grid();
    ensure_reduction(red, grid, 2);
    k_precond_finish<float, 4><<<grid, RED_BLOCK, 0, s->stream>>>(nb, kind, mas_view(s), s->dinv.data(), r, z, sc,
                                                               red.partials.data(), red.counter.data());
    B2S_CHECK_LAUNCH();
}

static void ensure_bf16_inverses(b2s_solver* s)
{
    if(s->precond_kind == B2S_PRECOND_MAS && s->mas.inv16_generation != s->precond_generation)
    {
        mas_pack_bf16(s);
        s->mas.inv16_generation = s->precond_generation;
    }
}

// the FP32 copy of the value planes the mixed PCG's SpMV reads (once per assembly)
static void ensure_f32_planes(b2s_solver* s)
{
    Matrix& A = s->A;
    if(A.vals32_generation == A.generation)
        return;
    A.vals32.resize((size_t)9 * A.stride, 1.2);
    k_planes_f32<<<vec_grid(9 * A.stride), VEC_BLOCK, 0, s->stream>>>(9 * A.stride, A.vals.data(), A.vals32.data());
    B2S_CHECK_LAUNCH();
    build_row_groups(s, A);
    A.vals32_generation = A.generation;
}

// y = A x as the mixed PCG computes it (FP32 planes and products, x.(A x) in
// FP64 into d_dot, device); x, y: 3 floats per node, padded around the product
void spmv_mixed(b2s_solver* s, const float* x, float* y, double* d_dot)
{
    Matrix&       A  = s->A;
    PcgState&     P  = s->pcg;
    const int32_t nb = A.nb;
    cudaStream_t  st = s->stream;
    ensure_f32_planes(s);
    ensure_reduction(P.red, std::max(spmv_grid(A.nnz), reduction_grid()), 2);
    P.p32.resize(4 * (size_t)nb, 1.1);
    P.Ap32.resize(4 * (size_t)nb, 1.1);
    k_pad4<<<vec_grid(nb), VEC_BLOCK, 0, st>>>(nb, x, P.p32.data());
    B2S_CHECK_LAUNCH();
    B2S_CUDA(cudaMemsetAsync(P.Ap32.data(), 0, sizeof(float) * 4 * (size_t)nb, st));
    B2S_CUDA(cudaMemsetAsync(d_dot, 0, sizeof(double), st));  // stays 0 for an empty matrix
    spmv_f32_launch(s, A, P.p32.data(), P.Ap32.data(), P.red, d_dot, nullptr);
    k_unpad4<<<vec_grid(nb), VEC_BLOCK, 0, st>>>(nb, P.Ap32.data(), y);
    B2S_CHECK_LAUNCH();
}

// the FP32 SpMV (with its fused dot) launched back to back on the solver's
// stream, events around the batch: the kernel's average launch duration on
// the assembled matrix (the padded vectors' values do not change its work)
double spmv_mixed_timing(b2s_solver* s, int launches)
{
    Matrix&       A  = s->A;
    PcgState&     P  = s->pcg;
    const int32_t nb = A.nb;
    cudaStream_t  st = s->stream;
    B2S_REQUIRE(launches > 0, B2S_ERR_ARGUMENT, "launch count must be positive");
    ensure_f32_planes(s);
    ensure_reduction(P.red, std::max(spmv_grid(A.nnz), reduction_grid()), 2);
    P.p32.resize(4 * (size_t)nb, 1.1);
    P.Ap32.resize(4 * (size_t)nb, 1.1);
    s->dot_out.resize(4);
    B2S_CUDA(cudaMemsetAsync(P.p32.data(), 0, sizeof(float) * 4 * (size_t)nb, st));
    B2S_CUDA(cudaMemsetAsync(P.Ap32.data(), 0, sizeof(float) * 4 * (size_t)nb, st));
    spmv_f32_launch(s, A, P.p32.data(), P.Ap32.data(), P.red, s->dot_out.data(), nullptr);  // warm-up
    cudaEvent_t e0, e1;
    B2S_CUDA(cudaEventCreate(&e0));
    B2S_CUDA(cudaEventCreate(&e1));
    B2S_CUDA(cudaEventRecord(e0, st));
    for(int i = 0; i < launches; ++i)
        spmv_f32_launch(s, A, P.p32.data(), P.Ap32.data(), P.red, s->dot_out.data(), nullptr);
    B2S_CUDA(cudaEventRecord(e1, st));
    B2S_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    B2S_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    B2S_CUDA(cudaEventDestroy(e0));
    B2S_CUDA(cudaEventDestroy(e1));
    return (double)ms / launches;
}

// r, z: 3 floats per node (the ABI's layout), padded around the apply
void precond_apply_mixed(b2s_solver* s, const float* r, float* z)
{
    B2S_REQUIRE(s->precond_kind >= 0, B2S_ERR_STATE, "precond_apply before b2s_precond_assemble");
    ensure_bf16_inverses(s);
    ensure_reduction(s->red, reduction_grid(), 2);
    const int32_t nb = s->A.nb;
    PcgState&     P  = s->pcg;
    P.r32.resize(4 * (size_t)nb, 1.1);
    P.z32.resize(4 * (size_t)nb, 1.1);
    k_pad4<<<vec_grid(nb), VEC_BLOCK, 0, s->stream>>>(nb, r, P.r32.data());
    B2S_CHECK_LAUNCH();
    precond_launch_f32(s, s->precond_kind, P.r32.data(), P.z32.data(), nullptr, s->red);
    k_unpad4<<<vec_grid(nb), VEC_BLOCK, 0, s->stream>>>(nb, P.z32.data(), z);
    B2S_CHECK_LAUNCH();
    check_device_errors(s);
}

static void pcg_iteration_mixed(b2s_solver* s, int kind, double* x, int slot)
{
    PcgState&     P  = s->pcg;
    const Matrix& A  = s->A;
    cudaStream_t  st = s->stream;
    const int32_t nb = A.nb;
    cudaEvent_t*  ev = s->timing ? &s->iter_events[(size_t)slot * 4] : nullptr;
    if(ev)
        B2S_CUDA(record_timing_event(ev[0], st));
    spmv_f32_launch(s, A, P.p32.data(), P.Ap32.data(), P.red, &P.sc.data()->pAp, &P.sc.data()->converged);
    if(ev)
        B2S_CUDA(record_timing_event(ev[1], st));
    k_update_xr_mixed4<<<vec_grid(nb), VEC_BLOCK, 0, st>>>(nb, P.sc.data(), x, P.p32.data(), P.r32.data(),
                                                           P.Ap32.data());
    B2S_CHECK_LAUNCH();
    if(ev)
        B2S_CUDA(record_timing_event(ev[2], st));
    precond_launch_f32(s, kind, P.r32.data(), P.z32.data(), P.sc.data(), P.red);
    if(ev)
        B2S_CUDA(record_timing_event(ev[3], st));
    k_update_p_mixed4<<<vec_grid(nb), VEC_BLOCK, 0, st>>>(nb, P.sc.data(), P.z32.data(), P.p32.data(),
                                                         P.Ap32.data());
    B2S_CHECK_LAUNCH();
}

// Mixed precision: the matrix in FP32 (planes converted once per assembly),
// r, z, p, Ap in FP32, the solution x and every scalar (alpha, beta, r.z,
// p.Ap, r.r) in FP64, MAS inverses as BF16 of the diagonal-scaled inverse
// with FP32 accumulation. Every `replace_every` iterations the recursive
// residual is replaced by b - A x computed in FP64 with the FP64 matrix
// (p, z and r.z are kept: a reliable update); the stop is always confirmed
// by the FP64 residual, and a stop the FP64 residual does not confirm
// continues from the true residual (with p = z).
void pcg_solve_mixed(b2s_solver* s, const double* b, double* x, const b2s_pcg_options& o, b2s_pcg_stats& st_out)
{
    cudaStream_t st = s->stream;
    Matrix&      A  = s->A;
    PcgState&    P  = s->pcg;
    const int64_t n = 3 * (int64_t)A.nb;
    std::memset(&st_out, 0, sizeof(st_out));
    if(n == 0)
    {
        st_out.converged = 1;
        return;
    }
    const int32_t nb = A.nb;
    const int64_t n4 = 4 * (int64_t)nb;  // padded FP32 vectors
    P.r32.resize(n4, 1.1);
    P.z32.resize(n4, 1.1);
    P.p32.resize(n4, 1.1);
    P.Ap32.resize(n4, 1.1);
    P.tmp.resize(n, 1.1);
    P.sc.resize(1);
    if(!P.h_sc)
        B2S_CUDA(cudaMallocHost(&P.h_sc, sizeof(PcgScalars)));
    ensure_reduction(P.red, std::max(spmv_grid(A.nnz), reduction_grid()), 2);
    ensure_reduction(s->red, reduction_grid(), 2);
    device_error_flag(s);
    s->dot_out.resize(4);
    B2S_REQUIRE(A.nnz == 0 || A.has_trank, B2S_ERR_STATE, "matrix lacks the SpMV tile ranks");
    const int     ci       = o.check_interval > 0 ? o.check_interval : 1;
    const int64_t max_iter = o.max_iter > 0 ? o.max_iter : std::max<int64_t>(2 * n, 1);
    int           kind     = s->precond_kind;

    // FP32 matrix planes, BF16 MAS inverses (once per assembly / build)
    ensure_f32_planes(s);
    ensure_bf16_inverses(s);

    // r = b - A x0 (FP64), stored FP32
    if(o.x0_given)
        spmv_f64(s, A, x, P.tmp.data(), nullptr);
    else
    {
        B2S_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, st));
        B2S_CUDA(cudaMemsetAsync(P.tmp.data(), 0, sizeof(double) * n, st));
    }
    k_residual_f32<<<vec_grid(nb), VEC_BLOCK, 0, st>>>(nb, b, P.tmp.data(), P.r32.data());
    B2S_CHECK_LAUNCH();

    auto restart_from_r = [&](int k) -> double
    {
        // z = P r, p = z; returns r.z (FP64 sum); also leaves r.r in dot_out[1]
        precond_launch_f32(s, k, P.r32.data(), P.z32.data(), nullptr, s->red);
        k_dot2_f32<<<reduction_grid(), RED_BLOCK, 0, st>>>(n4, P.r32.data(), P.z32.data(), s->red.partials.data(),
                                                            s->red.counter.data(), s->dot_out.data());
        B2S_CHECK_LAUNCH();
        B2S_CUDA(cudaMemcpyAsync(P.p32.data(), P.z32.data(), sizeof(float) * n4, cudaMemcpyDeviceToDevice, st));
        double h2[2];
        B2S_CUDA(cudaMemcpyAsync(h2, s->dot_out.data(), sizeof(h2), cudaMemcpyDeviceToHost, st));
        B2S_CUDA(cudaStreamSynchronize(st));
        return h2[0];
    };
    launch_dot(s, b, b, n, s->dot_out.data() + 2);
    double bb = 0.0;
    B2S_CUDA(cudaMemcpyAsync(&bb, s->dot_out.data() + 2, sizeof(double), cudaMemcpyDeviceToHost, st));
    double rz0 = restart_from_r(kind);
    B2S_REQUIRE(std::isfinite(bb), B2S_ERR_NUMERIC, "non-finite right-hand side");
    bool bypass = false;
    if(kind != B2S_PRECOND_NONE && (rz0 < 0.0 || !std::isfinite(rz0)))
    {
        bypass = true;  // PSD guard: plain CG
        kind   = B2S_PRECOND_NONE;
        rz0    = restart_from_r(kind);
    }
    st_out.rz0      = rz0;
    st_out.bypassed = bypass ? 1 : 0;
    const double bnorm = std::sqrt(bb);
    auto true_residual = [&]() -> double
    {
        spmv_f64(s, A, x, P.tmp.data(), nullptr);
        k_res_norms<<<reduction_grid(), RED_BLOCK, 0, st>>>(n, b, P.tmp.data(), s->red.partials.data(),
                                                            s->red.counter.data(), s->dot_out.data());
        B2S_CHECK_LAUNCH();
        double h2[2];
        B2S_CUDA(cudaMemcpyAsync(h2, s->dot_out.data(), sizeof(h2), cudaMemcpyDeviceToHost, st));
        B2S_CUDA(cudaStreamSynchronize(st));
        return h2[1] > 0 ? std::sqrt(h2[0] / h2[1]) : 0.0;
    };
    auto replace_residual = [&]()
    {
        spmv_f64(s, A, x, P.tmp.data(), nullptr);
        k_residual_f32<<<vec_grid(nb), VEC_BLOCK, 0, st>>>(nb, b, P.tmp.data(), P.r32.data());
        B2S_CHECK_LAUNCH();
    };
    if(rz0 == 0.0 || bb == 0.0)
    {
        st_out.converged = 1;
        st_out.rel_res   = true_residual();
        return;
    }

    PcgScalars h{};
    h.rz        = rz0;
    h.rz_tol    = o.tol * std::fabs(rz0);
    h.rr_tol    = (o.tol * bnorm) * (o.tol * bnorm);
    h.stop_rule = o.stop_rule;
    h.max_iter  = max_iter;
    int64_t iter_total = 0, replacements = 0, last_replace = 0;
    bool    done = false;
    while(!done)
    {
        h.converged = 0;
        h.iter      = iter_total;
        h.iter_conv = 0;
        B2S_CUDA(cudaMemcpyAsync(P.sc.data(), &h, sizeof(h), cudaMemcpyHostToDevice, st));
        B2S_CUDA(cudaMemsetAsync(P.Ap32.data(), 0, sizeof(float) * n4, st));
        bool use_graph = o.use_graph && st != nullptr;
        if(s->timing)
            ensure_iter_events(s, ci);
        if(use_graph)
        {
            const void*   ptrs[12] = {x,          A.vals32.data(), A.rows.data(),     P.r32.data(),
                                      s->mas.inv16.data(), s->dinv.data(), P.red.partials.data(), s->mas.Z.data(),
                                      A.cols.data(), P.p32.data(), P.Ap32.data(), P.z32.data()};
            const int64_t ints[6]  = {A.nnz, A.nb, kind, ci, s->mas.initialized ? s->mas.total : -1,
                                      s->mas.L + (s->timing ? 1000 : 0)};
            size_t hk = 1469598103934665603ull;
            for(const void* q : ptrs)
                hk = (hk ^ (size_t)q) * 1099511628211ull;
            for(int64_t q : ints)
                hk = (hk ^ (size_t)q) * 1099511628211ull;
            if(!P.graph_mixed || P.graph_mixed_key != hk)
            {
                if(P.graph_mixed)
                {
                    cudaGraphExecDestroy(P.graph_mixed);
                    P.graph_mixed = nullptr;
                }
                cudaGraph_t     g      = nullptr;
                const long long before = g_kernel_launches;
                B2S_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
                for(int it = 0; it < ci; ++it)
                    pcg_iteration_mixed(s, kind, x, it);
                B2S_CUDA(cudaStreamEndCapture(st, &g));
                P.graph_mixed_kernels = g_kernel_launches - before;
                g_kernel_launches     = before;
                cudaError_t e         = cudaGraphInstantiate(&P.graph_mixed, g, 0);
                cudaGraphDestroy(g);
                if(e != cudaSuccess)
                {
                    P.graph_mixed = nullptr;
                    use_graph     = false;
                    cudaGetLastError();
                }
                else
                    P.graph_mixed_key = hk;
            }
        }
        long long iter_before = h.iter;
        while(true)
        {
            if(use_graph)
            {
                B2S_CUDA(cudaGraphLaunch(P.graph_mixed, st));
                g_kernel_launches += P.graph_mixed_kernels;
            }
            else
                for(int it = 0; it < ci; ++it)
                    pcg_iteration_mixed(s, kind, x, it);
            B2S_CUDA(cudaMemcpyAsync(P.h_sc, P.sc.data(), sizeof(PcgScalars), cudaMemcpyDeviceToHost, st));
            B2S_CUDA(cudaStreamSynchronize(st));
            if(s->timing)
            {
                const long long live = std::min<long long>(P.h_sc->iter - iter_before, ci);
                for(long long it = 0; it < live; ++it)
                {
                    float a = 0.f, c = 0.f;
                    B2S_CUDA(cudaEventElapsedTime(&a, s->iter_events[it * 4 + 0], s->iter_events[it * 4 + 1]));
                    B2S_CUDA(cudaEventElapsedTime(&c, s->iter_events[it * 4 + 2], s->iter_events[it * 4 + 3]));
                    s->timers.spmv_ms += a;
                    s->timers.spmv_launches += 1;
                    s->timers.precond_apply_ms += c;
                    s->timers.precond_apply_launches += 1;
                }
            }
            iter_before = P.h_sc->iter;
            if(P.h_sc->converged != 0)
                break;
            if(o.replace_every > 0 && P.h_sc->iter - last_replace >= o.replace_every)
            {
                // reliable update: FP64 residual of the FP64 iterate, p and r.z kept
                replace_residual();
                ++replacements;
                last_replace = P.h_sc->iter;
            }
        }
        const PcgScalars r = *P.h_sc;
        iter_total         = r.iter;
        if(r.converged == 3)
            throw Error(B2S_ERR_NUMERIC, "mixed PCG breakdown: r.z non-finite at iteration " + std::to_string(r.iter));
        st_out.iterations_exact = r.converged == 1 ? r.iter_conv : r.iter;
        st_out.converged        = r.converged == 1 ? 1 : 0;
        st_out.rel_res          = true_residual();
        done                    = true;
        const bool verified = o.stop_rule != B2S_STOP_RELRES || st_out.rel_res <= o.tol;
        if(r.converged == 1 && !verified && replacements < 64 && iter_total < max_iter - 1)
        {
            // the FP32 recursion claimed a stop the FP64 residual does not
            // confirm: continue from the true residual
            replace_residual();
            ++replacements;
            last_replace = iter_total;
            h.rz         = restart_from_r(kind);
            done         = false;
        }
        else if(r.converged == 1 && !verified)
            st_out.converged = 0;
    }
    st_out.replacements = replacements;
    check_device_errors(s);
    if(st_out.converged)
        st_out.iterations = ci > 1 ? std::min<int64_t>(((st_out.iterations_exact + ci - 1) / ci) * ci, max_iter)
                                   : st_out.iterations_exact;
    else
        st_out.iterations = max_iter;
}
}  // namespace b2s
