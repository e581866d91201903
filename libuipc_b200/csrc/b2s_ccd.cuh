// The narrow phase of the line search's trajectory filter: per candidate
// pair (point-triangle or edge-edge, four vertex ids), the swept-box test
// expanded by dhat + thickness, then additive CCD (csrc/scene/elements.h:
// ccd_broadphase, accd_pair). Shared by the contact producer
// (b2s_generate_shell.cu) and the candidate detection (b2s_trajectory.cu).
#pragma once

#include <cstdint>

#include "scene/elements.h"

namespace b2s
{
// the trajectory filter's constants (simplex_trajectory_filter.cu:76, the
// ipc constitution's toi safety margin; lbvh_simplex_trajectory_filter.cu:18-21)
constexpr double CCD_ETA      = 0.1;
constexpr int    CCD_MAX_ITER = 1000;
constexpr double TOI_NONE     = 1.1;  // a pair without a hit within the step

namespace
{
// time of impact of every pair over the step alpha dx (TOI_NONE: none)
__global__ void k_contact_toi(int64_t np, const int32_t* __restrict__ pairs, const uint8_t* __restrict__ is_ee,
                              const double* __restrict__ x, const double* __restrict__ dx, double alpha, double dhat,
                              double xi, double eta, int max_iter, double* __restrict__ toi)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= np)
        return;
    const int32_t* V = pairs + 4 * p;
    double         X[12], dX[12];
    for(int i = 0; i < 4; ++i)
        for(int a = 0; a < 3; ++a)
        {
            X[3 * i + a]  = x[3 * (int64_t)V[i] + a];
            dX[3 * i + a] = alpha * dx[3 * (int64_t)V[i] + a];
        }
    double    t  = TOI_NONE;
    const int ee = is_ee[p];
    if(b2el::ccd_broadphase(X, dX, ee, dhat + xi))
    {
        double tt = TOI_NONE;
        if(b2el::accd_pair(X, dX, ee, eta, xi, max_iter, TOI_NONE, &tt))
            t = tt;
    }
    toi[p] = t;
}
}  // namespace
}  // namespace b2s
