// Flux models and face geometry of the conservation-law path, shared by the fused collocation
// kernels (claw_kernels.cuh) and the exact-quadrature Euler kernels (claw.cu).
//
//   ClawEuler    the compressible Euler system of examples/cl2d.cpp:67-126 (gamma 1.4) with its
//                local Lax-Friedrichs flux; exterior boundary state = interior state.
//   ClawLinear   f = A_0 u, g = A_1 u (Advection<true>), upwind flux
//                fh = 1/2 (n.A)(a + b) + 1/2 |n.A| (a - b), |n.A| per element side from a table
//                formed at set-up; exterior boundary state 0 (AdvectionHomogeneousBC<true>).
#pragma once

#include <cuda_runtime.h>

#include "launch.hpp"

namespace wdg
{
    struct ClawEuler
    {
        static constexpr double gamma = 1.4;
        __device__ static void flux(const ClawArgs &, const double *q, double *f, double *g)
        {
            const double rho = q[0], u = q[1] / q[0], v = q[2] / q[0], E = q[3];
            const double p = (gamma - 1.0) * (E - 0.5 * rho * (u * u + v * v));
            f[0] = rho * u;
            f[1] = rho * u * u + p;
            f[2] = rho * u * v;
            f[3] = u * (E + p);
            g[0] = rho * v;
            g[1] = rho * u * v;
            g[2] = rho * v * v + p;
            g[3] = v * (E + p);
        }
        __device__ static double speed(const double *q)
        {
            const double rho = q[0], u = q[1] / q[0], v = q[2] / q[0], E = q[3];
            const double p = (gamma - 1.0) * (E - 0.5 * rho * (u * u + v * v));
            return hypot(u, v) + sqrt(gamma * p / rho);
        }
        template <int NV>
        __device__ static void exterior(const double *q, double *x)
        {
#pragma unroll
            for (int d = 0; d < NV; ++d)
                x[d] = q[d];
        }
        template <int NV>
        __device__ static void numflux(const ClawArgs &a, int, int, double nx, double ny, const double *qL,
                                       const double *qR, double *fh)
        {
            double fL[4], gL[4], fR[4], gR[4];
            flux(a, qL, fL, gL);
            flux(a, qR, fR, gR);
            const double c = fmax(speed(qL), speed(qR));
#pragma unroll
            for (int d = 0; d < 4; ++d)
                fh[d] = 0.5 * nx * (fL[d] + fR[d]) + 0.5 * ny * (gL[d] + gR[d]) + 0.5 * c * (qL[d] - qR[d]);
        }
    };

    struct ClawLinear
    {
        template <int NV>
        __device__ static void flux_n(const ClawArgs &a, const double *q, double *f, double *g)
        {
#pragma unroll
            for (int d = 0; d < NV; ++d)
            {
                double s0 = 0.0, s1 = 0.0;
#pragma unroll
                for (int c = 0; c < NV; ++c)
                {
                    s0 += a.A[d + NV * c] * q[c];
                    s1 += a.A[d + NV * c + NV * NV] * q[c];
                }
                f[d] = s0;
                g[d] = s1;
            }
        }
        template <int NV>
        __device__ static void exterior(const double *, double *x)
        {
#pragma unroll
            for (int d = 0; d < NV; ++d)
                x[d] = 0.0;
        }
        template <int NV>
        __device__ static void numflux(const ClawArgs &a, int el, int side, double nx, double ny, const double *qL,
                                       const double *qR, double *fh)
        {
            const double *T = a.absA + (size_t)NV * NV * (4 * (size_t)el + side);
#pragma unroll
            for (int d = 0; d < NV; ++d)
            {
                double c = 0.0, u = 0.0;
#pragma unroll
                for (int k = 0; k < NV; ++k)
                {
                    const double nA = nx * a.A[d + NV * k] + ny * a.A[d + NV * k + NV * NV];
                    c += nA * (qL[k] + qR[k]);
                    u += T[d + NV * k] * (qL[k] - qR[k]);
                }
                fh[d] = 0.5 * c + 0.5 * u;
            }
        }
    };

    // outward unit normal and measure (length / 2) of side s of an element with corners c
    // (StraightEdge, wavedg/Edge.hpp:107-122); side s runs from corner p0 to p1: 0: 0 -> 1,
    // 1: 1 -> 2, 2: 3 -> 2, 3: 0 -> 3 (sides 2 and 3 against the counter-clockwise order)
    __device__ __forceinline__ void claw_side(const double *c, int s, double &nx, double &ny, double &meas)
    {
        const int p0 = (s == 0 || s == 3) ? 0 : (s == 1 ? 1 : 3), p1 = (s == 0) ? 1 : (s == 3 ? 3 : 2);
        const double dx = c[2 * p1] - c[2 * p0], dy = c[2 * p1 + 1] - c[2 * p0 + 1];
        const double len = sqrt(dx * dx + dy * dy), sgn = (s >= 2) ? -1.0 : 1.0;
        nx = sgn * dy / len;
        ny = -sgn * dx / len;
        meas = 0.5 * len;
    }
} // namespace wdg
