// Exterior states of the wave system's boundary codes, shared by the collocation and the
// exact-quadrature kernels.  Code 0 is the absorbing state wavedg/WaveEquation.hpp:77-84
// intends (the reference evaluates p_e before u_e), 1 reflecting (:64-69), 2 Dirichlet p = 0.
#pragma once

namespace wdg
{
    // exterior state of a boundary node: 0 absorbing, 1 reflecting, 2 Dirichlet p = 0
    template <typename Real>
    __device__ __forceinline__ void exterior(int code, Real nx, Real ny, const Real q[3], Real x[3])
    {
        if (code == 1)
        {
            x[0] = q[0];
            x[1] = (ny * ny - nx * nx) * q[1] - Real(2) * nx * ny * q[2];
            x[2] = -Real(2) * nx * ny * q[1] + (nx * nx - ny * ny) * q[2];
        }
        else if (code == 0)
        {
            const Real out = q[0] + nx * q[1] + ny * q[2];
            const Real tan = ny * q[1] - nx * q[2];
            x[1] = ny * tan + Real(0.5) * nx * out;
            x[2] = -nx * tan + Real(0.5) * ny * out;
            x[0] = nx * x[1] + ny * x[2];
        }
        else
        {
            x[0] = -q[0];
            x[1] = q[1];
            x[2] = q[2];
        }
    }

} // namespace wdg
