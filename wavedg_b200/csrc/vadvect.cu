// C-ABI: linear advection with a spatially varying coefficient, Advection<AQ> and
// AdvectionHomogeneousBC<AQ> with constant_coefficient = false (wavedg/Advection.hpp:59-273), on
// Gauss-Lobatto or Gauss-Legendre bases with either quadrature, MassMatrix<AQ>, as one fused
// kernel per operator application, RHS or time-stepping stage.
//
// The reference turns the coefficient and the geometry into operator tables once, at
// construction; this handle does the same on the host, with the same arithmetic:
//   volume  op(comp, c, d, p, el), the contravariant coefficient times the weights at volume
//           point p: the basis nodes with approx_quad = true (Div<true>, source/Div.cpp:6-54),
//           the Gauss-Legendre rule of Div<false> otherwise, the nodal coefficient interpolated
//           to it first (op_2d, source/Div.cpp:239-361);
//   faces   per element side and face point, in the element's own order, the two n_var x n_var
//           matrices that multiply the element's own and its neighbour's trace: w |E|/2 Fs with
//           Fs = R diag(-lambda/2 -+ |lambda|/2) R^T of n.A, A the face trace of each side's
//           coefficient (_ComputeFlux with a = -1, b = -1/2 and setup_flux_2d_c / _q,
//           source/EdgeFlux.cpp:31-88, 140-190, 430-494), + for the edge's first element and -
//           for its second (fb(side 1) = -fb(side 0)), the neighbour's matrix 0 on the boundary
//           (exterior state 0).
// The kernel (one warp per element, the element staged in shared memory) forms u at the volume
// points, the flux sum_c op(comp, c, d) u_c and its D / P contractions back to the nodes
// (div_2d_c and div_2d_q, source/Div.cpp:131-180, 469-589); per side the own trace and the
// neighbour's at the face points (Lobatto: nodal values, through the partner table of the
// collocation handle; Legendre: the interpolation of LegendreFaceProlongator along the lines of
// nodes normal to the side), the two matrices, back with P^T (flux_action_2d_c / _q,
// source/EdgeFlux.cpp:289-320, 553-624) and onto the nodes (the prolongator's transpose);
// then adds the result (the operators' action), or applies M^{-1} and writes the RHS or an
// RK4 / SSPRK3 stage.
// The flux matrices need a real eigen-decomposition of n.A: one variable, or symmetric
// coefficient matrices (cyclic Jacobi), are built.  FP64.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

#include "wave_impl.hpp"

using namespace wdg;

struct wdg_vadvect
{
    wdg_wave *w = nullptr;      // geometry, partner tables, argument staging
    int n = 0, nv = 0, Q = 0, Qf = 0;
    bool approx = true, legendre = false;
    double *d_Pv = nullptr, *d_Dv = nullptr, *d_Pf = nullptr;  // the rules' matrices (Q x n, Qf x n)
    double *d_xg = nullptr, *d_wg = nullptr, *d_e = nullptr;   // basis nodes, weights, phi(-1)
    double *d_op = nullptr, *d_G = nullptr;                    // volume and face tables
    double *d_Minv = nullptr;                                  // approx_quad = false: MassMatrix<false>^{-1}
    int *d_nb = nullptr; // Gauss-Legendre: per side (neighbour element * 4 + its side) * 2 + reversed, -1 boundary
    double *d_buf[3] = {nullptr, nullptr, nullptr};
};

namespace
{
    enum
    {
        VA_ACT = 16, // Advection::action: du += volume + interior faces
        VA_BC = 17,  // AdvectionHomogeneousBC::action: du += boundary faces
    };

    struct VArgs
    {
        ClawArgs c; // state, output, stage coefficients, geometry, partner table, error word
        const double *op, *G, *Pv, *Dv, *Pf, *xg, *wg, *e, *Minv;
        const int *nb;
        int n, nv, Q, Qf, approx, legendre;
    };

    __host__ __device__ inline int va_warp_doubles(int n, int nv, int Q, int Qf)
    {
        // su r (nv n^2 each) | Pu (nv n Q) | Uq (nv Q^2) | Fq (2 nv Q^2) | Df Pg (nv Q n each) | T0 T1 (4 n nv each)
        // | UF (4 Qf nv)
        return 2 * nv * n * n + nv * n * Q + 3 * nv * Q * Q + 2 * nv * Q * n + 8 * n * nv + 4 * Qf * nv;
    }

    __device__ inline int va_node(int n, int s, int k)
    {
        const int i = (s == 0 || s == 2) ? k : (s == 1 ? n - 1 : 0);
        const int j = (s == 1 || s == 3) ? k : (s == 2 ? n - 1 : 0);
        return i + n * j;
    }

    // LegendreFaceProlongator's node map (source/FaceProlongator.cpp:716-737): the node at
    // distance k from side s at position i along it
    __device__ inline int va_line(int n, int s, int i, int k)
    {
        const int x = (s == 0 || s == 2) ? i : (s == 1 ? n - 1 - k : k);
        const int y = (s == 1 || s == 3) ? i : (s == 2 ? n - 1 - k : k);
        return x + n * y;
    }

    __global__ void vadv_kernel(const VArgs A, int warps)
    {
        extern __shared__ double vsm[];
        const ClawArgs &a = A.c;
        const int n = A.n, nv = A.nv, Q = A.Q, Qf = A.Qf, nn = n * n, QQ = Q * Q, v2 = nv * nv;
        const bool ex = !A.approx;
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        double *su = vsm + (size_t)warp * va_warp_doubles(n, nv, Q, Qf);
        double *r = su + nv * nn, *Pu = r + nv * nn, *Uq = Pu + nv * n * Q, *Fq = Uq + nv * QQ;
        double *Df = Fq + 2 * nv * QQ, *Pg = Df + nv * Q * n, *T0 = Pg + nv * Q * n, *T1 = T0 + 4 * n * nv;
        double *UF = T1 + 4 * n * nv;
        const bool leg = A.legendre != 0;
        const long long limit = (long long)nn * a.nel;
        const bool vol = a.mode != VA_BC;
        for (int el = blockIdx.x * warps + warp; el < a.nel; el += gridDim.x * warps)
        {
            const double *xe = a.x + (size_t)nv * nn * el;
            for (int k = lane; k < nv * nn; k += 32)
            {
                su[k] = xe[k];
                r[k] = 0.0;
            }
            double c[8];
            for (int k = 0; k < 8; ++k)
                c[k] = __ldg(a.corners + 8 * (size_t)el + k);
            const uint32_t codes = __ldg(a.fcode + el);
            const int4 fb = __ldg(a.fbase + el);
            __syncwarp();
            if (vol)
            {
                const double *Uv = su;
                if (ex)
                {
                    // Pu(l, d, i) = sum_k P(i, k) u(d, k, l);  U(d, i, j) = sum_l P(j, l) Pu(l, d, i)
                    for (int o = lane; o < nv * n * Q; o += 32)
                    {
                        const int l = o % n, d = (o / n) % nv, i = o / (nv * n);
                        double t = 0.0;
                        for (int k = 0; k < n; ++k)
                            t += A.Pv[i + Q * k] * su[d + nv * (k + n * l)];
                        Pu[o] = t;
                    }
                    __syncwarp();
                    for (int o = lane; o < nv * QQ; o += 32)
                    {
                        const int d = o % nv, i = (o / nv) % Q, j = o / (nv * Q);
                        double t = 0.0;
                        for (int l = 0; l < n; ++l)
                            t += A.Pv[j + Q * l] * Pu[l + n * (d + nv * i)];
                        Uq[o] = t;
                    }
                    __syncwarp();
                    Uv = Uq;
                }
                // contravariant flux at the points: F(comp, d, p) = sum_c op(comp, c, d, p) U(c, p)
                for (int o = lane; o < nv * QQ; o += 32)
                {
                    const int d = o % nv, p = o / nv;
                    const double *T = A.op + ((size_t)el * QQ + p) * 2 * v2;
                    double f0 = 0.0, f1 = 0.0;
                    for (int cc = 0; cc < nv; ++cc)
                    {
                        const double u = Uv[cc + nv * p];
                        f0 += __ldg(T + cc + nv * d) * u;
                        f1 += __ldg(T + v2 + cc + nv * d) * u;
                    }
                    Fq[2 * o] = f0;
                    Fq[2 * o + 1] = f1;
                }
                __syncwarp();
                if (ex)
                {
                    // Df(j, d, k) = sum_i D(i, k) F0(d, i, j);  Pg(j, d, k) = sum_i P(i, k) F1(d, i, j)
                    for (int o = lane; o < nv * Q * n; o += 32)
                    {
                        const int j = o % Q, d = (o / Q) % nv, k = o / (nv * Q);
                        double df = 0.0, pg = 0.0;
                        for (int i = 0; i < Q; ++i)
                        {
                            const double *F = Fq + 2 * (d + nv * (i + Q * j));
                            df += A.Dv[i + Q * k] * F[0];
                            pg += A.Pv[i + Q * k] * F[1];
                        }
                        Df[o] = df;
                        Pg[o] = pg;
                    }
                    __syncwarp();
                    for (int o = lane; o < nv * nn; o += 32)
                    {
                        const int d = o % nv, k = (o / nv) % n, l = o / (nv * n);
                        double t = 0.0;
                        for (int j = 0; j < Q; ++j)
                            t += A.Pv[j + Q * l] * Df[j + Q * (d + nv * k)] + A.Dv[j + Q * l] * Pg[j + Q * (d + nv * k)];
                        r[o] = t;
                    }
                }
                else
                {
                    // (F, grad v)(i, j) = sum_l D(l, i) F0(d, l, j) + D(l, j) F1(d, i, l)
                    for (int o = lane; o < nv * nn; o += 32)
                    {
                        const int d = o % nv, i = (o / nv) % n, j = o / (nv * n);
                        double t = 0.0;
                        for (int l = 0; l < n; ++l)
                            t += A.Dv[l + n * i] * Fq[2 * (d + nv * (l + n * j))] +
                                 A.Dv[l + n * j] * Fq[2 * (d + nv * (i + n * l)) + 1];
                        r[o] = t;
                    }
                }
            }
            // the sides this call adds: interior (action), boundary (bc), or all
            auto wanted = [&](int s) -> bool
            {
                const bool bnd = ((codes >> (8 * s)) & 0x80u) != 0;
                return a.mode == VA_ACT ? !bnd : (a.mode == VA_BC ? bnd : true);
            };
            // the element's own traces T0(s, k, c) and its neighbours' T1(s, k, c) on the sides this
            // call adds (interior sides; 0 on the boundary): GLL nodal values through the partner
            // table, Gauss-Legendre sum_k phi_k(-1) u(line node k) (legendre_action_2d,
            // source/FaceProlongator.cpp:806-834)
            for (int o = lane; o < 4 * n; o += 32)
            {
                const int s = o / n, k = o - s * n;
                const uint32_t byte = (codes >> (8 * s)) & 0xffu;
                double *t0 = T0 + nv * o, *t1 = T1 + nv * o;
                for (int d = 0; d < nv; ++d)
                {
                    double v = 0.0;
                    if (leg)
                        for (int m = 0; m < n; ++m)
                            v += su[d + nv * va_line(n, s, k, m)] * A.e[m];
                    else
                        v = su[d + nv * va_node(n, s, k)];
                    t0[d] = v;
                    t1[d] = 0.0;
                }
                if ((byte & 0x80u) || !wanted(s))
                    continue;
                if (leg)
                {
                    const int code = __ldg(A.nb + 4 * (size_t)el + s);
                    const long long ne = code >> 3; // neighbour element
                    const int ns = (code >> 1) & 3, kk = (code & 1) ? n - 1 - k : k;
                    if (code < 0 || ne >= a.nel)
                    {
                        atomicOr(a.err, 2u);
                        continue;
                    }
                    const double *xn = a.x + (size_t)nv * nn * ne;
                    for (int d = 0; d < nv; ++d)
                    {
                        double v = 0.0;
                        for (int m = 0; m < n; ++m)
                            v += __ldg(xn + d + nv * va_line(n, ns, kk, m)) * A.e[m];
                        t1[d] = v;
                    }
                    continue;
                }
                const int off = (s == 0) ? fb.x : (s == 1) ? fb.y : (s == 2) ? fb.z : fb.w;
                const uint32_t sc = byte & 3u;
                const int stride = (sc == 0) ? 1 : (sc == 1) ? -1 : (sc == 2) ? n : -n; // in nodes
                const long long pn = (long long)(off / 3) + (long long)k * stride;
                if (off < 0 || pn < 0 || pn >= limit)
                    atomicOr(a.err, 2u);
                else
                    for (int d = 0; d < nv; ++d)
                        t1[d] = __ldg(a.x + (size_t)nv * pn + d);
            }
            __syncwarp();
            // face points: UF(s, q, d) = sum_c G_own(c, d) U_own(c) + G_nbr(c, d) U_nbr(c)
            for (int o = lane; o < 4 * Qf; o += 32)
            {
                const int s = o / Qf, q = o - s * Qf;
                double *uf = UF + nv * o;
                if (!wanted(s))
                {
                    for (int d = 0; d < nv; ++d)
                        uf[d] = 0.0;
                    continue;
                }
                double Uo[kJacobiMax], Un[kJacobiMax];
                for (int cc = 0; cc < nv; ++cc)
                {
                    if (ex)
                    {
                        double so = 0.0, sn = 0.0;
                        for (int j = 0; j < n; ++j)
                        {
                            const double p = A.Pf[q + Qf * j];
                            so += T0[cc + nv * (s * n + j)] * p;
                            sn += T1[cc + nv * (s * n + j)] * p;
                        }
                        Uo[cc] = so;
                        Un[cc] = sn;
                    }
                    else
                    {
                        Uo[cc] = T0[cc + nv * (s * n + q)];
                        Un[cc] = T1[cc + nv * (s * n + q)];
                    }
                }
                const double *G = A.G + (((size_t)el * 4 + s) * Qf + q) * 2 * v2;
                for (int d = 0; d < nv; ++d)
                {
                    double f = 0.0;
                    for (int cc = 0; cc < nv; ++cc)
                        f += __ldg(G + cc + nv * d) * Uo[cc] + __ldg(G + v2 + cc + nv * d) * Un[cc];
                    uf[d] = f;
                }
            }
            __syncwarp();
            // back to the face positions (P^T with approx_quad = false) into T0, then added to the
            // nodes: GLL at the face nodes, sides 0 and 2, then 1 and 3 (corners are shared by
            // neighbouring sides only); Gauss-Legendre along the lines, phi_k(-1) times the face
            // value, one side at a time (legendre_transpose_2d)
            for (int o = lane; o < 4 * n; o += 32)
            {
                const int s = o / n, k = o - s * n;
                for (int d = 0; d < nv; ++d)
                {
                    double f = 0.0;
                    if (wanted(s))
                    {
                        if (ex)
                            for (int q = 0; q < Qf; ++q)
                                f += UF[nv * (s * Qf + q) + d] * A.Pf[q + Qf * k];
                        else
                            f = UF[nv * (s * Qf + k) + d];
                    }
                    T0[nv * o + d] = f;
                }
            }
            __syncwarp();
            if (leg)
                for (int s = 0; s < 4; ++s)
                {
                    if (wanted(s))
                        for (int o = lane; o < nn; o += 32)
                        {
                            const int i = o % n, k = o / n, node = va_line(n, s, i, k);
                            for (int d = 0; d < nv; ++d)
                                r[nv * node + d] += T0[nv * (s * n + i) + d] * A.e[k];
                        }
                    __syncwarp();
                }
            else
                for (int pass = 0; pass < 2; ++pass)
                {
                    for (int o = lane; o < 2 * n; o += 32)
                    {
                        const int s = pass + 2 * (o / n), k = o % n;
                        if (!wanted(s))
                            continue;
                        const int node = va_node(n, s, k);
                        for (int d = 0; d < nv; ++d)
                            r[nv * node + d] += T0[nv * (s * n + k) + d];
                    }
                    __syncwarp();
                }
            if (a.mode == VA_ACT || a.mode == VA_BC)
            {
                for (int o = lane; o < nv * nn; o += 32)
                    a.out[(size_t)nv * nn * el + o] += r[o];
                __syncwarp();
                continue;
            }
            // M^{-1} and the output: lane per node
            for (int row = lane; row < nn; row += 32)
            {
                double y[kJacobiMax];
                if (ex)
                {
                    const double *Me = A.Minv + (size_t)nn * nn * el;
                    for (int d = 0; d < nv; ++d)
                        y[d] = 0.0;
                    for (int j = 0; j < nn; ++j)
                    {
                        const double m = __ldg(Me + row + (size_t)nn * j);
                        for (int d = 0; d < nv; ++d)
                            y[d] += m * r[nv * j + d];
                    }
                }
                else
                {
                    // MassMatrix<true>: w_i w_j det J at the basis node
                    const int i = row % n, j = row / n;
                    const double xi = A.xg[i], eta = A.xg[j];
                    const double Xx = 0.25 * ((1.0 - eta) * (c[2] - c[0]) + (1.0 + eta) * (c[4] - c[6]));
                    const double Yx = 0.25 * ((1.0 - eta) * (c[3] - c[1]) + (1.0 + eta) * (c[5] - c[7]));
                    const double Xe = 0.25 * ((1.0 - xi) * (c[6] - c[0]) + (1.0 + xi) * (c[4] - c[2]));
                    const double Ye = 0.25 * ((1.0 - xi) * (c[7] - c[1]) + (1.0 + xi) * (c[5] - c[3]));
                    const double m = A.wg[i] * A.wg[j] * (Xx * Ye - Yx * Xe);
                    for (int d = 0; d < nv; ++d)
                        y[d] = r[nv * row + d] / m;
                }
                const size_t g0 = (size_t)nv * (nn * (size_t)el + row);
                for (int d = 0; d < nv; ++d)
                {
                    const double qd = su[nv * row + d];
                    switch (a.mode)
                    {
                    case CLAW_RHS:
                        a.out[g0 + d] = y[d];
                        break;
                    case CLAW_RK4:
                    {
                        const double kd = (a.rk_a == 0.0) ? a.dt * y[d] : a.rk_a * a.du[g0 + d] + a.dt * y[d];
                        a.du[g0 + d] = kd;
                        a.out[g0 + d] = qd + a.rk_b * kd;
                        break;
                    }
                    case CLAW_SSP0:
                        a.out[g0 + d] = qd + a.dt * y[d];
                        break;
                    case CLAW_SSP1:
                        a.out[g0 + d] = 0.25 * (qd + 3.0 * a.base[g0 + d] + a.dt * y[d]);
                        break;
                    default:
                        a.out[g0 + d] = (a.base[g0 + d] + 2.0 * qd + 2.0 * a.dt * y[d]) / 3.0;
                        break;
                    }
                }
            }
            __syncwarp();
        }
    }

    // _ComputeFlux::flux with a = -1, b = -1/2 (source/EdgeFlux.cpp:31-88): Fs(c, d) for side
    // s of n.A; one variable in the closed form, else from the symmetric eigen-decomposition
    void side_flux(int nv, const double *nA, int s, double *Fs)
    {
        const double a = -1.0, b = -0.5, sgn = (s == 0) ? 1.0 : -1.0;
        if (nv == 1)
        {
            Fs[0] = 0.5 * a * nA[0] + sgn * b * std::abs(nA[0]);
            return;
        }
        double R[kJacobiMax * kJacobiMax], e[kJacobiMax];
        jacobi_eig(nv, nA, R, e);
        for (int cc = 0; cc < nv; ++cc)
            for (int d = 0; d < nv; ++d)
            {
                double acc = 0.0;
                for (int k = 0; k < nv; ++k)
                    acc += R[cc + nv * k] * (0.5 * a * e[k] + sgn * b * std::abs(e[k])) * R[d + nv * k];
                Fs[cc + nv * d] = acc;
            }
    }

    int node_of(int n, int s, int k)
    {
        const int i = (s == 0 || s == 2) ? k : (s == 1 ? n - 1 : 0);
        const int j = (s == 1 || s == 3) ? k : (s == 2 ? n - 1 : 0);
        return i + n * j;
    }

    // Div<true> (source/Div.cpp:6-54) or op_2d (source/Div.cpp:239-361) per element:
    // op(comp, c, d, p) from a(d, c, comp) at the volume points, times the weights
    void volume_table(const wdg_mesh &mesh, int n, int nv, int Q, bool approx, const double *a,
                      const std::vector<double> &xg, const std::vector<double> &wg, const std::vector<double> &xv,
                      const std::vector<double> &wv, const std::vector<double> &P, std::vector<double> &op)
    {
        const int v2 = nv * nv, nn = n * n, QQ = Q * Q;
        op.assign((size_t)2 * v2 * QQ * mesh.nel, 0.0);
        // a(d, c, comp, i, j, el) = a[d + nv (c + nv (comp + 2 (i + n (j + n el))))]
        auto A = [&](int d, int cc, int comp, int node, int el)
        { return a[d + nv * (cc + nv * (comp + 2 * (node + (size_t)nn * el)))]; };
        std::vector<double> PA((size_t)2 * v2 * n * Q);
        for (int el = 0; el < mesh.nel; ++el)
        {
            const double *cr = &mesh.corners[8 * (size_t)el];
            if (!approx)
            {
                // PA(comp, c, d, k, i) = sum_l P(i, l) a(d, c, comp, l, k)
                for (int k = 0; k < n; ++k)
                    for (int i = 0; i < Q; ++i)
                        for (int cc = 0; cc < nv; ++cc)
                            for (int d = 0; d < nv; ++d)
                            {
                                double a0 = 0.0, a1 = 0.0;
                                for (int l = 0; l < n; ++l)
                                {
                                    a0 += P[i + Q * l] * A(d, cc, 0, l + n * k, el);
                                    a1 += P[i + Q * l] * A(d, cc, 1, l + n * k, el);
                                }
                                PA[0 + 2 * (cc + nv * (d + nv * (k + n * (size_t)i)))] = a0;
                                PA[1 + 2 * (cc + nv * (d + nv * (k + n * (size_t)i)))] = a1;
                            }
            }
            for (int j = 0; j < Q; ++j)
                for (int i = 0; i < Q; ++i)
                {
                    double J[4];
                    const double xi = approx ? xg[i] : xv[i], eta = approx ? xg[j] : xv[j];
                    quad_jacobian(cr, xi, eta, J);
                    const double W = approx ? wg[j] * wg[i] : wv[i] * wv[j];
                    const double X_xi = J[0] * W, Y_xi = J[1] * W, X_eta = J[2] * W, Y_eta = J[3] * W;
                    double *T = &op[((size_t)el * QQ + i + Q * j) * 2 * v2];
                    for (int d = 0; d < nv; ++d)
                        for (int cc = 0; cc < nv; ++cc)
                        {
                            double a0, a1;
                            if (approx)
                            {
                                a0 = A(d, cc, 0, i + n * j, el);
                                a1 = A(d, cc, 1, i + n * j, el);
                            }
                            else
                            {
                                a0 = a1 = 0.0;
                                for (int k = 0; k < n; ++k)
                                {
                                    a0 += P[j + Q * k] * PA[0 + 2 * (cc + nv * (d + nv * (k + n * (size_t)i)))];
                                    a1 += P[j + Q * k] * PA[1 + 2 * (cc + nv * (d + nv * (k + n * (size_t)i)))];
                                }
                            }
                            T[cc + nv * d] = Y_eta * a0 - X_eta * a1;
                            T[v2 + cc + nv * d] = -Y_xi * a0 + X_xi * a1;
                        }
                }
        }
    }

    // the flux matrices of every element side in the element's own point order (setup_flux_2d_c,
    // source/EdgeFlux.cpp:140-190, or setup_flux_2d_q, :430-494, per edge in the edge's order,
    // the coefficient traces as LobattoFaceProlongator lays them out); G(t, c, d, q, s, el),
    // t = 0 the element's own trace, 1 its neighbour's
    int line_of(int n, int s, int i, int k)
    {
        const int x = (s == 0 || s == 2) ? i : (s == 1 ? n - 1 - k : k);
        const int y = (s == 1 || s == 3) ? i : (s == 2 ? n - 1 - k : k);
        return x + n * y;
    }

    int face_table(const wdg_mesh &mesh, int n, int nv, int Qf, bool approx, bool legendre, const double *a,
                   const std::vector<double> &e, const std::vector<double> &wg, const std::vector<double> &wf,
                   const std::vector<double> &Pf, std::vector<double> &G)
    {
        const int v2 = nv * nv, nn = n * n;
        G.assign((size_t)2 * v2 * Qf * 4 * mesh.nel, 0.0);
        auto A = [&](int flat, int comp, int node, int el)
        { return a[flat + v2 * (comp + 2 * (node + (size_t)nn * el))]; };
        // the coefficient's trace at position j of side s of element el (Lobatto: the face node;
        // Legendre: sum_k phi_k(-1) a(line node k), legendre_action_2d)
        auto trace = [&](int flat, int comp, int s, int j, int el)
        {
            if (!legendre)
                return A(flat, comp, node_of(n, s, j), el);
            double v = 0.0;
            for (int k = 0; k < n; ++k)
                v += A(flat, comp, line_of(n, s, j, k), el) * e[k];
            return v;
        };
        std::vector<double> F((size_t)2 * v2 * Qf), nA(v2), At((size_t)2 * v2 * n);
        for (int type = 0; type < 2; ++type)
        {
            const std::vector<EdgeRec> &list = type == 0 ? mesh.interior : mesh.boundary;
            for (const EdgeRec &E : list)
            {
                const double *cr = &mesh.corners[8 * (size_t)E.el0];
                const double dx = cr[2 * kSideTo[E.s0]] - cr[2 * kSideFrom[E.s0]];
                const double dy = cr[2 * kSideTo[E.s0] + 1] - cr[2 * kSideFrom[E.s0] + 1];
                const double len = std::sqrt(dx * dx + dy * dy), sg = (E.s0 >= 2) ? -1.0 : 1.0;
                const double nx = sg * dy / len, ny = -sg * dx / len, meas = 0.5 * len;
                for (int s = 0; s < 2; ++s)
                {
                    // side s's coefficient trace At(flat, comp, j) in the edge's node order
                    // (zero for the boundary's missing side)
                    for (int j = 0; j < n; ++j)
                        for (int comp = 0; comp < 2; ++comp)
                            for (int f = 0; f < v2; ++f)
                            {
                                double v = 0.0;
                                if (s == 0)
                                    v = trace(f, comp, E.s0, j, E.el0);
                                else if (type == 0)
                                    v = trace(f, comp, E.s1, E.delta < 0 ? n - 1 - j : j, E.el1);
                                At[f + v2 * (comp + 2 * (size_t)j)] = v;
                            }
                    for (int q = 0; q < Qf; ++q)
                    {
                        for (int f = 0; f < v2; ++f)
                        {
                            double a0, a1;
                            if (approx)
                            {
                                a0 = At[f + v2 * (0 + 2 * (size_t)q)];
                                a1 = At[f + v2 * (1 + 2 * (size_t)q)];
                            }
                            else
                            {
                                a0 = a1 = 0.0;
                                for (int j = 0; j < n; ++j)
                                {
                                    a0 += At[f + v2 * (0 + 2 * (size_t)j)] * Pf[q + Qf * j];
                                    a1 += At[f + v2 * (1 + 2 * (size_t)j)] * Pf[q + Qf * j];
                                }
                            }
                            nA[f] = nx * a0 + ny * a1;
                        }
                        if (nv > 1)
                        {
                            double amax = 0.0;
                            for (double v : nA)
                                amax = std::max(amax, std::abs(v));
                            for (int d = 0; d < nv; ++d)
                                for (int cc = 0; cc < d; ++cc)
                                    if (std::abs(nA[d + nv * cc] - nA[cc + nv * d]) > 1e-14 * amax)
                                        return fail(WDG_ERR_UNSUPPORTED,
                                                    "wdg_vadvect_create: n.A must be symmetric at every face point "
                                                    "(the flux uses a symmetric eigen-decomposition)");
                        }
                        double Fs[kJacobiMax * kJacobiMax];
                        side_flux(nv, nA.data(), s, Fs);
                        const double w = (approx ? wg[q] : wf[q]) * meas;
                        for (int f = 0; f < v2; ++f)
                            F[f + v2 * (s + 2 * (size_t)q)] = w * Fs[f];
                    }
                }
                // scatter: the first element in the edge's order with +, the second (if any) in its
                // own order with -, each with its own and its neighbour's matrix
                for (int q = 0; q < Qf; ++q)
                    for (int f = 0; f < v2; ++f)
                    {
                        double *g0 = &G[(((size_t)E.el0 * 4 + E.s0) * Qf + q) * 2 * v2];
                        g0[f] = F[f + v2 * (0 + 2 * (size_t)q)];
                        g0[v2 + f] = type == 0 ? F[f + v2 * (1 + 2 * (size_t)q)] : 0.0;
                        if (type == 0)
                        {
                            const int qe = E.delta < 0 ? Qf - 1 - q : q; // the edge's point at own point q
                            double *g1 = &G[(((size_t)E.el1 * 4 + E.s1) * Qf + q) * 2 * v2];
                            g1[f] = -F[f + v2 * (1 + 2 * (size_t)qe)];
                            g1[v2 + f] = -F[f + v2 * (0 + 2 * (size_t)qe)];
                        }
                    }
            }
        }
        return WDG_OK;
    }

    int upload(const std::vector<double> &v, double **d)
    {
        WDG_TRY(device_alloc(d, v.size()));
        return device_put(*d, v);
    }

    int check(const wdg_vadvect *h) { return h ? WDG_OK : fail(WDG_ERR_ARG, "null advection handle"); }
    long long nvals(const wdg_vadvect *h) { return (long long)h->nv * h->n * h->n * h->w->nel; }

    int va_warps(const wdg_vadvect *h)
    {
        const size_t per = sizeof(double) * (size_t)va_warp_doubles(h->n, h->nv, h->Q, h->Qf);
        return (int)std::max<size_t>(1, std::min<size_t>(4, (size_t)(200 * 1024) / per));
    }

    int va_launch(wdg_vadvect *h, const ClawArgs &c)
    {
        VArgs A{};
        A.c = c;
        A.op = h->d_op;
        A.G = h->d_G;
        A.Pv = h->d_Pv;
        A.Dv = h->d_Dv;
        A.Pf = h->d_Pf;
        A.xg = h->d_xg;
        A.wg = h->d_wg;
        A.e = h->d_e;
        A.nb = h->d_nb;
        A.Minv = h->d_Minv;
        A.n = h->n;
        A.nv = h->nv;
        A.Q = h->Q;
        A.Qf = h->Qf;
        A.approx = h->approx ? 1 : 0;
        A.legendre = h->legendre ? 1 : 0;
        const int warps = va_warps(h);
        const size_t smem = sizeof(double) * (size_t)va_warp_doubles(h->n, h->nv, h->Q, h->Qf) * warps;
        const unsigned blocks = (unsigned)std::max(1, std::min((c.nel + warps - 1) / warps, 148 * 16));
        vadv_kernel<<<blocks, 32 * warps, smem, h->w->stream>>>(A, warps);
        WDG_CUDA(cudaGetLastError());
        return WDG_OK;
    }

    int accumulate(wdg_vadvect *h, int mode, const double *u, double *du, const char *name)
    {
        WDG_TRY(check(h));
        if (!u || !du || u == du)
            return fail(WDG_ERR_ARG, (std::string(name) + ": distinct u and du arrays required").c_str());
        DeviceScope g(h->w->device);
        HostArg a[2];
        WDG_TRY(bind_arg(h->w, 0, u, (size_t)nvals(h), true, false, a[0]));
        WDG_TRY(bind_arg(h->w, 1, du, (size_t)nvals(h), true, true, a[1]));
        ClawArgs c = claw_args(h->w, a[0].dev, a[1].dev);
        c.mode = mode;
        WDG_TRY(va_launch(h, c));
        return finish_args(h->w, a, 2);
    }
} // namespace

extern "C"
{
    int wdg_vadvect_create(const wdg_mesh *mesh, int n_colloc, int basis_type, int n_var, const double *a,
                           int approx_quad, int device, wdg_vadvect **out)
    {
        if (!mesh || !a || !out)
            return fail(WDG_ERR_ARG, "wdg_vadvect_create: null argument");
        *out = nullptr;
        if (n_var < 1 || n_var > kJacobiMax)
            return fail(WDG_ERR_UNSUPPORTED, "wdg_vadvect_create: n_var must be 1..8");
        if (n_colloc < kMinN || n_colloc > kMaxN)
            return fail(WDG_ERR_UNSUPPORTED, "wdg_vadvect_create: n_colloc must be 2..9");
        if (basis_type != WDG_GAUSS_LEGENDRE && basis_type != WDG_GAUSS_LOBATTO)
            return fail(WDG_ERR_ARG, "wdg_vadvect_create: basis_type must be WDG_GAUSS_LEGENDRE or WDG_GAUSS_LOBATTO");
        const int n = n_colloc, nv = n_var;
        const bool approx = approx_quad != 0, legendre = basis_type == WDG_GAUSS_LEGENDRE;
        // default rules: Div<false> p = (n-2) + (n-1) + 1 + (n-1) (source/Div.cpp:313-330),
        // EdgeFlux<false> p = 2 (n-1) + 2 + (n-1) (source/EdgeFlux.cpp:496-512); exact to 2 (1 + p/2) - 1
        const int Q = approx ? n : 1 + ((n - 2) + (n - 1) + 1 + (n - 1)) / 2;
        const int Qf = approx ? n : 1 + (2 * (n - 1) + 2 + (n - 1)) / 2;
        std::vector<double> xg(n), wg(n), xv(Q), wv(Q), xf(Qf), wf(Qf), P((size_t)Q * n), D((size_t)Q * n),
            Pf((size_t)Qf * n), e(n), op, G, Mf, Mi;
        if (legendre)
            gauss_legendre(n, xg.data(), wg.data());
        else
            gauss_lobatto(n, xg.data(), wg.data());
        const double minus1 = -1.0;
        interp_matrix(n, xg.data(), 1, &minus1, e.data()); // phi_k(-1)
        if (approx)
        {
            xv = xg;
            wv = wg;
            xf = xg;
            wf = wg;
        }
        else
        {
            gauss_legendre(Q, xv.data(), wv.data());
            gauss_legendre(Qf, xf.data(), wf.data());
        }
        interp_matrix(n, xg.data(), Q, xv.data(), P.data());
        lagrange_deriv_at(n, xg.data(), Q, xv.data(), D.data());
        interp_matrix(n, xg.data(), Qf, xf.data(), Pf.data());
        volume_table(*mesh, n, nv, Q, approx, a, xg, wg, xv, wv, P, op);
        WDG_TRY(face_table(*mesh, n, nv, Qf, approx, legendre, a, e, wg, wf, Pf, G));
        if (!approx)
            WDG_TRY(exact_mass(*mesh, n, xg.data(), 1 + (2 * (n - 1) + 2) / 2, Mf, Mi));
        // Legendre: each side's neighbour and its side, and whether the edge runs against it
        std::vector<int> nb;
        if (legendre)
        {
            nb.assign(4 * (size_t)mesh->nel, -1);
            for (const EdgeRec &E : mesh->interior)
            {
                const int rev = E.delta < 0 ? 1 : 0;
                nb[4 * (size_t)E.el0 + E.s0] = ((E.el1 * 4 + E.s1) << 1) | rev;
                nb[4 * (size_t)E.el1 + E.s1] = ((E.el0 * 4 + E.s0) << 1) | rev;
            }
        }

        wdg_vadvect *h = new wdg_vadvect;
        h->n = n;
        h->nv = nv;
        h->Q = Q;
        h->Qf = Qf;
        h->approx = approx;
        h->legendre = legendre;
        int st = wdg_wave_create(mesh, n, nullptr, WDG_FP64, device, &h->w);
        if (st != WDG_OK)
        {
            wdg_vadvect_destroy(h);
            return st;
        }
        DeviceScope g(h->w->device);
        auto chk = [&](int r)
        {
            if (st == WDG_OK)
                st = r;
        };
        chk(upload(P, &h->d_Pv));
        chk(upload(D, &h->d_Dv));
        chk(upload(Pf, &h->d_Pf));
        chk(upload(xg, &h->d_xg));
        chk(upload(wg, &h->d_wg));
        chk(upload(op, &h->d_op));
        chk(upload(G, &h->d_G));
        chk(upload(e, &h->d_e));
        if (!approx)
            chk(upload(Mi, &h->d_Minv));
        if (legendre)
        {
            chk(device_alloc(&h->d_nb, nb.size()));
            if (st == WDG_OK)
                chk(device_put(h->d_nb, nb));
        }
        if (st == WDG_OK)
        {
            static std::mutex mu;
            static uint64_t set = 0;
            std::lock_guard<std::mutex> lock(mu);
            const int dev = h->w->device & 63;
            if (!(set & (1ull << dev)))
            {
                const cudaError_t e =
                    cudaFuncSetAttribute(vadv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
                if (e != cudaSuccess)
                    st = cuda_fail(e, "cudaFuncSetAttribute(vadv_kernel)");
                else
                    set |= 1ull << dev;
            }
        }
        if (st != WDG_OK)
        {
            wdg_vadvect_destroy(h);
            return st;
        }
        *out = h;
        return WDG_OK;
    }

    void wdg_vadvect_destroy(wdg_vadvect *h)
    {
        if (!h)
            return;
        if (h->w)
        {
            DeviceScope g(h->w->device);
            for (double *p : {h->d_Pv, h->d_Dv, h->d_Pf, h->d_xg, h->d_wg, h->d_e, h->d_op, h->d_G, h->d_Minv,
                              h->d_buf[0], h->d_buf[1], h->d_buf[2]})
                if (p)
                    cudaFree(p);
            if (h->d_nb)
                cudaFree(h->d_nb);
        }
        if (h->w)
            wdg_wave_destroy(h->w);
        delete h;
    }

    int wdg_vadvect_set_stream(wdg_vadvect *h, void *stream)
    {
        WDG_TRY(check(h));
        return wdg_wave_set_stream(h->w, stream);
    }
    int wdg_vadvect_sync(wdg_vadvect *h)
    {
        WDG_TRY(check(h));
        return wdg_wave_sync(h->w);
    }

    int wdg_vadvect_action(wdg_vadvect *h, const double *u, double *du)
    {
        return accumulate(h, VA_ACT, u, du, "wdg_vadvect_action");
    }
    int wdg_vadvect_bc_action(wdg_vadvect *h, const double *u, double *du)
    {
        return accumulate(h, VA_BC, u, du, "wdg_vadvect_bc_action");
    }

    // dudt = M^{-1} (Advection::action + AdvectionHomogeneousBC::action), the time derivative of
    // examples/advec2d.cpp
    int wdg_vadvect_rhs(wdg_vadvect *h, const double *u, double *dudt)
    {
        WDG_TRY(check(h));
        if (!u || !dudt || u == dudt)
            return fail(WDG_ERR_ARG, "wdg_vadvect_rhs: distinct u and dudt arrays required");
        DeviceScope g(h->w->device);
        HostArg a[2];
        WDG_TRY(bind_arg(h->w, 0, u, (size_t)nvals(h), true, false, a[0]));
        WDG_TRY(bind_arg(h->w, 1, dudt, (size_t)nvals(h), false, true, a[1]));
        ClawArgs c = claw_args(h->w, a[0].dev, a[1].dev);
        c.mode = CLAW_RHS;
        WDG_TRY(va_launch(h, c));
        return finish_args(h->w, a, 2);
    }

    // nsteps of ode::RungeKutta4 (method 0) or ode::SSPRK3 (method 1, the stepper of
    // examples/advec2d.cpp) on u in place, one fused launch per stage; *t advances by nsteps dt
    int wdg_vadvect_steps(wdg_vadvect *h, int method, double *u, double dt, double *t, int nsteps)
    {
        WDG_TRY(check(h));
        if (!u || !t || nsteps < 0 || (method != 0 && method != 1))
            return fail(WDG_ERR_ARG, "wdg_vadvect_steps: method 0 (RK4) or 1 (SSPRK3), nsteps >= 0");
        DeviceScope g(h->w->device);
        for (int k = 0; k < 3; ++k)
            if (!h->d_buf[k])
                WDG_TRY(device_alloc(&h->d_buf[k], (size_t)nvals(h)));
        HostArg ha;
        WDG_TRY(bind_arg(h->w, 2, u, (size_t)nvals(h), true, true, ha));
        double *ud = ha.dev;
        ClawArgs a = claw_args(h->w, ud, nullptr);
        a.dt = dt;
        for (int s = 0; s < nsteps; ++s)
        {
            if (method == 0)
            {
                // the rotation of the wave path: reads u, B, C, B, C and writes B, C, B, C, u
                double *B = h->d_buf[0], *Cb = h->d_buf[1];
                a.du = h->d_buf[2];
                const double *src = ud;
                for (int st = 0; st < 5; ++st)
                {
                    double *dst = (st == 4) ? ud : ((st % 2 == 0) ? B : Cb);
                    a.x = src;
                    a.out = dst;
                    a.mode = CLAW_RK4;
                    a.rk_a = rk4a[st];
                    a.rk_b = rk4b[st];
                    WDG_TRY(va_launch(h, a));
                    src = dst;
                }
            }
            else
            {
                a.base = ud;
                a.x = ud;
                a.out = h->d_buf[0];
                a.mode = CLAW_SSP0;
                WDG_TRY(va_launch(h, a));
                a.x = h->d_buf[0];
                a.out = h->d_buf[1];
                a.mode = CLAW_SSP1;
                WDG_TRY(va_launch(h, a));
                a.x = h->d_buf[1];
                a.out = ud;
                a.mode = CLAW_SSP2;
                WDG_TRY(va_launch(h, a));
            }
            *t += dt;
        }
        return finish_args(h->w, &ha, 1);
    }
}
