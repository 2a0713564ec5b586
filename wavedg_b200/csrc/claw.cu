// C-ABI: the nonlinear conservation-law path for the compressible Euler system of
// examples/cl2d.cpp (DivF2D<true>, EdgeFluxF2D<true>, the Lobatto prolongators and
// MassMatrix<true> with the example's flux and local Lax-Friedrichs numerical flux), and the
// fused RHS / time stepping it shares with linear advection (claw_kernels.cuh).
//
// State layout: the reference's u(d, i, j, el) with d = density, x-momentum, y-momentum,
// energy (4 values per node).  FP64.  Geometry, partner tables and argument staging are those
// of an internal collocation handle.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "claw_model.cuh"
#include "wave_impl.hpp"

using namespace wdg;

struct wdg_claw
{
    wdg_wave *w = nullptr;
    int n = 0, nv = 4;
    double *d_buf[4] = {nullptr, nullptr, nullptr, nullptr}; // stepping: RK4 B, C, register; SSPRK3 y1, y2
    // approx_quad = false: the exact operators' geometry and M^{-1} (an internal exact handle,
    // whose collocation handle is w), the volume rule (q points) and the face rule (qf points)
    wdg_waveq *exact = nullptr;
    int q = 0, qf = 0;
    double *d_xv = nullptr, *d_wv = nullptr, *d_Pv = nullptr, *d_Dv = nullptr, *d_wf = nullptr, *d_Pf = nullptr;
};

namespace wdg
{
    ClawArgs claw_args(const wdg_wave *w, const double *x, double *out)
    {
        ClawArgs a{};
        a.x = x;
        a.out = out;
        a.corners = w->d_corners;
        a.fbase = w->d_fbase;
        a.fcode = w->d_fcode;
        a.err = w->d_err;
        a.nel = w->nel;
        return a;
    }

    // nsteps of ode::RungeKutta4 (method 0) or ode::SSPRK3 (method 1) on device array u (in
    // place) with the fused kernel of flux model `model`; bufs: 3 arrays of u's size
    int claw_steps(wdg_wave *w, int model, int nv, const double *A, const double *absA, double *const *bufs, int method,
                   double *u, double dt, double *t, int nsteps)
    {
        ClawArgs a = claw_args(w, u, nullptr);
        a.A = A;
        a.absA = absA;
        a.dt = dt;
        for (int s = 0; s < nsteps; ++s)
        {
            if (method == 0)
            {
                // the rotation of the wave path: reads u, B, C, B, C and writes B, C, B, C, u
                double *B = bufs[0], *Cb = bufs[1];
                a.du = bufs[2];
                const double *src = u;
                for (int st = 0; st < 5; ++st)
                {
                    double *dst = (st == 4) ? u : ((st % 2 == 0) ? B : Cb);
                    a.x = src;
                    a.out = dst;
                    a.mode = CLAW_RK4;
                    a.rk_a = rk4a[st];
                    a.rk_b = rk4b[st];
                    WDG_CUDA(launch_claw(model, w->n, nv, a, w->stream));
                    src = dst;
                }
            }
            else
            {
                // y1 = u + dt f(u); y2 = (y1 + 3 u + dt f(y1)) / 4; u = (u + 2 y2 + 2 dt f(y2)) / 3
                double *y1 = bufs[0], *y2 = bufs[1];
                a.base = u;
                a.x = u;
                a.out = y1;
                a.mode = CLAW_SSP0;
                WDG_CUDA(launch_claw(model, w->n, nv, a, w->stream));
                a.x = y1;
                a.out = y2;
                a.mode = CLAW_SSP1;
                WDG_CUDA(launch_claw(model, w->n, nv, a, w->stream));
                a.x = y2;
                a.out = u;
                a.mode = CLAW_SSP2;
                WDG_CUDA(launch_claw(model, w->n, nv, a, w->stream));
            }
            *t += dt;
        }
        return WDG_OK;
    }
} // namespace wdg

namespace
{
    // ------------------------------------------------------------------ approx_quad = false
    // The Euler operators of examples/cl2d.cpp as shipped (DivF2D<false>, EdgeFluxF2D<false>,
    // MassMatrix<false>; wavedg/DivF.hpp:262-394, wavedg/EdgeFluxF.hpp:182-254) fused per
    // element, a warp each: u interpolated to the q x q volume points (P), the physical flux
    // there, its contravariant form with the Jacobian at the points and the weights, the D and
    // P contractions back to the nodes; per side the element's own nodal trace and its
    // neighbour's (partner table; boundary: the own trace, exterior = interior) interpolated
    // to the qf face points, the local Lax-Friedrichs flux with the element's own normal times
    // w_i |E|/2, projected back and subtracted; then the dense inverse mass matrix, and the RHS
    // or one RK4 / SSPRK3 stage.
    struct QEArgs
    {
        ClawArgs c;
        const double *xv, *wv, *Pv, *Dv, *wf, *Pf, *Minv;
        int n, q, qf;
    };
    constexpr int kQENV = 4;

    __host__ __device__ inline int qe_warp_doubles(int n, int q, int qf)
    {
        // su r (4 n^2 each) | Pu (4 n q) | Uq (4 q^2) | Fq (8 q^2) | Df Pg (4 q n each) | T1 (4 n 4) | UF (4 qf 4)
        return 8 * n * n + 4 * n * q + 12 * q * q + 8 * q * n + 16 * n + 16 * qf;
    }

    __device__ inline void qe_jac(const double *c, double xi, double eta, double J[4])
    {
        J[0] = 0.25 * ((1.0 - eta) * (c[2] - c[0]) + (1.0 + eta) * (c[4] - c[6]));
        J[1] = 0.25 * ((1.0 - eta) * (c[3] - c[1]) + (1.0 + eta) * (c[5] - c[7]));
        J[2] = 0.25 * ((1.0 - xi) * (c[6] - c[0]) + (1.0 + xi) * (c[4] - c[2]));
        J[3] = 0.25 * ((1.0 - xi) * (c[7] - c[1]) + (1.0 + xi) * (c[5] - c[3]));
    }
    __device__ inline int qe_node(int n, int s, int k)
    {
        const int i = (s == 0 || s == 2) ? k : (s == 1 ? n - 1 : 0);
        const int j = (s == 1 || s == 3) ? k : (s == 2 ? n - 1 : 0);
        return i + n * j;
    }
    __global__ void qeuler_kernel(const QEArgs A, int warps)
    {
        extern __shared__ double esm[];
        const ClawArgs &a = A.c;
        const int n = A.n, q = A.q, qf = A.qf, nn = n * n, qq = q * q, NV = kQENV;
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        double *su = esm + (size_t)warp * qe_warp_doubles(n, q, qf);
        double *r = su + NV * nn, *Pu = r + NV * nn, *Uq = Pu + NV * n * q, *Fq = Uq + NV * qq, *Df = Fq + 2 * NV * qq;
        double *Pg = Df + NV * q * n, *T1 = Pg + NV * q * n, *UF = T1 + 4 * n * NV;
        const long long limit = (long long)nn * a.nel;
        for (int el = blockIdx.x * warps + warp; el < a.nel; el += gridDim.x * warps)
        {
            const double *xe = a.x + (size_t)NV * nn * el;
            for (int k = lane; k < NV * nn; k += 32)
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
            // Pu(l, d, i) = sum_k P(i, k) u(d, k, l)
            for (int o = lane; o < NV * n * q; o += 32)
            {
                const int l = o % n, d = (o / n) % NV, i = o / (NV * n);
                double t = 0.0;
                for (int k = 0; k < n; ++k)
                    t += A.Pv[i + q * k] * su[d + NV * (k + n * l)];
                Pu[o] = t;
            }
            __syncwarp();
            // U(d, i, j) = sum_l P(j, l) Pu(l, d, i)
            for (int o = lane; o < NV * qq; o += 32)
            {
                const int d = o % NV, i = (o / NV) % q, j = o / (NV * q);
                double t = 0.0;
                for (int l = 0; l < n; ++l)
                    t += A.Pv[j + q * l] * Pu[l + n * (d + NV * i)];
                Uq[o] = t;
            }
            __syncwarp();
            // contravariant fluxes at the points: F0(d, i, j), F1(d, i, j) at Fq[2 d (+1) + 2 NV (i + q j)]
            for (int o = lane; o < qq; o += 32)
            {
                const int i = o % q, j = o / q;
                double J[4], f[4], g[4];
                qe_jac(c, A.xv[i], A.xv[j], J);
                const double W = A.wv[i] * A.wv[j];
                const double Ye = J[3] * W, Xe = J[2] * W, Yx = J[1] * W, Xx = J[0] * W;
                ClawEuler::flux(a, Uq + NV * o, f, g);
                double *Fo = Fq + 2 * NV * o;
                for (int d = 0; d < NV; ++d)
                {
                    Fo[2 * d] = Ye * f[d] - Xe * g[d];
                    Fo[2 * d + 1] = -Yx * f[d] + Xx * g[d];
                }
            }
            __syncwarp();
            // Df(j, d, k) = sum_i D(i, k) F0(d, i, j);  Pg(j, d, k) = sum_i P(i, k) F1(d, i, j)
            for (int o = lane; o < NV * q * n; o += 32)
            {
                const int j = o % q, d = (o / q) % NV, k = o / (NV * q);
                double df = 0.0, pg = 0.0;
                for (int i = 0; i < q; ++i)
                {
                    df += A.Dv[i + q * k] * Fq[2 * d + 2 * NV * (i + q * j)];
                    pg += A.Pv[i + q * k] * Fq[2 * d + 1 + 2 * NV * (i + q * j)];
                }
                Df[o] = df;
                Pg[o] = pg;
            }
            // neighbour nodal traces T1(s, k, d); boundary: the own trace
            for (int o = lane; o < 4 * n; o += 32)
            {
                const int s = o / n, k = o - s * n;
                const uint32_t byte = (codes >> (8 * s)) & 0xffu;
                const double *own = su + NV * qe_node(n, s, k);
                double *t1 = T1 + NV * o;
                bool copy = (byte & 0x80u) != 0;
                if (!copy)
                {
                    const int off = (s == 0) ? fb.x : (s == 1) ? fb.y : (s == 2) ? fb.z : fb.w;
                    const uint32_t sc = byte & 3u;
                    const int stride = (sc == 0) ? 1 : (sc == 1) ? -1 : (sc == 2) ? n : -n; // in nodes
                    const long long pn = (long long)(off / 3) + (long long)k * stride;
                    if (off < 0 || pn < 0 || pn >= limit)
                    {
                        atomicOr(a.err, 2u);
                        copy = true;
                    }
                    else
                        for (int d = 0; d < NV; ++d)
                            t1[d] = __ldg(a.x + (size_t)NV * pn + d);
                }
                if (copy)
                    for (int d = 0; d < NV; ++d)
                        t1[d] = own[d];
            }
            __syncwarp();
            // volume result
            for (int o = lane; o < NV * nn; o += 32)
            {
                const int d = o % NV, k = (o / NV) % n, l = o / (NV * n);
                double t = 0.0;
                for (int j = 0; j < q; ++j)
                    t += A.Pv[j + q * l] * Df[j + q * (d + NV * k)] + A.Dv[j + q * l] * Pg[j + q * (d + NV * k)];
                r[o] = t;
            }
            // face points: UF(s, i, d) = w_i |E|/2 fh(n, own, neighbour)
            for (int o = lane; o < 4 * qf; o += 32)
            {
                const int s = o / qf, i = o - s * qf;
                double nx, ny, meas, qL[4] = {0, 0, 0, 0}, qR[4] = {0, 0, 0, 0};
                claw_side(c, s, nx, ny, meas);
                for (int j = 0; j < n; ++j)
                {
                    const double pw = A.Pf[i + qf * j];
                    const double *own = su + NV * qe_node(n, s, j), *nb = T1 + NV * (s * n + j);
                    for (int d = 0; d < NV; ++d)
                    {
                        qL[d] += own[d] * pw;
                        qR[d] += nb[d] * pw;
                    }
                }
                double fh[4];
                ClawEuler::numflux<4>(a, el, s, nx, ny, qL, qR, fh);
                const double ds = A.wf[i] * meas;
                for (int d = 0; d < NV; ++d)
                    UF[NV * o + d] = fh[d] * ds;
            }
            __syncwarp();
            if (a.mode == CLAW_DIV)
            {
                for (int o = lane; o < NV * nn; o += 32)
                    a.out[(size_t)NV * nn * el + o] += r[o];
                __syncwarp();
                continue;
            }
            // back to the face nodes, subtracted: sides 0 and 2, then 1 and 3
            for (int pass = 0; pass < 2; ++pass)
            {
                for (int o = lane; o < 2 * n; o += 32)
                {
                    const int s = pass + 2 * (o / n), k = o % n, node = qe_node(n, s, k);
                    for (int d = 0; d < NV; ++d)
                    {
                        double f = 0.0;
                        for (int i = 0; i < qf; ++i)
                            f += UF[NV * (s * qf + i) + d] * A.Pf[i + qf * k];
                        r[NV * node + d] -= f;
                    }
                }
                __syncwarp();
            }
            // M^{-1} (dense, per field) and the output: lane per row
            const double *Me = A.Minv + (size_t)nn * nn * el;
            for (int row = lane; row < nn; row += 32)
            {
                double y[4] = {0, 0, 0, 0};
                for (int j = 0; j < nn; ++j)
                {
                    const double m = __ldg(Me + row + (size_t)nn * j);
                    for (int d = 0; d < NV; ++d)
                        y[d] += m * r[NV * j + d];
                }
                const size_t g0 = (size_t)NV * (nn * (size_t)el + row);
                for (int d = 0; d < NV; ++d)
                {
                    const double qd = su[NV * row + d];
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

    // EdgeFluxF2D<false>::action on face traces (n, 4, 2, edges): thread per edge; both sides'
    // traces to the qf points, the flux with the first element's normal, back with P^T ds
    __global__ void qeuler_face_kernel(int n, int qf, int ne, const int *__restrict__ edges,
                                       const double *__restrict__ corners, const double *__restrict__ wf,
                                       const double *__restrict__ Pf, const double *ub, double *fb)
    {
        const int e = blockIdx.x * blockDim.x + threadIdx.x;
        if (e >= ne)
            return;
        const int el = edges[5 * (size_t)e], s = edges[5 * (size_t)e + 1];
        double c[8];
        for (int k = 0; k < 8; ++k)
            c[k] = corners[8 * (size_t)el + k];
        double nx, ny, meas;
        claw_side(c, s, nx, ny, meas);
        double acc[9][4];
        for (int k = 0; k < n; ++k)
            for (int d = 0; d < 4; ++d)
                acc[k][d] = 0.0;
        for (int i = 0; i < qf; ++i)
        {
            double qL[4] = {0, 0, 0, 0}, qR[4] = {0, 0, 0, 0};
            for (int j = 0; j < n; ++j)
                for (int d = 0; d < 4; ++d)
                {
                    qL[d] += ub[j + n * (d + 4 * (0 + 2 * (size_t)e))] * Pf[i + qf * j];
                    qR[d] += ub[j + n * (d + 4 * (1 + 2 * (size_t)e))] * Pf[i + qf * j];
                }
            double fh[4];
            ClawEuler::numflux<4>(ClawArgs{}, e, s, nx, ny, qL, qR, fh);
            const double ds = wf[i] * meas;
            for (int d = 0; d < 4; ++d)
                for (int k = 0; k < n; ++k)
                    acc[k][d] += fh[d] * Pf[i + qf * k] * ds;
        }
        for (int k = 0; k < n; ++k)
            for (int d = 0; d < 4; ++d)
            {
                fb[k + n * (d + 4 * (0 + 2 * (size_t)e))] = acc[k][d];
                fb[k + n * (d + 4 * (1 + 2 * (size_t)e))] = -acc[k][d];
            }
    }

    int qe_warps(const wdg_claw *h)
    {
        const size_t per = sizeof(double) * (size_t)qe_warp_doubles(h->n, h->q, h->qf);
        return (int)std::max<size_t>(1, std::min<size_t>(4, (size_t)(200 * 1024) / per));
    }

    int qe_launch(wdg_claw *h, const ClawArgs &c)
    {
        QEArgs A{};
        A.c = c;
        A.xv = h->d_xv;
        A.wv = h->d_wv;
        A.Pv = h->d_Pv;
        A.Dv = h->d_Dv;
        A.wf = h->d_wf;
        A.Pf = h->d_Pf;
        A.Minv = waveq_minv(h->exact);
        A.n = h->n;
        A.q = h->q;
        A.qf = h->qf;
        const int warps = qe_warps(h);
        const size_t smem = sizeof(double) * (size_t)qe_warp_doubles(h->n, h->q, h->qf) * warps;
        const unsigned blocks = (unsigned)std::max(1, std::min((c.nel + warps - 1) / warps, 148 * 16));
        qeuler_kernel<<<blocks, 32 * warps, smem, h->w->stream>>>(A, warps);
        WDG_CUDA(cudaGetLastError());
        return WDG_OK;
    }

    // the fused stage launches of claw_steps, for the exact operators
    int qe_steps(wdg_claw *h, int method, double *u, double dt, double *t, int nsteps)
    {
        ClawArgs a = claw_args(h->w, u, nullptr);
        a.dt = dt;
        for (int s = 0; s < nsteps; ++s)
        {
            if (method == 0)
            {
                double *B = h->d_buf[0], *Cb = h->d_buf[1];
                a.du = h->d_buf[2];
                const double *src = u;
                for (int st = 0; st < 5; ++st)
                {
                    double *dst = (st == 4) ? u : ((st % 2 == 0) ? B : Cb);
                    a.x = src;
                    a.out = dst;
                    a.mode = CLAW_RK4;
                    a.rk_a = rk4a[st];
                    a.rk_b = rk4b[st];
                    WDG_TRY(qe_launch(h, a));
                    src = dst;
                }
            }
            else
            {
                a.base = u;
                a.x = u;
                a.out = h->d_buf[0];
                a.mode = CLAW_SSP0;
                WDG_TRY(qe_launch(h, a));
                a.x = h->d_buf[0];
                a.out = h->d_buf[1];
                a.mode = CLAW_SSP1;
                WDG_TRY(qe_launch(h, a));
                a.x = h->d_buf[1];
                a.out = u;
                a.mode = CLAW_SSP2;
                WDG_TRY(qe_launch(h, a));
            }
            *t += dt;
        }
        return WDG_OK;
    }

    long long nvals(const wdg_claw *h) { return (long long)h->nv * h->n * h->n * h->w->nel; }

    int ensure_bufs(wdg_claw *h)
    {
        for (int k = 0; k < 3; ++k)
            if (!h->d_buf[k])
                WDG_TRY(device_alloc(&h->d_buf[k], (size_t)nvals(h)));
        return WDG_OK;
    }

    int check(wdg_claw *h) { return h ? WDG_OK : fail(WDG_ERR_ARG, "null conservation-law handle"); }

    int upload(const std::vector<double> &v, double **d)
    {
        WDG_TRY(device_alloc(d, v.size()));
        WDG_CUDA(cudaMemcpy(*d, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice));
        return WDG_OK;
    }

    // the 2n-point Gauss-Legendre rules of DivF2D<false> and EdgeFluxF2D<false>
    // (source/DivF.cpp:59, source/EdgeFluxF.cpp:55) and their matrices on the GLL basis
    int exact_tables(wdg_claw *h)
    {
        const int n = h->n, q = 2 * n;
        h->q = h->qf = q;
        std::vector<double> x(n), wg(n), xq(q), wq(q), P((size_t)q * n), D((size_t)q * n);
        gauss_lobatto(n, x.data(), wg.data());
        gauss_legendre(q, xq.data(), wq.data());
        interp_matrix(n, x.data(), q, xq.data(), P.data());
        lagrange_deriv_at(n, x.data(), q, xq.data(), D.data());
        WDG_TRY(upload(xq, &h->d_xv));
        WDG_TRY(upload(wq, &h->d_wv));
        WDG_TRY(upload(P, &h->d_Pv));
        WDG_TRY(upload(D, &h->d_Dv));
        WDG_TRY(upload(wq, &h->d_wf));
        WDG_TRY(upload(P, &h->d_Pf));
        static std::mutex mu;
        static uint64_t set = 0;
        std::lock_guard<std::mutex> lock(mu);
        const int dev = h->w->device & 63;
        if (!(set & (1ull << dev)))
        {
            WDG_CUDA(cudaFuncSetAttribute(qeuler_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
            set |= 1ull << dev;
        }
        return WDG_OK;
    }
} // namespace

extern "C"
{
    int wdg_euler_create(const wdg_mesh *mesh, int n_colloc, int device, wdg_claw **out)
    {
        if (!mesh || !out)
            return fail(WDG_ERR_ARG, "wdg_euler_create: null argument");
        *out = nullptr;
        wdg_wave *w = nullptr;
        WDG_TRY(wdg_wave_create(mesh, n_colloc, nullptr, WDG_FP64, device, &w));
        wdg_claw *h = new wdg_claw;
        h->w = w;
        h->n = n_colloc;
        h->nv = 4;
        *out = h;
        return WDG_OK;
    }

    // examples/cl2d.cpp as shipped (approx_quad = false): DivF2D<false>, EdgeFluxF2D<false> on
    // 2n-point Gauss-Legendre rules and MassMatrix<false>
    int wdg_euler_create_exact(const wdg_mesh *mesh, int n_colloc, int device, wdg_claw **out)
    {
        if (!mesh || !out)
            return fail(WDG_ERR_ARG, "wdg_euler_create_exact: null argument");
        *out = nullptr;
        wdg_waveq *q = nullptr;
        WDG_TRY(wdg_waveq_create(mesh, n_colloc, nullptr, device, &q));
        wdg_claw *h = new wdg_claw;
        h->exact = q;
        wdg_waveq_wave(q, &h->w);
        h->n = n_colloc;
        h->nv = 4;
        DeviceScope g(h->w->device);
        const int st = exact_tables(h);
        if (st != WDG_OK)
        {
            wdg_claw_destroy(h);
            return st;
        }
        *out = h;
        return WDG_OK;
    }

    void wdg_claw_destroy(wdg_claw *h)
    {
        if (!h)
            return;
        {
            DeviceScope g(h->w ? h->w->device : 0);
            for (double *p : h->d_buf)
                if (p)
                    cudaFree(p);
            for (double *p : {h->d_xv, h->d_wv, h->d_Pv, h->d_Dv, h->d_wf, h->d_Pf})
                if (p)
                    cudaFree(p);
        }
        if (h->exact)
            wdg_waveq_destroy(h->exact); // owns w
        else if (h->w)
            wdg_wave_destroy(h->w);
        delete h;
    }

    int wdg_claw_set_stream(wdg_claw *h, void *stream)
    {
        WDG_TRY(check(h));
        return wdg_wave_set_stream(h->w, stream);
    }
    int wdg_claw_sync(wdg_claw *h)
    {
        WDG_TRY(check(h));
        return wdg_wave_sync(h->w);
    }

    // DivF2D<true>::action: divF += (F(u), grad v)
    int wdg_claw_div(wdg_claw *h, const double *u, double *divF)
    {
        WDG_TRY(check(h));
        if (!u || !divF || u == divF)
            return fail(WDG_ERR_ARG, "wdg_claw_div: distinct u and divF arrays required");
        DeviceScope g(h->w->device);
        HostArg a[2];
        WDG_TRY(bind_arg(h->w, 0, u, (size_t)nvals(h), true, false, a[0]));
        WDG_TRY(bind_arg(h->w, 1, divF, (size_t)nvals(h), true, true, a[1]));
        ClawArgs c = claw_args(h->w, a[0].dev, a[1].dev);
        c.mode = CLAW_DIV;
        if (h->exact)
            WDG_TRY(qe_launch(h, c));
        else
            WDG_CUDA(launch_claw(0, h->n, h->nv, c, h->w->stream));
        return finish_args(h->w, a, 2);
    }

    // EdgeFluxF2D<true>::action on face traces uB (n, 4, 2, n_edges(face_type)) -> fB (may alias uB)
    int wdg_claw_flux(wdg_claw *h, int face_type, const double *uB, double *fB)
    {
        WDG_TRY(check(h));
        if (!uB || !fB || (face_type != WDG_INTERIOR && face_type != WDG_BOUNDARY))
            return fail(WDG_ERR_ARG, "wdg_claw_flux: bad arguments");
        DeviceScope g(h->w->device);
        wdg_wave *w = h->w;
        const int ne = face_type == WDG_INTERIOR ? w->nI : w->nB;
        const size_t cnt = (size_t)h->n * 4 * 2 * ne;
        if (ne == 0)
            return WDG_OK;
        HostArg a[2];
        const bool same = uB == fB;
        WDG_TRY(bind_arg(w, 0, uB, cnt, true, same, a[0]));
        if (!same)
            WDG_TRY(bind_arg(w, 1, fB, cnt, false, true, a[1]));
        const int *edges = face_type == WDG_INTERIOR ? w->d_edgesI : w->d_edgesB;
        double *fd = same ? a[0].dev : a[1].dev;
        if (h->exact)
        {
            qeuler_face_kernel<<<(ne + 127) / 128, 128, 0, w->stream>>>(h->n, h->qf, ne, edges, w->d_corners, h->d_wf,
                                                                        h->d_Pf, a[0].dev, fd);
            WDG_CUDA(cudaGetLastError());
        }
        else
            WDG_CUDA(launch_euler_face_flux(h->n, ne, edges, w->d_corners, a[0].dev, fd, w->stream));
        return finish_args(w, a, same ? 1 : 2);
    }

    // the time derivative of examples/cl2d.cpp:171-220 (either quadrature)
    int wdg_claw_rhs(wdg_claw *h, const double *u, double *dudt)
    {
        WDG_TRY(check(h));
        if (!u || !dudt || u == dudt)
            return fail(WDG_ERR_ARG, "wdg_claw_rhs: distinct u and dudt arrays required");
        DeviceScope g(h->w->device);
        HostArg a[2];
        WDG_TRY(bind_arg(h->w, 0, u, (size_t)nvals(h), true, false, a[0]));
        WDG_TRY(bind_arg(h->w, 1, dudt, (size_t)nvals(h), false, true, a[1]));
        ClawArgs c = claw_args(h->w, a[0].dev, a[1].dev);
        c.mode = CLAW_RHS;
        if (h->exact)
            WDG_TRY(qe_launch(h, c));
        else
            WDG_CUDA(launch_claw(0, h->n, h->nv, c, h->w->stream));
        return finish_args(h->w, a, 2);
    }

    // nsteps of ode::RungeKutta4 (method 0) or ode::SSPRK3 (method 1, the stepper of
    // examples/cl2d.cpp) on u in place; *t advances by nsteps dt
    int wdg_claw_steps(wdg_claw *h, int method, double *u, double dt, double *t, int nsteps)
    {
        WDG_TRY(check(h));
        if (!u || !t || nsteps < 0 || (method != 0 && method != 1))
            return fail(WDG_ERR_ARG, "wdg_claw_steps: method 0 (RK4) or 1 (SSPRK3), nsteps >= 0");
        DeviceScope g(h->w->device);
        WDG_TRY(ensure_bufs(h));
        HostArg a;
        WDG_TRY(bind_arg(h->w, 2, u, (size_t)nvals(h), true, true, a));
        if (h->exact)
            WDG_TRY(qe_steps(h, method, a.dev, dt, t, nsteps));
        else
            WDG_TRY(claw_steps(h->w, 0, h->nv, nullptr, nullptr, h->d_buf, method, a.dev, dt, t, nsteps));
        return finish_args(h->w, &a, 1);
    }
}
