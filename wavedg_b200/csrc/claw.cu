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
#include <vector>

#include "wave_impl.hpp"

using namespace wdg;

struct wdg_claw
{
    wdg_wave *w = nullptr;
    int n = 0, nv = 4;
    double *d_buf[4] = {nullptr, nullptr, nullptr, nullptr}; // stepping: RK4 B, C, register; SSPRK3 y1, y2
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
    long long nvals(const wdg_claw *h) { return (long long)h->nv * h->n * h->n * h->w->nel; }

    int ensure_bufs(wdg_claw *h)
    {
        for (int k = 0; k < 3; ++k)
            if (!h->d_buf[k])
                WDG_TRY(device_alloc(&h->d_buf[k], (size_t)nvals(h)));
        return WDG_OK;
    }

    int check(wdg_claw *h) { return h ? WDG_OK : fail(WDG_ERR_ARG, "null conservation-law handle"); }
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

    void wdg_claw_destroy(wdg_claw *h)
    {
        if (!h)
            return;
        {
            DeviceScope g(h->w ? h->w->device : 0);
            for (double *p : h->d_buf)
                if (p)
                    cudaFree(p);
        }
        if (h->w)
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
        WDG_CUDA(launch_euler_face_flux(h->n, ne, face_type == WDG_INTERIOR ? w->d_edgesI : w->d_edgesB, w->d_corners,
                                        a[0].dev, same ? a[0].dev : a[1].dev, w->stream));
        return finish_args(w, a, same ? 1 : 2);
    }

    // the time derivative of examples/cl2d.cpp:171-220 (approx_quad = true)
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
        WDG_TRY(claw_steps(h->w, 0, h->nv, nullptr, nullptr, h->d_buf, method, a.dev, dt, t, nsteps));
        return finish_args(h->w, &a, 1);
    }
}
