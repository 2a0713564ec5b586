// C-ABI: WaveHoltz (source/WaveHoltz.cpp) on the fused stage kernel.
//
// A period is nt RK4 steps = 5 nt stage launches; the cos(omega t) filter
// accumulation acc += c_it * p is fused into the fifth stage of every step and
// kept in FP64 whatever the stepping precision.  Each period is captured once
// into a CUDA graph on a private stream and replayed; the residual of the
// fixed-point update is reduced in FP64 in the same pass that forms
// W <- S W + pi0.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "wave_impl.hpp"

using namespace wdg;

struct wdg_waveholtz
{
    wdg_wave *w = nullptr;
    double omega = 0, T = 0, dt = 0;
    int nt = 0;
    std::vector<double> c_filter; // c_it, it = 1..nt
    double c0 = 0;                // 0.5 dt K(0)
    cudaStream_t cs = nullptr;    // private capture stream
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    double *d_W = nullptr, *d_acc = nullptr, *d_pi0 = nullptr;
    void *d_F = nullptr; // forcing in the stepping precision
    cudaGraphExec_t g_S = nullptr, g_pi0 = nullptr;
    double pi0_norm = 0;
    wdg_waveq *q = nullptr; // exact quadrature (approx_quad = false): periods on its operators
};

namespace
{
    double K(const wdg_waveholtz *h, double t) { return h->omega / M_PI * (std::cos(h->omega * t) - 0.25); }

    // run `body` on the private stream, ordered after and before the handle's stream
    template <class Body>
    int on_private_stream(wdg_waveholtz *h, Body body)
    {
        wdg_wave *w = h->w;
        cudaStream_t user = w->stream;
        WDG_CUDA(cudaEventRecord(h->ev_in, user));
        WDG_CUDA(cudaStreamWaitEvent(h->cs, h->ev_in, 0));
        w->stream = h->cs;
        int s = body();
        w->stream = user;
        cudaError_t e = cudaEventRecord(h->ev_out, h->cs);
        if (e == cudaSuccess)
            e = cudaStreamWaitEvent(user, h->ev_out, 0);
        if (s == WDG_OK && e != cudaSuccess)
            return cuda_fail(e, "stream ordering");
        return s;
    }

    template <typename Real>
    int period(wdg_waveholtz *h, bool forced)
    {
        wdg_wave *w = h->w;
        if (h->q)
            return waveq_period(h->q, static_cast<double *>(w->d_state[0]), h->dt, h->nt,
                                forced ? static_cast<const double *>(h->d_F) : nullptr, h->omega, h->d_acc,
                                h->c_filter.data());
        RKExtras x;
        x.acc = h->d_acc;
        x.c_filter = h->c_filter.data();
        if (forced)
        {
            x.F = h->d_F;
            x.omega = h->omega;
        }
        double t = 0.0;
        return rk4_run<Real>(w, static_cast<Real *>(w->d_state[0]), h->dt, t, h->nt, x);
    }

    // prologue + one period, from d_W (S) or from zero (pi0), as a graph
    int record_period(wdg_waveholtz *h, bool forced, cudaGraphExec_t *exec)
    {
        wdg_wave *w = h->w;
        const bool fp32 = w->precision == WDG_FP32;
        WDG_CUDA(cudaStreamBeginCapture(h->cs, cudaStreamCaptureModeThreadLocal));
        int s = WDG_OK;
        cudaError_t e = cudaSuccess;
        if (forced)
        {
            e = cudaMemsetAsync(w->d_state[0], 0, w->real_size() * (size_t)w->ndof, h->cs);
            if (e == cudaSuccess)
                e = cudaMemsetAsync(h->d_acc, 0, sizeof(double) * (size_t)w->ndof, h->cs);
        }
        else
        {
            e = fp32 ? launch_scale_into<float>(h->d_W, static_cast<float *>(w->d_state[0]), h->d_acc, h->c0, w->ndof, h->cs)
                     : launch_scale_into<double>(h->d_W, static_cast<double *>(w->d_state[0]), h->d_acc, h->c0, w->ndof, h->cs);
        }
        if (e != cudaSuccess)
            s = cuda_fail(e, "WaveHoltz prologue");
        if (s == WDG_OK)
            s = fp32 ? period<float>(h, forced) : period<double>(h, forced);
        cudaGraph_t graph = nullptr;
        e = cudaStreamEndCapture(h->cs, &graph);
        if (s != WDG_OK)
        {
            if (graph)
                cudaGraphDestroy(graph);
            return s;
        }
        if (e != cudaSuccess)
            return cuda_fail(e, "cudaStreamEndCapture");
        e = cudaGraphInstantiate(exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess)
            return cuda_fail(e, "cudaGraphInstantiate");
        return WDG_OK;
    }

    int run_period(wdg_waveholtz *h, bool forced)
    {
        cudaGraphExec_t *g = forced ? &h->g_pi0 : &h->g_S;
        if (!*g)
            WDG_TRY(record_period(h, forced, g));
        WDG_CUDA(cudaGraphLaunch(*g, h->cs));
        return WDG_OK;
    }

    // F (FP64, host or device) -> d_F in the stepping precision
    int set_forcing(wdg_waveholtz *h, const double *F)
    {
        wdg_wave *w = h->w;
        bool dev = false;
        WDG_TRY(is_device_ptr(w, F, dev));
        const double *src = F;
        if (!dev)
        {
            WDG_TRY(ensure_stage(w, 2));
            WDG_CUDA(cudaMemcpyAsync(w->d_stage[2], F, sizeof(double) * w->ndof, cudaMemcpyHostToDevice, h->cs));
            src = w->d_stage[2];
        }
        if (w->precision == WDG_FP32)
            WDG_CUDA(launch_convert<double, float>(src, static_cast<float *>(h->d_F), w->ndof, h->cs));
        else
            WDG_CUDA(cudaMemcpyAsync(h->d_F, src, sizeof(double) * w->ndof, cudaMemcpyDeviceToDevice, h->cs));
        return WDG_OK;
    }

    int copy_in(wdg_waveholtz *h, double *dst, const double *src)
    {
        WDG_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * h->w->ndof, cudaMemcpyDefault, h->cs));
        return WDG_OK;
    }

    int finish_host(wdg_waveholtz *h)
    {
        WDG_CUDA(cudaStreamSynchronize(h->cs));
        return check_device_error(h->w);
    }
} // namespace

extern "C"
{
    int wdg_waveholtz_create(wdg_wave *w, double omega, wdg_waveholtz **out)
    {
        if (!w || !out || !(omega > 0.0))
            return fail(WDG_ERR_ARG, "wdg_waveholtz_create: need a discretisation and omega > 0");
        if (w->halo)
            return fail(WDG_ERR_UNSUPPORTED, "wdg_waveholtz_create: not available on a domain of a decomposed mesh");
        *out = nullptr;
        wdg_waveholtz *h = new wdg_waveholtz;
        h->w = w;
        h->omega = omega;
        // WaveHoltz::WaveHoltz (source/WaveHoltz.cpp:24-29)
        h->T = 2.0 * M_PI / omega;
        const double p = w->n;
        h->dt = 0.5 * w->min_h / (p * p);
        h->nt = (int)std::ceil(h->T / h->dt);
        h->dt = h->T / h->nt;
        h->c0 = 0.5 * h->dt * K(h, 0.0);
        // filter weights at the accumulated step times, as WaveHoltz::S / pi0 form them
        h->c_filter.resize(h->nt);
        double t = 0.0;
        for (int it = 1; it <= h->nt; ++it)
        {
            t += h->dt;
            h->c_filter[it - 1] = ((it == h->nt) ? 0.5 : 1.0) * h->dt * K(h, t);
        }
        int dev_prev = 0;
        cudaGetDevice(&dev_prev);
        cudaSetDevice(w->device);
        // state buffers must exist before a period is captured into a graph
        int s = ensure_states(w);
        cudaError_t e = (s == WDG_OK) ? cudaStreamCreateWithFlags(&h->cs, cudaStreamNonBlocking) : cudaSuccess;
        if (e == cudaSuccess)
            e = cudaEventCreateWithFlags(&h->ev_in, cudaEventDisableTiming);
        if (e == cudaSuccess)
            e = cudaEventCreateWithFlags(&h->ev_out, cudaEventDisableTiming);
        const size_t nd = (size_t)w->ndof;
        if (e == cudaSuccess)
            e = cudaMalloc(&h->d_W, sizeof(double) * nd + 64);
        if (e == cudaSuccess)
            e = cudaMalloc(&h->d_acc, sizeof(double) * nd + 64);
        if (e == cudaSuccess)
            e = cudaMalloc(&h->d_pi0, sizeof(double) * nd + 64);
        if (e == cudaSuccess)
            e = cudaMalloc(&h->d_F, w->real_size() * nd + 64);
        if (s == WDG_OK && e != cudaSuccess)
            s = cuda_fail(e, "wdg_waveholtz_create");
        cudaSetDevice(dev_prev);
        if (s != WDG_OK)
        {
            const std::string msg = wdg_last_error();
            wdg_waveholtz_destroy(h);
            return fail(s, msg);
        }
        *out = h;
        return WDG_OK;
    }

    // WaveHoltz(omega, mesh, basis, bc, approx_quad = false): the same iteration on the exact-
    // quadrature operators of q (which must outlive the handle)
    int wdg_waveholtz_create_exact(wdg_waveq *q, double omega, wdg_waveholtz **out)
    {
        if (!q || !out)
            return fail(WDG_ERR_ARG, "wdg_waveholtz_create_exact: null argument");
        *out = nullptr;
        wdg_wave *w = nullptr;
        WDG_TRY(wdg_waveq_wave(q, &w));
        WDG_TRY(waveq_prepare(q));
        wdg_waveholtz *h = nullptr;
        WDG_TRY(wdg_waveholtz_create(w, omega, &h));
        h->q = q;
        *out = h;
        return WDG_OK;
    }

    void wdg_waveholtz_destroy(wdg_waveholtz *h)
    {
        if (!h)
            return;
        int dev_prev = 0;
        cudaGetDevice(&dev_prev);
        cudaSetDevice(h->w->device);
        if (h->cs)
            cudaStreamSynchronize(h->cs);
        if (h->g_S)
            cudaGraphExecDestroy(h->g_S);
        if (h->g_pi0)
            cudaGraphExecDestroy(h->g_pi0);
        for (void *p : {(void *)h->d_W, (void *)h->d_acc, (void *)h->d_pi0, h->d_F})
            if (p)
                cudaFree(p);
        if (h->ev_in)
            cudaEventDestroy(h->ev_in);
        if (h->ev_out)
            cudaEventDestroy(h->ev_out);
        if (h->cs)
            cudaStreamDestroy(h->cs);
        cudaSetDevice(dev_prev);
        delete h;
    }

    int wdg_waveholtz_params(const wdg_waveholtz *h, double *T, double *dt, int *nt)
    {
        if (!h)
            return fail(WDG_ERR_ARG, "null WaveHoltz handle");
        if (T) *T = h->T;
        if (dt) *dt = h->dt;
        if (nt) *nt = h->nt;
        return WDG_OK;
    }

    int wdg_waveholtz_pi0(wdg_waveholtz *h, double *wout, const double *F)
    {
        if (!h || !wout || !F)
            return fail(WDG_ERR_ARG, "wdg_waveholtz_pi0: bad arguments");
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(h->w->device);
        int s = on_private_stream(h, [&]() -> int
        {
            WDG_TRY(set_forcing(h, F));
            WDG_TRY(run_period(h, true));
            return copy_in(h, wout, h->d_acc);
        });
        if (s == WDG_OK)
            s = finish_host(h);
        cudaSetDevice(prev);
        return s;
    }

    int wdg_waveholtz_S(wdg_waveholtz *h, double *W)
    {
        if (!h || !W)
            return fail(WDG_ERR_ARG, "wdg_waveholtz_S: bad arguments");
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(h->w->device);
        int s = on_private_stream(h, [&]() -> int
        {
            WDG_TRY(copy_in(h, h->d_W, W));
            WDG_TRY(run_period(h, false));
            return copy_in(h, W, h->d_acc);
        });
        if (s == WDG_OK)
            s = finish_host(h);
        cudaSetDevice(prev);
        return s;
    }

    int wdg_waveholtz_postprocess(wdg_waveholtz *h, double *H, const double *W)
    {
        if (!h || !H || !W)
            return fail(WDG_ERR_ARG, "wdg_waveholtz_postprocess: bad arguments");
        wdg_wave *w = h->w;
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(w->device);
        int s = on_private_stream(h, [&]() -> int
        {
            WDG_TRY(copy_in(h, h->d_W, W));
            // P = M^{-1}(A + B) W in FP64 (the postprocess is a single RHS)
            if (h->q)
                WDG_TRY(waveq_rhs_device(h->q, h->d_W, h->d_acc));
            StageArgs<double> a{};
            a.u = h->d_W;
            a.out = h->d_acc;
            a.corners = w->d_corners;
            a.fbase = w->d_fbase;
            a.fcode = w->d_fcode;
            a.nel = w->nel;
            a.tile = default_tile(w->n, false, kDefaultStages);
            a.stages = kDefaultStages;
            a.family = w->family;
            a.flags = F_ALL;
            a.use_tma = 1;
            a.err = w->d_err;
            if (!h->q)
                WDG_CUDA(launch_stage<double>(w->n, false, a, 0, h->cs));
            bool dev = false;
            WDG_TRY(is_device_ptr(w, H, dev));
            const long long npts = w->ndof / 3;
            if (dev)
            {
                WDG_CUDA(launch_wh_post(h->d_W, h->d_acc, h->omega, npts, H, h->cs));
                return WDG_OK;
            }
            WDG_TRY(ensure_stage(w, 1));
            WDG_CUDA(launch_wh_post(h->d_W, h->d_acc, h->omega, npts, w->d_stage[1], h->cs));
            WDG_CUDA(cudaMemcpyAsync(H, w->d_stage[1], sizeof(double) * 2 * npts, cudaMemcpyDeviceToHost, h->cs));
            return WDG_OK;
        });
        if (s == WDG_OK)
            s = finish_host(h);
        cudaSetDevice(prev);
        return s;
    }

    int wdg_waveholtz_solve(wdg_waveholtz *h, const double *F, double tol, int maxit, double *W, int *iters,
                            double *residual)
    {
        if (!h || !F || !W || !iters || !residual || maxit < 0)
            return fail(WDG_ERR_ARG, "wdg_waveholtz_solve: bad arguments");
        wdg_wave *w = h->w;
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(w->device);
        *iters = 0;
        *residual = INFINITY;
        int s = on_private_stream(h, [&]() -> int
        {
            // pi0 and its norm (examples/waveholtz2d.cpp:137-141)
            WDG_TRY(set_forcing(h, F));
            WDG_TRY(run_period(h, true));
            WDG_CUDA(cudaMemcpyAsync(h->d_pi0, h->d_acc, sizeof(double) * w->ndof, cudaMemcpyDeviceToDevice, h->cs));
            WDG_CUDA(launch_sumsq<double>(h->d_pi0, nullptr, w->ndof, w->d_scratch, w->d_result, h->cs));
            WDG_CUDA(cudaMemcpyAsync(w->h_result, w->d_result, sizeof(double), cudaMemcpyDeviceToHost, h->cs));
            WDG_TRY(finish_host(h));
            h->pi0_norm = std::sqrt(w->h_result[0]);
            const double pz = (h->pi0_norm > 0) ? h->pi0_norm : 1.0;
            WDG_TRY(copy_in(h, h->d_W, W));
            // fixed-point loop (examples/waveholtz2d.cpp:165-185)
            for (int it = 1; it <= maxit; ++it)
            {
                WDG_TRY(run_period(h, false));
                WDG_CUDA(launch_wh_update(h->d_W, h->d_acc, h->d_pi0, w->ndof, w->d_scratch, w->d_result, h->cs));
                WDG_CUDA(cudaMemcpyAsync(w->h_result, w->d_result, sizeof(double), cudaMemcpyDeviceToHost, h->cs));
                WDG_TRY(finish_host(h));
                *iters = it;
                *residual = std::sqrt(w->h_result[0]) / pz;
                if (*residual < tol)
                    break;
            }
            return copy_in(h, W, h->d_W);
        });
        if (s == WDG_OK)
            s = finish_host(h);
        cudaSetDevice(prev);
        if (s == WDG_OK && !(*residual < tol))
            return fail(WDG_ERR_NOT_CONVERGED, "WaveHoltz iteration did not reach the tolerance in maxit iterations");
        return s;
    }
}
