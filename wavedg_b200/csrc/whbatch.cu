// C-ABI: batched WaveHoltz -- many independent Helmholtz solves (each its own mesh,
// degree, frequency and forcing) advanced together: per RK stage one persistent launch
// per polynomial degree over a work list of (solve, chunk) items, the degrees' launches
// running concurrently on forked streams.  Blocks of steps are captured once
// into a CUDA graph on a private stream and replayed until every solve has finished;
// each solve's step counter, period ends, residual and status live on the device
// (WhbState), so a replay needs no host decision.  Iteration and residual follow the
// reference's fixed-point loop (examples/waveholtz2d.cpp:165-185; WaveHoltz.cpp:55-121).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "wave_impl.hpp"

using namespace wdg;

// the solves of one degree: one launch per RK stage.  The filter stage (the fifth) stages the
// FP64 filter accumulator through its slots as well; the other four stop their slots before
// it, so FP32 launches of those stages fit more CTAs per SM (`_nf`: no filter)
struct WhbGroup
{
    int n = 0, s_lo = 0, s_hi = 0, it_lo = 0, it_hi = 0;
    int slot_bytes = 0, warp_scratch = 0, grid = 0;
    int slot_nf = 0, grid_nf = 0;
    size_t smem = 0, smem_nf = 0;
    cudaStream_t st = nullptr; // forked stream of the captured graph (groups run concurrently)
    cudaEvent_t done = nullptr;
};

struct wdg_whbatch
{
    int device = 0, precision = WDG_FP64, n = 0;
    // solves are held sorted by degree; perm[i] is the caller's index of internal solve i
    std::vector<int> perm;
    std::vector<WhbGroup> groups;
    cudaEvent_t fork = nullptr;
    std::vector<wdg_wave *> w;
    std::vector<double> omega, T, dt, c0;
    std::vector<int> nt, nchunks, item0, chunk;
    std::vector<size_t> part_cap;
    int nitems = 0, rounds = 1, ring = 2;
    cudaStream_t cs = nullptr;
    std::vector<double *> d_W, d_acc, d_part;
    std::vector<void *> d_F;
    WhbState *d_state = nullptr;
    WhbState *h_state = nullptr; // pinned
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
};

namespace
{
    constexpr int kGraphSteps = 32; // RK4 steps per captured graph

    double K(double omega, double t) { return omega / M_PI * (std::cos(omega * t) - 0.25); }

    struct Dev
    {
        int prev = -1;
        explicit Dev(int d)
        {
            cudaGetDevice(&prev);
            cudaSetDevice(d);
        }
        ~Dev()
        {
            if (prev >= 0)
                cudaSetDevice(prev);
        }
    };

    // launch shape: chunk = rounds x unit(n) per solve; one launch per degree group
    int shape(wdg_whbatch *b, int rounds, int ring)
    {
        const bool fp32 = b->precision == WDG_FP32;
        std::vector<int> chunk(b->n), nch(b->n), it0(b->n);
        int items = 0;
        for (int s = 0; s < b->n; ++s)
        {
            chunk[s] = rounds * ws_chunk_unit(b->w[s]->n);
            nch[s] = (b->w[s]->nel + chunk[s] - 1) / chunk[s];
            it0[s] = items;
            items += nch[s];
        }
        std::vector<WhbGroup> gs = b->groups;
        for (WhbGroup &g : gs)
        {
            const int ch = rounds * ws_chunk_unit(g.n);
            g.slot_bytes = ws_slot_bytes(g.n, fp32, ch, true, true);
            g.slot_nf = ws_slot_bytes(g.n, fp32, ch, true, false);
            g.warp_scratch = ws_warp_scratch_bytes(g.n, fp32);
            g.smem = (size_t)whb_smem_bytes(g.n, g.slot_bytes, g.warp_scratch, ring, fp32);
            g.smem_nf = (size_t)whb_smem_bytes(g.n, g.slot_nf, g.warp_scratch, ring, fp32);
            if (g.smem > 227 * 1024)
                return fail(WDG_ERR_ARG, "batched WaveHoltz: chunk x ring too large for shared memory");
            g.it_lo = it0[g.s_lo];
            g.it_hi = it0[g.s_hi - 1] + nch[g.s_hi - 1];
            int grid = 0, grid_nf = 0;
            WDG_CUDA(fp32 ? whb_occupancy<float>(g.n, true, g.smem, &grid)
                          : whb_occupancy<double>(g.n, true, g.smem, &grid));
            WDG_CUDA(fp32 ? whb_occupancy<float>(g.n, false, g.smem_nf, &grid_nf)
                          : whb_occupancy<double>(g.n, false, g.smem_nf, &grid_nf));
            g.grid = std::max(1, std::min(grid, g.it_hi - g.it_lo));
            g.grid_nf = std::max(1, std::min(grid_nf, g.it_hi - g.it_lo));
        }
        // partial sums: nchunks x consumer warps x 2 per solve, grown as needed
        for (int s = 0; s < b->n; ++s)
        {
            const size_t need = (size_t)nch[s] * kWsConsumers * 2;
            if (need > b->part_cap[s])
            {
                if (b->d_part[s])
                    cudaFree(b->d_part[s]);
                b->d_part[s] = nullptr;
                b->part_cap[s] = 0;
                WDG_CUDA(cudaMalloc(&b->d_part[s], sizeof(double) * need));
                b->part_cap[s] = need;
            }
        }
        b->groups = gs;
        b->chunk = chunk;
        b->nchunks = nch;
        b->item0 = it0;
        b->nitems = items;
        b->rounds = rounds;
        b->ring = ring;
        if (b->graph)
        {
            cudaGraphExecDestroy(b->graph);
            b->graph = nullptr;
        }
        return WDG_OK;
    }

    template <typename Real>
    WhbArgs<Real> make_args(const wdg_whbatch *b, const WhbGroup &g, int stage)
    {
        WhbArgs<Real> a{};
        a.nsolves = b->n;
        a.s_lo = g.s_lo;
        a.s_hi = g.s_hi;
        a.it_lo = g.it_lo;
        a.it_hi = g.it_hi;
        a.stage = stage;
        a.ring = b->ring;
        a.slot_bytes = stage == 4 ? g.slot_bytes : g.slot_nf;
        a.warp_scratch = g.warp_scratch;
        a.state = b->d_state;
        a.err = b->w[0]->d_err;
        for (int s = 0; s < b->n; ++s)
        {
            const wdg_wave *w = b->w[s];
            WhbSolve<Real> &P = a.s[s];
            for (int k = 0; k < 3; ++k)
                P.buf[k] = static_cast<Real *>(w->d_state[k]);
            P.du = static_cast<Real *>(w->d_du);
            P.F = static_cast<const Real *>(b->d_F[s]);
            P.acc = b->d_acc[s];
            P.W = b->d_W[s];
            P.part = b->d_part[s];
            P.corners = w->d_corners;
            P.fbase = w->d_fbase;
            P.fcode = w->d_fcode;
            P.nel = w->nel;
            P.n = w->n;
            P.chunk = b->chunk[s];
            P.item0 = b->item0[s];
            P.nt = b->nt[s];
            P.dt = b->dt[s];
            P.omega = b->omega[s];
            P.c0 = b->c0[s];
        }
        return a;
    }

    template <typename Real>
    cudaError_t launch_group(const wdg_whbatch *b, const WhbGroup &g, int stage, cudaStream_t st)
    {
        const WhbArgs<Real> a = make_args<Real>(b, g, stage);
        return stage == 4 ? launch_whb_stage<Real>(a, g.n, g.grid, g.smem, st)
                          : launch_whb_stage<Real>(a, g.n, g.grid_nf, g.smem_nf, st);
    }

    // kGraphSteps steps (per stage one launch per degree group, the groups on forked streams,
    // then the step-end update) as one graph
    int record(wdg_whbatch *b)
    {
        const bool fp32 = b->precision == WDG_FP32;
        const bool fork = b->groups.size() > 1;
        WDG_CUDA(cudaStreamBeginCapture(b->cs, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = cudaSuccess;
        for (int k = 0; k < kGraphSteps && e == cudaSuccess; ++k)
        {
            for (int stg = 0; stg < 5 && e == cudaSuccess; ++stg)
            {
                if (fork)
                    e = cudaEventRecord(b->fork, b->cs);
                for (const WhbGroup &g : b->groups)
                {
                    cudaStream_t st = fork ? g.st : b->cs;
                    if (e == cudaSuccess && fork)
                        e = cudaStreamWaitEvent(st, b->fork, 0);
                    if (e == cudaSuccess)
                        e = fp32 ? launch_group<float>(b, g, stg, st) : launch_group<double>(b, g, stg, st);
                    if (e == cudaSuccess && fork)
                        e = cudaEventRecord(g.done, st);
                }
                for (const WhbGroup &g : b->groups)
                    if (e == cudaSuccess && fork)
                        e = cudaStreamWaitEvent(b->cs, g.done, 0);
            }
            if (e == cudaSuccess)
                e = launch_whb_step_end(b->d_state, b->n, b->cs);
        }
        cudaGraph_t gph = nullptr;
        const cudaError_t e2 = cudaStreamEndCapture(b->cs, &gph);
        if (e != cudaSuccess || e2 != cudaSuccess)
        {
            if (gph)
                cudaGraphDestroy(gph);
            return cuda_fail(e != cudaSuccess ? e : e2, "batched WaveHoltz: graph capture");
        }
        e = cudaGraphInstantiate(&b->graph, gph, 0);
        cudaGraphDestroy(gph);
        if (e != cudaSuccess)
            return cuda_fail(e, "cudaGraphInstantiate");
        b->graph_steps = kGraphSteps;
        return WDG_OK;
    }

    // state and filter of solve s set to zero (the start of every solve)
    int zero_period(wdg_whbatch *b, int s)
    {
        wdg_wave *w = b->w[s];
        WDG_CUDA(cudaMemsetAsync(w->d_state[0], 0, w->real_size() * (size_t)w->ndof, b->cs));
        WDG_CUDA(cudaMemsetAsync(b->d_acc[s], 0, sizeof(double) * (size_t)w->ndof, b->cs));
        return WDG_OK;
    }

    // order the private stream after every solve handle's stream, so inputs the caller wrote
    // there (forcing, warm starts) are complete before the batch reads them
    int after_callers(wdg_whbatch *b)
    {
        std::vector<cudaStream_t> seen;
        for (const wdg_wave *w : b->w)
        {
            if (std::find(seen.begin(), seen.end(), w->stream) != seen.end())
                continue;
            seen.push_back(w->stream);
            WDG_CUDA(cudaEventRecord(b->fork, w->stream));
            WDG_CUDA(cudaStreamWaitEvent(b->cs, b->fork, 0));
        }
        return WDG_OK;
    }

    // known_pi0sq > 0 (warm starts only): |pi0|^2 given, so the solve skips its pi0 period
    WhbState fresh_state(const wdg_whbatch *b, int s, bool warm, double tol, int maxit, int stall_limit,
                         double known_pi0sq = 0.0)
    {
        WhbState S{};
        S.k = 0;
        S.phase = (warm && !(known_pi0sq > 0.0)) ? 0 : 1;
        S.pi0sq = warm ? known_pi0sq : 0.0;
        S.active = 1;
        S.zero_start = warm ? 0 : 1;
        S.nt = b->nt[s];
        S.nparts = b->nchunks[s] * kWsConsumers;
        S.maxit = maxit;
        S.stall_limit = stall_limit;
        S.status = -1;
        S.residual = INFINITY;
        S.best = INFINITY;
        S.tol = tol;
        S.part = b->d_part[s];
        return S;
    }
} // namespace

extern "C"
{
    int wdg_whbatch_create(int n_solves, wdg_wave *const *waves, const double *omegas, wdg_whbatch **out)
    {
        if (!out || !waves || !omegas || n_solves < 1 || n_solves > kMaxBatch)
            return fail(WDG_ERR_ARG, "wdg_whbatch_create: 1..64 solves, each a discretisation and a frequency");
        *out = nullptr;
        for (int s = 0; s < n_solves; ++s)
        {
            if (!waves[s] || !(omegas[s] > 0.0))
                return fail(WDG_ERR_ARG, "wdg_whbatch_create: every solve needs a discretisation and omega > 0");
            if (waves[s]->device != waves[0]->device || waves[s]->precision != waves[0]->precision)
                return fail(WDG_ERR_ARG, "wdg_whbatch_create: all solves must share the device and the precision");
            for (int r = 0; r < s; ++r)
                if (waves[r] == waves[s])
                    return fail(WDG_ERR_ARG, "wdg_whbatch_create: a discretisation may appear once per batch");
        }
        wdg_whbatch *b = new wdg_whbatch;
        b->device = waves[0]->device;
        b->precision = waves[0]->precision;
        b->n = n_solves;
        Dev g(b->device);
        int st = upload_rk4_tables(b->device);
        b->d_W.assign(n_solves, nullptr);
        b->d_acc.assign(n_solves, nullptr);
        b->d_part.assign(n_solves, nullptr);
        b->part_cap.assign(n_solves, 0);
        b->d_F.assign(n_solves, nullptr);
        // internal order: sorted by degree (stable), one group of solves per degree
        b->perm.resize(n_solves);
        for (int s = 0; s < n_solves; ++s)
            b->perm[s] = s;
        std::stable_sort(b->perm.begin(), b->perm.end(), [&](int x, int y) { return waves[x]->n < waves[y]->n; });
        for (int s = 0; s < n_solves; ++s)
        {
            const int nn = waves[b->perm[s]]->n;
            if (b->groups.empty() || b->groups.back().n != nn)
            {
                WhbGroup gr;
                gr.n = nn;
                gr.s_lo = s;
                b->groups.push_back(gr);
            }
            b->groups.back().s_hi = s + 1;
        }
        for (int s = 0; s < n_solves && st == WDG_OK; ++s)
        {
            const int u = b->perm[s];
            wdg_wave *w = waves[u];
            b->w.push_back(w);
            b->omega.push_back(omegas[u]);
            // WaveHoltz::WaveHoltz (source/WaveHoltz.cpp:24-29)
            const double T = 2.0 * M_PI / omegas[u];
            const double p = w->n;
            double dt = 0.5 * w->min_h / (p * p);
            const int nt = (int)std::ceil(T / dt);
            dt = T / nt;
            b->T.push_back(T);
            b->dt.push_back(dt);
            b->nt.push_back(nt);
            b->c0.push_back(0.5 * dt * K(omegas[u], 0.0));
            st = ensure_states(w);
            const size_t nd = (size_t)w->ndof;
            cudaError_t e = cudaSuccess;
            if (st == WDG_OK)
                e = cudaMalloc(&b->d_W[s], sizeof(double) * nd);
            if (st == WDG_OK && e == cudaSuccess)
                e = cudaMalloc(&b->d_acc[s], sizeof(double) * nd);
            if (st == WDG_OK && e == cudaSuccess)
                e = cudaMalloc(&b->d_F[s], w->real_size() * nd);
            if (st == WDG_OK && e != cudaSuccess)
                st = cuda_fail(e, "wdg_whbatch_create");
        }
        cudaError_t e = cudaSuccess;
        if (st == WDG_OK)
            e = cudaStreamCreateWithFlags(&b->cs, cudaStreamNonBlocking);
        if (st == WDG_OK && e == cudaSuccess)
            e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
        for (WhbGroup &gr : b->groups)
        {
            if (st == WDG_OK && e == cudaSuccess)
                e = cudaStreamCreateWithFlags(&gr.st, cudaStreamNonBlocking);
            if (st == WDG_OK && e == cudaSuccess)
                e = cudaEventCreateWithFlags(&gr.done, cudaEventDisableTiming);
        }
        if (st == WDG_OK && e == cudaSuccess)
            e = cudaMalloc(&b->d_state, sizeof(WhbState) * n_solves);
        if (st == WDG_OK && e == cudaSuccess)
            e = cudaMallocHost(&b->h_state, sizeof(WhbState) * n_solves);
        if (st == WDG_OK && e != cudaSuccess)
            st = cuda_fail(e, "wdg_whbatch_create");
        if (st == WDG_OK)
            st = shape(b, 1, 2);
        if (st != WDG_OK)
        {
            const std::string msg = wdg_last_error();
            wdg_whbatch_destroy(b);
            return fail(st, msg);
        }
        *out = b;
        return WDG_OK;
    }

    void wdg_whbatch_destroy(wdg_whbatch *b)
    {
        if (!b)
            return;
        Dev g(b->device);
        if (b->cs)
            cudaStreamSynchronize(b->cs);
        if (b->graph)
            cudaGraphExecDestroy(b->graph);
        for (double *p : b->d_W)
            if (p)
                cudaFree(p);
        for (double *p : b->d_acc)
            if (p)
                cudaFree(p);
        for (double *p : b->d_part)
            if (p)
                cudaFree(p);
        for (void *p : b->d_F)
            if (p)
                cudaFree(p);
        if (b->d_state)
            cudaFree(b->d_state);
        if (b->h_state)
            cudaFreeHost(b->h_state);
        for (WhbGroup &gr : b->groups)
        {
            if (gr.done)
                cudaEventDestroy(gr.done);
            if (gr.st)
                cudaStreamDestroy(gr.st);
        }
        if (b->fork)
            cudaEventDestroy(b->fork);
        if (b->cs)
            cudaStreamDestroy(b->cs);
        delete b;
    }

    int wdg_whbatch_params(const wdg_whbatch *b, int solve, double *T, double *dt, int *nt)
    {
        if (!b || solve < 0 || solve >= b->n)
            return fail(WDG_ERR_ARG, "wdg_whbatch_params: bad arguments");
        const int i = (int)(std::find(b->perm.begin(), b->perm.end(), solve) - b->perm.begin());
        if (T) *T = b->T[i];
        if (dt) *dt = b->dt[i];
        if (nt) *nt = b->nt[i];
        return WDG_OK;
    }

    int wdg_whbatch_set_launch(wdg_whbatch *b, int rounds, int ring)
    {
        if (!b || rounds < 1 || rounds > 16 || ring < 2 || ring > 6)
            return fail(WDG_ERR_ARG, "wdg_whbatch_set_launch: rounds 1..16, ring 2..6");
        Dev g(b->device);
        return shape(b, rounds, ring);
    }

    int wdg_whbatch_get_launch(const wdg_whbatch *b, int *rounds, int *ring, int *grid)
    {
        if (!b)
            return fail(WDG_ERR_ARG, "null batch");
        if (rounds) *rounds = b->rounds;
        if (ring) *ring = b->ring;
        if (grid)
        {
            *grid = 0;
            for (const WhbGroup &gr : b->groups)
                *grid += gr.grid_nf;
        }
        return WDG_OK;
    }

    int wdg_whbatch_solve(wdg_whbatch *b, const double *const *F, double tol, int maxit, int stall_limit,
                          double *const *W, const int *warm, double *pi0_norm, int *iters, double *residuals,
                          int *status)
    {
        if (!b || !F || !W || maxit < 1 || stall_limit < 0 || !(tol > 0.0))
            return fail(WDG_ERR_ARG, "wdg_whbatch_solve: bad arguments");
        for (int s = 0; s < b->n; ++s)
            if (!F[s] || !W[s])
                return fail(WDG_ERR_ARG, "wdg_whbatch_solve: every solve needs F and W");
        Dev g(b->device);
        WDG_TRY(after_callers(b));
        for (int s = 0; s < b->n; ++s)
        {
            wdg_wave *w = b->w[s];
            const size_t nd = (size_t)w->ndof;
            // forcing in the stepping precision (d_W serves as the FP64 staging buffer)
            const int u = b->perm[s]; // the caller's index of internal solve s
            WDG_CUDA(cudaMemcpyAsync(b->d_W[s], F[u], sizeof(double) * nd, cudaMemcpyDefault, b->cs));
            if (b->precision == WDG_FP32)
                WDG_CUDA(launch_convert<double, float>(b->d_W[s], static_cast<float *>(b->d_F[s]), (long long)nd,
                                                       b->cs));
            else
                WDG_CUDA(cudaMemcpyAsync(b->d_F[s], b->d_W[s], sizeof(double) * nd, cudaMemcpyDeviceToDevice, b->cs));
            // zero start: fixed-point periods from W = 0 (the first yields pi0); warm start:
            // a pi0 period from zero first (its norm scales the residual), then from W --
            // or, with |pi0| given, straight from W (state W, filter 0.5 dt K(0) W)
            const bool ws = warm && warm[u];
            const double known = (ws && pi0_norm && pi0_norm[u] > 0.0) ? pi0_norm[u] * pi0_norm[u] : 0.0;
            if (ws)
                WDG_CUDA(cudaMemcpyAsync(b->d_W[s], W[u], sizeof(double) * nd, cudaMemcpyDefault, b->cs));
            else
                WDG_CUDA(cudaMemsetAsync(b->d_W[s], 0, sizeof(double) * nd, b->cs));
            if (known > 0.0)
            {
                if (b->precision == WDG_FP32)
                    WDG_CUDA(launch_scale_into<float>(b->d_W[s], static_cast<float *>(w->d_state[0]), b->d_acc[s],
                                                      b->c0[s], (long long)nd, b->cs));
                else
                    WDG_CUDA(launch_scale_into<double>(b->d_W[s], static_cast<double *>(w->d_state[0]),
                                                       b->d_acc[s], b->c0[s], (long long)nd, b->cs));
            }
            else
                WDG_TRY(zero_period(b, s));
            b->h_state[s] = fresh_state(b, s, ws, tol, maxit, stall_limit, known);
        }
        WDG_CUDA(cudaMemcpyAsync(b->d_state, b->h_state, sizeof(WhbState) * b->n, cudaMemcpyHostToDevice, b->cs));
        if (!b->graph)
            WDG_TRY(record(b));
        // replay blocks of steps until no solve is running; bounded by the longest possible
        // run (maxit + 1 periods of the longest period)
        long long limit = 0;
        for (int s = 0; s < b->n; ++s)
            limit = std::max<long long>(limit, (long long)(maxit + 1) * b->nt[s]);
        long long steps = 0;
        bool running = true;
        while (running && steps <= limit + b->graph_steps)
        {
            WDG_CUDA(cudaGraphLaunch(b->graph, b->cs));
            steps += b->graph_steps;
            WDG_CUDA(cudaMemcpyAsync(b->h_state, b->d_state, sizeof(WhbState) * b->n, cudaMemcpyDeviceToHost, b->cs));
            WDG_CUDA(cudaStreamSynchronize(b->cs));
            WDG_TRY(check_device_error(b->w[0]));
            running = false;
            for (int s = 0; s < b->n; ++s)
                running = running || b->h_state[s].active;
        }
        for (int s = 0; s < b->n; ++s)
        {
            const int u = b->perm[s];
            WDG_CUDA(cudaMemcpyAsync(W[u], b->d_W[s], sizeof(double) * b->w[s]->ndof, cudaMemcpyDefault, b->cs));
            if (iters)
                iters[u] = b->h_state[s].iter;
            if (residuals)
                residuals[u] = b->h_state[s].residual;
            if (status)
                status[u] = b->h_state[s].status;
            if (pi0_norm)
                pi0_norm[u] = std::sqrt(std::max(0.0, b->h_state[s].pi0sq));
        }
        WDG_CUDA(cudaStreamSynchronize(b->cs));
        if (running)
            return fail(WDG_ERR_TIMEOUT, "batched WaveHoltz: solves still running past the step limit");
        return WDG_OK;
    }

    // time `steps` batch steps of every (rounds, ring) that fits and keep the fastest
    int wdg_whbatch_autotune(wdg_whbatch *b, int steps, float *best_ms_per_step)
    {
        if (!b || steps < 1)
            return fail(WDG_ERR_ARG, "wdg_whbatch_autotune: bad arguments");
        Dev g(b->device);
        for (int s = 0; s < b->n; ++s)
        {
            WDG_CUDA(cudaMemsetAsync(b->d_F[s], 0, b->w[s]->real_size() * (size_t)b->w[s]->ndof, b->cs));
            WDG_CUDA(cudaMemsetAsync(b->d_W[s], 0, sizeof(double) * (size_t)b->w[s]->ndof, b->cs));
            WDG_TRY(zero_period(b, s));
        }
        cudaEvent_t e0, e1;
        WDG_CUDA(cudaEventCreate(&e0));
        WDG_CUDA(cudaEventCreate(&e1));
        float best = 1e30f;
        int br = b->rounds, bg = b->ring, st = WDG_OK;
        for (int rounds = 1; rounds <= 4 && st == WDG_OK; ++rounds)
            for (int ring = 2; ring <= 4 && st == WDG_OK; ++ring)
            {
                if (shape(b, rounds, ring) != WDG_OK)
                    continue;
                for (int s = 0; s < b->n; ++s)
                {
                    b->h_state[s] = fresh_state(b, s, false, 0.0, 1, 0);
                    b->h_state[s].nt = 1 << 30; // no period ends while timing
                }
                cudaError_t e = cudaMemcpyAsync(b->d_state, b->h_state, sizeof(WhbState) * b->n,
                                                cudaMemcpyHostToDevice, b->cs);
                if (e == cudaSuccess && record(b) != WDG_OK)
                    e = cudaErrorUnknown;
                const int reps = std::max(1, (steps + kGraphSteps - 1) / kGraphSteps);
                if (e == cudaSuccess)
                    e = cudaGraphLaunch(b->graph, b->cs); // warm-up
                if (e == cudaSuccess)
                    e = cudaEventRecord(e0, b->cs);
                for (int r = 0; r < reps && e == cudaSuccess; ++r)
                    e = cudaGraphLaunch(b->graph, b->cs);
                if (e == cudaSuccess)
                    e = cudaEventRecord(e1, b->cs);
                if (e == cudaSuccess)
                    e = cudaEventSynchronize(e1);
                if (e != cudaSuccess)
                {
                    st = cuda_fail(e, "wdg_whbatch_autotune");
                    break;
                }
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                ms /= (float)(reps * kGraphSteps);
                if (ms < best)
                {
                    best = ms;
                    br = rounds;
                    bg = ring;
                }
            }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (st == WDG_OK)
            st = shape(b, br, bg);
        if (st == WDG_OK)
            st = check_device_error(b->w[0]);
        if (best_ms_per_step)
            *best_ms_per_step = best;
        return st;
    }
}
