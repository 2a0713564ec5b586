// Batched WaveHoltz: per RK stage, one persistent launch per polynomial degree over a work
// list of (solve, chunk) items of the batch's solves of that degree (included by kernels.cu).
//
// Every solve has its own mesh, frequency, period length nt and state; a launch covers the
// solves [s_lo, s_hi) of one degree, whose chunks are listed back to back (items
// it_lo .. it_hi).  A CTA walks items it_lo + blockIdx.x, + G, ... skipping solves that have
// finished, and runs the same producer / consumer pair as the single-solve kernel on each
// item.  Per-solve stage scalars come from the solve's own step counter k:  forcing scale
// -sin(omega (k + c_s) dt) / omega, filter weight dt K((k + 1) dt) (halved on the last step
// of a period).
//
// Each iteration is one forced period from the current iterate W (by linearity of the
// scheme this equals S W + pi0 of the reference's loop): the state starts at W, the
// filter at 0.5 dt K(0) W.  On the last stage of a period the consumer epilogue
// finishes the filter, writes W' and restarts state and filter from it, and leaves
// per-chunk partial sums of (W' - W)^2 and W'^2; whb_step_end_kernel reduces them in a
// fixed order and updates the solve's residual and status.  A warm-started solve first
// runs one forced period from zero only to obtain |pi0|, the residual's scale.
namespace wdg
{
    __constant__ double c_rk4a[5], c_rk4b[5], c_rk4c[5];

    // shared memory: [2 S mbarriers | pad 128][per solve: forcing scale, filter weight (FP64)]
    //                [x (n), w (n)][per solve: k, phase, active][first item per solve, + end]
    //                [pad 128][S slots][consumer scratch]
    __host__ __device__ inline int whb_slots_offset(int n, int real_size)
    {
        return (128 + 16 * kMaxBatch + 2 * n * real_size + 3 * kMaxBatch * 4 + 4 * (kMaxBatch + 1) + 127) & ~127;
    }

    // CTAs per SM the registers are budgeted for: FP32 stages of degree <= 4 fit three
    // (at most 65536 / (3 x 160) registers a thread, no spills); the rest keep two
    template <int N, typename Real>
    constexpr int whb_min_blocks() { return (sizeof(Real) == 4 && N <= 5) ? 3 : 2; }

    // LAST: the fifth RK stage (filter, period ends); the other four compile without that code
    template <int N, typename Real, bool LAST>
    __global__ void __launch_bounds__(kWsThreads, whb_min_blocks<N, Real>()) whb_stage_kernel(const __grid_constant__ WhbArgs<Real> a)
    {
        const int S = a.ring, G = gridDim.x, st = a.stage;
        extern __shared__ __align__(128) unsigned char smem[];
        uint64_t *full = reinterpret_cast<uint64_t *>(smem);
        uint64_t *done = full + S;
        double *sc = reinterpret_cast<double *>(smem + 128);                // per solve: fscale, acc_c
        Real *xt = reinterpret_cast<Real *>(smem + 128 + 16 * kMaxBatch); // GLL nodes, then weights
        Real *wt = xt + N;
        int *act = reinterpret_cast<int *>(smem + 128 + 16 * kMaxBatch + 2 * N * sizeof(Real)); // k, phase, active
        int *it0 = act + 3 * kMaxBatch; // first item of each solve; it0[s_hi] = it_hi
        unsigned char *slots = smem + whb_slots_offset(N, (int)sizeof(Real));
        unsigned char *scratch = slots + S * a.slot_bytes;

        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        if (threadIdx.x == 0)
        {
            for (int q = 0; q < S; ++q)
            {
                mbar_init(&full[q], 1 + 32); // the bulk-copy arrive + one cp.async arrive per producer lane
                mbar_init(&done[q], kWsConsumers);
            }
            fence_mbar_init();
        }
        for (int q = threadIdx.x; q < 2 * N; q += blockDim.x)
            xt[q] = (q < N) ? Tab<Real>::x(N, q) : Tab<Real>::w(N, q - N);
        for (int q = a.s_lo + (int)threadIdx.x; q < a.s_hi; q += blockDim.x)
        {
            const int k = a.state[q].k;
            act[3 * q] = k;
            act[3 * q + 1] = a.state[q].phase;
            act[3 * q + 2] = a.state[q].active;
            // the solve's stage scalars, once per CTA rather than once per item:
            // forcing F s(t), s(t) = -sin(omega t) / omega at the stage time (WaveHoltz.cpp:57-68);
            // filter weight of the step's end dt K(t), halved on the period's last step
            const WhbSolve<Real> &P = a.s[q];
            const double ts = (k + c_rk4c[st]) * P.dt;
            sc[2 * q] = -sin(P.omega * ts) / P.omega;
            const double t1 = (k + 1) * P.dt;
            sc[2 * q + 1] = LAST ? ((k + 1 == P.nt) ? 0.5 : 1.0) * P.dt * (P.omega / M_PI * (cos(P.omega * t1) - 0.25))
                                 : 0.0;
            it0[q] = P.item0;
        }
        if (threadIdx.x == 0)
            it0[a.s_hi] = a.it_hi;
        __syncthreads();

        // item -> solve: the launch's solves' items are contiguous and ascending.  A thread's
        // successive items mostly fall in the solve of its previous one: try that first.
        int hint = a.s_lo;
        auto solve_of = [&](int item)
        {
            if (item >= it0[hint] && item < it0[hint + 1])
                return hint;
            int lo = a.s_lo, hi = a.s_hi - 1;
            while (lo < hi)
            {
                const int mid = (lo + hi + 1) >> 1;
                if (it0[mid] <= item)
                    lo = mid;
                else
                    hi = mid - 1;
            }
            hint = lo;
            return lo;
        };
        // the next item of this CTA at or after k whose solve is still running; producer and
        // consumers walk the same sequence, so their ring positions agree
        auto advance = [&](int k)
        {
            while (k < a.it_hi && !act[3 * solve_of(k) + 2])
                k += G;
            return k;
        };
        WsChunk<Real> c{};
        auto build = [&](int item)
        {
            const int si = solve_of(item);
            const WhbSolve<Real> &P = a.s[si];
            const int ci = item - it0[si];
            const int k = act[3 * si], phase = act[3 * si + 1];
            // the RK4 buffer rotation A -> B -> C -> B -> C -> A
            const int src = (st == 0) ? 0 : (st % 2 == 1) ? 1 : 2;
            const int dst = LAST ? 0 : (st % 2 == 0) ? 1 : 2;
            c.u = P.buf[src];
            c.out = P.buf[dst];
            c.du = P.du;
            c.F = P.F;
            c.acc = P.acc;
            c.corners = P.corners;
            c.fbase = P.fbase;
            c.fcode = P.fcode;
            c.err = a.err;
            c.nel = P.nel;
            c.chunk = P.chunk;
            c.el0 = ci * P.chunk;
            c.ne = min(P.chunk, P.nel - c.el0);
            c.flags = F_ALL | F_FORCE | (st > 0 ? F_READ_DU : 0) | (LAST ? F_FILTER : 0);
            c.rk_a = (Real)c_rk4a[st];
            c.rk_b = (Real)c_rk4b[st];
            c.dt = (Real)P.dt;
            c.fscale = (Real)sc[2 * si];
            c.acc_c = sc[2 * si + 1];
            c.pend = (LAST && k + 1 == P.nt) ? (phase == 0 ? 2 : 1) : 0;
            c.W = P.W;
            c.c0 = P.c0;
            c.part = P.part + (size_t)ci * kWsConsumers * 2;
        };

        const int first = a.it_lo + (int)blockIdx.x;
        if (warp == kWsConsumers)
        {
            // ------------------------------------------------------------ producer
            int kl = advance(first), nl = 0; // next item to load, loads issued
            for (; nl < S && kl < a.it_hi; ++nl)
            {
                build(kl);
                ws_load<N, Real, true>(c, slots + (nl % S) * a.slot_bytes, &full[nl % S], lane);
                kl = advance(kl + G);
            }
            int ks = advance(first), m = 0; // next item to store, stores done
            bool ok = true;
            for (; ks < a.it_hi; ++m)
            {
                const int q = m % S;
                if (!__all_sync(0xffffffffu, mbar_wait(&done[q], (m / S) & 1)))
                {
                    ok = false;
                    break;
                }
                build(ks);
                ws_store<N, Real, true>(c, slots + q * a.slot_bytes, lane);
                ks = advance(ks + G);
                if (kl < a.it_hi)
                {
                    if (lane == 0)
                        bulk_wait_read(); // the store above has read the slot
                    __syncwarp();
                    build(kl);
                    ws_load<N, Real, true>(c, slots + q * a.slot_bytes, &full[q], lane);
                    kl = advance(kl + G);
                    ++nl;
                }
            }
            if (!ok && lane == 0)
            {
                // a consumer gave up: record it, let the loads already issued land, leave
                atomicOr(a.err, 1u);
                for (int r = m; r < nl; ++r)
                    mbar_wait(&full[r % S], (r / S) & 1);
            }
            if (lane == 0)
                bulk_wait_all();
            return;
        }

        // ---------------------------------------------------------------- consumers
        Real *Rc = reinterpret_cast<Real *>(scratch + warp * a.warp_scratch);
        int kc = advance(first);
        for (int m = 0; kc < a.it_hi; ++m)
        {
            const int q = m % S;
            if (!__all_sync(0xffffffffu, mbar_wait(&full[q], (m / S) & 1)))
            {
                if (lane == 0)
                    atomicOr(a.err, 1u);
                break;
            }
            build(kc);
            ws_consume<N, Real, true, LAST>(c, slots + q * a.slot_bytes, Rc, xt, wt, warp, lane);
            // results are in the slot: hand them to the async proxy, then release the slot
            fence_async_smem();
            __syncwarp();
            if (lane == 0)
                mbar_arrive(&done[q]);
            kc = advance(kc + G);
        }
    }

    // After the fifth stage of every step: advance each running solve's step counter; at the
    // end of a period reduce its partial sums in a fixed order and update residual and status
    // (examples/waveholtz2d.cpp:165-185: ||W - W_prev|| / ||pi0|| against tol, maxit).
    __global__ void whb_step_end_kernel(WhbState *state, int nsolves)
    {
        const int s = blockIdx.x;
        if (s >= nsolves)
            return;
        WhbState &P = state[s];
        if (!P.active)
            return;
        const int k = P.k + 1;
        if (k < P.nt)
        {
            __syncthreads();
            if (threadIdx.x == 0)
                P.k = k;
            return;
        }
        __shared__ double sd[256], sn[256];
        double d = 0.0, nrm = 0.0;
        for (int i = threadIdx.x; i < P.nparts; i += blockDim.x)
        {
            d += P.part[2 * i];
            nrm += P.part[2 * i + 1];
        }
        sd[threadIdx.x] = d;
        sn[threadIdx.x] = nrm;
        __syncthreads();
        for (int h = blockDim.x / 2; h > 0; h >>= 1)
        {
            if ((int)threadIdx.x < h)
            {
                sd[threadIdx.x] += sd[threadIdx.x + h];
                sn[threadIdx.x] += sn[threadIdx.x + h];
            }
            __syncthreads();
        }
        if (threadIdx.x != 0)
            return;
        P.k = 0;
        if (P.phase == 0)
        {
            P.pi0sq = sn[0];
            P.phase = 1;
            return;
        }
        if (P.iter == 0 && P.zero_start)
            P.pi0sq = sn[0]; // the first period from zero is pi0 itself
        const double scale = P.pi0sq > 0.0 ? sqrt(P.pi0sq) : 1.0;
        P.residual = sqrt(sd[0]) / scale;
        P.iter += 1;
        if (P.residual < P.best)
        {
            P.best = P.residual;
            P.stall = 0;
        }
        else
            P.stall += 1;
        if (P.residual < P.tol)
        {
            P.active = 0;
            P.status = 0;
        }
        else if (P.iter >= P.maxit)
        {
            P.active = 0;
            P.status = 1;
        }
        else if (P.stall_limit > 0 && P.stall >= P.stall_limit)
        {
            P.active = 0;
            P.status = 2;
        }
    }

    int whb_smem_bytes(int n, int slot_bytes, int warp_scratch, int ring, bool fp32)
    {
        return whb_slots_offset(n, fp32 ? 4 : 8) + ring * slot_bytes + kWsConsumers * warp_scratch;
    }

#define WDG_WHB_CASES(X) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9)
    template <typename K>
    cudaError_t whb_occupancy_of(K kern, size_t smem, int *per_sm)
    {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, kern, kWsThreads, smem);
        return e;
    }
    template <typename Real>
    cudaError_t whb_occupancy(int n, bool last, size_t smem, int *grid)
    {
        int dev = 0, per_sm = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaError_t e = cudaErrorInvalidValue;
        switch (n)
        {
#define WDG_X(NV)                                                                                           \
    case NV:                                                                                                \
        if (last)                                                                                           \
            e = whb_occupancy_of(whb_stage_kernel<NV, Real, true>, smem, &per_sm);                          \
        else                                                                                                \
            e = whb_occupancy_of(whb_stage_kernel<NV, Real, false>, smem, &per_sm);                         \
        break;
            WDG_WHB_CASES(WDG_X)
#undef WDG_X
        default:
            break;
        }
        if (e == cudaSuccess)
            e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        *grid = std::max(1, per_sm) * sms;
        return e;
    }
    template <typename Real>
    cudaError_t launch_whb_stage(const WhbArgs<Real> &a, int n, int grid, size_t smem, cudaStream_t s)
    {
        const bool last = a.stage == 4;
        switch (n)
        {
#define WDG_X(NV)                                                                \
    case NV:                                                                     \
        if (last)                                                                \
            whb_stage_kernel<NV, Real, true><<<grid, kWsThreads, smem, s>>>(a);  \
        else                                                                     \
            whb_stage_kernel<NV, Real, false><<<grid, kWsThreads, smem, s>>>(a); \
        break;
            WDG_WHB_CASES(WDG_X)
#undef WDG_X
        default:
            return cudaErrorInvalidValue;
        }
        return cudaGetLastError();
    }
#undef WDG_WHB_CASES
    cudaError_t launch_whb_step_end(WhbState *state, int nsolves, cudaStream_t s)
    {
        whb_step_end_kernel<<<nsolves, 256, 0, s>>>(state, nsolves);
        return cudaGetLastError();
    }
    int upload_rk4_tables(int device)
    {
        static std::mutex mu;
        static uint64_t done = 0;
        std::lock_guard<std::mutex> lock(mu);
        if (device < 0 || device >= 64)
            return fail(WDG_ERR_ARG, "device ordinal out of range");
        if (done & (1ull << device))
            return WDG_OK;
        WDG_CUDA(cudaMemcpyToSymbol(c_rk4a, rk4a, sizeof(double) * 5));
        WDG_CUDA(cudaMemcpyToSymbol(c_rk4b, rk4b, sizeof(double) * 5));
        WDG_CUDA(cudaMemcpyToSymbol(c_rk4c, rk4c, sizeof(double) * 5));
        done |= (1ull << device);
        return WDG_OK;
    }
    template cudaError_t launch_whb_stage<double>(const WhbArgs<double> &, int, int, size_t, cudaStream_t);
    template cudaError_t launch_whb_stage<float>(const WhbArgs<float> &, int, int, size_t, cudaStream_t);
    template cudaError_t whb_occupancy<double>(int, bool, size_t, int *);
    template cudaError_t whb_occupancy<float>(int, bool, size_t, int *);
} // namespace wdg
