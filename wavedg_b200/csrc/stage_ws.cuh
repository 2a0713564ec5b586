// Warp-specialised RK stage kernel (included by kernels.cu).
//
// One CTA = one producer warp + kWsConsumers consumer warps, persistent over
// chunks of C consecutive elements (C a multiple of 4, so every chunk of u, du
// and geometry is a whole number of 16-byte units in HBM).
//
//   producer   ring of S chunk slots in shared memory.  For each chunk it
//              waits until the slot is free, loads u, du and the element
//              geometry with cp.async.bulk on the slot's `full` mbarrier, and
//              once every consumer warp has arrived on the slot's `done`
//              mbarrier it stores u' and du' back with cp.async.bulk straight
//              from the slot (the results are written in place).
//   consumers  a warp owns whole elements (EPW of them when an element's n^2
//              nodes fit a warp, else one element with several nodes per
//              lane) and never waits for another warp: contravariant fluxes go
//              to a per-warp scratch, a __syncwarp, then each node lane
//              contracts along both directions; face lanes (one per face node)
//              form the upwind flux into a per-warp face buffer; node lanes
//              add it, apply M^{-1} and the RK update, and write u', du' into
//              the slot.
//
// Neighbour traces are read from the stage's input array in global memory
// (L2) by the face lanes, issued before the volume work so their latency
// overlaps it; the slot copy of u cannot serve them because other warps
// overwrite their elements in place.
//
// Used for RK launches whose arrays are 16-byte aligned; every other launch
// takes the tiled kernel.

namespace wdg
{
    template <int N>
    struct WsShape
    {
        static constexpr int NN = N * N, ND = 3 * NN, NF = 4 * N;
        static constexpr int EPW = (NN <= 32) ? 32 / NN : 1;    // elements per warp-round
        static constexpr int NODES = EPW * NN, NPL = (NODES + 31) / 32; // node slots per lane
        static constexpr int FACES = EPW * NF, FPL = (FACES + 31) / 32; // face slots per lane
    };
    constexpr int kWsConsumers = 8;
    constexpr int kWsThreads = 32 * (kWsConsumers + 1);

    int ws_epw(int n) { return (n * n <= 32) ? 32 / (n * n) : 1; }

    // shared-memory layout (bytes), identical on host and device:
    //   [2 S mbarriers | pad to 128][D (n^2), w (n), x (n) | pad to 128][S slots][consumer scratch]
    //   slot    = u (C, 3 n^2) | du (C, 3 n^2) | corners (C, 8 doubles) | fbase (C, int4) | fcode (C, u32)
    //   scratch = per warp, per element of a round: fluxes [n^2][6], face fluxes [4 n][3]
    struct WsLayout
    {
        int ub, slot, tab, slots, scratch, warp_scratch, total;
    };
    template <typename Real>
    __host__ __device__ inline WsLayout ws_layout(int n, int chunk, int stages)
    {
        WsLayout L;
        const int nn = n * n, epw = (nn <= 32) ? 32 / nn : 1;
        L.ub = chunk * 3 * nn * (int)sizeof(Real);
        L.slot = 2 * L.ub + chunk * 84;
        L.tab = 128;
        L.slots = (L.tab + (nn + 2 * n) * (int)sizeof(Real) + 127) & ~127;
        L.scratch = L.slots + stages * L.slot;
        L.warp_scratch = ((epw * (6 * nn + 12 * n) * (int)sizeof(Real)) + 15) & ~15;
        L.total = L.scratch + kWsConsumers * L.warp_scratch;
        return L;
    }

    __device__ __forceinline__ void mbar_arrive(uint64_t *bar)
    {
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
    }

    template <typename Real>
    struct Vec2;
    template <>
    struct Vec2<double>
    {
        using T = double2;
    };
    template <>
    struct Vec2<float>
    {
        using T = float2;
    };

    template <int N, typename Real, bool EXTRA>
    __global__ void __launch_bounds__(kWsThreads, 3) ws_stage_kernel(const StageArgs<Real> a)
    {
        using Sh = WsShape<N>;
        using R2 = typename Vec2<Real>::T;
        constexpr int NN = Sh::NN, ND = Sh::ND, NF = Sh::NF, EPW = Sh::EPW;
        constexpr int NPL = Sh::NPL, FPL = Sh::FPL;
        const int C = a.chunk, S = a.ring, G = gridDim.x;
        const int flags = a.flags;
        const bool has_du = (flags & F_READ_DU) != 0;
        const int nchunks = (a.nel + C - 1) / C;
        const WsLayout L = ws_layout<Real>(N, C, S);

        extern __shared__ __align__(128) unsigned char smem[];
        uint64_t *full = reinterpret_cast<uint64_t *>(smem);
        uint64_t *done = full + S;
        Real *Dt = reinterpret_cast<Real *>(smem + L.tab); // D[l + N i] = phi_i'(x_l)
        Real *wt = Dt + NN, *xt = wt + N;
        unsigned char *slots = smem + L.slots;

        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        if (threadIdx.x == 0)
        {
            for (int q = 0; q < S; ++q)
            {
                mbar_init(&full[q], 1);
                mbar_init(&done[q], kWsConsumers);
            }
            fence_mbar_init();
        }
        for (int q = threadIdx.x; q < NN + 2 * N; q += blockDim.x)
            Dt[q] = (q < NN) ? Tab<Real>::D(N, q) : (q < NN + N) ? Tab<Real>::w(N, q - NN) : Tab<Real>::x(N, q - NN - N);
        __syncthreads();

        // this CTA's chunks: k_m = blockIdx.x + m G
        const int M = ((int)blockIdx.x < nchunks) ? (nchunks - 1 - (int)blockIdx.x) / G + 1 : 0;
        auto chunk_el0 = [&](int m) { return ((int)blockIdx.x + m * G) * C; };

        if (warp == kWsConsumers)
        {
            // ------------------------------------------------------------ producer
            auto load = [&](int m)
            {
                const int el0 = chunk_el0(m), ne = min(C, a.nel - el0), q = m % S;
                unsigned char *base = slots + q * L.slot;
                if (ne == C)
                {
                    if (lane == 0)
                    {
                        mbar_expect_tx(&full[q], (uint32_t)(L.ub * (has_du ? 2 : 1) + C * 84));
                        bulk_g2s(base, a.u + (size_t)el0 * ND, (uint32_t)L.ub, &full[q]);
                        if (has_du)
                            bulk_g2s(base + L.ub, a.du + (size_t)el0 * ND, (uint32_t)L.ub, &full[q]);
                        unsigned char *g = base + 2 * L.ub;
                        bulk_g2s(g, a.corners + 8 * (size_t)el0, (uint32_t)(64 * C), &full[q]);
                        bulk_g2s(g + 64 * C, a.fbase + el0, (uint32_t)(16 * C), &full[q]);
                        bulk_g2s(g + 80 * C, a.fcode + el0, (uint32_t)(4 * C), &full[q]);
                    }
                }
                else
                {
                    // ragged last chunk: plain copies by the warp, then an ordinary arrive
                    Real *us = reinterpret_cast<Real *>(base), *dus = us + C * ND;
                    for (int i = lane; i < ne * ND; i += 32)
                    {
                        us[i] = a.u[(size_t)el0 * ND + i];
                        if (has_du)
                            dus[i] = a.du[(size_t)el0 * ND + i];
                    }
                    double *cw = reinterpret_cast<double *>(base + 2 * L.ub);
                    for (int i = lane; i < ne * 8; i += 32)
                        cw[i] = a.corners[8 * (size_t)el0 + i];
                    int4 *bw = reinterpret_cast<int4 *>(base + 2 * L.ub + 64 * C);
                    uint32_t *kw = reinterpret_cast<uint32_t *>(base + 2 * L.ub + 80 * C);
                    for (int i = lane; i < ne; i += 32)
                    {
                        bw[i] = a.fbase[el0 + i];
                        kw[i] = a.fcode[el0 + i];
                    }
                    __threadfence_block();
                    __syncwarp();
                    if (lane == 0)
                        mbar_arrive(&full[q]);
                }
            };
            for (int m = 0; m < min(S, M); ++m)
                load(m);
            int m = 0;
            for (; m < M; ++m)
            {
                const int q = m % S, el0 = chunk_el0(m), ne = min(C, a.nel - el0);
                // a warp-uniform verdict, so no lane leaves while others go on
                if (!__all_sync(0xffffffffu, mbar_wait(&done[q], (m / S) & 1)))
                    break;
                unsigned char *base = slots + q * L.slot;
                if (ne == C)
                {
                    if (lane == 0)
                    {
                        bulk_s2g(a.out + (size_t)el0 * ND, base, (uint32_t)L.ub);
                        bulk_s2g(a.du + (size_t)el0 * ND, base + L.ub, (uint32_t)L.ub);
                        bulk_commit();
                    }
                }
                else
                {
                    const Real *us = reinterpret_cast<const Real *>(base), *dus = us + C * ND;
                    for (int i = lane; i < ne * ND; i += 32)
                    {
                        a.out[(size_t)el0 * ND + i] = us[i];
                        a.du[(size_t)el0 * ND + i] = dus[i];
                    }
                }
                if (m + S < M)
                {
                    if (lane == 0)
                        bulk_wait_read(); // the store above has read the slot
                    __syncwarp();
                    load(m + S);
                }
            }
            if (m < M)
            {
                // a consumer gave up: record it, let the loads already issued land, leave
                if (lane == 0)
                {
                    atomicOr(a.err, 1u);
                    for (int r = m; r < min(m + S, M); ++r)
                        mbar_wait(&full[r % S], (r / S) & 1);
                }
            }
            if (lane == 0)
                bulk_wait_all();
            return;
        }

        // ---------------------------------------------------------------- consumers
        const int cw = warp;
        const int R = C / (kWsConsumers * EPW); // warp-rounds per chunk
        Real *X = reinterpret_cast<Real *>(smem + L.scratch + cw * L.warp_scratch); // [EPW][NN][6]
        Real *Fb = X + EPW * NN * 6;                                                  // [EPW][NF][3]

        for (int m = 0; m < M; ++m)
        {
            const int q = m % S, el0 = chunk_el0(m), ne = min(C, a.nel - el0);
            if (!__all_sync(0xffffffffu, mbar_wait(&full[q], (m / S) & 1)))
            {
                if (lane == 0)
                    atomicOr(a.err, 1u);
                break;
            }
            unsigned char *base = slots + q * L.slot;
            Real *us = reinterpret_cast<Real *>(base);
            Real *dus = us + C * ND;
            const double *cs = reinterpret_cast<const double *>(base + 2 * L.ub);
            const int *fbs = reinterpret_cast<const int *>(base + 2 * L.ub + 64 * C);
            const uint32_t *fks = reinterpret_cast<const uint32_t *>(base + 2 * L.ub + 80 * C);

            for (int r = 0; r < R; ++r)
            {
                const int eb = (cw * R + r) * EPW; // first chunk-local element of this round

                // ---- node lanes: metrics, contravariant fluxes (source/Div.cpp:5-53), M^{-1}
                Real minv[NPL];
                Real fv[NPL][3];
                double av[NPL][3];
#pragma unroll
                for (int p = 0; p < NPL; ++p)
                {
                    const int v = lane + 32 * p;
                    const int ei = v / NN, node = v - ei * NN, le = eb + ei;
                    minv[p] = 0;
                    if (v >= Sh::NODES || le >= ne)
                        continue;
                    const int i = node % N, j = node / N;
                    const Real *qn = us + le * ND + 3 * node;
                    const Real q0 = qn[0], q1 = qn[1], q2 = qn[2];
                    const double2 *c2 = reinterpret_cast<const double2 *>(cs + 8 * le);
                    const double2 c01 = c2[0], c23 = c2[1], c45 = c2[2], c67 = c2[3];
                    const Real xi = xt[i], eta = xt[j];
                    // QuadElement::jacobian (source/Element.cpp:21-27)
                    const Real Xxi = Real(0.25) * ((Real(1) - eta) * Real(c23.x - c01.x) + (Real(1) + eta) * Real(c45.x - c67.x));
                    const Real Yxi = Real(0.25) * ((Real(1) - eta) * Real(c23.y - c01.y) + (Real(1) + eta) * Real(c45.y - c67.y));
                    const Real Xeta = Real(0.25) * ((Real(1) - xi) * Real(c67.x - c01.x) + (Real(1) + xi) * Real(c45.x - c23.x));
                    const Real Yeta = Real(0.25) * ((Real(1) - xi) * Real(c67.y - c01.y) + (Real(1) + xi) * Real(c45.y - c23.y));
                    const Real W = wt[i] * wt[j];
                    const Real WYe = W * Yeta, WXe = W * Xeta, WYx = W * Yxi, WXx = W * Xxi;
                    Real *x = X + (ei * NN + node) * 6;
                    // [F_p F_u | F_v G_p | G_u G_v]
                    reinterpret_cast<R2 *>(x)[0] = R2{WYe * q1 - WXe * q2, WYe * q0};
                    reinterpret_cast<R2 *>(x)[1] = R2{-WXe * q0, -WYx * q1 + WXx * q2};
                    reinterpret_cast<R2 *>(x)[2] = R2{-WYx * q0, WXx * q0};
                    // MassMatrix<true>: w_i w_j det J (source/MassMatrix.cpp:6-28)
                    minv[p] = Real(1) / (W * (Xxi * Yeta - Yxi * Xeta));
                    if (EXTRA)
                    {
                        const size_t g = (size_t)(el0 + le) * ND + 3 * node;
#pragma unroll
                        for (int c = 0; c < 3; ++c)
                        {
                            fv[p][c] = (flags & F_FORCE) ? a.F[g + c] : Real(0);
                            av[p][c] = (flags & F_FILTER) ? a.acc[g + c] : 0.0;
                        }
                    }
                }

                // ---- face lanes: own trace, and the partner trace from L2 (issued now, used later)
                Real fo[FPL][3], fx[FPL][3];
                uint32_t fbyte[FPL];
#pragma unroll
                for (int p = 0; p < FPL; ++p)
                {
                    const int f = lane + 32 * p;
                    const int ei = f / NF, fl = f - ei * NF, le = eb + ei;
                    fbyte[p] = 0x40u; // inactive
                    if (f >= Sh::FACES || le >= ne)
                        continue;
                    const int s = fl / N, k = fl - s * N;
                    const uint32_t byte = (fks[le] >> (8 * s)) & 0xffu;
                    const Real *own = us + le * ND + 3 * face_node(N, s, k);
                    fo[p][0] = own[0];
                    fo[p][1] = own[1];
                    fo[p][2] = own[2];
                    fbyte[p] = byte;
                    if (byte & 0x80u)
                    {
                        if (!(flags & F_BND))
                            fbyte[p] = 0x40u;
                        continue;
                    }
                    if (!(flags & F_INT))
                    {
                        fbyte[p] = 0x40u;
                        continue;
                    }
                    const int off = fbs[4 * le + s] + k * partner_stride<N>(byte);
                    if (off < 0 || off + 3 > a.nel * ND)
                    {
                        atomicOr(a.err, 2u);
                        fbyte[p] = 0x40u;
                        continue;
                    }
                    fx[p][0] = __ldg(a.u + off);
                    fx[p][1] = __ldg(a.u + off + 1);
                    fx[p][2] = __ldg(a.u + off + 2);
                }
                __syncwarp();

                // ---- volume: du(i,j) = sum_l D(l,i) F(l,j) + D(l,j) G(i,l)  (div_2d_c, source/Div.cpp:131-179)
                Real rv[NPL][3];
#pragma unroll
                for (int p = 0; p < NPL; ++p)
                {
                    rv[p][0] = rv[p][1] = rv[p][2] = 0;
                    const int v = lane + 32 * p;
                    const int ei = v / NN, node = v - ei * NN, le = eb + ei;
                    if (v >= Sh::NODES || le >= ne || !(flags & F_VOL))
                        continue;
                    const int i = node % N, j = node / N;
                    const Real *xe = X + ei * NN * 6;
#pragma unroll
                    for (int l = 0; l < N; ++l)
                    {
                        const Real di = Dt[l + N * i], dj = Dt[l + N * j];
                        const Real *xf = xe + (l + N * j) * 6; // F at (l, j)
                        const Real *xg = xe + (i + N * l) * 6; // G at (i, l)
                        const R2 f01 = reinterpret_cast<const R2 *>(xf)[0];
                        const Real f2 = xf[2], g0 = xg[3];
                        const R2 g12 = reinterpret_cast<const R2 *>(xg)[2];
                        rv[p][0] += di * f01.x + dj * g0;
                        rv[p][1] += di * f01.y + dj * g12.x;
                        rv[p][2] += di * f2 + dj * g12.y;
                    }
                }

                // ---- upwind face fluxes (EdgeFlux / WaveBC closed form) into the face buffer
#pragma unroll
                for (int p = 0; p < FPL; ++p)
                {
                    const int f = lane + 32 * p;
                    const int ei = f / NF, fl = f - ei * NF, le = eb + ei;
                    if (f >= Sh::FACES || le >= ne)
                        continue;
                    Real *o = Fb + (ei * NF + fl) * 3;
                    const uint32_t byte = fbyte[p];
                    if (byte == 0x40u)
                    {
                        o[0] = o[1] = o[2] = 0;
                        continue;
                    }
                    const int s = fl / N, k = fl - s * N;
                    const int p0 = (0x0310 >> (4 * s)) & 0xf, p1 = (0x3221 >> (4 * s)) & 0xf; // side s runs p0 -> p1
                    const double *c = cs + 8 * le;
                    const double dx = c[2 * p1] - c[2 * p0], dy = c[2 * p1 + 1] - c[2 * p0 + 1];
                    const double s2 = dx * dx + dy * dy, rs = rsqrt(s2);
                    const double sgn = (s >= 2) ? -1.0 : 1.0;
                    const Real nx = (Real)(sgn * dy * rs), ny = (Real)(-sgn * dx * rs);
                    const Real hm = (Real)(0.25 * s2 * rs);
                    Real xq[3];
                    if (byte & 0x80u)
                        exterior<Real>((int)((byte >> 3) & 3u), nx, ny, fo[p], xq);
                    else
                    {
                        xq[0] = fx[p][0];
                        xq[1] = fx[p][1];
                        xq[2] = fx[p][2];
                    }
                    Real fl3[3] = {0, 0, 0};
                    upwind<Real>(nx, ny, wt[k] * hm, fo[p], xq, fl3);
                    o[0] = fl3[0];
                    o[1] = fl3[1];
                    o[2] = fl3[2];
                }
                __syncwarp();

                // ---- combine, M^{-1}, RK update in place (wavedg/ode.hpp:66-93)
#pragma unroll
                for (int p = 0; p < NPL; ++p)
                {
                    const int v = lane + 32 * p;
                    const int ei = v / NN, node = v - ei * NN, le = eb + ei;
                    if (v >= Sh::NODES || le >= ne)
                        continue;
                    const int i = node % N, j = node / N;
                    const Real *fe = Fb + ei * NF * 3;
                    Real r0 = rv[p][0], r1 = rv[p][1], r2 = rv[p][2];
                    // face slots (side * N + face node) through node (i, j)
                    const int sa = (j == 0) ? i : (j == N - 1) ? 2 * N + i : -1;
                    const int sb = (i == N - 1) ? N + j : (i == 0) ? 3 * N + j : -1;
                    if (sa >= 0)
                    {
                        r0 += fe[3 * sa];
                        r1 += fe[3 * sa + 1];
                        r2 += fe[3 * sa + 2];
                    }
                    if (sb >= 0)
                    {
                        r0 += fe[3 * sb];
                        r1 += fe[3 * sb + 1];
                        r2 += fe[3 * sb + 2];
                    }
                    if (EXTRA && (flags & F_FORCE))
                    {
                        r0 += a.fscale * fv[p][0];
                        r1 += a.fscale * fv[p][1];
                        r2 += a.fscale * fv[p][2];
                    }
                    if (flags & F_MINV)
                    {
                        r0 *= minv[p];
                        r1 *= minv[p];
                        r2 *= minv[p];
                    }
                    Real *un = us + le * ND + 3 * node;
                    Real *dn = dus + le * ND + 3 * node;
                    const Real d0 = has_du ? a.rk_a * dn[0] + a.dt * r0 : a.dt * r0;
                    const Real d1 = has_du ? a.rk_a * dn[1] + a.dt * r1 : a.dt * r1;
                    const Real d2 = has_du ? a.rk_a * dn[2] + a.dt * r2 : a.dt * r2;
                    const Real u0 = un[0] + a.rk_b * d0, u1 = un[1] + a.rk_b * d1, u2 = un[2] + a.rk_b * d2;
                    dn[0] = d0;
                    dn[1] = d1;
                    dn[2] = d2;
                    un[0] = u0;
                    un[1] = u1;
                    un[2] = u2;
                    if (EXTRA && (flags & F_FILTER))
                    {
                        const size_t g = (size_t)(el0 + le) * ND + 3 * node;
                        a.acc[g] = av[p][0] + a.acc_c * (double)u0;
                        a.acc[g + 1] = av[p][1] + a.acc_c * (double)u1;
                        a.acc[g + 2] = av[p][2] + a.acc_c * (double)u2;
                    }
                }
            }
            // results are in the slot: hand them to the async proxy, then release the slot
            fence_async_smem();
            __syncwarp();
            if (lane == 0)
                mbar_arrive(&done[q]);
        }
    }

    template <int N, typename Real>
    static cudaError_t launch_ws_n(const StageArgs<Real> &a, int grid_limit, cudaStream_t s)
    {
        const bool extra = (a.flags & (F_FORCE | F_FILTER)) != 0;
        auto kern = extra ? ws_stage_kernel<N, Real, true> : ws_stage_kernel<N, Real, false>;
        const size_t smem = (size_t)ws_layout<Real>(N, a.chunk, a.ring).total;
        int dev = 0;
        cudaGetDevice(&dev);
        static bool attr_set[2][64] = {};
        if (!attr_set[extra][dev & 63])
        {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
            if (e != cudaSuccess)
                return e;
            attr_set[extra][dev & 63] = true;
        }
        // resident CTAs per device for this footprint; cached per (device, variant)
        static int c_grid[2][64];
        static size_t c_smem[2][64];
        const int slot = dev & 63;
        if (c_smem[extra][slot] != smem + 1)
        {
            int per_sm = 0, sms = 0;
            cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kWsThreads, smem);
            if (e != cudaSuccess)
                return e;
            e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            if (e != cudaSuccess)
                return e;
            c_grid[extra][slot] = std::max(1, per_sm) * sms;
            c_smem[extra][slot] = smem + 1;
        }
        const int nchunks = (a.nel + a.chunk - 1) / a.chunk;
        int grid = c_grid[extra][slot];
        if (grid_limit > 0)
            grid = std::min(grid, grid_limit);
        grid = std::min(grid, nchunks);
        kern<<<grid, kWsThreads, smem, s>>>(a);
        return cudaGetLastError();
    }
} // namespace wdg
