// Warp-specialised RK stage kernel (included by kernels.cu).
//
// One CTA = one producer warp + kWsConsumers consumer warps, persistent over
// chunks of C consecutive elements (C a multiple of 4, so every chunk of u, du
// and geometry is a whole number of 16-byte units in HBM).
//
//   producer   ring of S chunk slots in shared memory.  For each chunk it
//              waits until the slot is free, loads u, du and the element
//              geometry with cp.async.bulk, and gathers every face node's
//              neighbour trace from the stage's input array with cp.async
//              (8- or 4-byte pieces; the mesh is unstructured), all on the
//              slot's `full` mbarrier.  Once every consumer warp has arrived
//              on the slot's `done` mbarrier it stores u' and du' back with
//              cp.async.bulk straight from the slot (results are in place).
//   consumers  a warp owns EW = floor(32 / n) whole elements per round, one
//              lane per grid line of each, all three fields per lane:
//                column pass  lane m holds column i = m: forms the eta-fluxes G
//                             of the column in registers and contracts them
//                             with D (compile-time constants) into 3 n sums;
//                             adds the upwind flux of the column's two face
//                             nodes (sides 0 and 2); writes the sums to a
//                             per-warp scratch.
//                row pass     lane m holds row j = m: xi-fluxes F, the xi
//                             contraction, the face nodes of sides 3 and 1,
//                             then per node the column pass's sums, M^{-1}
//                             and the RK update, in place.  The row pass works
//                             on contiguous 3 n-value runs, so its shared
//                             memory accesses are free of bank conflicts.
//              Warps sync only with __syncwarp; a chunk is released when all
//              consumer warps have arrived on its `done` barrier.
//
// The neighbour traces are gathered from global memory even when the
// neighbour sits in the same chunk: consumer warps overwrite their elements
// in place, so the slot's copy of u cannot serve another warp.  The gather
// runs on the producer's lanes ahead of time, so no consumer waits on L2.
//
// Used for RK launches whose arrays are 16-byte aligned; every other launch
// takes the tiled kernel.

namespace wdg
{
    template <int N>
    struct WsShape
    {
        static constexpr int NN = N * N, ND = 3 * NN, NF = 4 * N;
        static constexpr int EW = 32 / N; // elements per warp-round, one lane per line
    };
    constexpr int kWsThreads = 32 * (kWsConsumers + 1);

    int ws_epw(int n) { return 32 / n; }

    // shared-memory layout (bytes), identical on host and device:
    //   [2 S mbarriers | pad to 128][x (n), w (n) | pad to 128][S slots][consumer scratch]
    //   slot    = u (C, 3 n^2) | du (C, 3 n^2) | halo (C, 4 n, 3) | corners (C, 8 doubles) | fcode (C, u32)
    //   scratch = per warp, per element of a round: column-pass sums [n^2][3]
    struct WsLayout
    {
        int slot, tab, slots, scratch, warp_scratch, total;
    };
    template <typename Real>
    __host__ __device__ inline WsLayout ws_layout(int n, int chunk, int stages, bool staged = false);

    __device__ __forceinline__ void mbar_arrive(uint64_t *bar)
    {
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
    }
    // arrive on `bar` once this thread's earlier cp.async copies have landed; counts as
    // one of the barrier's expected arrivals
    __device__ __forceinline__ void cp_async_mbar_arrive(uint64_t *bar)
    {
        asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
    }

    // Upwind flux of face node k of side SIDE of one element (own trace `own`),
    // subtracted into r: the closed form of EdgeFlux (source/EdgeFlux.cpp:7-139)
    // with the side's outward normal and measure (StraightEdge, wavedg/Edge.hpp:107-122)
    // and the exterior state of WaveBC for boundary sides.
    template <int N, typename Real, int SIDE>
    __device__ __forceinline__ void ws_face(uint32_t codes, int flags, const double2 c01, const double2 c23,
                                            const double2 c45, const double2 c67, Real wk, int k,
                                            const Real *own, const Real *halo_e, Real &r0, Real &r1, Real &r2)
    {
        const uint32_t byte = (codes >> (8 * SIDE)) & 0xffu;
        const bool bnd = (byte & 0x80u) != 0;
        if (bnd ? !(flags & F_BND) : !(flags & F_INT))
            return;
        // side SIDE runs from corner p0 to p1: 0: 0->1, 1: 1->2, 2: 3->2, 3: 0->3
        const double2 a0 = (SIDE == 0 || SIDE == 3) ? c01 : (SIDE == 1) ? c23 : c67;
        const double2 a1 = (SIDE == 0) ? c23 : (SIDE == 3) ? c67 : c45;
        Real nx, ny, h;
        if constexpr (sizeof(Real) == 4)
        {
            // FP32 stepping: the side's length and normal in FP32 from FP64 corner differences
            const float dx = (float)(a1.x - a0.x), dy = (float)(a1.y - a0.y);
            const float s2 = dx * dx + dy * dy, rs = rsqrtf(s2);
            const float sgn = (SIDE >= 2) ? -1.f : 1.f;
            nx = sgn * dy * rs;
            ny = -sgn * dx * rs;
            h = wk * (0.25f * s2 * rs);
        }
        else
        {
            const double dx = a1.x - a0.x, dy = a1.y - a0.y;
            const double s2 = dx * dx + dy * dy, rs = rsqrt(s2);
            const double sgn = (SIDE >= 2) ? -1.0 : 1.0;
            nx = (Real)(sgn * dy * rs);
            ny = (Real)(-sgn * dx * rs);
            h = wk * (Real)(0.25 * s2 * rs);
        }
        const Real q[3] = {own[0], own[1], own[2]};
        Real x[3];
        if (bnd)
            exterior<Real>((int)((byte >> 3) & 3u), nx, ny, q, x);
        else
        {
            const Real *hp = halo_e + 3 * (SIDE * N + k);
            x[0] = hp[0];
            x[1] = hp[1];
            x[2] = hp[2];
        }
        Real r[3] = {r0, r1, r2};
        upwind<Real>(nx, ny, h, q, x, r);
        r0 = r[0];
        r1 = r[1];
        r2 = r[2];
    }

    // One chunk of one RK stage as both roles see it (the single-solve kernel fills it from
    // its launch arguments, the batched kernel from its solve table).
    template <typename Real>
    struct WsChunk
    {
        const Real *u;  // state in (the stage's input array; neighbour traces come from it)
        Real *out;      // u' (never aliases u)
        Real *du;       // RK register, read (stages > 0) and written in place
        const Real *F;  // forcing (F_FORCE)
        double *acc;    // FP64 filter accumulator (F_FILTER)
        const double *corners;
        const int4 *fbase;
        const uint32_t *fcode;
        unsigned *err;
        int nel, el0, ne, chunk, flags;
        int nread; // readable values of u for neighbour traces (0: nel * 3 n^2)
        Real rk_a, rk_b, dt, fscale;
        double acc_c;
        // batched WaveHoltz, last stage of a period: 1 = fixed-point update W <- filter,
        // 2 = end of the separate pi0 period (only its norm is kept); 0 = neither
        int pend;
        double *W;    // FP64 iterate
        double c0;    // 0.5 dt K(0): the filter's first term at a period start
        double *part; // this chunk's partial sums: per consumer warp (sum (W' - W)^2, sum W'^2)
    };

    // slot offsets (bytes) of an n, chunk-C slot:
    //   u (C, 3 n^2) | du (C, 3 n^2) | halo (C, 4 n, 3) | corners (C, 8 doubles) | fcode (C, u32)
    //   [ | F (C, 3 n^2) | filter (C, 3 n^2, FP64) ]   staged: FP32 launches with forcing / filter
    // Staging F and the filter through the slot keeps their latency off the consumers; FP64
    // launches read them directly, since the larger slot would cost a CTA per SM.
    struct WsSlot
    {
        int ub, hb, cb, kb, fb, ab, bytes;
    };
    template <typename Real, bool EXTRA>
    struct WsStage
    {
        static constexpr bool value = EXTRA && sizeof(Real) == 4;
    };
    template <typename Real>
    __host__ __device__ inline WsSlot ws_slot(int n, int chunk, bool staged = false)
    {
        WsSlot o;
        o.ub = chunk * 3 * n * n * (int)sizeof(Real);
        o.hb = 2 * o.ub;
        o.cb = o.hb + chunk * 12 * n * (int)sizeof(Real);
        o.kb = o.cb + chunk * 64;
        o.fb = o.kb + chunk * 4;
        o.ab = o.fb + (staged ? o.ub : 0);
        o.bytes = o.ab + (staged ? chunk * 3 * n * n * 8 : 0);
        return o;
    }

    // ---------------------------------------------------------------- producer: load one chunk
    // u, du, corners and side codes by cp.async.bulk on `full` (plain copies for a ragged
    // chunk), then the neighbour traces of every interior face node by cp.async, one lane
    // per (element, side); the table reads of a batch go out together, so a chunk costs one
    // L2 round trip per batch rather than one per face node.
    template <int N, typename Real, bool EXTRA = false>
    __device__ __forceinline__ void ws_load(const WsChunk<Real> &c, unsigned char *base, uint64_t *full, int lane)
    {
        constexpr int ND = 3 * N * N, NF = 4 * N;
        constexpr bool STG = WsStage<Real, EXTRA>::value;
        const WsSlot o = ws_slot<Real>(N, c.chunk, STG);
        const bool has_du = (c.flags & F_READ_DU) != 0;
        const bool sF = STG && (c.flags & F_FORCE), sA = STG && (c.flags & F_FILTER);
        const int el0 = c.el0, ne = c.ne, C = c.chunk;
        if (ne == C)
        {
            if (lane == 0)
            {
                mbar_expect_tx(full, (uint32_t)(o.ub * ((has_du ? 2 : 1) + (sF ? 1 : 0)) + C * 68 +
                                                 (sA ? C * ND * 8 : 0)));
                bulk_g2s(base, c.u + (size_t)el0 * ND, (uint32_t)o.ub, full);
                if (has_du)
                    bulk_g2s(base + o.ub, c.du + (size_t)el0 * ND, (uint32_t)o.ub, full);
                bulk_g2s(base + o.cb, c.corners + 8 * (size_t)el0, (uint32_t)(64 * C), full);
                bulk_g2s(base + o.kb, c.fcode + el0, (uint32_t)(4 * C), full);
                if (sF)
                    bulk_g2s(base + o.fb, c.F + (size_t)el0 * ND, (uint32_t)o.ub, full);
                if (sA)
                    bulk_g2s(base + o.ab, c.acc + (size_t)el0 * ND, (uint32_t)(C * ND * 8), full);
            }
        }
        else
        {
            Real *us = reinterpret_cast<Real *>(base), *dus = us + C * ND;
            for (int i = lane; i < ne * ND; i += 32)
            {
                us[i] = c.u[(size_t)el0 * ND + i];
                if (has_du)
                    dus[i] = c.du[(size_t)el0 * ND + i];
                if (sF)
                    reinterpret_cast<Real *>(base + o.fb)[i] = c.F[(size_t)el0 * ND + i];
                if (sA)
                    reinterpret_cast<double *>(base + o.ab)[i] = c.acc[(size_t)el0 * ND + i];
            }
            double *cw = reinterpret_cast<double *>(base + o.cb);
            for (int i = lane; i < ne * 8; i += 32)
                cw[i] = c.corners[8 * (size_t)el0 + i];
            uint32_t *kw = reinterpret_cast<uint32_t *>(base + o.kb);
            for (int i = lane; i < ne; i += 32)
                kw[i] = c.fcode[el0 + i];
            __threadfence_block();
            __syncwarp();
            if (lane == 0)
                mbar_arrive(full);
        }
        if (c.flags & F_INT)
        {
            Real *halo = reinterpret_cast<Real *>(base + o.hb);
            const int limit = c.nread > 0 ? c.nread : c.nel * ND;
            constexpr int B = 4; // (element, side) pairs per lane per batch
            for (int p0 = 0; p0 < ne * 4; p0 += 32 * B)
            {
                uint32_t code[B];
                int off[B];
#pragma unroll
                for (int b = 0; b < B; ++b)
                {
                    const int pr = p0 + 32 * b + lane, le = pr >> 2, s = pr & 3;
                    code[b] = 0x80u;
                    off[b] = -1;
                    if (pr < ne * 4)
                    {
                        code[b] = (__ldg(c.fcode + el0 + le) >> (8 * s)) & 0xffu;
                        off[b] = __ldg(reinterpret_cast<const int *>(c.fbase + el0 + le) + s);
                    }
                }
#pragma unroll
                for (int b = 0; b < B; ++b)
                {
                    const int pr = p0 + 32 * b + lane, le = pr >> 2, s = pr & 3;
                    if (code[b] & 0x80u)
                        continue; // boundary side (or past the chunk): no neighbour
                    const int stride = partner_stride<N>(code[b]);
                    if (off[b] < 0 || off[b] + (N - 1) * stride < 0 || off[b] + 3 > limit ||
                        off[b] + (N - 1) * stride + 3 > limit)
                    {
                        atomicOr(c.err, 2u);
                        continue;
                    }
                    Real *dst = halo + 3 * (le * NF + s * N);
#pragma unroll
                    for (int k = 0; k < N; ++k)
                    {
                        const Real *src = c.u + off[b] + k * stride;
                        cp_async<sizeof(Real)>(dst + 3 * k, src);
                        cp_async<sizeof(Real)>(dst + 3 * k + 1, src + 1);
                        cp_async<sizeof(Real)>(dst + 3 * k + 2, src + 2);
                    }
                }
            }
        }
        cp_async_mbar_arrive(full);
    }

    // ---------------------------------------------------------------- producer: store one chunk
    template <int N, typename Real, bool EXTRA = false>
    __device__ __forceinline__ void ws_store(const WsChunk<Real> &c, const unsigned char *base, int lane)
    {
        constexpr int ND = 3 * N * N;
        constexpr bool STG = WsStage<Real, EXTRA>::value;
        const WsSlot o = ws_slot<Real>(N, c.chunk, STG);
        const bool sA = STG && (c.flags & F_FILTER);
        const int el0 = c.el0, ne = c.ne;
        if (ne == c.chunk)
        {
            if (lane == 0)
            {
                bulk_s2g(c.out + (size_t)el0 * ND, base, (uint32_t)o.ub);
                bulk_s2g(c.du + (size_t)el0 * ND, base + o.ub, (uint32_t)o.ub);
                if (sA)
                    bulk_s2g(c.acc + (size_t)el0 * ND, base + o.ab, (uint32_t)(c.chunk * ND * 8));
                bulk_commit();
            }
        }
        else
        {
            const Real *us = reinterpret_cast<const Real *>(base), *dus = us + c.chunk * ND;
            const double *as = reinterpret_cast<const double *>(base + o.ab);
            for (int i = lane; i < ne * ND; i += 32)
            {
                c.out[(size_t)el0 * ND + i] = us[i];
                c.du[(size_t)el0 * ND + i] = dus[i];
                if (sA)
                    c.acc[(size_t)el0 * ND + i] = as[i];
            }
        }
    }

    // ---------------------------------------------------------------- consumer: one chunk
    // Warp `cw` takes rounds of EW whole elements; Rc is its scratch for the column sums.
    template <int N, typename Real, bool EXTRA, bool BATCH>
    __device__ __forceinline__ void ws_consume(const WsChunk<Real> &c, unsigned char *base, Real *Rc,
                                               const Real *xtab, const Real *wtab, int cw, int lane)
    {
        using Sh = WsShape<N>;
        constexpr int NN = Sh::NN, ND = Sh::ND, NF = Sh::NF, EW = Sh::EW;
        constexpr bool STG = WsStage<Real, EXTRA>::value;
        const WsSlot o = ws_slot<Real>(N, c.chunk, STG);
        const int flags = c.flags;
        // forcing and filter: staged in the slot (chunk-local index) or read in place
        const Real *Fx = STG ? reinterpret_cast<const Real *>(base + o.fb) - (size_t)c.el0 * ND : c.F;
        double *Ax = STG ? reinterpret_cast<double *>(base + o.ab) - (size_t)c.el0 * ND : c.acc;
        const bool has_du = (flags & F_READ_DU) != 0;
        const int R = c.chunk / (kWsConsumers * EW); // warp-rounds per chunk
        const int el_l = lane / N, ln = lane - el_l * N; // element of the round, grid line
        const bool lane_on = lane < EW * N;
        const Real xm = lane_on ? xtab[ln] : Real(0), wm = lane_on ? wtab[ln] : Real(0);
        Real *us = reinterpret_cast<Real *>(base);
        Real *dus = us + c.chunk * ND;
        const Real *halo = reinterpret_cast<const Real *>(base + o.hb);
        const double *cs = reinterpret_cast<const double *>(base + o.cb);
        const uint32_t *fks = reinterpret_cast<const uint32_t *>(base + o.kb);
        double dsum = 0.0, nsum = 0.0;

        for (int r = 0; r < R; ++r)
        {
                const int le = (cw * R + r) * EW + el_l; // chunk-local element of this lane
                const bool act = lane_on && le < c.ne;
                double2 c01, c23, c45, c67;
                uint32_t codes = 0;
                const Real *halo_e = halo + le * NF * 3;
                Real *ue = us + le * ND;
                Real *rc = Rc + el_l * NN * 3; // this element's column-pass sums, (node, field)
                if (act)
                {
                    const double2 *c2 = reinterpret_cast<const double2 *>(cs + 8 * le);
                    c01 = c2[0];
                    c23 = c2[1];
                    c45 = c2[2];
                    c67 = c2[3];
                    codes = fks[le];

                    // ---- column pass: column i = ln.  Contravariant eta-fluxes of the wave system
                    // (source/Div.cpp:5-53): G = W (-y_xi u + x_xi v, -y_xi p, x_xi p); along a
                    // column x_eta, y_eta are constant and x_xi, y_xi vary linearly with eta.
                    const int i = ln;
                    const Real wi = wm;
                    const Real dx0 = Real(c23.x - c01.x), dx1 = Real(c45.x - c67.x);
                    const Real dy0 = Real(c23.y - c01.y), dy1 = Real(c45.y - c67.y);
                    Real sp[N], su[N], sv[N];
#pragma unroll
                    for (int j = 0; j < N; ++j)
                        sp[j] = su[j] = sv[j] = 0;
                    if (flags & F_VOL)
                    {
#pragma unroll
                        for (int l = 0; l < N; ++l)
                        {
                            const Real el = Tab<Real>::x(N, l);
                            const Real Xxi = Real(0.25) * ((Real(1) - el) * dx0 + (Real(1) + el) * dx1);
                            const Real Yxi = Real(0.25) * ((Real(1) - el) * dy0 + (Real(1) + el) * dy1);
                            const Real W = wi * Tab<Real>::w(N, l);
                            const Real *nd = ue + 3 * (i + N * l);
                            const Real p = nd[0], u = nd[1], v = nd[2];
                            const Real WYx = W * Yxi, WXx = W * Xxi;
                            const Real Gp = -WYx * u + WXx * v, Gu = -WYx * p, Gv = WXx * p;
                            // du(i, j) += sum_l D(l, j) G(i, l)  (div_2d_c, source/Div.cpp:131-179)
#pragma unroll
                            for (int j = 0; j < N; ++j)
                            {
                                const Real d = Tab<Real>::D(N, l + N * j);
                                sp[j] += d * Gp;
                                su[j] += d * Gu;
                                sv[j] += d * Gv;
                            }
                        }
                    }
                    // face nodes of the column: (i, 0) on side 0, (i, n-1) on side 2, face-node index i
                    ws_face<N, Real, 0>(codes, flags, c01, c23, c45, c67, wi, i, ue + 3 * i, halo_e, sp[0], su[0], sv[0]);
                    ws_face<N, Real, 2>(codes, flags, c01, c23, c45, c67, wi, i, ue + 3 * (i + N * (N - 1)), halo_e,
                                        sp[N - 1], su[N - 1], sv[N - 1]);
#pragma unroll
                    for (int j = 0; j < N; ++j)
                    {
                        Real *o = rc + 3 * (i + N * j);
                        o[0] = sp[j];
                        o[1] = su[j];
                        o[2] = sv[j];
                    }
                }
                __syncwarp();
                if (act)
                {
                    // ---- row pass: row j = ln.  F = W (y_eta u - x_eta v, y_eta p, -x_eta p); along a
                    // row x_xi, y_xi are constant and x_eta, y_eta vary linearly with xi.
                    const int j = ln;
                    const Real eta = xm, wj = wm;
                    const Real Xxi = Real(0.25) * ((Real(1) - eta) * Real(c23.x - c01.x) + (Real(1) + eta) * Real(c45.x - c67.x));
                    const Real Yxi = Real(0.25) * ((Real(1) - eta) * Real(c23.y - c01.y) + (Real(1) + eta) * Real(c45.y - c67.y));
                    const Real ex0 = Real(c67.x - c01.x), ex1 = Real(c45.x - c23.x);
                    const Real ey0 = Real(c67.y - c01.y), ey1 = Real(c45.y - c23.y);
                    Real *row = ue + 3 * N * j;
                    Real q0[N], q1[N], q2[N], mv[N];
                    Real ap[N], au[N], av[N];
#pragma unroll
                    for (int l = 0; l < N; ++l)
                    {
                        q0[l] = row[3 * l];
                        q1[l] = row[3 * l + 1];
                        q2[l] = row[3 * l + 2];
                        ap[l] = au[l] = av[l] = 0;
                    }
#pragma unroll
                    for (int l = 0; l < N; ++l)
                    {
                        const Real xl = Tab<Real>::x(N, l);
                        const Real Xeta = Real(0.25) * ((Real(1) - xl) * ex0 + (Real(1) + xl) * ex1);
                        const Real Yeta = Real(0.25) * ((Real(1) - xl) * ey0 + (Real(1) + xl) * ey1);
                        const Real W = Tab<Real>::w(N, l) * wj;
                        // MassMatrix<true>: w_i w_j det J (source/MassMatrix.cpp:6-28)
                        if constexpr (sizeof(Real) == 4)
                            mv[l] = __frcp_rn(W * (Xxi * Yeta - Yxi * Xeta));
                        else
                            mv[l] = Real(1) / (W * (Xxi * Yeta - Yxi * Xeta));
                        if (flags & F_VOL)
                        {
                            const Real WYe = W * Yeta, WXe = W * Xeta;
                            const Real Fp = WYe * q1[l] - WXe * q2[l], Fu = WYe * q0[l], Fv = -WXe * q0[l];
                            // du(i, j) += sum_l D(l, i) F(l, j)
#pragma unroll
                            for (int i = 0; i < N; ++i)
                            {
                                const Real d = Tab<Real>::D(N, l + N * i);
                                ap[i] += d * Fp;
                                au[i] += d * Fu;
                                av[i] += d * Fv;
                            }
                        }
                    }
                    // face nodes of the row: (0, j) on side 3, (n-1, j) on side 1, face-node index j
                    ws_face<N, Real, 3>(codes, flags, c01, c23, c45, c67, wj, j, row, halo_e, ap[0], au[0], av[0]);
                    ws_face<N, Real, 1>(codes, flags, c01, c23, c45, c67, wj, j, row + 3 * (N - 1), halo_e,
                                        ap[N - 1], au[N - 1], av[N - 1]);

                    // ---- epilogue per node of the row: + column-pass sums, forcing, M^{-1}, RK
                    // update in place (wavedg/ode.hpp:66-93); the row is this lane's alone
                    Real *drow = dus + le * ND + 3 * N * j;
#pragma unroll
                    for (int i = 0; i < N; ++i)
                    {
                        const Real *cr = rc + 3 * (i + N * j);
                        Real r0 = ap[i] + cr[0], r1 = au[i] + cr[1], r2 = av[i] + cr[2];
                        const size_t g = (size_t)(c.el0 + le) * ND + 3 * (i + N * j);
                        if (EXTRA && (flags & F_FORCE))
                        {
                            r0 += c.fscale * Fx[g];
                            r1 += c.fscale * Fx[g + 1];
                            r2 += c.fscale * Fx[g + 2];
                        }
                        if (flags & F_MINV)
                        {
                            r0 *= mv[i];
                            r1 *= mv[i];
                            r2 *= mv[i];
                        }
                        Real *dn = drow + 3 * i;
                        const Real d0 = has_du ? c.rk_a * dn[0] + c.dt * r0 : c.dt * r0;
                        const Real d1 = has_du ? c.rk_a * dn[1] + c.dt * r1 : c.dt * r1;
                        const Real d2 = has_du ? c.rk_a * dn[2] + c.dt * r2 : c.dt * r2;
                        Real uo[3] = {q0[i] + c.rk_b * d0, q1[i] + c.rk_b * d1, q2[i] + c.rk_b * d2};
                        dn[0] = d0;
                        dn[1] = d1;
                        dn[2] = d2;
                        if (BATCH && c.pend)
                        {
                            // last step of a period: the filter's last term completes the period's
                            // result; the state and the filter restart from the new iterate
#pragma unroll
                            for (int f = 0; f < 3; ++f)
                            {
                                const double fin = Ax[g + f] + c.acc_c * (double)uo[f];
                                nsum += fin * fin;
                                double w0;
                                if (c.pend == 1)
                                {
                                    const double dw = fin - c.W[g + f];
                                    dsum += dw * dw;
                                    c.W[g + f] = fin;
                                    w0 = fin;
                                }
                                else
                                    w0 = c.W[g + f];
                                Ax[g + f] = c.c0 * w0;
                                uo[f] = (Real)w0;
                            }
                        }
                        else if (EXTRA && (flags & F_FILTER))
                        {
                            Ax[g] += c.acc_c * (double)uo[0];
                            Ax[g + 1] += c.acc_c * (double)uo[1];
                            Ax[g + 2] += c.acc_c * (double)uo[2];
                        }
                        row[3 * i] = uo[0];
                        row[3 * i + 1] = uo[1];
                        row[3 * i + 2] = uo[2];
                    }
                }
                __syncwarp(); // the scratch is reused by the next round
        }
        if (BATCH && c.pend)
        {
#pragma unroll
            for (int sh = 16; sh > 0; sh >>= 1)
            {
                dsum += __shfl_xor_sync(0xffffffffu, dsum, sh);
                nsum += __shfl_xor_sync(0xffffffffu, nsum, sh);
            }
            if (lane == 0)
            {
                c.part[2 * cw] = dsum;
                c.part[2 * cw + 1] = nsum;
            }
        }
    }

    template <typename Real>
    __host__ __device__ inline WsLayout ws_layout(int n, int chunk, int stages, bool staged)
    {
        WsLayout L;
        const int nn = n * n, ew = 32 / n;
        L.slot = ws_slot<Real>(n, chunk, staged).bytes;
        L.tab = 128;
        L.slots = (L.tab + 2 * n * (int)sizeof(Real) + 127) & ~127;
        L.scratch = L.slots + stages * L.slot;
        L.warp_scratch = ((ew * 3 * nn * (int)sizeof(Real)) + 15) & ~15;
        L.total = L.scratch + kWsConsumers * L.warp_scratch;
        return L;
    }

    template <int N, typename Real, bool EXTRA>
    __global__ void __launch_bounds__(kWsThreads, 2) ws_stage_kernel(const StageArgs<Real> a)
    {
        const int C = a.chunk, S = a.ring, G = gridDim.x;
        const int e0 = a.el_begin, e1 = a.el_end > 0 ? a.el_end : a.nel; // this launch's elements
        const int nchunks = (e1 - e0 + C - 1) / C;
        const WsLayout L = ws_layout<Real>(N, C, S, WsStage<Real, EXTRA>::value);

        extern __shared__ __align__(128) unsigned char smem[];
        uint64_t *full = reinterpret_cast<uint64_t *>(smem);
        uint64_t *done = full + S;
        Real *xt = reinterpret_cast<Real *>(smem + L.tab); // GLL nodes, then weights
        Real *wt = xt + N;
        unsigned char *slots = smem + L.slots;

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
        __syncthreads();

        // this CTA's chunks: k_m = blockIdx.x + m G
        const int M = ((int)blockIdx.x < nchunks) ? (nchunks - 1 - (int)blockIdx.x) / G + 1 : 0;
        WsChunk<Real> c{};
        c.u = a.u;
        c.out = a.out;
        c.du = a.du;
        c.F = a.F;
        c.acc = a.acc;
        c.corners = a.corners;
        c.fbase = a.fbase;
        c.fcode = a.fcode;
        c.err = a.err;
        c.nel = a.nel;
        c.nread = a.nread;
        c.chunk = C;
        c.flags = a.flags;
        c.rk_a = a.rk_a;
        c.rk_b = a.rk_b;
        c.dt = a.dt;
        c.fscale = a.fscale;
        c.acc_c = a.acc_c;
        auto at = [&](int m)
        {
            c.el0 = e0 + ((int)blockIdx.x + m * G) * C;
            c.ne = min(C, e1 - c.el0);
        };
        const uint64_t wlim = wait_limit(a.wait_ns);

        if (warp == kWsConsumers)
        {
            // ------------------------------------------------------------ producer
            // test hook: chunk test_skip - 1 is never loaded, so every wait on it runs out
            for (int m = 0; m < min(S, M); ++m)
            {
                at(m);
                if (m + 1 != a.test_skip)
                    ws_load<N, Real, EXTRA>(c, slots + (m % S) * L.slot, &full[m % S], lane);
            }
            int m = 0;
            for (; m < M; ++m)
            {
                const int q = m % S;
                // a warp-uniform verdict, so no lane leaves while others go on
                if (!__all_sync(0xffffffffu, mbar_wait(&done[q], (m / S) & 1, wlim)))
                    break;
                at(m);
                ws_store<N, Real, EXTRA>(c, slots + q * L.slot, lane);
                if (m + S < M)
                {
                    if (lane == 0)
                        bulk_wait_read(); // the store above has read the slot
                    __syncwarp();
                    at(m + S);
                    if (m + S + 1 != a.test_skip)
                        ws_load<N, Real, EXTRA>(c, slots + q * L.slot, &full[q], lane);
                }
            }
            if (m < M)
            {
                // a consumer gave up: record it, let the loads already issued land, leave
                if (lane == 0)
                {
                    atomicOr(a.err, 1u);
                    for (int r = m; r < min(m + S, M); ++r)
                        mbar_wait(&full[r % S], (r / S) & 1, wlim);
                }
            }
            if (lane == 0)
                bulk_wait_all();
            return;
        }

        // ---------------------------------------------------------------- consumers
        Real *Rc = reinterpret_cast<Real *>(smem + L.scratch + warp * L.warp_scratch); // [EW][NN][3] column sums
        for (int m = 0; m < M; ++m)
        {
            const int q = m % S;
            if (!__all_sync(0xffffffffu, mbar_wait(&full[q], (m / S) & 1, wlim)))
            {
                if (lane == 0)
                    atomicOr(a.err, 1u);
                break;
            }
            at(m);
            ws_consume<N, Real, EXTRA, false>(c, slots + q * L.slot, Rc, xt, wt, warp, lane);
            // results are in the slot: hand them to the async proxy, then release the slot
            fence_async_smem();
            __syncwarp();
            if (lane == 0)
                mbar_arrive(&done[q]);
        }
    }

    // whether a launch's shared memory (the forcing / filter staging included) fits a CTA
    template <int N, typename Real>
    static bool ws_fits(const StageArgs<Real> &a)
    {
        const bool extra = (a.flags & (F_FORCE | F_FILTER)) != 0;
        const size_t smem = (size_t)ws_layout<Real>(N, a.chunk, a.ring, extra && WsStage<Real, true>::value).total;
        return smem <= 227 * 1024;
    }

    template <int N, typename Real>
    static cudaError_t launch_ws_n(const StageArgs<Real> &a, int grid_limit, cudaStream_t s)
    {
        const bool extra = (a.flags & (F_FORCE | F_FILTER)) != 0;
        auto kern = extra ? ws_stage_kernel<N, Real, true> : ws_stage_kernel<N, Real, false>;
        const size_t smem = (size_t)(extra ? ws_layout<Real>(N, a.chunk, a.ring, WsStage<Real, true>::value).total
                                           : ws_layout<Real>(N, a.chunk, a.ring).total);

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
        const int span = (a.el_end > 0 ? a.el_end : a.nel) - a.el_begin;
        const int nchunks = (span + a.chunk - 1) / a.chunk;
        int grid = c_grid[extra][slot];
        if (grid_limit > 0)
            grid = std::min(grid, grid_limit);
        grid = std::min(grid, nchunks);
        if (grid < 1)
            return cudaSuccess; // an empty range
        kern<<<grid, kWsThreads, smem, s>>>(a);
        return cudaGetLastError();
    }
} // namespace wdg
