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
    constexpr int kWsConsumers = 4;
    constexpr int kWsThreads = 32 * (kWsConsumers + 1);

    int ws_epw(int n) { return 32 / n; }

    // shared-memory layout (bytes), identical on host and device:
    //   [2 S mbarriers | pad to 128][x (n), w (n) | pad to 128][S slots][consumer scratch]
    //   slot    = u (C, 3 n^2) | du (C, 3 n^2) | halo (C, 4 n, 3) | corners (C, 8 doubles) | fcode (C, u32)
    //   scratch = per warp, per element of a round: column-pass sums [n^2][3]
    struct WsLayout
    {
        int ub, hb, cb, kb, slot, tab, slots, scratch, warp_scratch, total;
    };
    template <typename Real>
    __host__ __device__ inline WsLayout ws_layout(int n, int chunk, int stages)
    {
        WsLayout L;
        const int nn = n * n, ew = 32 / n;
        L.ub = chunk * 3 * nn * (int)sizeof(Real);
        L.hb = 2 * L.ub;                                   // halo
        L.cb = L.hb + chunk * 12 * n * (int)sizeof(Real);  // corners
        L.kb = L.cb + chunk * 64;                          // side codes
        L.slot = L.kb + chunk * 4;
        L.tab = 128;
        L.slots = (L.tab + 2 * n * (int)sizeof(Real) + 127) & ~127;
        L.scratch = L.slots + stages * L.slot;
        L.warp_scratch = ((ew * 3 * nn * (int)sizeof(Real)) + 15) & ~15;
        L.total = L.scratch + kWsConsumers * L.warp_scratch;
        return L;
    }

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
        const double dx = a1.x - a0.x, dy = a1.y - a0.y;
        const double s2 = dx * dx + dy * dy, rs = rsqrt(s2);
        const double sgn = (SIDE >= 2) ? -1.0 : 1.0;
        const Real nx = (Real)(sgn * dy * rs), ny = (Real)(-sgn * dx * rs);
        const Real h = wk * (Real)(0.25 * s2 * rs);
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

    template <int N, typename Real, bool EXTRA>
    __global__ void __launch_bounds__(kWsThreads, 2) ws_stage_kernel(const StageArgs<Real> a)
    {
        using Sh = WsShape<N>;
        constexpr int NN = Sh::NN, ND = Sh::ND, NF = Sh::NF, EW = Sh::EW;
        const int C = a.chunk, S = a.ring, G = gridDim.x;
        const int flags = a.flags;
        const bool has_du = (flags & F_READ_DU) != 0;
        const int nchunks = (a.nel + C - 1) / C;
        const WsLayout L = ws_layout<Real>(N, C, S);

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
                        mbar_expect_tx(&full[q], (uint32_t)(L.ub * (has_du ? 2 : 1) + C * 68));
                        bulk_g2s(base, a.u + (size_t)el0 * ND, (uint32_t)L.ub, &full[q]);
                        if (has_du)
                            bulk_g2s(base + L.ub, a.du + (size_t)el0 * ND, (uint32_t)L.ub, &full[q]);
                        bulk_g2s(base + L.cb, a.corners + 8 * (size_t)el0, (uint32_t)(64 * C), &full[q]);
                        bulk_g2s(base + L.kb, a.fcode + el0, (uint32_t)(4 * C), &full[q]);
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
                    double *cw = reinterpret_cast<double *>(base + L.cb);
                    for (int i = lane; i < ne * 8; i += 32)
                        cw[i] = a.corners[8 * (size_t)el0 + i];
                    uint32_t *kw = reinterpret_cast<uint32_t *>(base + L.kb);
                    for (int i = lane; i < ne; i += 32)
                        kw[i] = a.fcode[el0 + i];
                    __threadfence_block();
                    __syncwarp();
                    if (lane == 0)
                        mbar_arrive(&full[q]);
                }
                // neighbour traces of every interior face node of the chunk: one lane per
                // (element, side); the table reads of a batch go out together, so a chunk
                // costs one L2 round trip per batch rather than one per face node
                if (flags & F_INT)
                {
                    Real *halo = reinterpret_cast<Real *>(base + L.hb);
                    const int limit = a.nel * ND;
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
                                code[b] = (__ldg(a.fcode + el0 + le) >> (8 * s)) & 0xffu;
                                off[b] = __ldg(reinterpret_cast<const int *>(a.fbase + el0 + le) + s);
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
                                atomicOr(a.err, 2u);
                                continue;
                            }
                            Real *dst = halo + 3 * (le * NF + s * N);
#pragma unroll
                            for (int k = 0; k < N; ++k)
                            {
                                const Real *src = a.u + off[b] + k * stride;
                                cp_async<sizeof(Real)>(dst + 3 * k, src);
                                cp_async<sizeof(Real)>(dst + 3 * k + 1, src + 1);
                                cp_async<sizeof(Real)>(dst + 3 * k + 2, src + 2);
                            }
                        }
                    }
                }
                cp_async_mbar_arrive(&full[q]);
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
        const int R = C / (kWsConsumers * EW); // warp-rounds per chunk
        Real *Rc = reinterpret_cast<Real *>(smem + L.scratch + cw * L.warp_scratch); // [EW][NN][3] column-pass sums
        const int el_l = lane / N, ln = lane - el_l * N; // element of the round, grid line
        const bool lane_on = lane < EW * N;
        const Real xm = lane_on ? xt[ln] : Real(0), wm = lane_on ? wt[ln] : Real(0);

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
            const Real *halo = reinterpret_cast<const Real *>(base + L.hb);
            const double *cs = reinterpret_cast<const double *>(base + L.cb);
            const uint32_t *fks = reinterpret_cast<const uint32_t *>(base + L.kb);

            for (int r = 0; r < R; ++r)
            {
                const int le = (cw * R + r) * EW + el_l; // chunk-local element of this lane
                const bool act = lane_on && le < ne;
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
                        const size_t g = (size_t)(el0 + le) * ND + 3 * (i + N * j);
                        if (EXTRA && (flags & F_FORCE))
                        {
                            r0 += a.fscale * a.F[g];
                            r1 += a.fscale * a.F[g + 1];
                            r2 += a.fscale * a.F[g + 2];
                        }
                        if (flags & F_MINV)
                        {
                            r0 *= mv[i];
                            r1 *= mv[i];
                            r2 *= mv[i];
                        }
                        Real *dn = drow + 3 * i;
                        const Real d0 = has_du ? a.rk_a * dn[0] + a.dt * r0 : a.dt * r0;
                        const Real d1 = has_du ? a.rk_a * dn[1] + a.dt * r1 : a.dt * r1;
                        const Real d2 = has_du ? a.rk_a * dn[2] + a.dt * r2 : a.dt * r2;
                        const Real u0 = q0[i] + a.rk_b * d0, u1 = q1[i] + a.rk_b * d1, u2 = q2[i] + a.rk_b * d2;
                        dn[0] = d0;
                        dn[1] = d1;
                        dn[2] = d2;
                        row[3 * i] = u0;
                        row[3 * i + 1] = u1;
                        row[3 * i + 2] = u2;
                        if (EXTRA && (flags & F_FILTER))
                        {
                            a.acc[g] += a.acc_c * (double)u0;
                            a.acc[g + 1] += a.acc_c * (double)u1;
                            a.acc[g + 2] += a.acc_c * (double)u2;
                        }
                    }
                }
                __syncwarp(); // the scratch is reused by the next round
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
