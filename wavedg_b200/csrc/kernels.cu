// Device kernels of libwdg_b200 (sm_100a).
//
// The hot kernel is `stage_kernel`: one pass over the state per RK stage that
// fuses what the reference does in eight separate loops per time derivative
// and two per RK stage (Div::action, FaceProlongator::action, EdgeFlux::action,
// FaceProlongator::t for interior and boundary faces, apply_bc_2d, the forcing
// add, MassMatrix::inv, and the low-storage RK update of wavedg/ode.hpp:66-93).
//
//   * A CTA owns tiles of E consecutive elements (E a multiple of 4) and loops
//     over them persistently.  Each tile's state block, RK register and
//     geometry (4 corners, neighbour table) are contiguous in HBM and are
//     staged into shared memory with cp.async.bulk (the TMA engine) on an
//     mbarrier, double-buffered so tile k+2 is in flight while k computes.
//   * The volume term is sum-factorised: every node forms its six contravariant
//     fluxes once in shared memory, then contracts n entries along each
//     direction with the 1-D derivative matrix held in registers.  The
//     matrices are n x n with n <= 9, far too small for tensor cores.
//   * Metrics are recomputed from the 4 corners (source/Element.cpp:21-27)
//     instead of streaming the reference's 18-doubles-per-node `op` table.
//   * Each element evaluates the upwind flux on its own faces with its own
//     outward normal; since C = n_x A0 + n_y A1 has eigenvalues {0, +-1},
//     |C| = C^2 and the reference's per-node 3x3 flux matrices
//     (source/EdgeFlux.cpp:7-139) collapse to a closed form.  Interior edges
//     are evaluated twice (once per side) and nothing is scattered, so no
//     face-trace array and no atomics are needed.
//   * Neighbour traces come from shared memory when the neighbour is in the
//     tile, otherwise from global memory (L2) with loads issued before the
//     volume work so their latency overlaps it.
//
// All bounded waits give up after a fixed number of polls, set a bit in the
// device error word and return; no kernel traps.
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstdio>
#include <mutex>
#include <vector>

#include "common.hpp"
#include "launch.hpp"
#include "wave_bc.cuh"

namespace wdg
{
    // ------------------------------------------------------------------ tables
    struct BasisTab
    {
        double x[kMaxN], w[kMaxN], D[kMaxN * kMaxN];     // GLL nodes, weights, D[l + n j] = phi_j'(x_l)
        double gx[kMaxN], gw[kMaxN], B[kMaxN * kMaxN];   // n-point Gauss-Legendre and B[q + n j] = phi_j(gx_q)
        float xf[kMaxN], wf[kMaxN], Df[kMaxN * kMaxN];
    };
    __constant__ BasisTab c_tab[kMaxN + 1];

    constexpr int kMaxThreads = 320; // threads per CTA of the stage kernel (launch bound)

    bool degree_supported(int n) { return n == 2 || n == 3 || n == 4 || n == 5 || n == 6 || n == 7 || n == 8 || n == 9; }

    int max_tile(int n) { return (kMaxThreads / (n + 8)) & ~3; }

    template <typename Real>
    size_t stage_smem_bytes(int n, int tile, int flags, int stages);

    // largest tile (multiple of 4, <= 512 threads) with which two CTAs of a
    // `stages`-deep pipeline share an SM
    int default_tile(int n, bool fp32, int stages)
    {
        const size_t budget = (227 * 1024) / 3 - 1024;
        for (int e = max_tile(n); e >= 4; e -= 4)
        {
            const size_t b = fp32 ? stage_smem_bytes<float>(n, e, F_RK, stages)
                                  : stage_smem_bytes<double>(n, e, F_RK, stages);
            if (b <= budget)
                return e;
        }
        return 4;
    }

    int upload_basis_tables(int device)
    {
        static std::mutex mu;
        static uint64_t done = 0;
        std::lock_guard<std::mutex> lock(mu);
        if (device < 0 || device >= 64)
            return fail(WDG_ERR_ARG, "device ordinal out of range");
        if (done & (1ull << device))
            return WDG_OK;
        std::vector<BasisTab> tab(kMaxN + 1);
        for (int n = kMinN; n <= kMaxN; ++n)
        {
            BasisTab &T = tab[n];
            gauss_lobatto(n, T.x, T.w);
            deriv_matrix(n, T.x, T.D);
            gauss_legendre(n, T.gx, T.gw);
            interp_matrix(n, T.x, n, T.gx, T.B);
            for (int k = 0; k < n; ++k)
            {
                T.xf[k] = (float)T.x[k];
                T.wf[k] = (float)T.w[k];
            }
            for (int k = 0; k < n * n; ++k)
                T.Df[k] = (float)T.D[k];
        }
        WDG_CUDA(cudaMemcpyToSymbol(c_tab, tab.data(), sizeof(BasisTab) * (kMaxN + 1)));
        done |= (1ull << device);
        return WDG_OK;
    }

    template <typename Real>
    struct Tab;
    template <>
    struct Tab<double>
    {
        static __device__ __forceinline__ double x(int n, int i) { return c_tab[n].x[i]; }
        static __device__ __forceinline__ double w(int n, int i) { return c_tab[n].w[i]; }
        static __device__ __forceinline__ double D(int n, int k) { return c_tab[n].D[k]; }
    };
    template <>
    struct Tab<float>
    {
        static __device__ __forceinline__ float x(int n, int i) { return c_tab[n].xf[i]; }
        static __device__ __forceinline__ float w(int n, int i) { return c_tab[n].wf[i]; }
        static __device__ __forceinline__ float D(int n, int k) { return c_tab[n].Df[k]; }
    };

    __constant__ int c_from[4] = {0, 1, 3, 0};
    __constant__ int c_to[4] = {1, 2, 2, 3};

    // --------------------------------------------------------- PTX helpers
    __device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

    __device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
    {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    }
    __device__ __forceinline__ void fence_mbar_init()
    {
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
    {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                     : "memory");
    }
    // 1-D bulk copy global -> shared through the TMA unit; dst, src and bytes
    // are multiples of 16 (checked by the host before use_tma is set)
    __device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
    {
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                smem_u32(dst)),
            "l"(src), "r"(bytes), "r"(smem_u32(bar))
            : "memory");
    }
    __device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
    {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        return ok != 0;
    }
    // try_wait with a suspend-time hint: the thread sleeps until the phase
    // completes or the hint (ns) runs out, instead of spinning on the issue port
    __device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t *bar, uint32_t parity)
    {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(smem_u32(bar)), "r"(parity), "r"(100000u)
            : "memory");
        return ok != 0;
    }
    __device__ __forceinline__ uint64_t globaltimer_ns()
    {
        uint64_t t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        return t;
    }
    // bounded wait: gives up after limit_ns of wall time (the copies it waits for take
    // microseconds; the limit only guards against a lost completion).  Stage launches pass the
    // handle's limit (StageArgs::wait_ns, 2 s unless set); other kernels use the default.
    __device__ __forceinline__ uint64_t wait_limit(unsigned long long ns) { return ns ? ns : kWaitLimitNs; }
    __device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint64_t limit_ns = kWaitLimitNs)
    {
        if (mbar_try_wait(bar, parity))
            return true;
        const uint64_t t0 = globaltimer_ns();
        for (;;)
        {
            if (mbar_try_wait_sleep(bar, parity))
                return true;
            if (globaltimer_ns() - t0 > limit_ns)
                return false;
        }
    }

    // ------------------------------------------------------------- geometry
    // QuadElement::jacobian (source/Element.cpp:21-27) at (xi, eta):
    // J = [x_xi, y_xi, x_eta, y_eta]; corners c = (x0,y0, x1,y1, x2,y2, x3,y3)
    template <typename Real>
    __device__ __forceinline__ void jacobian(const double *c, Real xi, Real eta, Real J[4])
    {
        J[0] = Real(0.25) * ((Real(1) - eta) * Real(c[2] - c[0]) + (Real(1) + eta) * Real(c[4] - c[6]));
        J[1] = Real(0.25) * ((Real(1) - eta) * Real(c[3] - c[1]) + (Real(1) + eta) * Real(c[5] - c[7]));
        J[2] = Real(0.25) * ((Real(1) - xi) * Real(c[6] - c[0]) + (Real(1) + xi) * Real(c[4] - c[2]));
        J[3] = Real(0.25) * ((Real(1) - xi) * Real(c[7] - c[1]) + (Real(1) + xi) * Real(c[5] - c[3]));
    }

    // outward unit normal and measure (= length / 2) of side f of an element
    // (StraightEdge, wavedg/Edge.hpp:107-122)
    __device__ __forceinline__ void side_normal(const double *c, int f, double &nx, double &ny, double &meas)
    {
        const int a = c_from[f], b = c_to[f];
        const double dx = c[2 * b] - c[2 * a], dy = c[2 * b + 1] - c[2 * a + 1];
        const double s = hypot(dx, dy);
        const double sgn = (f == 2 || f == 3) ? -1.0 : 1.0;
        nx = sgn * dy / s;
        ny = -sgn * dx / s;
        meas = s / 2;
    }

    // upwind numerical flux through a face with outward normal n, weight
    // h = w_k * meas / 2:  r -= h [C (q + x) + |C| (q - x)],  |C| = C^2
    template <typename Real>
    __device__ __forceinline__ void upwind(Real nx, Real ny, Real h, const Real q[3], const Real x[3], Real r[3])
    {
        const Real sp = q[0] + x[0], su = q[1] + x[1], sv = q[2] + x[2];
        const Real jp = q[0] - x[0], ju = q[1] - x[1], jv = q[2] - x[2];
        const Real nj = nx * ju + ny * jv;
        r[0] -= h * (nx * su + ny * sv + jp);
        r[1] -= h * (nx * sp + nx * nj);
        r[2] -= h * (ny * sp + ny * nj);
    }

    // face-node k of side f -> node (i, j):  f0 (k,0)  f1 (n-1,k)  f2 (k,n-1)  f3 (0,k)
    // (the reference's mapV2E, source/FaceProlongator.cpp:508-514)
    __device__ __forceinline__ int face_node(int n, int f, int k)
    {
        const int i = (f == 0 || f == 2) ? k : (f == 1 ? n - 1 : 0);
        const int j = (f == 1 || f == 3) ? k : (f == 2 ? n - 1 : 0);
        return i + n * j;
    }

    // ------------------------------------------------------- stage kernel
    // per-thread asynchronous global -> shared copies (LDGSTS); used for the
    // neighbour traces, which are scattered 8-byte pieces unsuited to TMA
    template <int BYTES>
    __device__ __forceinline__ void cp_async(void *dst, const void *src)
    {
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_u32(dst)), "l"(src), "n"(BYTES)
                     : "memory");
    }
    __device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
    template <int PENDING>
    __device__ __forceinline__ void cp_async_wait()
    {
        asm volatile("cp.async.wait_group %0;" ::"n"(PENDING) : "memory");
    }

    __device__ __forceinline__ void bulk_s2g(void *dst, const void *src, uint32_t bytes)
    {
        asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_u32(src)),
                     "r"(bytes)
                     : "memory");
    }
    __device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
    __device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
    __device__ __forceinline__ void bulk_wait_read1() { asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory"); }
    __device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
    __device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

    template <int N>
    __device__ __forceinline__ int partner_stride(uint32_t byte)
    {
        const uint32_t c = byte & 3u;
        return (c == 0) ? 3 : (c == 1) ? -3 : (c == 2) ? 3 * N : -3 * N;
    }

    // Shared-memory layout of one CTA (E elements per tile, ND = 3 n^2 values per
    // element, NF = 4 n face nodes per element):
    //   [S <= 4 mbarriers][buffer 0 .. S-1][halo 0][halo 1][face flux][G][Rx][Ms][basis x, w]
    //   buffer    = u tile | du tile (stages > 0) | corners (8 doubles) | partner bases (int4) | codes (u32)
    //   halo      = (E, NF, 3) neighbour traces from outside the tile, filled by cp.async
    //   face flux = (E, NF, 3) upwind flux contribution of every face node
    //   G, Rx     = (E, 3, n^2) eta-fluxes and xi-derivatives
    //   Ms        = (E, n^2) inverse diagonal mass
    template <typename Real>
    size_t stage_smem_bytes(int n, int tile, int flags, int stages)
    {
        const size_t nd = 3 * (size_t)n * n;
        const bool du = (flags & F_RK) != 0; // RK launches stage du' in place, whether or not they read du
        const size_t ub = (size_t)tile * nd * sizeof(Real);
        const size_t bufb = ub * (du ? 2 : 1) + (size_t)tile * 84;
        const size_t face = (size_t)tile * 12 * n * sizeof(Real);
        const size_t minv = (size_t)tile * n * n * sizeof(Real);
        const size_t basis = (2 * n * sizeof(Real) + 15) & ~size_t(15);
        return 32 + (size_t)stages * bufb + 3 * face + 2 * ub + minv + basis;
    }

    // n line threads (one per row / column) and 8 face threads (two per side) per element
    int stage_threads(int n, int tile) { return (n + 8) * tile; }

    template <int N, typename Real, bool RK>
    __global__ void __launch_bounds__(kMaxThreads, 2) stage_kernel(const StageArgs<Real> a)
    {
        constexpr int NN = N * N, ND = 3 * NN, NF = 4 * N;
        const int E = a.tile;
        const int flags = a.flags;
        const bool has_du = RK && (flags & F_READ_DU);
        const int ntiles = (a.nel + E - 1) / E;
        const int G = gridDim.x;
        const int TL = N * E; // line threads; the next 8 E threads are face threads

        extern __shared__ __align__(128) unsigned char smem[];
        const int ub = E * ND * (int)sizeof(Real);
        // RK launches keep a du tile in every buffer: stage 0 does not read du but
        // still stages du' there for the bulk store
        const int bufb = ub * (RK ? 2 : 1) + E * 84;
        const int gofs = ub * (RK ? 2 : 1); // geometry block within a buffer
        const int S = a.stages;             // pipeline depth: tiles in flight + 1
        uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
        unsigned char *buf0 = smem + 32;
        Real *halo = reinterpret_cast<Real *>(buf0 + S * bufb); // 2 x (E, NF, 3)
        Real *fc = halo + 2 * E * NF * 3;                       // (E, NF, 3)
        Real *Gs = fc + E * NF * 3;                             // (E, 3, NN)
        Real *Rx = Gs + 3 * NN * E;                             // (E, 3, NN)
        Real *Ms = Rx + 3 * NN * E;                             // (E, NN)
        Real *bx = Ms + NN * E;                                 // nodes (N), weights (N)
        const Real *xs = bx, *ws = bx + N;

        const int t = threadIdx.x;
        // line role: t = e * N + m -> element e, row (phase 1) / column (phase 2) m, all 3 components
        const bool line = t < TL;
        const int le = t / N, lm = t - (t / N) * N;
        // face role: t - TL = (fe * 4 + ff) * 2 + fh -> nodes fh, fh + 2, ... of side ff of element fe
        const bool face = !line;
        const int fe = (t - TL) >> 3, ff = ((t - TL) >> 1) & 3, fh = (t - TL) & 1;

        if (t == 0)
        {
            for (int q = 0; q < S; ++q)
                mbar_init(&bars[q], 1);
            fence_mbar_init();
        }
        if (t < 2 * N)
            bx[t] = (t < N) ? Tab<Real>::x(N, t) : Tab<Real>::w(N, t - N);

        auto tma_tile = [&](int k) { return a.use_tma && (k + 1) * E <= a.nel; };
        auto issue_tma = [&](int k, int b)
        {
            if (k >= ntiles || !tma_tile(k))
                return;
            const size_t el0 = (size_t)k * E;
            unsigned char *base = buf0 + b * bufb;
            mbar_expect_tx(&bars[b], (uint32_t)(ub * (has_du ? 2 : 1) + E * 84));
            bulk_g2s(base, a.u + el0 * ND, (uint32_t)ub, &bars[b]);
            if (has_du)
                bulk_g2s(base + ub, a.du + el0 * ND, (uint32_t)ub, &bars[b]);
            unsigned char *g = base + gofs;
            bulk_g2s(g, a.corners + 8 * el0, (uint32_t)(64 * E), &bars[b]);
            bulk_g2s(g + 64 * E, a.fbase + el0, (uint32_t)(16 * E), &bars[b]);
            bulk_g2s(g + 80 * E, a.fcode + el0, (uint32_t)(4 * E), &bars[b]);
        };
        // partner base of this face thread's side in tile k (-1: none), and its stride
        auto load_partner = [&](int k, int &base, int &stride)
        {
            base = -1;
            stride = 0;
            const int el = k * E + fe;
            if (!face || fe >= E || k >= ntiles || el >= a.nel || !(flags & F_INT))
                return;
            const uint32_t byte = (__ldg(a.fcode + el) >> (8 * ff)) & 0xffu;
            if (byte & 0x80u)
                return;
            base = __ldg(reinterpret_cast<const int *>(a.fbase + el) + ff);
            stride = partner_stride<N>(byte);
        };
        // start copying the side's exterior traces for tile k (those outside the tile) into halo slot hb
        auto issue_halo = [&](int k, int hb, int base, int stride)
        {
            if (base < 0 || k >= ntiles)
                return;
            const int lo = k * E * ND, hi = min(k * E + E, a.nel) * ND;
            Real *dst = halo + ((hb * E + fe) * NF + ff * N) * 3;
#pragma unroll
            for (int kk = 0; kk < N; ++kk)
            {
                if ((kk & 1) != fh)
                    continue;
                const int off = base + kk * stride;
                if (off >= lo && off < hi)
                    continue; // read from the staged tile instead
                if (off < 0 || off + 3 > (a.nread > 0 ? a.nread : a.nel * ND))
                {
                    atomicOr(a.err, 2u);
                    continue;
                }
                cp_async<sizeof(Real)>(dst + 3 * kk, a.u + off);
                cp_async<sizeof(Real)>(dst + 3 * kk + 1, a.u + off + 1);
                cp_async<sizeof(Real)>(dst + 3 * kk + 2, a.u + off + 2);
            }
        };

        // Pipeline: tile T_m (the m-th tile of this CTA) lives in buffer m % S.  Its bulk
        // load is issued at the end of iteration m - S + 1, into the buffer of tile
        // m - S whose bulk store has had a full iteration to drain, so S - 2 tiles are
        // in flight ahead of the one being computed.
        int bad = 0;
        if (t == 0)
            for (int q = 0; q < S - 1; ++q)
                issue_tma(blockIdx.x + q * G, q);
        int pbase, pstride;
        load_partner(blockIdx.x, pbase, pstride);
        issue_halo(blockIdx.x, 0, pbase, pstride);
        cp_async_commit();
        load_partner(blockIdx.x + G, pbase, pstride); // issued at the top of iteration 0
        __syncthreads(); // mbarrier initialisation and the basis table are visible

        int it = 0;
        for (int k = blockIdx.x; k < ntiles; k += G, ++it)
        {
            const int b = it % S; // data buffer of this tile
            const int h = it & 1; // halo slot of this tile
            const int el0 = k * E;
            const int ne = min(E, a.nel - el0);
            Real *us = reinterpret_cast<Real *>(buf0 + b * bufb);
            Real *dus = reinterpret_cast<Real *>(buf0 + b * bufb + ub);
            const double *cs = reinterpret_cast<const double *>(buf0 + b * bufb + gofs);
            const int *ps = reinterpret_cast<const int *>(cs + 8 * E);            // (4, E) partner bases
            const uint32_t *is = reinterpret_cast<const uint32_t *>(ps + 4 * E); // (E) codes
            const bool tin = tma_tile(k);
            const bool tout = RK && a.tma_out && (k + 1) * E <= a.nel;

            // every thread waits (sleeping) on this tile's bulk loads
            if (tin && !mbar_wait(&bars[b], (it / S) & 1, wait_limit(a.wait_ns)))
                bad = 1;
            if (!tin)
            {
                for (int q = t; q < ne * ND; q += blockDim.x)
                    us[q] = a.u[(size_t)el0 * ND + q];
                if (has_du)
                    for (int q = t; q < ne * ND; q += blockDim.x)
                        dus[q] = a.du[(size_t)el0 * ND + q];
                double *cw = const_cast<double *>(cs);
                for (int q = t; q < ne * 8; q += blockDim.x)
                    cw[q] = a.corners[8 * (size_t)el0 + q];
                for (int q = t; q < ne; q += blockDim.x)
                {
                    reinterpret_cast<int4 *>(const_cast<int *>(ps))[q] = a.fbase[el0 + q];
                    const_cast<uint32_t *>(is)[q] = a.fcode[el0 + q];
                }
                __syncthreads();
            }

            // ---------------- phase 1: xi-lines and face fluxes
            if (line && le < ne)
            {
                // row j = lm of element le.  Contravariant fluxes (source/Div.cpp:5-53 for the
                // wave system): F = W (y_eta u - x_eta v, y_eta p, -x_eta p),
                // G = W (-y_xi u + x_xi v, -y_xi p, x_xi p); x_xi, y_xi are constant along a
                // row of the bilinear map, x_eta, y_eta vary linearly with xi.
                const double *c = cs + 8 * le;
                const Real eta = xs[lm], wj = ws[lm];
                const Real Xxi = Real(0.25) * ((Real(1) - eta) * Real(c[2] - c[0]) + (Real(1) + eta) * Real(c[4] - c[6]));
                const Real Yxi = Real(0.25) * ((Real(1) - eta) * Real(c[3] - c[1]) + (Real(1) + eta) * Real(c[5] - c[7]));
                const Real ex0 = Real(c[6] - c[0]), ex1 = Real(c[4] - c[2]);
                const Real ey0 = Real(c[7] - c[1]), ey1 = Real(c[5] - c[3]);
                const Real *row = us + le * ND + 3 * N * lm;
                Real *g0 = Gs + le * 3 * NN + N * lm;
                Real *m0 = Ms + le * NN + N * lm;
                // xi-contraction du(i, j) += sum_l D(l, i) F(l, j) (div_2d_c, source/Div.cpp:131-179),
                // accumulated l-outer so the 3 N sums are independent
                Real ap[N], au[N], av[N];
#pragma unroll
                for (int i = 0; i < N; ++i)
                    ap[i] = au[i] = av[i] = 0;
#pragma unroll
                for (int l = 0; l < N; ++l)
                {
                    const Real xl = xs[l];
                    const Real Xeta = Real(0.25) * ((Real(1) - xl) * ex0 + (Real(1) + xl) * ex1);
                    const Real Yeta = Real(0.25) * ((Real(1) - xl) * ey0 + (Real(1) + xl) * ey1);
                    const Real W = ws[l] * wj;
                    const Real p = row[3 * l], u = row[3 * l + 1], v = row[3 * l + 2];
                    const Real WYe = Yeta * W, WXe = Xeta * W, WYx = Yxi * W, WXx = Xxi * W;
                    const Real Fp = WYe * u - WXe * v;
                    const Real Fu = WYe * p;
                    const Real Fv = -WXe * p;
                    g0[l] = -WYx * u + WXx * v;
                    g0[NN + l] = -WYx * p;
                    g0[2 * NN + l] = WXx * p;
                    // MassMatrix<true>: w_i w_j detJ (source/MassMatrix.cpp:6-28)
                    m0[l] = Real(1) / (W * (Xxi * Yeta - Yxi * Xeta));
#pragma unroll
                    for (int i = 0; i < N; ++i)
                    {
                        const Real d = Tab<Real>::D(N, l + N * i);
                        ap[i] += d * Fp;
                        au[i] += d * Fu;
                        av[i] += d * Fv;
                    }
                }
                Real *r0 = Rx + le * 3 * NN + N * lm;
#pragma unroll
                for (int i = 0; i < N; ++i)
                {
                    r0[i] = ap[i];
                    r0[NN + i] = au[i];
                    r0[2 * NN + i] = av[i];
                }
            }
            if (face)
            {
                // the next tile's traces start now; this tile's (started one iteration earlier) have landed
                issue_halo(k + G, h ^ 1, pbase, pstride);
                cp_async_commit();
                cp_async_wait<1>();
                load_partner(k + 2 * G, pbase, pstride);
                if (fe < ne)
                {
                    const uint32_t byte = (is[fe] >> (8 * ff)) & 0xffu;
                    const bool bnd = (byte & 0x80u) != 0;
                    Real *o = fc + (fe * NF + ff * N) * 3;
                    if (bnd ? (flags & F_BND) : (flags & F_INT))
                    {
                        // outward normal and measure of the side (StraightEdge, wavedg/Edge.hpp:107-122)
                        const double *c = cs + 8 * fe;
                        const int p0 = c_from[ff], p1 = c_to[ff];
                        const double dx = c[2 * p1] - c[2 * p0], dy = c[2 * p1 + 1] - c[2 * p0 + 1];
                        const double s2 = dx * dx + dy * dy, rs = rsqrt(s2);
                        const double sgn = (ff >= 2) ? -1.0 : 1.0;
                        const Real nx = (Real)(sgn * dy * rs), ny = (Real)(-sgn * dx * rs);
                        const Real hm = (Real)(0.25 * s2 * rs); // half the side measure
                        const int code = (int)((byte >> 3) & 3u);
                        const int base = ps[4 * fe + ff] - el0 * ND, stride = partner_stride<N>(byte);
                        const Real *hb = halo + ((h * E + fe) * NF + ff * N) * 3;
                        // own face node kk: (kk,0) (n-1,kk) (kk,n-1) (0,kk) for sides 0..3
                        const int o0 = (ff == 1) ? 3 * (N - 1) : (ff == 2) ? 3 * N * (N - 1) : 0;
                        const int os = (ff == 0 || ff == 2) ? 3 : 3 * N;
                        const Real *own = us + fe * ND + o0;
#pragma unroll
                        for (int kk = 0; kk < N; ++kk)
                        {
                            if ((kk & 1) != fh)
                                continue;
                            const Real q[3] = {own[kk * os], own[kk * os + 1], own[kk * os + 2]};
                            Real x[3];
                            if (bnd)
                                exterior<Real>(code, nx, ny, q, x);
                            else
                            {
                                const int loc = base + kk * stride;
                                const Real *src = (loc >= 0 && loc < ne * ND) ? us + loc : hb + 3 * kk;
                                x[0] = src[0];
                                x[1] = src[1];
                                x[2] = src[2];
                            }
                            Real fl[3] = {0, 0, 0};
                            upwind<Real>(nx, ny, Tab<Real>::w(N, kk) * hm, q, x, fl);
                            o[3 * kk] = fl[0];
                            o[3 * kk + 1] = fl[1];
                            o[3 * kk + 2] = fl[2];
                        }
                    }
                    else
                    {
#pragma unroll
                        for (int kk = 0; kk < N; ++kk)
                            if ((kk & 1) == fh)
                            {
                                o[3 * kk] = 0;
                                o[3 * kk + 1] = 0;
                                o[3 * kk + 2] = 0;
                            }
                    }
                }
            }
            if (__syncthreads_or(bad))
            {
                // leave after bounded waits for the copies still in flight
                if (t == 0)
                {
                    atomicOr(a.err, 1u);
                    for (int q = 1; q < S - 1; ++q)
                    {
                        const int kq = k + q * G;
                        if (kq < ntiles && tma_tile(kq))
                            mbar_wait(&bars[(it + q) % S], ((it + q) / S) & 1, wait_limit(a.wait_ns));
                    }
                    bulk_wait_all();
                }
                cp_async_wait<0>();
                return;
            }

            // ---------------- phase 2: eta-lines, face terms, M^{-1}, epilogue (in place)
            if (line && le < ne)
            {
                // column i = lm of element le: du(i, j) += sum_l D(l, j) G(i, l)
                const int i = lm;
                const Real *gc = Gs + le * 3 * NN + i;
                const Real *rc = Rx + le * 3 * NN + i;
                // eta-contraction, l-outer: 3 N independent sums seeded with the xi part
                Real sp[N], su[N], sv[N];
#pragma unroll
                for (int j = 0; j < N; ++j)
                {
                    sp[j] = (flags & F_VOL) ? rc[N * j] : Real(0);
                    su[j] = (flags & F_VOL) ? rc[NN + N * j] : Real(0);
                    sv[j] = (flags & F_VOL) ? rc[2 * NN + N * j] : Real(0);
                }
                if (flags & F_VOL)
                {
#pragma unroll
                    for (int l = 0; l < N; ++l)
                    {
                        const Real gp = gc[N * l], gu = gc[NN + N * l], gv = gc[2 * NN + N * l];
#pragma unroll
                        for (int j = 0; j < N; ++j)
                        {
                            const Real d = Tab<Real>::D(N, l + N * j);
                            sp[j] += d * gp;
                            su[j] += d * gu;
                            sv[j] += d * gv;
                        }
                    }
                }
                const Real *fce = fc + le * NF * 3;
                const Real *mc = Ms + le * NN + i;
                Real *uc = us + le * ND + 3 * i;
                Real *duc = dus + le * ND + 3 * i;
                const size_t gb = (size_t)(el0 + le) * ND + 3 * i;
#pragma unroll
                for (int j = 0; j < N; ++j)
                {
                    Real r[3] = {sp[j], su[j], sv[j]};
                    // face-flux slots (side * N + face node) through node (i, j)
                    int sl[2] = {-1, -1}, ns = 0;
                    if (j == 0) sl[ns++] = 0 * N + i;
                    if (j == N - 1) sl[ns++] = 2 * N + i;
                    if (i == N - 1 && ns < 2) sl[ns++] = 1 * N + j;
                    if (i == 0 && ns < 2) sl[ns++] = 3 * N + j;
                    for (int q = 0; q < ns; ++q)
                    {
                        const Real *o = fce + 3 * sl[q];
                        r[0] += o[0];
                        r[1] += o[1];
                        r[2] += o[2];
                    }
                    if (flags & F_FORCE)
                        for (int d = 0; d < 3; ++d)
                            r[d] += a.F[gb + 3 * N * j + d] * a.fscale;
                    if (flags & F_MINV)
                    {
                        const Real m = mc[N * j];
                        r[0] *= m;
                        r[1] *= m;
                        r[2] *= m;
                    }
                    Real *un = uc + 3 * N * j;
                    if (RK)
                    {
                        Real *dn = duc + 3 * N * j;
#pragma unroll
                        for (int d = 0; d < 3; ++d)
                        {
                            const Real dv = has_du ? a.rk_a * dn[d] + a.dt * r[d] : a.dt * r[d];
                            dn[d] = dv;
                            un[d] = un[d] + a.rk_b * dv;
                        }
                    }
                    else
                    {
                        un[0] = r[0];
                        un[1] = r[1];
                        un[2] = r[2];
                    }
                }
                if (tout)
                    fence_async_smem();
            }

            // ---------------- end of tile: write back, refill the previous tile's buffer
            __syncthreads();
            const bool filter = RK && (flags & F_FILTER);
            if (tout && t == 0)
            {
                bulk_s2g(a.out + (size_t)el0 * ND, us, (uint32_t)ub);
                bulk_s2g(a.du + (size_t)el0 * ND, dus, (uint32_t)ub);
                bulk_commit();
            }
            if (!tout || filter)
            {
                const size_t g0 = (size_t)el0 * ND;
                for (int q = t; q < ne * ND; q += blockDim.x)
                {
                    const Real v = us[q];
                    if (!tout)
                    {
                        if (RK)
                        {
                            a.out[g0 + q] = v;
                            a.du[g0 + q] = dus[q];
                        }
                        else
                            a.out[g0 + q] = (flags & F_ACCUM) ? a.out[g0 + q] + v : v;
                    }
                    if (filter)
                        a.acc[g0 + q] += a.acc_c * (double)v;
                }
                __syncthreads();
            }
            if (t == 0)
            {
                // the buffer refilled next held tile it+1-S+... i.e. tile it-1 (S >= 2): its
                // store (committed one iteration ago) must have finished reading shared memory
                if (tout)
                    bulk_wait_read1();
                else
                    bulk_wait_read();
                issue_tma(k + (S - 1) * G, (it + S - 1) % S);
            }
        }
        cp_async_wait<0>();
        if (t == 0)
            bulk_wait_all();
    }

    // ------------------------------------------------ warp-per-element kernel
    // A warp owns EPW = 32 / n^2 elements (n <= 5) or one element with NPL =
    // ceil(n^2 / 32) nodes per lane (n >= 6); every lane holds whole nodes.
    //   * the node's state, RK register, the element's 4 corners and its face
    //     table come straight from global memory in coalesced loads; face lanes
    //     issue the loads of their partner's trace (L2) before any arithmetic;
    //   * metrics and the six contravariant fluxes are formed per node and
    //     exchanged through a per-warp scratch in shared memory (__syncwarp, no
    //     CTA barrier); the 1-D derivative columns of the lane sit in registers;
    //   * the upwind flux, forcing, M^{-1} and the RK update finish in registers
    //     and are stored coalesced.
    // Warps never wait for one another, so memory latency is covered by the many
    // warps resident per SM.
    template <int N>
    struct WarpShape
    {
        static constexpr int NN = N * N;
        static constexpr int EPW = (NN <= 32) ? 32 / NN : 1;
        static constexpr int NPL = (NN <= 32) ? 1 : (NN + 31) / 32;
    };
    constexpr int kWarpThreads = 256;

    template <typename Real>
    size_t warp_smem_bytes(int n)
    {
        const int nn = n * n, epw = (nn <= 32) ? 32 / nn : 1;
        const size_t dtab = ((size_t)nn * sizeof(Real) + 15) & ~size_t(15);
        return dtab + (size_t)(kWarpThreads / 32) * epw * nn * 6 * sizeof(Real);
    }

    template <int N, typename Real, bool RK>
    __global__ void __launch_bounds__(kWarpThreads, 3) warp_stage_kernel(const StageArgs<Real> a)
    {
        constexpr int NN = N * N, EPW = WarpShape<N>::EPW, NPL = WarpShape<N>::NPL;
        const int flags = a.flags;
        const bool has_du = RK && (flags & F_READ_DU);
        extern __shared__ __align__(16) unsigned char wsmem[];
        Real *Dsm = reinterpret_cast<Real *>(wsmem);
        Real *X = reinterpret_cast<Real *>(wsmem + ((NN * sizeof(Real) + 15) & ~size_t(15))) +
                  (threadIdx.x >> 5) * (EPW * NN * 6); // this warp's scratch: [slot][6][NN]
        if (NPL > 1)
        {
            for (int q = threadIdx.x; q < NN; q += blockDim.x)
                Dsm[q] = Tab<Real>::D(N, q);
            __syncthreads();
        }
        const int lane = threadIdx.x & 31;
        const int el_base = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * EPW;
        if (el_base >= a.nel)
            return;

        int node[NPL], slot[NPL], el[NPL];
        bool act[NPL];
#pragma unroll
        for (int p = 0; p < NPL; ++p)
        {
            node[p] = (NPL == 1) ? lane % NN : lane + 32 * p;
            slot[p] = (NPL == 1) ? lane / NN : 0;
            el[p] = el_base + slot[p];
            act[p] = ((NPL == 1) ? (lane < EPW * NN) : (node[p] < NN)) && el[p] < a.nel;
        }
        // derivative columns D(., i), D(., j) of a single-node lane
        Real Di[NPL == 1 ? N : 1], Dj[NPL == 1 ? N : 1];
        if (NPL == 1)
        {
            const int i = node[0] % N, j = node[0] / N;
#pragma unroll
            for (int l = 0; l < (NPL == 1 ? N : 1); ++l)
            {
                Di[l] = Tab<Real>::D(N, l + N * i);
                Dj[l] = Tab<Real>::D(N, l + N * j);
            }
        }

        // ---- loads: node state, RK register, side inputs, partner traces
        Real q[NPL][3], dv[NPL][3], xf[NPL][2][3], Fv[NPL][3], ov[NPL][3];
        double accv[NPL][3];
        int nfc[NPL], fcs[NPL][2], fck[NPL][2];
        uint32_t fbyte[NPL][2];
#pragma unroll
        for (int p = 0; p < NPL; ++p)
        {
            nfc[p] = 0;
            if (!act[p])
                continue;
            const size_t g = ((size_t)el[p] * NN + node[p]) * 3;
#pragma unroll
            for (int c = 0; c < 3; ++c)
            {
                q[p][c] = a.u[g + c];
                dv[p][c] = has_du ? a.du[g + c] : Real(0);
                Fv[p][c] = (flags & F_FORCE) ? a.F[g + c] : Real(0);
                ov[p][c] = (!RK && (flags & F_ACCUM)) ? a.out[g + c] : Real(0);
                accv[p][c] = (RK && (flags & F_FILTER)) ? a.acc[g + c] : 0.0;
            }
            const int i = node[p] % N, j = node[p] / N;
            if (j == 0) { fcs[p][nfc[p]] = 0; fck[p][nfc[p]++] = i; }
            if (i == N - 1) { fcs[p][nfc[p]] = 1; fck[p][nfc[p]++] = j; }
            if (j == N - 1 && nfc[p] < 2) { fcs[p][nfc[p]] = 2; fck[p][nfc[p]++] = i; }
            if (i == 0 && nfc[p] < 2) { fcs[p][nfc[p]] = 3; fck[p][nfc[p]++] = j; }
            if (nfc[p] == 0)
                continue;
            const int4 fb = a.fbase[el[p]];
            const uint32_t code = a.fcode[el[p]];
#pragma unroll
            for (int s = 0; s < 2; ++s)
            {
                if (s >= nfc[p])
                    continue;
                const int f = fcs[p][s];
                const uint32_t byte = (code >> (8 * f)) & 0xffu;
                fbyte[p][s] = byte;
                if ((byte & 0x80u) || !(flags & F_INT))
                    continue;
                const int off = ((f == 0) ? fb.x : (f == 1) ? fb.y : (f == 2) ? fb.z : fb.w) +
                                fck[p][s] * partner_stride<N>(byte);
                if (off < 0 || off + 3 > (a.nread > 0 ? a.nread : a.nel * 3 * NN))
                {
                    atomicOr(a.err, 2u);
                    fbyte[p][s] = 0x40u; // skip this face
                    continue;
                }
                xf[p][s][0] = __ldg(a.u + off);
                xf[p][s][1] = __ldg(a.u + off + 1);
                xf[p][s][2] = __ldg(a.u + off + 2);
            }
        }

        // ---- metrics and contravariant fluxes at the nodes (source/Div.cpp:5-53)
        Real minv[NPL];
#pragma unroll
        for (int p = 0; p < NPL; ++p)
        {
            minv[p] = 0;
            if (!act[p])
                continue;
            const int i = node[p] % N, j = node[p] / N;
            const double2 *cp = reinterpret_cast<const double2 *>(a.corners + 8 * (size_t)el[p]);
            double c[8];
#pragma unroll
            for (int k = 0; k < 4; ++k)
            {
                const double2 v = __ldg(cp + k);
                c[2 * k] = v.x;
                c[2 * k + 1] = v.y;
            }
            Real J[4];
            jacobian<Real>(c, Tab<Real>::x(N, i), Tab<Real>::x(N, j), J);
            const Real W = Tab<Real>::w(N, i) * Tab<Real>::w(N, j);
            const Real Yeta = J[3] * W, Xeta = J[2] * W, Yxi = J[1] * W, Xxi = J[0] * W;
            Real *x = X + slot[p] * (6 * NN) + node[p];
            x[0 * NN] = Yeta * q[p][1] - Xeta * q[p][2];
            x[1 * NN] = Yeta * q[p][0];
            x[2 * NN] = -Xeta * q[p][0];
            x[3 * NN] = -Yxi * q[p][1] + Xxi * q[p][2];
            x[4 * NN] = -Yxi * q[p][0];
            x[5 * NN] = Xxi * q[p][0];
            minv[p] = Real(1) / (W * (J[0] * J[3] - J[1] * J[2]));
        }
        __syncwarp();

        // ---- volume, faces, M^{-1}, epilogue
#pragma unroll
        for (int p = 0; p < NPL; ++p)
        {
            if (!act[p])
                continue;
            const int i = node[p] % N, j = node[p] / N;
            Real r[3] = {0, 0, 0};
            if (flags & F_VOL)
            {
                const Real *x = X + slot[p] * (6 * NN);
#pragma unroll
                for (int l = 0; l < N; ++l)
                {
                    const Real di = (NPL == 1) ? Di[l % (NPL == 1 ? N : 1)] : Dsm[l + N * i];
                    const Real dj = (NPL == 1) ? Dj[l % (NPL == 1 ? N : 1)] : Dsm[l + N * j];
                    const int fl = l + N * j, gl = i + N * l;
                    r[0] += di * x[fl] + dj * x[3 * NN + gl];
                    r[1] += di * x[NN + fl] + dj * x[4 * NN + gl];
                    r[2] += di * x[2 * NN + fl] + dj * x[5 * NN + gl];
                }
            }
            if (nfc[p] > 0)
            {
                const double *c = a.corners + 8 * (size_t)el[p];
#pragma unroll
                for (int s = 0; s < 2; ++s)
                {
                    if (s >= nfc[p])
                        continue;
                    const uint32_t byte = fbyte[p][s];
                    const bool bnd = (byte & 0x80u) != 0;
                    if ((byte == 0x40u) || (bnd ? !(flags & F_BND) : !(flags & F_INT)))
                        continue;
                    const int f = fcs[p][s];
                    const double dx = __ldg(c + 2 * c_to[f]) - __ldg(c + 2 * c_from[f]);
                    const double dy = __ldg(c + 2 * c_to[f] + 1) - __ldg(c + 2 * c_from[f] + 1);
                    const double s2 = dx * dx + dy * dy, rs = rsqrt(s2);
                    const double sgn = (f >= 2) ? -1.0 : 1.0;
                    const Real nx = (Real)(sgn * dy * rs), ny = (Real)(-sgn * dx * rs);
                    Real x[3];
                    if (bnd)
                        exterior<Real>((int)((byte >> 3) & 3u), nx, ny, q[p], x);
                    else
                    {
                        x[0] = xf[p][s][0];
                        x[1] = xf[p][s][1];
                        x[2] = xf[p][s][2];
                    }
                    upwind<Real>(nx, ny, Tab<Real>::w(N, fck[p][s]) * (Real)(0.25 * s2 * rs), q[p], x, r);
                }
            }
            if (flags & F_FORCE)
                for (int c = 0; c < 3; ++c)
                    r[c] += Fv[p][c] * a.fscale;
            if (flags & F_MINV)
                for (int c = 0; c < 3; ++c)
                    r[c] *= minv[p];
            const size_t g = ((size_t)el[p] * NN + node[p]) * 3;
            if (RK)
            {
#pragma unroll
                for (int c = 0; c < 3; ++c)
                {
                    const Real dn = has_du ? a.rk_a * dv[p][c] + a.dt * r[c] : a.dt * r[c];
                    const Real un = q[p][c] + a.rk_b * dn;
                    a.du[g + c] = dn;
                    a.out[g + c] = un;
                    if (flags & F_FILTER)
                        a.acc[g + c] = accv[p][c] + a.acc_c * (double)un;
                }
            }
            else
            {
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    a.out[g + c] = (flags & F_ACCUM) ? ov[p][c] + r[c] : r[c];
            }
        }
    }

} // namespace wdg

#include "stage_ws.cuh"
#include "stage_ws_batch.cuh"
#include "claw_kernels.cuh"

namespace wdg
{
    int ws_chunk_unit(int n) { return kWsConsumers * ws_epw(n); }

    cudaError_t launch_claw(int model, int n, int nv, const ClawArgs &a, cudaStream_t s)
    {
        return model == 0 ? launch_claw_m<ClawEuler>(n, nv, a, s) : launch_claw_m<ClawLinear>(n, nv, a, s);
    }
    cudaError_t launch_euler_face_flux(int n, int ne, const int *edges, const double *corners, const double *ub,
                                       double *fb, cudaStream_t s)
    {
        if (ne == 0)
            return cudaSuccess;
        const long long tot = (long long)n * ne;
        euler_face_flux_kernel<<<(unsigned)((tot + 127) / 128), 128, 0, s>>>(n, ne, edges, corners, ub, fb);
        return cudaGetLastError();
    }
    int ws_slot_bytes(int n, bool fp32, int chunk, bool extra, bool filter)
    {
        const bool staged = extra && (fp32 ? WsStage<float, true>::value : WsStage<double, true>::value);
        const WsSlot o = fp32 ? ws_slot<float>(n, chunk, staged) : ws_slot<double>(n, chunk, staged);
        return (staged && !filter) ? o.ab : o.bytes;
    }
    int ws_warp_scratch_bytes(int n, bool fp32)
    {
        return fp32 ? ws_layout<float>(n, 0, 0).warp_scratch : ws_layout<double>(n, 0, 0).warp_scratch;
    }
    size_t ws_smem_bytes(int n, bool fp32, int chunk, int ring)
    {
        return fp32 ? (size_t)ws_layout<float>(n, chunk, ring).total : (size_t)ws_layout<double>(n, chunk, ring).total;
    }
    int ws_default_chunk(int n, bool fp32)
    {
        const size_t budget = (227 * 1024) / 3 - 1024;
        const int unit = ws_chunk_unit(n);
        for (int r = 4; r >= 1; --r)
            if (ws_smem_bytes(n, fp32, r * unit, kWsDefaultRing) <= budget)
                return r * unit;
        return unit;
    }

    template <int N, typename Real, bool RK>
    static cudaError_t launch_warp_n(const StageArgs<Real> &a, cudaStream_t s)
    {
        auto kern = warp_stage_kernel<N, Real, RK>;
        const size_t smem = warp_smem_bytes<Real>(N);
        constexpr int EPW = WarpShape<N>::EPW;
        const long long warps = ((long long)a.nel + EPW - 1) / EPW;
        const int wpb = kWarpThreads / 32;
        const long long blocks = (warps + wpb - 1) / wpb;
        kern<<<(unsigned)blocks, kWarpThreads, smem, s>>>(a);
        return cudaGetLastError();
    }

    template <int N, typename Real, bool RK>
    static cudaError_t launch_stage_n(const StageArgs<Real> &a, int grid_limit, cudaStream_t s)
    {
        auto kern = stage_kernel<N, Real, RK>;
        const size_t smem = stage_smem_bytes<Real>(N, a.tile, a.flags | (RK ? F_RK : 0), a.stages);
        // the largest footprint any flag set can ask for, set once
        static bool attr_set[64] = {};
        int dev = 0;
        cudaGetDevice(&dev);
        if (!attr_set[dev & 63])
        {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
            if (e != cudaSuccess)
                return e;
            attr_set[dev & 63] = true;
        }
        const int threads = stage_threads(N, a.tile);
        const int ntiles = (a.nel + a.tile - 1) / a.tile;
        // resident CTAs per device for this (threads, smem); cached, one entry per device
        static int c_dev[64], c_threads[64], c_grid[64];
        static size_t c_smem[64];
        const int slot = dev & 63;
        if (c_threads[slot] != threads || c_smem[slot] != smem || c_dev[slot] != dev + 1)
        {
            int per_sm = 0, sms = 0;
            cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
            if (e != cudaSuccess)
                return e;
            e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            if (e != cudaSuccess)
                return e;
            c_grid[slot] = std::max(1, per_sm) * sms;
            c_threads[slot] = threads;
            c_smem[slot] = smem;
            c_dev[slot] = dev + 1;
        }
        int grid = c_grid[slot];
        if (grid_limit > 0)
            grid = std::min(grid, grid_limit);
        grid = std::min(grid, ntiles);
        kern<<<grid, threads, smem, s>>>(a);
        return cudaGetLastError();
    }

    template <typename Real>
    cudaError_t launch_stage(int n, bool rk, const StageArgs<Real> &a, int grid_limit, cudaStream_t s)
    {
        // a launch over part of the elements exists only in the warp-specialised family
        const bool partial = a.el_begin != 0 || (a.el_end > 0 && a.el_end != a.nel);
#define WDG_CASE(NV)                                                                       \
    case NV:                                                                               \
        if (a.family == 2 && rk && a.use_tma && a.tma_out && ws_fits<NV, Real>(a))         \
            return launch_ws_n<NV, Real>(a, grid_limit, s);                                \
        if (partial)                                                                       \
            return cudaErrorNotSupported;                                                  \
        if (a.family == 0)                                                                 \
            return rk ? launch_warp_n<NV, Real, true>(a, s) : launch_warp_n<NV, Real, false>(a, s); \
        return rk ? launch_stage_n<NV, Real, true>(a, grid_limit, s)                       \
                  : launch_stage_n<NV, Real, false>(a, grid_limit, s);
        switch (n)
        {
            WDG_CASE(2)
            WDG_CASE(3)
            WDG_CASE(4)
            WDG_CASE(5)
            WDG_CASE(6)
            WDG_CASE(7)
            WDG_CASE(8)
            WDG_CASE(9)
        default:
            return cudaErrorInvalidValue;
        }
#undef WDG_CASE
    }

    template cudaError_t launch_stage<double>(int, bool, const StageArgs<double> &, int, cudaStream_t);
    template cudaError_t launch_stage<float>(int, bool, const StageArgs<float> &, int, cudaStream_t);
    template size_t stage_smem_bytes<double>(int, int, int, int);
    template size_t stage_smem_bytes<float>(int, int, int, int);

    // --------------------------------------------- reference-layout kernels
    static inline int blocks_for(long long n, int threads) { return (int)std::min<long long>((n + threads - 1) / threads, 1 << 30); }

    // LobattoFaceProlongator::action (FaceProlongator.cpp:565-590): thread per (i, d, side, edge)
    __global__ void prolong_kernel(int n, int nedges, const int *__restrict__ edges, int interior,
                                   const double *__restrict__ u, double *__restrict__ uf)
    {
        const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
        const long long total = (long long)n * 3 * 2 * nedges;
        if (q >= total)
            return;
        const int i = (int)(q % n), d = (int)((q / n) % 3), s = (int)((q / (3 * n)) % 2);
        const int e = (int)(q / (6 * n));
        const int *E = edges + 5 * (size_t)e;
        double v = 0.0;
        if (s == 0 || interior)
        {
            const int el = E[2 * s], f = E[2 * s + 1];
            const int k = (s == 1 && E[4] < 0) ? (n - 1 - i) : i;
            v = u[d + 3 * ((size_t)el * n * n + face_node(n, f, k))];
        }
        uf[q] = v;
    }

    // LobattoFaceProlongator::t (FaceProlongator.cpp:650-672) as a gather:
    // thread per (d, node, el) adds the traces of the faces through its node
    __global__ void prolong_t_kernel(int n, int nel, const int *__restrict__ face_edge,
                                     const uint32_t *__restrict__ finfo, int want_boundary,
                                     const double *__restrict__ uf, double *__restrict__ u)
    {
        const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
        if (q >= 3LL * n * n * nel)
            return;
        const int d = (int)(q % 3);
        const long long nodeg = q / 3;
        const int node = (int)(nodeg % (n * n));
        const int el = (int)(nodeg / (n * n));
        const int i = node % n, j = node / n;
        const uint32_t info = finfo[el];
        double add = 0.0;
        for (int f = 0; f < 4; ++f)
        {
            int k;
            if (f == 0 && j == 0) k = i;
            else if (f == 1 && i == n - 1) k = j;
            else if (f == 2 && j == n - 1) k = i;
            else if (f == 3 && i == 0) k = j;
            else continue;
            const uint32_t byte = (info >> (8 * f)) & 0xffu;
            const bool bnd = (byte & 0x80u) != 0;
            if (bnd != (want_boundary != 0))
                continue;
            const int slot = face_edge[4 * (size_t)el + f];
            const int edge = slot >> 1, side = slot & 1;
            const int ie = (side == 1 && (byte & 4u)) ? (n - 1 - k) : k;
            add += uf[ie + n * (d + 3 * (side + 2 * (size_t)edge))];
        }
        u[q] += add;
    }

    // normal of an edge = outward normal of its first element's side (Edge.hpp:107-122)
    __device__ __forceinline__ void edge_normal(const double *corners, const int *E, double &nx, double &ny,
                                                double &meas)
    {
        side_normal(corners + 8 * (size_t)E[0], E[1], nx, ny, meas);
    }

    // EdgeFlux<true>::action (EdgeFlux.cpp:289-325): thread per (i, edge)
    __global__ void edge_flux_kernel(int n, int nedges, const int *__restrict__ edges,
                                     const double *__restrict__ corners, const double *ub, double *fb)
    {
        const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
        if (q >= (long long)n * nedges)
            return;
        const int i = (int)(q % n), e = (int)(q / n);
        double nx, ny, ms;
        edge_normal(corners, edges + 5 * (size_t)e, nx, ny, ms);
        double u0[3], u1[3], r[3] = {0, 0, 0};
        for (int d = 0; d < 3; ++d)
        {
            u0[d] = ub[i + n * (d + 3 * (0 + 2 * (size_t)e))];
            u1[d] = ub[i + n * (d + 3 * (1 + 2 * (size_t)e))];
        }
        upwind<double>(nx, ny, 0.5 * (c_tab[n].w[i] * ms), u0, u1, r);
        for (int d = 0; d < 3; ++d)
        {
            fb[i + n * (d + 3 * (0 + 2 * (size_t)e))] = r[d];
            fb[i + n * (d + 3 * (1 + 2 * (size_t)e))] = -r[d];
        }
    }

    // apply_bc_2d (WaveEquation.cpp:144-167): thread per (i, boundary edge)
    __global__ void apply_bc_kernel(int n, int nb, const int *__restrict__ edges, const int *__restrict__ codes,
                                    const double *__restrict__ corners, double *uB)
    {
        const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
        if (q >= (long long)n * nb)
            return;
        const int i = (int)(q % n), e = (int)(q / n);
        double nx, ny, ms;
        edge_normal(corners, edges + 5 * (size_t)e, nx, ny, ms);
        double v[3], x[3];
        for (int d = 0; d < 3; ++d)
            v[d] = uB[i + n * (d + 3 * (0 + 2 * (size_t)e))];
        exterior<double>(codes[e], nx, ny, v, x);
        for (int d = 0; d < 3; ++d)
            uB[i + n * (d + 3 * (1 + 2 * (size_t)e))] = x[d];
    }

    // MassMatrix<true>::action / ::inv (MassMatrix.cpp:55-82): thread per node
    __global__ void mass_kernel(int n, int nel, int n_var, const double *__restrict__ corners, const double *x,
                                double *y, int inverse)
    {
        const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
        if (q >= (long long)n * n * nel)
            return;
        const int node = (int)(q % (n * n));
        const int el = (int)(q / (n * n));
        const int i = node % n, j = node / n;
        double J[4];
        jacobian<double>(corners + 8 * (size_t)el, c_tab[n].x[i], c_tab[n].x[j], J);
        const double m = c_tab[n].w[i] * c_tab[n].w[j] * (J[0] * J[3] - J[1] * J[2]);
        for (int d = 0; d < n_var; ++d)
        {
            const size_t k = d + (size_t)n_var * q;
            y[k] = inverse ? x[k] / m : m * x[k];
        }
    }

    // physical coordinates at the GLL nodes or the Gauss-Legendre points
    // (QuadElement::physical_coordinates, source/Element.cpp:5-19)
    __global__ void coords_kernel(int n, int nel, const double *__restrict__ corners, int gl, double *xy)
    {
        const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
        if (q >= (long long)n * n * nel)
            return;
        const int node = (int)(q % (n * n));
        const int el = (int)(q / (n * n));
        const int i = node % n, j = node / n;
        const double xi = gl ? c_tab[n].gx[i] : c_tab[n].x[i];
        const double et = gl ? c_tab[n].gx[j] : c_tab[n].x[j];
        const double *c = corners + 8 * (size_t)el;
        const double b[4] = {0.25 * (1.0 - xi) * (1.0 - et), 0.25 * (1.0 + xi) * (1.0 - et),
                             0.25 * (1.0 + xi) * (1.0 + et), 0.25 * (1.0 - xi) * (1.0 + et)};
        double X = 0.0, Y = 0.0;
        for (int k = 0; k < 4; ++k)
        {
            X += c[2 * k] * b[k];
            Y += c[2 * k + 1] * b[k];
        }
        xy[2 * q] = X;
        xy[2 * q + 1] = Y;
    }

    // LinearFunctional2D::action (LinearFunctional.hpp:136-202): thread per
    // output node; f is either sampled (fq) or a sum of Gaussians (src)
    __global__ void linear_functional_kernel(int n, int nel, int n_var, const double *__restrict__ corners,
                                             const double *__restrict__ fq, int nsrc, const double *__restrict__ src,
                                             double scale, int comp, double *F)
    {
        const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
        if (q >= (long long)n * n * nel)
            return;
        const int node = (int)(q % (n * n));
        const int el = (int)(q / (n * n));
        const int i = node % n, j = node / n;
        const double *c = corners + 8 * (size_t)el;
        const BasisTab &T = c_tab[n];
        double acc[3] = {0, 0, 0};
        for (int l = 0; l < n; ++l)
            for (int k = 0; k < n; ++k)
            {
                const double xi = T.gx[k], et = T.gx[l];
                double J[4];
                jacobian<double>(c, xi, et, J);
                const double wgt = (J[0] * J[3] - J[1] * J[2]) * T.gw[k] * T.gw[l];
                const double bb = T.B[k + n * i] * T.B[l + n * j];
                if (fq)
                {
                    for (int d = 0; d < n_var; ++d)
                        acc[d] += fq[d + n_var * (k + n * (l + (size_t)n * el))] * wgt * bb;
                }
                else
                {
                    const double b4[4] = {0.25 * (1.0 - xi) * (1.0 - et), 0.25 * (1.0 + xi) * (1.0 - et),
                                          0.25 * (1.0 + xi) * (1.0 + et), 0.25 * (1.0 - xi) * (1.0 + et)};
                    double X = 0.0, Y = 0.0;
                    for (int m = 0; m < 4; ++m)
                    {
                        X += c[2 * m] * b4[m];
                        Y += c[2 * m + 1] * b4[m];
                    }
                    double s = 0.0;
                    for (int m = 0; m < nsrc; ++m)
                    {
                        const double dx = X - src[4 * m], dy = Y - src[4 * m + 1], sg = src[4 * m + 2];
                        s += src[4 * m + 3] * exp(-(dx * dx + dy * dy) / (2.0 * sg * sg));
                    }
                    acc[comp] += scale * s * wgt * bb;
                }
            }
        for (int d = 0; d < n_var; ++d)
            F[d + (size_t)n_var * q] = acc[d];
    }

    cudaError_t launch_prolong(const Geometry &g, int type, const double *u, double *uf, cudaStream_t s)
    {
        const int ne = (type == 0) ? g.nI : g.nB;
        const long long total = (long long)g.n * 6 * ne;
        if (total == 0)
            return cudaSuccess;
        prolong_kernel<<<blocks_for(total, 256), 256, 0, s>>>(g.n, ne, type == 0 ? g.edgesI : g.edgesB, type == 0,
                                                              u, uf);
        return cudaGetLastError();
    }
    cudaError_t launch_prolong_t(const Geometry &g, int type, const double *uf, double *u, cudaStream_t s)
    {
        const long long total = 3LL * g.n * g.n * g.nel;
        prolong_t_kernel<<<blocks_for(total, 256), 256, 0, s>>>(g.n, g.nel, g.face_edge, g.finfo, type == 1, uf, u);
        return cudaGetLastError();
    }
    cudaError_t launch_edge_flux(const Geometry &g, int type, const double *ub, double *fb, cudaStream_t s)
    {
        const int ne = (type == 0) ? g.nI : g.nB;
        const long long total = (long long)g.n * ne;
        if (total == 0)
            return cudaSuccess;
        edge_flux_kernel<<<blocks_for(total, 256), 256, 0, s>>>(g.n, ne, type == 0 ? g.edgesI : g.edgesB, g.corners,
                                                                ub, fb);
        return cudaGetLastError();
    }
    cudaError_t launch_apply_bc(const Geometry &g, double *uB, cudaStream_t s)
    {
        const long long total = (long long)g.n * g.nB;
        if (total == 0)
            return cudaSuccess;
        apply_bc_kernel<<<blocks_for(total, 256), 256, 0, s>>>(g.n, g.nB, g.edgesB, g.codesB, g.corners, uB);
        return cudaGetLastError();
    }
    cudaError_t launch_mass(const Geometry &g, int n_var, const double *x, double *y, bool inverse, cudaStream_t s)
    {
        const long long total = (long long)g.n * g.n * g.nel;
        mass_kernel<<<blocks_for(total, 256), 256, 0, s>>>(g.n, g.nel, n_var, g.corners, x, y, inverse ? 1 : 0);
        return cudaGetLastError();
    }
    cudaError_t launch_node_coords(const Geometry &g, bool gl, double *xy, cudaStream_t s)
    {
        const long long total = (long long)g.n * g.n * g.nel;
        coords_kernel<<<blocks_for(total, 256), 256, 0, s>>>(g.n, g.nel, g.corners, gl ? 1 : 0, xy);
        return cudaGetLastError();
    }
    cudaError_t launch_linear_functional(const Geometry &g, int n_var, const double *fq, double *F, cudaStream_t s)
    {
        const long long total = (long long)g.n * g.n * g.nel;
        linear_functional_kernel<<<blocks_for(total, 128), 128, 0, s>>>(g.n, g.nel, n_var, g.corners, fq, 0, nullptr,
                                                                        0.0, 0, F);
        return cudaGetLastError();
    }
    cudaError_t launch_load_gaussians(const Geometry &g, int nsrc, const double *src, double scale, int comp,
                                      double *F, cudaStream_t s)
    {
        const long long total = (long long)g.n * g.n * g.nel;
        linear_functional_kernel<<<blocks_for(total, 128), 128, 0, s>>>(g.n, g.nel, 3, g.corners, nullptr, nsrc, src,
                                                                        scale, comp, F);
        return cudaGetLastError();
    }

    // ----------------------------------------------------- element-wise
    template <typename A, typename B>
    __global__ void convert_kernel(const A *x, B *y, long long n)
    {
        for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
            y[q] = (B)x[q];
    }
    template <typename A, typename B>
    cudaError_t launch_convert(const A *x, B *y, long long n, cudaStream_t s)
    {
        if (n == 0)
            return cudaSuccess;
        convert_kernel<A, B><<<std::min(blocks_for(n, 256), 148 * 16), 256, 0, s>>>(x, y, n);
        return cudaGetLastError();
    }
    template cudaError_t launch_convert<double, float>(const double *, float *, long long, cudaStream_t);
    template cudaError_t launch_convert<float, double>(const float *, double *, long long, cudaStream_t);
    template cudaError_t launch_convert<double, double>(const double *, double *, long long, cudaStream_t);

    // WaveHoltz::S prologue (WaveHoltz.cpp:100-104): p <- x (in the stepping
    // precision), acc <- x * c (FP64)
    template <typename Real>
    __global__ void scale_into_kernel(const double *x, Real *p, double *acc, double c, long long n)
    {
        for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        {
            const double v = x[q];
            p[q] = (Real)v;
            acc[q] = v * c;
        }
    }
    template <typename Real>
    cudaError_t launch_scale_into(const double *x, Real *p, double *acc, double c, long long n, cudaStream_t s)
    {
        scale_into_kernel<Real><<<std::min(blocks_for(n, 256), 148 * 16), 256, 0, s>>>(x, p, acc, c, n);
        return cudaGetLastError();
    }
    template cudaError_t launch_scale_into<double>(const double *, double *, double *, double, long long, cudaStream_t);
    template cudaError_t launch_scale_into<float>(const double *, float *, double *, double, long long, cudaStream_t);

    // WaveHoltz::postprocess (WaveHoltz.cpp:123-145): H(0, i) = p_i, H(1, i) = -P_i / omega
    __global__ void wh_post_kernel(const double *W, const double *P, double omega, long long npts, double *H)
    {
        for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < npts; q += (long long)gridDim.x * blockDim.x)
        {
            H[2 * q] = W[3 * q];
            H[2 * q + 1] = -1.0 / omega * P[3 * q];
        }
    }
    cudaError_t launch_wh_post(const double *W, const double *P, double omega, long long npts, double *H, cudaStream_t s)
    {
        wh_post_kernel<<<std::min(blocks_for(npts, 256), 148 * 16), 256, 0, s>>>(W, P, omega, npts, H);
        return cudaGetLastError();
    }

    // -------------------------------------------------------- reductions
    constexpr int kRedBlocks = 1024, kRedThreads = 256;
    int reduce_scratch_doubles() { return kRedBlocks; }

    __device__ __forceinline__ double block_sum(double v)
    {
        __shared__ double part[32];
        for (int o = 16; o > 0; o >>= 1)
            v += __shfl_down_sync(0xffffffffu, v, o);
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        __syncthreads();
        if (lane == 0)
            part[w] = v;
        __syncthreads();
        v = (threadIdx.x < (blockDim.x >> 5)) ? part[threadIdx.x] : 0.0;
        if (w == 0)
            for (int o = 16; o > 0; o >>= 1)
                v += __shfl_down_sync(0xffffffffu, v, o);
        return v;
    }

    __global__ void finish_sum_kernel(const double *scratch, int nparts, double *out)
    {
        double v = 0.0;
        for (int q = threadIdx.x; q < nparts; q += blockDim.x)
            v += scratch[q];
        v = block_sum(v);
        if (threadIdx.x == 0)
            *out = v;
    }

    template <typename Real>
    __global__ void sumsq_kernel(const Real *x, const Real *y, long long n, double *scratch)
    {
        double v = 0.0;
        for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        {
            const double d = y ? (double)x[q] - (double)y[q] : (double)x[q];
            v += d * d;
        }
        v = block_sum(v);
        if (threadIdx.x == 0)
            scratch[blockIdx.x] = v;
    }

    template <typename Real>
    cudaError_t launch_sumsq(const Real *x, const Real *y, long long n, double *scratch, double *out, cudaStream_t s)
    {
        const int blocks = std::max(1, std::min(kRedBlocks, blocks_for(n, kRedThreads)));
        sumsq_kernel<Real><<<blocks, kRedThreads, 0, s>>>(x, y, n, scratch);
        finish_sum_kernel<<<1, kRedThreads, 0, s>>>(scratch, blocks, out);
        return cudaGetLastError();
    }
    template cudaError_t launch_sumsq<double>(const double *, const double *, long long, double *, double *, cudaStream_t);
    template cudaError_t launch_sumsq<float>(const float *, const float *, long long, double *, double *, cudaStream_t);

    template <typename Real>
    __global__ void energy_kernel(int n, int nel, const double *__restrict__ corners, const Real *u, double *scratch)
    {
        double v = 0.0;
        const long long total = (long long)n * n * nel;
        for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total; q += (long long)gridDim.x * blockDim.x)
        {
            const int node = (int)(q % (n * n));
            const int el = (int)(q / (n * n));
            const int i = node % n, j = node / n;
            double J[4];
            jacobian<double>(corners + 8 * (size_t)el, c_tab[n].x[i], c_tab[n].x[j], J);
            const double m = c_tab[n].w[i] * c_tab[n].w[j] * (J[0] * J[3] - J[1] * J[2]);
            const double p = u[3 * q], a = u[3 * q + 1], b = u[3 * q + 2];
            v += 0.5 * m * (p * p + a * a + b * b);
        }
        v = block_sum(v);
        if (threadIdx.x == 0)
            scratch[blockIdx.x] = v;
    }
    template <typename Real>
    cudaError_t launch_energy(const Geometry &g, const Real *u, double *scratch, double *out, cudaStream_t s)
    {
        const long long total = (long long)g.n * g.n * g.nel;
        const int blocks = std::max(1, std::min(kRedBlocks, blocks_for(total, kRedThreads)));
        energy_kernel<Real><<<blocks, kRedThreads, 0, s>>>(g.n, g.nel, g.corners, u, scratch);
        finish_sum_kernel<<<1, kRedThreads, 0, s>>>(scratch, blocks, out);
        return cudaGetLastError();
    }
    template cudaError_t launch_energy<double>(const Geometry &, const double *, double *, double *, cudaStream_t);
    template cudaError_t launch_energy<float>(const Geometry &, const float *, double *, double *, cudaStream_t);

    // examples/waveholtz2d.cpp:169-175: W <- acc + pi0, residual (W_new - W_prev)^2
    __global__ void wh_update_kernel(double *W, const double *acc, const double *pi0, long long n, double *scratch)
    {
        double v = 0.0;
        for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        {
            const double wn = pi0 ? acc[q] + pi0[q] : acc[q];
            const double d = wn - W[q];
            v += d * d;
            W[q] = wn;
        }
        v = block_sum(v);
        if (threadIdx.x == 0)
            scratch[blockIdx.x] = v;
    }
    cudaError_t launch_wh_update(double *W, const double *acc, const double *pi0, long long n, double *scratch,
                                 double *out, cudaStream_t s)
    {
        const int blocks = std::max(1, std::min(kRedBlocks, blocks_for(n, kRedThreads)));
        wh_update_kernel<<<blocks, kRedThreads, 0, s>>>(W, acc, pi0, n, scratch);
        finish_sum_kernel<<<1, kRedThreads, 0, s>>>(scratch, blocks, out);
        return cudaGetLastError();
    }
} // namespace wdg
