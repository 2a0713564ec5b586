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

    bool degree_supported(int n) { return n == 2 || n == 3 || n == 4 || n == 5 || n == 6 || n == 7 || n == 8 || n == 9; }

    int max_tile(int n) { return (512 / (n * n)) & ~3; }
    int default_tile(int n, bool fp32)
    {
        (void)fp32;
        return max_tile(n);
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
    // bounded: try_wait itself suspends for a hardware time slice per poll
    constexpr int kMaxPolls = 1 << 22;
    __device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
    {
        for (int it = 0; it < kMaxPolls; ++it)
            if (mbar_try_wait(bar, parity))
                return true;
        return false;
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

    // exterior state of a boundary node: 0 absorbing, 1 reflecting, 2 Dirichlet p = 0
    template <typename Real>
    __device__ __forceinline__ void exterior(int code, Real nx, Real ny, const Real q[3], Real x[3])
    {
        if (code == 1)
        {
            x[0] = q[0];
            x[1] = (ny * ny - nx * nx) * q[1] - Real(2) * nx * ny * q[2];
            x[2] = -Real(2) * nx * ny * q[1] + (nx * nx - ny * ny) * q[2];
        }
        else if (code == 0)
        {
            const Real out = q[0] + nx * q[1] + ny * q[2];
            const Real tan = ny * q[1] - nx * q[2];
            x[1] = ny * tan + Real(0.5) * nx * out;
            x[2] = -nx * tan + Real(0.5) * ny * out;
            x[0] = nx * x[1] + ny * x[2];
        }
        else
        {
            x[0] = -q[0];
            x[1] = q[1];
            x[2] = q[2];
        }
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
    template <int N, typename Real, bool RK>
    __global__ void __launch_bounds__(512) stage_kernel(const StageArgs<Real> a)
    {
        constexpr int NN = N * N, ND = 3 * NN;
        const int E = a.tile;
        const int flags = a.flags;
        const bool has_du = RK && (flags & F_READ_DU);
        const int ntiles = (a.nel + E - 1) / E;

        extern __shared__ __align__(128) unsigned char smem[];
        const size_t ub = (size_t)E * ND * sizeof(Real);
        const size_t bufb = ub * (has_du ? 2 : 1) + (size_t)E * (64 + 16 + 4);
        uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
        unsigned char *buf0 = smem + 16;
        Real *Fs = reinterpret_cast<Real *>(buf0 + 2 * bufb);
        Real *Gs = Fs + (size_t)3 * NN * E;
        Real *nrm = Gs + (size_t)3 * NN * E; // (3, 4, E): nx, ny, meas

        const int t = threadIdx.x;
        const int e = t / NN, node = t - e * NN;
        const int i = node % N, j = node / N;

        // faces through this node (corners lie on two)
        int fA = -1, kA = 0, fB = -1, kB = 0;
        {
            int fs[2] = {-1, -1}, ks[2] = {0, 0}, c = 0;
            if (j == 0) { fs[c] = 0; ks[c++] = i; }
            if (i == N - 1) { fs[c] = 1; ks[c++] = j; }
            if (j == N - 1 && c < 2) { fs[c] = 2; ks[c++] = i; }
            if (i == 0 && c < 2) { fs[c] = 3; ks[c++] = j; }
            fA = fs[0]; kA = ks[0]; fB = fs[1]; kB = ks[1];
        }

        if (t == 0)
        {
            mbar_init(&bars[0], 1);
            mbar_init(&bars[1], 1);
            fence_mbar_init();
        }
        __syncthreads();

        auto tile_full = [&](int k) { return (k + 1) * E <= a.nel; };
        auto issue = [&](int k, int b)
        {
            if (k >= ntiles || !a.use_tma || !tile_full(k))
                return;
            const size_t el0 = (size_t)k * E;
            unsigned char *base = buf0 + b * bufb;
            const uint32_t bytes = (uint32_t)(ub * (has_du ? 2 : 1) + (size_t)E * 84);
            mbar_expect_tx(&bars[b], bytes);
            bulk_g2s(base, a.u + el0 * ND, (uint32_t)ub, &bars[b]);
            if (has_du)
                bulk_g2s(base + ub, a.du + el0 * ND, (uint32_t)ub, &bars[b]);
            unsigned char *g = base + ub * (has_du ? 2 : 1);
            bulk_g2s(g, a.corners + 8 * el0, (uint32_t)(64 * E), &bars[b]);
            bulk_g2s(g + 64 * E, a.nbr + el0, (uint32_t)(16 * E), &bars[b]);
            bulk_g2s(g + 80 * E, a.finfo + el0, (uint32_t)(4 * E), &bars[b]);
        };
        if (t == 0)
        {
            issue(blockIdx.x, 0);
            issue(blockIdx.x + gridDim.x, 1);
        }

        Real Di[N], Dj[N];
#pragma unroll
        for (int l = 0; l < N; ++l)
        {
            Di[l] = Tab<Real>::D(N, l + N * i);
            Dj[l] = Tab<Real>::D(N, l + N * j);
        }
        const Real xi = Tab<Real>::x(N, i), eta = Tab<Real>::x(N, j);
        const Real wi = Tab<Real>::w(N, i), wj = Tab<Real>::w(N, j);
        const Real wA = (fA >= 0) ? Tab<Real>::w(N, kA) : Real(0);
        const Real wB = (fB >= 0) ? Tab<Real>::w(N, kB) : Real(0);

        int it = 0;
        for (int k = blockIdx.x; k < ntiles; k += gridDim.x, ++it)
        {
            const int b = it & 1;
            const uint32_t par = (it >> 1) & 1;
            const int el0 = k * E;
            const int ne = min(E, a.nel - el0);
            unsigned char *base = buf0 + b * bufb;
            Real *us = reinterpret_cast<Real *>(base);
            Real *dus = reinterpret_cast<Real *>(base + ub);
            double *cs = reinterpret_cast<double *>(base + ub * (has_du ? 2 : 1));
            int4 *ns = reinterpret_cast<int4 *>(cs + 8 * E);
            uint32_t *is = reinterpret_cast<uint32_t *>(ns + E);

            if (a.use_tma && tile_full(k))
            {
                const bool ok = mbar_wait(&bars[b], par);
                if (__syncthreads_or(!ok))
                {
                    // give the other buffer's copies a bounded chance to land, then leave
                    if (t == 0)
                    {
                        atomicOr(a.err, 1u);
                        const int kn = k + gridDim.x;
                        if (kn < ntiles && tile_full(kn))
                            mbar_wait(&bars[b ^ 1], ((it + 1) >> 1) & 1);
                    }
                    __syncthreads();
                    return;
                }
            }
            else
            {
                for (int q = t; q < ne * ND; q += blockDim.x)
                    us[q] = a.u[(size_t)el0 * ND + q];
                if (has_du)
                    for (int q = t; q < ne * ND; q += blockDim.x)
                        dus[q] = a.du[(size_t)el0 * ND + q];
                for (int q = t; q < ne * 8; q += blockDim.x)
                    cs[q] = a.corners[8 * (size_t)el0 + q];
                for (int q = t; q < ne; q += blockDim.x)
                {
                    ns[q] = a.nbr[el0 + q];
                    is[q] = a.finfo[el0 + q];
                }
                __syncthreads();
            }

            const bool act = e < ne;
            const size_t g = ((size_t)(el0 + e) * NN + node) * 3;
            const uint32_t info = act ? is[e] : 0u;
            const int4 nb4 = act ? ns[e] : make_int4(-1, -1, -1, -1);

            // neighbour traces that live outside the tile: issue the loads now
            Real xA[3] = {0, 0, 0}, xB[3] = {0, 0, 0};
            int srcA = 0, srcB = 0; // 0 none, 1 smem (index in nA/nB), 2 registers, 3 boundary
            int nA = 0, nB = 0;
            auto locate = [&](int f, int kk, int &src, int &sidx, Real x[3])
            {
                if (f < 0 || !act)
                    return;
                const uint32_t byte = (info >> (8 * f)) & 0xffu;
                if (byte & 0x80u)
                {
                    src = (flags & F_BND) ? 3 : 0;
                    return;
                }
                if (!(flags & F_INT))
                    return;
                const int nb = (f == 0) ? nb4.x : (f == 1) ? nb4.y : (f == 2) ? nb4.z : nb4.w;
                if (nb < 0 || nb >= a.nel)
                {
                    atomicOr(a.err, 2u);
                    return;
                }
                const int kn = (byte & 4u) ? (N - 1 - kk) : kk;
                const int nn = face_node(N, (int)(byte & 3u), kn);
                const int le = nb - el0;
                if (le >= 0 && le < ne)
                {
                    src = 1;
                    sidx = le * ND + 3 * nn;
                }
                else
                {
                    src = 2;
                    const Real *p = a.u + ((size_t)nb * NN + nn) * 3;
                    x[0] = __ldg(p);
                    x[1] = __ldg(p + 1);
                    x[2] = __ldg(p + 2);
                }
            };
            locate(fA, kA, srcA, nA, xA);
            locate(fB, kB, srcB, nB, xB);

            // per-DOF side inputs that are not staged
            Real Fv[3] = {0, 0, 0}, ov[3] = {0, 0, 0};
            double accv[3] = {0, 0, 0};
            if (act)
            {
                if (flags & F_FORCE)
                    for (int d = 0; d < 3; ++d)
                        Fv[d] = a.F[g + d];
                if (!RK && (flags & F_ACCUM))
                    for (int d = 0; d < 3; ++d)
                        ov[d] = a.out[g + d];
                if (RK && (flags & F_FILTER))
                    for (int d = 0; d < 3; ++d)
                        accv[d] = a.acc[g + d];
            }

            // phase A: contravariant fluxes and mass at this node; side normals
            Real q[3] = {0, 0, 0}, minv = 0;
            if (act)
            {
                q[0] = us[e * ND + 3 * node + 0];
                q[1] = us[e * ND + 3 * node + 1];
                q[2] = us[e * ND + 3 * node + 2];
                Real J[4];
                jacobian<Real>(cs + 8 * e, xi, eta, J);
                const Real W = wi * wj;
                const Real Yeta = J[3] * W, Xeta = J[2] * W, Yxi = J[1] * W, Xxi = J[0] * W;
                Real *F0 = Fs + (size_t)e * 3 * NN, *G0 = Gs + (size_t)e * 3 * NN;
                F0[node] = Yeta * q[1] - Xeta * q[2];
                F0[NN + node] = Yeta * q[0];
                F0[2 * NN + node] = -Xeta * q[0];
                G0[node] = -Yxi * q[1] + Xxi * q[2];
                G0[NN + node] = -Yxi * q[0];
                G0[2 * NN + node] = Xxi * q[0];
                minv = Real(1) / (wi * wj * (J[0] * J[3] - J[1] * J[2]));
            }
            if (t < 4 * ne)
            {
                const int ee = t >> 2, f = t & 3;
                double nx, ny, ms;
                side_normal(cs + 8 * ee, f, nx, ny, ms);
                nrm[(ee * 4 + f) * 3 + 0] = (Real)nx;
                nrm[(ee * 4 + f) * 3 + 1] = (Real)ny;
                nrm[(ee * 4 + f) * 3 + 2] = (Real)ms;
            }
            __syncthreads();

            // phase B: volume contraction + face fluxes
            if (act)
            {
                Real r[3] = {0, 0, 0};
                if (flags & F_VOL)
                {
                    const Real *F0 = Fs + (size_t)e * 3 * NN, *G0 = Gs + (size_t)e * 3 * NN;
#pragma unroll
                    for (int l = 0; l < N; ++l)
                    {
                        const int fl = l + N * j, gl = i + N * l;
                        r[0] += Di[l] * F0[fl] + Dj[l] * G0[gl];
                        r[1] += Di[l] * F0[NN + fl] + Dj[l] * G0[NN + gl];
                        r[2] += Di[l] * F0[2 * NN + fl] + Dj[l] * G0[2 * NN + gl];
                    }
                }
                auto face = [&](int f, int src, int sidx, Real x[3], Real wk)
                {
                    if (src == 0)
                        return;
                    const Real *nv = nrm + (e * 4 + f) * 3;
                    const Real nx = nv[0], ny = nv[1];
                    if (src == 1)
                    {
                        x[0] = us[sidx];
                        x[1] = us[sidx + 1];
                        x[2] = us[sidx + 2];
                    }
                    else if (src == 3)
                    {
                        const int code = (int)((info >> (8 * f + 3)) & 3u);
                        exterior<Real>(code, nx, ny, q, x);
                    }
                    upwind<Real>(nx, ny, Real(0.5) * (wk * nv[2]), q, x, r);
                };
                face(fA, srcA, nA, xA, wA);
                face(fB, srcB, nB, xB, wB);

                if (flags & F_FORCE)
                    for (int d = 0; d < 3; ++d)
                        r[d] += Fv[d] * a.fscale;
                if (flags & F_MINV)
                    for (int d = 0; d < 3; ++d)
                        r[d] *= minv;

                if (RK)
                {
                    for (int d = 0; d < 3; ++d)
                    {
                        const Real dn = has_du ? a.rk_a * dus[e * ND + 3 * node + d] + a.dt * r[d] : a.dt * r[d];
                        const Real un = q[d] + a.rk_b * dn;
                        a.du[g + d] = dn;
                        a.out[g + d] = un;
                        if (flags & F_FILTER)
                            a.acc[g + d] = accv[d] + a.acc_c * (double)un;
                    }
                }
                else
                {
                    for (int d = 0; d < 3; ++d)
                        a.out[g + d] = (flags & F_ACCUM) ? ov[d] + r[d] : r[d];
                }
            }
            __syncthreads();
            if (t == 0)
                issue(k + 2 * gridDim.x, b);
        }
    }

    template <typename Real>
    size_t stage_smem_bytes(int n, int tile, int flags)
    {
        const size_t nd = 3 * (size_t)n * n;
        const bool du = (flags & F_READ_DU) != 0;
        const size_t ub = (size_t)tile * nd * sizeof(Real);
        const size_t bufb = ub * (du ? 2 : 1) + (size_t)tile * 84;
        return 16 + 2 * bufb + 2 * ub + (size_t)tile * 12 * sizeof(Real);
    }

    template <int N, typename Real, bool RK>
    static cudaError_t launch_stage_n(const StageArgs<Real> &a, int grid_limit, cudaStream_t s)
    {
        auto kern = stage_kernel<N, Real, RK>;
        const size_t smem = stage_smem_bytes<Real>(N, a.tile, a.flags);
        // the largest footprint any flag set can ask for, set once
        static bool attr_set[64] = {};
        int dev = 0;
        cudaGetDevice(&dev);
        if (!attr_set[dev & 63])
        {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
            if (e != cudaSuccess)
                return e;
            attr_set[dev & 63] = true;
        }
        const int threads = a.tile * N * N;
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
#define WDG_CASE(NV)                                                                       \
    case NV:                                                                               \
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
    template size_t stage_smem_bytes<double>(int, int, int);
    template size_t stage_smem_bytes<float>(int, int, int);

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
