// Fused element kernels of the conservation-law path (included by kernels.cu, which owns the
// basis tables): u_t + div F(u) = 0 with nodal DG on GLL nodes, approximate quadrature.
//
// One warp per element, the element's values staged in shared memory:
//   volume   per node the physical flux (f, g) = F(u), its contravariant form
//            (W (y_eta f - x_eta g), W (-y_xi f + x_xi g)), and the D contraction
//            (DivF2D<true>::action, wavedg/DivF.hpp:203-260; Div<true> for a linear flux);
//   faces    per face node the numerical flux fh(n, u_own, u_nbr) with n the element's own
//            outward normal, subtracted times w_k |E| / 2 (EdgeFluxF2D<true>::action,
//            wavedg/EdgeFluxF.hpp:138-180, with the sign flip and transpose prolongation of
//            examples/cl2d.cpp:175-219); the neighbour's trace is read from the stage's input
//            through the partner table of the fused wave kernels;
//   mass     M^{-1} = 1 / (w_i w_j det J) (MassMatrix<true>);
//   output   the RHS, or one stage of ode::RungeKutta4 or ode::SSPRK3 (wavedg/ode.hpp:66-93,
//            145-186) applied in the same pass.
// Each face contribution uses the element's own normal and the numerical flux's antisymmetry
// fh(-n, b, a) = -fh(n, a, b), which holds exactly in floating point for both fluxes below, so
// the two elements of an edge add exactly opposite terms, as the reference's edge loop does.
//
// Flux models (ClawEuler, ClawLinear) and the side geometry: claw_model.cuh.

#include "claw_model.cuh"

namespace wdg
{
    template <class M, int NV>
    __device__ __forceinline__ void claw_flux(const ClawArgs &a, const double *q, double *f, double *g)
    {
        if constexpr (std::is_same<M, ClawLinear>::value)
            ClawLinear::flux_n<NV>(a, q, f, g);
        else
            M::flux(a, q, f, g);
    }

    constexpr int kClawWarps = 4;
    // doubles of a CTA's shared copy of the basis table (D, nodes, weights), kept even
    __host__ __device__ constexpr int claw_tab_doubles(int n) { return (n * n + 2 * n + 1) & ~1; }
    // doubles of one warp's staging: values, two fluxes, neighbour traces, masses, side geometry
    __host__ __device__ constexpr int claw_warp_doubles(int n, int nv)
    {
        return (3 * nv * n * n + 4 * n * nv + n * n + 12 + 1) & ~1;
    }

    // resident CTAs per SM the register budget is set for (the kernel is latency-bound: more
    // resident warps hide more of each warp's load -> compute -> store chain); degrees above 4
    // keep the compiler's own budget (their unrolled contractions would spill)
    template <int N, int NV>
    constexpr int claw_min_blocks()
    {
        return N > 5 ? 1 : NV <= 2 ? 6 : NV == 3 ? 5 : NV <= 6 ? 4 : 3;
    }

    template <int N, int NV, class M>
    __global__ void __launch_bounds__(32 * kClawWarps, claw_min_blocks<N, NV>()) claw_kernel(const ClawArgs a)
    {
        constexpr int NN = N * N, ND = NV * NN;
        extern __shared__ double csm[];
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        // the basis table (D, nodes, weights) in shared memory: the lanes of a warp read
        // different entries, which the constant cache would serve one address at a time
        double *sD = csm, *sx = sD + NN, *sw = sx + N;
        for (int k = threadIdx.x; k < NN; k += blockDim.x)
            sD[k] = Tab<double>::D(N, k);
        for (int k = threadIdx.x; k < N; k += blockDim.x)
        {
            sx[k] = Tab<double>::x(N, k);
            sw[k] = Tab<double>::w(N, k);
        }
        __syncthreads();
        // per warp: the element's values, the two contravariant fluxes, the neighbour traces
        // T(s, k, d) of its interior sides, the mass w_i w_j det J per node and (n_x, n_y, |E|/2)
        // per side
        double *q = csm + claw_tab_doubles(N) + (size_t)warp * claw_warp_doubles(N, NV), *Fs = q + ND, *Gs = Fs + ND,
               *T = Gs + ND, *mj = T + 4 * N * NV, *sn = mj + NN;
        const long long limit = (long long)a.nel * NN; // nodes a neighbour index may name
        for (int el = blockIdx.x * kClawWarps + warp; el < a.nel; el += gridDim.x * kClawWarps)
        {
            const double *xe = a.x + (size_t)el * ND;
            for (int k = lane; k < ND; k += 32)
                q[k] = xe[k];
            double c[8];
#pragma unroll
            for (int k = 0; k < 8; ++k)
                c[k] = __ldg(a.corners + 8 * (size_t)el + k);
            const uint32_t codes = __ldg(a.fcode + el);
            const int4 fb = __ldg(a.fbase + el);
            // the neighbour traces of the interior sides, copied asynchronously (cp.async) while
            // the volume term is formed; an index outside the state is reported and not read
            for (int o = lane; o < 4 * N; o += 32)
            {
                const int s = o / N, k = o - s * N;
                const uint32_t byte = (codes >> (8 * s)) & 0xffu;
                if (byte & 0x80u)
                    continue;
                const int off = (s == 0) ? fb.x : (s == 1) ? fb.y : (s == 2) ? fb.z : fb.w;
                const long long pn = (long long)(off / 3) + (long long)k * (partner_stride<N>(byte) / 3);
                if (off < 0 || pn < 0 || pn >= limit)
                    atomicOr(a.err, 2u);
                else
#pragma unroll
                    for (int d = 0; d < NV; ++d)
                        cp_async<8>(T + NV * o + d, a.x + (size_t)NV * pn + d);
            }
            cp_async_commit();
            if (lane < 4)
            {
                // one side per lane, each with a compile-time side index (keeps c in registers)
                double nx = 0.0, ny = 0.0, meas = 0.0;
                switch (lane)
                {
                case 0: claw_side(c, 0, nx, ny, meas); break;
                case 1: claw_side(c, 1, nx, ny, meas); break;
                case 2: claw_side(c, 2, nx, ny, meas); break;
                default: claw_side(c, 3, nx, ny, meas); break;
                }
                sn[3 * lane] = nx;
                sn[3 * lane + 1] = ny;
                sn[3 * lane + 2] = meas;
            }
            __syncwarp();
            // volume: contravariant fluxes per node
            for (int node = lane; node < NN; node += 32)
            {
                const int i = node % N, j = node / N;
                const double xi = sx[i], eta = sx[j];
                const double Xx = 0.25 * ((1.0 - eta) * (c[2] - c[0]) + (1.0 + eta) * (c[4] - c[6]));
                const double Yx = 0.25 * ((1.0 - eta) * (c[3] - c[1]) + (1.0 + eta) * (c[5] - c[7]));
                const double Xe = 0.25 * ((1.0 - xi) * (c[6] - c[0]) + (1.0 + xi) * (c[4] - c[2]));
                const double Ye = 0.25 * ((1.0 - xi) * (c[7] - c[1]) + (1.0 + xi) * (c[5] - c[3]));
                const double W = sw[i] * sw[j];
                mj[node] = W * (Xx * Ye - Yx * Xe); // MassMatrix<true>: w_i w_j det J
                double qq[NV], f[NV], g[NV];
#pragma unroll
                for (int d = 0; d < NV; ++d)
                    qq[d] = q[NV * node + d];
                claw_flux<M, NV>(a, qq, f, g);
#pragma unroll
                for (int d = 0; d < NV; ++d)
                {
                    Fs[NV * node + d] = (Ye * W) * f[d] - (Xe * W) * g[d];
                    Gs[NV * node + d] = -(Yx * W) * f[d] + (Xx * W) * g[d];
                }
            }
            cp_async_wait<0>();
            __syncwarp();
            for (int node = lane; node < NN; node += 32)
            {
                const int i = node % N, j = node / N;
                double r[NV];
#pragma unroll
                for (int d = 0; d < NV; ++d)
                {
                    double s = 0.0;
#pragma unroll
                    for (int l = 0; l < N; ++l)
                        s += sD[l + N * i] * Fs[NV * (l + N * j) + d] +
                             sD[l + N * j] * Gs[NV * (i + N * l) + d];
                    r[d] = s;
                }
                const size_t g0 = (size_t)el * ND + (size_t)NV * node;
                if (a.mode == CLAW_DIV)
                {
#pragma unroll
                    for (int d = 0; d < NV; ++d)
                        a.out[g0 + d] += r[d];
                    continue;
                }
                double qq[NV];
#pragma unroll
                for (int d = 0; d < NV; ++d)
                    qq[d] = q[NV * node + d];
                // faces through this node: side 0 (j = 0, k = i), 1 (i = n-1, k = j),
                // 2 (j = n-1, k = i), 3 (i = 0, k = j)
#pragma unroll
                for (int s = 0; s < 4; ++s)
                {
                    const bool on = (s == 0) ? (j == 0) : (s == 1) ? (i == N - 1) : (s == 2) ? (j == N - 1) : (i == 0);
                    if (!on)
                        continue;
                    const int k = (s == 0 || s == 2) ? i : j;
                    const uint32_t byte = (codes >> (8 * s)) & 0xffu;
                    double ext[NV];
                    if (byte & 0x80u)
                        M::template exterior<NV>(qq, ext);
                    else
                    {
                        const int off = (s == 0) ? fb.x : (s == 1) ? fb.y : (s == 2) ? fb.z : fb.w;
                        const long long pn = (long long)(off / 3) + (long long)k * (partner_stride<N>(byte) / 3);
                        const bool bad = off < 0 || pn < 0 || pn >= limit; // reported by the gather
#pragma unroll
                        for (int d = 0; d < NV; ++d)
                            ext[d] = bad ? qq[d] : T[NV * (s * N + k) + d];
                    }
                    const double nx = sn[3 * s], ny = sn[3 * s + 1], meas = sn[3 * s + 2];
                    double fh[NV];
                    M::template numflux<NV>(a, el, s, nx, ny, qq, ext, fh);
                    const double wk = sw[k] * meas;
#pragma unroll
                    for (int d = 0; d < NV; ++d)
                        r[d] -= wk * fh[d];
                }
                // M^{-1}: w_i w_j det J (MassMatrix<true>), formed with the volume term
                {
                    const double m = mj[node];
#pragma unroll
                    for (int d = 0; d < NV; ++d)
                        r[d] /= m;
                }
                switch (a.mode)
                {
                case CLAW_RHS:
#pragma unroll
                    for (int d = 0; d < NV; ++d)
                        a.out[g0 + d] = r[d];
                    break;
                case CLAW_RK4:
#pragma unroll
                    for (int d = 0; d < NV; ++d)
                    {
                        const double kd = (a.rk_a == 0.0) ? a.dt * r[d] : a.rk_a * a.du[g0 + d] + a.dt * r[d];
                        a.du[g0 + d] = kd;
                        a.out[g0 + d] = qq[d] + a.rk_b * kd;
                    }
                    break;
                case CLAW_SSP0:
#pragma unroll
                    for (int d = 0; d < NV; ++d)
                        a.out[g0 + d] = qq[d] + a.dt * r[d];
                    break;
                case CLAW_SSP1:
#pragma unroll
                    for (int d = 0; d < NV; ++d)
                        a.out[g0 + d] = 0.25 * (qq[d] + 3.0 * a.base[g0 + d] + a.dt * r[d]);
                    break;
                default: // CLAW_SSP2
#pragma unroll
                    for (int d = 0; d < NV; ++d)
                        a.out[g0 + d] = (a.base[g0 + d] + 2.0 * qq[d] + 2.0 * a.dt * r[d]) / 3.0;
                    break;
                }
            }
            __syncwarp(); // the element's staging is reused for the next one
        }
    }

    // EdgeFluxF2D<true>::action for the Euler system on face traces (n, 4, 2, edges): thread per
    // (face node, edge); fB = +- w_i |E| / 2 fh(n, side 0, side 1), n the outward normal of the
    // edge's first element (in place allowed: a thread reads its node's traces before writing)
    __global__ void euler_face_flux_kernel(int n, int ne, const int *__restrict__ edges, const double *__restrict__ corners,
                                           const double *ub, double *fb)
    {
        const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
        if (q >= (long long)n * ne)
            return;
        const int i = (int)(q % n), e = (int)(q / n);
        const int el = edges[5 * (size_t)e], s = edges[5 * (size_t)e + 1];
        double c[8];
        for (int k = 0; k < 8; ++k)
            c[k] = corners[8 * (size_t)el + k];
        double nx, ny, meas, qL[4], qR[4], fh[4];
        claw_side(c, s, nx, ny, meas);
        for (int d = 0; d < 4; ++d)
        {
            qL[d] = ub[i + n * (d + 4 * (0 + 2 * (size_t)e))];
            qR[d] = ub[i + n * (d + 4 * (1 + 2 * (size_t)e))];
        }
        ClawArgs none{};
        ClawEuler::numflux<4>(none, 0, 0, nx, ny, qL, qR, fh);
        const double wm = c_tab[n].w[i] * meas;
        for (int d = 0; d < 4; ++d)
        {
            fb[i + n * (d + 4 * (0 + 2 * (size_t)e))] = fh[d] * wm;
            fb[i + n * (d + 4 * (1 + 2 * (size_t)e))] = -fh[d] * wm;
        }
    }

    // shared memory of one CTA of claw_kernel
    inline size_t claw_smem(int n, int nv)
    {
        return sizeof(double) * (claw_tab_doubles(n) + (size_t)claw_warp_doubles(n, nv) * kClawWarps);
    }

    template <int N, int NV, class M>
    cudaError_t launch_claw_nv(const ClawArgs &a, cudaStream_t s)
    {
        const size_t smem = claw_smem(N, NV);
        auto kern = claw_kernel<N, NV, M>;
        if (smem > 48 * 1024)
        {
            static uint64_t set = 0; // devices whose attribute is set
            int dev = 0;
            cudaGetDevice(&dev);
            if (!(set & (1ull << (dev & 63))))
            {
                cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
                if (e != cudaSuccess)
                    return e;
                set |= 1ull << (dev & 63);
            }
        }
        const int blocks = std::max(1, std::min((a.nel + kClawWarps - 1) / kClawWarps, 148 * 16));
        kern<<<blocks, 32 * kClawWarps, smem, s>>>(a);
        return cudaGetLastError();
    }

    template <int N, class M>
    cudaError_t launch_claw_n(int nv, const ClawArgs &a, cudaStream_t s)
    {
        if constexpr (std::is_same<M, ClawEuler>::value)
            return nv == 4 ? launch_claw_nv<N, 4, M>(a, s) : cudaErrorInvalidValue;
        else
        {
            switch (nv)
            {
            case 1: return launch_claw_nv<N, 1, M>(a, s);
            case 2: return launch_claw_nv<N, 2, M>(a, s);
            case 3: return launch_claw_nv<N, 3, M>(a, s);
            case 4: return launch_claw_nv<N, 4, M>(a, s);
            case 5: return launch_claw_nv<N, 5, M>(a, s);
            case 6: return launch_claw_nv<N, 6, M>(a, s);
            case 7: return launch_claw_nv<N, 7, M>(a, s);
            case 8: return launch_claw_nv<N, 8, M>(a, s);
            default: return cudaErrorInvalidValue;
            }
        }
    }

    template <class M>
    cudaError_t launch_claw_m(int n, int nv, const ClawArgs &a, cudaStream_t s)
    {
        switch (n)
        {
        case 2: return launch_claw_n<2, M>(nv, a, s);
        case 3: return launch_claw_n<3, M>(nv, a, s);
        case 4: return launch_claw_n<4, M>(nv, a, s);
        case 5: return launch_claw_n<5, M>(nv, a, s);
        case 6: return launch_claw_n<6, M>(nv, a, s);
        case 7: return launch_claw_n<7, M>(nv, a, s);
        case 8: return launch_claw_n<8, M>(nv, a, s);
        case 9: return launch_claw_n<9, M>(nv, a, s);
        default: return cudaErrorInvalidValue;
        }
    }
} // namespace wdg
