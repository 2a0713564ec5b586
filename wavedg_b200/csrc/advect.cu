// C-ABI: the linear advection operator of the generic conservation-law path, constant
// coefficients, any number of variables (wavedg/Advection.hpp):
//
//   Advection<true>(n_var, mesh, basis, a, true)                :17-142
//     Div<true> with op_2d_cc (source/Div.cpp:5-53, div_2d_c :131-179) and
//     EdgeFlux<true> over interior edges, a = -1, b = -1/2 (source/EdgeFlux.cpp:7-139, 289-325)
//   AdvectionHomogeneousBC<true>(n_var, mesh, basis, a, true)   :144-273 (u = 0 outside)
//   MassMatrix<true>                                            source/MassMatrix.cpp:6-82
//
// a holds A_0 and A_1 as a(d, c, k) = a[d + nv (c + nv k)].  The upwind flux needs |n . A|;
// it is formed per edge on the host from a Jacobi eigen-decomposition, so A_0 and A_1 must
// be symmetric (the reference's general eigen-solver path for non-symmetric A is not built).
// FP64.  The RHS and RK4 run as one fused launch per evaluation or stage (claw_kernels.cuh:
// volume, both face terms with the upwind flux 1/2 (n.A)(a + b) + 1/2 |n.A| (a - b), mass
// inverse, RK update); the operator entry points (action, bc_action) keep component kernels in
// the reference layouts (u(d, i, j, el), face traces (i, d, side, edge)).  Geometry, edge and
// partner tables and argument staging are those of an internal collocation handle.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "wave_impl.hpp"

using namespace wdg;

struct wdg_advect
{
    wdg_wave *w = nullptr;
    int n = 0, nv = 0;
    double *d_a = nullptr;              // 2 nv^2
    double *d_x = nullptr, *d_wt = nullptr, *d_D = nullptr; // GLL nodes, weights, D(l, j)
    double *d_FI = nullptr, *d_FB = nullptr; // per edge and side: |E|/2 Fs(c, d), (nv, nv, 2, edges)
    double *d_uf = nullptr, *d_uB = nullptr;
    double *d_absA = nullptr;           // |n.A| per element side for the fused kernel, (nv, nv, 4, nel)
    double *d_rk = nullptr;             // RK4: the two rotation buffers and the register
};

namespace wdg
{
    // symmetric m x m eigen-decomposition, cyclic Jacobi: A = R diag(e) R^T (column-major)
    void jacobi_eig(int m, const double *A_, double *R, double *e)
    {
        double A[kJacobiMax * kJacobiMax];
        std::memcpy(A, A_, sizeof(double) * m * m);
        for (int i = 0; i < m * m; ++i)
            R[i] = (i % (m + 1) == 0) ? 1.0 : 0.0;
        for (int sweep = 0; sweep < 100; ++sweep)
        {
            double off = 0.0;
            for (int p = 0; p < m; ++p)
                for (int q = p + 1; q < m; ++q)
                    off += A[p + m * q] * A[p + m * q];
            if (off < 1e-300)
                break;
            for (int p = 0; p < m; ++p)
                for (int q = p + 1; q < m; ++q)
                {
                    const double apq = A[p + m * q];
                    if (apq == 0.0)
                        continue;
                    const double theta = (A[q + m * q] - A[p + m * p]) / (2.0 * apq);
                    const double t = (theta >= 0 ? 1.0 : -1.0) / (std::abs(theta) + std::sqrt(theta * theta + 1.0));
                    const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
                    for (int k = 0; k < m; ++k)
                    {
                        const double akp = A[k + m * p], akq = A[k + m * q];
                        A[k + m * p] = c * akp - sn * akq;
                        A[k + m * q] = sn * akp + c * akq;
                    }
                    for (int k = 0; k < m; ++k)
                    {
                        const double apk = A[p + m * k], aqk = A[q + m * k];
                        A[p + m * k] = c * apk - sn * aqk;
                        A[q + m * k] = sn * apk + c * aqk;
                    }
                    for (int k = 0; k < m; ++k)
                    {
                        const double rkp = R[k + m * p], rkq = R[k + m * q];
                        R[k + m * p] = c * rkp - sn * rkq;
                        R[k + m * q] = sn * rkp + c * rkq;
                    }
                }
        }
        for (int i = 0; i < m; ++i)
            e[i] = A[i + m * i];
    }

} // namespace wdg

namespace
{
    constexpr int kMaxVar = 8;

    __device__ __host__ inline void jac(const double *c, double xi, double eta, double J[4])
    {
        J[0] = 0.25 * ((1.0 - eta) * (c[2] - c[0]) + (1.0 + eta) * (c[4] - c[6]));
        J[1] = 0.25 * ((1.0 - eta) * (c[3] - c[1]) + (1.0 + eta) * (c[5] - c[7]));
        J[2] = 0.25 * ((1.0 - xi) * (c[6] - c[0]) + (1.0 + xi) * (c[4] - c[2]));
        J[3] = 0.25 * ((1.0 - xi) * (c[7] - c[1]) + (1.0 + xi) * (c[5] - c[3]));
    }
    __device__ inline int fnode(int n, int f, int k)
    {
        const int i = (f == 0 || f == 2) ? k : (f == 1 ? n - 1 : 0);
        const int j = (f == 1 || f == 3) ? k : (f == 2 ? n - 1 : 0);
        return i + n * j;
    }

    // Div<true> with constant coefficients: per node the contravariant fluxes
    // F_d = W sum_c (y_eta a(d,c,0) - x_eta a(d,c,1)) u_c, G_d = W sum_c (-y_xi a(d,c,0) + x_xi a(d,c,1)) u_c,
    // then du(d, i, j) += sum_l D(l, i) F_d(l, j) + D(l, j) G_d(i, l).  One CTA per element.
    __global__ void adv_div_kernel(int n, int nv, int nel, const double *__restrict__ corners,
                                   const double *__restrict__ a, const double *__restrict__ x,
                                   const double *__restrict__ wt, const double *__restrict__ D,
                                   const double *__restrict__ u, double *du)
    {
        extern __shared__ double sm[];
        const int nn = n * n, m = nv * nn, v2 = nv * nv;
        double *su = sm, *F = su + m, *G = F + m;
        const int t = threadIdx.x, T = blockDim.x;
        for (int el = blockIdx.x; el < nel; el += gridDim.x)
        {
            const double *ue = u + (size_t)m * el;
            for (int k = t; k < m; k += T)
                su[k] = ue[k];
            __syncthreads();
            const double *ce = corners + 8 * (size_t)el;
            for (int o = t; o < m; o += T)
            {
                const int d = o % nv, node = o / nv;
                double J[4];
                jac(ce, x[node % n], x[node / n], J);
                const double W = wt[node / n] * wt[node % n];
                const double Ye = J[3] * W, Xe = J[2] * W, Yx = J[1] * W, Xx = J[0] * W;
                double f = 0.0, g = 0.0;
                for (int c = 0; c < nv; ++c)
                {
                    const double a0 = a[d + nv * c], a1 = a[d + nv * c + v2], uc = su[c + nv * node];
                    f += (Ye * a0 - Xe * a1) * uc;
                    g += (-Yx * a0 + Xx * a1) * uc;
                }
                F[o] = f;
                G[o] = g;
            }
            __syncthreads();
            double *de = du + (size_t)m * el;
            for (int o = t; o < m; o += T)
            {
                const int d = o % nv, node = o / nv, i = node % n, j = node / n;
                double s = 0.0;
                for (int l = 0; l < n; ++l)
                    s += D[l + n * i] * F[d + nv * (l + n * j)] + D[l + n * j] * G[d + nv * (i + n * l)];
                de[o] += s;
            }
            __syncthreads();
        }
    }

    // LobattoFaceProlongator::action for nv variables: thread per (i, d, side, edge); the
    // boundary's side 1 is zero (u = 0 outside for the homogeneous boundary operator)
    __global__ void adv_prolong_kernel(int n, int nv, int ne, const int *__restrict__ edges, int interior,
                                       const double *__restrict__ u, double *__restrict__ uf)
    {
        const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
        if (q >= (long long)n * nv * 2 * ne)
            return;
        const int i = (int)(q % n), d = (int)((q / n) % nv), s = (int)((q / ((long long)n * nv)) % 2);
        const int e = (int)(q / ((long long)2 * n * nv));
        const int *E = edges + 5 * (size_t)e;
        double v = 0.0;
        if (s == 0 || interior)
        {
            const int el = E[2 * s], f = E[2 * s + 1];
            const int k = (s == 1 && E[4] < 0) ? (n - 1 - i) : i;
            v = u[d + nv * ((size_t)el * n * n + fnode(n, f, k))];
        }
        uf[q] = v;
    }

    // LobattoFaceProlongator::t for nv variables, as a gather: thread per (d, node, el)
    __global__ void adv_prolong_t_kernel(int n, int nv, int nel, const int *__restrict__ face_edge,
                                         const uint32_t *__restrict__ finfo, int want_boundary,
                                         const double *__restrict__ uf, double *__restrict__ u)
    {
        const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
        if (q >= (long long)nv * n * n * nel)
            return;
        const int d = (int)(q % nv);
        const long long nodeg = q / nv;
        const int node = (int)(nodeg % (n * n)), el = (int)(nodeg / (n * n));
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
            if (((byte & 0x80u) != 0) != (want_boundary != 0))
                continue;
            const int slot = face_edge[4 * (size_t)el + f];
            const int edge = slot >> 1, side = slot & 1;
            const int ie = (side == 1 && (byte & 4u)) ? (n - 1 - k) : k;
            add += uf[ie + n * (d + nv * (side + 2 * (size_t)edge))];
        }
        u[q] += add;
    }

    // EdgeFlux<true>::action for nv variables: uf_d = w_i sum_s sum_c Fs(c, d) u_s,c; side 0 <- uf,
    // side 1 <- -uf (safe in place: a thread reads its face node's traces before writing them)
    __global__ void adv_flux_kernel(int n, int nv, int ne, const double *__restrict__ Ft, const double *__restrict__ wt,
                                    const double *ub, double *fb)
    {
        const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
        if (q >= (long long)n * ne)
            return;
        const int i = (int)(q % n), e = (int)(q / n);
        const int v2 = nv * nv;
        double in[2][kMaxVar], out[kMaxVar];
        for (int s = 0; s < 2; ++s)
            for (int c = 0; c < nv; ++c)
                in[s][c] = ub[i + n * (c + nv * (s + 2 * (size_t)e))];
        const double *Fe = Ft + (size_t)2 * v2 * e;
        for (int d = 0; d < nv; ++d)
        {
            double acc = 0.0;
            for (int s = 0; s < 2; ++s)
                for (int c = 0; c < nv; ++c)
                    acc += (wt[i] * Fe[c + nv * (d + nv * s)]) * in[s][c];
            out[d] = acc;
        }
        for (int d = 0; d < nv; ++d)
        {
            fb[i + n * (d + nv * (0 + 2 * (size_t)e))] = out[d];
            fb[i + n * (d + nv * (1 + 2 * (size_t)e))] = -out[d];
        }
    }

    // per edge: |E|/2 Fs(c, d) for both sides, Fs = R diag(-lambda/2 -+ |lambda|/2) R^T of n . A
    // (_ComputeFlux::flux with a = -1, b = -1/2, source/EdgeFlux.cpp:31-88), normal of the
    // first element's side
    std::vector<double> flux_tables(const wdg_mesh &mesh, const std::vector<EdgeRec> &list, int nv, const double *a)
    {
        const int v2 = nv * nv;
        std::vector<double> F((size_t)2 * v2 * list.size());
        for (size_t e = 0; e < list.size(); ++e)
        {
            const double *cr = &mesh.corners[8 * (size_t)list[e].el0];
            const int s0 = list[e].s0;
            const double dx = cr[2 * kSideTo[s0]] - cr[2 * kSideFrom[s0]];
            const double dy = cr[2 * kSideTo[s0] + 1] - cr[2 * kSideFrom[s0] + 1];
            const double len = std::sqrt(dx * dx + dy * dy), sgn = (s0 >= 2) ? -1.0 : 1.0;
            const double nx = sgn * dy / len, ny = -sgn * dx / len, meas = 0.5 * len;
            double nA[kMaxVar * kMaxVar], R[kMaxVar * kMaxVar], ev[kMaxVar];
            for (int d = 0; d < v2; ++d)
                nA[d] = nx * a[d] + ny * a[d + v2];
            jacobi_eig(nv, nA, R, ev);
            for (int s = 0; s < 2; ++s)
            {
                const double sg = (s == 0) ? 1.0 : -1.0;
                for (int c = 0; c < nv; ++c)
                    for (int d = 0; d < nv; ++d)
                    {
                        double acc = 0.0;
                        for (int k = 0; k < nv; ++k)
                            acc += R[c + nv * k] * (-0.5 * ev[k] + sg * -0.5 * std::abs(ev[k])) * R[d + nv * k];
                        F[c + nv * (d + nv * (s + 2 * e))] = meas * acc;
                    }
            }
        }
        return F;
    }

    // |n.A| = R |diag(lambda)| R^T of n.A per element side, n the side's outward normal (the same
    // arithmetic as the fused kernel's claw_side), for the upwind flux of the fused kernel
    std::vector<double> abs_tables(const wdg_mesh &mesh, int nv, const double *a)
    {
        const int v2 = nv * nv;
        std::vector<double> T((size_t)v2 * 4 * mesh.nel);
        for (int el = 0; el < mesh.nel; ++el)
        {
            const double *c = &mesh.corners[8 * (size_t)el];
            for (int s = 0; s < 4; ++s)
            {
                const int p0 = (s == 0 || s == 3) ? 0 : (s == 1 ? 1 : 3), p1 = (s == 0) ? 1 : (s == 3 ? 3 : 2);
                const double dx = c[2 * p1] - c[2 * p0], dy = c[2 * p1 + 1] - c[2 * p0 + 1];
                const double len = std::sqrt(dx * dx + dy * dy), sgn = (s >= 2) ? -1.0 : 1.0;
                const double nx = sgn * dy / len, ny = -sgn * dx / len;
                double nA[kMaxVar * kMaxVar], R[kMaxVar * kMaxVar], ev[kMaxVar];
                for (int d = 0; d < v2; ++d)
                    nA[d] = nx * a[d] + ny * a[d + v2];
                jacobi_eig(nv, nA, R, ev);
                double *t = &T[(size_t)v2 * (4 * (size_t)el + s)];
                for (int d = 0; d < nv; ++d)
                    for (int k = 0; k < nv; ++k)
                    {
                        double acc = 0.0;
                        for (int m = 0; m < nv; ++m)
                            acc += R[d + nv * m] * std::abs(ev[m]) * R[k + nv * m];
                        t[d + nv * k] = acc;
                    }
            }
        }
        return T;
    }

    unsigned blocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

    long long nvals(const wdg_advect *h) { return (long long)h->nv * h->n * h->n * h->w->nel; }

    int div_dev(wdg_advect *h, const double *u, double *du)
    {
        wdg_wave *w = h->w;
        const size_t smem = sizeof(double) * 3 * h->nv * h->n * h->n;
        adv_div_kernel<<<(unsigned)std::min(w->nel, 148 * 16), 64, smem, w->stream>>>(h->n, h->nv, w->nel, w->d_corners,
                                                                                     h->d_a, h->d_x, h->d_wt, h->d_D, u, du);
        WDG_CUDA(cudaGetLastError());
        return WDG_OK;
    }
    int faces_dev(wdg_advect *h, int type, const double *u, double *du)
    {
        wdg_wave *w = h->w;
        const int ne = (type == 0) ? w->nI : w->nB;
        if (ne == 0)
            return WDG_OK;
        double *uf = (type == 0) ? h->d_uf : h->d_uB;
        const long long tot = (long long)h->n * h->nv * 2 * ne;
        adv_prolong_kernel<<<blocks(tot, 256), 256, 0, w->stream>>>(h->n, h->nv, ne, type == 0 ? w->d_edgesI : w->d_edgesB,
                                                                    type == 0, u, uf);
        adv_flux_kernel<<<blocks((long long)h->n * ne, 128), 128, 0, w->stream>>>(
            h->n, h->nv, ne, type == 0 ? h->d_FI : h->d_FB, h->d_wt, uf, uf);
        adv_prolong_t_kernel<<<blocks(nvals(h), 256), 256, 0, w->stream>>>(h->n, h->nv, w->nel, w->d_face_edge,
                                                                          w->d_finfo, type == 1, uf, du);
        WDG_CUDA(cudaGetLastError());
        return WDG_OK;
    }
    int action_dev(wdg_advect *h, const double *u, double *du)
    {
        WDG_TRY(div_dev(h, u, du));
        return faces_dev(h, 0, u, du);
    }
    int bc_dev(wdg_advect *h, const double *u, double *du) { return faces_dev(h, 1, u, du); }
    // dudt = M^{-1} (A u + B u): one fused launch (volume, both face terms with the upwind flux,
    // mass inverse; claw_kernels.cuh)
    int rhs_dev(wdg_advect *h, const double *u, double *dudt)
    {
        wdg_wave *w = h->w;
        ClawArgs c = claw_args(w, u, dudt);
        c.A = h->d_a;
        c.absA = h->d_absA;
        c.mode = CLAW_RHS;
        WDG_CUDA(launch_claw(1, h->n, h->nv, c, w->stream));
        return WDG_OK;
    }

    typedef int (*Unary)(wdg_advect *, const double *, double *);
    int entry(wdg_advect *h, const double *u, double *du, Unary f, bool accumulate)
    {
        if (!h || !u || !du)
            return fail(WDG_ERR_ARG, "null advection argument");
        if (u == du)
            return fail(WDG_ERR_ARG, "input and output arrays must differ");
        DeviceScope g(h->w->device);
        HostArg a[2];
        WDG_TRY(bind_arg(h->w, 0, u, (size_t)nvals(h), true, false, a[0]));
        WDG_TRY(bind_arg(h->w, 1, du, (size_t)nvals(h), accumulate, true, a[1]));
        WDG_TRY(f(h, a[0].dev, a[1].dev));
        return finish_args(h->w, a, 2);
    }
} // namespace

extern "C"
{
    int wdg_advect_create(const wdg_mesh *mesh, int n_colloc, int n_var, const double *a, int device, wdg_advect **out)
    {
        if (!mesh || !a || !out)
            return fail(WDG_ERR_ARG, "wdg_advect_create: null argument");
        *out = nullptr;
        if (n_var < 1 || n_var > kMaxVar)
            return fail(WDG_ERR_UNSUPPORTED, "wdg_advect_create: n_var must be 1..8");
        const int v2 = n_var * n_var;
        double amax = 0.0;
        for (int i = 0; i < 2 * v2; ++i)
            amax = std::max(amax, std::abs(a[i]));
        for (int k = 0; k < 2; ++k)
            for (int d = 0; d < n_var; ++d)
                for (int c = 0; c < d; ++c)
                    if (std::abs(a[d + n_var * c + v2 * k] - a[c + n_var * d + v2 * k]) > 1e-14 * amax)
                        return fail(WDG_ERR_UNSUPPORTED,
                                    "wdg_advect_create: the coefficient matrices must be symmetric (the upwind flux "
                                    "uses a symmetric eigen-decomposition)");
        wdg_wave *w = nullptr;
        WDG_TRY(wdg_wave_create(mesh, n_colloc, nullptr, WDG_FP64, device, &w));
        wdg_advect *h = new wdg_advect;
        h->w = w;
        h->n = n_colloc;
        h->nv = n_var;
        DeviceScope g(w->device);
        const int n = n_colloc;
        std::vector<double> x(n), wt(n), D((size_t)n * n), av(a, a + 2 * v2);
        gauss_lobatto(n, x.data(), wt.data());
        deriv_matrix(n, x.data(), D.data());
        const std::vector<double> FI = flux_tables(*mesh, mesh->interior, n_var, a);
        const std::vector<double> FB = flux_tables(*mesh, mesh->boundary, n_var, a);
        const std::vector<double> AB = abs_tables(*mesh, n_var, a);
        int st = WDG_OK;
        auto chk = [&](int r)
        {
            if (st == WDG_OK)
                st = r;
        };
        chk(device_alloc(&h->d_a, av.size()));
        chk(device_alloc(&h->d_x, x.size()));
        chk(device_alloc(&h->d_wt, wt.size()));
        chk(device_alloc(&h->d_D, D.size()));
        chk(device_alloc(&h->d_FI, FI.size()));
        chk(device_alloc(&h->d_FB, FB.size()));
        chk(device_alloc(&h->d_absA, AB.size()));
        chk(device_alloc(&h->d_uf, (size_t)n * n_var * 2 * w->nI));
        chk(device_alloc(&h->d_uB, (size_t)n * n_var * 2 * w->nB));
        if (st == WDG_OK)
        {
            chk(device_put(h->d_a, av));
            chk(device_put(h->d_x, x));
            chk(device_put(h->d_wt, wt));
            chk(device_put(h->d_D, D));
            chk(device_put(h->d_FI, FI));
            chk(device_put(h->d_FB, FB));
            chk(device_put(h->d_absA, AB));
        }
        if (st != WDG_OK)
        {
            wdg_advect_destroy(h);
            return st;
        }
        *out = h;
        return WDG_OK;
    }

    void wdg_advect_destroy(wdg_advect *h)
    {
        if (!h)
            return;
        {
            DeviceScope g(h->w ? h->w->device : 0);
            for (double *p : {h->d_a, h->d_x, h->d_wt, h->d_D, h->d_FI, h->d_FB, h->d_uf, h->d_uB, h->d_absA, h->d_rk})
                if (p)
                    cudaFree(p);
        }
        if (h->w)
            wdg_wave_destroy(h->w);
        delete h;
    }

    int wdg_advect_action(wdg_advect *h, const double *u, double *du) { return entry(h, u, du, action_dev, true); }
    int wdg_advect_bc_action(wdg_advect *h, const double *u, double *du) { return entry(h, u, du, bc_dev, true); }
    int wdg_advect_rhs(wdg_advect *h, const double *u, double *dudt) { return entry(h, u, dudt, rhs_dev, false); }

    int wdg_advect_rk4_steps(wdg_advect *h, double *u, double dt, double *t, int nsteps)
    {
        if (!h || !u || !t || nsteps < 0)
            return fail(WDG_ERR_ARG, "wdg_advect_rk4_steps: bad arguments");
        DeviceScope g(h->w->device);
        wdg_wave *w = h->w;
        const long long nd = nvals(h);
        if (!h->d_rk)
            WDG_TRY(device_alloc(&h->d_rk, 3 * (size_t)nd));
        double *bufs[3] = {h->d_rk, h->d_rk + nd, h->d_rk + 2 * nd};
        HostArg a;
        WDG_TRY(bind_arg(w, 0, u, (size_t)nd, true, true, a));
        // fused stage kernels (claw_kernels.cuh), the buffer rotation of the wave path
        WDG_TRY(claw_steps(w, 1, h->nv, h->d_a, h->d_absA, bufs, 0, a.dev, dt, t, nsteps));
        return finish_args(w, &a, 1);
    }
}
