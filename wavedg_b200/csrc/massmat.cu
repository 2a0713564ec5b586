// C-ABI: MassMatrix<AQ> (source/MassMatrix.cpp:6-227) and LinearFunctional2D
// (wavedg/LinearFunctional.hpp:61-202) on a Gauss-Lobatto or Gauss-Legendre basis, FP64 -- the
// set-up operators of the examples whose basis the wave handles do not cover
// (examples/advec2d.cpp: a Gauss-Legendre basis, the advection coefficient projected as
// M^{-1} (f, phi)).
//
//   approx_quad = true    M = diag(w_i w_j det J) at the basis nodes (MassMatrix<true>)
//   approx_quad = false   the element matrices on the (n + 1)-point Gauss-Legendre rule and their
//                         inverses (MassMatrix<false>), applied per element by one warp
//   load                  (f, phi) from f's values at the default n-point Gauss-Legendre points:
//                         f w_k w_l det J there, projected along y, then along x
//                         (LinearFunctional<2>::action), on the host, once per call
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "wave_impl.hpp"

using namespace wdg;

struct wdg_massmatrix
{
    wdg_wave *w = nullptr; // device, stream and argument staging
    const wdg_mesh *mesh_ = nullptr;
    int n = 0, nel = 0;
    bool approx = true;
    std::vector<double> corners;                 // (8, nel), for the load vector's geometry
    std::vector<double> xq, wq, B;               // the load vector's n-point rule, B(q, basis node)
    double *d_m = nullptr;                       // approx: w_i w_j det J per node
    double *d_M = nullptr, *d_Minv = nullptr;    // exact: element matrices and inverses (c, c, nel)
};

namespace
{
    __global__ void diag_kernel(const double *__restrict__ m, int nv, long long nodes, const double *x, double *y,
                                int inverse)
    {
        const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
        if (t >= nodes * nv)
            return;
        const double mi = m[t / nv];
        y[t] = inverse ? x[t] / mi : mi * x[t];
    }

    // y(d, i) = sum_j A(i, j) x(d, j) per element (A column-major, c x c); x and y may alias
    __global__ void dense_kernel(const double *__restrict__ A, int c, int nv, int nel, const double *x, double *y,
                                 int warps)
    {
        extern __shared__ double xs_all[];
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, m = nv * c;
        double *xs = xs_all + (size_t)warp * m;
        for (int el = blockIdx.x * warps + warp; el < nel; el += gridDim.x * warps)
        {
            const double *xe = x + (size_t)m * el;
            const double *Ae = A + (size_t)c * c * el;
            for (int o = lane; o < m; o += 32)
                xs[o] = xe[o];
            __syncwarp();
            for (int o = lane; o < m; o += 32)
            {
                const int i = o / nv, d = o - i * nv;
                double s = 0.0;
                for (int j = 0; j < c; ++j)
                    s += __ldg(Ae + i + (size_t)c * j) * xs[d + nv * j];
                y[(size_t)m * el + o] = s;
            }
            __syncwarp();
        }
    }

    int check(const wdg_massmatrix *h) { return h ? WDG_OK : fail(WDG_ERR_ARG, "null mass-matrix handle"); }

    int apply(wdg_massmatrix *h, int nv, const double *x, double *y, bool inverse)
    {
        const int c = h->n * h->n;
        const long long nodes = (long long)c * h->nel;
        if (h->approx)
        {
            const long long total = nodes * nv;
            diag_kernel<<<(unsigned)((total + 255) / 256), 256, 0, h->w->stream>>>(h->d_m, nv, nodes, x, y,
                                                                                  inverse ? 1 : 0);
        }
        else
        {
            const int warps = 4;
            const size_t smem = sizeof(double) * (size_t)warps * nv * c;
            if (smem > 48 * 1024)
                return fail(WDG_ERR_UNSUPPORTED, "mass matrix: n_var too large for one element in shared memory");
            const unsigned blocks = (unsigned)std::max(1, std::min((h->nel + warps - 1) / warps, 148 * 16));
            dense_kernel<<<blocks, 32 * warps, smem, h->w->stream>>>(inverse ? h->d_Minv : h->d_M, c, nv, h->nel, x, y,
                                                                      warps);
        }
        WDG_CUDA(cudaGetLastError());
        return WDG_OK;
    }
} // namespace

extern "C"
{
    int wdg_massmatrix_create(const wdg_mesh *mesh, int n_colloc, int basis_type, int approx_quad, int device,
                              wdg_massmatrix **out)
    {
        if (!mesh || !out)
            return fail(WDG_ERR_ARG, "wdg_massmatrix_create: null argument");
        *out = nullptr;
        if (n_colloc < kMinN || n_colloc > kMaxN)
            return fail(WDG_ERR_UNSUPPORTED, "wdg_massmatrix_create: n_colloc must be 2..9");
        if (basis_type != WDG_GAUSS_LEGENDRE && basis_type != WDG_GAUSS_LOBATTO)
            return fail(WDG_ERR_ARG, "wdg_massmatrix_create: basis_type must be WDG_GAUSS_LEGENDRE or WDG_GAUSS_LOBATTO");
        const int n = n_colloc, c = n * n;
        std::vector<double> xb(n), wb(n);
        if (basis_type == WDG_GAUSS_LEGENDRE)
            gauss_legendre(n, xb.data(), wb.data());
        else
            gauss_lobatto(n, xb.data(), wb.data());
        wdg_massmatrix *h = new wdg_massmatrix;
        h->n = n;
        h->nel = mesh->nel;
        h->approx = approx_quad != 0;
        h->corners = mesh->corners;
        h->xq.resize(n);
        h->wq.resize(n);
        h->B.resize((size_t)n * n);
        gauss_legendre(n, h->xq.data(), h->wq.data()); // LinearFunctional's default n-point rule
        interp_matrix(n, xb.data(), n, h->xq.data(), h->B.data());
        int st = wdg_wave_create(mesh, n, nullptr, WDG_FP64, device, &h->w);
        if (st == WDG_OK)
        {
            DeviceScope g(h->w->device);
            if (h->approx)
            {
                std::vector<double> m((size_t)c * h->nel);
                for (int el = 0; el < h->nel; ++el)
                    for (int j = 0; j < n; ++j)
                        for (int i = 0; i < n; ++i)
                        {
                            double J[4];
                            quad_jacobian(&mesh->corners[8 * (size_t)el], xb[i], xb[j], J);
                            m[i + n * j + (size_t)c * el] = wb[i] * wb[j] * (J[0] * J[3] - J[1] * J[2]);
                        }
                st = device_alloc(&h->d_m, m.size());
                if (st == WDG_OK)
                    st = device_put(h->d_m, m);
            }
            else
            {
                std::vector<double> Mf, Mi;
                st = exact_mass(*mesh, n, xb.data(), 1 + (2 * (n - 1) + 2) / 2, Mf, Mi);
                if (st == WDG_OK)
                    st = device_alloc(&h->d_M, Mf.size());
                if (st == WDG_OK)
                    st = device_put(h->d_M, Mf);
                if (st == WDG_OK)
                    st = device_alloc(&h->d_Minv, Mi.size());
                if (st == WDG_OK)
                    st = device_put(h->d_Minv, Mi);
            }
        }
        if (st != WDG_OK)
        {
            wdg_massmatrix_destroy(h);
            return st;
        }
        *out = h;
        return WDG_OK;
    }

    void wdg_massmatrix_destroy(wdg_massmatrix *h)
    {
        if (!h)
            return;
        if (h->w)
        {
            DeviceScope g(h->w->device);
            for (double *p : {h->d_m, h->d_M, h->d_Minv})
                if (p)
                    cudaFree(p);
            wdg_wave_destroy(h->w);
        }
        delete h;
    }

    int wdg_massmatrix_set_stream(wdg_massmatrix *h, void *stream)
    {
        WDG_TRY(check(h));
        return wdg_wave_set_stream(h->w, stream);
    }

    // MassMatrix::action: y = M x (x, y of n_var values per node)
    int wdg_massmatrix_action(wdg_massmatrix *h, int n_var, const double *x, double *y)
    {
        WDG_TRY(check(h));
        if (!x || !y || n_var < 1)
            return fail(WDG_ERR_ARG, "wdg_massmatrix_action: bad arguments");
        DeviceScope g(h->w->device);
        const size_t cnt = (size_t)n_var * h->n * h->n * h->nel;
        HostArg a[2];
        const bool same = x == y;
        WDG_TRY(bind_arg(h->w, 0, x, cnt, true, same, a[0]));
        if (!same)
            WDG_TRY(bind_arg(h->w, 1, y, cnt, false, true, a[1]));
        WDG_TRY(apply(h, n_var, a[0].dev, same ? a[0].dev : a[1].dev, false));
        return finish_args(h->w, a, same ? 1 : 2);
    }

    // MassMatrix::inv: x = M^{-1} x in place
    int wdg_massmatrix_inv(wdg_massmatrix *h, int n_var, double *x)
    {
        WDG_TRY(check(h));
        if (!x || n_var < 1)
            return fail(WDG_ERR_ARG, "wdg_massmatrix_inv: bad arguments");
        DeviceScope g(h->w->device);
        const size_t cnt = (size_t)n_var * h->n * h->n * h->nel;
        HostArg a;
        WDG_TRY(bind_arg(h->w, 0, x, cnt, true, true, a));
        WDG_TRY(apply(h, n_var, a.dev, a.dev, true));
        return finish_args(h->w, &a, 1);
    }

    // the points LinearFunctional2D::action evaluates f at: (x, y) of point k + n (l + n el),
    // the default n-point Gauss-Legendre rule mapped into element el (host array, 2 n^2 nel)
    int wdg_massmatrix_points(const wdg_massmatrix *h, double *xy)
    {
        WDG_TRY(check(h));
        if (!xy)
            return fail(WDG_ERR_ARG, "wdg_massmatrix_points: null argument");
        const int n = h->n;
        for (int el = 0; el < h->nel; ++el)
        {
            const double *c = &h->corners[8 * (size_t)el];
            for (int l = 0; l < n; ++l)
                for (int k = 0; k < n; ++k)
                {
                    const double xi = h->xq[k], eta = h->xq[l];
                    const double s0 = 0.25 * (1 - xi) * (1 - eta), s1 = 0.25 * (1 + xi) * (1 - eta);
                    const double s2 = 0.25 * (1 + xi) * (1 + eta), s3 = 0.25 * (1 - xi) * (1 + eta);
                    double *p = xy + 2 * (k + (size_t)n * (l + (size_t)n * el));
                    p[0] = s0 * c[0] + s1 * c[2] + s2 * c[4] + s3 * c[6];
                    p[1] = s0 * c[1] + s1 * c[3] + s2 * c[5] + s3 * c[7];
                }
        }
        return WDG_OK;
    }

    // LinearFunctional2D::action: F(d, i, j, el) = (f_d, phi_ij) from fq(d, point), f's values at
    // wdg_massmatrix_points (host array); F host or device
    int wdg_massmatrix_load(wdg_massmatrix *h, int n_var, const double *fq, double *F)
    {
        WDG_TRY(check(h));
        if (!fq || !F || n_var < 1)
            return fail(WDG_ERR_ARG, "wdg_massmatrix_load: bad arguments");
        const int n = h->n, nv = n_var;
        std::vector<double> out((size_t)nv * n * n * h->nel), Fq((size_t)nv * n * n), Pj((size_t)nv * n * n);
        for (int el = 0; el < h->nel; ++el)
        {
            const double *c = &h->corners[8 * (size_t)el];
            // f w_k w_l det J at the points
            for (int l = 0; l < n; ++l)
                for (int k = 0; k < n; ++k)
                {
                    double J[4];
                    quad_jacobian(c, h->xq[k], h->xq[l], J);
                    const double w = (J[0] * J[3] - J[1] * J[2]) * h->wq[k] * h->wq[l];
                    for (int d = 0; d < nv; ++d)
                        Fq[d + nv * (k + (size_t)n * l)] =
                            fq[d + nv * (k + (size_t)n * (l + (size_t)n * el))] * w;
                }
            // along y: P(d, k, j) = sum_l Fq(d, k, l) B(l, j); along x: F(d, i, j) = sum_k P(d, k, j) B(k, i)
            for (int j = 0; j < n; ++j)
                for (int k = 0; k < n; ++k)
                    for (int d = 0; d < nv; ++d)
                    {
                        double s = 0.0;
                        for (int l = 0; l < n; ++l)
                            s += Fq[d + nv * (k + (size_t)n * l)] * h->B[l + (size_t)n * j];
                        Pj[d + nv * (k + (size_t)n * j)] = s;
                    }
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i)
                    for (int d = 0; d < nv; ++d)
                    {
                        double s = 0.0;
                        for (int k = 0; k < n; ++k)
                            s += Pj[d + nv * (k + (size_t)n * j)] * h->B[k + (size_t)n * i];
                        out[d + nv * (i + (size_t)n * (j + (size_t)n * el))] = s;
                    }
        }
        DeviceScope g(h->w->device);
        bool dev = false;
        WDG_TRY(is_device_ptr(h->w, F, dev));
        if (dev)
        {
            WDG_CUDA(cudaMemcpyAsync(F, out.data(), out.size() * sizeof(double), cudaMemcpyHostToDevice, h->w->stream));
            WDG_CUDA(cudaStreamSynchronize(h->w->stream));
        }
        else
            std::copy(out.begin(), out.end(), F);
        return WDG_OK;
    }
}
