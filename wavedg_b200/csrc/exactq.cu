// C-ABI: the wave system with exact quadrature (approx_quad = false).
//
//   WaveEquation(mesh, basis, false)  source/WaveEquation.cpp:5-30
//     Div<false>       source/Div.cpp:312-361 (op_2d_cc), div_2d_q :469-588
//     EdgeFlux<false>  source/EdgeFlux.cpp:496-535, flux_action_2d_q :548-622
//   WaveBC(mesh, bc, basis, false)    source/WaveEquation.cpp:70-105, 190-215
//   MassMatrix<false>(mesh, basis)    source/MassMatrix.cpp:84-230; chol, solve_chol,
//                                     mult_chol in source/linalg.cpp:5-100
//
// Quadrature rules are the reference's defaults for bilinear elements (Gauss-Legendre):
// Div 1 + ((n-2) + (n-1) + 1) / 2 points per direction, EdgeFlux and MassMatrix
// 1 + (2 (n-1) + 2) / 2.  Face prolongation, the exterior states of the boundary codes and
// the argument staging are the collocation handle's (an internal wdg_wave, FP64).
//
// FP64 only.  The accuracy path for callers that set approx_quad = false.  The RHS and every
// RK4 stage (WaveHoltz periods included) are one fused launch, a warp per element
// (qfused_kernel: volume term, the four faces through the partner table, forcing, the dense
// inverse mass matrix formed at set-up from the block Cholesky factors, the stage update);
// the operator entry points (Div, EdgeFlux, the mass matrix and its inverse) keep component
// kernels in the reference layouts: one CTA per element for the volume term, one thread per
// edge for the face term, one warp per element for the dense mass products.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

#include "wave_bc.cuh"
#include "wave_impl.hpp"

using namespace wdg;

struct wdg_waveq
{
    wdg_wave *w = nullptr;
    int n = 0, nqd = 0, nqf = 0, nqm = 0;
    double *d_xd = nullptr, *d_wd = nullptr, *d_Pd = nullptr, *d_Dd = nullptr; // Div rule, P(i,k), D(i,k)
    double *d_wf = nullptr, *d_Pf = nullptr;                                   // face rule, P(i,k)
    double *d_nI = nullptr, *d_nB = nullptr; // per edge (n_x, n_y, |E| / 2)
    double *d_M = nullptr, *d_Minv = nullptr; // element mass matrices and their inverses (n^2, n^2, nel)
    double *d_uf = nullptr, *d_uB = nullptr; // face traces
};

namespace wdg
{
    // D(i, j) = phi_j'(xq_i) for the Lagrange basis on the nodes x, by the barycentric
    // derivative formula: at a node the diagonal form, elsewhere the quotient form
    // (lagrange_basis_deriv, source/lagrange_interpolation.cpp:33-50, 96-139)
    void lagrange_deriv_at(int n, const double *x, int nq, const double *xq, double *D)
    {
        std::vector<double> lw(n), B((size_t)nq * n);
        for (int i = 0; i < n; ++i)
        {
            double p = 1.0;
            for (int j = 0; j < n; ++j)
                if (j != i)
                    p *= x[i] - x[j];
            lw[i] = 1.0 / p;
        }
        const auto mm = std::minmax_element(lw.begin(), lw.end());
        const double diff = *mm.second - *mm.first;
        for (double &v : lw)
            v /= diff;
        interp_matrix(n, x, nq, xq, B.data());
        const double eps = 2.220446049250313e-16;
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < nq; ++i)
            {
                const double x0 = xq[i], p = B[i + (size_t)nq * j];
                int at = -1;
                for (int k = 0; k < n; ++k)
                    if (x0 == x[k] || std::abs(x0 - x[k]) <= eps)
                        at = k;
                double A = 0.0, S = 0.0;
                if (at >= 0)
                {
                    S = -lw[at];
                    for (int k = 0; k < n; ++k)
                        if (k != at)
                            A += lw[k] * (p - (k == j ? 1.0 : 0.0)) / (x0 - x[k]);
                }
                else
                    for (int k = 0; k < n; ++k)
                    {
                        const double t = lw[k] / (x0 - x[k]);
                        A += t * (p - (k == j ? 1.0 : 0.0)) / (x0 - x[k]);
                        S += t;
                    }
                D[i + (size_t)nq * j] = A / S;
            }
    }

    const double *waveq_minv(const wdg_waveq *h) { return h->d_Minv; }

    // MassMatrix<false> (source/MassMatrix.cpp:84-227) on the basis with nodes x: the element
    // mass matrices M(i, j) = sum_p w_p det J_p phi_i phi_j on the qm x qm Gauss-Legendre rule
    // (lower triangle, Cholesky in place; chol, linalg.cpp:5-30) and their inverses, solved
    // column by column (solve_chol, linalg.cpp:32-66); (n^2, n^2, nel) each
    int exact_mass(const wdg_mesh &mesh, int n, const double *x, int qm, std::vector<double> &Mf,
                   std::vector<double> &Mi)
    {
        const int c = n * n, q2 = qm * qm;
        std::vector<double> xm(qm), wm(qm), Bm((size_t)qm * n), L((size_t)c * c, 0.0), detJ(q2);
        Mf.assign((size_t)c * c * mesh.nel, 0.0);
        Mi.assign((size_t)c * c * mesh.nel, 0.0);
        gauss_legendre(qm, xm.data(), wm.data());
        interp_matrix(n, x, qm, xm.data(), Bm.data());
        int st = WDG_OK;
        for (int el = 0; el < mesh.nel && st == WDG_OK; ++el)
        {
            const double *cr = &mesh.corners[8 * (size_t)el];
            for (int p = 0; p < q2; ++p)
            {
                double J[4];
                quad_jacobian(cr, xm[p % qm], xm[p / qm], J);
                detJ[p] = J[0] * J[3] - J[2] * J[1];
            }
            double *M = L.data();
            std::fill(L.begin(), L.end(), 0.0);
            for (int j = 0; j < c; ++j)
                for (int i = j; i < c; ++i)
                {
                    double mij = 0.0;
                    for (int p = 0; p < q2; ++p)
                    {
                        const double bi = Bm[p % qm + qm * (i % n)] * Bm[p / qm + qm * (i / n)];
                        const double bj = Bm[p % qm + qm * (j % n)] * Bm[p / qm + qm * (j / n)];
                        mij += bi * bj * detJ[p] * wm[p % qm] * wm[p / qm];
                    }
                    M[i + c * j] = mij;
                    Mf[(size_t)c * c * el + i + c * j] = mij;
                    Mf[(size_t)c * c * el + j + c * i] = mij;
                }
            for (int k = 0; k < c && st == WDG_OK; ++k)
            {
                for (int j = k + 1; j < c; ++j)
                {
                    const double sc = M[j + c * k] / M[k + c * k];
                    for (int i = j; i < c; ++i)
                        M[i + c * j] -= sc * M[i + c * k];
                }
                if (!(M[k + c * k] > 0.0))
                    st = fail(WDG_ERR_ARG, "an element mass matrix is not positive definite");
                else
                {
                    const double sc = 1.0 / std::sqrt(M[k + c * k]);
                    for (int i = k; i < c; ++i)
                        M[i + c * k] *= sc;
                }
            }
            // M^{-1} column by column: solve_chol on the unit vectors (linalg.cpp:32-66)
            for (int col = 0; col < c && st == WDG_OK; ++col)
            {
                double *X = &Mi[(size_t)c * c * el + (size_t)c * col];
                for (int i = 0; i < c; ++i)
                    X[i] = (i == col) ? 1.0 : 0.0;
                for (int j = 0; j < c; ++j)
                {
                    X[j] /= M[j + c * j];
                    for (int i = j + 1; i < c; ++i)
                        X[i] -= M[i + c * j] * X[j];
                }
                for (int j = c - 1; j >= 0; --j)
                {
                    X[j] /= M[j + c * j];
                    for (int i = 0; i < j; ++i)
                        X[i] -= M[j + c * i] * X[j];
                }
            }
        }
        return st;
    }

} // namespace wdg

namespace
{
    constexpr int kMaxQ = 16;

    int qdiv(int n) { return 1 + ((n - 2) + (n - 1) + 1) / 2; }
    int qface(int n) { return 1 + (2 * (n - 1) + 2) / 2; }

    // QuadElement::jacobian (source/Element.cpp:21-27): J = (x_xi, y_xi, x_eta, y_eta)
    __host__ __device__ inline void jac(const double *c, double xi, double eta, double J[4])
    {
        J[0] = 0.25 * ((1.0 - eta) * (c[2] - c[0]) + (1.0 + eta) * (c[4] - c[6]));
        J[1] = 0.25 * ((1.0 - eta) * (c[3] - c[1]) + (1.0 + eta) * (c[5] - c[7]));
        J[2] = 0.25 * ((1.0 - xi) * (c[6] - c[0]) + (1.0 + xi) * (c[4] - c[2]));
        J[3] = 0.25 * ((1.0 - xi) * (c[7] - c[1]) + (1.0 + xi) * (c[5] - c[3]));
    }

    // ---------------------------------------------------------------- Div<false>
    // One CTA per element, shared memory per element: u, P u (one direction), U at the points,
    // the two contravariant fluxes, and the two half-contracted sums.  Accumulates into du.
    __global__ void qdiv_kernel(int n, int q, int nel, const double *__restrict__ corners,
                                const double *__restrict__ xd, const double *__restrict__ wd,
                                const double *__restrict__ Pd, const double *__restrict__ Dd,
                                const double *__restrict__ u, double *du)
    {
        extern __shared__ double sm[];
        const int nn = n * n, qq = q * q;
        double *su = sm;                 // (3, n, n)
        double *Pu = su + 3 * nn;        // (n, 3, q)
        double *Uq = Pu + 3 * n * q;     // (3, q, q)
        double *Fq = Uq + 3 * qq;        // (2, 3, q, q)
        double *Df = Fq + 6 * qq;        // (q, 3, n)
        double *Pg = Df + 3 * q * n;     // (q, 3, n)
        const int t = threadIdx.x, T = blockDim.x;
        for (int el = blockIdx.x; el < nel; el += gridDim.x)
        {
            const double *ue = u + (size_t)3 * nn * el;
            for (int k = t; k < 3 * nn; k += T)
                su[k] = ue[k];
            __syncthreads();
            // Pu(l, d, i) = sum_k P(i, k) u(d, k, l)
            for (int o = t; o < 3 * n * q; o += T)
            {
                const int l = o % n, d = (o / n) % 3, i = o / (3 * n);
                double s = 0.0;
                for (int k = 0; k < n; ++k)
                    s += Pd[i + q * k] * su[d + 3 * (k + n * l)];
                Pu[o] = s;
            }
            __syncthreads();
            // U(d, i, j) = sum_l P(j, l) Pu(l, d, i)
            for (int o = t; o < 3 * qq; o += T)
            {
                const int d = o % 3, i = (o / 3) % q, j = o / (3 * q);
                double s = 0.0;
                for (int l = 0; l < n; ++l)
                    s += Pd[j + q * l] * Pu[l + n * (d + 3 * i)];
                Uq[o] = s;
            }
            __syncthreads();
            // contravariant fluxes of the wave system at the points (op_2d_cc with the wave
            // table: F = W (y_eta u - x_eta v, y_eta p, -x_eta p), G = W (-y_xi u + x_xi v, -y_xi p, x_xi p))
            const double *ce = corners + 8 * (size_t)el;
            for (int o = t; o < qq; o += T)
            {
                const int i = o % q, j = o / q;
                double J[4];
                jac(ce, xd[i], xd[j], J);
                const double W = wd[i] * wd[j];
                const double Xxi = J[0] * W, Yxi = J[1] * W, Xeta = J[2] * W, Yeta = J[3] * W;
                const double *U = Uq + 3 * o;
                double *F = Fq + 6 * o;
                F[0] = Yeta * U[1] - Xeta * U[2];
                F[1] = -Yxi * U[1] + Xxi * U[2];
                F[2] = Yeta * U[0];
                F[3] = -Yxi * U[0];
                F[4] = -Xeta * U[0];
                F[5] = Xxi * U[0];
            }
            __syncthreads();
            // Df(j, d, k) = sum_i D(i, k) F(d, i, j);  Pg(j, d, k) = sum_i P(i, k) G(d, i, j)
            for (int o = t; o < 3 * q * n; o += T)
            {
                const int j = o % q, d = (o / q) % 3, k = o / (3 * q);
                double df = 0.0, pg = 0.0;
                for (int i = 0; i < q; ++i)
                {
                    df += Dd[i + q * k] * Fq[2 * d + 6 * (i + q * j)];
                    pg += Pd[i + q * k] * Fq[2 * d + 1 + 6 * (i + q * j)];
                }
                Df[o] = df;
                Pg[o] = pg;
            }
            __syncthreads();
            // du(d, k, l) += sum_j P(j, l) Df(j, d, k) + D(j, l) Pg(j, d, k)
            double *de = du + (size_t)3 * nn * el;
            for (int o = t; o < 3 * nn; o += T)
            {
                const int d = o % 3, k = (o / 3) % n, l = o / (3 * n);
                double s = 0.0;
                for (int j = 0; j < q; ++j)
                    s += Pd[j + q * l] * Df[j + q * (d + 3 * k)] + Dd[j + q * l] * Pg[j + q * (d + 3 * k)];
                de[o] += s;
            }
            __syncthreads();
        }
    }

    // ---------------------------------------------------------------- EdgeFlux<false>
    // One thread per edge: both sides' traces to the face points, upwind flux there (a = -1,
    // b = -1/2 of the wave system, in closed form: side 0 contributes -1/2 v (v . U0),
    // v = (1, n_x, n_y); side 1 +1/2 w (w . U1), w = (1, -n_x, -n_y)), weighted by
    // w_q |E| / 2, then back to the nodes; side 1 gets the negative.  fb may equal ub.
    __global__ void qflux_kernel(int n, int q, int ne, const double *__restrict__ nrm, const double *__restrict__ wf,
                                 const double *__restrict__ Pf, const double *ub, double *fb)
    {
        const int e = blockIdx.x * blockDim.x + threadIdx.x;
        if (e >= ne)
            return;
        const double nx = nrm[3 * e], ny = nrm[3 * e + 1], meas = nrm[3 * e + 2];
        double uf[kMaxQ][3];
        for (int i = 0; i < q; ++i)
        {
            double U0[3], U1[3];
            for (int d = 0; d < 3; ++d)
            {
                double a = 0.0, b = 0.0;
                for (int j = 0; j < n; ++j)
                {
                    a += ub[j + n * (d + 3 * (0 + 2 * (size_t)e))] * Pf[i + q * j];
                    b += ub[j + n * (d + 3 * (1 + 2 * (size_t)e))] * Pf[i + q * j];
                }
                U0[d] = a;
                U1[d] = b;
            }
            const double w = wf[i] * meas;
            const double s0 = -0.5 * w * (U0[0] + nx * U0[1] + ny * U0[2]);
            const double s1 = 0.5 * w * (U1[0] - nx * U1[1] - ny * U1[2]);
            uf[i][0] = s0 + s1;
            uf[i][1] = nx * (s0 - s1);
            uf[i][2] = ny * (s0 - s1);
        }
        for (int d = 0; d < 3; ++d)
            for (int i = 0; i < n; ++i)
            {
                double f = 0.0;
                for (int j = 0; j < q; ++j)
                    f += uf[j][d] * Pf[j + q * i];
                fb[i + n * (d + 3 * (0 + 2 * (size_t)e))] = f;
                fb[i + n * (d + 3 * (1 + 2 * (size_t)e))] = -f;
            }
    }

    // ---------------------------------------------------------------- MassMatrix<false>
    // x <- A x per element for a dense n^2 x n^2 matrix A (the element mass matrix, or its
    // inverse formed at set-up from the Cholesky factors), nv interleaved right-hand sides,
    // in place: one warp per element, the element's x staged in shared memory; lanes take
    // consecutive rows, so each column of A is read coalesced.
    __global__ void qdense_kernel(int c, int nel, int nv, const double *__restrict__ A, double *x)
    {
        extern __shared__ double sx[];
        const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
        double *xs = sx + (size_t)wib * nv * c;
        const int m = nv * c;
        for (int el = blockIdx.x * wpb + wib; el < nel; el += gridDim.x * wpb)
        {
            double *xe = x + (size_t)m * el;
            const double *Ae = A + (size_t)c * c * el;
            for (int o = lane; o < m; o += 32)
                xs[o] = xe[o];
            __syncwarp();
            for (int o = lane; o < m; o += 32)
            {
                const int i = o / nv, d = o - i * nv;
                double y = 0.0;
                for (int j = 0; j < c; ++j)
                    y += Ae[i + (size_t)c * j] * xs[d + nv * j];
                xe[o] = y;
            }
            __syncwarp();
        }
    }

    // ---------------------------------------------------------------- fused RHS / RK4 stage
    // One warp per element does what rhs_dev's chain of launches does, in one pass over the
    // element: the Gauss-point volume term of Div<false> (as qdiv_kernel), the four faces of
    // EdgeFlux<false> / WaveBC (the element's own nodal trace and its neighbour's, read through
    // the fused kernels' partner table, or the exterior state of the boundary code at the
    // nodes, both interpolated to the face rule; the closed-form upwind flux of qflux_kernel
    // with the element's own outward normal, which makes the two elements of an edge add
    // exactly opposite terms; projected back to the face nodes), the forcing s F, the dense
    // inverse mass matrix, then the RHS or the RK4 stage update (with the WaveHoltz filter on
    // the last stage).
    struct QFusedArgs
    {
        const double *x;      // state the RHS is evaluated at
        double *out;          // RHS: dudt; RK4: u'
        double *du;           // RK4 register
        const double *F;      // forcing (nullable) times fs
        double fs;
        double *acc;          // FP64 filter (stage 4, nullable) += acc_c u'
        double acc_c;
        const double *corners, *xd, *wd, *Pd, *Dd, *wf, *Pf, *Minv;
        const int4 *fbase;
        const uint32_t *fcode;
        unsigned *err;
        int n, q, qf, nel, rk; // rk: 0 RHS, 1 RK4 stage (rk_a == 0 on the first)
        double rk_a, rk_b, dt;
    };
    constexpr int kQWarps = 4;

    __host__ __device__ inline int qfused_warp_doubles(int n, int q, int qf)
    {
        // su r (3 n^2 each) | Pu (3 n q) | Uq (3 q^2) | Fq (7 q^2: six fluxes per point at an odd
        // stride, which spreads a warp's accesses over the shared-memory banks) | Df Pg (3 q n
        // each) | T1 (4 n 3) | UF (4 qf 3)
        return 6 * n * n + 3 * n * q + 10 * q * q + 6 * q * n + 12 * n + 12 * qf;
    }

    // outward unit normal and measure (length / 2) of side s (StraightEdge, wavedg/Edge.hpp:107-122);
    // side s runs from corner p0 to p1: 0: 0 -> 1, 1: 1 -> 2, 2: 3 -> 2, 3: 0 -> 3
    __device__ inline void qside(const double *c, int s, double &nx, double &ny, double &meas)
    {
        const int p0 = (s == 0 || s == 3) ? 0 : (s == 1 ? 1 : 3), p1 = (s == 0) ? 1 : (s == 3 ? 3 : 2);
        const double dx = c[2 * p1] - c[2 * p0], dy = c[2 * p1 + 1] - c[2 * p0 + 1];
        const double len = sqrt(dx * dx + dy * dy), sgn = (s >= 2) ? -1.0 : 1.0;
        nx = sgn * dy / len;
        ny = -sgn * dx / len;
        meas = 0.5 * len;
    }
    // partner walk of a side code (bits 0-1): +3, -3, +3n, -3n values per face node
    __device__ inline int qstride(int n, uint32_t byte)
    {
        const uint32_t c = byte & 3u;
        return (c == 0) ? 3 : (c == 1) ? -3 : (c == 2) ? 3 * n : -3 * n;
    }

    __device__ inline int qface_node(int n, int s, int k)
    {
        const int i = (s == 0 || s == 2) ? k : (s == 1 ? n - 1 : 0);
        const int j = (s == 1 || s == 3) ? k : (s == 2 ? n - 1 : 0);
        return i + n * j;
    }

    __global__ void __launch_bounds__(32 * kQWarps) qfused_kernel(const QFusedArgs a)
    {
        extern __shared__ double qsm[];
        const int n = a.n, q = a.q, qf = a.qf, nn = n * n, qq = q * q;
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        double *su = qsm + (size_t)warp * qfused_warp_doubles(n, q, qf);
        double *r = su + 3 * nn, *Pu = r + 3 * nn, *Uq = Pu + 3 * n * q, *Fq = Uq + 3 * qq, *Df = Fq + 7 * qq;
        double *Pg = Df + 3 * q * n, *T1 = Pg + 3 * q * n, *UF = T1 + 12 * n;
        const long long limit = 3LL * nn * a.nel;
        for (int el = blockIdx.x * kQWarps + warp; el < a.nel; el += gridDim.x * kQWarps)
        {
            const double *ue = a.x + (size_t)3 * nn * el;
            for (int k = lane; k < 3 * nn; k += 32)
            {
                su[k] = ue[k];
                r[k] = 0.0;
            }
            double c[8];
            for (int k = 0; k < 8; ++k)
                c[k] = __ldg(a.corners + 8 * (size_t)el + k);
            const uint32_t codes = __ldg(a.fcode + el);
            const int4 fb = __ldg(a.fbase + el);
            __syncwarp();
            // ---- volume (Div<false>): Pu, U at the points, fluxes, half contractions, back
            for (int o = lane; o < 3 * n * q; o += 32)
            {
                const int l = o % n, d = (o / n) % 3, i = o / (3 * n);
                double s = 0.0;
                for (int k = 0; k < n; ++k)
                    s += a.Pd[i + q * k] * su[d + 3 * (k + n * l)];
                Pu[o] = s;
            }
            __syncwarp();
            for (int o = lane; o < 3 * qq; o += 32)
            {
                const int d = o % 3, i = (o / 3) % q, j = o / (3 * q);
                double s = 0.0;
                for (int l = 0; l < n; ++l)
                    s += a.Pd[j + q * l] * Pu[l + n * (d + 3 * i)];
                Uq[o] = s;
            }
            __syncwarp();
            for (int o = lane; o < qq; o += 32)
            {
                const int i = o % q, j = o / q;
                double J[4];
                jac(c, a.xd[i], a.xd[j], J);
                const double W = a.wd[i] * a.wd[j];
                const double Xxi = J[0] * W, Yxi = J[1] * W, Xeta = J[2] * W, Yeta = J[3] * W;
                const double *U = Uq + 3 * o;
                double *Fo = Fq + 7 * o;
                Fo[0] = Yeta * U[1] - Xeta * U[2];
                Fo[1] = -Yxi * U[1] + Xxi * U[2];
                Fo[2] = Yeta * U[0];
                Fo[3] = -Yxi * U[0];
                Fo[4] = -Xeta * U[0];
                Fo[5] = Xxi * U[0];
            }
            __syncwarp();
            for (int o = lane; o < 3 * q * n; o += 32)
            {
                const int j = o % q, d = (o / q) % 3, k = o / (3 * q);
                double df = 0.0, pg = 0.0;
                for (int i = 0; i < q; ++i)
                {
                    df += a.Dd[i + q * k] * Fq[2 * d + 7 * (i + q * j)];
                    pg += a.Pd[i + q * k] * Fq[2 * d + 1 + 7 * (i + q * j)];
                }
                Df[o] = df;
                Pg[o] = pg;
            }
            // ---- neighbour / exterior nodal traces of the four sides, face-node order: T1(s, k, d)
            for (int o = lane; o < 4 * n; o += 32)
            {
                const int s = o / n, k = o - s * n;
                const uint32_t byte = (codes >> (8 * s)) & 0xffu;
                const double *own = su + 3 * qface_node(n, s, k);
                double *t1 = T1 + 3 * o;
                if (byte & 0x80u)
                {
                    double nx, ny, meas;
                    qside(c, s, nx, ny, meas);
                    const double qv[3] = {own[0], own[1], own[2]};
                    exterior<double>((int)((byte >> 3) & 3u), nx, ny, qv, t1);
                }
                else
                {
                    const int off = (s == 0) ? fb.x : (s == 1) ? fb.y : (s == 2) ? fb.z : fb.w;
                    const long long pos = (long long)off + (long long)k * qstride(n, byte);
                    if (off < 0 || pos < 0 || pos + 3 > limit)
                    {
                        atomicOr(a.err, 2u);
                        t1[0] = own[0];
                        t1[1] = own[1];
                        t1[2] = own[2];
                    }
                    else
                    {
                        t1[0] = __ldg(a.x + pos);
                        t1[1] = __ldg(a.x + pos + 1);
                        t1[2] = __ldg(a.x + pos + 2);
                    }
                }
            }
            __syncwarp();
            // volume result into r
            for (int o = lane; o < 3 * nn; o += 32)
            {
                const int d = o % 3, k = (o / 3) % n, l = o / (3 * n);
                double s = 0.0;
                for (int j = 0; j < q; ++j)
                    s += a.Pd[j + q * l] * Df[j + q * (d + 3 * k)] + a.Dd[j + q * l] * Pg[j + q * (d + 3 * k)];
                r[o] = s;
            }
            // ---- face points: both traces to the face rule, upwind flux: UF(s, i, d)
            for (int o = lane; o < 4 * qf; o += 32)
            {
                const int s = o / qf, i = o - s * qf;
                double nx, ny, meas;
                qside(c, s, nx, ny, meas);
                double U0[3] = {0.0, 0.0, 0.0}, U1[3] = {0.0, 0.0, 0.0};
                for (int j = 0; j < n; ++j)
                {
                    const double p = a.Pf[i + qf * j];
                    const double *own = su + 3 * qface_node(n, s, j), *nb = T1 + 3 * (s * n + j);
                    for (int d = 0; d < 3; ++d)
                    {
                        U0[d] += own[d] * p;
                        U1[d] += nb[d] * p;
                    }
                }
                const double w = a.wf[i] * meas;
                const double s0 = -0.5 * w * (U0[0] + nx * U0[1] + ny * U0[2]);
                const double s1 = 0.5 * w * (U1[0] - nx * U1[1] - ny * U1[2]);
                UF[3 * o] = s0 + s1;
                UF[3 * o + 1] = nx * (s0 - s1);
                UF[3 * o + 2] = ny * (s0 - s1);
            }
            __syncwarp();
            // back to the face nodes: sides 0 and 2, then 1 and 3 (corner nodes are shared only
            // by neighbouring sides)
            for (int pass = 0; pass < 2; ++pass)
            {
                for (int o = lane; o < 2 * n; o += 32)
                {
                    const int s = pass + 2 * (o / n), k = o % n;
                    const int node = qface_node(n, s, k);
                    for (int d = 0; d < 3; ++d)
                    {
                        double f = 0.0;
                        for (int j = 0; j < qf; ++j)
                            f += UF[3 * (s * qf + j) + d] * a.Pf[j + qf * k];
                        r[3 * node + d] += f;
                    }
                }
                __syncwarp();
            }
            // ---- forcing, then M^{-1} and the output: lane per row of the element's matrix
            if (a.F)
            {
                for (int o = lane; o < 3 * nn; o += 32)
                    r[o] += a.fs * __ldg(a.F + (size_t)3 * nn * el + o);
                __syncwarp();
            }
            const double *Me = a.Minv + (size_t)nn * nn * el;
            for (int row = lane; row < nn; row += 32)
            {
                double y[3] = {0.0, 0.0, 0.0};
                for (int j = 0; j < nn; ++j)
                {
                    const double m = __ldg(Me + row + (size_t)nn * j);
                    y[0] += m * r[3 * j];
                    y[1] += m * r[3 * j + 1];
                    y[2] += m * r[3 * j + 2];
                }
                const size_t g = (size_t)3 * (nn * (size_t)el + row);
                for (int d = 0; d < 3; ++d)
                {
                    if (!a.rk)
                    {
                        a.out[g + d] = y[d];
                        continue;
                    }
                    const double kd = (a.rk_a == 0.0) ? a.dt * y[d] : a.rk_a * a.du[g + d] + a.dt * y[d];
                    a.du[g + d] = kd;
                    const double un = su[3 * row + d] + a.rk_b * kd;
                    a.out[g + d] = un;
                    if (a.acc)
                        a.acc[g + d] += a.acc_c * un;
                }
            }
            __syncwarp();
        }
    }




    size_t face_count(const wdg_waveq *h, int type)
    {
        return (size_t)h->n * 3 * 2 * (type == 0 ? h->w->nI : h->w->nB);
    }

    // one launch of the fused kernel on the handle's tables (shared memory above 48 KB is opted
    // in once per device when the handle is created)
    int qfused_launch(wdg_waveq *h, QFusedArgs &a)
    {
        wdg_wave *w = h->w;
        a.corners = w->d_corners;
        a.xd = h->d_xd;
        a.wd = h->d_wd;
        a.Pd = h->d_Pd;
        a.Dd = h->d_Dd;
        a.wf = h->d_wf;
        a.Pf = h->d_Pf;
        a.Minv = h->d_Minv;
        a.fbase = w->d_fbase;
        a.fcode = w->d_fcode;
        a.err = w->d_err;
        a.n = h->n;
        a.q = h->nqd;
        a.qf = h->nqf;
        a.nel = w->nel;
        const size_t smem = sizeof(double) * kQWarps * qfused_warp_doubles(h->n, h->nqd, h->nqf);
        const unsigned blocks = (unsigned)std::max(1, std::min((w->nel + kQWarps - 1) / kQWarps, 148 * 16));
        qfused_kernel<<<blocks, 32 * kQWarps, smem, w->stream>>>(a);
        WDG_CUDA(cudaGetLastError());
        return WDG_OK;
    }

    // nsteps of ode::RungeKutta4 on device array u (not a rotation buffer), one fused launch per
    // stage: the rotation u -> B -> C -> B -> C -> u of the wave handle's buffers; with F, the
    // forcing F s(t) at the stage times; with acc, acc += c_filter[step] u after each step
    int qfused_rk4(wdg_waveq *h, double *u, double dt, double t, int nsteps, const double *F, double omega,
                   double *acc, const double *c_filter)
    {
        wdg_wave *w = h->w;
        WDG_TRY(ensure_states(w));
        double *B = static_cast<double *>(w->d_state[1]), *Cb = static_cast<double *>(w->d_state[2]);
        QFusedArgs a{};
        a.du = static_cast<double *>(w->d_du);
        a.rk = 1;
        a.dt = dt;
        a.F = F;
        for (int step = 0; step < nsteps; ++step)
        {
            const double *src = u;
            for (int st = 0; st < 5; ++st)
            {
                double *dst = (st == 4) ? u : ((st % 2 == 0) ? B : Cb);
                a.x = src;
                a.out = dst;
                a.rk_a = rk4a[st];
                a.rk_b = rk4b[st];
                a.fs = F ? -std::sin(omega * (t + rk4c[st] * dt)) / omega : 0.0;
                a.acc = (st == 4) ? acc : nullptr;
                a.acc_c = (st == 4 && acc) ? c_filter[step] : 0.0;
                WDG_TRY(qfused_launch(h, a));
                src = dst;
            }
            t += dt;
        }
        return WDG_OK;
    }

    // ---------------------------------------------------------------- device-side operators
    int div_dev(wdg_waveq *h, const double *u, double *du)
    {
        wdg_wave *w = h->w;
        const int n = h->n, q = h->nqd;
        const size_t smem = sizeof(double) * (3 * n * n + 3 * n * q + 3 * q * q + 6 * q * q + 6 * q * n);
        qdiv_kernel<<<(unsigned)std::min(w->nel, 148 * 16), 64, smem, w->stream>>>(n, q, w->nel, w->d_corners, h->d_xd,
                                                                                   h->d_wd, h->d_Pd, h->d_Dd, u, du);
        WDG_CUDA(cudaGetLastError());
        return WDG_OK;
    }
    int flux_dev(wdg_waveq *h, int type, const double *ub, double *fb)
    {
        wdg_wave *w = h->w;
        const int ne = (type == 0) ? w->nI : w->nB;
        if (ne == 0)
            return WDG_OK;
        qflux_kernel<<<(unsigned)((ne + 127) / 128), 128, 0, w->stream>>>(h->n, h->nqf, ne, type == 0 ? h->d_nI : h->d_nB,
                                                                          h->d_wf, h->d_Pf, ub, fb);
        WDG_CUDA(cudaGetLastError());
        return WDG_OK;
    }
    int mass_dev(wdg_waveq *h, int nv, double *x, bool inverse)
    {
        wdg_wave *w = h->w;
        const int c = h->n * h->n;
        const int wpb = (int)std::max<size_t>(1, std::min<size_t>(8, (48 * 1024) / (sizeof(double) * nv * c)));
        const size_t smem = sizeof(double) * wpb * nv * c; // at most 48 KB (nv <= 16, c <= 81: 10.4 KB a warp)
        qdense_kernel<<<(unsigned)std::min((w->nel + wpb - 1) / wpb, 148 * 32), 32 * wpb, smem, w->stream>>>(
            c, w->nel, nv, inverse ? h->d_Minv : h->d_M, x);
        WDG_CUDA(cudaGetLastError());
        return WDG_OK;
    }
    // du += Div u + Prol_I^T Flux_I Prol_I u
    int wave_dev(wdg_waveq *h, const double *u, double *du)
    {
        wdg_wave *w = h->w;
        WDG_TRY(div_dev(h, u, du));
        if (w->nI)
        {
            WDG_CUDA(launch_prolong(w->geo, 0, u, h->d_uf, w->stream));
            WDG_TRY(flux_dev(h, 0, h->d_uf, h->d_uf));
            WDG_CUDA(launch_prolong_t(w->geo, 0, h->d_uf, du, w->stream));
        }
        return WDG_OK;
    }
    // du += Prol_B^T Flux_B (exterior states) Prol_B u
    int bc_dev(wdg_waveq *h, const double *u, double *du)
    {
        wdg_wave *w = h->w;
        if (!w->nB)
            return WDG_OK;
        WDG_CUDA(launch_prolong(w->geo, 1, u, h->d_uB, w->stream));
        WDG_CUDA(launch_apply_bc(w->geo, h->d_uB, w->stream));
        WDG_TRY(flux_dev(h, 1, h->d_uB, h->d_uB));
        WDG_CUDA(launch_prolong_t(w->geo, 1, h->d_uB, du, w->stream));
        return WDG_OK;
    }
    // dudt = M^{-1} (A u + B u + s F), one fused launch
    int rhs_dev(wdg_waveq *h, const double *u, double *dudt, const double *F, double s)
    {
        QFusedArgs a{};
        a.x = u;
        a.out = dudt;
        a.F = F;
        a.fs = s;
        return qfused_launch(h, a);
    }

    typedef int (*Unary)(wdg_waveq *, const double *, double *);
    int accumulate_entry(wdg_waveq *h, const double *u, double *du, Unary f)
    {
        if (!h)
            return fail(WDG_ERR_ARG, "null exact-quadrature discretisation");
        if (u == du)
            return fail(WDG_ERR_ARG, "input and output arrays must differ");
        DeviceScope g(h->w->device);
        HostArg a[2];
        WDG_TRY(bind_arg(h->w, 0, u, h->w->ndof, true, false, a[0]));
        WDG_TRY(bind_arg(h->w, 1, du, h->w->ndof, true, true, a[1]));
        WDG_TRY(f(h, a[0].dev, a[1].dev));
        return finish_args(h->w, a, 2);
    }
} // namespace

namespace wdg
{
    // RK buffers and the resident state exist before a period is captured into a graph
    int waveq_prepare(wdg_waveq *h)
    {
        DeviceScope g(h->w->device);
        return ensure_states(h->w);
    }

    // One WaveHoltz period on the exact-quadrature operators, the sequence rk4_run runs on the
    // collocation kernels: nt RK4 steps of u' = M^{-1}(A u + B u + F s(t)), s(t) =
    // -sin(omega t) / omega at the stage times (F may be NULL), then acc += c_filter[step] u
    // after each step (source/WaveHoltz.cpp:55-121).  On the handle's current stream.
    int waveq_period(wdg_waveq *h, double *u, double dt, int nt, const double *F, double omega, double *acc,
                     const double *c_filter)
    {
        return qfused_rk4(h, u, dt, 0.0, nt, F, omega, acc, c_filter);
    }

    // P = M^{-1}(A + B) W on the exact operators (WaveHoltz::postprocess's RHS)
    int waveq_rhs_device(wdg_waveq *h, const double *u, double *dudt) { return rhs_dev(h, u, dudt, nullptr, 0.0); }
} // namespace wdg

extern "C"
{
    int wdg_waveq_create(const wdg_mesh *mesh, int n_colloc, const int *bc, int device, wdg_waveq **out)
    {
        if (!mesh || !out)
            return fail(WDG_ERR_ARG, "wdg_waveq_create: null argument");
        *out = nullptr;
        if (n_colloc < 2 || n_colloc > 9)
            return fail(WDG_ERR_UNSUPPORTED, "wdg_waveq_create: n_colloc must be 2..9");
        wdg_wave *w = nullptr;
        WDG_TRY(wdg_wave_create(mesh, n_colloc, bc, WDG_FP64, device, &w));
        wdg_waveq *h = new wdg_waveq;
        h->w = w;
        h->n = n_colloc;
        h->nqd = qdiv(n_colloc);
        h->nqf = qface(n_colloc);
        h->nqm = qface(n_colloc);
        DeviceScope g(w->device);
        {
            // the fused kernel's shared memory (70.4 KiB at n = 9), opted in once per device and
            // before any period is captured into a graph
            static std::mutex mu;
            static uint64_t set = 0;
            std::lock_guard<std::mutex> lock(mu);
            if (!(set & (1ull << (w->device & 63))))
            {
                const cudaError_t e = cudaFuncSetAttribute(qfused_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                           100 * 1024);
                if (e != cudaSuccess)
                {
                    wdg_wave_destroy(w);
                    delete h;
                    return cuda_fail(e, "cudaFuncSetAttribute(qfused_kernel)");
                }
                set |= 1ull << (w->device & 63);
            }
        }
        const int n = n_colloc, c = n * n;
        std::vector<double> x(n), wg(n);
        gauss_lobatto(n, x.data(), wg.data());
        // Div rule and its interpolation / derivative matrices
        std::vector<double> xd(h->nqd), wd(h->nqd), Pd((size_t)h->nqd * n), Dd((size_t)h->nqd * n);
        gauss_legendre(h->nqd, xd.data(), wd.data());
        interp_matrix(n, x.data(), h->nqd, xd.data(), Pd.data());
        lagrange_deriv_at(n, x.data(), h->nqd, xd.data(), Dd.data());
        // face rule
        std::vector<double> xf(h->nqf), wf(h->nqf), Pf((size_t)h->nqf * n);
        gauss_legendre(h->nqf, xf.data(), wf.data());
        interp_matrix(n, x.data(), h->nqf, xf.data(), Pf.data());
        // per edge: outward normal of elements[0] and |E| / 2 (StraightEdge, wavedg/Edge.hpp:107-122)
        auto normals = [&](const std::vector<EdgeRec> &list)
        {
            std::vector<double> nr(3 * list.size());
            for (size_t e = 0; e < list.size(); ++e)
            {
                const double *cr = &mesh->corners[8 * (size_t)list[e].el0];
                const int s = list[e].s0;
                const double dx = cr[2 * kSideTo[s]] - cr[2 * kSideFrom[s]];
                const double dy = cr[2 * kSideTo[s] + 1] - cr[2 * kSideFrom[s] + 1];
                const double len = std::sqrt(dx * dx + dy * dy), sgn = (s >= 2) ? -1.0 : 1.0;
                nr[3 * e] = sgn * dy / len;
                nr[3 * e + 1] = -sgn * dx / len;
                nr[3 * e + 2] = 0.5 * len;
            }
            return nr;
        };
        const std::vector<double> nI = normals(mesh->interior), nB = normals(mesh->boundary);
        std::vector<double> Mf, Mi;
        int st = exact_mass(*mesh, n, x.data(), h->nqm, Mf, Mi);
        auto chk = [&](int r)
        {
            if (st == WDG_OK)
                st = r;
        };
        chk(device_alloc(&h->d_xd, xd.size()));
        chk(device_alloc(&h->d_wd, wd.size()));
        chk(device_alloc(&h->d_Pd, Pd.size()));
        chk(device_alloc(&h->d_Dd, Dd.size()));
        chk(device_alloc(&h->d_wf, wf.size()));
        chk(device_alloc(&h->d_Pf, Pf.size()));
        chk(device_alloc(&h->d_nI, nI.size()));
        chk(device_alloc(&h->d_nB, nB.size()));
        chk(device_alloc(&h->d_M, Mf.size()));
        chk(device_alloc(&h->d_Minv, Mi.size()));
        chk(device_alloc(&h->d_uf, face_count(h, 0)));
        chk(device_alloc(&h->d_uB, face_count(h, 1)));
        if (st == WDG_OK)
        {
            chk(device_put(h->d_xd, xd));
            chk(device_put(h->d_wd, wd));
            chk(device_put(h->d_Pd, Pd));
            chk(device_put(h->d_Dd, Dd));
            chk(device_put(h->d_wf, wf));
            chk(device_put(h->d_Pf, Pf));
            chk(device_put(h->d_nI, nI));
            chk(device_put(h->d_nB, nB));
            chk(device_put(h->d_M, Mf));
            chk(device_put(h->d_Minv, Mi));
        }
        if (st == WDG_OK)
        {
            const int smax = (int)(sizeof(double) * (3 * c + 3 * n * h->nqd + 9 * h->nqd * h->nqd + 6 * h->nqd * n));
            if (smax > 48 * 1024)
            {
                const cudaError_t e = cudaFuncSetAttribute(qdiv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smax);
                if (e != cudaSuccess)
                    st = cuda_fail(e, "wdg_waveq_create: shared memory attribute");
            }
        }
        if (st != WDG_OK)
        {
            wdg_waveq_destroy(h);
            return st;
        }
        *out = h;
        return WDG_OK;
    }

    void wdg_waveq_destroy(wdg_waveq *h)
    {
        if (!h)
            return;
        {
            DeviceScope g(h->w ? h->w->device : 0);
            for (double *p : {h->d_xd, h->d_wd, h->d_Pd, h->d_Dd, h->d_wf, h->d_Pf, h->d_nI, h->d_nB, h->d_M, h->d_Minv, h->d_uf,
                              h->d_uB})
                if (p)
                    cudaFree(p);
        }
        if (h->w)
            wdg_wave_destroy(h->w);
        delete h;
    }

    int wdg_waveq_rules(const wdg_waveq *h, int *n_div, int *n_face, int *n_mass)
    {
        if (!h)
            return fail(WDG_ERR_ARG, "null exact-quadrature discretisation");
        if (n_div)
            *n_div = h->nqd;
        if (n_face)
            *n_face = h->nqf;
        if (n_mass)
            *n_mass = h->nqm;
        return WDG_OK;
    }

    int wdg_waveq_wave(const wdg_waveq *h, wdg_wave **wave)
    {
        if (!h || !wave)
            return fail(WDG_ERR_ARG, "wdg_waveq_wave: null argument");
        *wave = h->w;
        return WDG_OK;
    }

    int wdg_waveq_div_action(wdg_waveq *h, const double *u, double *du) { return accumulate_entry(h, u, du, div_dev); }
    int wdg_waveq_wave_action(wdg_waveq *h, const double *u, double *du) { return accumulate_entry(h, u, du, wave_dev); }
    int wdg_waveq_wavebc_action(wdg_waveq *h, const double *u, double *du) { return accumulate_entry(h, u, du, bc_dev); }

    int wdg_waveq_edge_flux(wdg_waveq *h, int type, const double *ub, double *fb)
    {
        if (!h || (type != 0 && type != 1) || !ub || !fb)
            return fail(WDG_ERR_ARG, "wdg_waveq_edge_flux: bad arguments");
        DeviceScope g(h->w->device);
        const size_t cnt = face_count(h, type);
        HostArg a[2];
        if (ub == fb)
        {
            WDG_TRY(bind_arg(h->w, 0, ub, cnt, true, true, a[0]));
            WDG_TRY(flux_dev(h, type, a[0].dev, a[0].dev));
            return finish_args(h->w, a, 1);
        }
        WDG_TRY(bind_arg(h->w, 0, ub, cnt, true, false, a[0]));
        WDG_TRY(bind_arg(h->w, 1, fb, cnt, false, true, a[1]));
        WDG_TRY(flux_dev(h, type, a[0].dev, a[1].dev));
        return finish_args(h->w, a, 2);
    }

    int wdg_waveq_mass_inv(wdg_waveq *h, int n_var, double *x)
    {
        if (!h || n_var < 1 || n_var > 16)
            return fail(WDG_ERR_ARG, "wdg_waveq_mass_inv: bad arguments");
        DeviceScope g(h->w->device);
        HostArg a;
        WDG_TRY(bind_arg(h->w, 0, x, (size_t)n_var * h->n * h->n * h->w->nel, true, true, a));
        WDG_TRY(mass_dev(h, n_var, a.dev, true));
        return finish_args(h->w, &a, 1);
    }

    int wdg_waveq_mass_action(wdg_waveq *h, int n_var, const double *x, double *y)
    {
        if (!h || n_var < 1 || n_var > 16 || !x || !y)
            return fail(WDG_ERR_ARG, "wdg_waveq_mass_action: bad arguments");
        DeviceScope g(h->w->device);
        const size_t cnt = (size_t)n_var * h->n * h->n * h->w->nel;
        HostArg a[2];
        WDG_TRY(bind_arg(h->w, 0, x, cnt, true, false, a[0]));
        WDG_TRY(bind_arg(h->w, 1, y, cnt, false, true, a[1]));
        if (a[1].dev != a[0].dev)
            WDG_CUDA(cudaMemcpyAsync(a[1].dev, a[0].dev, sizeof(double) * cnt, cudaMemcpyDeviceToDevice, h->w->stream));
        WDG_TRY(mass_dev(h, n_var, a[1].dev, false));
        return finish_args(h->w, a, 2);
    }

    int wdg_waveq_rhs(wdg_waveq *h, const double *u, double *dudt, const double *F, double s)
    {
        if (!h || !u || !dudt)
            return fail(WDG_ERR_ARG, "wdg_waveq_rhs: bad arguments");
        if (u == dudt)
            return fail(WDG_ERR_ARG, "input and output arrays must differ");
        DeviceScope g(h->w->device);
        HostArg a[3];
        int na = 2;
        WDG_TRY(bind_arg(h->w, 0, u, h->w->ndof, true, false, a[0]));
        WDG_TRY(bind_arg(h->w, 1, dudt, h->w->ndof, false, true, a[1]));
        if (F)
        {
            WDG_TRY(bind_arg(h->w, 2, F, h->w->ndof, true, false, a[2]));
            na = 3;
        }
        WDG_TRY(rhs_dev(h, a[0].dev, a[1].dev, F ? a[2].dev : nullptr, s));
        return finish_args(h->w, a, na);
    }

    int wdg_waveq_rk4_steps(wdg_waveq *h, double *u, double dt, double *t, int nsteps)
    {
        if (!h || !u || !t || nsteps < 0)
            return fail(WDG_ERR_ARG, "wdg_waveq_rk4_steps: bad arguments");
        DeviceScope g(h->w->device);
        wdg_wave *w = h->w;
        HostArg a;
        WDG_TRY(bind_arg(w, 0, u, w->ndof, true, true, a));
        WDG_TRY(qfused_rk4(h, a.dev, dt, *t, nsteps, nullptr, 0.0, nullptr, nullptr));
        for (int s = 0; s < nsteps; ++s)
            *t += dt; // ode::RungeKutta4::step advances t once per step
        return finish_args(w, &a, 1);
    }
}
