// wdg_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the oracle).
//
// A plain, serial C++ restatement of the reference's algorithm for the 2D wave
// hot path, written to be read line by line against the reference sources
// cited below.  It is the checker for the CUDA path: the tests, smoke() and
// bench.py's CPU-baseline leg are the only callers.  It shares no code with
// the product library (wavedg_b200/csrc), and it is itself pinned against the
// reference library (oracle/_ref, built from the reference's sources) by the
// golden vectors in tests/golden/.
//
// Layouts are the reference's (column-major, first index fastest):
//   state  u(d, i, j, el)       d in {p, u_x, u_y}       (docs/docs.md:55-61)
//   traces uf(i, d, side, edge)                          (FaceProlongator.hpp:43)
//
// Boundary codes per boundary edge: 0 absorbing (outflow, with the exterior
// state computed in dependency order -- the reference's absorb_2d assigns p_ext
// before u_ext, wavedg/WaveEquation.hpp:77-84), 1 reflecting (reflect_2d,
// WaveEquation.hpp:64-69), 2 Dirichlet p = 0 (mirror state p_ext = -p, u_ext = u;
// not implemented for 2D by the reference, WaveEquation.cpp:80-81).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

namespace
{
    using vec = std::vector<double>;

    // ---------------------------------------------------------------- mesh
    struct Edge
    {
        int el[2] = {-1, -1};
        int side[2] = {-1, -1};
        int delta = 1;
        bool interior = false;
        double x0[2], dx[2]; // StraightEdge (Edge.hpp:107-122)
        double n[2], meas;
    };

    struct Mesh
    {
        int nel = 0;
        vec corners; // (2, 4, nel)
        std::vector<Edge> edges;
        std::vector<int> interior, boundary; // indices into edges, in id order
    };

    // Mesh2D::from_vertices (source/Mesh2D.cpp:5-92).  Side s of an element runs
    // from corner emap1[s] to corner emap2[s]; an edge is created the first time
    // a vertex pair is met (so edge ids follow element order, then side order),
    // the second element to meet it becomes elements[1] and
    // delta = +1 iff it traverses the pair in the same direction.  Keys are
    // 64-bit here (the reference's int key can overflow past ~46k vertices).
    Mesh *make_mesh(int nv, const double *xy, int nel, const int *q)
    {
        static const int emap1[] = {0, 1, 3, 0};
        static const int emap2[] = {1, 2, 2, 3};
        Mesh *m = new Mesh;
        m->nel = nel;
        m->corners.resize(8 * (size_t)nel);
        for (int el = 0; el < nel; ++el)
            for (int c = 0; c < 4; ++c)
            {
                m->corners[8 * (size_t)el + 2 * c] = xy[2 * q[4 * el + c]];
                m->corners[8 * (size_t)el + 2 * c + 1] = xy[2 * q[4 * el + c] + 1];
            }
        std::unordered_map<int64_t, int> seen;
        seen.reserve(4 * (size_t)nel);
        for (int el = 0; el < nel; ++el)
            for (int s = 0; s < 4; ++s)
            {
                const int C0 = q[4 * el + emap1[s]], C1 = q[4 * el + emap2[s]];
                const int64_t key = (int64_t)std::min(C0, C1) + (int64_t)nv * std::max(C0, C1);
                auto it = seen.find(key);
                if (it == seen.end())
                {
                    Edge E;
                    E.el[0] = el;
                    E.side[0] = s;
                    E.x0[0] = xy[2 * C0];
                    E.x0[1] = xy[2 * C0 + 1];
                    E.dx[0] = xy[2 * C1] - xy[2 * C0];
                    E.dx[1] = xy[2 * C1 + 1] - xy[2 * C0 + 1];
                    const double len = std::hypot(E.dx[0], E.dx[1]);
                    const double sgn = (s == 2 || s == 3) ? -1 : 1;
                    E.n[0] = sgn * E.dx[1] / len;
                    E.n[1] = -sgn * E.dx[0] / len;
                    E.meas = len / 2;
                    seen.emplace(key, (int)m->edges.size());
                    m->edges.push_back(E);
                }
                else
                {
                    Edge &E = m->edges[it->second];
                    const int first = q[4 * E.el[0] + emap1[E.side[0]]];
                    E.el[1] = el;
                    E.side[1] = s;
                    E.interior = true;
                    E.delta = (C0 == first) ? 1 : -1;
                }
            }
        for (int e = 0; e < (int)m->edges.size(); ++e)
            (m->edges[e].interior ? m->interior : m->boundary).push_back(e);
        return m;
    }

    // --------------------------------------------------------- quadrature
    // Legendre P_k(x) and P_k'(x) by the three-term recurrence
    void legendre(int k, double x, double &P, double &dP)
    {
        double p0 = 1.0, p1 = x;
        if (k == 0)
        {
            P = 1.0;
            dP = 0.0;
            return;
        }
        for (int j = 2; j <= k; ++j)
        {
            const double p2 = ((2.0 * j - 1.0) * x * p1 - (j - 1.0) * p0) / j;
            p0 = p1;
            p1 = p2;
        }
        P = p1;
        dP = k * (x * p1 - p0) / (x * x - 1.0);
    }

    // Gauss-Lobatto rule (QuadratureRule.cpp:32-97): interior nodes are the roots
    // of P'_{n-1}; found by Newton from Chebyshev-Lobatto guesses, mirrored so the
    // rule is exactly symmetric.  w = 2 / (n(n-1) P_{n-1}(x)^2)  (:93-94).
    void gll(int n, double *x, double *w)
    {
        x[0] = -1.0;
        x[n - 1] = 1.0;
        for (int i = 1; i < n / 2 + (n & 1); ++i)
        {
            double t = -std::cos(M_PI * i / (n - 1));
            for (int it = 0; it < 100; ++it)
            {
                // f = P'_{n-1}, f' = P''_{n-1} = (2t P' - (n-1)n P)/(1-t^2)
                double P, dP;
                legendre(n - 1, t, P, dP);
                const double d2P = (2.0 * t * dP - (n - 1.0) * n * P) / (1.0 - t * t);
                const double step = dP / d2P;
                t -= step;
                if (std::abs(step) < 1e-17)
                    break;
            }
            x[i] = t;
            x[n - 1 - i] = -t;
        }
        if (n & 1)
            x[n / 2] = 0.0;
        for (int i = 0; i < n; ++i)
        {
            double P, dP;
            legendre(n - 1, x[i], P, dP);
            if (x[i] == 1.0 || x[i] == -1.0)
                P = (x[i] > 0 || ((n - 1) % 2 == 0)) ? 1.0 : -1.0;
            w[i] = 2.0 / (n * (n - 1) * P * P);
        }
    }

    // Gauss-Legendre rule (QuadratureRule.cpp:99-160): roots of P_n by Newton,
    // w = 2 / ((1 - x^2) P_n'(x)^2)
    void gl(int n, double *x, double *w)
    {
        for (int i = 0; i < (n + 1) / 2; ++i)
        {
            double t = -std::cos(M_PI * (i + 0.75) / (n + 0.5));
            for (int it = 0; it < 100; ++it)
            {
                double P, dP;
                legendre(n, t, P, dP);
                const double step = P / dP;
                t -= step;
                if (std::abs(step) < 1e-17)
                    break;
            }
            x[i] = t;
            x[n - 1 - i] = -t;
        }
        if (n & 1)
            x[n / 2] = 0.0;
        for (int i = 0; i < n; ++i)
        {
            double P, dP;
            legendre(n, x[i], P, dP);
            w[i] = 2.0 / ((1.0 - x[i] * x[i]) * dP * dP);
        }
    }

    // barycentric weights normalised by (max - min)  (lagrange_interpolation.cpp:52-72)
    void bary(const double *x, int n, double *lw)
    {
        for (int i = 0; i < n; ++i)
        {
            double p = 1.0;
            for (int j = 0; j < n; ++j)
                if (j != i)
                    p *= x[i] - x[j];
            lw[i] = 1.0 / p;
        }
        const auto mm = std::minmax_element(lw, lw + n);
        const double diff = *mm.second - *mm.first;
        for (int i = 0; i < n; ++i)
            lw[i] /= diff;
    }

    // D(l, j) = phi_j'(x_l) at the nodes (lagrange_basis_deriv at xeval = xgrid,
    // the "atnode" branch of lagrange_derivative, lagrange_interpolation.cpp:96-139)
    void deriv_matrix(int n, const double *x, double *D)
    {
        double lw[16];
        bary(x, n, lw);
        for (int j = 0; j < n; ++j)
            for (int l = 0; l < n; ++l)
            {
                double A = 0.0;
                const double p = (l == j) ? 1.0 : 0.0;
                for (int k = 0; k < n; ++k)
                    if (k != l)
                        A += lw[k] * (p - (k == j ? 1.0 : 0.0)) / (x[l] - x[k]);
                D[l + n * j] = A / (-lw[l]);
            }
    }

    // B(i, j) = phi_j(xq_i)  (lagrange_basis, lagrange_interpolation.cpp:14-31, 74-94)
    void interp_matrix(int n, const double *x, int nq, const double *xq, double *B)
    {
        double lw[16];
        bary(x, n, lw);
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < nq; ++i)
            {
                double A = 0.0, Bs = 0.0, val = NAN;
                for (int k = 0; k < n; ++k)
                {
                    const double xd = xq[i] - x[k];
                    if (xq[i] == x[k] || std::abs(xd) <= 2.220446049250313e-16)
                    {
                        val = (k == j) ? 1.0 : 0.0;
                        break;
                    }
                    const double C = lw[k] / xd;
                    A += C * (k == j ? 1.0 : 0.0);
                    Bs += C;
                }
                B[i + nq * j] = std::isnan(val) ? A / Bs : val;
            }
    }

    // ------------------------------------------------------ element metrics
    // QuadElement::jacobian / physical_coordinates (source/Element.cpp:5-27)
    void jacobian(const double *c, double xi, double eta, double J[4])
    {
        J[0] = 0.25 * ((1.0 - eta) * (c[2] - c[0]) + (1.0 + eta) * (c[4] - c[6]));
        J[1] = 0.25 * ((1.0 - eta) * (c[3] - c[1]) + (1.0 + eta) * (c[5] - c[7]));
        J[2] = 0.25 * ((1.0 - xi) * (c[6] - c[0]) + (1.0 + xi) * (c[4] - c[2]));
        J[3] = 0.25 * ((1.0 - xi) * (c[7] - c[1]) + (1.0 + xi) * (c[5] - c[3]));
    }
    void physical(const double *c, double xi, double eta, double X[2])
    {
        const double b[] = {0.25 * (1.0 - xi) * (1.0 - eta), 0.25 * (1.0 + xi) * (1.0 - eta),
                            0.25 * (1.0 + xi) * (1.0 + eta), 0.25 * (1.0 - xi) * (1.0 + eta)};
        X[0] = X[1] = 0.0;
        for (int i = 0; i < 4; ++i)
        {
            X[0] += c[2 * i] * b[i];
            X[1] += c[2 * i + 1] * b[i];
        }
    }

    // ------------------------------------------------------------ operator
    // cyclic Jacobi eigen-decomposition of a symmetric 3x3 matrix A (column-major):
    // A = R diag(e) R^T.  Stands in for the dgeevx_ call of real_eig (eig.cpp:29-73);
    // for the symmetric C = n_x A_0 + n_y A_1 of the wave system R is orthogonal,
    // so the reference's R^{-T} (dgels_) is R.
    void sym_eig3(const double *A_, double *R, double *e)
    {
        double A[9];
        std::memcpy(A, A_, sizeof A);
        for (int i = 0; i < 9; ++i)
            R[i] = (i % 4 == 0) ? 1.0 : 0.0;
        for (int sweep = 0; sweep < 50; ++sweep)
        {
            double off = 0.0;
            for (int p = 0; p < 3; ++p)
                for (int q = p + 1; q < 3; ++q)
                    off += A[p + 3 * q] * A[p + 3 * q];
            if (off < 1e-300)
                break;
            for (int p = 0; p < 3; ++p)
                for (int q = p + 1; q < 3; ++q)
                {
                    const double apq = A[p + 3 * q];
                    if (apq == 0.0)
                        continue;
                    const double theta = (A[q + 3 * q] - A[p + 3 * p]) / (2.0 * apq);
                    const double t = (theta >= 0 ? 1.0 : -1.0) / (std::abs(theta) + std::sqrt(theta * theta + 1.0));
                    const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                    for (int k = 0; k < 3; ++k) // A <- A G
                    {
                        const double akp = A[k + 3 * p], akq = A[k + 3 * q];
                        A[k + 3 * p] = c * akp - s * akq;
                        A[k + 3 * q] = s * akp + c * akq;
                    }
                    for (int k = 0; k < 3; ++k) // A <- G^T A
                    {
                        const double apk = A[p + 3 * k], aqk = A[q + 3 * k];
                        A[p + 3 * k] = c * apk - s * aqk;
                        A[q + 3 * k] = s * apk + c * aqk;
                    }
                    for (int k = 0; k < 3; ++k) // R <- R G
                    {
                        const double rkp = R[k + 3 * p], rkq = R[k + 3 * q];
                        R[k + 3 * p] = c * rkp - s * rkq;
                        R[k + 3 * q] = s * rkp + c * rkq;
                    }
                }
        }
        for (int i = 0; i < 3; ++i)
            e[i] = A[i + 3 * i];
    }

    struct Op
    {
        const Mesh &m;
        int n, nel, ndof;
        vec x, w, D;        // GLL nodes, weights, D(l, j)
        vec op;             // Div<true> table (2, 3, 3, n, n, nel)
        vec mass;           // (n, n, nel)
        std::vector<int> v2eI, v2eB; // (n, 2, nI), (n, 2, nB)
        vec FI, FB;         // EdgeFlux tables (n, 3, 3, 2, nedges)
        std::vector<int> bc;

        Op(const Mesh &m_, int n_, const int *codes) : m(m_), n(n_), nel(m_.nel), ndof(3 * n_ * n_ * m_.nel)
        {
            x.resize(n);
            w.resize(n);
            D.resize(n * n);
            gll(n, x.data(), w.data());
            deriv_matrix(n, x.data(), D.data());
            bc.assign(codes, codes + m.boundary.size());

            // wave system A table (source/WaveEquation.cpp:10-18): a(c, d, k)
            static const double a[] = {0, 1, 0, 1, 0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0};
            const int c2d = n * n;
            // Div<true> constructor (source/Div.cpp:5-53)
            op.resize((size_t)2 * 9 * c2d * nel);
            mass.resize((size_t)c2d * nel);
            for (int el = 0; el < nel; ++el)
                for (int i = 0; i < c2d; ++i)
                {
                    double J[4];
                    jacobian(&m.corners[8 * (size_t)el], x[i % n], x[i / n], J);
                    const double W = w[i / n] * w[i % n];
                    const double Y_eta = J[3] * W, X_eta = J[2] * W, Y_xi = J[1] * W, X_xi = J[0] * W;
                    for (int d = 0; d < 3; ++d)
                        for (int c = 0; c < 3; ++c)
                        {
                            const double a0 = a[c + 3 * d], a1 = a[c + 3 * d + 9];
                            op[0 + 2 * (d + 3 * (c + 3 * (i + (size_t)c2d * el)))] = Y_eta * a0 - X_eta * a1;
                            op[1 + 2 * (d + 3 * (c + 3 * (i + (size_t)c2d * el)))] = -Y_xi * a0 + X_xi * a1;
                        }
                    // MassMatrix<true> (source/MassMatrix.cpp:6-28): w_i w_j detJ
                    mass[i + (size_t)c2d * el] = w[i % n] * w[i / n] * (J[0] * J[3] - J[1] * J[2]);
                }
            build_v2e(m.interior, true, v2eI);
            build_v2e(m.boundary, false, v2eB);
            build_flux(m.interior, FI, a);
            build_flux(m.boundary, FB, a);
        }

        // LobattoFaceProlongator (source/FaceProlongator.cpp:497-539)
        void build_v2e(const std::vector<int> &list, bool interior, std::vector<int> &v2e)
        {
            const int N = (int)list.size();
            v2e.assign((size_t)2 * n * N, -1);
            auto map = [this](int i, int f, int el)
            {
                const int mm = (f == 0 || f == 2) ? i : (f == 1) ? (n - 1) : 0;
                const int nn = (f == 1 || f == 3) ? i : (f == 2) ? (n - 1) : 0;
                return mm + n * (nn + n * el);
            };
            for (int e = 0; e < N; ++e)
            {
                const Edge &E = m.edges[list[e]];
                for (int i = 0; i < n; ++i)
                    v2e[i + n * (0 + 2 * (size_t)e)] = map(i, E.side[0], E.el[0]);
                if (interior)
                    for (int i = 0; i < n; ++i)
                    {
                        const int j = (E.delta > 0) ? i : (n - 1 - i);
                        v2e[i + n * (1 + 2 * (size_t)e)] = map(j, E.side[1], E.el[1]);
                    }
            }
        }

        // setup_flux_2d_cc_c + _ComputeFlux::flux (source/EdgeFlux.cpp:7-139) with the
        // default a = -1, b = -1/2 (upwind): Fs = R^{-T} diag(a/2 e + sgn b|e|) R^T,
        // stored times w_i * ds
        void build_flux(const std::vector<int> &list, vec &F, const double *a)
        {
            const int N = (int)list.size();
            const double fa = -1.0, fb = -0.5;
            F.resize((size_t)n * 9 * 2 * N);
            for (int e = 0; e < N; ++e)
            {
                const Edge &E = m.edges[list[e]];
                double nA[9], R[9], ev[3];
                for (int d = 0; d < 9; ++d)
                    nA[d] = E.n[0] * a[d] + E.n[1] * a[d + 9];
                sym_eig3(nA, R, ev);
                for (int s = 0; s < 2; ++s)
                {
                    const double sgn = (s == 0) ? 1.0 : -1.0;
                    double Fs[9];
                    for (int i = 0; i < 3; ++i)
                        for (int j = 0; j < 3; ++j)
                        {
                            double acc = 0.0;
                            for (int k = 0; k < 3; ++k)
                                acc += R[i + 3 * k] * (0.5 * fa * ev[k] + sgn * fb * std::abs(ev[k])) * R[j + 3 * k];
                            Fs[i + 3 * j] = acc;
                        }
                    for (int i = 0; i < n; ++i)
                    {
                        const double ww = w[i] * E.meas;
                        for (int d = 0; d < 3; ++d)
                            for (int c = 0; c < 3; ++c)
                                F[i + n * (c + 3 * (d + 3 * (s + 2 * (size_t)e)))] = ww * Fs[c + 3 * d];
                    }
                }
            }
        }

        // div_2d_c (source/Div.cpp:131-179): du += D^T F + D^T G, accumulates
        void div(const double *u, double *du) const
        {
            std::vector<double> Fq((size_t)2 * n * 3 * n);
            auto FQ = [&](int k, int a, int d, int b) -> double & { return Fq[k + 2 * (a + n * (d + 3 * (size_t)b))]; };
            for (int el = 0; el < nel; ++el)
            {
                for (int j = 0; j < n; ++j)
                    for (int i = 0; i < n; ++i)
                        for (int d = 0; d < 3; ++d)
                        {
                            double Fd = 0.0, Gd = 0.0;
                            for (int c = 0; c < 3; ++c)
                            {
                                const size_t node = i + n * (j + (size_t)n * el);
                                const double uij = u[c + 3 * node];
                                Fd += op[0 + 2 * (c + 3 * (d + 3 * node))] * uij;
                                Gd += op[1 + 2 * (c + 3 * (d + 3 * node))] * uij;
                            }
                            FQ(0, i, d, j) = Fd;
                            FQ(1, j, d, i) = Gd;
                        }
                for (int j = 0; j < n; ++j)
                    for (int i = 0; i < n; ++i)
                        for (int d = 0; d < 3; ++d)
                        {
                            double s = 0.0;
                            for (int l = 0; l < n; ++l)
                                s += D[l + n * i] * FQ(0, l, d, j) + D[l + n * j] * FQ(1, l, d, i);
                            du[d + 3 * (i + n * (j + (size_t)n * el))] += s;
                        }
            }
        }

        // lobatto_action_2d (FaceProlongator.cpp:565-590): zero, then gather
        void prolong(bool interior, const double *u, double *uf) const
        {
            const auto &v2e = interior ? v2eI : v2eB;
            const int N = (int)(interior ? m.interior.size() : m.boundary.size());
            std::fill(uf, uf + (size_t)n * 3 * 2 * N, 0.0);
            for (int e = 0; e < N; ++e)
                for (int s = 0; s < (interior ? 2 : 1); ++s)
                    for (int i = 0; i < n; ++i)
                        for (int d = 0; d < 3; ++d)
                            uf[i + n * (d + 3 * (s + 2 * (size_t)e))] = u[d + 3 * (size_t)v2e[i + n * (s + 2 * (size_t)e)]];
        }

        // lobatto_transpose_2d (FaceProlongator.cpp:650-672): scatter-add
        void prolong_t(bool interior, const double *uf, double *u) const
        {
            const auto &v2e = interior ? v2eI : v2eB;
            const int N = (int)(interior ? m.interior.size() : m.boundary.size());
            for (int e = 0; e < N; ++e)
                for (int s = 0; s < (interior ? 2 : 1); ++s)
                    for (int i = 0; i < n; ++i)
                        for (int d = 0; d < 3; ++d)
                            u[d + 3 * (size_t)v2e[i + n * (s + 2 * (size_t)e)]] += uf[i + n * (d + 3 * (s + 2 * (size_t)e))];
        }

        // flux_action_2d_c (EdgeFlux.cpp:289-325): uf = sum_s Fs^T u_s; side 0 <- uf,
        // side 1 <- -uf  (safe in place)
        void flux(bool interior, const double *ub, double *fb) const
        {
            const auto &F = interior ? FI : FB;
            const int N = (int)(interior ? m.interior.size() : m.boundary.size());
            std::vector<double> uf((size_t)n * 3);
            for (int e = 0; e < N; ++e)
            {
                std::fill(uf.begin(), uf.end(), 0.0);
                for (int s = 0; s < 2; ++s)
                    for (int d = 0; d < 3; ++d)
                        for (int c = 0; c < 3; ++c)
                            for (int i = 0; i < n; ++i)
                                uf[i + n * d] += F[i + n * (c + 3 * (d + 3 * (s + 2 * (size_t)e)))] * ub[i + n * (c + 3 * (s + 2 * (size_t)e))];
                for (int d = 0; d < 3; ++d)
                    for (int i = 0; i < n; ++i)
                    {
                        fb[i + n * (d + 3 * (0 + 2 * (size_t)e))] = uf[i + n * d];
                        fb[i + n * (d + 3 * (1 + 2 * (size_t)e))] = -uf[i + n * d];
                    }
            }
        }

        // apply_bc_2d (WaveEquation.cpp:144-167) with the exterior states above
        void apply_bc(double *uB) const
        {
            const int N = (int)m.boundary.size();
            for (int e = 0; e < N; ++e)
            {
                const double *nn = m.edges[m.boundary[e]].n;
                for (int i = 0; i < n; ++i)
                {
                    double vi[3], ve[3];
                    for (int d = 0; d < 3; ++d)
                        vi[d] = uB[i + n * (d + 3 * (0 + 2 * (size_t)e))];
                    if (bc[e] == 1)
                    {
                        ve[0] = vi[0];
                        ve[1] = (nn[1] * nn[1] - nn[0] * nn[0]) * vi[1] - 2.0 * nn[0] * nn[1] * vi[2];
                        ve[2] = -2.0 * nn[0] * nn[1] * vi[1] + (nn[0] * nn[0] - nn[1] * nn[1]) * vi[2];
                    }
                    else if (bc[e] == 0)
                    {
                        const double out = vi[0] + nn[0] * vi[1] + nn[1] * vi[2];
                        const double tan = nn[1] * vi[1] - nn[0] * vi[2];
                        ve[1] = nn[1] * tan + 0.5 * nn[0] * out;
                        ve[2] = -nn[0] * tan + 0.5 * nn[1] * out;
                        ve[0] = nn[0] * ve[1] + nn[1] * ve[2];
                    }
                    else
                    {
                        ve[0] = -vi[0];
                        ve[1] = vi[1];
                        ve[2] = vi[2];
                    }
                    for (int d = 0; d < 3; ++d)
                        uB[i + n * (d + 3 * (1 + 2 * (size_t)e))] = ve[d];
                }
            }
        }

        // WaveEquation::action (WaveEquation.cpp:54-68): du += div + prol^T flux prol
        void wave_action(const double *u, double *du) const
        {
            div(u, du);
            std::vector<double> uf((size_t)n * 3 * 2 * m.interior.size());
            prolong(true, u, uf.data());
            flux(true, uf.data(), uf.data());
            prolong_t(true, uf.data(), du);
        }

        // WaveBC::action (WaveEquation.cpp:190-215)
        void bc_action(const double *u, double *du) const
        {
            std::vector<double> uB((size_t)n * 3 * 2 * m.boundary.size());
            prolong(false, u, uB.data());
            apply_bc(uB.data());
            flux(false, uB.data(), uB.data());
            prolong_t(false, uB.data(), du);
        }

        // MassMatrix<true>::inv / action (MassMatrix.cpp:55-82)
        void mass_inv(int nv, double *xv) const
        {
            const size_t np = (size_t)n * n * nel;
            for (size_t i = 0; i < np; ++i)
                for (int d = 0; d < nv; ++d)
                    xv[d + nv * i] /= mass[i];
        }
        void mass_action(int nv, const double *xv, double *y) const
        {
            const size_t np = (size_t)n * n * nel;
            for (size_t i = 0; i < np; ++i)
                for (int d = 0; d < nv; ++d)
                    y[d + nv * i] = mass[i] * xv[d + nv * i];
        }

        // the examples' time derivative: M^{-1}(A u + B u + s F)
        void rhs(const double *u, double *du, const double *F, double s) const
        {
            std::fill(du, du + ndof, 0.0);
            wave_action(u, du);
            bc_action(u, du);
            if (F)
                for (int i = 0; i < ndof; ++i)
                    du[i] += F[i] * s;
            mass_inv(3, du);
        }
    };

    // ode::RungeKutta4::step (wavedg/ode.hpp:66-93), Carpenter-Kennedy 2N-storage
    const double rk4a[5] = {0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
                            -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0};
    const double rk4b[5] = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
                            1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
                            2277821191437.0 / 14882151754819.0};
    const double rk4c[5] = {0.0, 1432997174477.0 / 9575080441755.0, 2526269341429.0 / 6820363962896.0,
                            2006345519317.0 / 3224310063776.0, 2802321613138.0 / 2924317926251.0};

    template <class F>
    void rk4_step(int nd, double dt, F f, double &t, double *u, vec &p, vec &du)
    {
        f(p.data(), t, u);
        for (int i = 0; i < nd; ++i)
        {
            du[i] = dt * p[i];
            u[i] += rk4b[0] * du[i];
        }
        for (int st = 1; st < 5; ++st)
        {
            f(p.data(), t + rk4c[st] * dt, u);
            for (int i = 0; i < nd; ++i)
            {
                du[i] = rk4a[st] * du[i] + dt * p[i];
                u[i] += rk4b[st] * du[i];
            }
        }
        t += dt;
    }

    // cyclic Jacobi eigen-decomposition of a symmetric m x m matrix (column-major), m <= 8:
    // A = R diag(e) R^T (the symmetric case of real_eig, eig.cpp:29-73)
    void sym_eig(int m, const double *A_, double *R, double *e)
    {
        double A[64];
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

    // Advection<true> with constant coefficients (wavedg/Advection.hpp:17-142: Div<true> and
    // EdgeFlux<true> with a = -1, b = -1/2 for any n_var) and AdvectionHomogeneousBC<true>
    // (:144-273: u = 0 outside), for symmetric coefficient matrices A_0, A_1 (n_var x n_var,
    // a(d, c, k) = a[d + nv (c + nv k)]); the Lobatto prolongation and mass of Op.
    struct OpA
    {
        const Op base;
        const Mesh &m;
        int n, nv, nel, ndof;
        vec a, FI, FB; // coefficients; flux tables (n, nv, nv, 2, edges), times w_i |E|/2

        OpA(const Mesh &m_, int n_, int nv_, const double *a_)
            : base(m_, n_, std::vector<int>(m_.boundary.size(), 0).data()), m(m_), n(n_), nv(nv_), nel(m_.nel),
              ndof(nv_ * n_ * n_ * m_.nel), a(a_, a_ + 2 * nv_ * nv_)
        {
            flux_table(m.interior, FI);
            flux_table(m.boundary, FB);
        }

        void flux_table(const std::vector<int> &list, vec &F) const
        {
            const int N = (int)list.size(), v2 = nv * nv;
            F.resize((size_t)n * v2 * 2 * N);
            for (int e = 0; e < N; ++e)
            {
                const Edge &E = m.edges[list[e]];
                double nA[64], R[64], ev[8];
                for (int d = 0; d < v2; ++d)
                    nA[d] = E.n[0] * a[d] + E.n[1] * a[d + v2];
                sym_eig(nv, nA, R, ev);
                for (int s = 0; s < 2; ++s)
                {
                    const double sgn = (s == 0) ? 1.0 : -1.0;
                    for (int c = 0; c < nv; ++c)
                        for (int d = 0; d < nv; ++d)
                        {
                            double acc = 0.0;
                            for (int k = 0; k < nv; ++k)
                                acc += R[c + nv * k] * (-0.5 * ev[k] + sgn * -0.5 * std::abs(ev[k])) * R[d + nv * k];
                            for (int i = 0; i < n; ++i)
                                F[i + n * (c + nv * (d + nv * (s + 2 * (size_t)e)))] = base.w[i] * E.meas * acc;
                        }
                }
            }
        }
        // div_2d_c with the op table of op_2d_cc (Div.cpp:5-53, 131-179): du += D^T F + D^T G
        void div(const double *u, double *du) const
        {
            const int nn = n * n, v2 = nv * nv;
            vec Fx((size_t)nv * nn), Gy((size_t)nv * nn);
            for (int el = 0; el < nel; ++el)
            {
                const double *ue = u + (size_t)nv * nn * el;
                for (int i = 0; i < nn; ++i)
                {
                    double J[4];
                    jacobian(&m.corners[8 * (size_t)el], base.x[i % n], base.x[i / n], J);
                    const double W = base.w[i / n] * base.w[i % n];
                    const double Ye = J[3] * W, Xe = J[2] * W, Yx = J[1] * W, Xx = J[0] * W;
                    for (int d = 0; d < nv; ++d)
                    {
                        double f = 0.0, g = 0.0;
                        for (int c = 0; c < nv; ++c)
                        {
                            const double a0 = a[d + nv * c], a1 = a[d + nv * c + v2];
                            f += (Ye * a0 - Xe * a1) * ue[c + nv * i];
                            g += (-Yx * a0 + Xx * a1) * ue[c + nv * i];
                        }
                        Fx[d + nv * i] = f;
                        Gy[d + nv * i] = g;
                    }
                }
                for (int j = 0; j < n; ++j)
                    for (int i = 0; i < n; ++i)
                        for (int d = 0; d < nv; ++d)
                        {
                            double sum = 0.0;
                            for (int l = 0; l < n; ++l)
                                sum += base.D[l + n * i] * Fx[d + nv * (l + n * j)] + base.D[l + n * j] * Gy[d + nv * (i + n * l)];
                            du[d + nv * (i + n * (j + (size_t)n * el))] += sum;
                        }
            }
        }
        void prolong(bool interior, const double *u, double *uf) const
        {
            const auto &v2e = interior ? base.v2eI : base.v2eB;
            const int N = (int)(interior ? m.interior.size() : m.boundary.size());
            std::fill(uf, uf + (size_t)n * nv * 2 * N, 0.0);
            for (int e = 0; e < N; ++e)
                for (int s = 0; s < (interior ? 2 : 1); ++s)
                    for (int i = 0; i < n; ++i)
                        for (int d = 0; d < nv; ++d)
                            uf[i + n * (d + nv * (s + 2 * (size_t)e))] = u[d + nv * (size_t)v2e[i + n * (s + 2 * (size_t)e)]];
        }
        void prolong_t(bool interior, const double *uf, double *u) const
        {
            const auto &v2e = interior ? base.v2eI : base.v2eB;
            const int N = (int)(interior ? m.interior.size() : m.boundary.size());
            for (int e = 0; e < N; ++e)
                for (int s = 0; s < (interior ? 2 : 1); ++s)
                    for (int i = 0; i < n; ++i)
                        for (int d = 0; d < nv; ++d)
                            u[d + nv * (size_t)v2e[i + n * (s + 2 * (size_t)e)]] += uf[i + n * (d + nv * (s + 2 * (size_t)e))];
        }
        // flux_action_2d_c (EdgeFlux.cpp:289-325) for nv variables
        void flux(bool interior, const double *ub, double *fb) const
        {
            const auto &F = interior ? FI : FB;
            const int N = (int)(interior ? m.interior.size() : m.boundary.size());
            vec uf((size_t)n * nv);
            for (int e = 0; e < N; ++e)
            {
                std::fill(uf.begin(), uf.end(), 0.0);
                for (int s = 0; s < 2; ++s)
                    for (int d = 0; d < nv; ++d)
                        for (int c = 0; c < nv; ++c)
                            for (int i = 0; i < n; ++i)
                                uf[i + n * d] += F[i + n * (c + nv * (d + nv * (s + 2 * (size_t)e)))] *
                                                 ub[i + n * (c + nv * (s + 2 * (size_t)e))];
                for (int d = 0; d < nv; ++d)
                    for (int i = 0; i < n; ++i)
                    {
                        fb[i + n * (d + nv * (0 + 2 * (size_t)e))] = uf[i + n * d];
                        fb[i + n * (d + nv * (1 + 2 * (size_t)e))] = -uf[i + n * d];
                    }
            }
        }
        void action(const double *u, double *du) const
        {
            div(u, du);
            vec uf((size_t)n * nv * 2 * m.interior.size());
            prolong(true, u, uf.data());
            flux(true, uf.data(), uf.data());
            prolong_t(true, uf.data(), du);
        }
        void bc_action(const double *u, double *du) const
        {
            vec uB((size_t)n * nv * 2 * m.boundary.size());
            prolong(false, u, uB.data()); // side 1 stays 0: u = 0 outside
            flux(false, uB.data(), uB.data());
            prolong_t(false, uB.data(), du);
        }
        void rhs(const double *u, double *du) const
        {
            std::fill(du, du + ndof, 0.0);
            action(u, du);
            bc_action(u, du);
            base.mass_inv(nv, du);
        }
    };

    // The compressible Euler system of examples/cl2d.cpp:67-126 (gamma = 1.4): physical flux
    // (f in fg[0..3], g in fg[4..7]), wave speed |v| + sqrt(gamma p / rho), and the local
    // Lax-Friedrichs flux 1/2 n.(F(qL) + F(qR)) + 1/2 max(speed) (qL - qR).
    constexpr double kGammaE = 1.4;
    void euler_flux(const double q[4], double fg[8])
    {
        const double rho = q[0], u = q[1] / q[0], v = q[2] / q[0], E = q[3];
        const double p = (kGammaE - 1.0) * (E - 0.5 * rho * (u * u + v * v));
        fg[0] = rho * u;
        fg[1] = rho * u * u + p;
        fg[2] = rho * u * v;
        fg[3] = u * (E + p);
        fg[4] = rho * v;
        fg[5] = rho * u * v;
        fg[6] = rho * v * v + p;
        fg[7] = v * (E + p);
    }
    double euler_speed(const double q[4])
    {
        const double rho = q[0], u = q[1] / q[0], v = q[2] / q[0], E = q[3];
        const double p = (kGammaE - 1.0) * (E - 0.5 * rho * (u * u + v * v));
        return std::hypot(u, v) + std::sqrt(kGammaE * p / rho);
    }
    void euler_llf(const double nrm[2], const double qL[4], const double qR[4], double fh[4])
    {
        double fL[8], fR[8];
        euler_flux(qL, fL);
        euler_flux(qR, fR);
        const double c = std::max(euler_speed(qL), euler_speed(qR));
        for (int d = 0; d < 4; ++d)
            fh[d] = 0.5 * nrm[0] * (fL[d] + fR[d]) + 0.5 * nrm[1] * (fL[4 + d] + fR[4 + d]) + 0.5 * c * (qL[d] - qR[d]);
    }

    // The nonlinear conservation-law operators with approximate quadrature on GLL nodes for the
    // Euler system: DivF2D<true>::action (wavedg/DivF.hpp:203-260), EdgeFluxF2D<true>::action
    // (wavedg/EdgeFluxF.hpp:138-180), and the time derivative of examples/cl2d.cpp:171-220
    // (exterior boundary state = interior state), with the Lobatto prolongation and mass of Op.
    struct OpE
    {
        static constexpr int nv = 4;
        const Op base;
        const Mesh &m;
        int n, nel, ndof;

        OpE(const Mesh &m_, int n_)
            : base(m_, n_, std::vector<int>(m_.boundary.size(), 0).data()), m(m_), n(n_), nel(m_.nel),
              ndof(nv * n_ * n_ * m_.nel)
        {
        }
        void div(const double *u, double *du) const
        {
            const int nn = n * n;
            vec F0((size_t)nv * nn), F1((size_t)nv * nn); // F0(l, d, j) at l + n (d + nv j); F1(l, d, i) likewise
            for (int el = 0; el < nel; ++el)
            {
                const double *ue = u + (size_t)nv * nn * el;
                for (int j = 0; j < n; ++j)
                    for (int i = 0; i < n; ++i)
                    {
                        double J[4], fg[8];
                        jacobian(&m.corners[8 * (size_t)el], base.x[i], base.x[j], J);
                        const double W = base.w[i] * base.w[j];
                        const double Ye = J[3] * W, Xe = J[2] * W, Yx = J[1] * W, Xx = J[0] * W;
                        euler_flux(ue + nv * (i + n * j), fg);
                        for (int d = 0; d < nv; ++d)
                        {
                            F0[i + n * (d + nv * j)] = Ye * fg[d] - Xe * fg[4 + d];
                            F1[j + n * (d + nv * i)] = -Yx * fg[d] + Xx * fg[4 + d];
                        }
                    }
                for (int j = 0; j < n; ++j)
                    for (int i = 0; i < n; ++i)
                        for (int d = 0; d < nv; ++d)
                        {
                            double s = 0.0;
                            for (int l = 0; l < n; ++l)
                                s += base.D[l + n * i] * F0[l + n * (d + nv * j)] + base.D[l + n * j] * F1[l + n * (d + nv * i)];
                            du[d + nv * (i + n * (j + (size_t)n * el))] += s;
                        }
            }
        }
        void prolong(bool interior, const double *u, double *uf) const
        {
            const auto &v2e = interior ? base.v2eI : base.v2eB;
            const int N = (int)(interior ? m.interior.size() : m.boundary.size());
            std::fill(uf, uf + (size_t)n * nv * 2 * N, 0.0);
            for (int e = 0; e < N; ++e)
                for (int s = 0; s < (interior ? 2 : 1); ++s)
                    for (int i = 0; i < n; ++i)
                        for (int d = 0; d < nv; ++d)
                            uf[i + n * (d + nv * (s + 2 * (size_t)e))] = u[d + nv * (size_t)v2e[i + n * (s + 2 * (size_t)e)]];
        }
        void prolong_t(bool interior, const double *uf, double *u) const
        {
            const auto &v2e = interior ? base.v2eI : base.v2eB;
            const int N = (int)(interior ? m.interior.size() : m.boundary.size());
            for (int e = 0; e < N; ++e)
                for (int s = 0; s < (interior ? 2 : 1); ++s)
                    for (int i = 0; i < n; ++i)
                        for (int d = 0; d < nv; ++d)
                            u[d + nv * (size_t)v2e[i + n * (s + 2 * (size_t)e)]] += uf[i + n * (d + nv * (s + 2 * (size_t)e))];
        }
        // fB(i, d, 0) = W_i |E|/2 fh(n, u0, u1), fB(i, d, 1) = -fB(i, d, 0); n = outward normal of elements[0]
        void flux(bool interior, const double *ub, double *fb) const
        {
            const auto &list = interior ? m.interior : m.boundary;
            const int N = (int)list.size();
            double qL[4], qR[4], fh[4];
            for (int e = 0; e < N; ++e)
            {
                const Edge &E = m.edges[list[e]];
                for (int i = 0; i < n; ++i)
                {
                    for (int d = 0; d < nv; ++d)
                    {
                        qL[d] = ub[i + n * (d + nv * (0 + 2 * (size_t)e))];
                        qR[d] = ub[i + n * (d + nv * (1 + 2 * (size_t)e))];
                    }
                    euler_llf(E.n, qL, qR, fh);
                    for (int d = 0; d < nv; ++d)
                    {
                        const double fl = fh[d] * base.w[i] * E.meas;
                        fb[i + n * (d + nv * (0 + 2 * (size_t)e))] = fl;
                        fb[i + n * (d + nv * (1 + 2 * (size_t)e))] = -fl;
                    }
                }
            }
        }
        void rhs(const double *u, double *du) const
        {
            std::fill(du, du + ndof, 0.0);
            div(u, du);
            vec uI((size_t)n * nv * 2 * m.interior.size()), uB((size_t)n * nv * 2 * m.boundary.size());
            prolong(true, u, uI.data());
            flux(true, uI.data(), uI.data());
            for (double &x : uI)
                x = -x;
            prolong_t(true, uI.data(), du);
            prolong(false, u, uB.data());
            for (size_t e = 0; e < m.boundary.size(); ++e)
                for (int d = 0; d < nv; ++d)
                    for (int i = 0; i < n; ++i)
                        uB[i + n * (d + nv * (1 + 2 * e))] = uB[i + n * (d + nv * (0 + 2 * e))];
            flux(false, uB.data(), uB.data());
            for (double &x : uB)
                x = -x;
            prolong_t(false, uB.data(), du);
            base.mass_inv(nv, du);
        }
    };

    // D(i, j) = phi_j'(xq_i) at points off (or on) the nodes: lagrange_basis_deriv with the
    // two branches of lagrange_derivative (lagrange_interpolation.cpp:33-50, 96-139)
    void deriv_at(int n, const double *x, int nq, const double *xq, double *D)
    {
        double lw[16], B[16 * 16];
        bary(x, n, lw);
        interp_matrix(n, x, nq, xq, B);
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < nq; ++i)
            {
                const double x0 = xq[i], p = B[i + nq * j];
                int at = -1;
                for (int k = 0; k < n; ++k)
                    if (x0 == x[k] || std::abs(x0 - x[k]) <= 2.220446049250313e-16)
                        at = k;
                double A = 0.0, Bs = 0.0;
                if (at >= 0)
                {
                    Bs = -lw[at];
                    for (int k = 0; k < n; ++k)
                        if (k != at)
                            A += lw[k] * (p - (k == j ? 1.0 : 0.0)) / (x0 - x[k]);
                }
                else
                    for (int k = 0; k < n; ++k)
                    {
                        const double t = lw[k] / (x0 - x[k]);
                        A += t * (p - (k == j ? 1.0 : 0.0)) / (x0 - x[k]);
                        Bs += t;
                    }
                D[i + nq * j] = A / Bs;
            }
    }

    // The wave system with approx_quad = false (exact quadrature): Div<false>
    // (source/Div.cpp:312-361 with op_2d_cc, and div_2d_q :469-588), EdgeFlux<false>
    // (source/EdgeFlux.cpp:496-535, flux_action_2d_q :548-622), MassMatrix<false>
    // (source/MassMatrix.cpp:84-230 with chol / solve_chol / mult_chol, linalg.cpp:5-100).
    // Default rules (Gauss-Legendre): Div p = 1 + ((n-2) + (n-1) + 1) / 2 points,
    // EdgeFlux and MassMatrix p = 1 + (2 (n-1) + 2) / 2.  Prolongation and exterior states
    // are the Lobatto ones of Op.
    struct OpQ
    {
        const Op base;
        const Mesh &m;
        int n, nel, ndof, nqd, nqf, nqm;
        vec xd, wd, Pd, Dd; // Div rule and P(i, k) = phi_k(xq_i), D(i, k) = phi_k'(xq_i)
        vec xf, wf, Pf;     // face rule
        vec L;              // Cholesky factors of the element mass matrices (c2d, c2d, nel)

        OpQ(const Mesh &m_, int n_, const int *codes)
            : base(m_, n_, codes), m(m_), n(n_), nel(m_.nel), ndof(3 * n_ * n_ * m_.nel)
        {
            nqd = 1 + ((n - 2) + (n - 1) + 1) / 2;
            nqf = 1 + (2 * (n - 1) + 2) / 2;
            nqm = nqf;
            xd.resize(nqd);
            wd.resize(nqd);
            gl(nqd, xd.data(), wd.data());
            Pd.resize(nqd * n);
            Dd.resize(nqd * n);
            interp_matrix(n, base.x.data(), nqd, xd.data(), Pd.data());
            deriv_at(n, base.x.data(), nqd, xd.data(), Dd.data());
            xf.resize(nqf);
            wf.resize(nqf);
            gl(nqf, xf.data(), wf.data());
            Pf.resize(nqf * n);
            interp_matrix(n, base.x.data(), nqf, xf.data(), Pf.data());
            // element mass matrices on the nqm x nqm rule, lower triangle, then chol
            vec xm(nqm), wm(nqm), Bm(nqm * n);
            gl(nqm, xm.data(), wm.data());
            interp_matrix(n, base.x.data(), nqm, xm.data(), Bm.data());
            const int c = n * n, q2 = nqm * nqm;
            L.assign((size_t)c * c * nel, 0.0);
            vec detJ(q2);
            for (int el = 0; el < nel; ++el)
            {
                const double *cr = &m.corners[8 * (size_t)el];
                for (int p = 0; p < q2; ++p)
                {
                    double J[4];
                    jacobian(cr, xm[p % nqm], xm[p / nqm], J);
                    detJ[p] = J[0] * J[3] - J[2] * J[1];
                }
                double *M = &L[(size_t)c * c * el];
                for (int j = 0; j < c; ++j)
                    for (int i = j; i < c; ++i)
                    {
                        double mij = 0.0;
                        for (int p = 0; p < q2; ++p)
                        {
                            const double bi = Bm[p % nqm + nqm * (i % n)] * Bm[p / nqm + nqm * (i / n)];
                            const double bj = Bm[p % nqm + nqm * (j % n)] * Bm[p / nqm + nqm * (j / n)];
                            mij += bi * bj * detJ[p] * wm[p % nqm] * wm[p / nqm];
                        }
                        M[i + c * j] = mij;
                    }
                for (int k = 0; k < c; ++k)
                {
                    for (int j = k + 1; j < c; ++j)
                    {
                        const double sc = M[j + c * k] / M[k + c * k];
                        for (int i = j; i < c; ++i)
                            M[i + c * j] -= sc * M[i + c * k];
                    }
                    const double sc = 1.0 / std::sqrt(M[k + c * k]);
                    for (int i = k; i < c; ++i)
                        M[i + c * k] *= sc;
                }
            }
        }

        // div_2d_q: u -> quadrature points, contravariant fluxes, (F, grad v) back; accumulates
        void div(const double *u, double *du) const
        {
            const int q = nqd;
            vec Pu((size_t)n * 3 * q), Uq((size_t)3 * q * q), Fq((size_t)2 * 3 * q * q), Df((size_t)q * 3 * n),
                Pg((size_t)q * 3 * n);
            for (int el = 0; el < nel; ++el)
            {
                const double *ue = u + (size_t)3 * n * n * el;
                const double *cr = &m.corners[8 * (size_t)el];
                for (int i = 0; i < q; ++i)
                    for (int l = 0; l < n; ++l)
                        for (int d = 0; d < 3; ++d)
                        {
                            double s = 0.0;
                            for (int k = 0; k < n; ++k)
                                s += Pd[i + q * k] * ue[d + 3 * (k + n * l)];
                            Pu[l + n * (d + 3 * i)] = s;
                        }
                for (int j = 0; j < q; ++j)
                    for (int i = 0; i < q; ++i)
                        for (int d = 0; d < 3; ++d)
                        {
                            double s = 0.0;
                            for (int l = 0; l < n; ++l)
                                s += Pd[j + q * l] * Pu[l + n * (d + 3 * i)];
                            Uq[d + 3 * (i + q * j)] = s;
                        }
                for (int j = 0; j < q; ++j)
                    for (int i = 0; i < q; ++i)
                    {
                        double J[4];
                        jacobian(cr, xd[i], xd[j], J);
                        const double W = wd[i] * wd[j];
                        const double Xxi = J[0] * W, Yxi = J[1] * W, Xeta = J[2] * W, Yeta = J[3] * W;
                        const double *U = &Uq[3 * (i + q * j)];
                        double *F = &Fq[2 * 3 * (i + q * j)];
                        // wave system: a(0,1,0) = a(1,0,0) = a(0,2,1) = a(2,0,1) = 1
                        F[0] = Yeta * U[1] - Xeta * U[2];
                        F[1] = -Yxi * U[1] + Xxi * U[2];
                        F[2] = Yeta * U[0];
                        F[3] = -Yxi * U[0];
                        F[4] = -Xeta * U[0];
                        F[5] = Xxi * U[0];
                    }
                for (int j = 0; j < q; ++j)
                    for (int k = 0; k < n; ++k)
                        for (int d = 0; d < 3; ++d)
                        {
                            double df = 0.0, pg = 0.0;
                            for (int i = 0; i < q; ++i)
                            {
                                df += Dd[i + q * k] * Fq[2 * d + 6 * (i + q * j)];
                                pg += Pd[i + q * k] * Fq[2 * d + 1 + 6 * (i + q * j)];
                            }
                            Df[j + q * (d + 3 * k)] = df;
                            Pg[j + q * (d + 3 * k)] = pg;
                        }
                double *de = du + (size_t)3 * n * n * el;
                for (int l = 0; l < n; ++l)
                    for (int k = 0; k < n; ++k)
                        for (int d = 0; d < 3; ++d)
                        {
                            double s = 0.0;
                            for (int j = 0; j < q; ++j)
                                s += Pd[j + q * l] * Df[j + q * (d + 3 * k)] + Dd[j + q * l] * Pg[j + q * (d + 3 * k)];
                            de[d + 3 * (k + n * l)] += s;
                        }
            }
        }

        // flux_action_2d_q: traces -> face points, upwind flux (w_q |E|/2 Fs), back; side 1 = -side 0
        void flux(bool interior, const double *ub, double *fb) const
        {
            const int q = nqf;
            const std::vector<int> &list = interior ? m.interior : m.boundary;
            const int N = (int)list.size();
            static const double a[] = {0, 1, 0, 1, 0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0};
            vec uf((size_t)q * 3);
            for (int e = 0; e < N; ++e)
            {
                const Edge &E = m.edges[list[e]];
                double nA[9], R[9], ev[3], Fs[2][9];
                for (int d = 0; d < 9; ++d)
                    nA[d] = E.n[0] * a[d] + E.n[1] * a[d + 9];
                sym_eig3(nA, R, ev);
                for (int s = 0; s < 2; ++s)
                {
                    const double sgn = (s == 0) ? 1.0 : -1.0;
                    for (int i = 0; i < 3; ++i)
                        for (int j = 0; j < 3; ++j)
                        {
                            double acc = 0.0;
                            for (int k = 0; k < 3; ++k)
                                acc += R[i + 3 * k] * (0.5 * -1.0 * ev[k] + sgn * -0.5 * std::abs(ev[k])) * R[j + 3 * k];
                            Fs[s][i + 3 * j] = acc;
                        }
                }
                std::fill(uf.begin(), uf.end(), 0.0);
                for (int s = 0; s < 2; ++s)
                    for (int i = 0; i < q; ++i)
                    {
                        double Uq[3];
                        for (int d = 0; d < 3; ++d)
                        {
                            double v = 0.0;
                            for (int j = 0; j < n; ++j)
                                v += ub[j + n * (d + 3 * (s + 2 * (size_t)e))] * Pf[i + q * j];
                            Uq[d] = v;
                        }
                        const double w = wf[i] * E.meas;
                        for (int d = 0; d < 3; ++d)
                        {
                            double f = 0.0;
                            for (int c = 0; c < 3; ++c)
                                f += (w * Fs[s][c + 3 * d]) * Uq[c];
                            uf[i + q * d] += f;
                        }
                    }
                for (int d = 0; d < 3; ++d)
                    for (int i = 0; i < n; ++i)
                    {
                        double f = 0.0;
                        for (int j = 0; j < q; ++j)
                            f += uf[j + q * d] * Pf[j + q * i];
                        fb[i + n * (d + 3 * (0 + 2 * (size_t)e))] = f;
                        fb[i + n * (d + 3 * (1 + 2 * (size_t)e))] = -f;
                    }
            }
        }

        void wave_action(const double *u, double *du) const
        {
            div(u, du);
            vec uf((size_t)n * 3 * 2 * m.interior.size());
            base.prolong(true, u, uf.data());
            flux(true, uf.data(), uf.data());
            base.prolong_t(true, uf.data(), du);
        }
        void bc_action(const double *u, double *du) const
        {
            vec uB((size_t)n * 3 * 2 * m.boundary.size());
            base.prolong(false, u, uB.data());
            base.apply_bc(uB.data());
            flux(false, uB.data(), uB.data());
            base.prolong_t(false, uB.data(), du);
        }
        // solve_chol: L \ x, then L^T \ x, nv right-hand sides interleaved per node
        void mass_inv(int nv, double *x) const
        {
            const int c = n * n;
            for (int el = 0; el < nel; ++el)
            {
                const double *M = &L[(size_t)c * c * el];
                double *X = x + (size_t)nv * c * el;
                for (int j = 0; j < c; ++j)
                {
                    for (int d = 0; d < nv; ++d)
                        X[d + nv * j] /= M[j + c * j];
                    for (int i = j + 1; i < c; ++i)
                        for (int d = 0; d < nv; ++d)
                            X[d + nv * i] -= M[i + c * j] * X[d + nv * j];
                }
                for (int j = c - 1; j >= 0; --j)
                {
                    for (int d = 0; d < nv; ++d)
                        X[d + nv * j] /= M[j + c * j];
                    for (int i = 0; i < j; ++i)
                        for (int d = 0; d < nv; ++d)
                            X[d + nv * i] -= M[j + c * i] * X[d + nv * j];
                }
            }
        }
        // mult_chol: y = L (L^T x)
        void mass_action(int nv, const double *x, double *y) const
        {
            const int c = n * n;
            std::copy(x, x + (size_t)nv * c * nel, y);
            for (int el = 0; el < nel; ++el)
            {
                const double *M = &L[(size_t)c * c * el];
                double *Y = y + (size_t)nv * c * el;
                for (int i = 0; i < c; ++i)
                    for (int d = 0; d < nv; ++d)
                    {
                        double t = 0.0;
                        for (int j = i; j < c; ++j)
                            t += M[j + c * i] * Y[d + nv * j];
                        Y[d + nv * i] = t;
                    }
                for (int i = c - 1; i >= 0; --i)
                    for (int d = 0; d < nv; ++d)
                    {
                        double t = 0.0;
                        for (int j = 0; j <= i; ++j)
                            t += M[i + c * j] * Y[d + nv * j];
                        Y[d + nv * i] = t;
                    }
            }
        }
        void rhs(const double *u, double *du, const double *F = nullptr, double s = 0.0) const
        {
            std::fill(du, du + ndof, 0.0);
            wave_action(u, du);
            bc_action(u, du);
            if (F)
                for (int i = 0; i < ndof; ++i)
                    du[i] += F[i] * s;
            mass_inv(3, du);
        }
    };

    double min_h(const Mesh &m)
    {
        double h = INFINITY;
        for (const Edge &E : m.edges)
            h = std::min(h, 2.0 * E.meas);
        return h;
    }

    // WaveHoltz (source/WaveHoltz.cpp:5-145)
    // WaveHoltz over either operator set (collocation Op or exact-quadrature OpQ)
    struct WHBase
    {
        double omega = 0, T = 0, dt = 0;
        int nt = 0, ndof = 0;
        virtual ~WHBase() = default;
        virtual void pi0(double *u, const double *F) const = 0;
        virtual void S(double *u) const = 0;
        virtual void postprocess(double *H, const double *U) const = 0;
    };
    template <class O>
    struct WHT : WHBase
    {
        const O &op;
        mutable vec p, q, du;
        WHT(const O &o, double om) : op(o), p(o.ndof), q(o.ndof), du(o.ndof)
        {
            omega = om;
            ndof = o.ndof;
            T = 2.0 * M_PI / omega;
            const double h = min_h(o.m);
            const double pp = o.n;
            dt = 0.5 * h / (pp * pp);
            nt = (int)std::ceil(T / dt);
            dt = T / nt;
        }
        double K(double t) const { return omega / M_PI * (std::cos(omega * t) - 0.25); }
        void pi0(double *u, const double *F) const override
        {
            auto f = [this, F](double *vt, double t, const double *v)
            { op.rhs(v, vt, F, -1.0 / omega * std::sin(omega * t)); };
            std::fill(p.begin(), p.end(), 0.0);
            std::fill(u, u + op.ndof, 0.0);
            double t = 0.0;
            for (int it = 1; it <= nt; ++it)
            {
                rk4_step(op.ndof, dt, f, t, p.data(), q, du);
                const double c = ((it == nt) ? 0.5 : 1.0) * dt * K(t);
                for (int i = 0; i < op.ndof; ++i)
                    u[i] += c * p[i];
            }
        }
        void S(double *u) const override
        {
            auto f = [this](double *vt, double, const double *v)
            { op.rhs(v, vt, nullptr, 0.0); };
            for (int i = 0; i < op.ndof; ++i)
            {
                p[i] = u[i];
                u[i] *= 0.5 * dt * K(0.0);
            }
            double t = 0.0;
            for (int it = 1; it <= nt; ++it)
            {
                rk4_step(op.ndof, dt, f, t, p.data(), q, du);
                const double c = ((it == nt) ? 0.5 : 1.0) * dt * K(t);
                for (int i = 0; i < op.ndof; ++i)
                    u[i] += c * p[i];
            }
        }
        void postprocess(double *H, const double *U) const override
        {
            op.rhs(U, p.data(), nullptr, 0.0);
            for (int i = 0; i < op.ndof / 3; ++i)
            {
                H[2 * i] = U[3 * i];
                H[2 * i + 1] = -1.0 / omega * p[3 * i];
            }
        }
    };

    double norm2(int nd, const double *a)
    {
        double r = 0.0;
        for (int i = 0; i < nd; ++i)
            r += a[i] * a[i];
        return std::sqrt(r);
    }
    double err2(int nd, const double *a, const double *b)
    {
        double r = 0.0;
        for (int i = 0; i < nd; ++i)
        {
            const double d = a[i] - b[i];
            r += d * d;
        }
        return std::sqrt(r);
    }
} // namespace

extern "C"
{
    void *orc_mesh_create(int nv, const double *xy, int nel, const int *quads) { return make_mesh(nv, xy, nel, quads); }
    // Mesh2D::from_file (source/Mesh2D.cpp:94-128): info.txt "n_pts n_elem", coordinates.txt
    // "x y" per point, elements.txt four point indices per element, then from_vertices;
    // nullptr if a file is missing or short
    void *orc_mesh_from_file(const char *dir)
    {
        // C stdio, not iostreams: this library may share a process with another C++ runtime
        const std::string d(dir);
        FILE *info = std::fopen((d + "/info.txt").c_str(), "r");
        FILE *coo = std::fopen((d + "/coordinates.txt").c_str(), "r");
        FILE *els = std::fopen((d + "/elements.txt").c_str(), "r");
        int np = 0, ne = 0;
        bool ok = info && coo && els && std::fscanf(info, "%d %d", &np, &ne) == 2 && np >= 1 && ne >= 1;
        std::vector<double> xy(ok ? 2 * (size_t)np : 0);
        std::vector<int> q(ok ? 4 * (size_t)ne : 0);
        for (size_t i = 0; ok && i < xy.size(); ++i)
            ok = std::fscanf(coo, "%lf", &xy[i]) == 1;
        for (size_t i = 0; ok && i < q.size(); ++i)
            ok = std::fscanf(els, "%d", &q[i]) == 1;
        for (FILE *f : {info, coo, els})
            if (f)
                std::fclose(f);
        return ok ? make_mesh(np, xy.data(), ne, q.data()) : nullptr;
    }
    void orc_mesh_destroy(void *m) { delete static_cast<Mesh *>(m); }
    int orc_mesh_n_elem(void *m) { return static_cast<Mesh *>(m)->nel; }
    int orc_mesh_n_edges(void *m, int type)
    {
        Mesh *M = static_cast<Mesh *>(m);
        return (int)(type == 0 ? M->interior.size() : M->boundary.size());
    }
    double orc_mesh_min_h(void *m) { return min_h(*static_cast<Mesh *>(m)); }
    void orc_mesh_edges(void *m, int type, int *out)
    {
        Mesh *M = static_cast<Mesh *>(m);
        const auto &list = (type == 0) ? M->interior : M->boundary;
        for (size_t e = 0; e < list.size(); ++e)
        {
            const Edge &E = M->edges[list[e]];
            out[5 * e + 0] = E.el[0];
            out[5 * e + 1] = E.side[0];
            out[5 * e + 2] = type == 0 ? E.el[1] : -1;
            out[5 * e + 3] = type == 0 ? E.side[1] : -1;
            out[5 * e + 4] = type == 0 ? E.delta : 1;
        }
    }
    void orc_mesh_boundary_midpoints(void *m, double *xy)
    {
        Mesh *M = static_cast<Mesh *>(m);
        for (size_t e = 0; e < M->boundary.size(); ++e)
        {
            const Edge &E = M->edges[M->boundary[e]];
            xy[2 * e] = E.x0[0] + E.dx[0] * 0.5;
            xy[2 * e + 1] = E.x0[1] + E.dx[1] * 0.5;
        }
    }

    void orc_basis(int n, double *x, double *w, double *D)
    {
        gll(n, x, w);
        deriv_matrix(n, x, D);
    }

    void *orc_op_create(void *m, int n, const int *bc) { return new Op(*static_cast<Mesh *>(m), n, bc); }
    void orc_op_destroy(void *o) { delete static_cast<Op *>(o); }
    void orc_node_coords(void *o, double *xy)
    {
        Op *op = static_cast<Op *>(o);
        const int n = op->n;
        for (int el = 0; el < op->nel; ++el)
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i)
                    physical(&op->m.corners[8 * (size_t)el], op->x[i], op->x[j], &xy[2 * (i + n * (j + (size_t)n * el))]);
    }
    void orc_div(void *o, const double *u, double *du) { static_cast<Op *>(o)->div(u, du); }
    void orc_wave_action(void *o, const double *u, double *du) { static_cast<Op *>(o)->wave_action(u, du); }
    void orc_bc_action(void *o, const double *u, double *du) { static_cast<Op *>(o)->bc_action(u, du); }
    void orc_prolong(void *o, int type, const double *u, double *uf) { static_cast<Op *>(o)->prolong(type == 0, u, uf); }
    void orc_prolong_t(void *o, int type, const double *uf, double *u) { static_cast<Op *>(o)->prolong_t(type == 0, uf, u); }
    void orc_flux(void *o, int type, const double *uf, double *fb) { static_cast<Op *>(o)->flux(type == 0, uf, fb); }
    void orc_apply_bc(void *o, double *uB) { static_cast<Op *>(o)->apply_bc(uB); }
    void orc_mass_inv(void *o, int nv, double *x) { static_cast<Op *>(o)->mass_inv(nv, x); }
    void orc_mass_action(void *o, int nv, const double *x, double *y) { static_cast<Op *>(o)->mass_action(nv, x, y); }
    void orc_rhs(void *o, const double *u, double *du) { static_cast<Op *>(o)->rhs(u, du, nullptr, 0.0); }
    void orc_rhs_forced(void *o, const double *u, double *du, const double *F, double s) { static_cast<Op *>(o)->rhs(u, du, F, s); }

    void orc_rk4(void *o, double dt, int nsteps, double *t, double *u)
    {
        Op *op = static_cast<Op *>(o);
        vec p(op->ndof), du(op->ndof);
        auto f = [op](double *dudt, double, const double *v)
        { op->rhs(v, dudt, nullptr, 0.0); };
        for (int s = 0; s < nsteps; ++s)
            rk4_step(op->ndof, dt, f, *t, u, p, du);
    }

    // LinearFunctional2D::action (wavedg/LinearFunctional.hpp:61-74, 136-202): (f, phi)
    // with the n-point Gauss-Legendre rule, f a sum of Gaussians in component comp
    void orc_load_gaussians(void *o, int nsrc, const double *cx, const double *cy, const double *sigma,
                            const double *amp, double scale, int comp, int mass_inv, double *F)
    {
        Op *op = static_cast<Op *>(o);
        const int n = op->n, nq = n;
        vec xq(nq), wq(nq), B((size_t)nq * n);
        gl(nq, xq.data(), wq.data());
        interp_matrix(n, op->x.data(), nq, xq.data(), B.data());
        vec Fq((size_t)3 * nq * nq), P((size_t)3 * nq * n);
        for (int el = 0; el < op->nel; ++el)
        {
            const double *c = &op->m.corners[8 * (size_t)el];
            for (int l = 0; l < nq; ++l)
                for (int k = 0; k < nq; ++k)
                {
                    double X[2], J[4];
                    physical(c, xq[k], xq[l], X);
                    jacobian(c, xq[k], xq[l], J);
                    double s = 0.0;
                    for (int q = 0; q < nsrc; ++q)
                    {
                        const double dx = X[0] - cx[q], dy = X[1] - cy[q];
                        s += amp[q] * std::exp(-(dx * dx + dy * dy) / (2.0 * sigma[q] * sigma[q]));
                    }
                    const double wgt = (J[0] * J[3] - J[1] * J[2]) * wq[k] * wq[l];
                    for (int d = 0; d < 3; ++d)
                        Fq[d + 3 * (k + nq * l)] = ((d == comp) ? scale * s : 0.0) * wgt;
                }
            for (int j = 0; j < n; ++j)
                for (int k = 0; k < nq; ++k)
                    for (int d = 0; d < 3; ++d)
                    {
                        double s = 0.0;
                        for (int l = 0; l < nq; ++l)
                            s += Fq[d + 3 * (k + nq * l)] * B[l + nq * j];
                        P[d + 3 * (k + nq * j)] = s;
                    }
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i)
                    for (int d = 0; d < 3; ++d)
                    {
                        double s = 0.0;
                        for (int k = 0; k < nq; ++k)
                            s += P[d + 3 * (k + nq * j)] * B[k + nq * i];
                        F[d + 3 * (i + n * (j + (size_t)n * el))] = s;
                    }
        }
        if (mass_inv)
            op->mass_inv(3, F);
    }

    double orc_norm(int nd, const double *x) { return norm2(nd, x); }
    double orc_error(int nd, const double *x, const double *y) { return err2(nd, x, y); }

    void *orc_opa_create(void *m, int n, int nv, const double *a) { return new OpA(*static_cast<Mesh *>(m), n, nv, a); }
    void orc_opa_destroy(void *o) { delete static_cast<OpA *>(o); }
    void orc_opa_action(void *o, const double *u, double *du) { static_cast<OpA *>(o)->action(u, du); }
    void orc_opa_bc_action(void *o, const double *u, double *du) { static_cast<OpA *>(o)->bc_action(u, du); }
    void orc_opa_rhs(void *o, const double *u, double *du) { static_cast<OpA *>(o)->rhs(u, du); }
    void orc_opa_rk4(void *o, double dt, int nsteps, double *t, double *u)
    {
        OpA *op = static_cast<OpA *>(o);
        vec p(op->ndof), du(op->ndof);
        auto f = [op](double *dudt, double, const double *v) { op->rhs(v, dudt); };
        for (int s = 0; s < nsteps; ++s)
            rk4_step(op->ndof, dt, f, *t, u, p, du);
    }
    void *orc_ope_create(void *m, int n) { return new OpE(*static_cast<Mesh *>(m), n); }
    void orc_ope_destroy(void *o) { delete static_cast<OpE *>(o); }
    void orc_ope_div(void *o, const double *u, double *du) { static_cast<OpE *>(o)->div(u, du); }
    void orc_ope_flux(void *o, int type, const double *ub, double *fb) { static_cast<OpE *>(o)->flux(type == 0, ub, fb); }
    void orc_ope_prolong(void *o, int type, const double *u, double *ub) { static_cast<OpE *>(o)->prolong(type == 0, u, ub); }
    void orc_ope_rhs(void *o, const double *u, double *du) { static_cast<OpE *>(o)->rhs(u, du); }
    // method 0: ode::RungeKutta4; 1: ode::SSPRK3 (wavedg/ode.hpp:145-186), step for step
    void orc_ope_steps(void *o, int method, double dt, int nsteps, double *t, double *u)
    {
        OpE *op = static_cast<OpE *>(o);
        const int nd = op->ndof;
        vec p(nd), du(nd), y(nd);
        auto f = [op](double *dudt, double, const double *v) { op->rhs(v, dudt); };
        for (int s = 0; s < nsteps; ++s)
        {
            if (method == 0)
            {
                rk4_step(nd, dt, f, *t, u, p, du);
                continue;
            }
            f(p.data(), *t, u);
            for (int i = 0; i < nd; ++i)
                y[i] = u[i] + dt * p[i];
            f(p.data(), *t + dt, y.data());
            for (int i = 0; i < nd; ++i)
                y[i] = 0.25 * (y[i] + 3.0 * u[i] + dt * p[i]);
            f(p.data(), *t + 0.5 * dt, y.data());
            for (int i = 0; i < nd; ++i)
                u[i] = (u[i] + 2.0 * y[i] + 2.0 * dt * p[i]) / 3.0;
            *t += dt;
        }
    }
    void *orc_opq_create(void *m, int n, const int *bc) { return new OpQ(*static_cast<Mesh *>(m), n, bc); }
    void orc_opq_destroy(void *o) { delete static_cast<OpQ *>(o); }
    void orc_opq_div(void *o, const double *u, double *du) { static_cast<OpQ *>(o)->div(u, du); }
    void orc_opq_flux(void *o, int type, const double *uf, double *fb) { static_cast<OpQ *>(o)->flux(type == 0, uf, fb); }
    void orc_opq_wave_action(void *o, const double *u, double *du) { static_cast<OpQ *>(o)->wave_action(u, du); }
    void orc_opq_bc_action(void *o, const double *u, double *du) { static_cast<OpQ *>(o)->bc_action(u, du); }
    void orc_opq_mass_inv(void *o, int nv, double *x) { static_cast<OpQ *>(o)->mass_inv(nv, x); }
    void orc_opq_mass_action(void *o, int nv, const double *x, double *y) { static_cast<OpQ *>(o)->mass_action(nv, x, y); }
    void orc_opq_rhs(void *o, const double *u, double *du) { static_cast<OpQ *>(o)->rhs(u, du); }
    void orc_opq_rk4(void *o, double dt, int nsteps, double *t, double *u)
    {
        OpQ *op = static_cast<OpQ *>(o);
        vec p(op->ndof), du(op->ndof);
        auto f = [op](double *dudt, double, const double *v) { op->rhs(v, dudt); };
        for (int s = 0; s < nsteps; ++s)
            rk4_step(op->ndof, dt, f, *t, u, p, du);
    }
    void *orc_wh_create(void *o, double omega) { return static_cast<WHBase *>(new WHT<Op>(*static_cast<Op *>(o), omega)); }
    void *orc_whq_create(void *o, double omega) { return static_cast<WHBase *>(new WHT<OpQ>(*static_cast<OpQ *>(o), omega)); }
    void orc_wh_destroy(void *w) { delete static_cast<WHBase *>(w); }
    void orc_wh_params(void *w, double *T, double *dt, int *nt)
    {
        WHBase *wh = static_cast<WHBase *>(w);
        *T = wh->T;
        *dt = wh->dt;
        *nt = wh->nt;
    }
    void orc_wh_pi0(void *w, double *u, const double *F) { static_cast<WHBase *>(w)->pi0(u, F); }
    void orc_wh_S(void *w, double *u) { static_cast<WHBase *>(w)->S(u); }
    void orc_wh_postprocess(void *w, double *H, const double *U) { static_cast<WHBase *>(w)->postprocess(H, U); }
    // examples/waveholtz2d.cpp:165-185 from W (in/out)
    int orc_wh_solve(void *w, const double *pi0, double tol, int maxit, double *W, double *err_out)
    {
        WHBase *wh = static_cast<WHBase *>(w);
        const int nd = wh->ndof;
        const double pz = norm2(nd, pi0);
        vec prev(nd);
        int it;
        double err = 0.0;
        for (it = 1; it <= maxit; ++it)
        {
            std::copy(W, W + nd, prev.begin());
            wh->S(W);
            for (int i = 0; i < nd; ++i)
                W[i] += pi0[i];
            err = err2(nd, W, prev.data()) / pz;
            if (err < tol)
                break;
        }
        *err_out = err;
        return it;
    }
}
