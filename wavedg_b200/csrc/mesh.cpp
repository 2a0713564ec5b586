// Host-side set-up: mesh connectivity, quadrature, and the face tables the
// kernels read.  Runs once per mesh / discretisation; nothing here is on the
// per-stage path.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <string>
#include <unordered_map>

#include "common.hpp"

namespace wdg
{
    thread_local std::string g_last_error;

    int fail(int code, const std::string &msg)
    {
        g_last_error = msg;
        return code;
    }
    int cuda_fail(cudaError_t e, const char *what)
    {
        g_last_error = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
        return WDG_ERR_CUDA;
    }
    void clear_error() { g_last_error.clear(); }

    // Legendre P_k and P_k' by recurrence (P_k' only away from +-1)
    static void legendre(int k, double x, double &P, double &dP)
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
            const double p2 = ((2 * j - 1) * x * p1 - (j - 1) * p0) / j;
            p0 = p1;
            p1 = p2;
        }
        P = p1;
        dP = (x * x == 1.0) ? 0.0 : k * (x * p1 - p0) / (x * x - 1.0);
    }

    // Interior GLL nodes are the roots of P'_{n-1}; Newton on
    // f = P'_{n-1}, f' = (2x P' - n(n-1) P)/(1 - x^2), started at the
    // Chebyshev-Lobatto points and mirrored so the rule is exactly symmetric
    // (the flux weights of the two sides of an edge must agree).
    // Weights 2 / (n (n-1) P_{n-1}(x)^2) as in QuadratureRule::gauss_lobatto.
    void gauss_lobatto(int n, double *x, double *w)
    {
        x[0] = -1.0;
        x[n - 1] = 1.0;
        for (int i = 1; i < (n + 1) / 2; ++i)
        {
            double t = -std::cos(M_PI * i / (n - 1));
            for (int it = 0; it < 64; ++it)
            {
                double P, dP;
                legendre(n - 1, t, P, dP);
                const double step = dP * (1.0 - t * t) / (2.0 * t * dP - (n - 1.0) * n * P);
                t -= step;
                if (std::fabs(step) < 1e-16)
                    break;
            }
            x[i] = t;
            x[n - 1 - i] = -t;
        }
        if (n & 1)
            x[n / 2] = 0.0;
        for (int i = 0; i < (n + 1) / 2; ++i)
        {
            double P, dP;
            legendre(n - 1, x[i], P, dP);
            w[i] = w[n - 1 - i] = 2.0 / (n * (n - 1) * P * P);
        }
    }

    // roots of P_n by Newton; w = 2 / ((1 - x^2) P_n'(x)^2)
    void gauss_legendre(int n, double *x, double *w)
    {
        for (int i = 0; i < (n + 1) / 2; ++i)
        {
            double t = -std::cos(M_PI * (i + 0.75) / (n + 0.5));
            for (int it = 0; it < 64; ++it)
            {
                double P, dP;
                legendre(n, t, P, dP);
                const double step = P / dP;
                t -= step;
                if (std::fabs(step) < 1e-16)
                    break;
            }
            x[i] = t;
            x[n - 1 - i] = -t;
        }
        if (n & 1)
            x[n / 2] = 0.0;
        for (int i = 0; i < (n + 1) / 2; ++i)
        {
            double P, dP;
            legendre(n, x[i], P, dP);
            w[i] = w[n - 1 - i] = 2.0 / ((1.0 - x[i] * x[i]) * dP * dP);
        }
    }

    // barycentric weights lambda_j = 1 / prod_{k != j} (x_j - x_k)
    static void barycentric(int n, const double *x, double *lam)
    {
        for (int j = 0; j < n; ++j)
        {
            double p = 1.0;
            for (int k = 0; k < n; ++k)
                if (k != j)
                    p *= x[j] - x[k];
            lam[j] = 1.0 / p;
        }
    }

    // D[l + n j] = phi_j'(x_l): (lam_j / lam_l) / (x_l - x_j) off the diagonal,
    // minus the row sum on it
    void deriv_matrix(int n, const double *x, double *D)
    {
        double lam[kMaxN + 1];
        barycentric(n, x, lam);
        for (int l = 0; l < n; ++l)
        {
            double diag = 0.0;
            for (int j = 0; j < n; ++j)
            {
                if (j == l)
                    continue;
                const double d = (lam[j] / lam[l]) / (x[l] - x[j]);
                D[l + n * j] = d;
                diag -= d;
            }
            D[l + n * l] = diag;
        }
    }

    // B[i + nq j] = phi_j(xq_i), second barycentric form
    void interp_matrix(int n, const double *x, int nq, const double *xq, double *B)
    {
        double lam[kMaxN + 1];
        barycentric(n, x, lam);
        for (int i = 0; i < nq; ++i)
        {
            int hit = -1;
            double den = 0.0;
            for (int k = 0; k < n; ++k)
            {
                if (xq[i] == x[k])
                    hit = k;
                den += lam[k] / (xq[i] - x[k]);
            }
            for (int j = 0; j < n; ++j)
                B[i + nq * j] = (hit >= 0) ? (j == hit ? 1.0 : 0.0) : (lam[j] / (xq[i] - x[j])) / den;
        }
    }

    int build_face_tables(const wdg_mesh &m, const int *bc, FaceTables &ft)
    {
        const int nel = m.nel;
        ft.nbr.assign(4 * (size_t)nel, -1);
        ft.info.assign(nel, 0u);
        ft.face_edge.assign(4 * (size_t)nel, -1);
        std::vector<uint8_t> seen(4 * (size_t)nel, 0);
        auto set = [&](int el, int f, uint32_t byte, int nb, int edge_slot) -> int
        {
            if (el < 0 || el >= nel || f < 0 || f > 3)
                return fail(WDG_ERR_ARG, "mesh edge table references an element or side out of range");
            if (seen[4 * (size_t)el + f]++)
                return fail(WDG_ERR_ARG, "mesh has an element side shared by more than two elements");
            ft.info[el] |= byte << (8 * f);
            ft.nbr[4 * (size_t)el + f] = nb;
            ft.face_edge[4 * (size_t)el + f] = edge_slot;
            return WDG_OK;
        };
        for (size_t e = 0; e < m.interior.size(); ++e)
        {
            const EdgeRec &E = m.interior[e];
            if (E.s0 < 0 || E.s0 > 3 || E.s1 < 0 || E.s1 > 3)
                return fail(WDG_ERR_ARG, "interior edge with side out of range");
            const uint32_t flip = (E.delta < 0) ? 4u : 0u;
            WDG_TRY(set(E.el0, E.s0, (uint32_t)E.s1 | flip, E.el1, (int)(2 * e + 0)));
            WDG_TRY(set(E.el1, E.s1, (uint32_t)E.s0 | flip, E.el0, (int)(2 * e + 1)));
        }
        for (size_t e = 0; e < m.boundary.size(); ++e)
        {
            const EdgeRec &E = m.boundary[e];
            const int code = bc ? bc[e] : 0;
            if (code < 0 || code > 2)
                return fail(WDG_ERR_ARG, "boundary code must be 0 (absorbing), 1 (reflecting) or 2 (Dirichlet p=0)");
            WDG_TRY(set(E.el0, E.s0, 0x80u | ((uint32_t)code << 3), -1, (int)(2 * e)));
        }
        for (size_t k = 0; k < seen.size(); ++k)
            if (!seen[k])
                return fail(WDG_ERR_ARG, "mesh edge tables leave an element side without an edge");
        return WDG_OK;
    }

    static int face_node_host(int n, int f, int k)
    {
        const int i = (f == 0 || f == 2) ? k : (f == 1 ? n - 1 : 0);
        const int j = (f == 1 || f == 3) ? k : (f == 2 ? n - 1 : 0);
        return i + n * j;
    }

    void build_partner_tables(const FaceTables &ft, int n, std::vector<int> &fbase, std::vector<uint32_t> &fcode)
    {
        const size_t nel = ft.info.size();
        fbase.assign(4 * nel, -1);
        fcode.assign(nel, 0u);
        for (size_t el = 0; el < nel; ++el)
            for (int f = 0; f < 4; ++f)
            {
                const uint32_t byte = (ft.info[el] >> (8 * f)) & 0xffu;
                if (byte & 0x80u)
                {
                    fcode[el] |= byte << (8 * f);
                    continue;
                }
                const int nb = ft.nbr[4 * el + f], fs = (int)(byte & 3u);
                const bool flip = (byte & 4u) != 0;
                const int nn0 = face_node_host(n, fs, flip ? n - 1 : 0);
                const int nn1 = face_node_host(n, fs, flip ? n - 2 : 1);
                const int step = nn1 - nn0;
                const uint32_t code = (step == 1) ? 0u : (step == -1) ? 1u : (step == n) ? 2u : 3u;
                fbase[4 * el + f] = 3 * (nb * n * n + nn0);
                fcode[el] |= code << (8 * f);
            }
    }

    static double edge_length(const double *c, int s)
    {
        const double dx = c[2 * kSideTo[s]] - c[2 * kSideFrom[s]];
        const double dy = c[2 * kSideTo[s] + 1] - c[2 * kSideFrom[s] + 1];
        return std::hypot(dx, dy);
    }

    static void finish_mesh(wdg_mesh &m)
    {
        double h = INFINITY;
        for (const EdgeRec &E : m.interior)
            h = std::min(h, edge_length(&m.corners[8 * (size_t)E.el0], E.s0));
        for (const EdgeRec &E : m.boundary)
            h = std::min(h, edge_length(&m.corners[8 * (size_t)E.el0], E.s0));
        m.min_h = h;
    }
} // namespace wdg

using namespace wdg;

extern "C"
{
    const char *wdg_last_error(void) { return g_last_error.c_str(); }
    int wdg_version(void) { return 1; }

    int wdg_gauss_lobatto(int n, double *x, double *w, double *D)
    {
        if (n < 2 || n > 32 || !x || !w)
            return fail(WDG_ERR_ARG, "wdg_gauss_lobatto: need 2 <= n <= 32 and non-null x, w");
        gauss_lobatto(n, x, w);
        if (D)
        {
            if (n > kMaxN + 1)
                return fail(WDG_ERR_ARG, "wdg_gauss_lobatto: D only for n <= 10");
            deriv_matrix(n, x, D);
        }
        return WDG_OK;
    }

    // Edges are created in order of first appearance over (element, side);
    // the second element meeting a vertex pair closes the edge, and delta is
    // +1 iff it walks the pair in the same direction as the first element.
    int wdg_mesh_from_vertices(int n_vert, const double *xy, int n_elem, const int *quads, wdg_mesh **out)
    {
        if (!out || !xy || !quads || n_vert < 3 || n_elem < 1)
            return fail(WDG_ERR_ARG, "wdg_mesh_from_vertices: bad arguments");
        *out = nullptr;
        wdg_mesh *m = new wdg_mesh;
        m->nel = n_elem;
        m->corners.resize(8 * (size_t)n_elem);
        for (int el = 0; el < n_elem; ++el)
            for (int c = 0; c < 4; ++c)
            {
                const int v = quads[4 * (size_t)el + c];
                if (v < 0 || v >= n_vert)
                {
                    delete m;
                    return fail(WDG_ERR_ARG, "wdg_mesh_from_vertices: vertex index out of range");
                }
                m->corners[8 * (size_t)el + 2 * c] = xy[2 * (size_t)v];
                m->corners[8 * (size_t)el + 2 * c + 1] = xy[2 * (size_t)v + 1];
            }
        std::vector<EdgeRec> all;
        std::vector<uint8_t> is_int;
        all.reserve(2 * (size_t)n_elem + 64);
        std::unordered_map<int64_t, int> map;
        map.reserve(4 * (size_t)n_elem);
        for (int el = 0; el < n_elem; ++el)
            for (int s = 0; s < 4; ++s)
            {
                const int C0 = quads[4 * (size_t)el + kSideFrom[s]];
                const int C1 = quads[4 * (size_t)el + kSideTo[s]];
                const int64_t key = (int64_t)std::min(C0, C1) + (int64_t)n_vert * std::max(C0, C1);
                auto it = map.find(key);
                if (it == map.end())
                {
                    map.emplace(key, (int)all.size());
                    all.push_back({el, s, -1, -1, 1});
                    is_int.push_back(0);
                }
                else
                {
                    EdgeRec &E = all[it->second];
                    if (is_int[it->second])
                    {
                        delete m;
                        return fail(WDG_ERR_ARG, "wdg_mesh_from_vertices: edge shared by more than two elements");
                    }
                    const int first = quads[4 * (size_t)E.el0 + kSideFrom[E.s0]];
                    E.el1 = el;
                    E.s1 = s;
                    E.delta = (C0 == first) ? 1 : -1;
                    is_int[it->second] = 1;
                }
            }
        for (size_t e = 0; e < all.size(); ++e)
            (is_int[e] ? m->interior : m->boundary).push_back(all[e]);
        finish_mesh(*m);
        *out = m;
        return WDG_OK;
    }

    int wdg_mesh_uniform_rect(int nx, double ax, double bx, int ny, double ay, double by, wdg_mesh **out)
    {
        if (nx < 1 || ny < 1 || !out)
            return fail(WDG_ERR_ARG, "wdg_mesh_uniform_rect: bad arguments");
        const int np = (nx + 1) * (ny + 1);
        std::vector<double> xy(2 * (size_t)np);
        std::vector<int> q(4 * (size_t)nx * ny);
        const double dx = (bx - ax) / nx, dy = (by - ay) / ny;
        for (int j = 0; j <= ny; ++j)
            for (int i = 0; i <= nx; ++i)
            {
                xy[2 * (i + (size_t)(nx + 1) * j)] = ax + dx * i;
                xy[2 * (i + (size_t)(nx + 1) * j) + 1] = ay + dy * j;
            }
        auto l = [nx](int i, int j) { return i + (nx + 1) * j; };
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i)
            {
                int *e = &q[4 * (i + (size_t)nx * j)];
                e[0] = l(i, j);
                e[1] = l(i + 1, j);
                e[2] = l(i + 1, j + 1);
                e[3] = l(i, j + 1);
            }
        return wdg_mesh_from_vertices(np, xy.data(), nx * ny, q.data(), out);
    }

    int wdg_mesh_from_tables(int n_elem, const double *corners, int n_interior, const int *ie, int n_boundary,
                             const int *be, wdg_mesh **out)
    {
        if (!out || !corners || n_elem < 1 || n_interior < 0 || n_boundary < 0 || (n_interior && !ie) ||
            (n_boundary && !be))
            return fail(WDG_ERR_ARG, "wdg_mesh_from_tables: bad arguments");
        *out = nullptr;
        wdg_mesh *m = new wdg_mesh;
        m->nel = n_elem;
        m->corners.assign(corners, corners + 8 * (size_t)n_elem);
        for (int e = 0; e < n_interior; ++e)
            m->interior.push_back({ie[5 * e], ie[5 * e + 1], ie[5 * e + 2], ie[5 * e + 3], ie[5 * e + 4]});
        for (int e = 0; e < n_boundary; ++e)
            m->boundary.push_back({be[5 * e], be[5 * e + 1], -1, -1, 1});
        FaceTables ft; // validates the tables
        int s = build_face_tables(*m, nullptr, ft);
        if (s != WDG_OK)
        {
            delete m;
            return s;
        }
        finish_mesh(*m);
        *out = m;
        return WDG_OK;
    }

    void wdg_mesh_destroy(wdg_mesh *m) { delete m; }
    int wdg_mesh_n_elem(const wdg_mesh *m) { return m ? m->nel : fail(WDG_ERR_ARG, "null mesh"); }
    int wdg_mesh_n_edges(const wdg_mesh *m, int type)
    {
        if (!m || (type != WDG_INTERIOR && type != WDG_BOUNDARY))
            return fail(WDG_ERR_ARG, "wdg_mesh_n_edges: bad arguments");
        return (int)(type == WDG_INTERIOR ? m->interior.size() : m->boundary.size());
    }
    int wdg_mesh_edges(const wdg_mesh *m, int type, int *out)
    {
        if (!m || !out || (type != WDG_INTERIOR && type != WDG_BOUNDARY))
            return fail(WDG_ERR_ARG, "wdg_mesh_edges: bad arguments");
        const auto &L = (type == WDG_INTERIOR) ? m->interior : m->boundary;
        for (size_t e = 0; e < L.size(); ++e)
        {
            out[5 * e] = L[e].el0;
            out[5 * e + 1] = L[e].s0;
            out[5 * e + 2] = L[e].el1;
            out[5 * e + 3] = L[e].s1;
            out[5 * e + 4] = L[e].delta;
        }
        return WDG_OK;
    }
    int wdg_mesh_min_h(const wdg_mesh *m, double *h)
    {
        if (!m || !h)
            return fail(WDG_ERR_ARG, "wdg_mesh_min_h: bad arguments");
        *h = m->min_h;
        return WDG_OK;
    }
    int wdg_mesh_boundary_midpoints(const wdg_mesh *m, double *xy)
    {
        if (!m || !xy)
            return fail(WDG_ERR_ARG, "wdg_mesh_boundary_midpoints: bad arguments");
        for (size_t e = 0; e < m->boundary.size(); ++e)
        {
            const EdgeRec &E = m->boundary[e];
            const double *c = &m->corners[8 * (size_t)E.el0];
            const double x0 = c[2 * kSideFrom[E.s0]], y0 = c[2 * kSideFrom[E.s0] + 1];
            const double x1 = c[2 * kSideTo[E.s0]], y1 = c[2 * kSideTo[E.s0] + 1];
            xy[2 * e] = x0 + (x1 - x0) * 0.5;
            xy[2 * e + 1] = y0 + (y1 - y0) * 0.5;
        }
        return WDG_OK;
    }

    // Mesh2D::from_file (source/Mesh2D.cpp:94-128): <dir>/info.txt holds "n_points n_elements",
    // coordinates.txt one "x y" line per point, elements.txt four 0-based point indices per
    // element; the mesh is then built as from_vertices does.  Unlike the reference, a short
    // or unreadable file is an error rather than uninitialised data.
    int wdg_mesh_from_file(const char *dir, wdg_mesh **out)
    {
        if (!dir || !out)
            return fail(WDG_ERR_ARG, "wdg_mesh_from_file: bad arguments");
        *out = nullptr;
        const std::string d(dir);
        std::ifstream info(d + "/info.txt");
        if (!info)
            return fail(WDG_ERR_ARG, "wdg_mesh_from_file: cannot open " + d + "/info.txt");
        long long np = 0, ne = 0;
        if (!(info >> np >> ne) || np < 3 || ne < 1 || np > (1ll << 30) || ne > (1ll << 29))
            return fail(WDG_ERR_ARG, "wdg_mesh_from_file: " + d + "/info.txt must hold two positive counts");
        std::ifstream coo(d + "/coordinates.txt");
        if (!coo)
            return fail(WDG_ERR_ARG, "wdg_mesh_from_file: cannot open " + d + "/coordinates.txt");
        std::vector<double> xy(2 * (size_t)np);
        for (long long i = 0; i < 2 * np; ++i)
            if (!(coo >> xy[(size_t)i]))
                return fail(WDG_ERR_ARG, "wdg_mesh_from_file: " + d + "/coordinates.txt has fewer than " +
                                             std::to_string(np) + " points");
        std::ifstream el(d + "/elements.txt");
        if (!el)
            return fail(WDG_ERR_ARG, "wdg_mesh_from_file: cannot open " + d + "/elements.txt");
        std::vector<int> q(4 * (size_t)ne);
        for (long long i = 0; i < 4 * ne; ++i)
            if (!(el >> q[(size_t)i]))
                return fail(WDG_ERR_ARG, "wdg_mesh_from_file: " + d + "/elements.txt has fewer than " +
                                             std::to_string(ne) + " elements");
        return wdg_mesh_from_vertices((int)np, xy.data(), (int)ne, q.data(), out);
    }

    // dg::to_file (examples/examples.hpp:14-19): n doubles, raw native byte order; u on the
    // host or on a GPU
    int wdg_write_raw(const char *fname, long long n, const double *u)
    {
        if (!fname || n < 0 || (n > 0 && !u))
            return fail(WDG_ERR_ARG, "wdg_write_raw: bad arguments");
        std::vector<double> host;
        const double *src = u;
        cudaPointerAttributes at{};
        if (n > 0 && cudaPointerGetAttributes(&at, u) == cudaSuccess && at.type == cudaMemoryTypeDevice)
        {
            host.resize((size_t)n);
            WDG_CUDA(cudaMemcpy(host.data(), u, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost));
            src = host.data();
        }
        cudaGetLastError(); // a host pointer on a machine without a GPU leaves an error behind
        std::ofstream f(fname, std::ios::out | std::ios::binary);
        if (!f)
            return fail(WDG_ERR_ARG, std::string("wdg_write_raw: cannot open ") + fname);
        f.write(reinterpret_cast<const char *>(src), (std::streamsize)(sizeof(double) * (size_t)n));
        if (!f)
            return fail(WDG_ERR_ARG, std::string("wdg_write_raw: short write to ") + fname);
        return WDG_OK;
    }

    // the inverse of wdg_write_raw: exactly n doubles (a file of another size is an error)
    int wdg_read_raw(const char *fname, long long n, double *u)
    {
        if (!fname || n < 0 || (n > 0 && !u))
            return fail(WDG_ERR_ARG, "wdg_read_raw: bad arguments");
        std::ifstream f(fname, std::ios::in | std::ios::binary | std::ios::ate);
        if (!f)
            return fail(WDG_ERR_ARG, std::string("wdg_read_raw: cannot open ") + fname);
        const long long bytes = (long long)f.tellg();
        if (bytes != (long long)sizeof(double) * n)
            return fail(WDG_ERR_ARG, std::string("wdg_read_raw: ") + fname + " holds " + std::to_string(bytes) +
                                         " bytes, expected " + std::to_string(sizeof(double) * n));
        f.seekg(0);
        std::vector<double> host((size_t)n);
        f.read(reinterpret_cast<char *>(host.data()), (std::streamsize)bytes);
        if (!f)
            return fail(WDG_ERR_ARG, std::string("wdg_read_raw: short read from ") + fname);
        cudaPointerAttributes at{};
        if (n > 0 && cudaPointerGetAttributes(&at, u) == cudaSuccess && at.type == cudaMemoryTypeDevice)
            WDG_CUDA(cudaMemcpy(u, host.data(), (size_t)bytes, cudaMemcpyHostToDevice));
        else
        {
            cudaGetLastError();
            if (n > 0)
                std::memcpy(u, host.data(), (size_t)bytes);
        }
        return WDG_OK;
    }
}
