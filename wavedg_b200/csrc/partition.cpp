// Element -> rank maps for distributing one mesh over several GPUs, the two methods of
// Mesh2D::distribute (source/Mesh2D.cpp:233-382) without MPI: every rank calls the same
// deterministic host code on the global mesh and obtains the same map.
//
//   rcb  recursive coordinate bisection: a part of p ranks is cut across the principal axis of
//        its element centres into d equal-count pieces, d the smallest prime divisor of p; the
//        first piece keeps the part's rank, the others take the next new ranks in breadth-first
//        order; pieces of more than one rank are cut again (source/Mesh2D.cpp:233-294).
//   rcm  reverse Cuthill-McKee order of the edge-adjacency graph, cut into n_parts blocks of
//        consecutive elements (source/Mesh2D.cpp:312-382).
//
// The split rules, the rank numbering and the graph walk are the reference's, so that a
// decomposition has the same shape as the reference's MPI runs.  Two defects of its principal
// axis are not carried over: the mean of y is accumulated from the x coordinates
// (source/Mesh2D.cpp:194-196), and the axis divides by the covariance, which is zero for an
// axis-aligned part (:209); here the mean of y is y's, and a part with zero covariance is cut
// across its axis of larger variance.  The selection (std::nth_element) and the degree sort
// (std::sort) are the C++ library's, as in the reference's build.
#include <algorithm>
#include <cmath>
#include <queue>
#include <tuple>
#include <vector>

#include "common.hpp"

using namespace wdg;

namespace
{
    struct Centre
    {
        int id;
        double x, y, pc;
    };

    // projection of every centre of [first, last) on the first principal axis of the set
    void principal_axis(Centre *first, Centre *last)
    {
        const int n = (int)(last - first);
        double xm = 0.0, ym = 0.0;
        for (Centre *u = first; u != last; ++u)
        {
            xm += u->x;
            ym += u->y;
        }
        xm /= n;
        ym /= n;
        double vx = 0.0, vy = 0.0, cv = 0.0;
        const double inv = n > 1 ? 1.0 / (n - 1) : 1.0;
        for (Centre *u = first; u != last; ++u)
        {
            const double s = u->x - xm, t = u->y - ym;
            vx += s * s * inv;
            vy += t * t * inv;
            cv += s * t * inv;
        }
        double ex, ey;
        if (cv != 0.0)
        {
            // eigenvector of [[vx, cv], [cv, vy]] for its larger eigenvalue, scaled so ey = 1
            const double disc = std::sqrt((vx - vy) * (vx - vy) + 4.0 * cv * cv);
            ex = (disc + vx - vy) / (2.0 * cv);
            ey = 1.0;
        }
        else if (vx >= vy)
        {
            ex = 1.0;
            ey = 0.0;
        }
        else
        {
            ex = 0.0;
            ey = 1.0;
        }
        for (Centre *u = first; u != last; ++u)
            u->pc = ex * (u->x - xm) + ey * (u->y - ym);
    }

    int smallest_prime_divisor(int n)
    {
        if (n % 2 == 0)
            return 2;
        for (int k = 3; k * k <= n; k += 2)
            if (n % k == 0)
                return k;
        return n;
    }

    void rcb(const wdg_mesh &m, int nparts, int *e2p)
    {
        const int nel = m.nel;
        std::vector<Centre> a(nel);
        for (int el = 0; el < nel; ++el)
        {
            // the bilinear map at the reference-element centre: the mean of the four corners
            const double *c = m.corners.data() + 8 * (size_t)el;
            a[el] = {el, 0.25 * (c[0] + c[2] + c[4] + c[6]), 0.25 * (c[1] + c[3] + c[5] + c[7]), 0.0};
            e2p[el] = 0;
        }
        if (nparts < 2)
            return;
        std::queue<std::tuple<int, int, int>> q;
        q.push(std::make_tuple(0, nel, nparts));
        int rank = 1;
        auto by_pc = [](const Centre &u, const Centre &v) { return u.pc < v.pc; };
        while (!q.empty())
        {
            const auto [first, last, p] = q.front();
            q.pop();
            principal_axis(a.data() + first, a.data() + last);
            const int d = smallest_prime_divisor(p), next = p / d;
            std::vector<int> pos(d + 1);
            for (int k = 0; k <= d; ++k)
                pos[k] = first + (int)((long long)k * (last - first) / d);
            for (int k = 1; k < d; ++k)
                std::nth_element(a.data() + pos[k - 1], a.data() + pos[k], a.data() + last, by_pc);
            for (int k = 1; k < d; ++k, ++rank)
                for (int i = pos[k]; i < pos[k + 1]; ++i)
                    e2p[a[i].id] = rank;
            if (next > 1)
                for (int k = 0; k < d; ++k)
                    q.push(std::make_tuple(pos[k], pos[k + 1], next));
        }
    }

    int rcm(const wdg_mesh &m, int nparts, int *e2p)
    {
        const int nel = m.nel;
        std::vector<std::vector<int>> adj(nel);
        for (const EdgeRec &e : m.interior)
        {
            adj[e.el0].push_back(e.el1);
            adj[e.el1].push_back(e.el0);
        }
        int start = 0;
        for (int k = 1; k < nel; ++k)
            if (adj[k].size() < adj[start].size())
                start = k;
        std::vector<char> seen(nel, 0);
        std::vector<int> order;
        order.reserve(nel);
        std::queue<int> q;
        q.push(start);
        while (!q.empty())
        {
            const int k = q.front();
            q.pop();
            if (seen[k])
                continue;
            seen[k] = 1;
            order.push_back(k);
            std::vector<int> v = adj[k];
            std::sort(v.begin(), v.end(), [&adj](int i, int j) { return adj[i].size() < adj[j].size(); });
            for (int j : v)
                q.push(j);
        }
        if ((int)order.size() != nel)
            return fail(WDG_ERR_ARG, "wdg_mesh_partition: the mesh is not connected (reverse Cuthill-McKee reached "
                                     "only part of it)");
        // the reversed order, cut into n_parts blocks of consecutive elements
        for (int k = 0; k < nparts; ++k)
        {
            const int b = (int)((long long)k * nel / nparts), e = (int)((long long)(k + 1) * nel / nparts);
            for (int i = b; i < e; ++i)
                e2p[order[nel - 1 - i]] = k;
        }
        return WDG_OK;
    }
} // namespace

extern "C"
{
    int wdg_mesh_partition(const wdg_mesh *m, int n_parts, int method, int *e2p)
    {
        if (!m || !e2p || n_parts < 1 || n_parts > m->nel || method < 0 || method > 1)
            return fail(WDG_ERR_ARG, "wdg_mesh_partition: 1 <= n_parts <= n_elem and method 0 (rcb) or 1 (rcm)");
        if (method == 0)
        {
            rcb(*m, n_parts, e2p);
            return WDG_OK;
        }
        return rcm(*m, n_parts, e2p);
    }
}
