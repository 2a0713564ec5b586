// Internal declarations shared by the host translation units of libwdg_b200.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "wdg_b200.h"

namespace wdg
{
    // ---- errors: thread-local message + status code -----------------------
    int fail(int code, const std::string &msg);
    int cuda_fail(cudaError_t e, const char *what);
    void clear_error();

#define WDG_CUDA(...)                                    \
    do                                                   \
    {                                                    \
        cudaError_t _e = (__VA_ARGS__);                  \
        if (_e != cudaSuccess)                           \
            return ::wdg::cuda_fail(_e, #__VA_ARGS__);   \
    } while (0)

#define WDG_TRY(...)             \
    do                           \
    {                            \
        int _s = (__VA_ARGS__);  \
        if (_s != WDG_OK)        \
            return _s;           \
    } while (0)

    constexpr int kMinN = 2;
    constexpr int kMaxN = 9;

    // ---- host mesh -----------------------------------------------------------
    // Element sides run from corner kSideFrom[s] to corner kSideTo[s]
    // (side 0: v0->v1, 1: v1->v2, 2: v3->v2, 3: v0->v3; source/Mesh2D.cpp:10-11).
    constexpr int kSideFrom[4] = {0, 1, 3, 0};
    constexpr int kSideTo[4] = {1, 2, 2, 3};

    // QuadElement::jacobian (source/Element.cpp:21-27) of the bilinear map of the corners
    // c = (x0, y0, ..., x3, y3) at (xi, eta): J = (x_xi, y_xi, x_eta, y_eta)
    __host__ __device__ inline void quad_jacobian(const double *c, double xi, double eta, double J[4])
    {
        J[0] = 0.25 * ((1.0 - eta) * (c[2] - c[0]) + (1.0 + eta) * (c[4] - c[6]));
        J[1] = 0.25 * ((1.0 - eta) * (c[3] - c[1]) + (1.0 + eta) * (c[5] - c[7]));
        J[2] = 0.25 * ((1.0 - xi) * (c[6] - c[0]) + (1.0 + xi) * (c[4] - c[2]));
        J[3] = 0.25 * ((1.0 - xi) * (c[7] - c[1]) + (1.0 + xi) * (c[5] - c[3]));
    }

    struct EdgeRec
    {
        int el0, s0, el1, s1, delta;
    };
} // namespace wdg

struct wdg_mesh
{
    int nel = 0;
    std::vector<double> corners;             // (2, 4, nel)
    std::vector<wdg::EdgeRec> interior;      // Mesh2D::edge(i, INTERIOR) order
    std::vector<wdg::EdgeRec> boundary;      // Mesh2D::edge(i, BOUNDARY) order
    double min_h = 0.0;
};

namespace wdg
{
    // GLL rule and derivative matrix for n nodes (host, double)
    void gauss_lobatto(int n, double *x, double *w);
    void deriv_matrix(int n, const double *x, double *D);
    void gauss_legendre(int n, double *x, double *w);
    void interp_matrix(int n, const double *x, int nq, const double *xq, double *B);

    // the packed per-element face table the kernels read (see wave.cu)
    struct FaceTables
    {
        std::vector<int> nbr;            // (4, nel): neighbour element or -1
        std::vector<uint32_t> info;      // (nel): byte f = side' | flip<<2 | code<<3 | boundary<<7
        std::vector<int> face_edge;      // (4, nel): edge index within its type list, or -1
    };
    int build_face_tables(const wdg_mesh &m, const int *bc, FaceTables &ft);

    // What the stage kernel reads per element side: the DOF offset of the
    // partner node that faces this side's face-node 0 (-1 on the boundary),
    // and a byte: bits 0-1 stride code (partner offset for face-node k is
    // base + k * {+3, -3, +3n, -3n}[code]), bits 3-4 boundary code, bit 7 boundary.
    void build_partner_tables(const FaceTables &ft, int n, std::vector<int> &fbase, std::vector<uint32_t> &fcode);
} // namespace wdg
