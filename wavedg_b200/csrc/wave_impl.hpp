// Internal layout of the wdg_wave handle, shared by wave.cu and waveholtz.cu.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "common.hpp"
#include "launch.hpp"

struct wdg_wave
{
    int device = 0;
    cudaStream_t stream = 0;
    int n = 0, nel = 0, precision = WDG_FP64, tile = 0, max_ctas = 0, stages = wdg::kDefaultStages;
    int family = 0; // fused-kernel family: 0 warp-per-element, 1 tiled TMA pipeline, 2 warp-specialised
    int ws_chunk = 0, ws_ring = wdg::kWsDefaultRing; // family 2 launch shape
    long long ndof = 0;
    long long halo = 0; // values of neighbour traces appended after the elements in each state
                        // buffer (a domain of a decomposed mesh; 0 otherwise)
    int nI = 0, nB = 0;
    double min_h = 0.0;

    // geometry (device)
    double *d_corners = nullptr;
    int4 *d_nbr = nullptr;
    uint32_t *d_finfo = nullptr;
    int *d_face_edge = nullptr;
    int4 *d_fbase = nullptr;
    uint32_t *d_fcode = nullptr;
    int *d_edgesI = nullptr, *d_edgesB = nullptr, *d_codes = nullptr;
    wdg::Geometry geo;

    // state buffers in the stepping precision: [0] resident state, [1], [2] rotation
    void *d_state[3] = {nullptr, nullptr, nullptr};
    void *d_du = nullptr;
    // FP64 staging for host-pointer calls (lazily allocated)
    double *d_stage[3] = {nullptr, nullptr, nullptr};
    // reductions
    double *d_scratch = nullptr;
    double *d_result = nullptr; // 8 doubles
    double *h_result = nullptr; // pinned, 8 doubles
    unsigned *d_err = nullptr;
    unsigned long long wait_ns = 0; // limit of the stage kernels' bounded waits (0: kWaitLimitNs)
    int test_skip = 0;              // test hook: 1 + chunk the next RK launch leaves unloaded
    double *d_src = nullptr;    // gaussian source table
    int src_cap = 0;

    size_t real_size() const { return precision == WDG_FP32 ? sizeof(float) : sizeof(double); }
};

namespace wdg
{
    // which memory an argument lives in
    int is_device_ptr(const wdg_wave *w, const void *p, bool &dev);
    int ensure_stage(wdg_wave *w, int k);
    int ensure_states(wdg_wave *w);
    int check_device_error(wdg_wave *w);
    int sync(wdg_wave *w);

    // Low-storage RK4 (wavedg/ode.hpp:66-93) on buffer A (stepping precision),
    // rotating A->B->C->B->C->A per step.  Optional forcing F * s(t_stage) with
    // s(t) = -sin(omega t)/omega and FP64 filter acc += c_it * u after each step.
    struct RKExtras
    {
        const void *F = nullptr;   // forcing in the stepping precision (nullable)
        double omega = 0.0;        // s(t) = -sin(omega t)/omega when F != nullptr
        double *acc = nullptr;     // FP64 filter (nullable)
        const double *c_filter = nullptr; // per-step filter weights (host array, nsteps)
    };
    template <typename Real>
    int rk4_run(wdg_wave *w, Real *A, double dt, double &t, int nsteps, const RKExtras &x);
    // stage st of the RK4 step that starts at time t; with F, forcing F * s(t + c_st dt),
    // s(t) = -sin(omega t) / omega; with acc (stage 4 only), the filter acc += acc_c * u_new
    // el_begin, el_end: update elements [el_begin, el_end) only (el_end 0: all; the
    // warp-specialised kernel only, el_begin a multiple of 4)
    template <typename Real>
    int rk4_stage(wdg_wave *w, int st, double dt, double t = 0.0, const void *F = nullptr, double omega = 0.0,
                  double *acc = nullptr, double acc_c = 0.0, int el_begin = 0, int el_end = 0);

    extern const double rk4a[5], rk4b[5], rk4c[5];

    // fused conservation-law kernels (claw.cu): launch arguments on a handle's geometry, and
    // nsteps of RK4 (method 0) or SSPRK3 (method 1) on device array u; bufs: 3 arrays of u's size
    // D(i, j) = phi_j'(xq_i) of the Lagrange basis on nodes x at points xq (barycentric, the
    // reference's lagrange_basis_deriv); the element inverse mass matrices of an exact handle
    void lagrange_deriv_at(int n, const double *x, int nq, const double *xq, double *D);
    const double *waveq_minv(const wdg_waveq *h);
    // MassMatrix<false>'s element matrices and inverses for the basis with nodes x on the
    // qm x qm Gauss-Legendre rule, (n^2, n^2, nel) each
    int exact_mass(const wdg_mesh &mesh, int n, const double *x, int qm, std::vector<double> &Mf,
                   std::vector<double> &Mi);
    // symmetric m x m (m <= kJacobiMax) eigen-decomposition by cyclic Jacobi rotations:
    // A = R diag(e) R^T, column-major
    constexpr int kJacobiMax = 8;
    void jacobi_eig(int m, const double *A, double *R, double *e);

    ClawArgs claw_args(const wdg_wave *w, const double *x, double *out);
    int claw_steps(wdg_wave *w, int model, int nv, const double *A, const double *absA, double *const *bufs, int method,
                   double *u, double dt, double *t, int nsteps);

    // An FP64 array argument of a C-ABI call: the caller's device pointer, or a staging buffer
    // filled from (and, for outputs, copied back to) the caller's host array.
    struct HostArg
    {
        const double *host_in = nullptr;
        double *host_out = nullptr;
        double *dev = nullptr;
        size_t count = 0;
    };
    // slot: which of the handle's staging buffers a host array of at most ndof values uses
    int bind_arg(wdg_wave *w, int slot, const double *p, size_t count, bool read, bool write, HostArg &a);
    // copy host outputs back, release temporaries, wait when any argument was host memory
    int finish_args(wdg_wave *w, HostArg *args, int nargs);

    // host helpers shared by the C-ABI files: make `device` current for a scope; cudaMalloc of
    // count elements (at least one) reported as a library error; upload a host vector
    struct DeviceScope
    {
        int prev = -1;
        explicit DeviceScope(int device)
        {
            cudaGetDevice(&prev);
            if (prev != device)
                cudaSetDevice(device);
        }
        ~DeviceScope()
        {
            if (prev >= 0)
                cudaSetDevice(prev);
        }
    };
    template <typename T>
    int device_alloc(T **p, size_t count)
    {
        cudaError_t e = cudaMalloc((void **)p, sizeof(T) * (count ? count : 1));
        if (e != cudaSuccess)
        {
            *p = nullptr;
            return cuda_fail(e, "cudaMalloc");
        }
        return WDG_OK;
    }
    template <typename T>
    int device_put(T *d, const std::vector<T> &h)
    {
        if (!h.empty())
        {
            cudaError_t e = cudaMemcpy(d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice);
            if (e != cudaSuccess)
                return cuda_fail(e, "cudaMemcpy");
        }
        return WDG_OK;
    }

    // exact-quadrature periods for WaveHoltz (exactq.cu)
    int waveq_prepare(wdg_waveq *q);
    int waveq_period(wdg_waveq *q, double *u, double dt, int nt, const double *F, double omega, double *acc,
                     const double *c_filter);
    int waveq_rhs_device(wdg_waveq *q, const double *u, double *dudt);
} // namespace wdg
