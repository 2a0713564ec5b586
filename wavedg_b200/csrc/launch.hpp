// Internal launch interface between the C-ABI layer (wave.cu, waveholtz.cu)
// and the kernels (kernels.cu).  Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace wdg
{
    // stage-kernel flags
    enum : int
    {
        F_VOL = 1,        // volume term  (Div<true>)
        F_INT = 2,        // interior-face flux (WaveEquation's EdgeFlux)
        F_BND = 4,        // boundary-face flux (WaveBC)
        F_MINV = 8,       // multiply by the inverse diagonal mass matrix
        F_ACCUM = 16,     // out += result (operator mode)
        F_FORCE = 32,     // + fscale * F before M^{-1}
        F_READ_DU = 64,   // RK stage > 0: du = a du + dt r (stage 0 never reads du)
        F_FILTER = 128,   // acc += acc_c * u_new  (FP64 WaveHoltz filter)
        F_RK = 256,       // shared-memory sizing only: the launch uses the RK epilogue
        F_ALL = F_VOL | F_INT | F_BND | F_MINV,
    };

    template <typename Real>
    struct StageArgs
    {
        const Real *u;        // state in
        Real *out;            // operator mode: result; RK mode: u_new (never aliases u)
        Real *du;             // RK register (RK mode)
        const Real *F;        // forcing load vector (F_FORCE)
        double *acc;          // filter accumulator (F_FILTER)
        const double *corners;
        const int4 *fbase;    // per side: DOF offset of the partner of face-node 0, -1 on the boundary
        const uint32_t *fcode;// per side: stride code | bc code << 3 | boundary << 7
        int nel;
        int flags;
        int tile;             // elements per tile (multiple of 4)
        int use_tma;          // 1: full tiles are loaded with cp.async.bulk
        int tma_out;          // 1: full tiles of u' and du' are stored with cp.async.bulk (RK mode)
        int stages;           // pipeline depth (2..4): tiles whose bulk loads are in flight + 1
        int family;           // 0: warp-per-element kernel, 1: tiled TMA-pipeline kernel,
                              // 2: warp-specialised kernel (RK launches on aligned arrays; else tiled)
        int chunk;            // family 2: elements per chunk (a multiple of 8 x elements per warp-round)
        int ring;             // family 2: chunk slots in the shared-memory ring (2..6)
        Real rk_a, rk_b, dt, fscale;
        double acc_c;
        unsigned *err;        // device error word (bit 0: wait timeout, bit 1: bad neighbour index)
        int nread;            // values of u neighbour traces may come from (0: nel * 3 n^2; a domain
                              // of a decomposed mesh appends its halo traces after its elements)
        unsigned long long wait_ns; // limit of every bounded device-side wait (0: kWaitLimitNs)
        int test_skip;        // test hook (family 2): 1 + the number of the chunk every CTA leaves
                              // unloaded, so the waits on it run out; 0 (none) in every other launch
        int el_begin, el_end; // family 2: the launch updates elements [el_begin, el_end) only
                              // (el_end 0: nel; el_begin a multiple of 4); other families: all
    };

    struct Geometry
    {
        int n = 0, nel = 0;
        const double *corners = nullptr;   // (8, nel)
        const int4 *nbr = nullptr;         // (nel)
        const uint32_t *finfo = nullptr;   // (nel)
        const int *face_edge = nullptr;    // (4, nel): 2*edge + side
        const int *edgesI = nullptr;       // (5, nI)
        const int *edgesB = nullptr;       // (5, nB)
        int nI = 0, nB = 0;
        const int *codesB = nullptr;       // (nB)
    };

    int upload_basis_tables(int device);   // once per device
    bool degree_supported(int n);
    int default_tile(int n, bool fp32, int stages);
    // the warp-specialised kernel for RK launches (operator launches take the tiled one)
    inline int default_family(int) { return 2; }
    constexpr int kDefaultStages = 3;
    int max_tile(int n);

    // warp-specialised family: chunk = 8 consumer warps x elements per warp-round x rounds
    int ws_chunk_unit(int n);                 // the smallest valid chunk
    size_t ws_smem_bytes(int n, bool fp32, int chunk, int ring);
    constexpr int kWsDefaultRing = 2;
    int ws_default_chunk(int n, bool fp32);   // most rounds (<= 4) whose default ring fits 3 CTAs per SM

    // one launch of the fused conservation-law kernels (claw_kernels.cuh)
    struct ClawArgs
    {
        const double *x;      // state the RHS is evaluated at (neighbour traces come from it)
        double *out;          // CLAW_RHS: dudt; CLAW_DIV: += volume term; RK4: u'; SSPRK3: stage result
        double *du;           // RK4 register, in place
        const double *base;   // SSPRK3 stages 1 and 2: u(t)
        const double *corners;
        const int4 *fbase;    // partner tables of the wave kernels (3 values per node): /3 gives nodes
        const uint32_t *fcode;
        const double *A;      // ClawLinear: A_0, A_1 as a(d, c, k) = A[d + nv (c + nv k)]
        const double *absA;   // ClawLinear: |n.A| per element side, (nv, nv, 4, nel)
        unsigned *err;
        int nel, mode;
        double rk_a, rk_b, dt;
    };
    enum
    {
        CLAW_RHS = 0,
        CLAW_DIV = 1,
        CLAW_RK4 = 2,
        CLAW_SSP0 = 3,
        CLAW_SSP1 = 4,
        CLAW_SSP2 = 5
    };

    // model 0: compressible Euler (n_var 4), 1: linear with constant coefficients (n_var 1..8)
    cudaError_t launch_claw(int model, int n, int nv, const ClawArgs &a, cudaStream_t s);
    cudaError_t launch_euler_face_flux(int n, int ne, const int *edges, const double *corners, const double *ub,
                                       double *fb, cudaStream_t s);

    // default limit of a bounded device-side wait (a lost copy completion; never reached otherwise)
    constexpr unsigned long long kWaitLimitNs = 2000000000ull;

    // warp-specialised stage kernels: one producer warp + kWsConsumers consumer warps per CTA
    constexpr int kWsConsumers = 4;
    // one ring slot of an n, chunk-element chunk (extra: of a launch with forcing and filter;
    // filter false: a staged launch that does not touch the filter, whose slot stops before
    // the filter accumulator's region, the slot's last)
    int ws_slot_bytes(int n, bool fp32, int chunk, bool extra = false, bool filter = true);
    int ws_warp_scratch_bytes(int n, bool fp32);    // one consumer warp's scratch

    // ---- batched WaveHoltz (kernels in stage_ws_batch.cuh, C-ABI in whbatch.cu)
    constexpr int kMaxBatch = 64;

    template <typename Real>
    struct WhbSolve
    {
        Real *buf[3]; // rotation buffers: [0] the state between steps, [1], [2]
        Real *du;
        const Real *F;
        double *acc, *W, *part;
        const double *corners;
        const int4 *fbase;
        const uint32_t *fcode;
        int nel, n, chunk, item0; // item0: the solve's first work item
        int nt;
        double dt, omega, c0;
    };

    struct WhbState
    {
        int k;      // step within the current period
        int phase;  // 0: the pi0 period of a warm start, 1: fixed-point periods
        int active; // 0 once converged, out of iterations or stalled
        int iter;   // fixed-point updates done
        int stall;  // consecutive updates without a new smallest residual
        int zero_start, nt, nparts;
        int maxit, stall_limit, status, pad; // status: 0 converged, 1 iteration limit, 2 stalled, -1 running
        double pi0sq, residual, best, tol;
        double *part;
    };

    // one launch covers the solves [s_lo, s_hi) (all of one degree) and their items [it_lo, it_hi)
    template <typename Real>
    struct WhbArgs
    {
        int nsolves, s_lo, s_hi, it_lo, it_hi, stage, ring;
        int slot_bytes, warp_scratch;
        WhbState *state;
        unsigned *err;
        WhbSolve<Real> s[kMaxBatch];
    };

    extern const double rk4a[5], rk4b[5], rk4c[5];
    int upload_rk4_tables(int device); // once per device
    int whb_smem_bytes(int n, int slot_bytes, int warp_scratch, int ring, bool fp32);
    template <typename Real>
    cudaError_t launch_whb_stage(const WhbArgs<Real> &a, int n, int grid, size_t smem, cudaStream_t s);
    template <typename Real>
    cudaError_t whb_occupancy(int n, bool last, size_t smem, int *grid); // last: the fifth stage's kernel
    cudaError_t launch_whb_step_end(WhbState *state, int nsolves, cudaStream_t s);

    // fused stage: RK = true for the time-stepping epilogue
    template <typename Real>
    cudaError_t launch_stage(int n, bool rk, const StageArgs<Real> &a, int grid_limit, cudaStream_t s);
    template <typename Real>
    size_t stage_smem_bytes(int n, int tile, int flags, int stages);

    // reference-layout component kernels (FP64)
    cudaError_t launch_prolong(const Geometry &g, int type, const double *u, double *uf, cudaStream_t s);
    cudaError_t launch_prolong_t(const Geometry &g, int type, const double *uf, double *u, cudaStream_t s);
    cudaError_t launch_edge_flux(const Geometry &g, int type, const double *ub, double *fb, cudaStream_t s);
    cudaError_t launch_apply_bc(const Geometry &g, double *uB, cudaStream_t s);
    cudaError_t launch_mass(const Geometry &g, int n_var, const double *x, double *y, bool inverse, cudaStream_t s);
    cudaError_t launch_node_coords(const Geometry &g, bool gauss_legendre, double *xy, cudaStream_t s);
    cudaError_t launch_linear_functional(const Geometry &g, int n_var, const double *fq, double *F, cudaStream_t s);
    cudaError_t launch_load_gaussians(const Geometry &g, int nsrc, const double *src /*(4, nsrc) device*/,
                                      double scale, int comp, double *F, cudaStream_t s);

    // element-wise helpers
    template <typename A, typename B>
    cudaError_t launch_convert(const A *x, B *y, long long n, cudaStream_t s);
    template <typename Real>
    cudaError_t launch_scale_into(const double *x, Real *p, double *acc, double c, long long n, cudaStream_t s);
    cudaError_t launch_wh_post(const double *W, const double *P, double omega, long long npts, double *H,
                               cudaStream_t s);

    // FP64 reductions: result written to *out (device); scratch holds >= reduce_scratch_doubles()
    int reduce_scratch_doubles();
    template <typename Real>
    cudaError_t launch_sumsq(const Real *x, const Real *y, long long n, double *scratch, double *out, cudaStream_t s);
    template <typename Real>
    cudaError_t launch_energy(const Geometry &g, const Real *u, double *scratch, double *out, cudaStream_t s);
    // WaveHoltz update: W_new = acc + pi0 (pi0 may be null); out = sum (W_new - W)^2; W <- W_new
    cudaError_t launch_wh_update(double *W, const double *acc, const double *pi0, long long n, double *scratch,
                                 double *out, cudaStream_t s);
} // namespace wdg
