// C-ABI: the GPU discretisation handle, the reference-operator drop-ins and
// the fused RHS / RK4 entry points.
#include <cuda_runtime.h>

#include <string>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "wave_impl.hpp"

using namespace wdg;

namespace wdg
{
    // Carpenter-Kennedy 5-stage 2N-storage coefficients (wavedg/ode.hpp:68-70)
    const double rk4a[5] = {0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
                            -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0};
    const double rk4b[5] = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
                            1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
                            2277821191437.0 / 14882151754819.0};
    const double rk4c[5] = {0.0, 1432997174477.0 / 9575080441755.0, 2526269341429.0 / 6820363962896.0,
                            2006345519317.0 / 3224310063776.0, 2802321613138.0 / 2924317926251.0};

    int is_device_ptr(const wdg_wave *w, const void *p, bool &dev)
    {
        cudaPointerAttributes at;
        cudaError_t e = cudaPointerGetAttributes(&at, p);
        if (e != cudaSuccess)
        {
            cudaGetLastError();
            dev = false;
            return WDG_OK;
        }
        if (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged)
        {
            if (at.type == cudaMemoryTypeDevice && at.device != w->device)
                return fail(WDG_ERR_ARG, "array lives on another GPU than the discretisation");
            dev = true;
        }
        else
            dev = false;
        return WDG_OK;
    }

    int ensure_stage(wdg_wave *w, int k)
    {
        if (!w->d_stage[k])
        {
            cudaError_t e = cudaMalloc(&w->d_stage[k], sizeof(double) * (size_t)w->ndof + 64);
            if (e != cudaSuccess)
            {
                w->d_stage[k] = nullptr;
                return cuda_fail(e, "cudaMalloc(staging)");
            }
        }
        return WDG_OK;
    }

    // the three state buffers and the RK register, allocated on first use so
    // that operator-only handles (WaveEquation, WaveBC, MassMatrix drop-ins)
    // hold geometry only
    int ensure_states(wdg_wave *w)
    {
        for (int k = 0; k < 3; ++k)
            if (!w->d_state[k])
            {
                cudaError_t e = cudaMalloc(&w->d_state[k], w->real_size() * (size_t)(w->ndof + w->halo) + 64);
                if (e != cudaSuccess)
                {
                    w->d_state[k] = nullptr;
                    return cuda_fail(e, "cudaMalloc(state)");
                }
            }
        if (!w->d_du)
        {
            cudaError_t e = cudaMalloc(&w->d_du, w->real_size() * (size_t)w->ndof + 64);
            if (e != cudaSuccess)
            {
                w->d_du = nullptr;
                return cuda_fail(e, "cudaMalloc(du)");
            }
        }
        return WDG_OK;
    }

    int check_device_error(wdg_wave *w)
    {
        unsigned err = 0;
        WDG_CUDA(cudaMemcpyAsync(&err, w->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, w->stream));
        WDG_CUDA(cudaStreamSynchronize(w->stream));
        if (err)
        {
            WDG_CUDA(cudaMemsetAsync(w->d_err, 0, sizeof(unsigned), w->stream));
            if (err & 1u)
                return fail(WDG_ERR_TIMEOUT, "a bounded device-side wait expired (TMA copy did not complete)");
            return fail(WDG_ERR_ARG, "device kernel met a neighbour index outside the mesh");
        }
        return WDG_OK;
    }

    int sync(wdg_wave *w)
    {
        WDG_CUDA(cudaStreamSynchronize(w->stream));
        return check_device_error(w);
    }

    static bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

    template <typename Real>
    static StageArgs<Real> base_args(const wdg_wave *w)
    {
        StageArgs<Real> a{};
        a.corners = w->d_corners;
        a.fbase = w->d_fbase;
        a.fcode = w->d_fcode;
        a.nel = w->nel;
        a.tile = w->tile;
        a.stages = w->stages;
        a.family = w->family;
        a.chunk = w->ws_chunk;
        a.ring = w->ws_ring;
        a.err = w->d_err;
        a.nread = w->halo ? (int)(w->ndof + w->halo) : 0;
        a.wait_ns = w->wait_ns;
        return a;
    }

    template <typename Real>
    int rk4_run(wdg_wave *w, Real *A, double dt, double &t, int nsteps, const RKExtras &x)
    {
        WDG_TRY(ensure_states(w));
        Real *B = static_cast<Real *>(w->d_state[1]);
        Real *Cb = static_cast<Real *>(w->d_state[2]);
        Real *du = static_cast<Real *>(w->d_du);
        if (A == B || A == Cb)
            return fail(WDG_ERR_ARG, "rk4: state buffer aliases the rotation buffers");
        StageArgs<Real> a = base_args<Real>(w);
        a.du = du;
        a.dt = (Real)dt;
        // test hook (wdg_test_skip_chunk): the first stage launch of this call only
        a.test_skip = w->test_skip;
        w->test_skip = 0;
        for (int s = 0; s < nsteps; ++s)
        {
            const Real *src = A;
            for (int st = 0; st < 5; ++st)
            {
                Real *dst = (st == 4) ? A : ((st % 2 == 0) ? B : Cb);
                a.u = src;
                a.out = dst;
                a.flags = F_ALL | (st > 0 ? F_READ_DU : 0);
                a.rk_a = (Real)rk4a[st];
                a.rk_b = (Real)rk4b[st];
                a.use_tma = aligned16(src) ? 1 : 0;
                a.tma_out = aligned16(dst) ? 1 : 0;
                if (x.F)
                {
                    a.flags |= F_FORCE;
                    a.F = static_cast<const Real *>(x.F);
                    const double ts = t + rk4c[st] * dt;
                    a.fscale = (Real)(-1.0 / x.omega * std::sin(x.omega * ts));
                }
                if (st == 4 && x.acc)
                {
                    a.flags |= F_FILTER;
                    a.acc = x.acc;
                    a.acc_c = x.c_filter[s];
                }
                cudaError_t e = launch_stage<Real>(w->n, true, a, w->max_ctas, w->stream);
                if (e != cudaSuccess)
                    return cuda_fail(e, "stage kernel launch");
                a.test_skip = 0;
                src = dst;
            }
            t += dt;
        }
        return WDG_OK;
    }
    template int rk4_run<double>(wdg_wave *, double *, double, double &, int, const RKExtras &);
    template int rk4_run<float>(wdg_wave *, float *, double, double &, int, const RKExtras &);

    // stage st (0..4) of one RK4 step on the resident buffers, the rotation of rk4_run:
    // reads A, B, C, B, C and writes B, C, B, C, A (A = the resident state)
    template <typename Real>
    int rk4_stage(wdg_wave *w, int st, double dt, double t, const void *F, double omega, double *acc, double acc_c,
                  int el_begin, int el_end)
    {
        WDG_TRY(ensure_states(w));
        Real *buf[3] = {static_cast<Real *>(w->d_state[0]), static_cast<Real *>(w->d_state[1]),
                        static_cast<Real *>(w->d_state[2])};
        static const int src_of[5] = {0, 1, 2, 1, 2}, dst_of[5] = {1, 2, 1, 2, 0};
        StageArgs<Real> a = base_args<Real>(w);
        a.du = static_cast<Real *>(w->d_du);
        a.dt = (Real)dt;
        a.u = buf[src_of[st]];
        a.out = buf[dst_of[st]];
        a.flags = F_ALL | (st > 0 ? F_READ_DU : 0);
        a.rk_a = (Real)rk4a[st];
        a.rk_b = (Real)rk4b[st];
        a.use_tma = aligned16(a.u) ? 1 : 0;
        a.tma_out = aligned16(a.out) ? 1 : 0;
        if (F)
        {
            a.flags |= F_FORCE;
            a.F = static_cast<const Real *>(F);
            a.fscale = (Real)(-1.0 / omega * std::sin(omega * (t + rk4c[st] * dt)));
        }
        if (st == 4 && acc)
        {
            a.flags |= F_FILTER;
            a.acc = acc;
            a.acc_c = acc_c;
        }
        a.el_begin = el_begin;
        a.el_end = el_end;
        cudaError_t e = launch_stage<Real>(w->n, true, a, w->max_ctas, w->stream);
        if (e == cudaErrorNotSupported)
            return fail(WDG_ERR_UNSUPPORTED, "rk4 stage over part of the elements: needs the warp-specialised kernel "
                                             "(wdg_wave_set_kernel 2) with its chunk and ring fitting shared memory");
        if (e != cudaSuccess)
            return cuda_fail(e, "stage kernel launch");
        return WDG_OK;
    }
    template int rk4_stage<double>(wdg_wave *, int, double, double, const void *, double, double *, double, int, int);
    template int rk4_stage<float>(wdg_wave *, int, double, double, const void *, double, double *, double, int, int);
} // namespace wdg

namespace
{
    template <typename T>
    int dalloc(T **p, size_t count)
    {
        cudaError_t e = cudaMalloc((void **)p, sizeof(T) * std::max<size_t>(count, 1));
        if (e != cudaSuccess)
        {
            *p = nullptr;
            return cuda_fail(e, "cudaMalloc");
        }
        return WDG_OK;
    }
    template <typename T>
    int upload(T *d, const T *h, size_t count)
    {
        if (count)
            WDG_CUDA(cudaMemcpy(d, h, sizeof(T) * count, cudaMemcpyHostToDevice));
        return WDG_OK;
    }

    constexpr size_t kMaxSmem = 227 * 1024;
    size_t smem_for(const wdg_wave *w, int tile, int stages)
    {
        return w->precision == WDG_FP32 ? stage_smem_bytes<float>(w->n, tile, F_RK, stages)
                                        : stage_smem_bytes<double>(w->n, tile, F_RK, stages);
    }

    struct DeviceGuard
    {
        int prev = -1;
        explicit DeviceGuard(int dev)
        {
            cudaGetDevice(&prev);
            if (prev != dev)
                cudaSetDevice(dev);
        }
        ~DeviceGuard()
        {
            if (prev >= 0)
                cudaSetDevice(prev);
        }
    };

    using Arg = wdg::HostArg;

    int bind(wdg_wave *w, int slot, const double *p, size_t count, bool read, bool write, Arg &a)
    {
        if (!p)
            return fail(WDG_ERR_ARG, "null array argument");
        bool dev = false;
        WDG_TRY(is_device_ptr(w, p, dev));
        a.count = count;
        if (dev)
        {
            a.dev = const_cast<double *>(p);
            return WDG_OK;
        }
        if (count > (size_t)w->ndof)
        {
            // larger than a state vector (face traces): use a temporary
            WDG_CUDA(cudaMallocAsync((void **)&a.dev, sizeof(double) * count, w->stream));
            a.host_out = write ? const_cast<double *>(p) : nullptr;
            a.host_in = p;
            if (read)
                WDG_CUDA(cudaMemcpyAsync(a.dev, p, sizeof(double) * count, cudaMemcpyHostToDevice, w->stream));
            a.count = count | (size_t(1) << 62); // mark as temporary
            return WDG_OK;
        }
        WDG_TRY(ensure_stage(w, slot));
        a.dev = w->d_stage[slot];
        a.host_in = p;
        a.host_out = write ? const_cast<double *>(p) : nullptr;
        if (read)
            WDG_CUDA(cudaMemcpyAsync(a.dev, p, sizeof(double) * count, cudaMemcpyHostToDevice, w->stream));
        return WDG_OK;
    }

    // copy host outputs back, release temporaries, and wait when any argument was host memory
    int finish(wdg_wave *w, Arg *args, int nargs)
    {
        bool any_host = false;
        for (int k = 0; k < nargs; ++k)
        {
            Arg &a = args[k];
            const bool temp = (a.count >> 62) & 1;
            const size_t cnt = a.count & ~(size_t(3) << 62);
            if (a.host_out)
                WDG_CUDA(cudaMemcpyAsync(a.host_out, a.dev, sizeof(double) * cnt, cudaMemcpyDeviceToHost, w->stream));
            if (a.host_in || a.host_out)
                any_host = true;
            if (temp)
                WDG_CUDA(cudaFreeAsync(a.dev, w->stream));
        }
        if (any_host)
            return sync(w);
        return WDG_OK;
    }

    int launch_op(wdg_wave *w, const double *u, double *out, int flags, const double *F, double s)
    {
        StageArgs<double> a = base_args<double>(w);
        // operator launches always run the FP64 kernel, whatever the stepping precision
        a.tile = default_tile(w->n, false, kDefaultStages);
        a.stages = kDefaultStages;
        a.family = w->family;
        a.u = u;
        a.out = out;
        a.flags = flags;
        a.F = F;
        a.fscale = s;
        a.use_tma = ((uintptr_t)u & 15u) == 0;
        a.tma_out = 0;
        cudaError_t e = launch_stage<double>(w->n, false, a, w->max_ctas, w->stream);
        if (e != cudaSuccess)
            return cuda_fail(e, "stage kernel launch (operator mode)");
        return WDG_OK;
    }

    // a domain of a decomposed mesh (halo traces) only steps stage by stage, with its halo
    // filled by the caller; whole-operator and whole-step calls would treat its cut sides as
    // boundary sides
    int whole_mesh_only(const wdg_wave *w, const char *what)
    {
        if (w && w->halo)
            return fail(WDG_ERR_UNSUPPORTED, std::string(what) +
                                                 ": not available on a domain of a decomposed mesh (use wdg_rk4_stage)");
        return WDG_OK;
    }

    int op_entry(wdg_wave *w, const double *u, double *du, int flags)
    {
        if (!w)
            return fail(WDG_ERR_ARG, "null discretisation");
        WDG_TRY(whole_mesh_only(w, "operator action"));
        DeviceGuard g(w->device);
        if (u == du)
            return fail(WDG_ERR_ARG, "input and output arrays must differ");
        Arg a[2];
        WDG_TRY(bind(w, 0, u, w->ndof, true, false, a[0]));
        WDG_TRY(bind(w, 1, du, w->ndof, true, true, a[1]));
        WDG_TRY(launch_op(w, a[0].dev, a[1].dev, flags | F_ACCUM, nullptr, 0.0));
        return finish(w, a, 2);
    }

    size_t face_count(const wdg_wave *w, int type) { return (size_t)w->n * 3 * 2 * (type == 0 ? w->nI : w->nB); }

    template <typename Real>
    int upload_state(wdg_wave *w, const double *u)
    {
        WDG_TRY(ensure_states(w));
        bool dev = false;
        WDG_TRY(is_device_ptr(w, u, dev));
        const double *src = u;
        if (!dev)
        {
            WDG_TRY(ensure_stage(w, 0));
            WDG_CUDA(cudaMemcpyAsync(w->d_stage[0], u, sizeof(double) * w->ndof, cudaMemcpyHostToDevice, w->stream));
            src = w->d_stage[0];
        }
        WDG_CUDA(launch_convert<double, Real>(src, static_cast<Real *>(w->d_state[0]), w->ndof, w->stream));
        if (!dev)
            return sync(w);
        return WDG_OK;
    }

    template <typename Real>
    int download_state(wdg_wave *w, double *u)
    {
        WDG_TRY(ensure_states(w));
        bool dev = false;
        WDG_TRY(is_device_ptr(w, u, dev));
        double *dst = u;
        if (!dev)
        {
            WDG_TRY(ensure_stage(w, 0));
            dst = w->d_stage[0];
        }
        WDG_CUDA(launch_convert<Real, double>(static_cast<const Real *>(w->d_state[0]), dst, w->ndof, w->stream));
        if (!dev)
        {
            WDG_CUDA(cudaMemcpyAsync(u, dst, sizeof(double) * w->ndof, cudaMemcpyDeviceToHost, w->stream));
            return sync(w);
        }
        return WDG_OK;
    }
} // namespace

namespace wdg
{
    int bind_arg(wdg_wave *w, int slot, const double *p, size_t count, bool read, bool write, HostArg &a)
    {
        return bind(w, slot, p, count, read, write, a);
    }
    int finish_args(wdg_wave *w, HostArg *args, int nargs) { return finish(w, args, nargs); }
} // namespace wdg

extern "C"
{
    int wdg_supported_degrees(int *n_colloc, int cap)
    {
        int c = 0;
        for (int n = kMinN; n <= kMaxN; ++n)
            if (degree_supported(n))
            {
                if (n_colloc && c < cap)
                    n_colloc[c] = n;
                ++c;
            }
        return c;
    }

    int wdg_wave_create(const wdg_mesh *mesh, int n_colloc, const int *bc, int precision, int device, wdg_wave **out)
    {
        if (!mesh || !out)
            return fail(WDG_ERR_ARG, "wdg_wave_create: null argument");
        *out = nullptr;
        if (!degree_supported(n_colloc))
            return fail(WDG_ERR_UNSUPPORTED, "wdg_wave_create: no kernels for this n_colloc (built: 2..9)");
        if (precision != WDG_FP64 && precision != WDG_FP32)
            return fail(WDG_ERR_ARG, "wdg_wave_create: precision must be WDG_FP64 or WDG_FP32");
        if (3LL * n_colloc * n_colloc * mesh->nel >= (1LL << 31))
            return fail(WDG_ERR_UNSUPPORTED, "wdg_wave_create: more than 2^31 DOF on one GPU");
        int ndev = 0;
        WDG_CUDA(cudaGetDeviceCount(&ndev));
        if (device < 0)
            WDG_CUDA(cudaGetDevice(&device));
        if (device >= ndev)
            return fail(WDG_ERR_ARG, "wdg_wave_create: no such device");
        DeviceGuard guard(device);
        WDG_TRY(upload_basis_tables(device));

        FaceTables ft;
        WDG_TRY(build_face_tables(*mesh, bc, ft));

        wdg_wave *w = new wdg_wave;
        w->device = device;
        w->n = n_colloc;
        w->nel = mesh->nel;
        w->precision = precision;
        w->ndof = 3LL * n_colloc * n_colloc * mesh->nel;
        w->nI = (int)mesh->interior.size();
        w->nB = (int)mesh->boundary.size();
        w->min_h = mesh->min_h;
        w->tile = default_tile(n_colloc, precision == WDG_FP32, w->stages);
        w->family = default_family(n_colloc);
        w->ws_chunk = ws_default_chunk(n_colloc, precision == WDG_FP32);

        int s = WDG_OK;
        auto chk = [&](int r)
        {
            if (s == WDG_OK)
                s = r;
        };
        const size_t nel = mesh->nel;
        chk(dalloc(&w->d_corners, 8 * nel));
        chk(dalloc(&w->d_nbr, nel));
        chk(dalloc(&w->d_finfo, nel));
        chk(dalloc(&w->d_face_edge, 4 * nel));
        chk(dalloc(&w->d_fbase, nel));
        chk(dalloc(&w->d_fcode, nel));
        chk(dalloc(&w->d_edgesI, 5 * (size_t)w->nI));
        chk(dalloc(&w->d_edgesB, 5 * (size_t)w->nB));
        chk(dalloc(&w->d_codes, (size_t)w->nB));
        chk(dalloc(&w->d_scratch, (size_t)reduce_scratch_doubles()));
        chk(dalloc(&w->d_result, 8));
        chk(dalloc(&w->d_err, 1));
        if (s == WDG_OK)
        {
            cudaError_t e = cudaMallocHost(&w->h_result, 8 * sizeof(double));
            if (e != cudaSuccess)
                chk(cuda_fail(e, "cudaMallocHost"));
        }
        if (s == WDG_OK)
        {
            std::vector<int> ei(5 * (size_t)w->nI), eb(5 * (size_t)w->nB), codes(w->nB);
            for (int e = 0; e < w->nI; ++e)
            {
                const EdgeRec &E = mesh->interior[e];
                int *r = &ei[5 * (size_t)e];
                r[0] = E.el0; r[1] = E.s0; r[2] = E.el1; r[3] = E.s1; r[4] = E.delta;
            }
            for (int e = 0; e < w->nB; ++e)
            {
                const EdgeRec &E = mesh->boundary[e];
                int *r = &eb[5 * (size_t)e];
                r[0] = E.el0; r[1] = E.s0; r[2] = -1; r[3] = -1; r[4] = 1;
                codes[e] = bc ? bc[e] : 0;
            }
            std::vector<int4> nb4(nel);
            for (size_t el = 0; el < nel; ++el)
                nb4[el] = make_int4(ft.nbr[4 * el], ft.nbr[4 * el + 1], ft.nbr[4 * el + 2], ft.nbr[4 * el + 3]);
            chk(upload(w->d_corners, mesh->corners.data(), 8 * nel));
            chk(upload(w->d_nbr, nb4.data(), nel));
            chk(upload(w->d_finfo, ft.info.data(), nel));
            chk(upload(w->d_face_edge, ft.face_edge.data(), 4 * nel));
            std::vector<int> fbase;
            std::vector<uint32_t> fcode;
            build_partner_tables(ft, n_colloc, fbase, fcode);
            chk(upload(reinterpret_cast<int *>(w->d_fbase), fbase.data(), 4 * nel));
            chk(upload(w->d_fcode, fcode.data(), nel));
            chk(upload(w->d_edgesI, ei.data(), ei.size()));
            chk(upload(w->d_edgesB, eb.data(), eb.size()));
            chk(upload(w->d_codes, codes.data(), codes.size()));
            if (s == WDG_OK)
            {
                cudaError_t e = cudaMemset(w->d_err, 0, sizeof(unsigned));
                if (e != cudaSuccess)
                    chk(cuda_fail(e, "cudaMemset"));
            }
        }
        Geometry &g = w->geo;
        g.n = w->n;
        g.nel = w->nel;
        g.corners = w->d_corners;
        g.nbr = w->d_nbr;
        g.finfo = w->d_finfo;
        g.face_edge = w->d_face_edge;
        g.edgesI = w->d_edgesI;
        g.edgesB = w->d_edgesB;
        g.nI = w->nI;
        g.nB = w->nB;
        g.codesB = w->d_codes;
        if (s != WDG_OK)
        {
            const std::string msg = wdg_last_error();
            wdg_wave_destroy(w);
            return fail(s, msg);
        }
        *out = w;
        return WDG_OK;
    }

    void wdg_wave_destroy(wdg_wave *w)
    {
        if (!w)
            return;
        DeviceGuard g(w->device);
        cudaStreamSynchronize(w->stream);
        void *ptrs[] = {w->d_corners, w->d_nbr, w->d_finfo, w->d_face_edge, w->d_fbase, w->d_fcode, w->d_edgesI,
                        w->d_edgesB, w->d_codes,
                        w->d_state[0], w->d_state[1], w->d_state[2], w->d_du, w->d_stage[0], w->d_stage[1],
                        w->d_stage[2], w->d_scratch, w->d_result, w->d_err, w->d_src};
        for (void *p : ptrs)
            if (p)
                cudaFree(p);
        if (w->h_result)
            cudaFreeHost(w->h_result);
        delete w;
    }

    int wdg_wave_info(const wdg_wave *w, int *n, int *nel, long long *ndof, int *precision)
    {
        if (!w)
            return fail(WDG_ERR_ARG, "null discretisation");
        if (n) *n = w->n;
        if (nel) *nel = w->nel;
        if (ndof) *ndof = w->ndof;
        if (precision) *precision = w->precision;
        return WDG_OK;
    }

    int wdg_wave_set_stream(wdg_wave *w, void *stream)
    {
        if (!w)
            return fail(WDG_ERR_ARG, "null discretisation");
        w->stream = static_cast<cudaStream_t>(stream);
        return WDG_OK;
    }

    int wdg_wave_sync(wdg_wave *w)
    {
        if (!w)
            return fail(WDG_ERR_ARG, "null discretisation");
        DeviceGuard g(w->device);
        return sync(w);
    }

    static int ws_set(wdg_wave *w, int chunk, int ring)
    {
        const bool fp32 = w->precision == WDG_FP32;
        if (chunk == 0)
            chunk = ws_default_chunk(w->n, fp32);
        if (ring == 0)
            ring = kWsDefaultRing;
        const int unit = ws_chunk_unit(w->n);
        if (chunk < unit || chunk % unit || chunk > 64 * unit)
            return fail(WDG_ERR_ARG, "warp-specialised kernel: the chunk must be a multiple of 8 warps x elements per warp");
        if (ring < 2 || ring > 6)
            return fail(WDG_ERR_ARG, "warp-specialised kernel: the ring holds 2 to 6 chunks");
        if (ws_smem_bytes(w->n, fp32, chunk, ring) > kMaxSmem)
            return fail(WDG_ERR_ARG, "warp-specialised kernel: chunk x ring too large for shared memory");
        w->ws_chunk = chunk;
        w->ws_ring = ring;
        return WDG_OK;
    }

    int wdg_wave_set_tile(wdg_wave *w, int tile)
    {
        if (!w)
            return fail(WDG_ERR_ARG, "null discretisation");
        if (w->family == 2)
            return ws_set(w, tile, w->ws_ring);
        if (tile == 0)
            tile = default_tile(w->n, w->precision == WDG_FP32, w->stages);
        if (tile < 4 || (tile & 3) || tile > max_tile(w->n))
            return fail(WDG_ERR_ARG, "tile must be a positive multiple of 4 with (3 n + 8) * tile <= 512 threads");
        if (smem_for(w, tile, w->stages) > kMaxSmem)
            return fail(WDG_ERR_ARG, "tile too large for shared memory at this pipeline depth");
        w->tile = tile;
        return WDG_OK;
    }
    int wdg_wave_set_stages(wdg_wave *w, int stages)
    {
        if (w && w->family == 2)
        {
            if (stages < 0 || stages == 1 || stages > 6)
                return fail(WDG_ERR_ARG, "wdg_wave_set_stages: the ring holds 2 to 6 chunks (0 = default)");
            int chunk = w->ws_chunk;
            const int unit = ws_chunk_unit(w->n), ring = stages ? stages : kWsDefaultRing;
            while (chunk > unit && ws_smem_bytes(w->n, w->precision == WDG_FP32, chunk, ring) > kMaxSmem)
                chunk -= unit;
            return ws_set(w, chunk, ring);
        }
        if (!w || stages < 0 || stages == 1 || stages > 4)
            return fail(WDG_ERR_ARG, "wdg_wave_set_stages: stages must be 2, 3 or 4 (0 = default)");
        if (stages == 0)
            stages = kDefaultStages;
        int tile = w->tile;
        while (tile > 4 && smem_for(w, tile, stages) > kMaxSmem)
            tile -= 4;
        if (smem_for(w, tile, stages) > kMaxSmem)
            return fail(WDG_ERR_ARG, "wdg_wave_set_stages: no tile fits shared memory at this depth");
        w->stages = stages;
        w->tile = tile;
        return WDG_OK;
    }

    int wdg_wave_set_wait_limit(wdg_wave *w, double seconds)
    {
        if (!w || !(seconds > 0.0) || seconds > 60.0)
            return fail(WDG_ERR_ARG, "wdg_wave_set_wait_limit: the limit must be in (0, 60] seconds");
        w->wait_ns = std::max(1ull, (unsigned long long)(seconds * 1e9));
        return WDG_OK;
    }

    int wdg_test_skip_chunk(wdg_wave *w, int chunk)
    {
        if (!w || chunk < -1)
            return fail(WDG_ERR_ARG, "wdg_test_skip_chunk: chunk must be >= 0 (or -1: none)");
        w->test_skip = chunk + 1;
        return WDG_OK;
    }

    int wdg_test_set_partner(wdg_wave *w, int elem, int side, int offset, int *previous)
    {
        if (!w || elem < 0 || elem >= w->nel || side < 0 || side > 3)
            return fail(WDG_ERR_ARG, "wdg_test_set_partner: element or side out of range");
        DeviceGuard g(w->device);
        int *p = reinterpret_cast<int *>(w->d_fbase + elem) + side;
        int old = 0;
        WDG_CUDA(cudaMemcpyAsync(&old, p, sizeof(int), cudaMemcpyDeviceToHost, w->stream));
        WDG_CUDA(cudaStreamSynchronize(w->stream));
        WDG_CUDA(cudaMemcpyAsync(p, &offset, sizeof(int), cudaMemcpyHostToDevice, w->stream));
        WDG_CUDA(cudaStreamSynchronize(w->stream));
        if (previous)
            *previous = old;
        return WDG_OK;
    }

    int wdg_wave_set_kernel(wdg_wave *w, int family)
    {
        if (!w || family < -1 || family > 2)
            return fail(WDG_ERR_ARG,
                        "wdg_wave_set_kernel: 0 (warp per element), 1 (tiled), 2 (warp-specialised) or -1 (default)");
        w->family = (family < 0) ? default_family(w->n) : family;
        return WDG_OK;
    }

    int wdg_wave_get_launch(const wdg_wave *w, int *family, int *tile, int *stages, int *max_ctas)
    {
        if (!w)
            return fail(WDG_ERR_ARG, "null discretisation");
        if (family) *family = w->family;
        if (tile) *tile = (w->family == 2) ? w->ws_chunk : w->tile;
        if (stages) *stages = (w->family == 2) ? w->ws_ring : w->stages;
        if (max_ctas) *max_ctas = w->max_ctas;
        return WDG_OK;
    }

    // Time `steps` RK4 steps of every (tile, stages) candidate on the resident
    // state with dt = 0 (state unchanged, traffic identical) and keep the fastest.
    int wdg_wave_autotune(wdg_wave *w, int steps, float *best_ms_per_step)
    {
        if (!w || steps < 1)
            return fail(WDG_ERR_ARG, "wdg_wave_autotune: bad arguments");
        DeviceGuard g(w->device);
        WDG_TRY(ensure_states(w));
        cudaEvent_t e0, e1;
        WDG_CUDA(cudaEventCreate(&e0));
        WDG_CUDA(cudaEventCreate(&e1));
        const int save_tile = w->tile, save_stages = w->stages, save_family = w->family;
        const int save_chunk = w->ws_chunk, save_ring = w->ws_ring;
        float best = 1e30f;
        int bt = save_tile, bs = save_stages, bf = save_family, bc = save_chunk, br = save_ring, s = WDG_OK;
        RKExtras none;
        // candidates: the warp-per-element kernel; every fitting tiled (tile, depth); every
        // warp-specialised (chunk of 1..4 rounds, ring of 2..6) that fits shared memory
        struct Cand
        {
            int family, a, b;
        };
        std::vector<Cand> cands;
        cands.push_back({0, save_tile, save_stages});
        for (int st = 2; st <= 4; ++st)
            for (int tile = 4; tile <= max_tile(w->n); tile += 4)
                if (smem_for(w, tile, st) <= kMaxSmem)
                    cands.push_back({1, tile, st});
        for (int r = 1; r <= 4; ++r)
            for (int ring = 2; ring <= 6; ++ring)
                if (ws_smem_bytes(w->n, w->precision == WDG_FP32, r * ws_chunk_unit(w->n), ring) <= kMaxSmem)
                    cands.push_back({2, r * ws_chunk_unit(w->n), ring});
        for (size_t ci = 0; ci < cands.size() && s == WDG_OK; ++ci)
            {
                const Cand &cd = cands[ci];
                w->family = cd.family;
                w->tile = (cd.family == 1) ? cd.a : save_tile;
                w->stages = (cd.family == 1) ? cd.b : save_stages;
                w->ws_chunk = (cd.family == 2) ? cd.a : save_chunk;
                w->ws_ring = (cd.family == 2) ? cd.b : save_ring;
                double t = 0.0;
                auto run = [&](int n) -> int
                {
                    return w->precision == WDG_FP64
                               ? rk4_run<double>(w, static_cast<double *>(w->d_state[0]), 0.0, t, n, none)
                               : rk4_run<float>(w, static_cast<float *>(w->d_state[0]), 0.0, t, n, none);
                };
                s = run(1);
                if (s != WDG_OK)
                    break;
                if (cudaEventRecord(e0, w->stream) != cudaSuccess)
                {
                    s = cuda_fail(cudaGetLastError(), "cudaEventRecord");
                    break;
                }
                s = run(steps);
                if (s != WDG_OK)
                    break;
                cudaEventRecord(e1, w->stream);
                cudaEventSynchronize(e1);
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                ms /= steps;
                if (ms < best)
                {
                    best = ms;
                    bt = w->tile;
                    bs = w->stages;
                    bf = w->family;
                    bc = w->ws_chunk;
                    br = w->ws_ring;
                }
            }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        w->tile = (s == WDG_OK) ? bt : save_tile;
        w->stages = (s == WDG_OK) ? bs : save_stages;
        w->family = (s == WDG_OK) ? bf : save_family;
        w->ws_chunk = (s == WDG_OK) ? bc : save_chunk;
        w->ws_ring = (s == WDG_OK) ? br : save_ring;
        if (s == WDG_OK)
            s = sync(w);
        if (best_ms_per_step)
            *best_ms_per_step = best;
        return s;
    }

    int wdg_wave_set_max_ctas(wdg_wave *w, int max_ctas)
    {
        if (!w || max_ctas < 0)
            return fail(WDG_ERR_ARG, "wdg_wave_set_max_ctas: bad arguments");
        w->max_ctas = max_ctas;
        return WDG_OK;
    }

    int wdg_wave_get_tile(const wdg_wave *w, int *tile)
    {
        if (!w || !tile)
            return fail(WDG_ERR_ARG, "null argument");
        *tile = (w->family == 2) ? w->ws_chunk : w->tile;
        return WDG_OK;
    }

    int wdg_wave_node_coords(wdg_wave *w, double *xy)
    {
        if (!w)
            return fail(WDG_ERR_ARG, "null discretisation");
        DeviceGuard g(w->device);
        const size_t cnt = 2 * (size_t)w->n * w->n * w->nel;
        Arg a;
        WDG_TRY(bind(w, 0, xy, cnt, false, true, a));
        WDG_CUDA(launch_node_coords(w->geo, false, a.dev, w->stream));
        return finish(w, &a, 1);
    }

    int wdg_quad_points(wdg_wave *w, double *xy)
    {
        if (!w)
            return fail(WDG_ERR_ARG, "null discretisation");
        DeviceGuard g(w->device);
        const size_t cnt = 2 * (size_t)w->n * w->n * w->nel;
        Arg a;
        WDG_TRY(bind(w, 0, xy, cnt, false, true, a));
        WDG_CUDA(launch_node_coords(w->geo, true, a.dev, w->stream));
        return finish(w, &a, 1);
    }

    int wdg_div_action(wdg_wave *w, const double *u, double *du) { return op_entry(w, u, du, F_VOL); }
    int wdg_wave_action(wdg_wave *w, const double *u, double *du) { return op_entry(w, u, du, F_VOL | F_INT); }
    int wdg_wavebc_action(wdg_wave *w, const double *u, double *du) { return op_entry(w, u, du, F_BND); }

    int wdg_face_prolong(wdg_wave *w, int type, const double *u, double *uf)
    {
        WDG_TRY(whole_mesh_only(w, "wdg_face_prolong"));
        if (!w || (type != 0 && type != 1))
            return fail(WDG_ERR_ARG, "wdg_face_prolong: bad arguments");
        DeviceGuard g(w->device);
        Arg a[2];
        WDG_TRY(bind(w, 0, u, w->ndof, true, false, a[0]));
        WDG_TRY(bind(w, 1, uf, face_count(w, type), false, true, a[1]));
        WDG_CUDA(launch_prolong(w->geo, type, a[0].dev, a[1].dev, w->stream));
        return finish(w, a, 2);
    }

    int wdg_face_prolong_t(wdg_wave *w, int type, const double *uf, double *u)
    {
        WDG_TRY(whole_mesh_only(w, "wdg_face_prolong_t"));
        if (!w || (type != 0 && type != 1))
            return fail(WDG_ERR_ARG, "wdg_face_prolong_t: bad arguments");
        DeviceGuard g(w->device);
        Arg a[2];
        WDG_TRY(bind(w, 0, uf, face_count(w, type), true, false, a[0]));
        WDG_TRY(bind(w, 1, u, w->ndof, true, true, a[1]));
        WDG_CUDA(launch_prolong_t(w->geo, type, a[0].dev, a[1].dev, w->stream));
        return finish(w, a, 2);
    }

    int wdg_edge_flux(wdg_wave *w, int type, const double *ub, double *fb)
    {
        WDG_TRY(whole_mesh_only(w, "wdg_edge_flux"));
        if (!w || (type != 0 && type != 1))
            return fail(WDG_ERR_ARG, "wdg_edge_flux: bad arguments");
        DeviceGuard g(w->device);
        const size_t cnt = face_count(w, type);
        Arg a[2];
        if (ub == fb)
        {
            WDG_TRY(bind(w, 0, ub, cnt, true, true, a[0]));
            WDG_CUDA(launch_edge_flux(w->geo, type, a[0].dev, a[0].dev, w->stream));
            return finish(w, a, 1);
        }
        WDG_TRY(bind(w, 0, ub, cnt, true, false, a[0]));
        WDG_TRY(bind(w, 1, fb, cnt, false, true, a[1]));
        WDG_CUDA(launch_edge_flux(w->geo, type, a[0].dev, a[1].dev, w->stream));
        return finish(w, a, 2);
    }

    int wdg_apply_bc(wdg_wave *w, double *uB)
    {
        WDG_TRY(whole_mesh_only(w, "wdg_apply_bc"));
        if (!w)
            return fail(WDG_ERR_ARG, "null discretisation");
        DeviceGuard g(w->device);
        Arg a;
        WDG_TRY(bind(w, 0, uB, face_count(w, 1), true, true, a));
        WDG_CUDA(launch_apply_bc(w->geo, a.dev, w->stream));
        return finish(w, &a, 1);
    }

    int wdg_mass_action(wdg_wave *w, int n_var, const double *x, double *y)
    {
        if (!w || n_var < 1 || n_var > 16)
            return fail(WDG_ERR_ARG, "wdg_mass_action: bad arguments");
        DeviceGuard g(w->device);
        const size_t cnt = (size_t)n_var * w->n * w->n * w->nel;
        Arg a[2];
        WDG_TRY(bind(w, 0, x, cnt, true, false, a[0]));
        WDG_TRY(bind(w, 1, y, cnt, false, true, a[1]));
        WDG_CUDA(launch_mass(w->geo, n_var, a[0].dev, a[1].dev, false, w->stream));
        return finish(w, a, 2);
    }

    int wdg_mass_inv(wdg_wave *w, int n_var, double *x)
    {
        if (!w || n_var < 1 || n_var > 16)
            return fail(WDG_ERR_ARG, "wdg_mass_inv: bad arguments");
        DeviceGuard g(w->device);
        const size_t cnt = (size_t)n_var * w->n * w->n * w->nel;
        Arg a;
        WDG_TRY(bind(w, 0, x, cnt, true, true, a));
        WDG_CUDA(launch_mass(w->geo, n_var, a.dev, a.dev, true, w->stream));
        return finish(w, &a, 1);
    }

    int wdg_rhs(wdg_wave *w, const double *u, double *dudt, const double *F, double s)
    {
        WDG_TRY(whole_mesh_only(w, "wdg_rhs"));
        if (!w)
            return fail(WDG_ERR_ARG, "null discretisation");
        if (u == dudt)
            return fail(WDG_ERR_ARG, "wdg_rhs: input and output arrays must differ");
        DeviceGuard g(w->device);
        Arg a[3];
        WDG_TRY(bind(w, 0, u, w->ndof, true, false, a[0]));
        WDG_TRY(bind(w, 1, dudt, w->ndof, false, true, a[1]));
        int nargs = 2;
        if (F)
        {
            WDG_TRY(bind(w, 2, F, w->ndof, true, false, a[2]));
            nargs = 3;
        }
        WDG_TRY(launch_op(w, a[0].dev, a[1].dev, F_ALL | (F ? F_FORCE : 0), F ? a[2].dev : nullptr, s));
        return finish(w, a, nargs);
    }

    int wdg_rk4_steps(wdg_wave *w, double *u, double dt, double *t, int nsteps)
    {
        WDG_TRY(whole_mesh_only(w, "wdg_rk4_steps"));
        if (!w || !u || !t || nsteps < 0)
            return fail(WDG_ERR_ARG, "wdg_rk4_steps: bad arguments");
        DeviceGuard g(w->device);
        bool dev = false;
        WDG_TRY(is_device_ptr(w, u, dev));
        RKExtras none;
        if (w->precision == WDG_FP64 && dev)
            return rk4_run<double>(w, u, dt, *t, nsteps, none);
        if (w->precision == WDG_FP64)
        {
            WDG_TRY(ensure_states(w));
            double *A = static_cast<double *>(w->d_state[0]);
            WDG_CUDA(cudaMemcpyAsync(A, u, sizeof(double) * w->ndof, cudaMemcpyHostToDevice, w->stream));
            WDG_TRY(rk4_run<double>(w, A, dt, *t, nsteps, none));
            WDG_CUDA(cudaMemcpyAsync(u, A, sizeof(double) * w->ndof, cudaMemcpyDeviceToHost, w->stream));
            return sync(w);
        }
        WDG_TRY(upload_state<float>(w, u));
        WDG_TRY(rk4_run<float>(w, static_cast<float *>(w->d_state[0]), dt, *t, nsteps, none));
        WDG_TRY(download_state<float>(w, u));
        return dev ? WDG_OK : sync(w);
    }

    int wdg_state_upload(wdg_wave *w, const double *u)
    {
        if (!w || !u)
            return fail(WDG_ERR_ARG, "wdg_state_upload: bad arguments");
        DeviceGuard g(w->device);
        return w->precision == WDG_FP64 ? upload_state<double>(w, u) : upload_state<float>(w, u);
    }

    int wdg_state_download(wdg_wave *w, double *u)
    {
        if (!w || !u)
            return fail(WDG_ERR_ARG, "wdg_state_download: bad arguments");
        DeviceGuard g(w->device);
        return w->precision == WDG_FP64 ? download_state<double>(w, u) : download_state<float>(w, u);
    }

    int wdg_state_device_ptr(wdg_wave *w, void **p)
    {
        if (!w || !p)
            return fail(WDG_ERR_ARG, "wdg_state_device_ptr: bad arguments");
        DeviceGuard g(w->device);
        WDG_TRY(ensure_states(w));
        *p = w->d_state[0];
        return WDG_OK;
    }

    int wdg_state_rk4_steps(wdg_wave *w, double dt, double *t, int nsteps)
    {
        WDG_TRY(whole_mesh_only(w, "wdg_state_rk4_steps"));
        if (!w || !t || nsteps < 0)
            return fail(WDG_ERR_ARG, "wdg_state_rk4_steps: bad arguments");
        DeviceGuard g(w->device);
        RKExtras none;
        if (w->precision == WDG_FP64)
            return rk4_run<double>(w, static_cast<double *>(w->d_state[0]), dt, *t, nsteps, none);
        return rk4_run<float>(w, static_cast<float *>(w->d_state[0]), dt, *t, nsteps, none);
    }

    int wdg_state_energy(wdg_wave *w, double *energy)
    {
        if (!w || !energy)
            return fail(WDG_ERR_ARG, "wdg_state_energy: bad arguments");
        DeviceGuard g(w->device);
        WDG_TRY(ensure_states(w));
        if (w->precision == WDG_FP64)
            WDG_CUDA(launch_energy<double>(w->geo, static_cast<const double *>(w->d_state[0]), w->d_scratch,
                                           w->d_result, w->stream));
        else
            WDG_CUDA(launch_energy<float>(w->geo, static_cast<const float *>(w->d_state[0]), w->d_scratch,
                                          w->d_result, w->stream));
        WDG_CUDA(cudaMemcpyAsync(w->h_result, w->d_result, sizeof(double), cudaMemcpyDeviceToHost, w->stream));
        WDG_TRY(sync(w));
        *energy = w->h_result[0];
        return WDG_OK;
    }

    int wdg_linear_functional(wdg_wave *w, int n_var, const double *fq, double *F)
    {
        if (!w || n_var < 1 || n_var > 3)
            return fail(WDG_ERR_ARG, "wdg_linear_functional: n_var must be 1..3");
        DeviceGuard g(w->device);
        const size_t cnt = (size_t)n_var * w->n * w->n * w->nel;
        Arg a[2];
        WDG_TRY(bind(w, 0, fq, cnt, true, false, a[0]));
        WDG_TRY(bind(w, 1, F, cnt, false, true, a[1]));
        WDG_CUDA(launch_linear_functional(w->geo, n_var, a[0].dev, a[1].dev, w->stream));
        return finish(w, a, 2);
    }

    int wdg_load_gaussians(wdg_wave *w, int nsrc, const double *cx, const double *cy, const double *sigma,
                           const double *amp, double scale, int comp, int mass_inv, double *F)
    {
        if (!w || nsrc < 0 || comp < 0 || comp > 2 || (nsrc > 0 && (!cx || !cy || !sigma || !amp)))
            return fail(WDG_ERR_ARG, "wdg_load_gaussians: bad arguments");
        DeviceGuard g(w->device);
        if (nsrc > w->src_cap)
        {
            if (w->d_src)
                cudaFree(w->d_src);
            w->d_src = nullptr;
            w->src_cap = 0;
            WDG_TRY(dalloc(&w->d_src, 4 * (size_t)nsrc));
            w->src_cap = nsrc;
        }
        std::vector<double> tab(4 * (size_t)std::max(nsrc, 1));
        for (int k = 0; k < nsrc; ++k)
        {
            tab[4 * k] = cx[k];
            tab[4 * k + 1] = cy[k];
            tab[4 * k + 2] = sigma[k];
            tab[4 * k + 3] = amp[k];
        }
        if (nsrc)
            WDG_CUDA(cudaMemcpyAsync(w->d_src, tab.data(), sizeof(double) * 4 * nsrc, cudaMemcpyHostToDevice, w->stream));
        Arg a;
        WDG_TRY(bind(w, 1, F, w->ndof, false, true, a));
        WDG_CUDA(launch_load_gaussians(w->geo, nsrc, w->d_src, scale, comp, a.dev, w->stream));
        if (mass_inv)
            WDG_CUDA(launch_mass(w->geo, 3, a.dev, a.dev, true, w->stream));
        // the source table is read asynchronously: wait before it can be reused
        int s = finish(w, &a, 1);
        if (s == WDG_OK && !a.host_out)
            s = sync(w);
        return s;
    }

    int wdg_norm(wdg_wave *w, const double *x, double *result)
    {
        return wdg_error(w, x, nullptr, result);
    }

    int wdg_error(wdg_wave *w, const double *x, const double *y, double *result)
    {
        if (!w || !x || !result)
            return fail(WDG_ERR_ARG, "wdg_error: bad arguments");
        DeviceGuard g(w->device);
        Arg a[2];
        WDG_TRY(bind(w, 0, x, w->ndof, true, false, a[0]));
        int nargs = 1;
        if (y)
        {
            WDG_TRY(bind(w, 1, y, w->ndof, true, false, a[1]));
            nargs = 2;
        }
        WDG_CUDA(launch_sumsq<double>(a[0].dev, y ? a[1].dev : nullptr, w->ndof, w->d_scratch, w->d_result, w->stream));
        WDG_CUDA(cudaMemcpyAsync(w->h_result, w->d_result, sizeof(double), cudaMemcpyDeviceToHost, w->stream));
        WDG_TRY(finish(w, a, nargs));
        WDG_TRY(sync(w));
        *result = std::sqrt(w->h_result[0]);
        return WDG_OK;
    }
}
