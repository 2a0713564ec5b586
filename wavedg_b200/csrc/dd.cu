// C-ABI: a domain of a decomposed mesh (one rank's share of the elements).
//
// The reference distributes a mesh over MPI ranks (Mesh2D::distribute, source/Mesh2D.cpp:384-592)
// and exchanges the face traces of cut edges before every operator application
// (FaceVector::send_recv, source/FEMVector.cpp:153-216).  Here a domain is an ordinary
// discretisation of its own elements whose state buffers carry, after the elements, one
// n x 3 trace per cut side (the "halo"); the cut sides' partner offsets point into it, so
// the fused stage kernels read a neighbour on another rank exactly as they read a local one.
// Per RK stage the host fills the halo of the stage's input buffer (gather the traces the
// other ranks need with wdg_halo_gather, move them with NCCL or any transport, write the
// received ones with wdg_halo_put) and runs the stage (wdg_rk4_stage).  Every element's
// arithmetic is the one of the undivided mesh, so the decomposed result is the same.
#include <cuda_runtime.h>

#include <vector>

#include "wave_impl.hpp"

using namespace wdg;

namespace
{
    // out[3 j + f] = u[idx[j] + f]; an index outside the elements' values is skipped and
    // recorded in the handle's error word (bit 1, as a bad neighbour index)
    template <typename Real>
    __global__ void halo_gather_kernel(const Real *__restrict__ u, const int *__restrict__ idx, int count,
                                       long long limit, unsigned *err, Real *__restrict__ out)
    {
        for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < count; j += gridDim.x * blockDim.x)
        {
            const int o = idx[j];
            if (o < 0 || o + 3 > limit)
            {
                atomicOr(err, 2u);
                continue;
            }
            out[3 * j] = u[o];
            out[3 * j + 1] = u[o + 1];
            out[3 * j + 2] = u[o + 2];
        }
    }

} // namespace

extern "C"
{
    int wdg_mesh_partner_table(const wdg_mesh *mesh, int n_colloc, const int *bc, int *fbase, unsigned *fcode)
    {
        if (!mesh || !fbase || !fcode || n_colloc < 2 || n_colloc > 9)
            return fail(WDG_ERR_ARG, "wdg_mesh_partner_table: bad arguments");
        FaceTables ft;
        WDG_TRY(build_face_tables(*mesh, bc, ft));
        std::vector<int> fb;
        std::vector<uint32_t> fc;
        build_partner_tables(ft, n_colloc, fb, fc);
        std::copy(fb.begin(), fb.end(), fbase);
        std::copy(fc.begin(), fc.end(), fcode);
        return WDG_OK;
    }

    int wdg_wave_create_halo(const wdg_mesh *mesh, int n_colloc, const int *bc, int precision, int device, int n_halo,
                             const int *halo_elem, const int *halo_side, wdg_wave **out)
    {
        if (!mesh || !out || n_halo < 0 || (n_halo > 0 && (!halo_elem || !halo_side)))
            return fail(WDG_ERR_ARG, "wdg_wave_create_halo: bad arguments");
        *out = nullptr;
        FaceTables ft;
        WDG_TRY(build_face_tables(*mesh, bc, ft));
        std::vector<int> fb;
        std::vector<uint32_t> fc;
        build_partner_tables(ft, n_colloc, fb, fc);
        const long long nd = 3LL * n_colloc * n_colloc * mesh->nel;
        if (nd + 3LL * n_colloc * n_halo >= (1LL << 31))
            return fail(WDG_ERR_UNSUPPORTED, "wdg_wave_create_halo: more than 2^31 values in a state buffer");
        for (int j = 0; j < n_halo; ++j)
        {
            const int el = halo_elem[j], f = halo_side[j];
            if (el < 0 || el >= mesh->nel || f < 0 || f > 3)
                return fail(WDG_ERR_ARG, "wdg_wave_create_halo: halo side out of range");
            const uint32_t byte = (fc[el] >> (8 * f)) & 0xffu;
            if (!(byte & 0x80u))
                return fail(WDG_ERR_ARG, "wdg_wave_create_halo: a halo side must be a boundary side of the local mesh");
            // partner: trace j of the halo, face node k at + 3 k (stride code 0), interior
            fb[4 * (size_t)el + f] = (int)(nd + 3LL * n_colloc * j);
            fc[el] &= ~(0xffu << (8 * f));
        }
        wdg_wave *w = nullptr;
        WDG_TRY(wdg_wave_create(mesh, n_colloc, bc, precision, device, &w));
        DeviceScope g(w->device);
        w->halo = 3LL * n_colloc * n_halo;
        cudaError_t e = cudaMemcpy(w->d_fbase, fb.data(), sizeof(int) * fb.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(w->d_fcode, fc.data(), sizeof(uint32_t) * fc.size(), cudaMemcpyHostToDevice);
        int s = (e == cudaSuccess) ? ensure_states(w) : cuda_fail(e, "wdg_wave_create_halo: partner tables");
        if (s != WDG_OK)
        {
            wdg_wave_destroy(w);
            return s;
        }
        *out = w;
        return WDG_OK;
    }

    int wdg_halo_info(const wdg_wave *w, long long *elements_values, long long *halo_values)
    {
        if (!w)
            return fail(WDG_ERR_ARG, "null discretisation");
        if (elements_values)
            *elements_values = w->ndof;
        if (halo_values)
            *halo_values = w->halo;
        return WDG_OK;
    }

    int wdg_halo_gather(wdg_wave *w, int buffer, const int *idx, int count, void *out)
    {
        if (!w || buffer < 0 || buffer > 2 || count < 0 || (count > 0 && (!idx || !out)))
            return fail(WDG_ERR_ARG, "wdg_halo_gather: bad arguments");
        if (count == 0)
            return WDG_OK;
        DeviceScope g(w->device);
        WDG_TRY(ensure_states(w));
        const unsigned grid = (unsigned)std::min(148 * 8, (count + 255) / 256);
        if (w->precision == WDG_FP32)
            halo_gather_kernel<float><<<grid, 256, 0, w->stream>>>(static_cast<const float *>(w->d_state[buffer]), idx,
                                                                   count, w->ndof, w->d_err, static_cast<float *>(out));
        else
            halo_gather_kernel<double><<<grid, 256, 0, w->stream>>>(static_cast<const double *>(w->d_state[buffer]),
                                                                    idx, count, w->ndof, w->d_err,
                                                                    static_cast<double *>(out));
        WDG_CUDA(cudaGetLastError());
        return WDG_OK;
    }

    int wdg_halo_put(wdg_wave *w, int buffer, long long offset, const void *src, long long count)
    {
        if (!w || buffer < 0 || buffer > 2 || offset < 0 || count < 0 || offset + count > w->halo || (count && !src))
            return fail(WDG_ERR_ARG, "wdg_halo_put: bad arguments");
        if (count == 0)
            return WDG_OK;
        DeviceScope g(w->device);
        WDG_TRY(ensure_states(w));
        char *dst = static_cast<char *>(w->d_state[buffer]) + w->real_size() * (size_t)(w->ndof + offset);
        WDG_CUDA(cudaMemcpyAsync(dst, src, w->real_size() * (size_t)count, cudaMemcpyDefault, w->stream));
        return WDG_OK;
    }

    int wdg_rk4_stage(wdg_wave *w, int stage, double dt)
    {
        if (!w || stage < 0 || stage > 4)
            return fail(WDG_ERR_ARG, "wdg_rk4_stage: stage must be 0..4");
        DeviceScope g(w->device);
        return w->precision == WDG_FP32 ? rk4_stage<float>(w, stage, dt) : rk4_stage<double>(w, stage, dt);
    }

    int wdg_rk4_stage_forced(wdg_wave *w, int stage, double dt, double t, const void *F, double omega, double *acc,
                             double acc_c)
    {
        if (!w || stage < 0 || stage > 4 || (F && !(omega != 0.0)))
            return fail(WDG_ERR_ARG, "wdg_rk4_stage_forced: stage must be 0..4 and omega nonzero with a forcing");
        DeviceScope g(w->device);
        bool dev = true;
        if (F)
            WDG_TRY(is_device_ptr(w, F, dev));
        if (dev && acc)
            WDG_TRY(is_device_ptr(w, acc, dev));
        if (!dev)
            return fail(WDG_ERR_ARG, "wdg_rk4_stage_forced: F and acc must be device arrays");
        return w->precision == WDG_FP32 ? rk4_stage<float>(w, stage, dt, t, F, omega, acc, acc_c)
                                        : rk4_stage<double>(w, stage, dt, t, F, omega, acc, acc_c);
    }

    int wdg_rk4_stage_elems(wdg_wave *w, int stage, double dt, double t, const void *F, double omega, double *acc,
                            double acc_c, int el_begin, int el_end)
    {
        if (!w || stage < 0 || stage > 4 || (F && !(omega != 0.0)))
            return fail(WDG_ERR_ARG, "wdg_rk4_stage_elems: stage must be 0..4 and omega nonzero with a forcing");
        if (el_begin < 0 || el_begin > el_end || el_end > w->nel || (el_begin & 3))
            return fail(WDG_ERR_ARG, "wdg_rk4_stage_elems: need 0 <= el_begin <= el_end <= n_elem, el_begin a "
                                     "multiple of 4");
        if (el_begin == el_end)
            return WDG_OK;
        DeviceScope g(w->device);
        bool dev = true;
        if (F)
            WDG_TRY(is_device_ptr(w, F, dev));
        if (dev && acc)
            WDG_TRY(is_device_ptr(w, acc, dev));
        if (!dev)
            return fail(WDG_ERR_ARG, "wdg_rk4_stage_elems: F and acc must be device arrays");
        return w->precision == WDG_FP32 ? rk4_stage<float>(w, stage, dt, t, F, omega, acc, acc_c, el_begin, el_end)
                                        : rk4_stage<double>(w, stage, dt, t, F, omega, acc, acc_c, el_begin, el_end);
    }
}
