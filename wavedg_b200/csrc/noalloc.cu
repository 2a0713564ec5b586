// An allocation-free variant of wdg_load_gaussians.
//
// wdg_load_gaussians stages the Gaussian source table (cx, cy, sigma, amp per
// source) in a device buffer it allocates on first use and regrows when a call
// brings more sources.  Some callers cannot let a library allocate device
// memory once they are running: real-time loops whose memory is fixed when they
// start (a cudaMalloc can fail there and synchronises the device), or hosts
// whose own allocator has reserved the GPU's memory.  For them
// wdg_load_gaussians_noalloc keeps the table in a fixed-size array that is part
// of the library image instead.
//
// The array's device address is looked up once per device and cached for the
// life of the process; it does not survive cudaDeviceReset, after which this
// entry point must not be called again.
#include <cuda_runtime.h>

#include <mutex>

#include "wave_impl.hpp"

using namespace wdg;

// (cx, cy, sigma, amp) per source; every GPU that loads the library holds
// these 32 KiB until the process exits
static constexpr int kMaxNoAllocSources = 1024;
static __device__ __align__(256) double g_source_table[4 * kMaxNoAllocSources];

namespace
{
    std::mutex g_mu;
    double *g_table_ptr[64] = {};

    // device address of the table on `device` (which must be current); looked up once per device
    int table_address(int device, double **out)
    {
        std::lock_guard<std::mutex> lock(g_mu);
        if (device < 0 || device >= 64)
            return fail(WDG_ERR_ARG, "wdg_load_gaussians_noalloc: device ordinal out of range");
        if (!g_table_ptr[device])
        {
            void *p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_source_table);
            if (e != cudaSuccess)
                return cuda_fail(e, "cudaGetSymbolAddress(g_source_table)");
            g_table_ptr[device] = static_cast<double *>(p);
        }
        *out = g_table_ptr[device];
        return WDG_OK;
    }

    struct CurrentDevice
    {
        int prev = -1;
        explicit CurrentDevice(int dev)
        {
            cudaGetDevice(&prev);
            if (prev != dev)
                cudaSetDevice(dev);
        }
        ~CurrentDevice()
        {
            if (prev >= 0)
                cudaSetDevice(prev);
        }
    };
} // namespace

extern "C" int wdg_load_gaussians_noalloc(wdg_wave *w, int nsrc, const double *cx, const double *cy,
                                          const double *sigma, const double *amp, double scale, int comp,
                                          int mass_inv, double *F)
{
    if (!w || !F || comp < 0 || comp > 2 || nsrc < 0 || (nsrc > 0 && (!cx || !cy || !sigma || !amp)))
        return fail(WDG_ERR_ARG, "wdg_load_gaussians_noalloc: bad arguments");
    if (nsrc > kMaxNoAllocSources)
        return fail(WDG_ERR_ARG, "wdg_load_gaussians_noalloc: at most 1024 sources per call (the fixed table "
                                 "size); use wdg_load_gaussians for more");
    CurrentDevice guard(w->device);
    bool dev = false;
    WDG_TRY(is_device_ptr(w, F, dev));
    if (!dev)
        return fail(WDG_ERR_ARG, "wdg_load_gaussians_noalloc: F must be device memory (no staging buffer is "
                                 "allocated)");
    double *tab = nullptr;
    WDG_TRY(table_address(w->device, &tab));
    // interleave the four source arrays into the table, one strided copy each
    const double *cols[4] = {cx, cy, sigma, amp};
    for (int k = 0; k < 4 && nsrc > 0; ++k)
        WDG_CUDA(cudaMemcpy2DAsync(tab + k, 4 * sizeof(double), cols[k], sizeof(double), sizeof(double), nsrc,
                                   cudaMemcpyDefault, w->stream));
    WDG_CUDA(launch_load_gaussians(w->geo, nsrc, tab, scale, comp, F, w->stream));
    if (mass_inv)
        WDG_CUDA(launch_mass(w->geo, 3, F, F, true, w->stream));
    return WDG_OK;
}
