// One NSSurfacelet analysis subband computed with scratch that lives in a
// static device array of this library instead of memory it allocates.
//
// Who needs it: callers that must not allocate device memory at the moment
// they transform — latency-critical loops that cannot absorb an allocator
// call (or the device-wide synchronisation a cudaFree implies), and
// applications whose own memory manager owns the whole device and forbids
// side allocations.  Such a caller creates the plan once at start-up (that
// step allocates the mask tables), makes one warm-up call per plan size
// there too, and then calls sfl_ns_analyze_subband_static as often as it
// likes from ordinary host code: the call itself allocates nothing, neither
// through cudaMalloc nor through any library.  It does launch kernels, so it
// cannot run inside a host function enqueued on a stream (cudaLaunchHostFunc
// callbacks may make no CUDA call at all).
//
// Warm-up: the first call on a device looks up the scratch's device address
// (cudaGetSymbolAddress), and under CUDA's lazy module loading the first
// launch of a kernel loads its code, which can take device memory; so the
// first call for each plan size belongs at start-up, before the
// allocation-free phase.  The cached address
// is per device and per process: after cudaDeviceReset the library's module
// is loaded anew and the cache is stale, so a process that resets a device
// must not call this entry point on it again.
//
// The scratch is g_static_scratch below, kNoAllocMaxPoints x 2 complex
// float32 values (4 MiB): the input spectrum and one work spectrum on the
// rfft grid.  Every GPU that loads the library holds it until the process
// exits.  All calls share it, so two calls that overlap on the GPU (on
// different streams, or from different threads without ordering) race on it
// and corrupt each other's results; calls must be ordered, e.g. on one
// stream.  Nothing in the scratch needs to start at zero: every element is
// written before it is read.
#include <cuda_runtime.h>

#include <mutex>

#include "ns_mask.cuh"
#include "passes.cuh"
#include "plan.h"
#include "regpass.cuh"

namespace sfl {

// Largest rfft grid, (n1/2+1) * n2 * n3, the static scratch holds.
constexpr long long kNoAllocMaxPoints = 262144;

static __device__ __align__(256) float2 g_static_scratch[2 * kNoAllocMaxPoints];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_mu;
float2* g_scratch_addr[kMaxDevices] = {};

// The device address of the static scratch on the current device.  In host
// code g_static_scratch names a host-side stand-in, not device memory, so the
// address is looked up once per device with cudaGetSymbolAddress.
float2* scratch_on_current_device() {
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) throw ArgError("device ordinal out of range for the static scratch table");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        cuda_check(cudaGetSymbolAddress(&p, g_static_scratch), "cudaGetSymbolAddress(static scratch)");
        g_scratch_addr[dev] = reinterpret_cast<float2*>(p);
    }
    return g_scratch_addr[dev];
}

// The plan's FFT set-up for length n; the plan made it at creation, so this
// never allocates.
FFTLen* planned_fft(NSPlan& P, int n) {
    auto it = P.ffts.find(n);
    if (it == P.ffts.end()) throw ArgError("the plan has no FFT set-up for length " + std::to_string(n));
    return it->second.get();
}

}  // namespace

void ns_analyze_subband_static(NSPlan& P, const void* x, void* band, int index, cudaStream_t st) {
    if (P.nch != 1) throw ArgError("sfl_ns_analyze_subband_static takes real (float32) plans only");
    if (index < 1 || index > P.S)
        throw ArgError("subband index " + std::to_string(index) + " out of range 1:" + std::to_string(P.S));
    if (P.H > kNoAllocMaxPoints)
        throw ArgError("the volume's rfft grid has " + std::to_string(P.H) + " points ((n1/2+1)*n2*n3), above the " +
                       std::to_string(kNoAllocMaxPoints) + " the static scratch of sfl_ns_analyze_subband_static holds");
    int item = 0;
    while (item < P.S && P.items_host[item].s != index) ++item;
    float2* X = scratch_on_current_device();
    float2* W = X + kNoAllocMaxPoints;
    const int hd[3] = {P.h1, P.dims[1], P.dims[2]};
    const float* xin = reinterpret_cast<const float*>(x);
    float* out = reinterpret_cast<float*>(band);

    // X = rfft3(x): R2C along axis 1 (two lines per complex FFT), then axes 2, 3
    {
        FFTLen* f = planned_fft(P, P.dims[0]);
        Lines gin = axis_lines(P.dims, 0), gout = axis_lines(hd, 0);
        int pairs = (gin.nlines + 1) / 2;
        if (!launch_reg<false>(f->sh.n, RLoadRPair{xin, ZMap{}, gin, 1}, RStoreHalfPair{X, ZMap{}, gout, f->sh.n},
                               f->sh.tw, pairs, 1, false, st, "ns_static_r2c"))
            launch_pass(LoadRPair{xin, ZMap{}, gin, 1}, StoreHalfPair{X, ZMap{}, gout}, f->sh, pairs, 1, false, st,
                        "ns_static_r2c");
    }
    for (int a = 1; a < 3; ++a) {
        FFTLen* f = planned_fft(P, hd[a]);
        Lines g = axis_lines(hd, a);
        if (!launch_reg<false>(f->sh.n, RLoadC{X, ZMap{}, g}, RStoreC{X, ZMap{}, g}, f->sh.tw, g.nlines, 1, true, st,
                               "ns_static_c2c"))
            launch_pass(LoadC{X, ZMap{}, g, 1.f}, StoreC{X, ZMap{}, g, 1.f}, f->sh, g.nlines, 1, false, st,
                        "ns_static_c2c");
    }
    // c = irfft3(X * M): masked inverse pass along axis 3, axis 2, then C2R
    {
        FFTLen* f = planned_fft(P, hd[2]);
        Lines g = axis_lines(hd, 2);
        const NSItem* it = P.items.as<NSItem>();
        if (!launch_reg<true>(f->sh.n, RLoadNSMask{X, P.tb, it, item, 0}, RStoreC{W, ZMap{}, g}, f->sh.tw, g.nlines,
                              1, true, st, "ns_static_mask"))
            launch_pass(LoadNSMask{X, P.tb, it, item, 0}, StoreC{W, ZMap{}, g, 1.f}, f->sh, g.nlines, 1, true, st,
                        "ns_static_mask");
    }
    {
        FFTLen* f = planned_fft(P, hd[1]);
        Lines g = axis_lines(hd, 1);
        if (!launch_reg<true>(f->sh.n, RLoadC{W, ZMap{}, g}, RStoreC{W, ZMap{}, g}, f->sh.tw, g.nlines, 1, true, st,
                              "ns_static_c2c"))
            launch_pass(LoadC{W, ZMap{}, g, 1.f}, StoreC{W, ZMap{}, g, 1.f}, f->sh, g.nlines, 1, true, st,
                        "ns_static_c2c");
    }
    {
        FFTLen* f = planned_fft(P, P.dims[0]);
        Lines gin = axis_lines(hd, 0), gout = axis_lines(P.dims, 0);
        int pairs = (gout.nlines + 1) / 2;
        float scale = 1.0f / (float)P.N;
        if (!launch_reg<true>(f->sh.n, RLoadHPair{W, ZMap{}, gin, f->sh.n}, RStoreRPair{out, ZMap{}, gout, 1, scale},
                              f->sh.tw, pairs, 1, false, st, "ns_static_c2r"))
            launch_pass(LoadHPair{W, ZMap{}, gin}, StoreRPair{out, ZMap{}, gout, 1, scale}, f->sh, pairs, 1, true, st,
                        "ns_static_c2r");
    }
}

}  // namespace sfl
