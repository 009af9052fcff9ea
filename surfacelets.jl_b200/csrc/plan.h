// Plan (workspace) state shared by the C ABI and the kernel drivers.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <string>
#include <vector>

#include "design.h"
#include "fft_core.cuh"

namespace sfl {

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct AllocError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct StateError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
// A bounded device wait of an earlier call ran out (the plan's status word).
struct TimeoutError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

void cuda_check(cudaError_t e, const char* what);

// Device allocation owned by a plan.
// One int in mapped, page-locked host memory: kernels store to it through
// `dev`, the host reads `host` without a copy or a synchronisation.
struct HostWord {
    int* host = nullptr;
    int* dev = nullptr;
    HostWord() = default;
    HostWord(const HostWord&) = delete;
    HostWord& operator=(const HostWord&) = delete;
    ~HostWord();
    void alloc();
    int read() const { return host ? *static_cast<volatile int*>(host) : 0; }
    void clear() {
        if (host) *static_cast<volatile int*>(host) = 0;
    }
};

struct DevMem {
    void* p = nullptr;
    size_t bytes = 0;
    DevMem() = default;
    DevMem(const DevMem&) = delete;
    DevMem& operator=(const DevMem&) = delete;
    DevMem(DevMem&& o) noexcept : p(o.p), bytes(o.bytes) {
        o.p = nullptr;
        o.bytes = 0;
    }
    DevMem& operator=(DevMem&& o) noexcept {
        std::swap(p, o.p);
        std::swap(bytes, o.bytes);
        return *this;
    }
    ~DevMem();
    void alloc(size_t n);
    template <class T>
    T* as() const { return reinterpret_cast<T*>(p); }
};

// Twiddle table and radix schedule of one FFT length, on the device.
struct FFTLen {
    FFTShape sh;
    DevMem tw;
};

// Per-subband descriptor of the NS cascade (device copy in NSPlan::items).
struct NSItem {
    int s;        // 1-based subband index
    int kind;     // 0 directional, 1 lowpass
    int lv;       // pyramid level (0 = finest); the lowpass uses J
    int i;        // hourglass 1..3
    int g;        // group (scale, hourglass): index of its mask table
    int wa_off, wb_off;    // float offsets of the two wedge planes
    int wa_lo, wa_hi, wa_dlo;   // 0-based axes and lo extent of plane a
    int wb_lo, wb_hi, wb_dlo;
};

// Where item z of a batched launch starts: a fixed stride, or the subband
// named by an NS item (offset (s-1)*sub_stride).
struct ZMap {
    const NSItem* items = nullptr;
    int item0 = 0;
    long long sub_stride = 0;
    long long zstride = 0;
    __device__ __forceinline__ long long off(int z) const {
        return items ? (long long)(items[item0 + z].s - 1) * sub_stride : (long long)z * zstride;
    }
};

// Mask tables on the device: the group masks (float64-designed, one rfft
// grid each), the level bandpasses (synthesis of a bank that is not tight),
// the lowpass's per-axis factors and the wedge planes.
struct NSMaskTables {
    const float* G = nullptr;       // [group][H]
    const float* Bl = nullptr;      // [level][H] (not tight only)
    const float* vec = nullptr;     // lowpass factors a1 | a2 | a3
    const float* planes = nullptr;
    long long H = 0;
    int h1 = 0, n2 = 0, n3 = 0;
    int tight = 1;
    int low_off[3] = {0, 0, 0};
};

// Support box of a mask group on the rfft grid: rows k1 < nk1 and the nk2
// columns |k2| <= b2 (k2 <= b2 or k2 >= n2 - b2; b2 >= n2 when all).
struct NSBox {
    int nk1 = 0, nk2 = 0, b2 = 0;
};

struct NSPlan {
    sfl_ns_params p{};
    int dims[3] = {0, 0, 0};
    int h1 = 0;
    long long N = 0;      // voxels
    long long H = 0;      // rfft grid points
    int S = 0;            // subbands
    int nch = 1;          // 1 real, 2 complex
    bool ndfb = false;    // the standalone directional bank (no pyramid, no lowpass)
    int group = 8;
    int ipc = 0;          // subbands a CTA of the slab axis-3 analysis pass takes (1, 2, 4, 8; 0: the default, mask_ipc)
    std::vector<NSItem> items_host;   // streaming / item order: directional ascending, then lowpass
    DevMem items;
    DevMem G, Bl, vec, planes;
    NSMaskTables tb;
    HostWord status;        // status word of bounded waits (0 = fine), written by the kernels
    // slab pipeline (spectra with the axis-1 pitch padded to P1)
    bool slab = false;
    int P1 = 0;
    long long SP = 0;               // P1 * n2 * n3
    std::vector<NSBox> boxes;       // per mask group, then the lowpass
    NSBox boxes_full;
    int sms = 148;
    std::map<int, std::unique_ptr<FFTLen>> ffts;
    DevMem X;        // nch spectra
    DevMem work;     // group spectra
    DevMem acc, comp;   // nch accumulators (+ Kahan compensation)
    DevMem band, maxbits;   // float32 subbands of a chunk and their peaks (bfloat16 coefficients)
    // streaming state
    int stream_mode = 0;    // 0 idle, 1 analyzing, 2 synthesizing
    int stream_pos = 0;
    int stream_chunk0 = 0;  // synthesis: first item of the mask group being staged
    NSDesign design;        // kept for the table export
};

struct DecPlan;
// DecPlan is complete only in dec.cu, which defines this deleter.
struct DecPlanDeleter {
    void operator()(DecPlan* d) const;
};

struct Plan {
    int kind = SFL_KIND_NS;
    int dtype = SFL_REAL32;
    int device = 0;
    std::unique_ptr<NSPlan> ns;
    std::unique_ptr<DecPlan, DecPlanDeleter> dec;
};

// FFT length set-up (twiddles designed in float64).
FFTLen* get_fft(std::map<int, std::unique_ptr<FFTLen>>& cache, int n);

// NS drivers (ns.cu)
void ns_plan_init(NSPlan& P, const sfl_ns_params& p, const int dims[3], int dtype, bool ndfb = false);
void ns_analyze(NSPlan& P, const void* x, void* c, cudaStream_t st, bool synth_masks);
void ns_synthesize(NSPlan& P, const void* c, void* x, cudaStream_t st, bool analysis_masks);
void ns_stream_analyze_begin(NSPlan& P, const void* x, cudaStream_t st);
int ns_stream_analyze_next(NSPlan& P, void* band, int* index, cudaStream_t st);
void ns_stream_synth_begin(NSPlan& P, cudaStream_t st);
int ns_stream_synth_next_index(NSPlan& P, int* index);
void ns_stream_synth_push(NSPlan& P, const void* band, cudaStream_t st);
void ns_stream_synth_end(NSPlan& P, void* x, cudaStream_t st);
// Group tables G, level bandpasses Bl and the per-table support boxes,
// designed in float64 on the device (ns_design.cu).
void ns_design_tables_device(NSPlan& P);
// Slab pipeline (ns_slab.cu).
bool ns_slab_supported(int n1, int n2, int n3);
// Launches from this thread run beside others on concurrent streams (a batch
// graph being captured): the slab pipeline's launch shapes then favour fewer,
// larger CTAs over filling the GPU alone.
void ns_set_concurrent(bool on);
void ns_use_slabs(NSPlan& P);
NSBox ns_make_box(int nk1, int b2, int n2);
NSBox ns_table_box(const std::vector<double>& g, int h1, int n2, int n3);
void ns_alloc_scratch(NSPlan& P);
void ns_slab_rfft3(NSPlan& P, const float* x, int es, float2* X, cudaStream_t st);
void ns_slab_analyze(NSPlan& P, const void* x, void* c, cudaStream_t st, bool synth_masks);
void ns_slab_synthesize(NSPlan& P, const void* c, void* x, cudaStream_t st, bool analysis_masks);
void ns_slab_irfft3(NSPlan& P, float2* A, float* x, int es, cudaStream_t st);
int ns_slab_chunk_end(const NSPlan& P, int i0);
void ns_slab_analyze_items(NSPlan& P, const float2* X, float* vol, ZMap vz, int es, int i0, int nz, bool synth_masks,
                           cudaStream_t st);
void ns_slab_synth_items(NSPlan& P, const float* vol, ZMap vz, int es, int i0, int nz, bool analysis_masks,
                         float2* acc, float2* comp, cudaStream_t st);
void ns_slab_denoise_items(NSPlan& P, const float2* X, int i0, int nz, const float* tau, float2* acc, float2* comp,
                           cudaStream_t st);
void ns_slab_stage_items(NSPlan& P, const float* vol, ZMap vz, int es, int i0, int nz, int slot0, int nch,
                         cudaStream_t st);
void ns_slab_accum_items(NSPlan& P, int i0, int nz, bool analysis_masks, float2* acc, float2* comp, int nch,
                         cudaStream_t st);
// The line pipeline's denoiser step on items [i0, i0 + nz): the analysis
// axis-3 and axis-2 passes, one fused axis-1 kernel (C2R, soft threshold,
// R2C), the synthesis axis-2 pass and the accumulation (ns.cu); for axis-1
// lengths with a register kernel.
bool ns_line_shrink_supported(const NSPlan& P);
void ns_line_denoise_items(NSPlan& P, const float2* X, int i0, int nz, const float* tau, float2* acc, float2* comp,
                           cudaStream_t st);
// Fused soft-threshold denoiser y = S(soft(A x, tau)) (ns_denoise.cu).
void ns_denoise(NSPlan& P, const float* x, float* y, const float* tau, cudaStream_t st);
// Item-range building blocks of the slab and line pipelines (ns.cu): the
// spectrum of a channel, the launch chunks, the analysis of items into
// volumes at vol + vz.off(z), their accumulation into a spectrum, and its
// inverse.  Spectra hold ns_spec_elems bins.
long long ns_spec_elems(const NSPlan& P);
void ns_forward_spectrum(NSPlan& P, const float* x, int es, float2* X, cudaStream_t st);
int ns_next_chunk(const NSPlan& P, int i0);
void ns_analyze_range(NSPlan& P, const float2* X, float* vol, ZMap vz, int es, int i0, int nz, bool synth_masks,
                      cudaStream_t st);
void ns_acc_clear(NSPlan& P, float2* acc, float2* comp, cudaStream_t st);
// Decimated design tables composed on the device from their host factors
// (dec_design.cu): V_K into V[K] (float32, half-K grids) and one IRC stage's
// four slice planes (float2, nKh x nm).
void ritf_masks_device(const int n[3], const std::vector<double> P[3][3], float* const V[3], cudaStream_t st);
void irc_slices_device(const IRCFactors& F, float2* const out[4], cudaStream_t st);
// The plan's Kahan compensation grid of channel ch (spectrum-sized).
float2* ns_comp_grid(NSPlan& P, int ch);
// Runs out one bounded mbarrier wait on purpose (no copy in flight) so that
// the plan's status word records a timeout.
void ns_selftest_wait(NSPlan& P, cudaStream_t st);
void ns_accumulate_range(NSPlan& P, const float* vol, ZMap vz, int es, int i0, int nz, bool analysis_masks,
                         float2* acc, float2* comp, cudaStream_t st);
void ns_inverse_spectrum(NSPlan& P, float2* A, float* x, int es, cudaStream_t st);
// ns_accumulate_range in two halves: the forward transforms of nz volumes into
// work slots slot0.. (nch channels on the slab pipeline, 1 on the line
// pipeline), then the accumulation of items [i0, i0 + nz) from slots 0..nz-1.
void ns_stage_range(NSPlan& P, const float* vol, ZMap vz, int es, int i0, int nz, int slot0, int nch,
                    cudaStream_t st);
void ns_accum_staged(NSPlan& P, int i0, int nz, bool analysis_masks, float2* acc, float2* comp, int nch,
                     cudaStream_t st);
ZMap ns_subband_map(const NSPlan& P, int i0, int es);
// bfloat16 coefficients with a float32 scale per subband (ns_bf16.cu).
void ns_analyze_bf16(NSPlan& P, const float* x, void* c, float* scales, cudaStream_t st);
void ns_synthesize_bf16(NSPlan& P, const void* c, const float* scales, float* x, cudaStream_t st);
// One analysis subband with static scratch (noalloc.cu).
void ns_analyze_subband_static(NSPlan& P, const void* x, void* band, int index, cudaStream_t st);

// Decimated drivers (dec.cu)
void dec_plan_create(Plan& plan, const sfl_surf_params& p, const int dims[3], int dtype);
int dec_nsubbands(const DecPlan& d);
long long dec_ncoeffs(const DecPlan& d);
void dec_subband_info(const DecPlan& d, int i, int shape[3], long long* offset);
void dec_analyze(DecPlan& d, const void* x, void* c, cudaStream_t st);
void dec_synthesize(DecPlan& d, const void* c, void* x, cudaStream_t st);
void dec_adjoint_analyze(DecPlan& d, const void* c, void* x, cudaStream_t st);
void dec_adjoint_synthesize(DecPlan& d, const void* x, void* c, cudaStream_t st);
const SurfDesign& dec_design(const DecPlan& d);
const float* dec_plan_table(const DecPlan& d, const std::string& name, int index, long long* count);

}  // namespace sfl
