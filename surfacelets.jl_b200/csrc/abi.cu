// extern "C" entry points of libsurfacelets_b200.so (declared in
// include/surfacelets_b200.h).  Every entry point catches the library's
// exceptions and turns them into a status code plus a thread-local message.
#include <algorithm>
#include <cuda_runtime.h>

#include <cstring>
#include <memory>
#include <mutex>
#include <map>
#include <string>
#include <vector>

#include "../../include/surfacelets_b200.h"
#include "design.h"
#include "plan.h"
#include "prof.h"

namespace sfl {

void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        if (e == cudaErrorMemoryAllocation) {
            cudaGetLastError();
            throw AllocError(std::string(what) + ": " + cudaGetErrorString(e));
        }
        throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
    }
}

DevMem::~DevMem() {
    if (p) cudaFree(p);
}

HostWord::~HostWord() {
    if (host) cudaFreeHost(host);
}

void HostWord::alloc() {
    if (host) return;
    cuda_check(cudaHostAlloc(reinterpret_cast<void**>(&host), sizeof(int), cudaHostAllocMapped), "cudaHostAlloc(status)");
    *static_cast<volatile int*>(host) = 0;
    cuda_check(cudaHostGetDevicePointer(reinterpret_cast<void**>(&dev), host, 0), "cudaHostGetDevicePointer(status)");
}

void DevMem::alloc(size_t n) {
    if (p) {
        cudaFree(p);
        p = nullptr;
    }
    bytes = n;
    cuda_check(cudaMalloc(&p, n ? n : 1), "cudaMalloc");
}

}  // namespace sfl

struct sfl_plan {
    sfl::Plan impl;
};

namespace {

thread_local std::string g_error;

template <class F>
int guarded(F&& f) {
    try {
        g_error.clear();
        return f();
    } catch (const sfl::ArgError& e) {
        g_error = e.what();
        return SFL_ERR_ARGUMENT;
    } catch (const sfl::DimError& e) {
        g_error = e.what();
        return SFL_ERR_DIMENSION;
    } catch (const sfl::AllocError& e) {
        g_error = e.what();
        return SFL_ERR_ALLOC;
    } catch (const sfl::CudaError& e) {
        g_error = e.what();
        return SFL_ERR_CUDA;
    } catch (const sfl::StateError& e) {
        g_error = e.what();
        return SFL_ERR_STATE;
    } catch (const sfl::TimeoutError& e) {
        g_error = e.what();
        return SFL_ERR_TIMEOUT;
    } catch (const std::bad_alloc&) {
        g_error = "host memory exhausted";
        return SFL_ERR_ALLOC;
    } catch (const std::exception& e) {
        g_error = e.what();
        return SFL_ERR_ARGUMENT;
    }
}

void need(const void* p, const char* what) {
    if (!p) throw sfl::ArgError(std::string(what) + " must not be NULL");
}

void dims_of(const int32_t* d, int out[3]) {
    need(d, "dims");
    for (int i = 0; i < 3; ++i) out[i] = d[i];
}

cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

void check_aligned(const void* p, int dtype, const char* what) {
    uintptr_t a = reinterpret_cast<uintptr_t>(p);
    size_t need_al = dtype == SFL_COMPLEX64 ? 8 : 4;
    if (a % need_al != 0)
        throw sfl::ArgError(std::string(what) + " is not aligned to its element type");
}

// Spectra (the item-range ABI) are copied in 16-byte blocks by the slab passes.
void check_spectrum_aligned(const void* p, const char* what) {
    if (reinterpret_cast<uintptr_t>(p) % 16 != 0) throw sfl::ArgError(std::string(what) + " is not 16-byte aligned");
}

// Runs f with the plan's device current, restoring the caller's afterwards.
template <class F>
void on_device(const sfl_plan* plan, F&& f) {
    int cur = 0;
    sfl::cuda_check(cudaGetDevice(&cur), "cudaGetDevice");
    if (cur != plan->impl.device) sfl::cuda_check(cudaSetDevice(plan->impl.device), "cudaSetDevice");
    try {
        f();
    } catch (...) {
        if (cur != plan->impl.device) cudaSetDevice(cur);
        throw;
    }
    if (cur != plan->impl.device) sfl::cuda_check(cudaSetDevice(cur), "cudaSetDevice");
}

// A bounded wait of an earlier call on this plan ran out: report it once (the
// word is cleared) before anything new is enqueued.  Results of the earlier
// call are not valid.
void check_timeout(const sfl_plan* plan) {
    if (plan->impl.kind != SFL_KIND_NS) return;
    sfl::NSPlan& N = *plan->impl.ns;
    const int v = N.status.read();
    if (v != 0) {
        N.status.clear();
        throw sfl::TimeoutError("a bounded device wait of an earlier call on this plan ran out (status " +
                                std::to_string(v) + "); that call's results are not valid");
    }
}

// Pipeline, group and axis-3 tile of an NS plan (the knobs of the tuner).
void ns_apply(sfl::NSPlan& N, int pipeline, int group, int ipc = -1) {
    if (ipc >= 0) N.ipc = ipc;
    cudaDeviceSynchronize();
    if (pipeline == SFL_PIPELINE_LINES) {
        if (N.slab) {
            N.slab = false;
            sfl::ns_alloc_scratch(N);
        }
    } else if (pipeline == SFL_PIPELINE_PLANES) {
        throw sfl::ArgError("the plane-major pipeline was retired: the slab pipeline is faster at every size it "
                            "supported");
    } else if (pipeline == SFL_PIPELINE_SLABS) {
        sfl::ns_use_slabs(N);
    } else {
        throw sfl::ArgError("unknown pipeline " + std::to_string(pipeline));
    }
    if (group >= 1 && std::min(group, N.S) != N.group) {
        N.group = std::min(group, N.S);
        sfl::ns_alloc_scratch(N);
    }
}

int ns_pipeline_of(const sfl::NSPlan& N) {
    return N.slab ? SFL_PIPELINE_SLABS : SFL_PIPELINE_LINES;
}

// Tuned (pipeline, group) per transform, size and element type, for the
// lifetime of the process; plans created later with the same key start tuned.
std::mutex g_tuned_mu;
struct Tuning {
    int pipeline, group, ipc;
};
std::map<std::string, Tuning> g_tuned;

std::string tune_key(const sfl::NSPlan& N, int dtype) {
    std::string k = (N.ndfb ? "ndfb" : "ns") + std::string(":");
    for (int i = 0; i < 3; ++i) k += std::to_string(N.dims[i]) + ",";
    k += std::to_string(dtype) + ":" + std::to_string(N.p.scales) + ":";
    for (int j = 0; j < N.p.scales; ++j) k += std::to_string(N.p.direction_levels[j]) + ",";
    k += ":" + std::to_string(N.p.bernstein_order) + ":" + std::to_string(N.p.halfband_order) + ":" +
         std::to_string(N.p.transition) + ":" + std::to_string(N.p.tight);
    return k;
}

void apply_tuned(sfl_plan* plan) {
    sfl::NSPlan& N = *plan->impl.ns;
    Tuning t;
    {
        std::lock_guard<std::mutex> lk(g_tuned_mu);
        auto it = g_tuned.find(tune_key(N, plan->impl.dtype));
        if (it == g_tuned.end()) return;
        t = it->second;
    }
    ns_apply(N, t.pipeline, t.group, t.ipc);
}

// One transform of a plan (the four operators of the C ABI).
void run_op(sfl_plan* plan, int op, const void* in, void* out, cudaStream_t st) {
    sfl::Plan& P = plan->impl;
    const bool ns = P.kind == SFL_KIND_NS;
    switch (op) {
        case SFL_OP_ANALYZE:
            ns ? sfl::ns_analyze(*P.ns, in, out, st, false) : sfl::dec_analyze(*P.dec, in, out, st);
            return;
        case SFL_OP_SYNTHESIZE:
            ns ? sfl::ns_synthesize(*P.ns, in, out, st, false) : sfl::dec_synthesize(*P.dec, in, out, st);
            return;
        case SFL_OP_ADJOINT_ANALYZE:
            ns ? sfl::ns_synthesize(*P.ns, in, out, st, true) : sfl::dec_adjoint_analyze(*P.dec, in, out, st);
            return;
        case SFL_OP_ADJOINT_SYNTHESIZE:
            ns ? sfl::ns_analyze(*P.ns, in, out, st, true) : sfl::dec_adjoint_synthesize(*P.dec, in, out, st);
            return;
        case SFL_OP_COPY_VOLUME: {
            int d[3];
            if (ns) {
                for (int i = 0; i < 3; ++i) d[i] = P.ns->dims[i];
            } else {
                for (int i = 0; i < 3; ++i) d[i] = sfl::dec_design(*P.dec).dims[i];
            }
            const size_t bytes = (size_t)d[0] * d[1] * d[2] * (P.dtype == SFL_COMPLEX64 ? 8 : 4);
            sfl::cuda_check(cudaMemcpyAsync(out, in, bytes, cudaMemcpyDefault, st), "cudaMemcpyAsync(volume)");
            return;
        }
    }
    throw sfl::ArgError("unknown operator " + std::to_string(op));
}

}  // namespace

struct sfl_batch {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int device = 0;
    ~sfl_batch() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

extern "C" {

const char* sfl_last_error(void) { return g_error.c_str(); }

const char* sfl_version(void) { return "surfacelets_b200 0.1.0 (sm_100a)"; }

int sfl_ns_check_params(const sfl_ns_params* p) {
    return guarded([&] {
        need(p, "params");
        sfl::ns_check_params(*p);
        return SFL_OK;
    });
}

int sfl_ns_check_size(const sfl_ns_params* p, const int32_t dims[3]) {
    return guarded([&] {
        need(p, "params");
        int d[3];
        dims_of(dims, d);
        sfl::ns_check_params(*p);
        sfl::ns_check_size(*p, d);
        return SFL_OK;
    });
}

int sfl_ns_nsubbands(const sfl_ns_params* p, int32_t* n) {
    return guarded([&] {
        need(p, "params");
        need(n, "n");
        sfl::ns_check_params(*p);
        *n = sfl::ns_nsubbands(*p);
        return SFL_OK;
    });
}

int sfl_ns_layout(const sfl_ns_params* p, int32_t* scale, int32_t* direction) {
    return guarded([&] {
        need(p, "params");
        sfl::ns_check_params(*p);
        int k = 0;
        if (scale) scale[k] = 0;
        if (direction) direction[k] = 0;
        ++k;
        for (int j = 1; j <= p->scales; ++j)
            for (int d = 1; d <= sfl::ns_nbands(*p, j); ++d, ++k) {
                if (scale) scale[k] = j;
                if (direction) direction[k] = d;
            }
        return SFL_OK;
    });
}

int sfl_surf_levels_from_int(int32_t L, int32_t out[3][3]) {
    return guarded([&] {
        need(out, "out");
        int o[3][3];
        sfl::surf_levels_from_int(L, o);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) out[i][j] = o[i][j];
        return SFL_OK;
    });
}

int sfl_surf_check_params(const sfl_surf_params* p) {
    return guarded([&] {
        need(p, "params");
        sfl::surf_check_params(*p);
        return SFL_OK;
    });
}

int sfl_surf_layout(const sfl_surf_params* p, const int32_t dims[3], int32_t* n, int32_t* sizes, int32_t* scale,
                    int32_t* hourglass, int32_t* wedge) {
    return guarded([&] {
        need(p, "params");
        int d[3];
        dims_of(dims, d);
        sfl::surf_check_params(*p);
        auto sz = sfl::surf_layout_sizes(*p, d);
        if (n) *n = (int32_t)sz.size();
        if (sizes)
            for (size_t i = 0; i < sz.size(); ++i)
                for (int k = 0; k < 3; ++k) sizes[3 * i + k] = sz[i][k];
        int k = 0;
        if (scale) scale[0] = 0;
        if (hourglass) hourglass[0] = 0;
        if (wedge) wedge[0] = 0;
        ++k;
        for (int j = 1; j <= p->scales; ++j)
            for (int K = 1; K <= 3; ++K) {
                int s = 0;
                for (int m = 0; m < 3; ++m)
                    if (m != K - 1) s += p->levels[j - 1][K - 1][m];
                for (int w = 1; w <= (1 << s); ++w, ++k) {
                    if (scale) scale[k] = j;
                    if (hourglass) hourglass[k] = K;
                    if (wedge) wedge[k] = w;
                }
            }
        return SFL_OK;
    });
}

int sfl_surf_redundancy(const sfl_surf_params* p, const int32_t dims[3], double* r) {
    return guarded([&] {
        need(p, "params");
        need(r, "r");
        int d[3];
        dims_of(dims, d);
        sfl::surf_check_params(*p);
        auto sz = sfl::surf_layout_sizes(*p, d);
        double tot = 0;
        for (auto& s : sz) tot += (double)s[0] * s[1] * s[2];
        *r = tot / ((double)d[0] * d[1] * d[2]);
        return SFL_OK;
    });
}

int sfl_ns_plan_create(const sfl_ns_params* p, const int32_t dims[3], int32_t dtype, sfl_plan** out) {
    return guarded([&] {
        need(p, "params");
        need(out, "out");
        *out = nullptr;
        if (dtype != SFL_REAL32 && dtype != SFL_COMPLEX64) throw sfl::ArgError("dtype must be SFL_REAL32 or SFL_COMPLEX64");
        int d[3];
        dims_of(dims, d);
        sfl::ns_check_params(*p);
        sfl::ns_check_size(*p, d);
        std::unique_ptr<sfl_plan> plan(new sfl_plan);
        plan->impl.kind = SFL_KIND_NS;
        plan->impl.dtype = dtype;
        sfl::cuda_check(cudaGetDevice(&plan->impl.device), "cudaGetDevice");
        plan->impl.ns.reset(new sfl::NSPlan);
        sfl::ns_plan_init(*plan->impl.ns, *p, d, dtype);
        apply_tuned(plan.get());
        *out = plan.release();
        return SFL_OK;
    });
}

static sfl_ns_params ndfb_as_ns(const sfl_ndfb_params& p) {
    if (p.levels < 0) throw sfl::ArgError("levels must be ≥ 0");
    if (!(p.transition >= 0)) throw sfl::ArgError("transition must be ≥ 0");
    sfl_ns_params q{};
    q.scales = 1;
    q.direction_levels[0] = p.levels;
    q.bernstein_order = p.bernstein_order;
    q.halfband_order = p.halfband_order;
    q.transition = p.transition;
    q.tight = p.tight;
    sfl::ns_check_params(q);
    return q;
}

int sfl_ndfb_check_params(const sfl_ndfb_params* p) {
    return guarded([&] {
        need(p, "params");
        ndfb_as_ns(*p);
        return SFL_OK;
    });
}

int sfl_ndfb_plan_create(const sfl_ndfb_params* p, const int32_t dims[3], int32_t dtype, sfl_plan** out) {
    return guarded([&] {
        need(p, "params");
        need(out, "out");
        *out = nullptr;
        if (dtype != SFL_REAL32 && dtype != SFL_COMPLEX64) throw sfl::ArgError("dtype must be SFL_REAL32 or SFL_COMPLEX64");
        int d[3];
        dims_of(dims, d);
        const sfl_ns_params q = ndfb_as_ns(*p);
        for (int i = 0; i < 3; ++i)
            if (d[i] < 1) throw sfl::DimError("volume size must be positive");
        std::unique_ptr<sfl_plan> plan(new sfl_plan);
        plan->impl.kind = SFL_KIND_NS;
        plan->impl.dtype = dtype;
        sfl::cuda_check(cudaGetDevice(&plan->impl.device), "cudaGetDevice");
        plan->impl.ns.reset(new sfl::NSPlan);
        sfl::ns_plan_init(*plan->impl.ns, q, d, dtype, true);
        apply_tuned(plan.get());
        *out = plan.release();
        return SFL_OK;
    });
}

int sfl_surf_plan_create(const sfl_surf_params* p, const int32_t dims[3], int32_t dtype, sfl_plan** out) {
    return guarded([&] {
        need(p, "params");
        need(out, "out");
        *out = nullptr;
        if (dtype != SFL_REAL32 && dtype != SFL_COMPLEX64) throw sfl::ArgError("dtype must be SFL_REAL32 or SFL_COMPLEX64");
        int d[3];
        dims_of(dims, d);
        sfl::surf_check_params(*p);
        sfl::surf_layout_sizes(*p, d);
        std::unique_ptr<sfl_plan> plan(new sfl_plan);
        plan->impl.kind = SFL_KIND_DECIMATED;
        plan->impl.dtype = dtype;
        sfl::cuda_check(cudaGetDevice(&plan->impl.device), "cudaGetDevice");
        sfl::dec_plan_create(plan->impl, *p, d, dtype);
        *out = plan.release();
        return SFL_OK;
    });
}

}  // extern "C"

extern "C" {

int sfl_plan_destroy(sfl_plan* plan) {
    return guarded([&] {
        if (!plan) return SFL_OK;
        on_device(plan, [&] {
            cudaDeviceSynchronize();
            plan->impl.dec.reset();
            plan->impl.ns.reset();
        });
        delete plan;
        return SFL_OK;
    });
}

int sfl_plan_info(const sfl_plan* plan, int32_t* kind, int32_t dims[3], int32_t* dtype, int32_t* nsubbands,
                  int64_t* ncoeffs) {
    return guarded([&] {
        need(plan, "plan");
        const sfl::Plan& P = plan->impl;
        if (kind) *kind = P.kind == SFL_KIND_NS && P.ns->ndfb ? SFL_KIND_NDFB : P.kind;
        if (dtype) *dtype = P.dtype;
        if (P.kind == SFL_KIND_NS) {
            const sfl::NSPlan& N = *P.ns;
            if (dims)
                for (int i = 0; i < 3; ++i) dims[i] = N.dims[i];
            if (nsubbands) *nsubbands = N.S;
            if (ncoeffs) *ncoeffs = N.N * N.S;
        } else {
            const sfl::SurfDesign& D = sfl::dec_design(*P.dec);
            if (dims)
                for (int i = 0; i < 3; ++i) dims[i] = D.dims[i];
            if (nsubbands) *nsubbands = sfl::dec_nsubbands(*P.dec);
            if (ncoeffs) *ncoeffs = sfl::dec_ncoeffs(*P.dec);
        }
        return SFL_OK;
    });
}

int sfl_subband_info(const sfl_plan* plan, int32_t i, int32_t shape[3], int64_t* offset) {
    return guarded([&] {
        need(plan, "plan");
        const sfl::Plan& P = plan->impl;
        int n = P.kind == SFL_KIND_NS ? P.ns->S : sfl::dec_nsubbands(*P.dec);
        if (i < 1 || i > n)
            throw sfl::ArgError("subband index " + std::to_string(i) + " out of range 1:" + std::to_string(n));
        int sh[3];
        long long off;
        if (P.kind == SFL_KIND_NS) {
            for (int k = 0; k < 3; ++k) sh[k] = P.ns->dims[k];
            off = (long long)(i - 1) * P.ns->N;
        } else {
            sfl::dec_subband_info(*P.dec, i, sh, &off);
        }
        if (shape)
            for (int k = 0; k < 3; ++k) shape[k] = sh[k];
        if (offset) *offset = off;
        return SFL_OK;
    });
}

int sfl_plan_status(sfl_plan* plan, int32_t* status, int32_t reset) {
    return guarded([&] {
        need(plan, "plan");
        need(status, "status");
        *status = 0;
        if (plan->impl.kind == SFL_KIND_NS) {
            on_device(plan, [&] {
                // the word is host memory the kernels store to: wait for the device's work first
                sfl::cuda_check(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
                *status = plan->impl.ns->status.read();
                if (reset) plan->impl.ns->status.clear();
            });
        }
        return SFL_OK;
    });
}

int sfl_plan_set_group(sfl_plan* plan, int32_t group) {
    return guarded([&] {
        need(plan, "plan");
        if (group < 1) throw sfl::ArgError("group must be ≥ 1, got " + std::to_string(group));
        if (plan->impl.kind == SFL_KIND_NS) {
            sfl::NSPlan& N = *plan->impl.ns;
            if (N.stream_mode != 0) throw sfl::ArgError("a streaming pass is in progress on this plan");
            int g = std::min<int>(group, N.S);
            on_device(plan, [&] {
                cudaDeviceSynchronize();
                N.group = g;
                sfl::ns_alloc_scratch(N);
            });
        }
        return SFL_OK;
    });
}

int sfl_plan_set_pipeline(sfl_plan* plan, int32_t pipeline) {
    return guarded([&] {
        need(plan, "plan");
        if (plan->impl.kind != SFL_KIND_NS) throw sfl::ArgError("pipeline selection applies to NSSurfacelet plans");
        sfl::NSPlan& N = *plan->impl.ns;
        if (N.stream_mode != 0) throw sfl::ArgError("a streaming pass is in progress on this plan");
        on_device(plan, [&] { ns_apply(N, pipeline, 0); });
        return SFL_OK;
    });
}

int sfl_plan_tuning(const sfl_plan* plan, int32_t* pipeline, int32_t* group) {
    return guarded([&] {
        need(plan, "plan");
        if (plan->impl.kind != SFL_KIND_NS) {
            if (pipeline) *pipeline = -1;
            if (group) *group = 0;
            return SFL_OK;
        }
        const sfl::NSPlan& N = *plan->impl.ns;
        if (pipeline) *pipeline = ns_pipeline_of(N);
        if (group) *group = N.group;
        return SFL_OK;
    });
}

int sfl_plan_autotune(sfl_plan* plan, const void* x, void* c, void* stream) {
    return guarded([&] {
        need(plan, "plan");
        need(x, "x");
        need(c, "c");
        if (plan->impl.kind != SFL_KIND_NS) return SFL_OK;   // the decimated transform has no knobs
        sfl::NSPlan& N = *plan->impl.ns;
        if (N.stream_mode != 0) throw sfl::ArgError("a streaming pass is in progress on this plan");
        check_aligned(x, plan->impl.dtype, "x");
        check_aligned(c, plan->impl.dtype, "c");
        on_device(plan, [&] {
            cudaStream_t st = as_stream(stream);
            cudaEvent_t e0, e1;
            sfl::cuda_check(cudaEventCreate(&e0), "cudaEventCreate");
            sfl::cuda_check(cudaEventCreate(&e1), "cudaEventCreate");
            // analysis, then synthesis of its coefficients into a scratch volume, twice after a warm-up
            sfl::DevMem y;
            y.alloc(sizeof(float) * (size_t)N.N * N.nch);
            auto time_it = [&](int pipe, int g, int ipc) {
                ns_apply(N, pipe, g, ipc);
                sfl::ns_analyze(N, x, c, st, false);   // warm-up
                sfl::cuda_check(cudaEventRecord(e0, st), "cudaEventRecord");
                for (int r = 0; r < 2; ++r) {
                    sfl::ns_analyze(N, x, c, st, false);
                    sfl::ns_synthesize(N, c, y.p, st, false);
                }
                sfl::cuda_check(cudaEventRecord(e1, st), "cudaEventRecord");
                sfl::cuda_check(cudaEventSynchronize(e1), "cudaEventSynchronize");
                float ms = 0;
                sfl::cuda_check(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
                return ms;
            };
            Tuning pick{ns_pipeline_of(N), N.group, N.ipc};
            float best = 1e30f;
            try {
                std::vector<int> pipes;
                if (sfl::ns_slab_supported(N.dims[0], N.dims[1], N.dims[2])) pipes.push_back(SFL_PIPELINE_SLABS);
                pipes.push_back(SFL_PIPELINE_LINES);
                // pipeline x group at the default tile, then the slab tile (subbands a CTA of the axis-3
                // analysis pass) for the best group
                for (int pipe : pipes)
                    for (int g : {2, 4, 8}) {
                        if (g > N.S && g != 2) continue;
                        const float ms = time_it(pipe, g, 0);
                        if (ms < best) {
                            best = ms;
                            pick = {pipe, g, 0};
                        }
                    }
                if (pick.pipeline == SFL_PIPELINE_SLABS)
                    for (int ipc : {1, 2, 4}) {
                        const float ms = time_it(pick.pipeline, pick.group, ipc);
                        if (ms < best) {
                            best = ms;
                            pick.ipc = ipc;
                        }
                    }
            } catch (...) {
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                throw;
            }
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            ns_apply(N, pick.pipeline, pick.group, pick.ipc);
            std::lock_guard<std::mutex> lk(g_tuned_mu);
            g_tuned[tune_key(N, plan->impl.dtype)] = pick;
        });
        return SFL_OK;
    });
}

int sfl_analyze(sfl_plan* plan, const void* x, void* c, void* stream) {
    return guarded([&] {
        need(plan, "plan");
        check_timeout(plan);
        need(x, "x");
        need(c, "c");
        check_aligned(x, plan->impl.dtype, "x");
        check_aligned(c, plan->impl.dtype, "c");
        on_device(plan, [&] {
            if (plan->impl.kind == SFL_KIND_NS)
                sfl::ns_analyze(*plan->impl.ns, x, c, as_stream(stream), false);
            else
                sfl::dec_analyze(*plan->impl.dec, x, c, as_stream(stream));
        });
        return SFL_OK;
    });
}

int sfl_synthesize(sfl_plan* plan, const void* c, void* x, void* stream) {
    return guarded([&] {
        need(plan, "plan");
        check_timeout(plan);
        need(x, "x");
        need(c, "c");
        check_aligned(x, plan->impl.dtype, "x");
        check_aligned(c, plan->impl.dtype, "c");
        on_device(plan, [&] {
            if (plan->impl.kind == SFL_KIND_NS)
                sfl::ns_synthesize(*plan->impl.ns, c, x, as_stream(stream), false);
            else
                sfl::dec_synthesize(*plan->impl.dec, c, x, as_stream(stream));
        });
        return SFL_OK;
    });
}

int sfl_adjoint_analyze(sfl_plan* plan, const void* c, void* x, void* stream) {
    return guarded([&] {
        need(plan, "plan");
        check_timeout(plan);
        need(x, "x");
        need(c, "c");
        check_aligned(x, plan->impl.dtype, "x");
        check_aligned(c, plan->impl.dtype, "c");
        on_device(plan, [&] {
            if (plan->impl.kind == SFL_KIND_NS)
                sfl::ns_synthesize(*plan->impl.ns, c, x, as_stream(stream), true);
            else
                sfl::dec_adjoint_analyze(*plan->impl.dec, c, x, as_stream(stream));
        });
        return SFL_OK;
    });
}

int sfl_adjoint_synthesize(sfl_plan* plan, const void* x, void* c, void* stream) {
    return guarded([&] {
        need(plan, "plan");
        check_timeout(plan);
        need(x, "x");
        need(c, "c");
        check_aligned(x, plan->impl.dtype, "x");
        check_aligned(c, plan->impl.dtype, "c");
        on_device(plan, [&] {
            if (plan->impl.kind == SFL_KIND_NS)
                sfl::ns_analyze(*plan->impl.ns, x, c, as_stream(stream), true);
            else
                sfl::dec_adjoint_synthesize(*plan->impl.dec, x, c, as_stream(stream));
        });
        return SFL_OK;
    });
}

static sfl::NSPlan& ns_of(sfl_plan* plan, const char* what = "streaming") {
    need(plan, "plan");
    if (plan->impl.kind != SFL_KIND_NS)
        throw sfl::ArgError(std::string(what) + " is supported by NSSurfacelet plans only");
    return *plan->impl.ns;
}

int sfl_plan_selftest_wait(sfl_plan* plan, void* stream) {
    return guarded([&] {
        sfl::NSPlan& N = ns_of(plan, "the bounded-wait self-test");
        on_device(plan, [&] { sfl::ns_selftest_wait(N, as_stream(stream)); });
        return SFL_OK;
    });
}

int sfl_plan_tile(sfl_plan* plan, int32_t set, int32_t* ipc) {
    return guarded([&] {
        sfl::NSPlan& N = ns_of(plan, "the axis-3 tile");
        need(ipc, "ipc");
        if (set) {
            if (*ipc != 0 && *ipc != 1 && *ipc != 2 && *ipc != 4 && *ipc != 8)
                throw sfl::ArgError("subbands a CTA must be 1, 2, 4 or 8 (0: the default), got " + std::to_string(*ipc));
            N.ipc = *ipc;
        } else {
            *ipc = N.ipc;
        }
        return SFL_OK;
    });
}

int sfl_stream_analyze_begin(sfl_plan* plan, const void* x, void* stream) {
    return guarded([&] {
        sfl::NSPlan& N = ns_of(plan);
        check_timeout(plan);
        need(x, "x");
        on_device(plan, [&] { sfl::ns_stream_analyze_begin(N, x, as_stream(stream)); });
        return SFL_OK;
    });
}

int sfl_stream_analyze_next(sfl_plan* plan, void* band, int32_t* index, void* stream) {
    return guarded([&] {
        sfl::NSPlan& N = ns_of(plan);
        check_timeout(plan);
        need(band, "band");
        need(index, "index");
        int r = SFL_OK, idx = 0;
        on_device(plan, [&] { r = sfl::ns_stream_analyze_next(N, band, &idx, as_stream(stream)); });
        if (r == SFL_OK) *index = idx;
        return r;
    });
}

int sfl_stream_synthesize_begin(sfl_plan* plan, void* stream) {
    return guarded([&] {
        sfl::NSPlan& N = ns_of(plan);
        check_timeout(plan);
        sfl::ns_stream_synth_begin(N, as_stream(stream));
        return SFL_OK;
    });
}

int sfl_stream_synthesize_next_index(sfl_plan* plan, int32_t* index) {
    return guarded([&] {
        sfl::NSPlan& N = ns_of(plan);
        need(index, "index");
        int idx = 0;
        int r = sfl::ns_stream_synth_next_index(N, &idx);
        if (r == SFL_OK) *index = idx;
        return r;
    });
}

int sfl_stream_synthesize_push(sfl_plan* plan, const void* band, void* stream) {
    return guarded([&] {
        sfl::NSPlan& N = ns_of(plan);
        check_timeout(plan);
        need(band, "band");
        on_device(plan, [&] { sfl::ns_stream_synth_push(N, band, as_stream(stream)); });
        return SFL_OK;
    });
}

int sfl_stream_synthesize_end(sfl_plan* plan, void* x, void* stream) {
    return guarded([&] {
        sfl::NSPlan& N = ns_of(plan);
        check_timeout(plan);
        need(x, "x");
        on_device(plan, [&] { sfl::ns_stream_synth_end(N, x, as_stream(stream)); });
        return SFL_OK;
    });
}

int sfl_ns_analyze_subband_static(sfl_plan* plan, const void* x, void* band, int32_t index, void* stream) {
    return guarded([&] {
        sfl::NSPlan& N = ns_of(plan, "sfl_ns_analyze_subband_static");
        need(x, "x");
        need(band, "band");
        check_aligned(x, plan->impl.dtype, "x");
        check_aligned(band, plan->impl.dtype, "band");
        on_device(plan, [&] { sfl::ns_analyze_subband_static(N, x, band, index, as_stream(stream)); });
        return SFL_OK;
    });
}

int sfl_ns_design_table(const sfl_ns_params* p, const int32_t dims[3], const char* name, int32_t index,
                        double* out, int64_t* count) {
    return guarded([&] {
        need(p, "params");
        need(name, "name");
        need(count, "count");
        int d[3];
        dims_of(dims, d);
        sfl::NSDesign D = sfl::ns_design(*p, d);
        const std::vector<double>* v = nullptr;
        std::vector<double> tmp;
        std::string nm(name);
        if (nm == "m1") {
            v = &D.m1;
        } else if (nm == "m2") {
            v = &D.m2;
        } else if (nm == "wedge") {
            int w = index % 64, plane = (index / 64) % 2, hi = (index / 128) % 3, j = index / 384;
            if (j >= p->scales) throw sfl::ArgError("wedge table index out of range");
            const sfl::WedgePlanes& W = D.wedges[j][hi][plane];
            if (w >= (int)W.w.size()) throw sfl::ArgError("wedge table index out of range");
            v = &W.w[w];
        } else if (nm == "group") {
            // plan order: g = 3 (scale - 1) + hourglass - 1
            if (index < 0 || index >= 3 * p->scales) throw sfl::ArgError("group index out of range");
            tmp = sfl::ns_group_mask(D, p->scales - 1 - index / 3, index % 3 + 1, true);
            v = &tmp;
        } else if (nm == "bandpass") {
            if (index < 0 || index >= p->scales) throw sfl::ArgError("level out of range");
            tmp = sfl::ns_group_mask(D, index, 1, false);
            v = &tmp;
        } else if (nm == "hourglass") {
            if (index < 0 || index >= 3) throw sfl::ArgError("hourglass index out of range");
            tmp = sfl::ns_hourglass_mask(D, index + 1);
            v = &tmp;
        } else if (nm == "pa" || nm == "pl") {
            int lv = index / 3, ax = index % 3;
            auto& tab = nm == "pa" ? D.pa : D.pl;
            if (lv < 0 || lv >= (int)tab.size()) throw sfl::ArgError("level out of range");
            v = &tab[lv][ax];
        } else {
            throw sfl::ArgError("unknown table " + nm);
        }
        *count = (int64_t)v->size();
        if (out) std::memcpy(out, v->data(), sizeof(double) * v->size());
        return SFL_OK;
    });
}

int sfl_ns_plan_table(sfl_plan* plan, const char* name, int32_t index, float* out, int64_t* count) {
    return guarded([&] {
        sfl::NSPlan& N = ns_of(plan);
        need(name, "name");
        need(count, "count");
        std::string nm(name);
        const sfl::DevMem* m = nullptr;
        int n = 0;
        if (nm == "group") {
            m = &N.G;
            n = N.ndfb ? 3 : 3 * N.p.scales;
        } else if (nm == "bandpass") {
            m = &N.Bl;
            n = N.p.tight ? 0 : (N.ndfb ? 1 : N.p.scales);
        } else {
            throw sfl::ArgError("unknown table " + nm);
        }
        if (index < 0 || index >= n) throw sfl::ArgError("table index out of range");
        *count = N.H;
        if (out)
            on_device(plan, [&] {
                sfl::cuda_check(cudaMemcpy(out, m->as<float>() + (size_t)index * N.H, sizeof(float) * N.H,
                                           cudaMemcpyDeviceToHost),
                                "table readback");
            });
        return SFL_OK;
    });
}

int sfl_surf_plan_table(sfl_plan* plan, const char* name, int32_t index, float* out, int64_t* count) {
    return guarded([&] {
        need(plan, "plan");
        need(name, "name");
        need(count, "count");
        if (plan->impl.kind != SFL_KIND_DECIMATED) throw sfl::ArgError("sfl_surf_plan_table takes Surfacelet plans");
        long long n = 0;
        const float* src = sfl::dec_plan_table(*plan->impl.dec, name, index, &n);
        *count = n;
        if (out)
            on_device(plan, [&] {
                sfl::cuda_check(cudaMemcpy(out, src, sizeof(float) * n, cudaMemcpyDeviceToHost), "table readback");
            });
        return SFL_OK;
    });
}

int sfl_surf_design_table(const sfl_surf_params* p, const int32_t dims[3], const char* name, int32_t index,
                          double* out, int64_t* count) {
    return guarded([&] {
        need(p, "params");
        need(name, "name");
        need(count, "count");
        int d[3];
        dims_of(dims, d);
        sfl::SurfDesign S = sfl::surf_design(*p, d);
        std::string nm(name);
        std::vector<double> tmp;
        if (nm == "ritf") {
            int lv = index / 3, K = index % 3;
            if (lv >= (int)S.scales.size()) throw sfl::ArgError("level out of range");
            tmp = S.scales[lv].V[K];
        } else if (nm == "irc") {
            int which = index % 4, stage = (index / 4) % 32, K = (index / 128) % 3, lv = index / 384;
            if (lv >= (int)S.scales.size() || stage >= (int)S.scales[lv].stages[K].size())
                throw sfl::ArgError("stage out of range");
            const sfl::IRCStage& st = S.scales[lv].stages[K][stage];
            const std::vector<std::complex<double>>& f = which < 2 ? st.ana[which] : st.syn[which - 2];
            for (auto z : f) {
                tmp.push_back(z.real());
                tmp.push_back(z.imag());
            }
        } else if (nm == "pyr_prof") {
            int lv = index / 3, ax = index % 3;
            if (lv >= (int)S.pyramid.size()) throw sfl::ArgError("level out of range");
            tmp = S.pyramid[lv].prof[ax];
        } else {
            throw sfl::ArgError("unknown table " + nm);
        }
        *count = (int64_t)tmp.size();
        if (out) std::memcpy(out, tmp.data(), sizeof(double) * tmp.size());
        return SFL_OK;
    });
}

int sfl_ns_analyze_bf16(sfl_plan* plan, const void* x, void* c, float* scales, void* stream) {
    return guarded([&] {
        need(x, "x");
        need(c, "c");
        need(scales, "scales");
        sfl::NSPlan& N = ns_of(plan, "bfloat16 coefficients");
        check_timeout(plan);
        if (N.stream_mode != 0) throw sfl::ArgError("a streaming pass is in progress on this plan");
        check_aligned(x, plan->impl.dtype, "x");
        if (reinterpret_cast<uintptr_t>(c) % 2 != 0) throw sfl::ArgError("c is not aligned to its element type");
        on_device(plan, [&] { sfl::ns_analyze_bf16(N, static_cast<const float*>(x), c, scales, as_stream(stream)); });
        return SFL_OK;
    });
}

int sfl_ns_synthesize_bf16(sfl_plan* plan, const void* c, const float* scales, void* x, void* stream) {
    return guarded([&] {
        need(x, "x");
        need(c, "c");
        need(scales, "scales");
        sfl::NSPlan& N = ns_of(plan, "bfloat16 coefficients");
        check_timeout(plan);
        if (N.stream_mode != 0) throw sfl::ArgError("a streaming pass is in progress on this plan");
        check_aligned(x, plan->impl.dtype, "x");
        if (reinterpret_cast<uintptr_t>(c) % 2 != 0) throw sfl::ArgError("c is not aligned to its element type");
        on_device(plan, [&] { sfl::ns_synthesize_bf16(N, c, scales, static_cast<float*>(x), as_stream(stream)); });
        return SFL_OK;
    });
}

int sfl_ns_denoise(sfl_plan* plan, const void* x, void* y, const float* tau, void* stream) {
    return guarded([&] {
        need(x, "x");
        need(y, "y");
        need(tau, "tau");
        sfl::NSPlan& N = ns_of(plan, "the denoiser");
        check_timeout(plan);
        if (N.stream_mode != 0) throw sfl::ArgError("a streaming pass is in progress on this plan");
        check_aligned(x, plan->impl.dtype, "x");
        check_aligned(y, plan->impl.dtype, "y");
        on_device(plan, [&] {
            sfl::ns_denoise(N, static_cast<const float*>(x), static_cast<float*>(y), tau, as_stream(stream));
        });
        return SFL_OK;
    });
}

// ── item ranges (sharding subbands across devices) ──────────────────────────

static sfl::NSPlan& range_plan(sfl_plan* plan) {
    sfl::NSPlan& N = ns_of(plan, "item ranges");
    if (N.stream_mode != 0) throw sfl::ArgError("a streaming pass is in progress on this plan");
    return N;
}

static void check_range(const sfl::NSPlan& N, int32_t first, int32_t count) {
    if (first < 0 || count < 0 || first + count > N.S)
        throw sfl::ArgError("stream positions [" + std::to_string(first) + ", " + std::to_string(first + count) +
                            ") are outside [0, " + std::to_string(N.S) + ")");
}

int sfl_ns_spectrum_elems(const sfl_plan* plan, int64_t* elems) {
    return guarded([&] {
        need(plan, "plan");
        need(elems, "elems");
        if (plan->impl.kind != SFL_KIND_NS) throw sfl::ArgError("item ranges are supported by NSSurfacelet plans only");
        *elems = sfl::ns_spec_elems(*plan->impl.ns);
        return SFL_OK;
    });
}

int sfl_ns_stream_order(const sfl_plan* plan, int32_t* subband_index) {
    return guarded([&] {
        need(plan, "plan");
        need(subband_index, "subband_index");
        if (plan->impl.kind != SFL_KIND_NS) throw sfl::ArgError("item ranges are supported by NSSurfacelet plans only");
        const sfl::NSPlan& N = *plan->impl.ns;
        for (int i = 0; i < N.S; ++i) subband_index[i] = N.items_host[i].s;
        return SFL_OK;
    });
}

int sfl_ns_forward_spectrum(sfl_plan* plan, const void* x, void* X, void* stream) {
    return guarded([&] {
        sfl::NSPlan& N = range_plan(plan);
        check_timeout(plan);
        need(x, "x");
        need(X, "X");
        check_spectrum_aligned(X, "X");
        check_aligned(x, plan->impl.dtype, "x");
        const long long E = sfl::ns_spec_elems(N);
        on_device(plan, [&] {
            for (int ch = 0; ch < N.nch; ++ch)
                sfl::ns_forward_spectrum(N, static_cast<const float*>(x) + ch, N.nch, static_cast<float2*>(X) + ch * E,
                                         as_stream(stream));
        });
        return SFL_OK;
    });
}

int sfl_ns_analyze_range(sfl_plan* plan, const void* X, int32_t first, int32_t count, void* c, void* stream) {
    return guarded([&] {
        sfl::NSPlan& N = range_plan(plan);
        check_timeout(plan);
        need(X, "X");
        check_spectrum_aligned(X, "X");
        need(c, "c");
        check_aligned(c, plan->impl.dtype, "c");
        check_range(N, first, count);
        const long long E = sfl::ns_spec_elems(N);
        on_device(plan, [&] {
            for (int ch = 0; ch < N.nch; ++ch)
                for (int i0 = first, i1; i0 < first + count; i0 = i1) {
                    i1 = std::min(sfl::ns_next_chunk(N, i0), first + count);
                    sfl::ZMap vz;
                    vz.zstride = N.N * N.nch;
                    float* base = static_cast<float*>(c) + (long long)(i0 - first) * N.N * N.nch + ch;
                    sfl::ns_analyze_range(N, static_cast<const float2*>(X) + ch * E, base, vz, N.nch, i0, i1 - i0,
                                          false, as_stream(stream));
                }
        });
        return SFL_OK;
    });
}

int sfl_ns_accumulate_range(sfl_plan* plan, const void* c, int32_t first, int32_t count, void* A, int32_t clear,
                            void* stream) {
    return guarded([&] {
        sfl::NSPlan& N = range_plan(plan);
        check_timeout(plan);
        need(c, "c");
        need(A, "A");
        check_spectrum_aligned(A, "A");
        check_aligned(c, plan->impl.dtype, "c");
        check_range(N, first, count);
        const long long E = sfl::ns_spec_elems(N);
        on_device(plan, [&] {
            for (int ch = 0; ch < N.nch; ++ch) {
                float2* acc = static_cast<float2*>(A) + ch * E;
                float2* comp = sfl::ns_comp_grid(N, ch);
                if (clear) sfl::ns_acc_clear(N, acc, comp, as_stream(stream));
                for (int i0 = first, i1; i0 < first + count; i0 = i1) {
                    i1 = std::min(sfl::ns_next_chunk(N, i0), first + count);
                    sfl::ZMap vz;
                    vz.zstride = N.N * N.nch;
                    const float* base = static_cast<const float*>(c) + (long long)(i0 - first) * N.N * N.nch + ch;
                    sfl::ns_accumulate_range(N, base, vz, N.nch, i0, i1 - i0, false, acc, comp, as_stream(stream));
                }
            }
        });
        return SFL_OK;
    });
}

int sfl_ns_inverse_spectrum(sfl_plan* plan, void* A, void* x, void* stream) {
    return guarded([&] {
        sfl::NSPlan& N = range_plan(plan);
        check_timeout(plan);
        need(A, "A");
        check_spectrum_aligned(A, "A");
        need(x, "x");
        check_aligned(x, plan->impl.dtype, "x");
        const long long E = sfl::ns_spec_elems(N);
        on_device(plan, [&] {
            for (int ch = 0; ch < N.nch; ++ch)
                sfl::ns_inverse_spectrum(N, static_cast<float2*>(A) + ch * E, static_cast<float*>(x) + ch, N.nch,
                                         as_stream(stream));
        });
        return SFL_OK;
    });
}

// ── batches: one CUDA graph over many transforms ─────────────────────────────

// Estimated work of one batch entry: the volume's voxels times (1 + coefficients a voxel); a volume copy
// counts as its voxels.
static double entry_work(const sfl_plan* plan, int op) {
    const sfl::Plan& P = plan->impl;
    double vox = 1, coef = 0;
    if (P.kind == SFL_KIND_NS) {
        vox = (double)P.ns->N;
        coef = (double)P.ns->S;
    } else {
        for (int d = 0; d < 3; ++d) vox *= sfl::dec_design(*P.dec).dims[d];
        coef = (double)sfl::dec_ncoeffs(*P.dec) / vox;
    }
    return op == SFL_OP_COPY_VOLUME ? vox : vox * (1 + coef);
}

int sfl_batch_create(int32_t n, sfl_plan* const* plans, const int32_t* ops, const void* const* inputs,
                     void* const* outputs, sfl_batch** out) {
    return guarded([&] {
        need(plans, "plans");
        need(ops, "ops");
        need(inputs, "inputs");
        need(outputs, "outputs");
        need(out, "out");
        *out = nullptr;
        if (n < 1) throw sfl::ArgError("a batch needs at least one transform, got " + std::to_string(n));
        const int dev = (need(plans[0], "plans[0]"), plans[0]->impl.device);
        // distinct plans run on up to kBranches concurrent branches; one plan always on the same branch, the
        // plans dealt out largest first to the branch with the least work so far (longest-processing-time
        // order), the work of an entry estimated as voxels x (1 + coefficients per voxel)
        constexpr int kBranches = 8;
        std::vector<const sfl_plan*> distinct;
        std::vector<double> work;
        std::vector<int> plan_of(n);
        std::vector<int> branch(n);
        for (int i = 0; i < n; ++i) {
            need(plans[i], "plans[i]");
            if (ops[i] < SFL_OP_ANALYZE || ops[i] > SFL_OP_COPY_VOLUME)
                throw sfl::ArgError("unknown operator " + std::to_string(ops[i]));
            need(inputs[i], "inputs[i]");
            need(outputs[i], "outputs[i]");
            if (plans[i]->impl.device != dev) throw sfl::ArgError("the plans of a batch must share one device");
            if (plans[i]->impl.kind == SFL_KIND_NS && plans[i]->impl.ns->stream_mode != 0)
                throw sfl::ArgError("a streaming pass is open on a plan of the batch");
            if (ops[i] != SFL_OP_COPY_VOLUME) {
                check_aligned(inputs[i], plans[i]->impl.dtype, "inputs[i]");
                check_aligned(outputs[i], plans[i]->impl.dtype, "outputs[i]");
            }
            auto it = std::find(distinct.begin(), distinct.end(), plans[i]);
            if (it == distinct.end()) {
                distinct.push_back(plans[i]);
                work.push_back(0.0);
                it = distinct.end() - 1;
            }
            plan_of[i] = (int)(it - distinct.begin());
            work[plan_of[i]] += entry_work(plans[i], ops[i]);
        }
        {
            std::vector<int> order(distinct.size());
            for (size_t k = 0; k < order.size(); ++k) order[k] = (int)k;
            std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return work[x] > work[y]; });
            std::vector<double> load(kBranches, 0.0);
            std::vector<int> br(distinct.size());
            for (int k : order) {
                const int to = (int)(std::min_element(load.begin(), load.end()) - load.begin());
                br[k] = to;
                load[to] += work[k];
            }
            for (int i = 0; i < n; ++i) branch[i] = br[plan_of[i]];
        }
        std::unique_ptr<sfl_batch> b(new sfl_batch());
        b->device = dev;
        on_device(plans[0], [&] {
            cudaStream_t s[kBranches] = {};
            cudaEvent_t fork = nullptr, join[kBranches] = {};
            auto cleanup = [&] {
                for (auto& e : join)
                    if (e) cudaEventDestroy(e);
                if (fork) cudaEventDestroy(fork);
                for (auto& x : s)
                    if (x) cudaStreamDestroy(x);
            };
            const bool prof = sfl::prof_on();
            try {
                for (auto& x : s) sfl::cuda_check(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking), "stream");
                sfl::cuda_check(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming), "event");
                for (auto& e : join) sfl::cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
                // the graph's branches run concurrently: launch shapes for that (the eager pass too, so that it
                // configures the kernels the capture records)
                struct Concurrent {
                    explicit Concurrent(bool on) { sfl::ns_set_concurrent(on); }
                    ~Concurrent() { sfl::ns_set_concurrent(false); }
                } concurrent(distinct.size() > 1);
                // one eager pass: validates the arguments and configures every kernel outside the capture
                for (int i = 0; i < n; ++i) run_op(plans[i], ops[i], inputs[i], outputs[i], s[0]);
                sfl::cuda_check(cudaStreamSynchronize(s[0]), "batch warm-up");
                sfl_profile_enable(0);
                sfl::cuda_check(cudaStreamBeginCapture(s[0], cudaStreamCaptureModeThreadLocal), "begin capture");
                try {
                    sfl::cuda_check(cudaEventRecord(fork, s[0]), "fork");
                    for (int k = 1; k < kBranches; ++k) sfl::cuda_check(cudaStreamWaitEvent(s[k], fork, 0), "fork");
                    for (int i = 0; i < n; ++i) run_op(plans[i], ops[i], inputs[i], outputs[i], s[branch[i]]);
                    for (int k = 1; k < kBranches; ++k) {
                        sfl::cuda_check(cudaEventRecord(join[k], s[k]), "join");
                        sfl::cuda_check(cudaStreamWaitEvent(s[0], join[k], 0), "join");
                    }
                } catch (...) {
                    cudaGraph_t g = nullptr;
                    cudaStreamEndCapture(s[0], &g);
                    if (g) cudaGraphDestroy(g);
                    throw;
                }
                sfl::cuda_check(cudaStreamEndCapture(s[0], &b->graph), "end capture");
                sfl::cuda_check(cudaGraphInstantiate(&b->exec, b->graph, 0), "cudaGraphInstantiate");
                sfl_profile_enable(prof ? 1 : 0);
            } catch (...) {
                sfl_profile_enable(prof ? 1 : 0);
                cleanup();
                throw;
            }
            cleanup();
        });
        *out = b.release();
        return SFL_OK;
    });
}

int sfl_batch_run(sfl_batch* batch, void* stream) {
    return guarded([&] {
        need(batch, "batch");
        int cur = 0;
        sfl::cuda_check(cudaGetDevice(&cur), "cudaGetDevice");
        if (cur != batch->device) sfl::cuda_check(cudaSetDevice(batch->device), "cudaSetDevice");
        cudaError_t e = cudaGraphLaunch(batch->exec, as_stream(stream));
        if (cur != batch->device) cudaSetDevice(cur);
        sfl::cuda_check(e, "cudaGraphLaunch");
        return SFL_OK;
    });
}

int sfl_batch_destroy(sfl_batch* batch) {
    return guarded([&] {
        if (!batch) return SFL_OK;
        int cur = 0;
        const int dev = batch->device;
        sfl::cuda_check(cudaGetDevice(&cur), "cudaGetDevice");
        if (cur != dev) cudaSetDevice(dev);
        delete batch;
        if (cur != dev) cudaSetDevice(cur);
        return SFL_OK;
    });
}

}  // extern "C"
