#include "prof.h"

#include <cuda_runtime.h>

#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/surfacelets_b200.h"

namespace sfl {

namespace {

struct Rec {
    std::string tag;
    cudaEvent_t a, b;
};

std::mutex g_mu;
bool g_on = false;
std::vector<Rec> g_recs;
std::map<std::string, double> g_bytes;

}  // namespace

bool prof_on() { return g_on; }

int prof_begin(const char* tag, cudaStream_t st) {
    if (!g_on) return -1;
    Rec r;
    r.tag = tag;
    if (cudaEventCreate(&r.a) != cudaSuccess || cudaEventCreate(&r.b) != cudaSuccess) return -1;
    cudaEventRecord(r.a, st);
    std::lock_guard<std::mutex> lk(g_mu);
    g_recs.push_back(r);
    return (int)g_recs.size() - 1;
}

void prof_end(int token, cudaStream_t st) {
    if (token < 0) return;
    std::lock_guard<std::mutex> lk(g_mu);
    if (token < (int)g_recs.size()) cudaEventRecord(g_recs[token].b, st);
}

void prof_bytes(const char* tag, double bytes) {
    if (!g_on) return;
    std::lock_guard<std::mutex> lk(g_mu);
    g_bytes[tag] += bytes;
}

}  // namespace sfl

extern "C" {

int sfl_profile_enable(int32_t on) {
    sfl::g_on = on != 0;
    return SFL_OK;
}

int sfl_profile_reset(void) {
    std::lock_guard<std::mutex> lk(sfl::g_mu);
    for (auto& r : sfl::g_recs) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    sfl::g_recs.clear();
    sfl::g_bytes.clear();
    return SFL_OK;
}

int sfl_profile_bytes(const char* tag, double* bytes) {
    std::lock_guard<std::mutex> lk(sfl::g_mu);
    double b = 0;
    for (auto& kv : sfl::g_bytes)
        if (!tag || kv.first == tag) b += kv.second;
    if (bytes) *bytes = b;
    return SFL_OK;
}

int sfl_profile_read(const char* tag, double* total_ms, int64_t* launches) {
    std::lock_guard<std::mutex> lk(sfl::g_mu);
    double tot = 0;
    int64_t n = 0;
    for (auto& r : sfl::g_recs) {
        if (tag && r.tag != tag) continue;
        if (cudaEventSynchronize(r.b) != cudaSuccess) return SFL_ERR_CUDA;
        float ms = 0;
        if (cudaEventElapsedTime(&ms, r.a, r.b) != cudaSuccess) return SFL_ERR_CUDA;
        tot += ms;
        ++n;
    }
    if (total_ms) *total_ms = tot;
    if (launches) *launches = n;
    return SFL_OK;
}

int sfl_profile_tags(char* buf, int64_t cap) {
    std::lock_guard<std::mutex> lk(sfl::g_mu);
    std::map<std::string, int> seen;
    std::string out;
    for (auto& r : sfl::g_recs)
        if (!seen.count(r.tag)) {
            seen[r.tag] = 1;
            out += r.tag + "\n";
        }
    if (buf && cap > 0) {
        std::strncpy(buf, out.c_str(), (size_t)cap - 1);
        buf[cap - 1] = 0;
    }
    return (int)out.size();
}

}  // extern "C"
