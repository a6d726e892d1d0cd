// Per-kernel CUDA-event timing on the context's stream (pfag_set_profile).
// Each instrumented launch is bracketed by an event pair recorded on the
// stream it runs on; pfag_profile_read synchronises, accumulates the elapsed
// times by kernel name and clears the record.
#include "pfag_internal.cuh"
#include <cstring>
#include <map>
#include <string>
#include <vector>

struct ProfRec { const char *name; cudaEvent_t a, b; };
struct ProfState {
    bool on = false;
    std::vector<ProfRec> recs;
    std::vector<cudaEvent_t> pool;
    std::map<std::string, std::pair<double, long>> acc;
};

static ProfState *PS(pfag_ctx *c) { return (ProfState *)c->prof; }

static cudaEvent_t take_event(ProfState *p) {
    if (!p->pool.empty()) { cudaEvent_t e = p->pool.back(); p->pool.pop_back(); return e; }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

void pfag_prof_begin(pfag_ctx *c, const char *name) {
    ProfState *p = PS(c);
    if (!p || !p->on) return;
    ProfRec r{name, take_event(p), take_event(p)};
    cudaEventRecord(r.a, c->stream);
    p->recs.push_back(r);
}

void pfag_prof_end(pfag_ctx *c) {
    ProfState *p = PS(c);
    if (!p || !p->on || p->recs.empty()) return;
    cudaEventRecord(p->recs.back().b, c->stream);
}

void pfag_prof_free(pfag_ctx *c) {
    ProfState *p = PS(c);
    if (!p) return;
    for (auto &r : p->recs) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
    for (auto e : p->pool) cudaEventDestroy(e);
    delete p;
    c->prof = nullptr;
}

bool pfag_prof_on(pfag_ctx *c) { return c && c->prof && PS(c)->on; }

extern "C" int pfag_set_profile(pfag_ctx *c, int on) {
    if (!c) return PFAG_E_ARG;
    if (!c->prof) c->prof = new ProfState();
    PS(c)->on = on != 0;
    return PFAG_OK;
}

extern "C" int pfag_profile_read(pfag_ctx *c, char *names, double *ms, long *launches, int cap) {
    if (!c || !c->prof) { pfag_set_error("profiling not enabled"); return PFAG_E_ARG; }
    ProfState *p = PS(c);
    PFAG_CUDA_CHECK(cudaStreamSynchronize(c->stream));
    for (auto &r : p->recs) {
        float t = 0.f;
        PFAG_CUDA_CHECK(cudaEventElapsedTime(&t, r.a, r.b));
        auto &e = p->acc[r.name];
        e.first += t;
        e.second += 1;
        p->pool.push_back(r.a);
        p->pool.push_back(r.b);
    }
    p->recs.clear();
    int k = 0;
    for (auto &kv : p->acc) {
        if (k >= cap) break;
        if (names) { std::strncpy(names + 64 * k, kv.first.c_str(), 63); names[64 * k + 63] = 0; }
        if (ms) ms[k] = kv.second.first;
        if (launches) launches[k] = kv.second.second;
        k++;
    }
    p->acc.clear();
    return k;
}
