// Snapshot output (saving_out_functions, useful_functions.cpp:66-99, and the
// file writer of run_with_active_gels.cpp:193-269) without stalling the steps.
//
// pfag_snapshot_async copies the saved state (phi, rho, lum, ECM) into a
// device staging area on the context's stream (device-to-device, ~0.2 ms for
// a 64-cell 1024^2 FP32 state) and then, on a copy stream that waits for that
// copy, into the caller's host buffers.  The steps that follow on the
// context's stream overlap the transfer; the next snapshot waits for the
// previous transfer before it refills the staging area.  Each call returns a
// ticket; pfag_snapshot_wait(ticket) returns once that snapshot's host copy is
// complete.  Host buffers should be pinned (cudaHostAlloc) for the copy to run
// asynchronously.
//
// pfag_write_text_snapshot writes one N x N table in the reference's text
// layout ("%.15f\n" per value, a blank line after every row,
// run_with_active_gels.cpp:215-229): the digits come from an exact integer
// computation of round-half-even(x * 10^15), formatted by several host
// threads.
#include "pfag_internal.cuh"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace {

constexpr int SNAP_TICKETS = 16;

struct SnapState {
    void *stage = nullptr;         // phi (nc), rho (nc), lum (ng), ECM (ng)
    cudaStream_t copy = nullptr;
    cudaEvent_t staged = nullptr;
    cudaEvent_t done[SNAP_TICKETS] = {};
    long next = 0;                 // next ticket
};

SnapState *SS(pfag_ctx *c) { return static_cast<SnapState *>(c->snap); }

int snap_init(pfag_ctx *c) {
    if (c->snap) return PFAG_OK;
    SnapState *s = new SnapState();
    c->snap = s;
    const size_t bytes = (2 * c->nc + 2 * c->ng) * c->rsz;
    PFAG_CUDA_CHECK(cudaMalloc(&s->stage, bytes));
    PFAG_CUDA_CHECK(cudaStreamCreateWithFlags(&s->copy, cudaStreamNonBlocking));
    PFAG_CUDA_CHECK(cudaEventCreateWithFlags(&s->staged, cudaEventDisableTiming));
    for (auto &e : s->done) PFAG_CUDA_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return PFAG_OK;
}

// %.15f of x as glibc prints it (round half to even on exact ties) for
// |x| < 2^63 / 10^15; false outside that range (the caller uses snprintf).
bool fixed15(double x, char *out, int *len) {
    if (!(x == x)) return false;
    const bool neg = std::signbit(x);
    double a = neg ? -x : x;
    if (a >= 9.0e3) return false;
    int e2;
    const double m = std::frexp(a, &e2);                       // a = m 2^e2, m in [0.5, 1)
    unsigned long long mant = (unsigned long long)std::ldexp(m, 53);   // exact: a = mant 2^(e2-53)
    const int shift = 53 - e2;                                 // a = mant / 2^shift
    unsigned __int128 num = (unsigned __int128)mant * 1000000000000000ULL;   // a 10^15 = num / 2^shift
    unsigned long long q;
    if (a == 0.0) {
        q = 0;
    } else if (shift >= 120) {
        q = 0;                                                 // below 2^-67: rounds to 0
    } else if (shift <= 0) {
        q = (unsigned long long)(num << (-shift));
    } else {
        const unsigned __int128 one = (unsigned __int128)1 << shift;
        unsigned __int128 qq = num >> shift;
        const unsigned __int128 rem = num & (one - 1);
        const unsigned __int128 half = one >> 1;
        if (rem > half || (rem == half && (qq & 1))) qq += 1;
        q = (unsigned long long)qq;
    }
    const unsigned long long ip = q / 1000000000000000ULL, fp = q % 1000000000000000ULL;
    char buf[48];
    int n = 0;
    if (neg) buf[n++] = '-';
    char tmp[24];
    int k = 0;
    unsigned long long v = ip;
    do { tmp[k++] = (char)('0' + v % 10); v /= 10; } while (v);
    while (k) buf[n++] = tmp[--k];
    buf[n++] = '.';
    unsigned long long f = fp;
    for (int d = 14; d >= 0; d--) { buf[n + d] = (char)('0' + f % 10); f /= 10; }
    n += 15;
    std::memcpy(out, buf, n);
    *len = n;
    return true;
}

template <typename real>
void format_rows(const real *t, int N, int i0, int i1, std::string &out) {
    out.clear();
    out.reserve((size_t)(i1 - i0) * ((size_t)N * 19 + 1));
    char b[64];
    for (int i = i0; i < i1; i++) {
        for (int j = 0; j < N; j++) {
            const double x = (double)t[(size_t)i * N + j];
            int len;
            if (!fixed15(x, b, &len)) len = std::snprintf(b, sizeof b, "%.15f", x);
            out.append(b, (size_t)len);
            out.push_back('\n');
        }
        out.push_back('\n');
    }
}

}  // namespace

void pfag_snapshot_free(pfag_ctx *c) {
    SnapState *s = SS(c);
    if (!s) return;
    if (s->copy) cudaStreamSynchronize(s->copy);
    if (s->stage) cudaFree(s->stage);
    if (s->staged) cudaEventDestroy(s->staged);
    for (auto e : s->done) if (e) cudaEventDestroy(e);
    if (s->copy) cudaStreamDestroy(s->copy);
    delete s;
    c->snap = nullptr;
}

extern "C" long pfag_snapshot_async(pfag_ctx *c, void *phi, void *rho, void *lum, void *ecm) {
    if (!c || !phi || !rho || !lum || !ecm) { pfag_set_error("null argument"); return PFAG_E_ARG; }
    PFAG_TRY(snap_init(c));
    SnapState *s = SS(c);
    const size_t rs = c->rsz;
    char *st = static_cast<char *>(s->stage);
    char *st_phi = st, *st_rho = st + c->nc * rs, *st_lum = st + 2 * c->nc * rs, *st_ecm = st_lum + c->ng * rs;
    // the staging area is free once the previous snapshot's host copy is done
    if (s->next > 0) PFAG_CUDA_CHECK(cudaStreamWaitEvent(c->stream, s->done[(s->next - 1) % SNAP_TICKETS], 0));
    PFAG_CUDA_CHECK(cudaMemcpyAsync(st_phi, c->phi, c->nc * rs, cudaMemcpyDeviceToDevice, c->stream));
    PFAG_CUDA_CHECK(cudaMemcpyAsync(st_rho, c->rho, c->nc * rs, cudaMemcpyDeviceToDevice, c->stream));
    PFAG_CUDA_CHECK(cudaMemcpyAsync(st_lum, c->lum, c->ng * rs, cudaMemcpyDeviceToDevice, c->stream));
    PFAG_CUDA_CHECK(cudaMemcpyAsync(st_ecm, c->ecm, c->ng * rs, cudaMemcpyDeviceToDevice, c->stream));
    PFAG_CUDA_CHECK(cudaEventRecord(s->staged, c->stream));
    PFAG_CUDA_CHECK(cudaStreamWaitEvent(s->copy, s->staged, 0));
    PFAG_CUDA_CHECK(cudaMemcpyAsync(phi, st_phi, c->nc * rs, cudaMemcpyDeviceToHost, s->copy));
    PFAG_CUDA_CHECK(cudaMemcpyAsync(rho, st_rho, c->nc * rs, cudaMemcpyDeviceToHost, s->copy));
    PFAG_CUDA_CHECK(cudaMemcpyAsync(lum, st_lum, c->ng * rs, cudaMemcpyDeviceToHost, s->copy));
    PFAG_CUDA_CHECK(cudaMemcpyAsync(ecm, st_ecm, c->ng * rs, cudaMemcpyDeviceToHost, s->copy));
    const long t = s->next++;
    PFAG_CUDA_CHECK(cudaEventRecord(s->done[t % SNAP_TICKETS], s->copy));
    return t;
}

extern "C" int pfag_snapshot_wait(pfag_ctx *c, long ticket) {
    if (!c || ticket < 0) { pfag_set_error("bad arguments"); return PFAG_E_ARG; }
    SnapState *s = SS(c);
    if (!s || ticket >= s->next) { pfag_set_error("no snapshot with ticket %ld", ticket); return PFAG_E_ARG; }
    // a slot reused by a later snapshot completes after this one: waiting on it is enough
    PFAG_CUDA_CHECK(cudaEventSynchronize(s->done[ticket % SNAP_TICKETS]));
    return PFAG_OK;
}

extern "C" int pfag_write_text_snapshot(const void *table, int precision, int N, const char *path) {
    if (!table || !path || N < 1 || (precision != 32 && precision != 64)) {
        pfag_set_error("bad arguments");
        return PFAG_E_ARG;
    }
    unsigned nt = std::thread::hardware_concurrency();
    nt = nt ? (nt > 16 ? 16 : nt) : 4;
    if ((int)nt > N) nt = (unsigned)N;
    std::vector<std::string> parts(nt);
    std::vector<std::thread> th;
    for (unsigned k = 0; k < nt; k++) {
        const int i0 = (int)((long)N * k / nt), i1 = (int)((long)N * (k + 1) / nt);
        th.emplace_back([&, k, i0, i1] {
            if (precision == 64) format_rows(static_cast<const double *>(table), N, i0, i1, parts[k]);
            else format_rows(static_cast<const float *>(table), N, i0, i1, parts[k]);
        });
    }
    for (auto &t : th) t.join();
    FILE *f = std::fopen(path, "wb");
    if (!f) { pfag_set_error("cannot open %s", path); return PFAG_E_ARG; }
    for (auto &p : parts) {
        if (std::fwrite(p.data(), 1, p.size(), f) != p.size()) {
            std::fclose(f);
            pfag_set_error("write failed: %s", path);
            return PFAG_E_ARG;
        }
    }
    std::fclose(f);
    return PFAG_OK;
}
