// Fused path: the same step as the plain path (and the reference loop body,
// main_code/run_with_active_gels.cpp:123-182), restricted to the sites that
// can change, with no host round trip: about 18 kernels per step (9 on the
// main stream, 9 on a side stream for the lumen/ECM work), replayed as one
// CUDA graph from the second step on.
//
// Exactness of the restriction.  Every per-cell write of the reference step
// lands in that cell's zone [xc-z, xc+z)^2, and hfunc_cell starts at zero, so
// outside the bounding rectangle B_n of all zones the cell has visited,
// hfunc_cell[n] is exactly 0 and phi[n] keeps its initial value.  Upload
// checks that the initial phi[n] is <= 0.5 outside the first zone; then the
// full-grid sums of the reference (centroid counts useful_functions.cpp:
// 208-219, areas :179-184, psi :315-318) equal sums over B_n, and psi skips
// only +0.0 terms (bit-identical).  Full-grid work arrays the reference fills
// (norm_grad_phi, J_x/J_y, prod_norm_delta, temp_phase, the parameter maps,
// pi_*) are recomputed on the fly where they are read.
//
// Spectral solve (rho_functions.cpp:409-471) per cell on its M x M box:
//   M = 32..256 (power of two): four passes on register-resident FFTs
//     A rows:    stresses pi_xx + i pi_yy and pi_xy, reaction R, class map, row FFTs
//     B columns: column FFTs, the k-space velocity (rho_functions.cpp:133-190),
//                Hermitian projection packing Re(v_x) + i Re(v_y), column IFFT
//     C2 rows:   row IFFT -> v; Fx = rho vx stored; Fy = rho vy differentiated
//                along the row (the separable form of update_fft_rho's divergence)
//     D2 columns: Fx differentiated along the column; rho + dt R + both terms in place
//   M = 16, 512, 1024: the same steps as five shared-memory radix-4 passes (kf_boxA..E)
//   any other even M up to 512 (the reference's default zone_size 200 gives
//     M = 398): Bluestein transforms over the register FFTs (pfag_bluestein.cuh;
//     kg_stress, kbl_rowsA, kbl_colsB, kg_velocity, kbl_colsC, kbl_rowsD1/D2,
//     kbl_colsE, kbl_rho).
// By linearity of the transform the new rho equals Re(IFFT(FFT(rho) + dt FFT(R)
// + D))/M^2 of the reference, without the round-trip transforms of rho and R.
#pragma once
#include "pfag_internal.cuh"
#include "pfag_fft.cuh"
#include "pfag_regfft.cuh"
#include "pfag_bluestein.cuh"
#include <cooperative_groups.h>
#include <cuda.h>
#include <cudaTypedefs.h>
#include <algorithm>
#include <climits>
#include <cmath>
#include <vector>
#include <cstdlib>
#include <map>
#include <type_traits>
#include <mutex>
#include <cstring>

namespace cg = cooperative_groups;

namespace {

// The dynamic shared-memory limit is an attribute of a kernel function, shared
// by every context of the process: raise it to the largest size any context
// needs and never lower it (contexts of different sizes can coexist).
inline int smem_at_least(const void *fn, size_t bytes) {
    static std::mutex mu;
    static std::map<const void *, size_t> cur;
    std::lock_guard<std::mutex> lock(mu);
    size_t &c = cur[fn];
    if (bytes <= c) return PFAG_OK;
    PFAG_CUDA_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    c = bytes;
    return PFAG_OK;
}

constexpr int FT = 256;           // threads per block of the fused kernels
constexpr int RT_I = 8;            // reshaping tile: RT_I zone rows x the full zone width

struct LumMaps;

struct FusedRes {
    void *Y1, *Y2;          // complex [Ntot][M][M]
    void *Rb;               // real [Ntot][M][M]   reaction -deg*rho + gen*P on the box
    unsigned char *clsT;    // [Ntot][M(j)][M(i)]  apical/basal/lateral class, transposed
    void *Jc;               // real [Ntot][2][W][W] normals on zone + 1 ring, W = 2z+2
    void *Jl;               // real [4][N][N] lumen / ECM normals
    int4 *rect;             // [Ntot] support rectangle (i0, i1, j0, j1), half-open
    double *part_a;         // [Ntot][tiles^2] per-cell area partials of the psi tiles
    double *part_r;         // [Ntot][tpc]
    double *part_e;         // [npsi] sum_ecm partials
    double *part_l;         // [2][coop_r]
    void *G;                // [N][N] lumen/ECM coupling term of the phi update (FP32 build)
    int *cK, *cdone, *ccnt; // per cell
    int *lK, *ldone, *lcnt; // [2] lumen, ECM
    int tpc;                // reshaping strips per cell
    int resh_threads;       // block size of the reshaping kernel (a thread per zone column, at most RESH_MAX_THREADS)
    size_t resh_smem;       // its per-warp, per-cell partial sums + strip tile
    size_t resh_tile;       // one staged strip (3 (RB+2) W reals)
    int ntl;                // lumen/ECM relaxation tiles per field (LRB rows x FT columns)
    size_t lum_tile;        // their staged tile (3 (LRB+2) (FT+2) reals)
    double *part_lt;        // [2][max(ntl, ltiles)] tile partial sums
    LumMaps *lmaps;         // FP32, N >= LT_W, N % 4 == 0: tensor maps of kl_relax_tma (else null)
    bool lum_tma;           // run the first lumen / ECM iterations as kl_relax_tma (pfag_set_lumen_tiles)
    int ltiles;             // kl_relax_tma's tiles per field
    int lt_blocks;          // its persistent grid
    size_t lt_smem;         // its stages, halo columns and barriers
    // side stream of the lumen/ECM kernels and its fork/join events
    cudaStream_t side;
    cudaEvent_t ev_psi, ev_area, ev_boxA, ev_lum;
    bool fork;
    int npsi;
    int coop_r;             // co-resident block count of the persistent kernel
    int coop_default;       // its value before any launch-shape setting
    long upd_default;       // the phi update's warp budget before any launch-shape setting
    bool generic;           // box not a power of two in 16..1024: Bluestein passes (M <= 512)
    int blue_L;             // their inner power-of-two length (>= 2M-1, at least 32)
    void *btw, *bcw, *bwf, *bhdi;   // their tables (pfag_bluestein.cuh), in the context's precision
    double *bh;             // the derivative kernel h in FP64 (table scratch)
    void *Gsp;              // pi_xy's half spectrum [Ntot][M][M/2+1] complex
    long upd_warps;         // co-resident warps of kf_update_rows (FP32)
    size_t upd_smem;        // its row ring
    int logm, rows_blk, grp_cols;
    size_t smemA, smemB, smemC, smemD, smemE;
    bool ring_pending;      // the rho ghost ring still has to be made to match its sources
    // cell sharding (pfag_shard_enable): [2][N][N] phi planes of the cells
    // before local cell 0 and after local cell Ntot-1, held by other contexts
    // and written here by the host between steps; null when unsharded
    void *nb_lo, *nb_hi;
    // the step split at psi (pfag_step_head / pfag_step_tail), each part
    // captured as its own graph: [0] head, [1] tail
    cudaGraph_t pgraph[2];
    cudaGraphExec_t pgexec[2];
    bool pgraph_ok[2];
    int pgraph_state[2];
    long pgraph_launches[2];
    bool head_pending;      // a head was enqueued and its tail not yet
    // one step captured as a CUDA graph after the first eager step
    cudaGraph_t graph;
    cudaGraphExec_t gexec;
    bool graph_ok;
    int graph_state;        // 0 not tried, 1 captured, -1 capture failed (eager from then on)
    long graph_key;         // host inputs the capture depends on (relaxation cap)
    long graph_launches;    // kernel launches in one replay
    long eager_steps;
};

template <typename real>
__device__ __forceinline__ int map_class_f(real ph, real l, real e, real pm, real pp) {
    // create_turnover_rates_tensions, rho_functions.cpp:324-353
    real c1l = ph * l, c1e = ph * e;
    int index;
    real mx;
    if (c1l > c1e) { index = 0; mx = c1l; } else { index = 1; mx = c1e; }
    real c1c2 = ph * pm;
    if (c1c2 > mx) { index = 2; mx = c1c2; }
    real c1c3 = ph * pp;
    if (c1c3 > mx) { index = 3; }
    return index == 3 ? 2 : index;
}

__device__ __forceinline__ double block_sum_d(double v) {
    __shared__ double sh[32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0)
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) r += sh[k];
    __syncthreads();
    return r;
}

// Fixed-order sum of n doubles by the calling warp (lane l adds elements
// l, l+32, ...; then a fixed shuffle tree); every lane returns the total.
__device__ __forceinline__ double warp_sum_fixed(const volatile double *p, int n) {
    const int l = threadIdx.x & 31;
    double a = 0.0;
    for (int k = l; k < n; k += 32) a += p[k];
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    return a;
}

// Asynchronous global -> shared copy of one 4-, 8- or 16-byte element (no
// register staging; a 16-byte one needs both addresses 16-byte aligned);
// cp_async_wait_all waits for this thread's copies.
template <typename T>
__device__ __forceinline__ void cp_async_elem(T *dst, const T *src) {
    static_assert(sizeof(T) == 4 || sizeof(T) == 8 || sizeof(T) == 16, "element size");
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d), "l"(src), "n"(sizeof(T)) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// True when every cell has a convergence stamp in (0, upto]; each warp reads
// the stamps in parallel (32 per round) and votes.
__device__ __forceinline__ bool all_done_upto(const int *done, int ncells, int upto) {
    bool ok = true;
    for (int base = 0; base < ncells; base += 32) {
        const int n = base + (threadIdx.x & 31);
        bool mine = true;
        if (n < ncells) {
            const int d = *(volatile const int *)&done[n];
            mine = d != 0 && d <= upto;
        }
        ok = __all_sync(0xffffffffu, mine) && ok;
        if (!ok) break;
    }
    return ok;
}

// ---- support-rectangle centroid (find_centres_cells, useful_functions.cpp:193-227)
template <typename real>
__global__ void kf_centroid(const real *__restrict__ phi, const int4 *__restrict__ rect, int N,
                            long long *__restrict__ acc) {
    const int n = blockIdx.y;
    const int4 r = rect[n];
    const real *p = phi + (size_t)n * N * N;
    // CR rows x 2 column slots per thread per round, all loads issued first
    constexpr int CR = 4;
    int c32 = 0, sx32 = 0, sy32 = 0;
    long long cnt = 0, sx = 0, sy = 0;
    for (int jb = r.z + threadIdx.x; jb < r.w; jb += 2 * blockDim.x)
    for (int ib = r.x + blockIdx.x; ib < r.y; ib += CR * gridDim.x) {
        const int j0 = jb, j1 = jb + blockDim.x;
        real v0[CR], v1[CR];
#pragma unroll
        for (int k = 0; k < CR; k++) {
            const int i = ib + k * gridDim.x;
            v0[k] = (i < r.y && j0 < r.w) ? p[(size_t)i * N + j0] : (real)0.0;
            v1[k] = (i < r.y && j1 < r.w) ? p[(size_t)i * N + j1] : (real)0.0;
        }
#pragma unroll
        for (int k = 0; k < CR; k++) {
            const int i = ib + k * gridDim.x;
            if (v0[k] > (real)0.5) { c32++; sx32 += i; sy32 += j0; }
            if (v1[k] > (real)0.5) { c32++; sx32 += i; sy32 += j1; }
        }
        // int partials stay far from overflow: at most 2 CR sites of index < 2^15 per round
        cnt += c32; sx += sx32; sy += sy32;
        c32 = sx32 = sy32 = 0;
    }
    for (int o = 16; o > 0; o >>= 1) {
        cnt += __shfl_down_sync(0xffffffffu, cnt, o);
        sx += __shfl_down_sync(0xffffffffu, sx, o);
        sy += __shfl_down_sync(0xffffffffu, sy, o);
    }
    if ((threadIdx.x & 31) == 0 && cnt) {
        atomicAdd((unsigned long long *)&acc[3 * n + 0], (unsigned long long)cnt);
        atomicAdd((unsigned long long *)&acc[3 * n + 1], (unsigned long long)sx);
        atomicAdd((unsigned long long *)&acc[3 * n + 2], (unsigned long long)sy);
    }
}

// centroid, zone check (clamped so no kernel can leave the grid), B_n union zone
// Cell n's centroid from its accumulators (integer division as the reference,
// useful_functions.cpp:222-223), clamped so that no kernel can leave the grid,
// the error bits it raises, and its support rectangle extended by the new zone.
__device__ __forceinline__ void centroid_of(const long long *__restrict__ acc, int n, int N, int zone, int &x,
                                            int &y, unsigned &errbits) {
    const long long c = acc[3 * n];
    errbits = 0;
    if (c == 0) {
        errbits |= ERRBIT_EMPTY_CELL;
        x = N / 2; y = N / 2;
    } else {
        x = (int)(acc[3 * n + 1] / c);
        y = (int)(acc[3 * n + 2] / c);
    }
    if (x - zone < 1 || x + zone > N - 1 || y - zone < 1 || y + zone > N - 1) {
        errbits |= ERRBIT_ZONE;
        x = min(max(x, zone + 1), N - 1 - zone);
        y = min(max(y, zone + 1), N - 1 - zone);
    }
}
__device__ __forceinline__ int4 rect_with_zone(int4 r, int x, int y, int zone) {
    r.x = min(r.x, x - zone); r.y = max(r.y, x + zone);
    r.z = min(r.z, y - zone); r.w = max(r.w, y + zone);
    return r;
}

__global__ void kf_centroid_finalize(const long long *__restrict__ acc, int Ntot, int N, int zone,
                                     int *__restrict__ xc, int *__restrict__ yc, int4 *__restrict__ rect,
                                     unsigned *__restrict__ err) {
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= Ntot) return;
    int x, y;
    unsigned eb;
    centroid_of(acc, n, N, zone, x, y, eb);
    if (eb) atomicOr(err, eb);
    xc[n] = x;
    yc[n] = y;
    rect[n] = rect_with_zone(rect[n], x, y, zone);
}

// ---- one pass over 16x32 tiles of the grid: h(phi) on every cell's zone
//      (compute_hfunc_3d_tables_kernels_loop_n, useful_functions.cpp:233-251),
//      psi = sum_n hfunc_cell[n] (:305-322), the cells' area partials
//      (sum_s_kernels, :168-190), h(lum), h(ECM) (:272-285) and the sum_ecm
//      partials (cell_phase_functions.cpp:376-386).
// Only the cells whose support rectangle B_n meets the tile are visited, in
// ascending order (warp 0 compacts them by ballots): hfunc_cell[n] is exactly
// 0 outside B_n, so psi is the reference's sum in the reference's order.
// Inside the zone h is formed from phi and stored, elsewhere in B_n the
// stored (stale) value is read.  Area partials: per cell and tile, the
// tile's warps' sums in warp order, written to part_a[n][tile].
constexpr int PT_R = 16, KR = PT_R / 8;   // tile rows (tiles are PT_R x 32), rows per thread
template <typename real>
__global__ void __launch_bounds__(256) kf_hpsi(const real *__restrict__ phi, real *__restrict__ hfunc,
                                               int4 *__restrict__ rect, const long long *__restrict__ cacc,
                                               int *__restrict__ xc, int *__restrict__ yc,
                                               unsigned *__restrict__ err, int Ntot, int N, int z,
                                               const real *__restrict__ lum, const real *__restrict__ ecm,
                                               real *__restrict__ psi, real *__restrict__ hl, real *__restrict__ he,
                                               double dx2, double *__restrict__ part_e, double *__restrict__ part_a) {
    __shared__ int list[1024];
    __shared__ int4 lrect[1024];              // indexed by cell
    __shared__ int2 lzone[1024];              // indexed by cell
    __shared__ unsigned hitm[32];             // per 32-cell chunk: cells whose B_n meets the tile
    __shared__ int nlist;
    __shared__ double wq[8][32];
    const int ti0 = blockIdx.y * PT_R, tj0 = blockIdx.x * 32;
    const int tile = blockIdx.y * gridDim.x + blockIdx.x, ntiles = gridDim.x * gridDim.y;
    // lum and ECM of this thread's sites: loaded first, used last
    real lv[KR], ev[KR];
#pragma unroll
    for (int k = 0; k < KR; k++) {
        const int i = ti0 + (threadIdx.x >> 5) + 8 * k, jj = tj0 + (threadIdx.x & 31);
        const bool ok = i < N && jj < N;
        lv[k] = ok ? lum[(size_t)i * N + jj] : (real)0.0;
        ev[k] = ok ? ecm[(size_t)i * N + jj] : (real)0.0;
    }
    {
        // every warp takes 32-cell chunks: this step's centroid (find_centres_cells)
        // from the sums over B_n; block (0, 0) publishes it for the later
        // kernels, every block uses its own copy (rect[n] may be old or new
        // here: the union is the same)
        const int nchunk = (Ntot + 31) / 32;
        for (int ch = threadIdx.x >> 5; ch < nchunk; ch += blockDim.x >> 5) {
            const int n = ch * 32 + (threadIdx.x & 31);
            bool hit = false;
            if (n < Ntot) {
                unsigned eb;
                int x, y;
                centroid_of(cacc, n, N, z, x, y, eb);
                const int4 r = rect_with_zone(rect[n], x, y, z);
                if (blockIdx.x == 0 && blockIdx.y == 0) {
                    if (eb) atomicOr(err, eb);
                    xc[n] = x;
                    yc[n] = y;
                    rect[n] = r;
                }
                hit = r.x < ti0 + PT_R && r.y > ti0 && r.z < tj0 + 32 && r.w > tj0;
                lrect[n] = r;
                lzone[n] = make_int2(x - z, y - z);
            }
            const unsigned m = __ballot_sync(0xffffffffu, hit);
            if ((threadIdx.x & 31) == 0) hitm[ch] = m;
        }
        __syncthreads();
        // the tile's cells in cell order (the order of the reference's psi sum)
        if (threadIdx.x < 32) {
            int cnt = 0;
            for (int ch = 0; ch < nchunk; ch++) {
                const unsigned m = hitm[ch];
                if ((m >> threadIdx.x) & 1u) list[cnt + __popc(m & ((1u << threadIdx.x) - 1u))] = ch * 32 + threadIdx.x;
                cnt += __popc(m);
            }
            if (threadIdx.x == 0) nlist = cnt;
        }
    }
    __syncthreads();
    const int nl = nlist;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int j = tj0 + lane;
    const size_t NN = (size_t)N * N;
    real ps[KR];
#pragma unroll
    for (int k = 0; k < KR; k++) ps[k] = (real)0.0;
    for (int q0 = 0; q0 < nl; q0 += 32) {
        const int qn = min(32, nl - q0);
        // CU cells per round, all their loads issued before any use
        constexpr int CU = 4;
        for (int u0 = 0; u0 < qn; u0 += CU) {
            real v[CU][KR];
            bool inz[CU][KR];
            real *hp[CU];
#pragma unroll
            for (int c = 0; c < CU; c++) {
                const int u = u0 + c;
                const bool live = u < qn;
                const int q = q0 + (live ? u : 0);
                const int n = list[q];
                const int4 r = lrect[n];
                const int zi0 = lzone[n].x, zj0 = lzone[n].y;
                hp[c] = hfunc + (size_t)n * NN;
                const real *pp = phi + (size_t)n * NN;
#pragma unroll
                for (int k = 0; k < KR; k++) {
                    const int i = ti0 + warp + 8 * k;
                    const bool ok = live && i < N && j < N && i >= r.x && i < r.y && j >= r.z && j < r.w;
                    inz[c][k] = ok && i >= zi0 && i < zi0 + 2 * z && j >= zj0 && j < zj0 + 2 * z;
                    const size_t o = (size_t)i * N + j;
                    v[c][k] = ok ? (inz[c][k] ? pp[o] : hp[c][o]) : (real)0.0;
                }
            }
#pragma unroll
            for (int c = 0; c < CU; c++) {
                double a = 0.0;
#pragma unroll
                for (int k = 0; k < KR; k++) {
                    real h = v[c][k];
                    if (inz[c][k]) {
                        h = h * h * ((real)3.0 - (real)2.0 * h);
                        hp[c][(size_t)(ti0 + warp + 8 * k) * N + j] = h;
                    }
                    ps[k] += h;                 // cells in list order
                    a += (double)h * dx2;
                }
                for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
                if (lane == 0 && u0 + c < qn) wq[warp][u0 + c] = a;
            }
        }
        __syncthreads();
        if (threadIdx.x < qn) {
            double t = 0.0;
#pragma unroll
            for (int w = 0; w < 8; w++) t += wq[w][threadIdx.x];
            part_a[(size_t)list[q0 + threadIdx.x] * ntiles + tile] = t;
        }
        __syncthreads();
    }
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < KR; k++) {
        const int i = ti0 + warp + 8 * k;
        if (i >= N || j >= N) continue;
        const size_t o = (size_t)i * N + j;
        psi[o] = ps[k];
        const real a = lv[k], b = ev[k];
        hl[o] = a * a * ((real)3.0 - (real)2.0 * a);
        const real hb = b * b * ((real)3.0 - (real)2.0 * b);
        he[o] = hb;
        acc += (double)hb * dx2;
    }
    const double t = block_sum_d(acc);
    if (threadIdx.x == 0) part_e[tile] = t;
}

// area s_n = sum of cell n's tile partials over the tiles B_n meets, in tile
// order (lanes take every 32nd tile, then a fixed summation tree): the calling
// warp returns it on every lane (sum_s_kernels, useful_functions.cpp:168-190)
__device__ __forceinline__ double cell_area(const double *__restrict__ part_a, const int4 *__restrict__ rect, int n,
                                            int tiles_x, int ntiles) {
    const int lane = threadIdx.x & 31;
    const int4 r = rect[n];
    const int tr0 = r.x / PT_R, tr1 = (r.y - 1) / PT_R, tc0 = r.z / 32, tc1 = (r.w - 1) / 32;
    const int w = tc1 - tc0 + 1, cnt = (tr1 - tr0 + 1) * w;
    double a = 0.0;
    for (int k = lane; k < cnt; k += 32) {
        const int tr = tr0 + k / w, tc = tc0 + k % w;
        a += part_a[(size_t)n * ntiles + tr * tiles_x + tc];
    }
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    return a;
}
// s_n and f0_n = alpha (s0 - s_n) (useful_functions.cpp:184-187), one warp per cell
__global__ void kf_area_tiles(const double *__restrict__ part_a, const int4 *__restrict__ rect, int tiles_x,
                              int ntiles, double alpha, double s0, double *__restrict__ s, double *__restrict__ f0) {
    const int n = blockIdx.x;
    const double a = cell_area(part_a, rect, n, tiles_x, ntiles);
    if (threadIdx.x == 0) {
        s[n] = a;
        f0[n] = alpha * (s0 - a);
    }
}

// ---- box passes -------------------------------------------------------------
struct BoxArgs {
    int N, z, M, logm, Ntot;
    double c4, sigma, dt, kfac, friction, dx;
    double inv_2s2, k_delta;     // 1/(2 sigma^2), 1/(sqrt(2 pi) sigma): FP32 folded constants
    double deg[3], gen[3], a_ort[3], a_tan[3], visc[3], bb[3];
    // phi planes of the index neighbours of cells 0 and Ntot-1 (n1 of cell 0
    // and n2 of cell Ntot-1, rho_functions.cpp:297-311): this context's own
    // cells Ntot-1 and 0, or planes held for a shard of a larger organoid
    const void *nb_lo, *nb_hi;
};

// the phi planes of cell n's index neighbours n1 = n-1 and n2 = n+1 (cyclic over the organoid)
template <typename real>
__device__ __forceinline__ void nb_planes(const real *phi, const BoxArgs &a, int n, const real *&p1,
                                          const real *&p2) {
    const size_t NN = (size_t)a.N * a.N;
    p1 = (n == 0) ? (const real *)a.nb_lo : phi + (size_t)(n - 1) * NN;
    p2 = (n == a.Ntot - 1) ? (const real *)a.nb_hi : phi + (size_t)(n + 1) * NN;
}

__device__ __forceinline__ int wrapk(int i, int M) { return i < M / 2 ? i : i - M; }

// Pass A: rows [i0, i0+R) of cell n's box
template <typename real>
__global__ void kf_boxA(const real *__restrict__ phi, const real *__restrict__ rho, const real *__restrict__ lum,
                        const real *__restrict__ ecm, const int *__restrict__ xc, const int *__restrict__ yc,
                        BoxArgs a, int R, typename Cplx<real>::type *__restrict__ Y1,
                        typename Cplx<real>::type *__restrict__ Y2, real *__restrict__ Rb,
                        unsigned char *__restrict__ clsT) {
    typedef typename Cplx<real>::type cx;
    extern __shared__ unsigned char smraw[];
    cx *tw = (cx *)smraw;
    const int M = a.M, N = a.N;
    cx *zz = tw + M;            // [2R][M]: rows of z1 then rows of z2
    fft_twiddles(tw, M);
    const int n = blockIdx.y, i0 = blockIdx.x * R;
    const int bi = xc[n] - a.z + 1, bj = yc[n] - a.z + 1;
    const real *p1, *p2;
    nb_planes<real>(phi, a, n, p1, p2);
    const size_t NN = (size_t)N * N;
    const real *p = phi + (size_t)n * NN;
    const real c4 = (real)a.c4, sigma = (real)a.sigma;
    for (int e = threadIdx.x; e < R * M; e += blockDim.x) {
        const int r = e >> a.logm, j = e & (M - 1);
        const int i = i0 + r;
        const int gi = bi + i, gj = bj + j;
        const size_t s = (size_t)gi * N + gj;
        const real f = p[s];
        const real dxp = p[s + N] - p[s - N];
        const real dyp = p[s + 1] - p[s - 1];
        const real g = sqrt(c4 * (dxp * dxp + dyp * dyp));
        const int cls = map_class_f<real>(f, lum[s], ecm[s], p1[s], p2[s]);
        const real rr = rho[(size_t)n * NN + s];
        const real at = (real)a.a_tan[cls], ao = (real)a.a_ort[cls], b = (real)a.bb[cls];
        // compute_pi_xx/yy/xy, rho_functions.cpp:47-51, :75-79, :105-109
        real xx = -at * rr * rr * rr + b * rr * rr * rr * rr;
        real yy = xx, xy = (real)0.0;
        if (g > (real)0.0) {
            xx += (at - ao) * rr * rr * rr * c4 * dxp * dxp / g / g;
            yy += (at - ao) * rr * rr * rr * c4 * dyp * dyp / g / g;
            xy += (at - ao) * rr * rr * rr * c4 * dxp * dyp / g / g;
        }
        // create_deg_gen with compute_prod_norm_delta, rho_functions.cpp:25, :205
        const real P = g * exp(-(f - (real)0.5) * (f - (real)0.5) / (real)2.0 / sigma / sigma) /
                       sqrt((real)(2.0 * M_PI)) / sigma;
        Rb[((size_t)n * M + i) * M + j] = -(real)a.deg[cls] * rr + (real)a.gen[cls] * P;
        clsT[((size_t)n * M + j) * M + i] = (unsigned char)cls;
        const int br = bitrev(j, a.logm);
        cx v1, v2;
        v1.x = xx; v1.y = yy;
        v2.x = xy; v2.y = (real)0.0;
        zz[(size_t)r * M + br] = v1;
        zz[(size_t)(R + r) * M + br] = v2;
    }
    __syncthreads();
    fft_stages(zz, 2 * R, M, a.logm, tw, false);
    for (int e = threadIdx.x; e < R * M; e += blockDim.x) {
        const int r = e >> a.logm, k = e & (M - 1);
        const size_t o = ((size_t)n * M + i0 + r) * M + k;
        Y1[o] = zz[(size_t)r * M + k];
        Y2[o] = zz[(size_t)(R + r) * M + k];
    }
}

// update_rho_velocity (rho_functions.cpp:153-186) at one wavevector
template <typename real, typename cx>
__device__ __forceinline__ void velocity_at(real kx, real ky, real et, real friction, cx pxx, cx pyy, cx pxy,
                                            cx &vx, cx &vy) {
    const real A = friction + (real)2.0 * et * (kx * kx + ky * ky / (real)2.0);
    const real D = -((real)4.0 * et * et * kx * kx * ky * ky + friction * friction +
                     (real)3.0 * et * friction * (kx * kx + ky * ky) +
                     (real)2.0 * et * et * (kx * kx * kx * kx + ky * ky * ky * ky));
    if constexpr (sizeof(real) == 4) {
        const real iD = (real)1.0 / D, iA = (real)1.0 / A;
        vy.x = (et * kx * ky * (kx * pxx.y + ky * pxy.y) - A * (ky * pyy.y + kx * pxy.y)) * iD;
        vy.y = (-et * kx * ky * (kx * pxx.x + ky * pxy.x) + A * (ky * pyy.x + kx * pxy.x)) * iD;
        vx.x = (kx * pxx.y + ky * pxy.y - et * kx * ky * vy.x) * iA;
        vx.y = (-kx * pxx.x - ky * pxy.x - et * kx * ky * vy.y) * iA;
        return;
    }
    vy.x = (real)0.0 + et * kx * ky * (kx * pxx.y + ky * pxy.y);
    vy.x -= A * (ky * pyy.y + kx * pxy.y);
    vy.x /= D;
    vy.y = (real)0.0 - et * kx * ky * (kx * pxx.x + ky * pxy.x);
    vy.y += A * (ky * pyy.x + kx * pxy.x);
    vy.y /= D;
    vx.x = (real)0.0 + (kx * pxx.y + ky * pxy.y - et * kx * ky * vy.x);
    vx.x /= A;
    vx.y = (real)0.0 + (-kx * pxx.x - ky * pxy.x - et * kx * ky * vy.y);
    vx.y /= A;
}

// Column slots of a pass B/D block: primaries c0..c0+np-1 (c <= M/2), then the
// partners M - c of the primaries that are not their own partner.
struct ColSlots {
    int np, ns;
    int col[64];
    int partner[32];
};

__device__ __forceinline__ void make_slots(ColSlots &cs, int c0, int G, int M) {
    cs.np = min(G, M / 2 + 1 - c0);
    cs.ns = cs.np;
    for (int s = 0; s < cs.np; s++) {
        const int c = c0 + s;
        cs.col[s] = c;
        const int pc = (M - c) % M;
        if (pc == c) cs.partner[s] = s;
        else { cs.col[cs.ns] = pc; cs.partner[s] = cs.ns; cs.ns++; }
    }
}

template <typename cx>
__device__ void load_cols(cx *dst, int sstride, const cx *__restrict__ src, const ColSlots &cs, int M, int logm) {
    for (int e = threadIdx.x; e < cs.ns * M; e += blockDim.x) {
        const int i = e / cs.ns, sl = e - i * cs.ns;
        dst[(size_t)sl * sstride + bitrev(i, logm)] = src[(size_t)i * M + cs.col[sl]];
    }
}

template <typename cx>
__device__ void store_cols(cx *__restrict__ dstg, const cx *src, int sstride, const ColSlots &cs, int M) {
    for (int e = threadIdx.x; e < cs.ns * M; e += blockDim.x) {
        const int i = e / cs.ns, sl = e - i * cs.ns;
        dstg[(size_t)i * M + cs.col[sl]] = src[(size_t)sl * sstride + i];
    }
}

// Enumerate the disjoint pairs {k, -k} of the slots; calls f(slot_a, kx_a, slot_b, kx_b).
template <typename F>
__device__ __forceinline__ void for_pairs(const ColSlots &cs, int M, F f) {
    const int half = M / 2;
    int total = 0;
    for (int s = 0; s < cs.np; s++) total += (cs.partner[s] == s) ? (half + 1) : M;
    for (int w = threadIdx.x; w < total; w += blockDim.x) {
        int rem = w, s = 0;
        for (; s < cs.np; s++) {
            const int cnt = (cs.partner[s] == s) ? (half + 1) : M;
            if (rem < cnt) break;
            rem -= cnt;
        }
        const int kx = rem, kx2 = (M - kx) % M;
        f(s, kx, cs.partner[s], kx2);
    }
}

template <typename real>
__global__ void kf_boxB(typename Cplx<real>::type *__restrict__ Y1, const typename Cplx<real>::type *__restrict__ Y2,
                        const unsigned char *__restrict__ clsT, BoxArgs a, int G) {
    typedef typename Cplx<real>::type cx;
    extern __shared__ unsigned char smraw[];
    const int M = a.M, S = M + 1;
    cx *tw = (cx *)smraw;
    fft_twiddles(tw, M);
    __shared__ ColSlots cs;
    const int n = blockIdx.y;
    if (threadIdx.x == 0) make_slots(cs, blockIdx.x * G, G, M);
    __syncthreads();
    cx *Z1 = tw + M, *Z2 = Z1 + (size_t)cs.ns * S;
    const cx *y1 = Y1 + (size_t)n * M * M, *y2 = Y2 + (size_t)n * M * M;
    load_cols(Z1, S, y1, cs, M, a.logm);
    load_cols(Z2, S, y2, cs, M, a.logm);
    __syncthreads();
    // both fields in one call: Z2 follows Z1 with the same stride
    fft_stages(Z1, 2 * cs.ns, S, a.logm, tw, false);
    const unsigned char *cl = clsT + (size_t)n * M * M;
    const real kf = (real)0.0;
    (void)kf;
    for_pairs(cs, M, [&](int sa, int ka, int sb, int kb) {
        const cx z1a = Z1[(size_t)sa * S + ka], z1b = Z1[(size_t)sb * S + kb];
        const cx z2a = Z2[(size_t)sa * S + ka], z2b = Z2[(size_t)sb * S + kb];
        // unpack the two real fields packed as pi_xx + i pi_yy
        cx pxx_a, pyy_a, pxx_b, pyy_b;
        pxx_a.x = (real)0.5 * (z1a.x + z1b.x); pxx_a.y = (real)0.5 * (z1a.y - z1b.y);
        pyy_a.x = (real)0.5 * (z1a.y + z1b.y); pyy_a.y = (real)0.5 * (z1b.x - z1a.x);
        pxx_b.x = pxx_a.x; pxx_b.y = -pxx_a.y;
        pyy_b.x = pyy_a.x; pyy_b.y = -pyy_a.y;
        const int ca = cs.col[sa], cb = cs.col[sb];
        const real kxa = (real)(a.kfac * wrapk(ka, M)), kya = (real)(a.kfac * wrapk(ca, M));
        const real kxb = (real)(a.kfac * wrapk(kb, M)), kyb = (real)(a.kfac * wrapk(cb, M));
        const real eta_a = (real)a.visc[cl[(size_t)ca * M + ka]];
        const real eta_b = (real)a.visc[cl[(size_t)cb * M + kb]];
        const real fr = (real)a.friction;
        cx vxa, vya, vxb, vyb;
        velocity_at<real, cx>(kxa, kya, eta_a, fr, pxx_a, pyy_a, z2a, vxa, vya);
        velocity_at<real, cx>(kxb, kyb, eta_b, fr, pxx_b, pyy_b, z2b, vxb, vyb);
        // Hermitian parts: H(X)(k) = (X(k) + conj(X(-k)))/2, packed H(vx) + i H(vy)
        cx hx, hy;
        hx.x = (real)0.5 * (vxa.x + vxb.x); hx.y = (real)0.5 * (vxa.y - vxb.y);
        hy.x = (real)0.5 * (vya.x + vyb.x); hy.y = (real)0.5 * (vya.y - vyb.y);
        cx pa, pb;
        pa.x = hx.x - hy.y; pa.y = hx.y + hy.x;
        pb.x = hx.x + hy.y; pb.y = hy.x - hx.y;
        Z1[(size_t)sa * S + ka] = pa;
        if (!(sa == sb && ka == kb)) Z1[(size_t)sb * S + kb] = pb;
    });
    __syncthreads();
    bitrev_permute(Z1, cs.ns, S, a.logm);
    fft_stages(Z1, cs.ns, S, a.logm, tw, true);
    store_cols(Y1 + (size_t)n * M * M, Z1, S, cs, M);
}

template <typename real>
__global__ void kf_boxC(const typename Cplx<real>::type *__restrict__ Y1, typename Cplx<real>::type *__restrict__ Y2,
                        const real *__restrict__ rho, const int *__restrict__ xc, const int *__restrict__ yc,
                        BoxArgs a, int R, real *__restrict__ vdx, real *__restrict__ vdy) {
    typedef typename Cplx<real>::type cx;
    extern __shared__ unsigned char smraw[];
    const int M = a.M, N = a.N;
    cx *tw = (cx *)smraw;
    cx *zz = tw + M;
    fft_twiddles(tw, M);
    const int n = blockIdx.y, i0 = blockIdx.x * R;
    const int bi = xc[n] - a.z + 1, bj = yc[n] - a.z + 1;
    for (int e = threadIdx.x; e < R * M; e += blockDim.x) {
        const int r = e >> a.logm, j = e & (M - 1);
        zz[(size_t)r * M + bitrev(j, a.logm)] = Y1[((size_t)n * M + i0 + r) * M + j];
    }
    __syncthreads();
    fft_stages(zz, R, M, a.logm, tw, true);
    const real mm = (real)((double)M * (double)M);
    const real *rh = rho + (size_t)n * N * N;
    // each thread owns the same set of e in both loops, so the permuted store
    // below may only be issued after every thread has read its values
    cx vals[8];
    int cntv = 0;
    for (int e = threadIdx.x; e < R * M; e += blockDim.x) {
        const int r = e >> a.logm, j = e & (M - 1);
        const cx v = zz[(size_t)r * M + j];
        const real rr = rh[(size_t)(bi + i0 + r) * N + bj + j];
        // load_fft_rho_v, rho_functions.cpp:279: rho * Re(IFFT(v)) / M^2
        cx q;
        q.x = rr * v.x / mm;
        q.y = rr * v.y / mm;
        if (vdx) {
            const size_t o = ((size_t)n * M + i0 + r) * M + j;
            vdx[o] = v.x / mm;
            vdy[o] = v.y / mm;
        }
        vals[cntv++] = q;
    }
    __syncthreads();
    cntv = 0;
    for (int e = threadIdx.x; e < R * M; e += blockDim.x) {
        const int r = e >> a.logm, j = e & (M - 1);
        zz[(size_t)r * M + bitrev(j, a.logm)] = vals[cntv++];
    }
    __syncthreads();
    fft_stages(zz, R, M, a.logm, tw, false);
    for (int e = threadIdx.x; e < R * M; e += blockDim.x) {
        const int r = e >> a.logm, k = e & (M - 1);
        Y2[((size_t)n * M + i0 + r) * M + k] = zz[(size_t)r * M + k];
    }
}

template <typename real>
__global__ void kf_boxD(typename Cplx<real>::type *__restrict__ Y1, const typename Cplx<real>::type *__restrict__ Y2,
                        BoxArgs a, int G) {
    typedef typename Cplx<real>::type cx;
    extern __shared__ unsigned char smraw[];
    const int M = a.M, S = M + 1;
    cx *tw = (cx *)smraw;
    fft_twiddles(tw, M);
    __shared__ ColSlots cs;
    const int n = blockIdx.y;
    if (threadIdx.x == 0) make_slots(cs, blockIdx.x * G, G, M);
    __syncthreads();
    cx *W = tw + M;
    load_cols(W, S, Y2 + (size_t)n * M * M, cs, M, a.logm);
    __syncthreads();
    fft_stages(W, cs.ns, S, a.logm, tw, false);
    const real dtk = (real)(a.dt * a.kfac);
    for_pairs(cs, M, [&](int sa, int ka, int sb, int kb) {
        const cx wa = W[(size_t)sa * S + ka], wb = W[(size_t)sb * S + kb];
        // (rho vx)^ = (W(k) + conj W(-k))/2, (rho vy)^ = (W(k) - conj W(-k))/(2i)
        cx A1, B1, A2, B2;
        A1.x = (real)0.5 * (wa.x + wb.x); A1.y = (real)0.5 * (wa.y - wb.y);
        B1.x = (real)0.5 * (wa.y + wb.y); B1.y = (real)0.5 * (wb.x - wa.x);
        A2.x = A1.x; A2.y = -A1.y;
        B2.x = B1.x; B2.y = -B1.y;
        const real ir1 = (real)wrapk(ka, M), jr1 = (real)wrapk(cs.col[sa], M);
        const real ir2 = (real)wrapk(kb, M), jr2 = (real)wrapk(cs.col[sb], M);
        // update_fft_rho, rho_functions.cpp:243-247: delta = -i dt k (ir A + jr B)
        cx F1, F2, D1, D2;
        F1.x = ir1 * A1.x + jr1 * B1.x; F1.y = ir1 * A1.y + jr1 * B1.y;
        F2.x = ir2 * A2.x + jr2 * B2.x; F2.y = ir2 * A2.y + jr2 * B2.y;
        D1.x = dtk * F1.y; D1.y = -dtk * F1.x;
        D2.x = dtk * F2.y; D2.y = -dtk * F2.x;
        cx ha, hb;
        ha.x = (real)0.5 * (D1.x + D2.x); ha.y = (real)0.5 * (D1.y - D2.y);
        hb.x = ha.x; hb.y = -ha.y;
        W[(size_t)sa * S + ka] = ha;
        if (!(sa == sb && ka == kb)) W[(size_t)sb * S + kb] = hb;
    });
    __syncthreads();
    bitrev_permute(W, cs.ns, S, a.logm);
    fft_stages(W, cs.ns, S, a.logm, tw, true);
    store_cols(Y1 + (size_t)n * M * M, W, S, cs, M);
}

template <typename real>
__global__ void kf_boxE(const typename Cplx<real>::type *__restrict__ Y1, const real *rho,
                        const real *__restrict__ Rb, real *rhon, const int *__restrict__ xc,
                        const int *__restrict__ yc, BoxArgs a, int R) {
    typedef typename Cplx<real>::type cx;
    extern __shared__ unsigned char smraw[];
    const int M = a.M, N = a.N;
    cx *tw = (cx *)smraw;
    cx *zz = tw + M;
    fft_twiddles(tw, M);
    const int n = blockIdx.y, i0 = blockIdx.x * R;
    const int bi = xc[n] - a.z + 1, bj = yc[n] - a.z + 1;
    for (int e = threadIdx.x; e < R * M; e += blockDim.x) {
        const int r = e >> a.logm, j = e & (M - 1);
        zz[(size_t)r * M + bitrev(j, a.logm)] = Y1[((size_t)n * M + i0 + r) * M + j];
    }
    __syncthreads();
    fft_stages(zz, R, M, a.logm, tw, true);
    const real mm = (real)((double)M * (double)M), dt = (real)a.dt;
    const size_t NN = (size_t)N * N;
    for (int e = threadIdx.x; e < R * M; e += blockDim.x) {
        const int r = e >> a.logm, j = e & (M - 1);
        const size_t s = (size_t)n * NN + (size_t)(bi + i0 + r) * N + bj + j;
        const real rr = rho[s];
        rhon[s] = rr + dt * Rb[((size_t)n * M + i0 + r) * M + j] + zz[(size_t)r * M + j].x / mm;
    }
}

// One box site of the active-gel stress and reaction (compute_pi_xx/yy/xy,
// rho_functions.cpp:32-115; create_deg_gen with compute_prod_norm_delta,
// :193-209, :13-30; the class of create_turnover_rates_tensions, :324-353):
// f and the central differences dxp, dyp of the cell's phi, its rho rr, and
// lum, ECM and the index neighbours' phi at the site.  FP64 keeps the
// reference's operation order; FP32 folds the constant factors.
template <typename real>
__device__ __forceinline__ void box_stress(const BoxArgs &a, real f, real dxp, real dyp, real rr, real lv, real ev,
                                           real pm, real pp, real &xx, real &yy, real &xy, real &rt, int &c) {
    const real c4 = (real)a.c4, sigma = (real)a.sigma;
    const real gg = sqrt(c4 * (dxp * dxp + dyp * dyp));
    c = map_class_f<real>(f, lv, ev, pm, pp);
    const real at = (real)a.a_tan[c], ao = (real)a.a_ort[c], b = (real)a.bb[c];
    xx = -at * rr * rr * rr + b * rr * rr * rr * rr;
    yy = xx;
    xy = (real)0.0;
    real P;
    if constexpr (sizeof(real) == 8) {
        if (gg > (real)0.0) {
            xx += (at - ao) * rr * rr * rr * c4 * dxp * dxp / gg / gg;
            yy += (at - ao) * rr * rr * rr * c4 * dyp * dyp / gg / gg;
            xy += (at - ao) * rr * rr * rr * c4 * dxp * dyp / gg / gg;
        }
        P = gg * exp(-(f - (real)0.5) * (f - (real)0.5) / (real)2.0 / sigma / sigma) / sqrt((real)(2.0 * M_PI)) /
            sigma;
    } else {
        if (gg > (real)0.0) {
            const real w = (at - ao) * rr * rr * rr * c4 / (gg * gg);
            xx += w * dxp * dxp;
            yy += w * dyp * dyp;
            xy += w * dxp * dyp;
        }
        const real d = f - (real)0.5;
        P = gg * (real)a.k_delta * __expf(-d * d * (real)a.inv_2s2);
    }
    rt = -(real)a.deg[c] * rr + (real)a.gen[c] * P;
}

// ---- box passes on register-resident FFTs (M = 32 .. 256) ----------------
template <int M> struct BoxGeom {
    static constexpr int TT = RegFFT<float2, M>::TT;          // threads per transform
    static constexpr int ROWS = (256 / TT < M) ? 256 / TT : M; // rows per block of the row passes
    static constexpr int THREADS = TT * ROWS;
    static constexpr int WG = 32 / TT;                       // thread groups per warp
};

// Pass A on register FFTs: one thread group per box row.
template <typename real, int M>
__global__ void __launch_bounds__(256, sizeof(real) == 4 ? 4 : 2) kr_boxA(const real *__restrict__ phi, const real *__restrict__ rho,
                                               const real *__restrict__ lum, const real *__restrict__ ecm,
                                               const int *__restrict__ xc, const int *__restrict__ yc, BoxArgs a,
                                               typename Cplx<real>::type *__restrict__ Y1,
                                               typename Cplx<real>::type *__restrict__ Y2, real *__restrict__ Rb,
                                               unsigned char *__restrict__ clsT) {
    typedef typename Cplx<real>::type cx;
    typedef RegFFT<cx, M> RF;
    constexpr int TT = RF::TT, E1 = RF::E1, ROWS = BoxGeom<M>::ROWS;
    extern __shared__ unsigned char smraw[];
    cx *tw = (cx *)smraw;
    cx *scr = tw + M;                                   // [ROWS][M] exchange scratch
    real *xys = (real *)(scr + ROWS * M);               // [ROWS][M] pi_xy, read back by the same thread
    unsigned char *cls = (unsigned char *)(xys + ROWS * M);  // [ROWS][M + 4]: padded against bank conflicts
    const int t = threadIdx.x % TT, g = threadIdx.x / TT;
    const int n = blockIdx.y, i0 = blockIdx.x * ROWS, i = i0 + g;
    const int N = a.N;
    const int bi = xc[n] - a.z + 1, bj = yc[n] - a.z + 1;
    const real *p1, *p2;
    nb_planes<real>(phi, a, n, p1, p2);
    const size_t NN = (size_t)N * N;
    const real *p = phi + (size_t)n * NN;
    // the block's phi rows with a one-site halo ([ROWS + 2][M + 2], in the FFT
    // exchange scratch, free until the first transform) and its rho rows (in
    // xys, each element read and then overwritten by the same thread) are
    // staged by cp.async, so only lum, ECM and the neighbour cells' phi are
    // read from global memory in the element loop
    constexpr int PW = M + 2;
    real *sphi = reinterpret_cast<real *>(scr);
    {
        const real *src = p + (size_t)(bi + i0 - 1) * N + (bj - 1);
        for (int e = threadIdx.x; e < (ROWS + 2) * PW; e += blockDim.x) {
            const int r = e / PW, cc = e - r * PW;
            cp_async_elem(sphi + e, src + (size_t)r * N + cc);
        }
        const real *rs = rho + (size_t)n * NN + (size_t)(bi + i0) * N + bj;
        for (int e = threadIdx.x; e < ROWS * M; e += blockDim.x) {
            const int r = e / M, cc = e - r * M;
            cp_async_elem(xys + e, rs + (size_t)r * N + cc);
        }
    }
    RegFFT<cx, M>::twiddles_kt(tw);
    cp_async_wait_all();
    __syncthreads();
    const size_t rowo = ((size_t)n * M + i) * M;
    cx v[E1];
#pragma unroll
    for (int q = 0; q < E1; q++) {
        const int j = RF::in_index(t, q);
        const size_t s = (size_t)(bi + i) * N + (bj + j);
        const int o = (g + 1) * PW + j + 1;
        const real f = sphi[o];
        const real dxp = sphi[o + PW] - sphi[o - PW];
        const real dyp = sphi[o + 1] - sphi[o - 1];
        real xx, yy, xy, rt;
        int c;
        box_stress<real>(a, f, dxp, dyp, xys[g * M + j], lum[s], ecm[s], p1[s], p2[s], xx, yy, xy, rt, c);
        Rb[rowo + j] = rt;
        cls[g * (M + 4) + j] = (unsigned char)c;
        xys[g * M + j] = xy;
        v[q].x = xx;
        v[q].y = yy;
    }
    __syncthreads();    // every group is done with the staged phi before scr becomes exchange space
    RF::template run<false, true>(v, t, scr + g * M, tw);
#pragma unroll
    for (int r = 0; r < RF::R2; r++)
#pragma unroll
        for (int k2 = 0; k2 < TT; k2++) Y1[rowo + RF::out_index(t, r, k2)] = v[r * TT + k2];
#pragma unroll
    for (int q = 0; q < E1; q++) {
        v[q].x = xys[g * M + RF::in_index(t, q)];
        v[q].y = (real)0.0;
    }
    RF::template run<false, true>(v, t, scr + g * M, tw);
#pragma unroll
    for (int r = 0; r < RF::R2; r++)
#pragma unroll
        for (int k2 = 0; k2 < TT; k2++) Y2[rowo + RF::out_index(t, r, k2)] = v[r * TT + k2];
    __syncthreads();
    // class map transposed, ROWS consecutive bytes per column, as 16-byte
    // stores (i0 and M are multiples of 16)
    static_assert(ROWS % 16 == 0 && M % 16 == 0, "16-byte class-map stores");
    for (int e = threadIdx.x; e < M * (ROWS / 16); e += blockDim.x) {
        const int j = e / (ROWS / 16), r0 = (e - j * (ROWS / 16)) * 16;
        unsigned w[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            w[q] = 0;
#pragma unroll
            for (int b = 0; b < 4; b++) w[q] |= (unsigned)cls[(r0 + 4 * q + b) * (M + 4) + j] << (8 * b);
        }
        *reinterpret_cast<uint4 *>(clsT + ((size_t)n * M + j) * M + i0 + r0) = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

// Column transforms of the slots held in shared memory (natural order in and
// out); each column's own storage is the exchange scratch of its transform.
template <typename cx, int M, bool INV>
__device__ __forceinline__ void columns_fft(cx *Z, int nseq_pad, const cx *tw) {
    typedef RegFFT<cx, M> RF;
    constexpr int TT = RF::TT, E1 = RF::E1, S = M + 1;
    const int t = threadIdx.x % TT, g = threadIdx.x / TT, ng = blockDim.x / TT;
    for (int base = 0; base < nseq_pad; base += ng) {
        const int seq = base + g;                  // nseq_pad is a multiple of the groups per warp
        if (seq < nseq_pad) {
            cx *col = Z + (size_t)seq * S;
            cx v[E1];
#pragma unroll
            for (int q = 0; q < E1; q++) v[q] = col[RF::in_index(t, q)];
            __syncwarp();
            RF::template run<INV, true>(v, t, col, tw);
#pragma unroll
            for (int r = 0; r < RF::R2; r++)
#pragma unroll
                for (int k2 = 0; k2 < TT; k2++) col[RF::out_index(t, r, k2)] = v[r * TT + k2];
        }
    }
}

// Column strips: NSP (a power of two) slots of M complex each, stride M + 1,
// loaded as cp.async copies (the caller waits), so all of a thread's elements
// are in flight at once.  Thread t always handles slot t % NSP and rows
// t / NSP + k * (BT / NSP), so the loop has shift-only indexing; slots past
// the block's columns are zeroed and never stored.
template <typename cx, int M, int NSP, int BT = 256>
__device__ __forceinline__ void issue_cols_fixed(cx *dst, const cx *__restrict__ src, const ColSlots &cs) {
    constexpr int S = M + 1, STEP = BT / NSP;
    static_assert(NSP <= BT && (NSP & (NSP - 1)) == 0, "NSP must be a power of two <= the block size");
    const int sl = threadIdx.x % NSP, i0 = threadIdx.x / NSP;
    const bool live = sl < cs.ns;
    const int col = live ? cs.col[sl] : 0;
#pragma unroll 8
    for (int i = i0; i < M; i += STEP) {
        if (live) {
            cp_async_elem(dst + (size_t)sl * S + i, src + (size_t)i * M + col);
        } else {
            cx v;
            v.x = 0;
            v.y = 0;
            dst[(size_t)sl * S + i] = v;
        }
    }
}

template <typename cx, int M, int NSP, int BT = 256>
__device__ __forceinline__ void store_cols_fixed(cx *__restrict__ dstg, const cx *src, const ColSlots &cs) {
    constexpr int S = M + 1, STEP = BT / NSP;
    const int sl = threadIdx.x % NSP, i0 = threadIdx.x / NSP;
    if (sl >= cs.ns) return;
    const int col = cs.col[sl];
#pragma unroll 8
    for (int i = i0; i < M; i += STEP) dstg[(size_t)i * M + col] = src[(size_t)sl * S + i];
}

// ---- the divergence of rho v in two passes instead of three --------------
// update_fft_rho (rho_functions.cpp:213-251) adds D = -i dt kfac (ir (rho vx)^
// + jr (rho vy)^) to rho^, and the new rho is Re(IFFT2(.))/M^2.  By linearity
// and because ir depends on the row wavenumber only (jr on the column one),
//   Re(IFFT2(-i ir FFT2(Fx)))/M^2 = Re(IFFT_i(-i ir FFT_i(Fx)))/M   (columns)
//   Re(IFFT2(-i jr FFT2(Fy)))/M^2 = Re(IFFT_j(-i jr FFT_j(Fy)))/M   (rows)
// with Fx = rho Re(vx), Fy = rho Re(vy) (load_fft_rho_v, :267-284): the
// transforms along the other direction cancel.  Re() keeps the Hermitian part
// of the multiplied spectrum, which for these odd multipliers is the spectrum
// with its Nyquist bin (ir or jr = -M/2, its own partner) set to zero.
//
// Pass C2 (rows): the inverse row transform of pass B's output gives vx + i vy;
// Fx is stored for pass D2, and Fy is differentiated along the row at once,
// dt kfac Re(IFFT_j(-i jr FFT_j(Fy)))/M stored beside it.  X holds Fx, the
// row term follows at X + Ntot M^2.
template <typename real, int M>
__global__ void __launch_bounds__(256, sizeof(real) == 4 ? 3 : 2) kr_boxC2(const typename Cplx<real>::type *__restrict__ Y1,
                                               real *__restrict__ X, const real *__restrict__ rho,
                                               const int *__restrict__ xc, const int *__restrict__ yc, BoxArgs a,
                                               real *__restrict__ vdx, real *__restrict__ vdy) {
    typedef typename Cplx<real>::type cx;
    typedef RegFFT<cx, M> RF;
    constexpr int TT = RF::TT, E1 = RF::E1, ROWS = BoxGeom<M>::ROWS;
    extern __shared__ unsigned char smraw[];
    cx *tw = (cx *)smraw;
    cx *scr = tw + M;
    RegFFT<cx, M>::twiddles_kt(tw);
    __syncthreads();
    const int t = threadIdx.x % TT, g = threadIdx.x / TT;
    const int n = blockIdx.y, i = blockIdx.x * ROWS + g;
    const int N = a.N;
    const int bi = xc[n] - a.z + 1, bj = yc[n] - a.z + 1;
    const size_t rowo = ((size_t)n * M + i) * M;
    real *Fx = X + rowo, *Dy = X + (size_t)a.Ntot * M * M + rowo;
    cx *sm = scr + g * M;
    cx v[E1];
#pragma unroll
    for (int q = 0; q < E1; q++) v[q] = Y1[rowo + RF::in_index(t, q)];
    RF::template run<true, true>(v, t, sm, tw);
    const real mm = (real)((double)M * (double)M);
    const real *rh = rho + (size_t)n * N * N + (size_t)(bi + i) * N + bj;
#pragma unroll
    for (int r = 0; r < RF::R2; r++)
#pragma unroll
        for (int k2 = 0; k2 < TT; k2++) {
            const int k = RF::out_index(t, r, k2);
            const cx val = v[r * TT + k2];
            const real rr = rh[k];
            Fx[k] = rr * val.x / mm;     // load_fft_rho_v, rho_functions.cpp:279
            cx fy;
            fy.x = rr * val.y / mm;
            fy.y = (real)0.0;
            if (vdx) { vdx[rowo + k] = val.x / mm; vdy[rowo + k] = val.y / mm; }
            sm[k] = fy;
        }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < E1; q++) v[q] = sm[RF::in_index(t, q)];
    __syncwarp();
    RF::template run<false, true>(v, t, sm, tw);
    // times -i jr, Nyquist bin zero
#pragma unroll
    for (int r = 0; r < RF::R2; r++)
#pragma unroll
        for (int k2 = 0; k2 < TT; k2++) {
            const int k = RF::out_index(t, r, k2);
            const real jr = (real)((k == M / 2) ? 0 : wrapk(k, M));
            const cx x = v[r * TT + k2];
            cx y;
            y.x = jr * x.y;
            y.y = -jr * x.x;
            sm[k] = y;
        }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < E1; q++) v[q] = sm[RF::in_index(t, q)];
    __syncwarp();
    RF::template run<true, true>(v, t, sm, tw);
    const real dtk = (real)(a.dt * a.kfac), inv_m = (real)(1.0 / (double)M);
#pragma unroll
    for (int r = 0; r < RF::R2; r++)
#pragma unroll
        for (int k2 = 0; k2 < TT; k2++) Dy[RF::out_index(t, r, k2)] = dtk * (v[r * TT + k2].x * inv_m);
}

// Pass D2 (columns): two real columns of Fx per complex transform (z = a + i b:
// the i-derivatives of a and b come back in the real and imaginary parts),
// then the new rho = rho + dt R + column term + row term, in place.
template <int M> struct BoxGeomD2 {
    static constexpr int TT = RegFFT<float2, M>::TT;
    static constexpr int GROUPS = 256 / TT;
    static constexpr int COLS = (2 * GROUPS < M) ? 2 * GROUPS : M;   // real columns per block
    static constexpr int NSQ = COLS / 2;                               // complex sequences per block
};
template <typename real, int M>
__global__ void __launch_bounds__(256, sizeof(real) == 4 ? 4 : 2) kr_boxD2(const real *__restrict__ X, real *__restrict__ rho,
                                                const real *__restrict__ Rb, const int *__restrict__ xc,
                                                const int *__restrict__ yc, BoxArgs a) {
    typedef typename Cplx<real>::type cx;
    constexpr int S = M + 1, NSQ = BoxGeomD2<M>::NSQ, COLS = BoxGeomD2<M>::COLS;
    constexpr int WG = BoxGeom<M>::WG;
    constexpr int NSP = (NSQ % WG == 0) ? NSQ : ((NSQ + WG - 1) / WG) * WG;   // padded to whole warps
    extern __shared__ unsigned char smraw[];
    cx *tw = (cx *)smraw;
    cx *Z = tw + M;                                   // [NSP][S]
    RegFFT<cx, M>::twiddles_kt(tw);
    const int n = blockIdx.y, c0 = blockIdx.x * COLS;
    const int N = a.N;
    const real *fx = X + (size_t)n * M * M, *dy = X + (size_t)a.Ntot * M * M + (size_t)n * M * M;
    // load column pairs: element (row i, pair p) -> Z[p][i], the two adjacent
    // reals of a pair as one cp.async copy (c0 + 2p is even, so it is aligned)
    constexpr int U = 4;
    for (int e = threadIdx.x; e < NSP * M; e += blockDim.x) {
        const int i = e / NSP, p = e - i * NSP;
        if (p < NSQ) {
            cp_async_elem(Z + (size_t)p * S + i, reinterpret_cast<const cx *>(fx + (size_t)i * M + c0 + 2 * p));
        } else {
            cx zz;
            zz.x = (real)0.0;
            zz.y = (real)0.0;
            Z[(size_t)p * S + i] = zz;
        }
    }
    cp_async_wait_all();
    __syncthreads();
    columns_fft<cx, M, false>(Z, NSP, tw);
    __syncthreads();
    // times -i ir, Nyquist bin zero
    for (int e = threadIdx.x; e < NSQ * M; e += blockDim.x) {
        const int p = e / M, k = e - p * M;
        const real ir = (real)((k == M / 2) ? 0 : wrapk(k, M));
        const cx x = Z[(size_t)p * S + k];
        cx y;
        y.x = ir * x.y;
        y.y = -ir * x.x;
        Z[(size_t)p * S + k] = y;
    }
    __syncthreads();
    columns_fft<cx, M, true>(Z, NSP, tw);
    __syncthreads();
    const real dtk = (real)(a.dt * a.kfac), inv_m = (real)(1.0 / (double)M), dt = (real)a.dt;
    const int bi = xc[n] - a.z + 1, bj = yc[n] - a.z + 1;
    real *rcell = rho + (size_t)n * N * N;
    const real *rb = Rb + (size_t)n * M * M;
    for (int e0 = threadIdx.x; e0 < NSQ * M; e0 += U * blockDim.x) {
        real ro[U][2], rr[U][2], yy[U][2];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int e = e0 + u * blockDim.x;
            if (e < NSQ * M) {
                const int i = e / NSQ, p = e - i * NSQ;
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int cc = c0 + 2 * p + h;
                    const size_t bo = (size_t)i * M + cc;
                    ro[u][h] = rcell[(size_t)(bi + i) * N + bj + cc];
                    rr[u][h] = rb[bo];
                    yy[u][h] = dy[bo];
                }
            }
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int e = e0 + u * blockDim.x;
            if (e < NSQ * M) {
                const int i = e / NSQ, p = e - i * NSQ;
                const cx w = Z[(size_t)p * S + i];
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int cc = c0 + 2 * p + h;
                    const real ti = dtk * ((h ? w.y : w.x) * inv_m);
                    rcell[(size_t)(bi + i) * N + bj + cc] = ro[u][h] + dt * rr[u][h] + (ti + yy[u][h]);
                }
            }
        }
    }
}

template <typename real, int M, int G, int BT>
__global__ void __launch_bounds__(BT, 1280 / BT) kr_boxB(typename Cplx<real>::type *__restrict__ Y1,
                                               const typename Cplx<real>::type *__restrict__ Y2,
                                               const unsigned char *__restrict__ clsT, BoxArgs a) {
    typedef typename Cplx<real>::type cx;
    constexpr int S = M + 1, WG = BoxGeom<M>::WG;
    extern __shared__ unsigned char smraw[];
    cx *tw = (cx *)smraw;
    RegFFT<cx, M>::twiddles_kt(tw);
    __shared__ ColSlots cs;
    const int n = blockIdx.y;
    if (threadIdx.x == 0) make_slots(cs, blockIdx.x * G, G, M);
    __syncthreads();
    constexpr int NSP = 2 * G;               // slots per block (primaries and partners, padded)
    static_assert(NSP % WG == 0, "slot count must be a multiple of the thread groups per warp");
    // pi_xy is real, so its 2-D spectrum at a pair's partner is the conjugate at
    // the primary: only the G primary columns of Y2 are transformed
    constexpr int NZ2 = ((G + WG - 1) / WG) * WG;   // padded to whole warps
    static_assert((NSP + NZ2) % WG == 0, "slot count must be a multiple of the thread groups per warp");
    cx *Z1 = tw + M, *Z2 = Z1 + (size_t)NSP * S;
    // the class map's columns of the block's slots (M bytes each, 16-byte
    // aligned rows of clsT) in flight while the spectra load
    unsigned char *scl = reinterpret_cast<unsigned char *>(Z2 + (size_t)NZ2 * S);   // [NSP][M]
    {
        constexpr int CH = M / 16;
        const unsigned char *cl = clsT + (size_t)n * M * M;
        for (int e = threadIdx.x; e < cs.ns * CH; e += BT) {
            const int sl = e / CH, q = e - sl * CH;
            cp_async_elem(reinterpret_cast<uint4 *>(scl + (size_t)sl * M) + q,
                          reinterpret_cast<const uint4 *>(cl + (size_t)cs.col[sl] * M) + q);
        }
    }
    issue_cols_fixed<cx, M, NSP, BT>(Z1, Y1 + (size_t)n * M * M, cs);
    issue_cols_fixed<cx, M, NZ2, BT>(Z2, Y2 + (size_t)n * M * M, cs);
    cp_async_wait_all();
    __syncthreads();
    columns_fft<cx, M, false>(Z1, NSP + NZ2, tw);   // Z2 follows Z1 with the same stride
    __syncthreads();
    for_pairs(cs, M, [&](int sa, int ka, int sb, int kb) {
        const cx z1a = Z1[(size_t)sa * S + ka], z1b = Z1[(size_t)sb * S + kb];
        const cx z2a = Z2[(size_t)sa * S + ka];
        cx z2b;
        z2b.x = z2a.x;
        z2b.y = -z2a.y;
        cx pxx_a, pyy_a, pxx_b, pyy_b;
        pxx_a.x = (real)0.5 * (z1a.x + z1b.x); pxx_a.y = (real)0.5 * (z1a.y - z1b.y);
        pyy_a.x = (real)0.5 * (z1a.y + z1b.y); pyy_a.y = (real)0.5 * (z1b.x - z1a.x);
        pxx_b.x = pxx_a.x; pxx_b.y = -pxx_a.y;
        pyy_b.x = pyy_a.x; pyy_b.y = -pyy_a.y;
        const int ca = cs.col[sa], cb = cs.col[sb];
        const real kxa = (real)(a.kfac * wrapk(ka, M)), kya = (real)(a.kfac * wrapk(ca, M));
        const real kxb = (real)(a.kfac * wrapk(kb, M)), kyb = (real)(a.kfac * wrapk(cb, M));
        const real eta_a = (real)a.visc[scl[(size_t)sa * M + ka]];
        const real eta_b = (real)a.visc[scl[(size_t)sb * M + kb]];
        const real fr = (real)a.friction;
        cx vxa, vya, vxb, vyb;
        velocity_at<real, cx>(kxa, kya, eta_a, fr, pxx_a, pyy_a, z2a, vxa, vya);
        velocity_at<real, cx>(kxb, kyb, eta_b, fr, pxx_b, pyy_b, z2b, vxb, vyb);
        cx hx, hy;
        hx.x = (real)0.5 * (vxa.x + vxb.x); hx.y = (real)0.5 * (vxa.y - vxb.y);
        hy.x = (real)0.5 * (vya.x + vyb.x); hy.y = (real)0.5 * (vya.y - vyb.y);
        cx pa, pb;
        pa.x = hx.x - hy.y; pa.y = hx.y + hy.x;
        pb.x = hx.x + hy.y; pb.y = hy.x - hx.y;
        Z1[(size_t)sa * S + ka] = pa;
        if (!(sa == sb && ka == kb)) Z1[(size_t)sb * S + kb] = pb;
    });
    __syncthreads();
    columns_fft<cx, M, true>(Z1, NSP, tw);
    __syncthreads();
    store_cols_fixed<cx, M, NSP, BT>(Y1 + (size_t)n * M * M, Z1, cs);
}

// ---- spectral solve for any even box size up to 512 that is not a power of
//      two (the reference's default zone_size 200, M = 398): the same steps as
//      the register passes with the Bluestein transforms of pfag_bluestein.cuh
//      (update_all_cortices, rho_functions.cpp:409-471).  Y1, Y2: [Ntot][M][M]
//      complex (Y2 also as two real [Ntot][M][M] planes: pi_xy, then the
//      fluxes); Rb: R; cm: the class map [Ntot][M][M] (row-major, not
//      transposed).

// stresses, reaction and class on the box: Y1 = pi_xx + i pi_yy, Y2 (as reals) = pi_xy
template <typename real>
__global__ void kg_stress(const real *__restrict__ phi, const real *__restrict__ rho, const real *__restrict__ lum,
                          const real *__restrict__ ecm, const int *__restrict__ xc, const int *__restrict__ yc,
                          BoxArgs a, typename Cplx<real>::type *__restrict__ Y1,
                          typename Cplx<real>::type *__restrict__ Y2, real *__restrict__ Rb,
                          unsigned char *__restrict__ cm) {
    const int n = blockIdx.y, M = a.M, N = a.N;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= M * M) return;
    const int i = e / M, j = e - i * M;
    const int bi = xc[n] - a.z + 1, bj = yc[n] - a.z + 1;
    const real *p1, *p2;
    nb_planes<real>(phi, a, n, p1, p2);
    const size_t NN = (size_t)N * N, s = (size_t)(bi + i) * N + (bj + j);
    const real *p = phi + (size_t)n * NN;
    real xx, yy, xy, rt;
    int c;
    box_stress<real>(a, p[s], p[s + N] - p[s - N], p[s + 1] - p[s - 1], rho[(size_t)n * NN + s], lum[s], ecm[s],
                     p1[s], p2[s], xx, yy, xy, rt, c);
    const size_t o = (size_t)n * M * M + e;
    Y1[o].x = xx;
    Y1[o].y = yy;
    reinterpret_cast<real *>(Y2)[o] = xy;   // a real plane, for a real-to-complex transform
    Rb[o] = rt;
    cm[o] = (unsigned char)c;
}

// k-space velocity (update_rho_velocity, rho_functions.cpp:133-190) on each
// pair {k, -k}: the pair's two spectra of pi_xx and pi_yy are unpacked from
// Y1, pi_xy's from its half spectrum (it is real, so its spectrum at -k is the
// conjugate at k), the
// velocity at k and at -k (each with the viscosity of its own index), and the
// Hermitian parts of vx and vy packed back as vx + i vy into Y1 at k and -k.
template <typename real>
__global__ void kg_velocity(typename Cplx<real>::type *__restrict__ Y1, const typename Cplx<real>::type *__restrict__ Hxy,
                            const unsigned char *__restrict__ cm, BoxArgs a) {
    typedef typename Cplx<real>::type cx;
    const int n = blockIdx.y, M = a.M;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= M * M) return;
    const int i = e / M, j = e - i * M;
    const int ib = (M - i) % M, jb = (M - j) % M, eb = ib * M + jb;
    if (eb < e) return;                      // the pair is done at its smaller index
    cx *y1 = Y1 + (size_t)n * M * M;
    const int H = M / 2 + 1;
    const cx *h = Hxy + (size_t)n * M * H;  // pi_xy's half spectrum [M][M/2+1]
    const unsigned char *cl = cm + (size_t)n * M * M;
    const cx z1a = y1[e], z1b = y1[eb];
    cx z2a, z2b;                             // pi_xy^ at k and at -k (its conjugate)
    if (j < H) {
        z2a = h[(size_t)i * H + j];
    } else {
        z2a = h[(size_t)ib * H + jb];
        z2a.y = -z2a.y;
    }
    z2b.x = z2a.x;
    z2b.y = -z2a.y;
    cx pxx_a, pyy_a, pxx_b, pyy_b;
    pxx_a.x = (real)0.5 * (z1a.x + z1b.x); pxx_a.y = (real)0.5 * (z1a.y - z1b.y);
    pyy_a.x = (real)0.5 * (z1a.y + z1b.y); pyy_a.y = (real)0.5 * (z1b.x - z1a.x);
    pxx_b.x = pxx_a.x; pxx_b.y = -pxx_a.y;
    pyy_b.x = pyy_a.x; pyy_b.y = -pyy_a.y;
    const real kxa = (real)(a.kfac * wrapk(i, M)), kya = (real)(a.kfac * wrapk(j, M));
    const real kxb = (real)(a.kfac * wrapk(ib, M)), kyb = (real)(a.kfac * wrapk(jb, M));
    const real fr = (real)a.friction;
    cx vxa, vya, vxb, vyb;
    velocity_at<real, cx>(kxa, kya, (real)a.visc[cl[e]], fr, pxx_a, pyy_a, z2a, vxa, vya);
    velocity_at<real, cx>(kxb, kyb, (real)a.visc[cl[eb]], fr, pxx_b, pyy_b, z2b, vxb, vyb);
    cx hx, hy;
    hx.x = (real)0.5 * (vxa.x + vxb.x); hx.y = (real)0.5 * (vxa.y - vxb.y);
    hy.x = (real)0.5 * (vya.x + vyb.x); hy.y = (real)0.5 * (vya.y - vyb.y);
    cx pa, pb;
    pa.x = hx.x - hy.y; pa.y = hx.y + hy.x;
    pb.x = hx.x + hy.y; pb.y = hy.x - hx.y;
    y1[e] = pa;
    if (eb != e) y1[eb] = pb;
}

// ---- phi update (cell_phase_functions.cpp:126-217) + normals
//      (useful_functions.cpp:356-388 with the periodic ghost map of :391-420)
// kf_update on shared-memory tiles: a block is a UR x UC tile of one cell's
// zone + ring (region W x W, W = 2z+2); phi, rho, T = psi - hfunc, h(lum) and
// h(ECM) are staged with a one-site halo, so T is formed once per site and
// the stencils read shared memory.  Normals on sites whose periodic ghost map
// is not the identity (a region touching the grid's ghost ring) read their
// mapped neighbours from global memory.  The FP32 build reads the lumen/ECM
// coupling term, which is the same for every cell, from G (kf_gel_coupling)
// and stages only phi, rho and T.
constexpr int UR = 16, UC = 64;

// The lumen / ECM part of the phi update's bracket (cell_phase_functions.cpp:
// 126-217): -beta_lum_cells h(lum) + eta_lum_cells lap9(h(lum)) / (4 dx^2)
// - beta_ECM_cells h(ECM) + eta_ECM_cells lap9(h(ECM)) / (4 dx^2).  No cell
// enters it, so the FP32 build forms it once per interior site here instead
// of once per cell and site in kf_update_tiled (rows and columns 0 and N-1,
// which no zone contains, are left alone).
template <typename real>
__global__ void kf_gel_coupling(const real *__restrict__ hl, const real *__restrict__ he, real *__restrict__ G,
                                DevParams P) {
    const int N = P.N;
    const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
    if (i < 1 || i > N - 2 || j < 1 || j > N - 2) return;
    const size_t k = (size_t)i * N + j;
    const real Ll = lap9<real>(hl[k], hl[k + N], hl[k - N], hl[k + 1], hl[k - 1], hl[k + N + 1], hl[k + N - 1],
                               hl[k - N - 1], hl[k - N + 1]);
    const real Le = lap9<real>(he[k], he[k + N], he[k - N], he[k + 1], he[k - 1], he[k + N + 1], he[k + N - 1],
                               he[k - N - 1], he[k - N + 1]);
    const real iq4 = (real)P.inv_q4;
    G[k] = -(real)P.beta_lum_cells * hl[k] + (real)P.eta_lum_cells * Ll * iq4 - (real)P.beta_ECM_cells * he[k] +
           (real)P.eta_ECM_cells * Le * iq4;
}

template <typename real>
__global__ void __launch_bounds__(256) kf_update_tiled(const real *__restrict__ phi, real *__restrict__ phin,
                                                       const real *__restrict__ rho, const real *__restrict__ hfunc,
                                                       const double *__restrict__ f0, const real *__restrict__ psi,
                                                       const real *__restrict__ hl, const real *__restrict__ he,
                                                       const int *__restrict__ xc, const int *__restrict__ yc,
                                                       DevParams P, real *__restrict__ Jc,
                                                       const real *__restrict__ G) {
    constexpr bool F32 = sizeof(real) == 4;
    constexpr int HR = UR + 2, HC = UC + 2, HRg = F32 ? 1 : HR;
    __shared__ real sphi[HR][HC], srho[HR][HC], sT[HR][HC], shl[HRg][HC], she[HRg][HC];
    const int n = blockIdx.z, N = P.N, z = P.zone, W = 2 * z + 2;
    const int r0 = blockIdx.y * UR, c0 = blockIdx.x * UC;        // region-local tile origin
    const int gi0 = xc[n] - z - 1 + r0, gj0 = yc[n] - z - 1 + c0;  // global origin
    const size_t NN = (size_t)N * N, base = (size_t)n * NN;
    for (int e = threadIdx.x; e < HR * HC; e += blockDim.x) {
        const int a = e / HC, b = e - a * HC;
        const int gi = min(max(gi0 - 1 + a, 0), N - 1), gj = min(max(gj0 - 1 + b, 0), N - 1);
        const size_t k = (size_t)gi * N + gj;
        sphi[a][b] = phi[base + k];
        srho[a][b] = rho[base + k];
        sT[a][b] = psi[k] - hfunc[base + k];
        if constexpr (!F32) {
            shl[a][b] = hl[k];
            she[a][b] = he[k];
        }
    }
    __syncthreads();
    const real dx = (real)P.dx, dt = (real)P.dt, tau = (real)P.tau, sigma = (real)P.sigma;
    const real c4 = (real)(1.0 / P.dx / P.dx / 4.0), inv2dx = (real)(1.0 / (2.0 * P.dx));
    const real q4 = (real)4.0 * dx * dx;
    const real fn0 = (real)f0[n];
    real *Jx = Jc + (size_t)n * 2 * W * W, *Jy = Jx + (size_t)W * W;
    for (int e = threadIdx.x; e < UR * UC; e += blockDim.x) {
        const int li = e / UC, lj = e - li * UC;
        const int rr = r0 + li, cc = c0 + lj;
        if (rr >= W || cc >= W) continue;
        const int gi = gi0 + li, gj = gj0 + lj;
        const int a = li + 1, b = lj + 1;                         // shared coordinates
        real ja, jb, g;
        if (gi >= 1 && gi <= N - 2 && gj >= 1 && gj <= N - 2) {
            ja = sphi[a + 1][b] - sphi[a - 1][b];
            jb = sphi[a][b + 1] - sphi[a][b - 1];
        } else {
            const size_t c = (size_t)ghost_src(gi, N) * N + ghost_src(gj, N);
            const real *p = phi + base;
            ja = p[c + N] - p[c - N];
            jb = p[c + 1] - p[c - 1];
        }
        const real q2 = c4 * (ja * ja + jb * jb);
        if constexpr (sizeof(real) == 8) g = sqrt(q2);
        else g = q2;                            // FP32 only tests g > 0 and uses rsqrt(q2)
        const size_t jo = (size_t)rr * W + cc;
        const size_t o = base + (size_t)gi * N + gj;
        const real f = sphi[a][b];
        real pn = f;
        if constexpr (sizeof(real) == 8) {
            // FP64: the reference's operation order, divisions included
            Jx[jo] = (g > (real)0.0) ? inv2dx * ja / g : (real)0.0;
            Jy[jo] = (g > (real)0.0) ? inv2dx * jb / g : (real)0.0;
            if (rr < 1 || rr > 2 * z || cc < 1 || cc > 2 * z) { phin[o] = f; continue; }
            if (g > (real)0.0) {
                pn -= (real)P.cpl / tau * (dt / dx / dx / (real)4.0) *
                      exp(-(f - (real)0.5) * (f - (real)0.5) / (real)2.0 / sigma / sigma) / sqrt((real)(2.0 * M_PI)) /
                      sigma * ((srho[a + 1][b] - srho[a - 1][b]) * ja + (srho[a][b + 1] - srho[a][b - 1]) * jb) / g;
            }
        } else {
            // FP32: constant factors folded, one reciprocal square root
            const real rg = (g > (real)0.0) ? rsqrtf(q2) : (real)0.0;
            Jx[jo] = inv2dx * ja * rg;
            Jy[jo] = inv2dx * jb * rg;
            if (rr < 1 || rr > 2 * z || cc < 1 || cc > 2 * z) { phin[o] = f; continue; }
            if (g > (real)0.0) {
                const real d = f - (real)0.5;
                pn -= (real)P.k_cpl * __expf(-d * d * (real)P.inv_2s2) *
                      ((srho[a + 1][b] - srho[a - 1][b]) * ja + (srho[a][b + 1] - srho[a][b - 1]) * jb) * rg;
            }
        }
        const real Tc = sT[a][b];
        const real LT = lap9<real>(Tc, sT[a + 1][b], sT[a - 1][b], sT[a][b + 1], sT[a][b - 1], sT[a + 1][b + 1],
                                   sT[a + 1][b - 1], sT[a - 1][b - 1], sT[a - 1][b + 1]);
        if constexpr (!F32) {
            const real Ll = lap9<real>(shl[a][b], shl[a + 1][b], shl[a - 1][b], shl[a][b + 1], shl[a][b - 1],
                                       shl[a + 1][b + 1], shl[a + 1][b - 1], shl[a - 1][b - 1], shl[a - 1][b + 1]);
            const real Le = lap9<real>(she[a][b], she[a + 1][b], she[a - 1][b], she[a][b + 1], she[a][b - 1],
                                       she[a + 1][b + 1], she[a + 1][b - 1], she[a - 1][b - 1], she[a - 1][b + 1]);
            pn += ((real)1.0 / tau) * f * ((real)1.0 - f) * dt *
                  (fn0 - (real)P.beta * Tc + (real)P.eta * LT / q4 - (real)P.beta_lum_cells * shl[a][b] +
                   (real)P.eta_lum_cells * Ll / q4 - (real)P.beta_ECM_cells * she[a][b] +
                   (real)P.eta_ECM_cells * Le / q4);
        } else {
            const real iq4 = (real)P.inv_q4;
            pn += (real)P.dt_tau * f * ((real)1.0 - f) *
                  (fn0 - (real)P.beta * Tc + (real)P.eta * LT * iq4 + G[(size_t)gi * N + gj]);
        }
        phin[o] = pn;
    }
}

// FP32 phi update + normals (cell_phase_functions.cpp:126-217,
// useful_functions.cpp:356-388) as a sliding window down the rows: a warp
// task is 30 columns x `rb` rows of one cell's zone + ring; lane l holds
// column cg*30 + l - 1 (lanes 0 and 31 only supply the left/right
// neighbours, read with warp shuffles).  Each thread keeps phi, rho and
// T = psi - hfunc of rows r-1, r, r+1 in registers; rows r+2 .. r+1+UPD_DEPTH
// of phi, rho, psi, hfunc and G are in flight as per-thread cp.async copies
// into a ring of UPD_DEPTH+1 shared-memory slots (a thread reads back only
// its own elements: no block barrier), one commit group per row; a row's
// slot is refilled one iteration after it was read.  Sites with a periodic
// ghost neighbour (a region touching the grid's ghost ring) take their
// normals from global memory through the ghost map.
constexpr int UPD_COLS = 30, UPD_DEPTH = 4, UPD_SLOTS = UPD_DEPTH + 1, UPD_THREADS = 256;
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int K>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(K) : "memory"); }

template <typename real>
__global__ void __launch_bounds__(UPD_THREADS, 5) kf_update_rows(const real *__restrict__ phi, real *__restrict__ phin,
                                                                 const real *__restrict__ rho,
                                                                 const real *__restrict__ hfunc,
                                                                 const double *__restrict__ f0,
                                                                 const real *__restrict__ psi,
                                                                 const real *__restrict__ G, const int *__restrict__ xc,
                                                                 const int *__restrict__ yc, DevParams P,
                                                                 real *__restrict__ Jc, int cgroups, int rchunks,
                                                                 int rb) {
    static_assert(sizeof(real) == 4, "the FP64 build keeps kf_update_tiled (reference operation order)");
    extern __shared__ float upd_ring[];                           // [UPD_SLOTS][5][UPD_THREADS]
    const int lane = threadIdx.x & 31;
    const int task = blockIdx.x * (UPD_THREADS >> 5) + (threadIdx.x >> 5);
    const int N = P.N, z = P.zone, W = 2 * z + 2;
    if (task >= P.Ntot * cgroups * rchunks) return;              // whole warps
    const int n = task / (cgroups * rchunks);
    const int rem = task - n * cgroups * rchunks;
    const int cg = rem / rchunks, rc = rem - cg * rchunks;
    const int cc = cg * UPD_COLS + lane - 1;                      // region column of this lane
    const int r0 = rc * rb, r1 = min(W, r0 + rb);
    const int gi0 = xc[n] - z - 1, gj0 = yc[n] - z - 1;         // region origin (grid)
    const int gj = gj0 + cc;
    const int gjc = min(max(gj, 0), N - 1);                      // clamped load column
    const bool out = lane >= 1 && lane <= UPD_COLS && cc < W;
    const size_t base = (size_t)n * N * N;
    // per-cell planes and 32-bit offsets (N^2 < 2^31)
    const real *__restrict__ pp = phi + base, *__restrict__ pr = rho + base, *__restrict__ ph = hfunc + base;
    auto row = [&](int r) { return (unsigned)(min(max(gi0 + r, 0), N - 1) * N + gjc); };
    float *ring = upd_ring + threadIdx.x;
    auto issue = [&](int r, int slot) {                          // row r into a ring slot, one commit group
        if (r <= r1) {
            const unsigned a = row(r);
            float *d = ring + slot * 5 * UPD_THREADS;
            cp_async_elem(d, pp + a);
            cp_async_elem(d + UPD_THREADS, pr + a);
            cp_async_elem(d + 2 * UPD_THREADS, psi + a);
            cp_async_elem(d + 3 * UPD_THREADS, ph + a);
            cp_async_elem(d + 4 * UPD_THREADS, G + a);
        }
        cp_async_commit();
    };
    const real dt_tau = (real)P.dt_tau, beta = (real)P.beta, eta = (real)P.eta, iq4 = (real)P.inv_q4;
    const real c4 = (real)(1.0 / P.dx / P.dx / 4.0), inv2dx = (real)(1.0 / (2.0 * P.dx));
    const real kcpl = (real)P.k_cpl, i2s2 = (real)P.inv_2s2;
    const real fn0 = (real)f0[n];
    real *Jx = Jc + (size_t)n * 2 * W * W, *Jy = Jx + (size_t)W * W;
    // rows r0+2 .. r0+1+UPD_DEPTH in flight (slot of row x: (x - r0 - 2) mod UPD_SLOTS)
#pragma unroll
    for (int k = 0; k < UPD_DEPTH; k++) issue(r0 + 2 + k, k);
    // window rows r-1, r, r+1 (phi p, rho q, T t) and G of row r
    real p0, p1, p2, q0, q1, q2, t0, t1, t2, g1;
    {
        const unsigned a = row(r0 - 1), b = row(r0), c = row(r0 + 1);
        p0 = pp[a]; p1 = pp[b]; p2 = pp[c];
        q0 = pr[a]; q1 = pr[b]; q2 = pr[c];
        t0 = psi[a] - ph[a]; t1 = psi[b] - ph[b]; t2 = psi[c] - ph[c];
        g1 = G[b];
    }
    real g2 = G[row(r0 + 1)];
    real tl0 = __shfl_up_sync(0xffffffffu, t0, 1), tr0 = __shfl_down_sync(0xffffffffu, t0, 1);
    real tl1 = __shfl_up_sync(0xffffffffu, t1, 1), tr1 = __shfl_down_sync(0xffffffffu, t1, 1);
    int rd = 0;                                                   // slot of row r+2
    for (int r = r0; r < r1; r++) {
        const int gi = gi0 + r;
        const bool zone = r >= 1 && r <= 2 * z && cc >= 1 && cc <= 2 * z;
        const real tl2 = __shfl_up_sync(0xffffffffu, t2, 1), tr2 = __shfl_down_sync(0xffffffffu, t2, 1);
        const real pl = __shfl_up_sync(0xffffffffu, p1, 1), prt = __shfl_down_sync(0xffffffffu, p1, 1);
        const real ql = __shfl_up_sync(0xffffffffu, q1, 1), qr = __shfl_down_sync(0xffffffffu, q1, 1);
        if (out) {
            real ja, jb;
            if (gi >= 1 && gi <= N - 2 && gj >= 1 && gj <= N - 2) {
                ja = p2 - p0;
                jb = prt - pl;
            } else {
                const unsigned c = (unsigned)(ghost_src(gi, N) * N + ghost_src(gj, N));
                ja = pp[c + N] - pp[c - N];
                jb = pp[c + 1] - pp[c - 1];
            }
            const real qq = c4 * (ja * ja + jb * jb);
            const real rg = (qq > (real)0.0) ? rsqrtf(qq) : (real)0.0;
            const unsigned jo = (unsigned)(r * W + cc);
            Jx[jo] = inv2dx * ja * rg;
            Jy[jo] = inv2dx * jb * rg;
            const real f = p1;
            real pn = f;
            if (zone) {
                if (qq > (real)0.0) {
                    const real d = f - (real)0.5;
                    pn -= kcpl * __expf(-d * d * i2s2) * ((q2 - q0) * ja + (qr - ql) * jb) * rg;
                }
                const real LT = lap9<real>(t1, t2, t0, tr1, tl1, tr2, tl2, tl0, tr0);
                pn += dt_tau * f * ((real)1.0 - f) * (fn0 - beta * t1 + eta * LT * iq4 + g1);
            }
            phin[base + (unsigned)(gi * N + gj)] = pn;
        }
        // slide the window down one row: row r+2 from its slot, then refill the
        // slot read one iteration ago with row r+2+UPD_DEPTH
        cp_async_wait<UPD_DEPTH - 1>();
        const float *sv = ring + rd * 5 * UPD_THREADS;
        p0 = p1; p1 = p2; p2 = sv[0];
        q0 = q1; q1 = q2; q2 = sv[UPD_THREADS];
        t0 = t1; t1 = t2; t2 = sv[2 * UPD_THREADS] - sv[3 * UPD_THREADS];
        g1 = g2; g2 = sv[4 * UPD_THREADS];
        tl0 = tl1; tr0 = tr1; tl1 = tl2; tr1 = tr2;
        const int wr = rd == 0 ? UPD_SLOTS - 1 : rd - 1;           // slot of row r+1, read last iteration
        issue(r + 2 + UPD_DEPTH, wr);
        rd = rd == UPD_SLOTS - 1 ? 0 : rd + 1;
    }
    cp_async_wait<0>();
}

// ---- persistent reshaping of all cells (cell_phase_functions.cpp:461-579)
struct ReshArgs {
    int N, z, Ntot, tpc, cap, rimax;   // tpc: strips per cell
    int it0;                  // first iteration the persistent kernel runs
    double A, B, scale, thr;
    int *K, *done, *cnt;
    double *part;
    unsigned *err;
};

// One reshaping strip of cell n (cell_phase_functions.cpp:486-552): zone
// rows [strip*RB, strip*RB + RB) of Q = P + F(P), a thread per zone column
// (strided by blockDim when the zone is wider than the block).  P's strip with its one-row, one-column ring and the
// normals' strip are staged in shared memory `sm` (3 (RB+2) W reals,
// W = 2z + 2) and the 3x3 / cross stencils read them there.  The ring, which
// no iteration writes, comes from `Pring` (the phi update's output, whose
// ring holds the old phi); the zone from P.  P's zone values are also stored
// into `Pout`: the reference keeps the penultimate iterate in phi (the copy
// phi <- phin at the top of its loop, cell_phase_functions.cpp:470-483), and
// iteration k's input is iterate k-1, so phi needs no copy after the loop.
// Returns this thread's sum of |Q - P| dx^2 / N_current
// (cell_phase_functions.cpp:554-561).  The caller synchronises the block
// before reusing `sm`.
template <typename real, int RB>
__device__ __forceinline__ double resh_tile(const real *__restrict__ P, const real *__restrict__ Pring,
                                            real *__restrict__ Q, real *__restrict__ Pout,
                                            const real *__restrict__ Jc, const int *__restrict__ xc,
                                            const int *__restrict__ yc, const ReshArgs &a, int n, int strip,
                                            real A, real B, real *sm) {
    const int N = a.N, z = a.z, Z = 2 * z, W = Z + 2;
    const size_t NN = (size_t)N * N;
    const int zi0 = xc[n] - z, zj0 = yc[n] - z;
    const int li0 = strip * RB;
    const int nr = min(RB, Z - li0);
    real *sP = sm, *sX = sm + (RB + 2) * W, *sY = sX + (RB + 2) * W;
    const size_t off = (size_t)n * NN + (size_t)(zi0 + li0 - 1) * N + (zj0 - 1);
    const real *p = P + off, *pr = Pring + off;
    const real *Jx = Jc + (size_t)n * 2 * W * W + (size_t)li0 * W, *Jy = Jx + (size_t)W * W;
    for (int c = threadIdx.x; c < W; c += blockDim.x) {
        const bool edge_col = (c == 0 || c == W - 1);
#pragma unroll
        for (int r = 0; r < RB + 2; r++) {
            if (r < nr + 2) {
                const int li = li0 + r - 1;                       // zone row; -1 and Z are the ring
                const bool ring = edge_col || li < 0 || li >= Z;
                cp_async_elem(sP + r * W + c, (ring ? pr : p) + (size_t)r * N + c);
            }
        }
    }
    // the normals' nr + 2 strip rows are contiguous in their W x W layout (and
    // in the tile): 16-byte copies when every address allows them
    {
        typedef typename std::conditional<sizeof(real) == 4, float4, double2>::type vec;
        constexpr int V = 16 / sizeof(real);
        const int nJ = (nr + 2) * W;
        const bool aligned = nJ % V == 0 &&
                             ((reinterpret_cast<size_t>(sX) | reinterpret_cast<size_t>(sY) |
                               reinterpret_cast<size_t>(Jx) | reinterpret_cast<size_t>(Jy)) & 15) == 0;
        if (aligned) {
            for (int k = threadIdx.x; k < nJ / V; k += blockDim.x) {
                cp_async_elem(reinterpret_cast<vec *>(sX) + k, reinterpret_cast<const vec *>(Jx) + k);
                cp_async_elem(reinterpret_cast<vec *>(sY) + k, reinterpret_cast<const vec *>(Jy) + k);
            }
        } else {
            for (int k = threadIdx.x; k < nJ; k += blockDim.x) {
                cp_async_elem(sX + k, Jx + k);
                cp_async_elem(sY + k, Jy + k);
            }
        }
    }
    cp_async_wait_all();
    __syncthreads();
    double acc = 0.0;
    float facc = 0.0f;
    const ReshConst kc = resh_const(a.A, a.B);
    for (int j = threadIdx.x; j < Z; j += blockDim.x) {       // zone columns (several per thread if Z > blockDim)
        const size_t qo = (size_t)n * NN + (size_t)(zi0 + li0) * N + zj0 + j;
        real *q = Q + qo, *po = Pout + qo;
        const int c = j + 1;
        // every row of the tile is computed (rows past the strip read stale tile
        // values and are not stored), so the loads a row shares with the next
        // one are not repeated
#pragma unroll
        for (int r = 0; r < RB; r++) {
            const bool live = r < nr;
            const int o = (r + 1) * W + c;
            real w[3][3];
#pragma unroll
            for (int di = 0; di < 3; di++)
#pragma unroll
                for (int dj = 0; dj < 3; dj++) w[di][dj] = sP[o + (di - 1) * W + dj - 1];
            const real old = w[1][1];
            if constexpr (sizeof(real) == 4) {
                const float nv = resh_update_f(kc, w, sX[o], sX[o + W], sX[o - W], sX[o + 1], sX[o - 1], sY[o],
                                               sY[o + W], sY[o - W], sY[o + 1], sY[o - 1], old);
                if (live) {
                    po[(size_t)r * N] = old;
                    q[(size_t)r * N] = nv;
                    facc += fabsf(nv - old);
                }
            } else {
                const real nv = resh_update<real>(A, B, w, sX[o], sX[o + W], sX[o - W], sX[o + 1], sX[o - 1],
                                                  sY[o], sY[o + W], sY[o - W], sY[o + 1], sY[o - 1], old);
                if (live) {
                    po[(size_t)r * N] = old;
                    q[(size_t)r * N] = nv;
                    acc += fabs((double)nv - (double)old) * a.scale;
                }
            }
        }
    }
    if constexpr (sizeof(real) == 4) acc = (double)facc * a.scale;
    return acc;
}

// Loop decision for cell n after iteration `it` (cell_phase_functions.cpp:
// 554-573) from its summed rdev; lane 0 of the deciding warp calls it.
__device__ __forceinline__ void resh_decide_cell(const ReshArgs &a, int n, int it, double rdev) {
    const int k = a.K[n] + 1;
    a.K[n] = k;
    bool stop = false;
    if (k - 1 > a.rimax) { atomicOr(a.err, ERRBIT_RELAX); stop = true; }
    if (rdev <= a.thr) stop = true;
    if (!stop && it == a.cap) { atomicOr(a.err, ERRBIT_ITER_CAP); stop = true; }
    if (stop) a.done[n] = it;
}

// Persistent reshaping of all cells (cell_phase_functions.cpp:461-579): the
// decision after iteration 1 (run by kf_resh_first; its per-strip partials
// part[n][tpc]), then iterations 2.. while a cell still moves; a task is one
// strip of one cell (resh_tile).  Iterate 0 is phin (the phi update's
// output), iterate 1 went to T; odd iterations read phin and write T, even
// ones read T and write phin, and every iteration stores its input into phi.
// rdev: each warp adds its tasks' sums into its own shared slot per cell (its
// tasks in a fixed order), the block writes per-cell partials, and after a
// grid barrier one warp per cell sums the blocks' partials in block order and
// takes the loop decision; a second barrier publishes it.  done[n] holds the
// iteration at which cell n stopped, so a block that reads it late still
// agrees on the iteration count.
constexpr int RESH_MAX_THREADS = 384;
template <typename real, int RB>
__device__ __forceinline__ void resh_loops(real *__restrict__ phi, real *__restrict__ phin, real *__restrict__ T,
                                           const real *__restrict__ Jc, const int *__restrict__ xc,
                                           const int *__restrict__ yc, const ReshArgs &a, double *wacc,
                                           cg::grid_group &grid) {
    const real A = (real)a.A, B = (real)a.B;
    const int strips = a.tpc;
    const int total = a.Ntot * strips;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    real *tile = reinterpret_cast<real *>(wacc + nw * a.Ntot);
    if (warp == 0) {
        for (int n = blockIdx.x; n < a.Ntot; n += gridDim.x) {
            const double rdev = warp_sum_fixed(a.part + (size_t)n * strips, strips);
            if (lane == 0) resh_decide_cell(a, n, a.it0 - 1, rdev);
        }
    }
    grid.sync();
    if (all_done_upto(a.done, a.Ntot, a.it0 - 1)) return;
    for (int it = a.it0; it <= a.cap; it++) {
        const real *P = (it & 1) ? phin : T;
        real *Q = (it & 1) ? T : phin;
        for (int k = threadIdx.x; k < nw * a.Ntot; k += blockDim.x) wacc[k] = 0.0;
        __syncthreads();
        for (int t = blockIdx.x; t < total; t += gridDim.x) {
            const int n = t / strips, strip = t - n * strips;
            const int d = *(volatile int *)&a.done[n];   // not written during this phase
            if (d != 0 && d < it) continue;
            double acc = resh_tile<real, RB>(P, phin, Q, phi, Jc, xc, yc, a, n, strip, A, B, tile);
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0) wacc[warp * a.Ntot + n] += acc;
            __syncthreads();
        }
        for (int n = threadIdx.x; n < a.Ntot; n += blockDim.x) {
            double sum = 0.0;
            for (int w2 = 0; w2 < nw; w2++) sum += wacc[w2 * a.Ntot + n];
            a.part[(size_t)n * gridDim.x + blockIdx.x] = sum;
        }
        grid.sync();
        if (warp == 0) {
            for (int n = blockIdx.x; n < a.Ntot; n += gridDim.x) {
                const int d = *(volatile int *)&a.done[n];
                if (d != 0 && d < it) continue;
                const double rdev = warp_sum_fixed(a.part + (size_t)n * gridDim.x, (int)gridDim.x);
                if (lane == 0) resh_decide_cell(a, n, it, rdev);
            }
        }
        grid.sync();
        if (all_done_upto(a.done, a.Ntot, it)) break;
    }
}

// Reshaping iteration 1 at full occupancy: one strip per block, P = phin
// (iterate 0) into Q = T, P stored into phi; per-strip partial sums (block
// order of warps fixed).
template <typename real, int RB>
__global__ void __maxnreg__(72) kf_resh_first(const real *__restrict__ P, real *__restrict__ Q,
                                                                   real *__restrict__ phi, const real *__restrict__ Jc,
                                                                   const int *__restrict__ xc,
                                                                   const int *__restrict__ yc, ReshArgs a) {
    extern __shared__ double tile_d[];
    const int n = blockIdx.y, strip = blockIdx.x;
    if (strip == 0 && threadIdx.x == 0) { a.K[n] = 0; a.done[n] = 0; }   // read from the next kernel on
    const double acc = resh_tile<real, RB>(P, P, Q, phi, Jc, xc, yc, a, n, strip, (real)a.A, (real)a.B,
                                           reinterpret_cast<real *>(tile_d));
    const double bs = block_sum_d(acc);
    if (threadIdx.x == 0) a.part[(size_t)n * a.tpc + strip] = bs;
}

// ---- persistent lumen / ECM update + reshaping
//      (cell_phase_functions.cpp:372-444, :709-871; useful_functions.cpp:422-462)
struct LumArgs {
    int N, cap, rimax, npsi;
    int it0;           // first iteration the persistent kernel runs
    double dx, dt, tau_lum, xi_lum, beta_lum_cells, eta_lum_cells, beta_lum_ECM;
    double alpha_ECM, tau_ECM, xi_ECM, beta_ECM_cells, eta_ECM_cells;
    double A, B, thr, rdev0;
    const double *part_e;
    double *part;      // [2][gridDim]
    int *K, *done, *cnt;
    unsigned *err;
    int no_copies;     // kl_relax_tma test hook: expect each stage's bytes but issue no copy, so no
                       // stage completes and the bounded waits run out (nothing in flight when they do)
    int wait_cap;      // kl_relax_tma: try_wait attempts per wait before it gives up
};

template <typename real>
__device__ __forceinline__ void dirichlet_val(int i, int j, int N, real side, real corner, real &v, bool &edge) {
    edge = (i == 0 || i == N - 1 || j == 0 || j == N - 1);
    if (edge) v = ((i == 0 || i == N - 1) && (j == 0 || j == N - 1)) ? corner : side;
}

// sum_ecm = sum h(ECM) dx^2 from the kf_psi block partials, fixed order
__global__ void kfl_sum_ecm(const double *__restrict__ part, int npart, double *__restrict__ out) {
    if (threadIdx.x < 32) {
        const double v = warp_sum_fixed(part, npart);
        if (threadIdx.x == 0) *out = v;
    }
}

// update_lumen_and_ECM (cell_phase_functions.cpp:372-444) with the boundary
// values of boundary_conditions_lumen_and_ECM (useful_functions.cpp:439-462)
template <typename real>
__global__ void kfl_update(const real *__restrict__ lum, const real *__restrict__ ecm, real *__restrict__ lumn,
                           real *__restrict__ ecmn, const real *__restrict__ psi, const real *__restrict__ hl,
                           const real *__restrict__ he, const double *__restrict__ sum_ecm, LumArgs a) {
    const int N = a.N;
    const int i = blockIdx.y * blockDim.y + threadIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0 && j == 0) {            // this step's loop counters of both fields (read from kl_relax on)
        for (int f = 0; f < 2; f++) { a.K[f] = 0; a.done[f] = 0; a.cnt[f] = 0; }
    }
    if (i >= N || j >= N) return;
    const size_t k = (size_t)i * N + j;
    if (i == 0 || i == N - 1 || j == 0 || j == N - 1) { lumn[k] = (real)0.0; ecmn[k] = (real)1.0; return; }
    const real dx = (real)a.dx, dt = (real)a.dt, q4 = (real)4.0 * dx * dx;
    const real elastic = (real)(a.alpha_ECM * ((double)N * (double)N * a.dx * a.dx - *sum_ecm));
    const real sv = psi[k];
    const real L = lap9<real>(sv, psi[k + N], psi[k - N], psi[k + 1], psi[k - 1], psi[k + N + 1], psi[k + N - 1],
                              psi[k - N - 1], psi[k - N + 1]);
    const real l = lum[k], e = ecm[k];
    real ln = l;
    ln += ((real)1.0 / (real)a.tau_lum) * l * ((real)1.0 - l) * dt *
          ((real)a.xi_lum - (real)a.beta_lum_cells * sv + (real)a.eta_lum_cells * L / q4 - (real)a.beta_lum_ECM * he[k]);
    real en = e;
    en += ((real)1.0 / (real)a.tau_ECM) * e * ((real)1.0 - e) * dt *
          (elastic + (real)a.xi_ECM - (real)a.beta_ECM_cells * sv + (real)a.eta_ECM_cells * L / q4 -
           (real)a.beta_lum_ECM * hl[k]);
    lumn[k] = ln;
    ecmn[k] = en;
}

// normals J = (1/(2dx)) grad(field_new) / |grad field_old| on every site, ghost
// sites through the periodic map (cell_phase_functions.cpp:722-771)
template <typename real>
__global__ void kfl_normals(const real *__restrict__ lum, const real *__restrict__ lumn, const real *__restrict__ ecm,
                            const real *__restrict__ ecmn, real *__restrict__ Jl, int N, double dx) {
    const int i = blockIdx.y * blockDim.y + threadIdx.y, j = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N || j >= N) return;
    const size_t NN = (size_t)N * N, k = (size_t)i * N + j;
    const size_t c = (size_t)ghost_src(i, N) * N + ghost_src(j, N);
    const real c4 = (real)(1.0 / dx / dx / 4.0), inv2dx = (real)(1.0 / (2.0 * dx));
#pragma unroll
    for (int f = 0; f < 2; f++) {
        const real *o = f ? ecm : lum;
        const real *nw = f ? ecmn : lumn;
        const real ga = o[c + N] - o[c - N], gb = o[c + 1] - o[c - 1];
        const real g = sqrt(c4 * (ga * ga + gb * gb));
        Jl[(size_t)(2 * f) * NN + k] = (g != (real)0.0) ? inv2dx * (nw[c + N] - nw[c - N]) / g : (real)0.0;
        Jl[(size_t)(2 * f + 1) * NN + k] = (g != (real)0.0) ? inv2dx * (nw[c + 1] - nw[c - 1]) / g : (real)0.0;
    }
}

// rows per tile of the persistent lumen / ECM iterations
constexpr int LUM_LRI = 4;

// Relaxation of the lumen and ECM fields (cell_phase_functions.cpp:774-869)
// from iteration a.it0 on, inside the persistent kernel kf_relax_loops.
template <typename real>
__device__ __forceinline__ void lum_loops(real *__restrict__ lum, real *__restrict__ lumn, real *__restrict__ ecm,
                                          real *__restrict__ ecmn, const real *__restrict__ Jl, const LumArgs &a,
                                          cg::grid_group &grid) {
    const int N = a.N;
    const size_t NN = (size_t)N * N;
    __shared__ int s_last, s_skip;
    // phase R: relaxation loops of both fields, iteration k reads P, writes Q.
    // Tiles of LRI rows x blockDim columns; one thread per column with its
    // column of the strip (plus a halo row each side) in registers and the
    // left/right neighbours from the adjacent lanes.
    const real A = (real)a.A, B = (real)a.B;
    const double dx2 = a.dx * a.dx;
    constexpr int LRI = LUM_LRI;
    const int lane = threadIdx.x & 31;
    const int tiles_i = (N + LRI - 1) / LRI, tiles_j = (N + blockDim.x - 1) / blockDim.x;
    const int ntiles = tiles_i * tiles_j;
    // iterations before it0 ran as separate kernels: nothing left to do?
    if (threadIdx.x < 32 && all_done_upto(a.done, 2, a.it0 - 1)) s_skip = 1;
    else if (threadIdx.x == 0) s_skip = 0;
    __syncthreads();
    if (s_skip) return;
    __syncthreads();
    for (int it = a.it0; it <= a.cap; it++) {
        for (int f = 0; f < 2; f++) {
            if (threadIdx.x == 0) {
                const int d = *(volatile int *)&a.done[f];
                s_skip = (d != 0 && d < it);
            }
            __syncthreads();
            const bool skip = s_skip;
            __syncthreads();
            if (skip) continue;
            real *P = (it & 1) ? (f ? ecmn : lumn) : (f ? ecm : lum);
            real *Q = (it & 1) ? (f ? ecm : lum) : (f ? ecmn : lumn);
            const real side = f ? (real)1.0 : (real)0.0;
            const real *Jx = Jl + (size_t)(2 * f) * NN, *Jy = Jl + (size_t)(2 * f + 1) * NN;
            double acc = 0.0;
            for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
                const int ti = tile / tiles_j, tj = tile - ti * tiles_j;
                const int i0 = ti * LRI;
                const int jraw = tj * blockDim.x + threadIdx.x;
                const bool col_ok = jraw < N;
                const int jj = min(jraw, N - 1);
                real pc[LRI + 2], pl[LRI + 2], pr[LRI + 2], xc_[LRI + 2], yc_[LRI + 2];
                real xl[LRI], xr[LRI], yl[LRI], yr[LRI];
#pragma unroll
                for (int r = 0; r < LRI + 2; r++) {
                    const int ii = min(max(i0 - 1 + r, 0), N - 1);
                    const size_t k = (size_t)ii * N + jj;
                    pc[r] = P[k];
                    xc_[r] = Jx[k];
                    yc_[r] = Jy[k];
                }
#pragma unroll
                for (int r = 0; r < LRI + 2; r++) {
                    pl[r] = __shfl_up_sync(0xffffffffu, pc[r], 1);
                    pr[r] = __shfl_down_sync(0xffffffffu, pc[r], 1);
                }
#pragma unroll
                for (int r = 0; r < LRI; r++) {
                    xl[r] = __shfl_up_sync(0xffffffffu, xc_[r + 1], 1);
                    xr[r] = __shfl_down_sync(0xffffffffu, xc_[r + 1], 1);
                    yl[r] = __shfl_up_sync(0xffffffffu, yc_[r + 1], 1);
                    yr[r] = __shfl_down_sync(0xffffffffu, yc_[r + 1], 1);
                }
                if (lane == 0 || lane == 31) {
                    const int jn = lane == 0 ? max(jj - 1, 0) : min(jj + 1, N - 1);
#pragma unroll
                    for (int r = 0; r < LRI + 2; r++) {
                        const int ii = min(max(i0 - 1 + r, 0), N - 1);
                        const real v = P[(size_t)ii * N + jn];
                        if (lane == 0) pl[r] = v; else pr[r] = v;
                    }
#pragma unroll
                    for (int r = 0; r < LRI; r++) {
                        const int ii = min(i0 + r, N - 1);
                        const size_t k = (size_t)ii * N + jn;
                        if (lane == 0) { xl[r] = Jx[k]; yl[r] = Jy[k]; } else { xr[r] = Jx[k]; yr[r] = Jy[k]; }
                    }
                }
#pragma unroll
                for (int r = 0; r < LRI; r++) {
                    const int ii = i0 + r;
                    if (ii < N && col_ok) {
                        real v;
                        bool edge;
                        dirichlet_val<real>(ii, jj, N, side, (real)0.0, v, edge);
                        if (!edge) {
                            real w[3][3];
                            w[0][0] = pl[r];     w[0][1] = pc[r];     w[0][2] = pr[r];
                            w[1][0] = pl[r + 1]; w[1][1] = pc[r + 1]; w[1][2] = pr[r + 1];
                            w[2][0] = pl[r + 2]; w[2][1] = pc[r + 2]; w[2][2] = pr[r + 2];
                            if constexpr (sizeof(real) == 4)
                                v = resh_update_f(resh_const(a.A, a.B), w, xc_[r + 1], xc_[r + 2], xc_[r], xr[r],
                                                  xl[r], yc_[r + 1], yc_[r + 2], yc_[r], yr[r], yl[r], w[1][1]);
                            else
                                v = resh_update<real>(A, B, w, xc_[r + 1], xc_[r + 2], xc_[r], xr[r], xl[r],
                                                      yc_[r + 1], yc_[r + 2], yc_[r], yr[r], yl[r], w[1][1]);
                        }
                        acc += fabs((double)v - (double)pc[r + 1]) * dx2;
                        Q[(size_t)ii * N + jj] = v;
                    }
                }
            }
            const double bs = block_sum_d(acc);
            if (threadIdx.x == 0) {
                a.part[(size_t)f * gridDim.x + blockIdx.x] = bs;
                __threadfence();
                const int ticket = atomicAdd(&a.cnt[f], 1);
                s_last = (ticket == (int)gridDim.x - 1);
            }
            __syncthreads();
            if (s_last && threadIdx.x < 32) {
                __threadfence();
                const double rdev = warp_sum_fixed(a.part + (size_t)f * gridDim.x, (int)gridDim.x);
                if (threadIdx.x == 0) {
                const int k2 = a.K[f] + 1;
                a.K[f] = k2;
                bool stop = false;
                if (k2 - 1 > a.rimax) { atomicOr(a.err, ERRBIT_RELAX); stop = true; }
                if (rdev <= a.thr) stop = true;
                if (!stop && it == a.cap) { atomicOr(a.err, ERRBIT_ITER_CAP); stop = true; }
                if (stop) a.done[f] = it;
                a.cnt[f] = 0;
                }
            }
            __syncthreads();
        }
        grid.sync();
        const int d0 = *(volatile int *)&a.done[0], d1 = *(volatile int *)&a.done[1];
        if (d0 != 0 && d0 <= it && d1 != 0 && d1 <= it) break;
    }
}

// One relaxation iteration `it` of field f = blockIdx.y (0 lumen, 1 ECM;
// cell_phase_functions.cpp:774-869) on a tile of LRB grid rows x blockDim
// columns, with the field and its normals staged in shared memory (one-site
// halo, clamped at the grid edge, where the Dirichlet sites take their side
// values and no stencil).  Fields already converged return at once.  The
// block's sum of |Q - P| dx^2 goes to part[f][block] (fixed order).
constexpr int LRB = 8;
template <typename real>
__global__ void __launch_bounds__(256) kl_relax(real *__restrict__ lum, real *__restrict__ lumn,
                                                real *__restrict__ ecm, real *__restrict__ ecmn,
                                                const real *__restrict__ Jl, LumArgs a, int it,
                                                double *__restrict__ part) {
    extern __shared__ double lsm_d[];
    const int f = blockIdx.y;
    {
        const int d = a.done[f];    // written only by kl_decide, between launches
        if (d != 0 && d < it) return;
    }
    const int N = a.N;
    const size_t NN = (size_t)N * N;
    const int TB = blockDim.x, TW = TB + 2;
    const int tiles_j = (N + TB - 1) / TB;
    const int ti = blockIdx.x / tiles_j, tj = blockIdx.x - ti * tiles_j;
    const int i0 = ti * LRB, j0 = tj * TB;
    real *sP = reinterpret_cast<real *>(lsm_d), *sX = sP + (LRB + 2) * TW, *sY = sX + (LRB + 2) * TW;
    const real *P = (it & 1) ? (f ? ecmn : lumn) : (f ? ecm : lum);
    real *Q = (it & 1) ? (f ? ecm : lum) : (f ? ecmn : lumn);
    const real *Jx = Jl + (size_t)(2 * f) * NN, *Jy = Jl + (size_t)(2 * f + 1) * NN;
#pragma unroll
    for (int r = 0; r < LRB + 2; r++) {
        const size_t row = (size_t)min(max(i0 - 1 + r, 0), N - 1) * N;
        for (int cc = threadIdx.x; cc < TW; cc += TB) {
            const size_t k = row + min(max(j0 - 1 + cc, 0), N - 1);
            cp_async_elem(sP + r * TW + cc, P + k);
            cp_async_elem(sX + r * TW + cc, Jx + k);
            cp_async_elem(sY + r * TW + cc, Jy + k);
        }
    }
    cp_async_wait_all();
    __syncthreads();
    const real A = (real)a.A, B = (real)a.B, side = f ? (real)1.0 : (real)0.0;
    const ReshConst kc = resh_const(a.A, a.B);
    const double dx2 = a.dx * a.dx;
    const int jj = j0 + threadIdx.x;
    double acc = 0.0;
    float facc = 0.0f;
    if (jj < N) {
        // every tile row holds staged (clamped) values: the stencil runs on all
        // of them, only the stores and sums are predicated, so the loads a row
        // shares with the next one are not repeated
#pragma unroll
        for (int r = 0; r < LRB; r++) {
            const int ii = i0 + r;
            const int o = (r + 1) * TW + threadIdx.x + 1;
            real w[3][3];
#pragma unroll
            for (int di = 0; di < 3; di++)
#pragma unroll
                for (int dj = 0; dj < 3; dj++) w[di][dj] = sP[o + (di - 1) * TW + dj - 1];
            const real old = w[1][1];
            real nv;
            if constexpr (sizeof(real) == 4)
                nv = resh_update_f(kc, w, sX[o], sX[o + TW], sX[o - TW], sX[o + 1], sX[o - 1], sY[o],
                                   sY[o + TW], sY[o - TW], sY[o + 1], sY[o - 1], old);
            else
                nv = resh_update<real>(A, B, w, sX[o], sX[o + TW], sX[o - TW], sX[o + 1], sX[o - 1], sY[o],
                                       sY[o + TW], sY[o - TW], sY[o + 1], sY[o - 1], old);
            if (ii < N) {
                real v;
                bool edge;
                dirichlet_val<real>(ii, jj, N, side, (real)0.0, v, edge);
                if (!edge) v = nv;
                if constexpr (sizeof(real) == 4) facc += fabsf(v - old);
                else acc += fabs((double)v - (double)old) * dx2;
                Q[(size_t)ii * N + jj] = v;
            }
        }
    }
    if constexpr (sizeof(real) == 4) acc = (double)facc * dx2;
    const double bs = block_sum_d(acc);
    if (threadIdx.x == 0) part[(size_t)f * gridDim.x + blockIdx.x] = bs;
}

// Loop decision after iteration `it` of kl_relax: one warp per field, the
// tiles' partials summed in tile order (cell_phase_functions.cpp:851-868).
__global__ void kl_decide(LumArgs a, int it, const double *__restrict__ part, int ntiles) {
    const int f = blockIdx.x;
    {
        const int d = a.done[f];
        if (d != 0 && d < it) return;
    }
    const double rdev = warp_sum_fixed(part + (size_t)f * ntiles, ntiles);
    if (threadIdx.x == 0) {
        const int k2 = a.K[f] + 1;
        a.K[f] = k2;
        bool stop = false;
        if (k2 - 1 > a.rimax) { atomicOr(a.err, ERRBIT_RELAX); stop = true; }
        if (rdev <= a.thr) stop = true;
        if (!stop && it == a.cap) { atomicOr(a.err, ERRBIT_ITER_CAP); stop = true; }
        if (stop) a.done[f] = it;
    }
}

// FP32 lumen / ECM relaxation iteration (the kl_relax step) on tiles of
// LT_R rows x LT_C columns staged by TMA (cp.async.bulk.tensor 2-D loads of
// P, J_x, J_y).  A box is LT_W = LT_C + 8 columns wide and starts LT_HX = 4
// columns left of the tile (a 16-byte aligned x, as TMA requires) and one row
// above it, so the tile's halo rows and columns come with it; sites outside
// the grid are zero-filled and feed only the Dirichlet border, which is
// overwritten.  A persistent block takes the tiles of the active fields in
// turn with LT_STAGES stages: the next tiles' copies are in flight while it
// computes one.  Copy completion is an mbarrier with a transaction count;
// every wait is bounded (ERRBIT_TIMEOUT, and the block drains its other
// copies before returning).  Tile partials of the rdev sum go to
// part[f][tile] in tile order, as kl_decide reads them.
constexpr int LT_R = 16, LT_C = 120, LT_W = 128, LT_HX = 4, LT_THREADS = 128, LT_STAGES = 2;
constexpr int LT_BOX = (LT_R + 2) * LT_W;                    // floats per plane per stage
struct LumMaps {
    CUtensorMap P[4];      // lum, lumn, ECM, ECMn as [N][N] FP32
    CUtensorMap J[4];      // the lumen / ECM normals: planes 0..3 of Jl
};
__device__ __forceinline__ unsigned lt_smem(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ bool lt_wait(unsigned bar, unsigned parity, int cap) {
    for (int k = 0; k < cap; k++) {
        unsigned ok;
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                     " selp.u32 %0, 1, 0, p;\n}\n"
                     : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
        if (ok) return true;
    }
    return false;
}
__device__ __forceinline__ void lt_load(const CUtensorMap *map, unsigned dst, unsigned bar, int x, int y) {
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n"
                 ::"r"(dst), "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(bar)
                 : "memory");
}

__global__ void __launch_bounds__(LT_THREADS) kl_relax_tma(const __grid_constant__ LumMaps maps,
                                                           float *__restrict__ lum, float *__restrict__ lumn,
                                                           float *__restrict__ ecm, float *__restrict__ ecmn,
                                                           LumArgs a, int it, double *__restrict__ part) {
    // TMA destinations 128-byte aligned (the dynamic allocation has 128 bytes
    // of slack for it; an aligned extern declaration would pad every kernel's
    // shared memory in this file)
    extern __shared__ unsigned char lt_raw[];
    float *tiles = reinterpret_cast<float *>(
        lt_raw + ((128u - (lt_smem(lt_raw) & 127u)) & 127u));                      // [stage][3][LT_R+2][LT_W]
    unsigned long long *bars = reinterpret_cast<unsigned long long *>(tiles + (size_t)LT_STAGES * 3 * LT_BOX);
    const int N = a.N;
    const int tj_n = (N + LT_C - 1) / LT_C, tpf = ((N + LT_R - 1) / LT_R) * tj_n;
    int fl[2], nf = 0;
    for (int f = 0; f < 2; f++) {
        const int d = a.done[f];                 // written only by kl_decide, between launches
        if (!(d != 0 && d < it)) fl[nf++] = f;
    }
    const int total = nf * tpf;
    if ((int)blockIdx.x >= total) return;
    const int c = threadIdx.x;
    if (c == 0) {
        for (int st = 0; st < LT_STAGES; st++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(lt_smem(&bars[st])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    constexpr unsigned BYTES = 3u * LT_BOX * sizeof(float);
    auto issue = [&](int k) {                    // copies of the block's k-th tile into stage k % LT_STAGES
        const int t = blockIdx.x + k * gridDim.x;
        if (t >= total) return;
        const int f = fl[t / tpf], loc = t - (t / tpf) * tpf;
        const int ti = loc / tj_n, tj = loc - ti * tj_n;
        const int st = k % LT_STAGES;
        const unsigned bar = lt_smem(&bars[st]);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(BYTES) : "memory");
        if (a.no_copies) return;
        float *dst = tiles + (size_t)st * 3 * LT_BOX;
        const int x = tj * LT_C - LT_HX, y = ti * LT_R - 1;        // x: a multiple of 4 floats
        lt_load(&maps.P[2 * f + (it & 1)], lt_smem(dst), bar, x, y);
        lt_load(&maps.J[2 * f], lt_smem(dst + LT_BOX), bar, x, y);
        lt_load(&maps.J[2 * f + 1], lt_smem(dst + 2 * LT_BOX), bar, x, y);
    };
    if (c == 0)
        for (int k = 0; k < LT_STAGES; k++) issue(k);
    const ReshConst kc = resh_const(a.A, a.B);
    const double dx2 = a.dx * a.dx;
    for (int k = 0;; k++) {
        const int t = blockIdx.x + k * gridDim.x;
        if (t >= total) break;
        const int f = fl[t / tpf], loc = t - (t / tpf) * tpf;
        const int ti = loc / tj_n, tj = loc - ti * tj_n;
        const int i0 = ti * LT_R, j0 = tj * LT_C;
        const int st = k % LT_STAGES;
        float *Q = (it & 1) ? (f ? ecm : lum) : (f ? ecmn : lumn);
        const unsigned parity = (unsigned)((k / LT_STAGES) & 1);
        const bool got = lt_wait(lt_smem(&bars[st]), parity, a.wait_cap);
        if (!__syncthreads_and(got)) {            // the same decision in every thread
            if (c == 0) {
                atomicOr(a.err, ERRBIT_TIMEOUT);
                // wait once more (bounded) for this stage's copies and for the
                // other stages' copies in flight before the block leaves
                for (int kk = k; kk < k + LT_STAGES; kk++)
                    if (blockIdx.x + kk * gridDim.x < total)
                        lt_wait(lt_smem(&bars[kk % LT_STAGES]), (unsigned)((kk / LT_STAGES) & 1), a.wait_cap);
            }
            __syncthreads();
            return;
        }
        // box row rr = tile row + 1, box column = tile column + LT_HX
        const float *sP = tiles + (size_t)st * 3 * LT_BOX + LT_HX, *sX = sP + LT_BOX, *sY = sX + LT_BOX;
        const float side_v = f ? 1.0f : 0.0f;
        const int jj = j0 + c;
        float facc = 0.0f;
        if (c < LT_C && jj < N) {
#pragma unroll 4
            for (int r = 0; r < LT_R; r++) {
                const int ii = i0 + r;
                if (ii >= N) break;
                const int o = (r + 1) * LT_W + c;
                float w[3][3];
#pragma unroll
                for (int di = 0; di < 3; di++)
#pragma unroll
                    for (int dj = 0; dj < 3; dj++) w[di][dj] = sP[o + (di - 1) * LT_W + dj - 1];
                const float old = w[1][1];
                const float nv = resh_update_f(kc, w, sX[o], sX[o + LT_W], sX[o - LT_W], sX[o + 1], sX[o - 1], sY[o],
                                               sY[o + LT_W], sY[o - LT_W], sY[o + 1], sY[o - 1], old);
                float v;
                bool edge;
                dirichlet_val<float>(ii, jj, N, side_v, 0.0f, v, edge);
                if (!edge) v = nv;
                facc += fabsf(v - old);
                Q[(size_t)ii * N + jj] = v;
            }
        }
        const double bs = block_sum_d((double)facc * dx2);    // ends with a block barrier
        if (c == 0) part[(size_t)f * tpf + loc] = bs;
        if (c == 0) issue(k + LT_STAGES);         // every thread is past this stage (barrier above)
    }
}

// The step ends with lum <- lumn, ECM <- ECMn (run_with_active_gels.cpp:179-181):
// after an odd iteration count the last iterate already sits in lum / ECM.
// Copies field f when its count is even and its loop stopped at an iteration
// in [lo, hi]; 16-byte vectors (cudaMalloc'd fields are 256-byte aligned),
// then the tail, over threads tid = 0 .. stride-1.
template <typename real>
__device__ __forceinline__ void lum_copy_fields(real *__restrict__ lum, const real *__restrict__ lumn,
                                                real *__restrict__ ecm, const real *__restrict__ ecmn,
                                                const int *__restrict__ K, const int *__restrict__ done, int N,
                                                int lo, int hi, size_t tid, size_t stride) {
    typedef typename std::conditional<sizeof(real) == 4, float4, double2>::type vec;
    constexpr int PER = 16 / sizeof(real);
    const size_t NN = (size_t)N * N, nv = NN / PER;
    for (int f = 0; f < 2; f++) {
        const int d = *(volatile const int *)&done[f];
        if ((*(volatile const int *)&K[f] & 1) || d < lo || d > hi) continue;
        real *dst = f ? ecm : lum;
        const real *src = f ? ecmn : lumn;
        for (size_t k = tid; k < nv; k += stride) reinterpret_cast<vec *>(dst)[k] = reinterpret_cast<const vec *>(src)[k];
        for (size_t k = nv * PER + tid; k < NN; k += stride) dst[k] = src[k];
    }
}
// the copy for fields whose loops stopped at iterations 1 .. hi (the regular kernels)
template <typename real>
__global__ void kl_copy(real *__restrict__ lum, const real *__restrict__ lumn, real *__restrict__ ecm,
                        const real *__restrict__ ecmn, const int *__restrict__ K, const int *__restrict__ done, int N,
                        int hi) {
    lum_copy_fields<real>(lum, lumn, ecm, ecmn, K, done, N, 1, hi, (size_t)blockIdx.x * blockDim.x + threadIdx.x,
                          (size_t)gridDim.x * blockDim.x);
}

// The next step's centroid sums (find_centres_cells, useful_functions.cpp:
// 193-227) over each cell's support rectangle of the reshaped phi: a warp
// takes CG rows of one rectangle at once (the loop over 32-column chunks is
// unrolled by 8, so up to 8 CG loads per lane are in flight), exact integer
// sums added atomically into acc (zeroed before
// the grid barrier that precedes this).  Nothing writes phi between the end
// of the reshaping loops and the next step's centroids.
template <typename real>
__device__ __forceinline__ void centroid_rows(const real *__restrict__ phi, const int4 *__restrict__ rect, int N,
                                              int Ntot, long long *__restrict__ acc) {
    constexpr int CG = 4;
    const int lane = threadIdx.x & 31;
    const int nw = blockDim.x >> 5;
    const int nwt = gridDim.x * nw;
    const int groups = (N + CG - 1) / CG;
    for (int t = blockIdx.x * nw + (threadIdx.x >> 5); t < Ntot * groups; t += nwt) {
        const int n = t / groups, i0 = (t - n * groups) * CG;
        const int4 r = rect[n];
        if (i0 + CG <= r.x || i0 >= r.y) continue;                 // warp-uniform
        const real *p = phi + (size_t)n * N * N;
        int cnt = 0, sx = 0, sy = 0;                               // < CG N sites of index < N per lane
#pragma unroll 8
        for (int j = r.z + lane; j < r.w; j += 32) {
            real v[CG];
#pragma unroll
            for (int k = 0; k < CG; k++) {
                const int i = i0 + k;
                v[k] = (i >= r.x && i < r.y) ? p[(size_t)i * N + j] : (real)0.0;
            }
#pragma unroll
            for (int k = 0; k < CG; k++)
                if (v[k] > (real)0.5) { cnt++; sx += i0 + k; sy += j; }
        }
        for (int o = 16; o > 0; o >>= 1) {
            cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
            sx += __shfl_xor_sync(0xffffffffu, sx, o);
            sy += __shfl_xor_sync(0xffffffffu, sy, o);
        }
        if (lane == 0 && cnt) {
            atomicAdd((unsigned long long *)&acc[3 * n + 0], (unsigned long long)cnt);
            atomicAdd((unsigned long long *)&acc[3 * n + 1], (unsigned long long)sx);
            atomicAdd((unsigned long long *)&acc[3 * n + 2], (unsigned long long)sy);
        }
    }
}

// The step's device-side loops in one persistent cooperative kernel: the
// cells' reshaping from iteration ra.it0 - 1's decision on, the next step's
// centroid sums of the reshaped cells, the lumen / ECM relaxation from
// iteration la.it0 on, then lum <- lumn, ECM <- ECMn for the fields whose
// loops ran here.
template <typename real, int RB>
__global__ void __launch_bounds__(RESH_MAX_THREADS, 2) kf_relax_loops(real *__restrict__ phi, real *__restrict__ phin,
                                                                    real *__restrict__ T, const real *__restrict__ Jc,
                                                                    const int *__restrict__ xc,
                                                                    const int *__restrict__ yc, ReshArgs ra,
                                                                    real *__restrict__ lum, real *__restrict__ lumn,
                                                                    real *__restrict__ ecm, real *__restrict__ ecmn,
                                                                    const real *__restrict__ Jl, LumArgs la,
                                                                    const int4 *__restrict__ rect,
                                                                    long long *__restrict__ cacc) {
    cg::grid_group grid = cg::this_grid();
    extern __shared__ double wacc[];          // [warps][Ntot], then the strip tile
    if (blockIdx.x == 0)                      // consumed by this step's kf_hpsi; refilled below
        for (int k = threadIdx.x; k < 3 * ra.Ntot; k += blockDim.x) cacc[k] = 0;
    resh_loops<real, RB>(phi, phin, T, Jc, xc, yc, ra, wacc, grid);   // ends with a grid barrier
    centroid_rows<real>(phi, rect, ra.N, ra.Ntot, cacc);
    lum_loops<real>(lum, lumn, ecm, ecmn, Jl, la, grid);
    lum_copy_fields<real>(lum, lumn, ecm, ecmn, la.K, la.done, la.N, la.it0, INT_MAX,
                          (size_t)blockIdx.x * blockDim.x + threadIdx.x, (size_t)gridDim.x * blockDim.x);
}

// ---- end of step: the periodic ghost ring of rho (boundary_conditions_cells,
//      useful_functions.cpp:391-420, applied to rhon at rho_functions.cpp:469)
template <typename real>
__global__ void kf_rho_ring(real *__restrict__ rho, int N) {
    const int n = blockIdx.y;
    real *p = rho + (size_t)n * N * N;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < 4 * N; k += gridDim.x * blockDim.x) {
        int i, j;
        if (k < N) { i = 0; j = k; }
        else if (k < 2 * N) { i = N - 1; j = k - N; }
        else if (k < 3 * N) { i = k - 2 * N; j = 0; }
        else { i = k - 3 * N; j = N - 1; }
        if ((k >= 2 * N) && (i == 0 || i == N - 1)) continue;
        p[(size_t)i * N + j] = p[(size_t)ghost_src(i, N) * N + ghost_src(j, N)];
    }
}

// upload: initial support rectangles and the exactness precondition
template <typename real>
__global__ void kf_outside_check(const real *__restrict__ phi, const int4 *__restrict__ rect, int N,
                                 unsigned *__restrict__ bad) {
    const int n = blockIdx.y;
    const int4 r = rect[n];
    const real *p = phi + (size_t)n * N * N;
    for (int i = blockIdx.x; i < N; i += gridDim.x)
        for (int j = threadIdx.x; j < N; j += blockDim.x) {
            if (i >= r.x && i < r.y && j >= r.z && j < r.w) continue;
            if (p[(size_t)i * N + j] > (real)0.5) atomicOr(bad, 1u);
        }
}

__global__ void kf_rect_init(int4 *rect, int Ntot, int N) {
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < Ntot) rect[n] = make_int4(N, 0, N, 0);   // empty; the first centroid sets it to the zone
}

// ---------------------------------------------------------------------------
FusedRes *F(pfag_ctx *c) { return (FusedRes *)c->fused; }

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library); null when the driver does not provide it
inline PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
        (void)cudaGetLastError();
    });
    return fn;
}
// [N][N] FP32 plane, boxes of LT_W columns x (LT_R + 2) rows, zero fill outside
inline bool encode_plane_map(CUtensorMap *m, const void *base, int N) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)N, (cuuint64_t)N};
    const cuuint64_t strides[1] = {(cuuint64_t)N * sizeof(float)};
    const cuuint32_t box[2] = {(cuuint32_t)LT_W, (cuuint32_t)(LT_R + 2)};
    const cuuint32_t es[2] = {1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void *>(base), dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

BoxArgs box_args(pfag_ctx *c) {
    BoxArgs a{};
    const DevParams &d = c->dp;
    a.N = c->N; a.z = c->zone; a.M = c->M; a.logm = F(c)->logm; a.Ntot = c->Ntot;
    a.c4 = 1.0 / d.dx / d.dx / 4.0; a.sigma = d.sigma; a.dt = d.dt; a.kfac = d.kfac; a.friction = d.friction;
    a.dx = d.dx;
    a.inv_2s2 = 1.0 / (2.0 * d.sigma * d.sigma);
    a.k_delta = 1.0 / (std::sqrt(2.0 * M_PI) * d.sigma);
    for (int k = 0; k < 3; k++) {
        a.deg[k] = d.deg[k]; a.gen[k] = d.gen[k]; a.a_ort[k] = d.a_ort[k]; a.a_tan[k] = d.a_tan[k];
        a.visc[k] = d.visc[k]; a.bb[k] = d.bb[k];
    }
    const FusedRes *r = F(c);
    const size_t plane = (size_t)c->N * c->N * (c->prec == 64 ? 8 : 4);
    a.nb_lo = r->nb_lo ? r->nb_lo : (const void *)((const char *)c->phi + (size_t)(c->Ntot - 1) * plane);
    a.nb_hi = r->nb_hi ? r->nb_hi : (const void *)c->phi;
    return a;
}

// Cooperative launch; when the runtime refuses the grid as larger than what
// can be co-resident, the grid is halved (the kernels stride over their work)
// and *blocks keeps the accepted size for later launches.
inline int launch_coop_t(const void *fn, int *blocks, int threads, void **args, size_t smem, cudaStream_t s) {
    for (;;) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(*blocks);
        cfg.blockDim = dim3(threads);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        const cudaError_t e = cudaLaunchKernelExC(&cfg, fn, args);
        if (e == cudaSuccess) return PFAG_OK;
        if (e == cudaErrorCooperativeLaunchTooLarge && *blocks > 1) {
            (void)cudaGetLastError();
            *blocks /= 2;
            continue;
        }
        cudaFuncAttributes fa{};
        cudaFuncGetAttributes(&fa, fn);
        pfag_set_error("cooperative launch of %d x %d threads (%d registers/thread, %zu B static smem): %s", *blocks,
                       threads, fa.numRegs, fa.sharedSizeBytes, cudaGetErrorString(e));
        return PFAG_E_CUDA;
    }
}


template <typename real>
struct Fused {
    typedef typename Cplx<real>::type cx;
    pfag_ctx *c;
    FusedRes *r;
    explicit Fused(pfag_ctx *ctx) : c(ctx), r(F(ctx)) {}
    real *R(void *p) { return (real *)p; }

    int configure() {
        const int M = c->M;
        int logm = 0;
        while ((1 << logm) < M) logm++;
        // power-of-two boxes from 16 to 1024: the hand-written FFT passes; any
        // other box up to 512: the Bluestein passes (kg_*, kbl_*)
        r->generic = (1 << logm) != M || M < 16 || M > 1024;
        if (M < 2) { pfag_set_error("zone_size %d gives no FFT box", c->zone); return PFAG_E_UNSUPPORTED; }
        if (r->generic) {
            if (M > 512 || (M & 1)) {
                pfag_set_error("fused path: FFT box %d (zone_size %d) is neither a power of two in 16..1024 nor an "
                               "even size up to 512; the plain path supports it", M, c->zone);
                return PFAG_E_UNSUPPORTED;
            }
            int L = 32;
            while (L < 2 * M - 1) L <<= 1;
            r->blue_L = L;
        }
        if (c->Ntot > 1024) { pfag_set_error("fused path supports at most 1024 cells"); return PFAG_E_UNSUPPORTED; }
        r->logm = logm;
        const size_t cs = sizeof(cx);
        if (!r->generic) {
        // rows per block for the row passes: keep the shared tile near 64 KB
        int R = std::max(1, std::min(8, (int)(65536 / (2 * (size_t)M * cs))));
        R = std::min(R, std::max(1, 8 * FT / M));   // pass C keeps <= 8 elements per thread in registers
        while (M % R) R--;
        r->rows_blk = R;
        int G = std::max(1, std::min(16, (int)(98304 / (4 * (size_t)(M + 1) * cs))));
        r->grp_cols = G;
        r->smemA = (M + 2 * (size_t)R * M) * cs;
        r->smemC = (M + (size_t)R * M) * cs;
        r->smemE = r->smemC;
        r->smemB = (M + 2 * 2 * (size_t)G * (M + 1)) * cs;
        r->smemD = (M + 2 * (size_t)G * (M + 1)) * cs;
        PFAG_TRY(smem_at_least((const void *)kf_boxA<real>, r->smemA));
        PFAG_TRY(smem_at_least((const void *)kf_boxB<real>, r->smemB));
        PFAG_TRY(smem_at_least((const void *)kf_boxC<real>, r->smemC));
        PFAG_TRY(smem_at_least((const void *)kf_boxD<real>, r->smemD));
        PFAG_TRY(smem_at_least((const void *)kf_boxE<real>, r->smemE));
        }
        int dev = 0, nsm = 0, per = 0;
        PFAG_CUDA_CHECK(cudaGetDevice(&dev));
        PFAG_CUDA_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        // one thread per zone column up to RESH_MAX_THREADS (wider zones: a thread takes several)
        r->resh_threads = std::min(32 * ((2 * c->zone + 31) / 32), RESH_MAX_THREADS);
        r->resh_tile = (size_t)3 * (RESH_RB + 2) * (2 * c->zone + 2) * sizeof(real);
        r->resh_smem = (size_t)(r->resh_threads / 32) * c->Ntot * sizeof(double) + r->resh_tile;
        if (r->resh_smem > 200 * 1024) { pfag_set_error("too many cells for the reshaping kernel's per-warp sums"); return PFAG_E_UNSUPPORTED; }
        PFAG_TRY(smem_at_least((const void *)kf_relax_loops<real, RESH_RB>, r->resh_smem));
        PFAG_TRY(smem_at_least((const void *)kf_resh_first<real, RESH_RB>, r->resh_tile));
        PFAG_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kf_relax_loops<real, RESH_RB>,
                                                                       r->resh_threads, r->resh_smem));
        if (per < 1) { pfag_set_error("relaxation kernel cannot be resident with %d threads", r->resh_threads); return PFAG_E_UNSUPPORTED; }
        r->coop_r = nsm * std::min(per, 8);
        r->tpc = (2 * c->zone + RESH_RB - 1) / RESH_RB;
        {
            // no more blocks than the loops have tasks (reshaping strips, lumen / ECM
            // tiles): a small organoid's persistent kernel leaves the rest of the
            // GPU to other contexts (sweep members)
            const long strips = (long)c->Ntot * r->tpc;
            const long tiles = (long)((c->N + LUM_LRI - 1) / LUM_LRI) * ((c->N + r->resh_threads - 1) / r->resh_threads);
            r->coop_r = (int)std::max(1L, std::min((long)r->coop_r, std::max(strips, tiles)));
        }
        r->ntl = ((c->N + LRB - 1) / LRB) * ((c->N + FT - 1) / FT);
        r->lum_tile = (size_t)3 * (LRB + 2) * (FT + 2) * sizeof(real);
        PFAG_TRY(smem_at_least((const void *)kl_relax<real>, r->lum_tile));
        r->ltiles = 0;                 // TMA-staged lumen iterations: set up in alloc, once Jl exists
        r->npsi = ((c->N + 31) / 32) * ((c->N + PT_R - 1) / PT_R);
        r->upd_warps = 0;
        r->upd_smem = (size_t)UPD_SLOTS * 5 * UPD_THREADS * sizeof(float);
        if constexpr (sizeof(real) == 4) {
            PFAG_TRY(smem_at_least((const void *)kf_update_rows<real>, r->upd_smem));
            PFAG_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kf_update_rows<real>, UPD_THREADS,
                                                                           r->upd_smem));
            r->upd_warps = (long)nsm * std::max(per, 1) * (UPD_THREADS / 32);
        }
        r->coop_default = r->coop_r;
        r->upd_default = r->upd_warps;
        return PFAG_OK;
    }

    int alloc() {
        PFAG_TRY(configure());
        const size_t mm = (size_t)c->M * c->M, rs = c->rsz, W = 2 * c->zone + 2;
        PFAG_CUDA_CHECK(cudaMalloc(&r->Y1, (size_t)c->Ntot * mm * 2 * rs));
        PFAG_CUDA_CHECK(cudaMalloc(&r->Y2, (size_t)c->Ntot * mm * 2 * rs));
        PFAG_CUDA_CHECK(cudaMalloc(&r->Rb, (size_t)c->Ntot * mm * rs));
        PFAG_CUDA_CHECK(cudaMalloc(&r->clsT, (size_t)c->Ntot * mm));
        if (r->generic) {
            const int M = c->M, L = r->blue_L;
            PFAG_CUDA_CHECK(cudaMalloc(&r->Gsp, (size_t)c->Ntot * M * (M / 2 + 1) * 2 * rs));
            PFAG_CUDA_CHECK(cudaMalloc(&r->btw, (size_t)L * 2 * rs));
            PFAG_CUDA_CHECK(cudaMalloc(&r->bcw, (size_t)M * 2 * rs));
            PFAG_CUDA_CHECK(cudaMalloc(&r->bwf, (size_t)L * 2 * rs));
            PFAG_CUDA_CHECK(cudaMalloc(&r->bhdi, (size_t)L * rs));
            PFAG_CUDA_CHECK(cudaMalloc(&r->bh, (size_t)M * sizeof(double)));
            const double dtk = c->dp.dt * c->dp.kfac;
            kbl_tables1<cx><<<(std::max(L, M) + 127) / 128, 128, 0, c->stream>>>(M, L, dtk, (cx *)r->btw,
                                                                                  (cx *)r->bcw, r->bh);
            PFAG_CUDA_CHECK(cudaGetLastError());
            kbl_tables2<cx><<<(L + 127) / 128, 128, 0, c->stream>>>(M, L, r->bh, (cx *)r->bwf, R(r->bhdi));
            PFAG_CUDA_CHECK(cudaGetLastError());
            PFAG_CUDA_CHECK(cudaStreamSynchronize(c->stream));
        }
        PFAG_CUDA_CHECK(cudaMalloc(&r->Jc, (size_t)c->Ntot * 2 * W * W * rs));
        PFAG_CUDA_CHECK(cudaMalloc(&r->Jl, 4 * c->ng * rs));
        if (sizeof(real) == 4) PFAG_CUDA_CHECK(cudaMalloc(&r->G, c->ng * rs));
        PFAG_CUDA_CHECK(cudaMalloc(&r->rect, sizeof(int4) * c->Ntot));
        {
            const size_t t = (size_t)((c->N + 31) / 32) * ((c->N + PT_R - 1) / PT_R);
            PFAG_CUDA_CHECK(cudaMalloc(&r->part_a, sizeof(double) * c->Ntot * t));
        }
        PFAG_CUDA_CHECK(cudaMalloc(&r->part_r, sizeof(double) * (size_t)c->Ntot * std::max(r->tpc, r->coop_r)));
        PFAG_CUDA_CHECK(cudaMalloc(&r->part_e, sizeof(double) * r->npsi));
        PFAG_CUDA_CHECK(cudaMalloc(&r->part_l, sizeof(double) * 2 * r->coop_r));
        if (sizeof(real) == 4 && c->N % 4 == 0 && c->N >= LT_W) {
            // TMA-staged lumen / ECM iterations: the maps hold the addresses of
            // this context's lum, lumn, ECM, ECMn and of the normals Jl, so
            // they are encoded after every one of them is allocated
            LumMaps mp;
            std::memset(&mp, 0, sizeof(mp));
            const size_t plane = (size_t)c->N * c->N * sizeof(float);
            void *pf[4] = {c->lum, c->lumn, c->ecm, c->ecmn};
            bool ok = r->Jl != nullptr;
            for (void *q : pf) ok = ok && q != nullptr;
            for (int k = 0; k < 4 && ok; k++) ok = encode_plane_map(&mp.P[k], pf[k], c->N);
            for (int k = 0; k < 4 && ok; k++) ok = encode_plane_map(&mp.J[k], (const char *)r->Jl + k * plane, c->N);
            if (ok) {
                r->lmaps = new LumMaps(mp);
                r->ltiles = ((c->N + LT_R - 1) / LT_R) * ((c->N + LT_C - 1) / LT_C);
                r->lt_smem = (size_t)LT_STAGES * 3 * LT_BOX * sizeof(float) + LT_STAGES * sizeof(long long) + 128;
                PFAG_TRY(smem_at_least((const void *)kl_relax_tma, r->lt_smem));
                int per = 0;
                PFAG_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kl_relax_tma, LT_THREADS,
                                                                               r->lt_smem));
                int dev = 0, nsm = 0;
                PFAG_CUDA_CHECK(cudaGetDevice(&dev));
                PFAG_CUDA_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
                r->lt_blocks = (int)std::min<long>(2L * r->ltiles, (long)nsm * std::max(1, per));
            }
        }
        PFAG_CUDA_CHECK(cudaMalloc(&r->part_lt, sizeof(double) * 2 * std::max(r->ntl, r->ltiles)));
        PFAG_CUDA_CHECK(cudaStreamCreateWithFlags(&r->side, cudaStreamNonBlocking));
        PFAG_CUDA_CHECK(cudaEventCreateWithFlags(&r->ev_psi, cudaEventDisableTiming));
        PFAG_CUDA_CHECK(cudaEventCreateWithFlags(&r->ev_boxA, cudaEventDisableTiming));
        PFAG_CUDA_CHECK(cudaEventCreateWithFlags(&r->ev_area, cudaEventDisableTiming));
        PFAG_CUDA_CHECK(cudaEventCreateWithFlags(&r->ev_lum, cudaEventDisableTiming));
        PFAG_CUDA_CHECK(cudaMalloc(&r->cK, sizeof(int) * (3 * c->Ntot + 8)));
        r->cdone = r->cK + c->Ntot;
        r->ccnt = r->cK + 2 * c->Ntot;
        r->lK = r->cK + 3 * c->Ntot;
        r->ldone = r->lK + 2;
        r->lcnt = r->lK + 4;
        PFAG_CUDA_CHECK(cudaMemset(r->cK, 0, sizeof(int) * (3 * c->Ntot + 8)));
        return PFAG_OK;
    }

    int upload_hook() {
        // full-grid centroid of the initial state, first support rectangle = first zone
        kf_rect_init<<<(c->Ntot + 127) / 128, 128, 0, c->stream>>>(r->rect, c->Ntot, c->N);
        PFAG_CUDA_CHECK(cudaMemsetAsync(c->d_cacc, 0, sizeof(long long) * 3 * c->Ntot, c->stream));
        int4 full = make_int4(0, c->N, 0, c->N);
        std::vector<int4> hf(c->Ntot, full);
        int4 *tmp = nullptr;
        PFAG_CUDA_CHECK(cudaMalloc(&tmp, sizeof(int4) * c->Ntot));
        PFAG_CUDA_CHECK(cudaMemcpyAsync(tmp, hf.data(), sizeof(int4) * c->Ntot, cudaMemcpyHostToDevice, c->stream));
        kf_centroid<real><<<dim3(64, c->Ntot), FT, 0, c->stream>>>(R(c->phi), tmp, c->N, c->d_cacc);
        kf_centroid_finalize<<<(c->Ntot + 127) / 128, 128, 0, c->stream>>>(c->d_cacc, c->Ntot, c->N, c->zone, c->d_xc,
                                                                           c->d_yc, r->rect, c->d_err);
        PFAG_CUDA_CHECK(cudaMemsetAsync(c->d_err + 1, 0, sizeof(unsigned), c->stream));
        kf_outside_check<real><<<dim3(64, c->Ntot), FT, 0, c->stream>>>(R(c->phi), r->rect, c->N, c->d_err + 1);
        PFAG_CUDA_CHECK(cudaMemcpyAsync(c->h_err, c->d_err, 2 * sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
        PFAG_CUDA_CHECK(cudaStreamSynchronize(c->stream));
        cudaFree(tmp);
        PFAG_CUDA_CHECK(cudaGetLastError());
        if (c->h_err[1]) {
            pfag_set_error("fused path precondition: a cell has phi > 0.5 outside its first zone; use the plain path");
            return PFAG_E_UNSUPPORTED;
        }
        if (c->h_err[0]) {
            PFAG_CUDA_CHECK(cudaMemsetAsync(c->d_err, 0, sizeof(unsigned), c->stream));
            pfag_set_error("initial zone leaves the grid or a cell is empty");
            return (c->h_err[0] & ERRBIT_EMPTY_CELL) ? PFAG_E_EMPTY_CELL : PFAG_E_ZONE;
        }
        r->ring_pending = true;
        return PFAG_OK;
    }

    // the phi update + normals on zone + ring (reads the old rho, like the
    // spectral solve, which therefore updates rho in place afterwards); runs
    // after pass A, once the side stream has turned the area partials into f0
    int launch_update() {
        cudaStream_t s = c->stream;
        if (r->fork) PFAG_CUDA_CHECK(cudaStreamWaitEvent(s, r->ev_area, 0));
        const int z = c->zone, W = 2 * z + 2;
        pfag_prof_begin(c, sizeof(real) == 4 ? "kf_update_rows" : "kf_update_tiled");
        if constexpr (sizeof(real) == 4) {
            // row chunks: as many warp tasks as fit on the GPU at once (one wave), with at
            // least 16 rows per task (a task loads 8 rows beyond the ones it updates)
            const int cg = (W + UPD_COLS - 1) / UPD_COLS;
            const long per_chunk = (long)c->Ntot * cg;
            const int nch = (int)std::max(1L, std::min((long)(W + 15) / 16, r->upd_warps / per_chunk));
            const int rb = (W + nch - 1) / nch;
            const long tasks = per_chunk * ((W + rb - 1) / rb);
            kf_update_rows<real><<<(unsigned)((tasks + 7) / 8), UPD_THREADS, r->upd_smem, s>>>(
                R(c->phi), R(c->phin), R(c->rho), R(c->hfunc), c->d_f0, R(c->psi), R(r->G), c->d_xc, c->d_yc, c->dp,
                R(r->Jc), cg, (W + rb - 1) / rb, rb);
        } else {
            dim3 gb((W + UC - 1) / UC, (W + UR - 1) / UR, c->Ntot);
            kf_update_tiled<real><<<gb, 256, 0, s>>>(R(c->phi), R(c->phin), R(c->rho), R(c->hfunc), c->d_f0,
                                                     R(c->psi), R(c->hlum), R(c->hecm), c->d_xc, c->d_yc, c->dp,
                                                     R(r->Jc), R(r->G));
        }
        PFAG_LAUNCHED(c);
        return PFAG_OK;
    }

    // enqueue one step (no host synchronisation; capturable).  part 0: the
    // whole step; 1: its head (centroids, h, this context's psi); 2: the rest,
    // once the host has completed psi over every shard of the organoid
    int enqueue(int part = 0) {
        cudaStream_t s = c->stream;
        const int N = c->N, Nt = c->Ntot, M = c->M, z = c->zone;
        const DevParams &d = c->dp;
        // 1-2. centroids (from the sums the previous step's persistent kernel,
        //    or the upload, left over B_n), hfunc on the zones, psi, area
        //    partials, h(lum), h(ECM), sum_ecm partials
        const int tiles = (N + 31) / 32, tiles_r = (N + PT_R - 1) / PT_R;
        if (part != 2) {
            pfag_prof_begin(c, "kf_hpsi");
            kf_hpsi<real><<<dim3(tiles, tiles_r), FT, 0, s>>>(R(c->phi), R(c->hfunc), r->rect, c->d_cacc, c->d_xc,
                                                               c->d_yc, c->d_err, Nt, N, z, R(c->lum), R(c->ecm),
                                                               R(c->psi), R(c->hlum), R(c->hecm), d.dx * d.dx,
                                                               r->part_e, r->part_a);
            PFAG_LAUNCHED(c);
            if (part == 1) {
                PFAG_CUDA_CHECK(cudaGetLastError());
                return PFAG_OK;
            }
        }
        // 3. areas and f0, then the lumen / ECM update and normals
        //    (cell_phase_functions.cpp:372-444, :722-771), which need only psi,
        //    h(lum) and h(ECM): on the side stream beside pass A, the phi
        //    update and the rest of the spectral solve.  The relaxation (6)
        //    rewrites lum and ECM, so it waits for pass A, which reads them.  No
        //    cooperative kernel runs beside the side stream: the main stream
        //    joins it before the persistent kernel.
        const bool fork = !pfag_prof_on(c);
        cudaStream_t s2 = fork ? r->side : s;
        r->fork = fork;
        if (fork) {
            PFAG_CUDA_CHECK(cudaEventRecord(r->ev_psi, s));
            PFAG_CUDA_CHECK(cudaStreamWaitEvent(s2, r->ev_psi, 0));
        }
        if (sizeof(real) == 4) {
            pfag_prof_begin(c, "kf_gel_coupling");
            kf_gel_coupling<real><<<dim3((N + 31) / 32, (N + 7) / 8), dim3(32, 8), 0, s2>>>(R(c->hlum), R(c->hecm),
                                                                                        R(r->G), c->dp);
            PFAG_LAUNCHED(c);
        }
        pfag_prof_begin(c, "kf_area_tiles");
        kf_area_tiles<<<Nt, 32, 0, s2>>>(r->part_a, r->rect, tiles, tiles * tiles_r, d.alpha, d.s0, c->d_s, c->d_f0);
        PFAG_LAUNCHED(c);
        if (fork) PFAG_CUDA_CHECK(cudaEventRecord(r->ev_area, s2));
        LumArgs la{};
        la.N = N; la.rimax = c->p.rimax; la.cap = c->relax_cap; la.npsi = r->npsi;
        la.dx = d.dx; la.dt = d.dt; la.tau_lum = d.tau_lum; la.xi_lum = d.xi_lum;
        la.beta_lum_cells = d.beta_lum_cells; la.eta_lum_cells = d.eta_lum_cells; la.beta_lum_ECM = d.beta_lum_ECM;
        la.alpha_ECM = d.alpha_ECM; la.tau_ECM = d.tau_ECM; la.xi_ECM = d.xi_ECM;
        la.beta_ECM_cells = d.beta_ECM_cells; la.eta_ECM_cells = d.eta_ECM_cells;
        la.A = d.A_resh; la.B = d.B_resh; la.thr = d.thr_lum; la.rdev0 = d.rdev0_lum;
        la.part_e = r->part_e; la.part = r->part_l; la.K = r->lK; la.done = r->ldone; la.cnt = r->lcnt;
        la.err = c->d_err;
        la.no_copies = (c->debug & 2) ? 1 : 0;               // pfag_set_debug bit 2: the TMA waits run out
        la.wait_cap = (c->debug & 2) ? (1 << 10) : (1 << 20);
        {
            pfag_prof_begin(c, "kfl_sum_ecm");
            kfl_sum_ecm<<<1, 32, 0, s2>>>(r->part_e, r->npsi, c->d_scal + 0);
            PFAG_LAUNCHED(c);
            const dim3 tb(32, 8), gb((N + 31) / 32, (N + 7) / 8);
            pfag_prof_begin(c, "kfl_update");
            kfl_update<real><<<gb, tb, 0, s2>>>(R(c->lum), R(c->ecm), R(c->lumn), R(c->ecmn), R(c->psi), R(c->hlum),
                                                R(c->hecm), c->d_scal + 0, la);
            PFAG_LAUNCHED(c);
            pfag_prof_begin(c, "kfl_normals");
            kfl_normals<real><<<gb, tb, 0, s2>>>(R(c->lum), R(c->lumn), R(c->ecm), R(c->ecmn), R(r->Jl), N, d.dx);
            PFAG_LAUNCHED(c);
        }
        // 4-5. spectral solve with the phi update after its pass A; the last
        //    column pass writes the new rho over each box in place
        //    (rho <- rhon of run_with_active_gels.cpp:175-178 on the box)
        const BoxArgs ba = box_args(c);
        const int Rr = r->rows_blk, G = r->grp_cols;
        cx *Y1 = (cx *)r->Y1, *Y2 = (cx *)r->Y2;
        if (r->generic) { PFAG_TRY(box_generic(ba)); }
        else if (M == 256) { PFAG_TRY(box_reg<256>(ba)); }
        else if (M == 128) { PFAG_TRY(box_reg<128>(ba)); }
        else if (M == 64) { PFAG_TRY(box_reg<64>(ba)); }
        else if (M == 32) { PFAG_TRY(box_reg<32>(ba)); }
        else {
        pfag_prof_begin(c, "kf_boxA");
        kf_boxA<real><<<dim3(M / Rr, Nt), FT, r->smemA, s>>>(R(c->phi), R(c->rho), R(c->lum), R(c->ecm), c->d_xc,
                                                             c->d_yc, ba, Rr, Y1, Y2, R(r->Rb), r->clsT);
        PFAG_LAUNCHED(c);
        if (r->fork) PFAG_CUDA_CHECK(cudaEventRecord(r->ev_boxA, s));
        PFAG_TRY(launch_update());
        const int ngrp = (M / 2 + 1 + G - 1) / G;
        pfag_prof_begin(c, "kf_boxB");
        kf_boxB<real><<<dim3(ngrp, Nt), FT, r->smemB, s>>>(Y1, Y2, r->clsT, ba, G); PFAG_LAUNCHED(c);
        pfag_prof_begin(c, "kf_boxC");
        kf_boxC<real><<<dim3(M / Rr, Nt), FT, r->smemC, s>>>(Y1, Y2, R(c->rho), c->d_xc, c->d_yc, ba, Rr,
                                                             c->debug ? R(c->d_vx) : nullptr,
                                                             c->debug ? R(c->d_vy) : nullptr);
        PFAG_LAUNCHED(c);
        pfag_prof_begin(c, "kf_boxD");
        kf_boxD<real><<<dim3(ngrp, Nt), FT, r->smemD, s>>>(Y1, Y2, ba, G); PFAG_LAUNCHED(c);
        pfag_prof_begin(c, "kf_boxE");
        kf_boxE<real><<<dim3(M / Rr, Nt), FT, r->smemE, s>>>(Y1, R(c->rho), R(r->Rb), R(c->rho), c->d_xc, c->d_yc,
                                                             ba, Rr);
        PFAG_LAUNCHED(c);
        }
        // 6. lumen / ECM relaxation: iterations 1 .. LUM_REGULAR as
        //    full-occupancy kernels on the side stream once pass A has read lum
        //    and ECM, and lum <- lumn, ECM <- ECMn for the fields that stopped
        //    there; the rest (if a field still moves) in the persistent kernel
        //    after the join below
        if (fork) PFAG_CUDA_CHECK(cudaStreamWaitEvent(s2, r->ev_boxA, 0));
        for (int it = 1; it <= LUM_REGULAR; it++) {
            if constexpr (sizeof(real) == 4) {
                if (r->lmaps && r->lum_tma) {
                    pfag_prof_begin(c, "kl_relax_tma");
                    kl_relax_tma<<<r->lt_blocks, LT_THREADS, r->lt_smem, s2>>>(
                        *r->lmaps, R(c->lum), R(c->lumn), R(c->ecm), R(c->ecmn), la, it, r->part_lt);
                    PFAG_LAUNCHED(c);
                    pfag_prof_begin(c, "kl_decide");
                    kl_decide<<<2, 32, 0, s2>>>(la, it, r->part_lt, r->ltiles);
                    PFAG_LAUNCHED(c);
                    continue;
                }
            }
            pfag_prof_begin(c, "kl_relax");
            kl_relax<real><<<dim3(r->ntl, 2), FT, r->lum_tile, s2>>>(R(c->lum), R(c->lumn), R(c->ecm), R(c->ecmn),
                                                                      R(r->Jl), la, it, r->part_lt);
            PFAG_LAUNCHED(c);
            pfag_prof_begin(c, "kl_decide");
            kl_decide<<<2, 32, 0, s2>>>(la, it, r->part_lt, r->ntl);
            PFAG_LAUNCHED(c);
        }
        pfag_prof_begin(c, "kl_copy");
        kl_copy<real><<<296, FT, 0, s2>>>(R(c->lum), R(c->lumn), R(c->ecm), R(c->ecmn), r->lK, r->ldone, N,
                                          LUM_REGULAR);
        PFAG_LAUNCHED(c);
        if (fork) PFAG_CUDA_CHECK(cudaEventRecord(r->ev_lum, s2));
        // 7. reshaping of the cells: iteration 1 at full occupancy, then the
        //    persistent kernel (its decision, iterations 2.., and the lumen /
        //    ECM iterations beyond LUM_REGULAR)
        {
            ReshArgs ra{};
            ra.N = N; ra.z = z; ra.Ntot = Nt; ra.tpc = r->tpc;
            ra.rimax = c->p.rimax; ra.cap = c->relax_cap;
            ra.A = d.A_resh; ra.B = d.B_resh; ra.scale = d.dx * d.dx / (double)d.Ncur; ra.thr = d.thr_cells;
            ra.K = r->cK; ra.done = r->cdone; ra.cnt = r->ccnt; ra.part = r->part_r; ra.err = c->d_err;
            ra.it0 = 2;
            la.it0 = LUM_REGULAR + 1;
            real *T = R(c->rhon);          // the fused path keeps rho in place: rhon is the reshaping scratch
            const dim3 gs(r->tpc, Nt);
            pfag_prof_begin(c, "kf_resh_first");
            kf_resh_first<real, RESH_RB><<<gs, r->resh_threads, r->resh_tile, s>>>(R(c->phin), T, R(c->phi), R(r->Jc),
                                                                                    c->d_xc, c->d_yc, ra);
            PFAG_LAUNCHED(c);
            real *a0 = R(c->phi), *a1 = R(c->phin), *a2 = T;
            const real *a3 = R(r->Jc);
            const int *a4 = c->d_xc, *a5 = c->d_yc;
            real *b0 = R(c->lum), *b1 = R(c->lumn), *b2 = R(c->ecm), *b3 = R(c->ecmn);
            const real *b4 = R(r->Jl);
            const int4 *c0 = r->rect;
            long long *c1 = c->d_cacc;
            void *args[] = {&a0, &a1, &a2, (void *)&a3, (void *)&a4, (void *)&a5, &ra,
                            &b0, &b1, &b2, &b3, (void *)&b4, &la, (void *)&c0, &c1};
            if (fork) PFAG_CUDA_CHECK(cudaStreamWaitEvent(s, r->ev_lum, 0));   // join the side stream
            pfag_prof_begin(c, "kf_relax_loops");
            PFAG_TRY(launch_coop_t((const void *)kf_relax_loops<real, RESH_RB>, &r->coop_r, r->resh_threads, args,
                                   r->resh_smem, s));
            PFAG_LAUNCHED(c);
        }
        // 8. periodic ghost ring of rho (boundary_conditions_cells(rhon),
        //    rho_functions.cpp:469).  Its sources, rows and columns 1 and N-2,
        //    lie outside every box (boxes span [xc-z+1, xc+z-2] with
        //    xc-z >= 1), so once the ring matches them it stays matched: it is
        //    applied in the first step after an upload only.
        if (r->ring_pending) {
            pfag_prof_begin(c, "kf_rho_ring");
            kf_rho_ring<real><<<dim3((4 * N + 255) / 256, Nt), 256, 0, s>>>(R(c->rho), N); PFAG_LAUNCHED(c);
        }
        PFAG_CUDA_CHECK(cudaGetLastError());
        return PFAG_OK;
    }

    // zone rows per reshaping strip
    static constexpr int RESH_RB = 8;
    // lumen/ECM relaxation iterations run as regular kernels before the persistent one
    static constexpr int LUM_REGULAR = 2;

    // primaries per block of the column passes (shared tile near 64 KB)
    static constexpr int GB = 4;

    BlueTabs<cx> blue_tabs() {
        BlueTabs<cx> tb;
        tb.tw = (const cx *)r->btw; tb.cw = (const cx *)r->bcw; tb.wf = (const cx *)r->bwf;
        tb.hdi = (const real *)r->bhdi;
        return tb;
    }

    // spectral solve on boxes of any even size up to 512 with Bluestein
    // transforms of inner length L: stresses; forward row transforms (pi_xx +
    // i pi_yy in place, pi_xy's rows in pairs to half spectra); forward column
    // transforms; the k-space velocity; inverse column transforms; inverse
    // row transforms with the fluxes and the row derivative; the column
    // derivative and the new rho on the box.  The phi update runs after the
    // stress kernel, which has read rho, lum and ECM.
    template <int L>
    int box_blue(const BoxArgs &ba) {
        typedef BlueGeom<real, L> BGm;
        cudaStream_t s = c->stream;
        const int M = c->M, Nt = c->Ntot, N = c->N, z = c->zone, H = M / 2 + 1;
        cx *Y1 = (cx *)r->Y1, *Y2 = (cx *)r->Y2, *Hs = (cx *)r->Gsp;
        const BlueTabs<cx> tb = blue_tabs();
        const size_t cs = sizeof(cx);
        const size_t tab_c = tabs_bytes<cx, L>(M, true, false), tab_d = tabs_bytes<cx, L>(M, false, true);
        const size_t sm_rows = (size_t)(1 + BGm::GPB) * L * cs + tab_c;
        const size_t sm_rowsD1 = (size_t)(1 + BGm::GPB) * L * cs + tab_c;
        const size_t sm_rowsD2 = (size_t)(1 + BGm::GPB) * L * cs + tab_d;
        const size_t sm_cols = ((size_t)L + (size_t)BGm::GPB * (L + 1)) * cs + tab_c;
        const size_t sm_colsE = ((size_t)L + (size_t)BGm::GPB * (L + 1)) * cs + tab_d;
        PFAG_TRY(smem_at_least((const void *)kbl_rowsA<real, L>, sm_rows));
        PFAG_TRY(smem_at_least((const void *)kbl_rowsD1<real, L>, sm_rowsD1));
        PFAG_TRY(smem_at_least((const void *)kbl_rowsD2<real, L>, sm_rowsD2));
        PFAG_TRY(smem_at_least((const void *)kbl_cols<real, L, false>, sm_cols));
        PFAG_TRY(smem_at_least((const void *)kbl_cols<real, L, true>, sm_cols));
        PFAG_TRY(smem_at_least((const void *)kbl_colsE<real, L>, sm_colsE));
        const dim3 g((M * M + 255) / 256, Nt);
        pfag_prof_begin(c, "kg_stress");
        kg_stress<real><<<g, 256, 0, s>>>(R(c->phi), R(c->rho), R(c->lum), R(c->ecm), c->d_xc, c->d_yc, ba, Y1, Y2,
                                          R(r->Rb), r->clsT);
        PFAG_LAUNCHED(c);
        if (r->fork) PFAG_CUDA_CHECK(cudaEventRecord(r->ev_boxA, s));
        PFAG_TRY(launch_update());
        {
            const long tasks = (long)Nt * (M + M / 2);
            pfag_prof_begin(c, "kbl_rowsA");
            kbl_rowsA<real, L><<<(unsigned)((tasks + BGm::GPB - 1) / BGm::GPB), BGm::THREADS, sm_rows, s>>>(
                Y1, (const real *)Y2, Hs, M, Nt, tb);
            PFAG_LAUNCHED(c);
        }
        ColSet<cx> y1s{Y1, (long)M * M, M, M, (M + BGm::GPB - 1) / BGm::GPB};
        ColSet<cx> hss{Hs, (long)M * H, H, H, (H + BGm::GPB - 1) / BGm::GPB};
        ColSet<cx> none{Y1, 0, M, 0, 0};
        pfag_prof_begin(c, "kbl_colsB");
        kbl_cols<real, L, false><<<(unsigned)((long)Nt * (y1s.nblk + hss.nblk)), BGm::THREADS, sm_cols, s>>>(
            y1s, hss, M, Nt, tb);
        PFAG_LAUNCHED(c);
        pfag_prof_begin(c, "kg_velocity");
        kg_velocity<real><<<g, 256, 0, s>>>(Y1, (const cx *)Hs, r->clsT, ba);
        PFAG_LAUNCHED(c);
        pfag_prof_begin(c, "kbl_colsC");
        kbl_cols<real, L, true><<<(unsigned)((long)Nt * y1s.nblk), BGm::THREADS, sm_cols, s>>>(y1s, none, M, Nt,
                                                                                                tb);
        PFAG_LAUNCHED(c);
        real *X = (real *)r->Y2;              // free once the row pass has read pi_xy: Fx, then the row term
        {
            const long tasks = (long)Nt * M;
            pfag_prof_begin(c, "kbl_rowsD1");
            kbl_rowsD1<real, L><<<(unsigned)((tasks + BGm::GPB - 1) / BGm::GPB), BGm::THREADS, sm_rowsD1, s>>>(
                Y1, X, R(c->rho), c->d_xc, c->d_yc, N, z, M, Nt, tb, c->debug ? R(c->d_vx) : nullptr,
                c->debug ? R(c->d_vy) : nullptr);
            PFAG_LAUNCHED(c);
            const long pairs = (long)Nt * (M / 2);
            pfag_prof_begin(c, "kbl_rowsD2");
            kbl_rowsD2<real, L><<<(unsigned)((pairs + BGm::GPB - 1) / BGm::GPB), BGm::THREADS, sm_rowsD2, s>>>(
                X, R(r->Rb), c->dp.dt, M, Nt, tb);
            PFAG_LAUNCHED(c);
        }
        {
            const long tasks = (long)Nt * ((M / 2 + BGm::GPB - 1) / BGm::GPB);
            pfag_prof_begin(c, "kbl_colsE");
            kbl_colsE<real, L><<<(unsigned)tasks, BGm::THREADS, sm_colsE, s>>>(X, M, Nt, tb);
            PFAG_LAUNCHED(c);
        }
        pfag_prof_begin(c, "kbl_rho");
        kbl_rho<real><<<g, 256, 0, s>>>(X, R(c->rho), c->d_xc, c->d_yc, N, z, M, Nt);
        PFAG_LAUNCHED(c);
        return PFAG_OK;
    }

    int box_generic(const BoxArgs &ba) {
        switch (r->blue_L) {
        case 32: return box_blue<32>(ba);
        case 64: return box_blue<64>(ba);
        case 128: return box_blue<128>(ba);
        case 256: return box_blue<256>(ba);
        case 512: return box_blue<512>(ba);
        case 1024: return box_blue<1024>(ba);
        default:
            pfag_set_error("no Bluestein pass for inner length %d", r->blue_L);
            return PFAG_E_UNSUPPORTED;
        }
    }

    template <int MM>
    int box_reg(const BoxArgs &ba) {
        typedef BoxGeom<MM> BG;
        cudaStream_t s = c->stream;
        const int Nt = c->Ntot;
        const size_t cs = sizeof(cx);
        const size_t smA = (MM + (size_t)BG::ROWS * MM) * cs + (size_t)BG::ROWS * MM * sizeof(real) +
                           (size_t)BG::ROWS * (MM + 4);
        const size_t smC = (MM + (size_t)BG::ROWS * MM) * cs;
        const int nsB = 2 * GB;
        const int nz2 = ((GB + BG::WG - 1) / BG::WG) * BG::WG;
        const size_t smB = (MM + (size_t)(nsB + nz2) * (MM + 1)) * cs + (size_t)nsB * MM;   // + class map columns
        PFAG_TRY(smem_at_least((const void *)kr_boxA<real, MM>, smA));
        PFAG_TRY(smem_at_least((const void *)kr_boxB<real, MM, GB, 256>, smB));
        typedef BoxGeomD2<MM> BD;
        constexpr int NSP2 = (BD::NSQ % BG::WG == 0) ? BD::NSQ : ((BD::NSQ + BG::WG - 1) / BG::WG) * BG::WG;
        const size_t smD2 = (MM + (size_t)NSP2 * (MM + 1)) * cs;
        PFAG_TRY(smem_at_least((const void *)kr_boxC2<real, MM>, smC));
        PFAG_TRY(smem_at_least((const void *)kr_boxD2<real, MM>, smD2));
        cx *Y1 = (cx *)r->Y1, *Y2 = (cx *)r->Y2;
        const dim3 grow(MM / BG::ROWS, Nt);
        pfag_prof_begin(c, "kr_boxA");
        kr_boxA<real, MM><<<grow, BG::THREADS, smA, s>>>(R(c->phi), R(c->rho), R(c->lum), R(c->ecm), c->d_xc, c->d_yc,
                                                          ba, Y1, Y2, R(r->Rb), r->clsT);
        PFAG_LAUNCHED(c);
        if (r->fork) PFAG_CUDA_CHECK(cudaEventRecord(r->ev_boxA, s));
        PFAG_TRY(launch_update());
        pfag_prof_begin(c, "kr_boxB");
        kr_boxB<real, MM, GB, 256><<<dim3((MM / 2 + 1 + GB - 1) / GB, Nt), 256, smB, s>>>(Y1, Y2, r->clsT, ba);
        PFAG_LAUNCHED(c);
        real *X = (real *)r->Y2;          // pass B is done with Y2: Fx, then the row term
        pfag_prof_begin(c, "kr_boxC2");
        kr_boxC2<real, MM><<<grow, BG::THREADS, smC, s>>>(Y1, X, R(c->rho), c->d_xc, c->d_yc, ba,
                                                           c->debug ? R(c->d_vx) : nullptr,
                                                           c->debug ? R(c->d_vy) : nullptr);
        PFAG_LAUNCHED(c);
        pfag_prof_begin(c, "kr_boxD2");
        kr_boxD2<real, MM><<<dim3(MM / BD::COLS, Nt), 256, smD2, s>>>(X, R(c->rho), R(r->Rb), c->d_xc, c->d_yc, ba);
        PFAG_LAUNCHED(c);
        return PFAG_OK;
    }

    // centroid sums over every support rectangle from the current phi (after
    // phi was changed between steps), for the next step's centroids
    int recentre() {
        PFAG_CUDA_CHECK(cudaMemsetAsync(c->d_cacc, 0, sizeof(long long) * 3 * c->Ntot, c->stream));
        kf_centroid<real><<<dim3(64, c->Ntot), FT, 0, c->stream>>>(R(c->phi), r->rect, c->N, c->d_cacc);
        PFAG_CUDA_CHECK(cudaGetLastError());
        return PFAG_OK;
    }

    int stats() {
        const int Nt = c->Ntot;
        if (std::getenv("PFAG_DEBUG_COOP")) {
            cudaFuncAttributes fr{};
            cudaFuncGetAttributes(&fr, (const void *)kf_relax_loops<real, RESH_RB>);
            std::fprintf(stderr, "pfag coop: relaxation loops %d blocks x %d threads (%d regs)\n", r->coop_r,
                         r->resh_threads, fr.numRegs);
        }
        std::vector<int> h(3 * Nt + 8);
        PFAG_CUDA_CHECK(cudaMemcpyAsync(h.data(), r->cK, sizeof(int) * (3 * Nt + 8), cudaMemcpyDeviceToHost, c->stream));
        PFAG_CUDA_CHECK(cudaStreamSynchronize(c->stream));
        int mx = 0, sm = 0;
        for (int n = 0; n < Nt; n++) {
            c->h_iflags[4 * Nt + n] = h[n];
            mx = std::max(mx, h[n]);
            sm += h[n];
        }
        c->stats.cell_iters_max = mx;
        c->stats.cell_iters_sum = sm;
        c->stats.lum_iters = h[3 * Nt + 0];
        c->stats.ecm_iters = h[3 * Nt + 1];
        return PFAG_OK;
    }
};

// Entry points instantiated once per precision (pfag_fused_f64.cu, pfag_fused_f32.cu).
template <typename real> int fused_alloc_t(pfag_ctx *c) { return Fused<real>(c).alloc(); }
template <typename real> int fused_stats_t(pfag_ctx *c) { return Fused<real>(c).stats(); }
template <typename real> int fused_recentre_t(pfag_ctx *c) { return Fused<real>(c).recentre(); }
template <typename real> int fused_upload_t(pfag_ctx *c) { return Fused<real>(c).upload_hook(); }
inline void fused_drop_graph(FusedRes *r) {
    if (r->graph_ok) { cudaGraphExecDestroy(r->gexec); cudaGraphDestroy(r->graph); }
    r->graph_ok = false;
    for (int k = 0; k < 2; k++) {
        if (r->pgraph_ok[k]) { cudaGraphExecDestroy(r->pgexec[k]); cudaGraphDestroy(r->pgraph[k]); }
        r->pgraph_ok[k] = false;
        r->pgraph_state[k] = 0;
    }
}

// One part of a step split at psi (part 1: head, 2: tail), graph-captured
// like the whole step once an eager step has run: the head after the first
// eager head-and-tail, the tail likewise.
template <typename real> int fused_step_part_t(pfag_ctx *c, int part, bool sync_host) {
    FusedRes *r = F(c);
    if ((part == 1) == r->head_pending) {
        pfag_set_error(part == 1 ? "step head enqueued twice without its tail" : "step tail without its head");
        return PFAG_E_ARG;
    }
    const int k = part - 1;
    const bool graphable = !pfag_prof_on(c) && !c->debug && !std::getenv("PFAG_NO_GRAPH");
    if (r->graph_key != (long)c->relax_cap) {
        fused_drop_graph(r);
        r->graph_state = 0;
        r->graph_key = (long)c->relax_cap;
    }
    if (graphable && r->pgraph_state[k] == 0 && r->eager_steps >= 1 && !r->ring_pending) {
        cudaStream_t s = c->stream;
        const long l0 = c->launches;
        r->pgraph_state[k] = -1;
        if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            const int rc = Fused<real>(c).enqueue(part);
            cudaGraph_t g = nullptr;
            const cudaError_t e = cudaStreamEndCapture(s, &g);
            if (rc == PFAG_OK && e == cudaSuccess && g && cudaGraphInstantiate(&r->pgexec[k], g, 0) == cudaSuccess) {
                r->pgraph[k] = g;
                r->pgraph_ok[k] = true;
                r->pgraph_state[k] = 1;
                r->pgraph_launches[k] = c->launches - l0;
            } else if (g) {
                cudaGraphDestroy(g);
            }
        }
        c->launches = l0;
        (void)cudaGetLastError();
    }
    if (r->pgraph_ok[k] && !r->ring_pending && graphable) {
        PFAG_CUDA_CHECK(cudaGraphLaunch(r->pgexec[k], c->stream));
        c->launches += r->pgraph_launches[k];
    } else {
        const int rc = Fused<real>(c).enqueue(part);
        if (rc != PFAG_OK) return rc;
        if (part == 2) {
            r->eager_steps++;
            r->ring_pending = false;
        }
    }
    r->head_pending = part == 1;
    if (sync_host && part == 2) {
        PFAG_CUDA_CHECK(cudaStreamSynchronize(c->stream));
        return Fused<real>(c).stats();
    }
    return PFAG_OK;
}

// One step.  The first step runs eagerly (kernel attributes and the
// persistent kernels' block counts settle there); the next one is captured
// into a CUDA graph that every later step replays with one launch.  Profiling,
// debug capture and PFAG_NO_GRAPH keep the eager path; a failed capture falls
// back to it for good.
template <typename real> int fused_step_t(pfag_ctx *c, bool sync_host) {
    FusedRes *r = F(c);
    if (r->head_pending) { pfag_set_error("a step head is waiting for its tail"); return PFAG_E_ARG; }
    const bool graphable = !pfag_prof_on(c) && !c->debug && !std::getenv("PFAG_NO_GRAPH");
    const long key = (long)c->relax_cap;
    if (r->graph_ok && r->graph_key != key) {
        fused_drop_graph(r);
        r->graph_state = 0;
    }
    if (graphable && r->graph_state == 0 && r->eager_steps >= 1 && !r->ring_pending) {
        cudaStream_t s = c->stream;
        const long l0 = c->launches;
        r->graph_state = -1;
        if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            const int rc = Fused<real>(c).enqueue();
            cudaGraph_t g = nullptr;
            const cudaError_t e = cudaStreamEndCapture(s, &g);
            if (rc == PFAG_OK && e == cudaSuccess && g && cudaGraphInstantiate(&r->gexec, g, 0) == cudaSuccess) {
                r->graph = g;
                r->graph_ok = true;
                r->graph_state = 1;
                r->graph_key = key;
                r->graph_launches = c->launches - l0;
            } else if (g) {
                cudaGraphDestroy(g);
            }
        }
        c->launches = l0;
        (void)cudaGetLastError();   // a refused capture leaves a non-sticky error
    }
    int rc = PFAG_OK;
    if (r->graph_ok && !r->ring_pending && graphable) {
        PFAG_CUDA_CHECK(cudaGraphLaunch(r->gexec, c->stream));
        c->launches += r->graph_launches;
    } else {
        rc = Fused<real>(c).enqueue();
        if (rc != PFAG_OK) return rc;
        r->eager_steps++;
        r->ring_pending = false;
    }
    if (sync_host) {
        PFAG_CUDA_CHECK(cudaStreamSynchronize(c->stream));
        rc = Fused<real>(c).stats();
    }
    return rc;
}

}  // namespace
