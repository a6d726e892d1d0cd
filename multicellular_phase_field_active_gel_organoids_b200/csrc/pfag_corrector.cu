// Learned coarse-grid corrector: the kernels of a small convolutional network
// (3x3 convolutions, BF16 weights and activations, FP32 accumulation) on the
// 5th-generation tensor cores, for its inference and its training on the GPU.
// No counterpart in the reference (its step has no learned part).
//
// Layout.  An activation tensor is BF16 [B][H+2][W+2][C] (NHWC with a
// one-site zero halo, C a multiple of 8): the halo is the convolution's zero
// padding, so every tap of every pixel reads memory of the same sample.
// Pixels are numbered q = y*(W+2) + x inside a sample.  A weight tensor is
// BF16 [Cout][9][Cin] (tap t = (dy+1)*3 + (dx+1)), i.e. a [Cout][K] matrix with
// K = 9 Cin ordered (tap, channel).
//
// Forward (kc_conv_fwd): implicit GEMM D[q][co] = sum_k A[q][k] B[co][k] over
// tiles of 128 consecutive pixels q0 .. q0+127 of the rows 1..H of a sample
// (halo columns included; their outputs are written as zero).  The CTA
// stages the pixels q0 - (W+2) - 1 .. q0 + 127 + (W+2) + 1 once in shared
// memory as [Cin/8][P][8] (16-byte rows: the canonical no-swizzle K-major
// core-matrix layout, 8 pixels x 8 channels per 128-byte core matrix); the A
// operand of tap t is the same buffer seen from pixel offset
// (W+2)+1 + dy*(W+2) + dx through its matrix descriptor, so there is no
// im2col copy.  One thread issues the 9 Cin/16 tcgen05.mma (M = 128, N = Cout,
// K = 16) into a TMEM accumulator, tcgen05.commit arrives on an mbarrier, and
// each warp reads its 32 rows back with tcgen05.ld for the epilogue (bias,
// GELU, BF16 stores; the pre-activation is kept for training).
//
// Weight gradient (kc_conv_wgrad): dW[co][t][ci] = sum_q dZ[q][co] X[q+off_t][ci]
// as D[co][ci] per tap with M = 128 (co, zero-padded), N = Cin, K = pixels:
// both operands MN-major from the staged [C/8][pixels][8] buffers (a core
// matrix is 8 pixels x 8 channels either way), 9 accumulators of Cin columns
// that live in TMEM across all tiles of the CTA, added to dW at the end.
// The input gradient is the forward kernel with the flipped, transposed
// weights (kc_flip).
//
// Every wait on an mbarrier is bounded; a wait that runs out sets bit 0 of
// *err and the kernel skips the rest of its work (the host reports it).
#include "pfag_internal.cuh"
#include <cuda_bf16.h>
#include <cstdint>

namespace {

constexpr int KC_THREADS = 128;
constexpr long KC_SPIN_LIMIT = 1L << 26;

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// no-swizzle matrix descriptor (version 1): start, leading and stride byte offsets
__device__ __forceinline__ uint64_t mdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// instruction descriptor of kind::f16: BF16 x BF16 -> F32, M = 128, N, majors
__host__ __device__ constexpr uint32_t idesc_bf16(int n, int a_mn, int b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
           ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

// bounded wait for the given phase parity; false if it ran out
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
    for (long it = 0; it < KC_SPIN_LIMIT; it++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// warp 0 allocates `ncols` TMEM columns (a power of two >= 32) and publishes the address
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, int ncols) {
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
                     "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
}

__device__ __forceinline__ void tmem_free(uint32_t taddr, int ncols) {
    if (threadIdx.x < 32)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 32 lanes x 16 columns of FP32 from TMEM (lane base encoded in taddr)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 16; k++) v[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ void cp16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
    return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

// Stage pixels [q_lo, q_lo + P) of sample b (zero outside 0 .. Q-1) as [C/8][P][8].
__device__ __forceinline__ void stage_pixels(unsigned char *dst, const __nv_bfloat16 *__restrict__ x, long sample_off,
                                             int q_lo, int P, int Q, int C) {
    const int chunks = C / 8;
    for (int e = threadIdx.x; e < P * chunks; e += blockDim.x) {
        const int c = e / P, p = e - c * P;
        const int q = q_lo + p;
        unsigned char *d = dst + ((size_t)c * P + p) * 16;
        if (q >= 0 && q < Q) cp16(d, x + (sample_off + q) * C + c * 8);
        else *reinterpret_cast<uint4 *>(d) = make_uint4(0, 0, 0, 0);
    }
}

// Y = act(conv3x3(X, W) + bias) on the padded layout.  cin in {16, 32, 64},
// cout in {16, 32}.  pre (optional): the pre-activation, same layout as Y.
template <int CIN, int COUT, bool GELU>
__global__ void __launch_bounds__(KC_THREADS) kc_conv_fwd(const __nv_bfloat16 *__restrict__ x,
                                                          const __nv_bfloat16 *__restrict__ w,
                                                          const float *__restrict__ bias,
                                                          __nv_bfloat16 *__restrict__ y, __nv_bfloat16 *__restrict__ pre,
                                                          int B, int H, int W, unsigned *__restrict__ err) {
    extern __shared__ __align__(128) unsigned char kc_smem[];
    __shared__ __align__(8) unsigned long long mbar_store;
    __shared__ uint32_t tmem_slot;
    const int Wp = W + 2, Q = (H + 2) * Wp;
    const int P = 128 + 2 * Wp + 2;
    const int tiles_per = (H * Wp + 127) / 128;
    const long ntiles = (long)B * tiles_per;
    unsigned char *ws = kc_smem;                                // weights [9 CIN/8][COUT][8]
    unsigned char *xs = kc_smem + (size_t)9 * CIN * COUT * 2;   // pixels [CIN/8][P][8]
    const uint32_t mbar = smem_addr(&mbar_store);
    // weights once: chunk c of row n at (c COUT + n) 16
    for (int e = threadIdx.x; e < 9 * CIN / 8 * COUT; e += blockDim.x) {
        const int c = e / COUT, n = e - c * COUT;
        cp16(ws + ((size_t)c * COUT + n) * 16, w + (size_t)n * 9 * CIN + c * 8);
    }
    if (threadIdx.x == 0) {
        mbar_init(mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tmem_alloc(&tmem_slot, 32);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;
    const uint32_t idesc = idesc_bf16(COUT, 0, 0);
    uint32_t phase = 0;
    bool ok = true;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const int b = (int)(tile / tiles_per), tb = (int)(tile - (long)b * tiles_per);
        const int q0 = Wp + tb * 128;
        const long soff = (long)b * Q;
        stage_pixels(xs, x, soff, q0 - Wp - 1, P, Q, CIN);
        cp_wait();
        proxy_fence();
        __syncthreads();
        tc_fence_after();
        if (threadIdx.x == 0) {
            const uint32_t xa = smem_addr(xs), wa = smem_addr(ws);
#pragma unroll 1
            for (int t = 0; t < 9; t++) {
                const int off = (t / 3 - 1) * Wp + (t % 3 - 1);
#pragma unroll
                for (int j = 0; j < CIN / 16; j++) {
                    const uint64_t a = mdesc(xa + (uint32_t)(((2 * j) * P + (Wp + 1 + off)) * 16), (uint32_t)P * 16, 128);
                    const uint64_t bd = mdesc(wa + (uint32_t)((t * (CIN / 8) + 2 * j) * COUT * 16), COUT * 16, 128);
                    mma_bf16(tmem, a, bd, idesc, (t | j) != 0);
                }
            }
            mma_commit(mbar);
        }
        if (!mbar_wait(mbar, phase)) {
            if (lane == 0) atomicOr(err, 1u);
            ok = false;
        }
        phase ^= 1;
        tc_fence_after();
        // row m = 32 warp + lane of D: pixel q0 + m (the loads run in every
        // lane whatever the wait gave: tcgen05.ld is warp-collective)
        const int q = q0 + 32 * warp + lane;
        const int yy = q / Wp, xx = q - yy * Wp;
        const bool valid = ok && q < (H + 1) * Wp && xx >= 1 && xx <= W;
        float acc[COUT];
#pragma unroll
        for (int h = 0; h < COUT / 16; h++) {
            float v[16];
            tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + 16 * h, v);
#pragma unroll
            for (int k = 0; k < 16; k++) acc[16 * h + k] = v[k];
        }
        if (q < (H + 1) * Wp) {
            __align__(16) __nv_bfloat16 out[COUT], pr[COUT];
#pragma unroll
            for (int k = 0; k < COUT; k++) {
                const float z = valid ? acc[k] + bias[k] : 0.0f;
                pr[k] = __float2bfloat16_rn(z);
                out[k] = __float2bfloat16_rn(valid ? (GELU ? gelu(z) : z) : 0.0f);
            }
            uint4 *dy = reinterpret_cast<uint4 *>(y + (soff + q) * COUT);
#pragma unroll
            for (int k = 0; k < COUT / 8; k++) dy[k] = reinterpret_cast<const uint4 *>(out)[k];
            if (pre) {
                uint4 *dp = reinterpret_cast<uint4 *>(pre + (soff + q) * COUT);
#pragma unroll
                for (int k = 0; k < COUT / 8; k++) dp[k] = reinterpret_cast<const uint4 *>(pr)[k];
            }
        }
        tc_fence_before();
        ok = __syncthreads_and(ok);   // every thread leaves the loop together
    }
    tc_fence_after();
    __syncthreads();
    tmem_free(tmem, 32);
}

// dW[co][t][ci] += sum_q dz[q][co] x[q + off_t][ci], db[co] += sum_q dz[q][co]
// (dz zero on halo sites).  CIN in {16, 32, 64}, COUT in {16, 32}.
template <int CIN, int COUT>
__global__ void __launch_bounds__(KC_THREADS) kc_conv_wgrad(const __nv_bfloat16 *__restrict__ x,
                                                            const __nv_bfloat16 *__restrict__ dz,
                                                            float *__restrict__ dw, float *__restrict__ db, int B, int H,
                                                            int W, unsigned *__restrict__ err) {
    extern __shared__ __align__(128) unsigned char kc_smem[];
    __shared__ __align__(8) unsigned long long mbar_store;
    __shared__ uint32_t tmem_slot;
    constexpr int NCOL = 9 * CIN <= 256 ? 256 : 512;      // TMEM columns: 9 accumulators of CIN
    const int Wp = W + 2, Q = (H + 2) * Wp;
    const int P = 128 + 2 * Wp + 2;
    const int tiles_per = (H * Wp + 127) / 128;
    const long ntiles = (long)B * tiles_per;
    unsigned char *gs = kc_smem;                             // dz [16][128][8]: co padded to 128
    unsigned char *xs = kc_smem + (size_t)16 * 128 * 16;     // x [CIN/8][P][8]
    const uint32_t mbar = smem_addr(&mbar_store);
    for (int e = threadIdx.x; e < 16 * 128; e += blockDim.x)
        *reinterpret_cast<uint4 *>(gs + (size_t)e * 16) = make_uint4(0, 0, 0, 0);
    if (threadIdx.x == 0) {
        mbar_init(mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tmem_alloc(&tmem_slot, NCOL);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;
    const uint32_t idesc = idesc_bf16(CIN, 1, 1);
    uint32_t phase = 0;
    bool ok = true, first = true;
    float bsum = 0.0f;                                        // db partial of channel threadIdx.x (< COUT)
    for (long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const int b = (int)(tile / tiles_per), tb = (int)(tile - (long)b * tiles_per);
        const int q0 = Wp + tb * 128;
        const long soff = (long)b * Q;
        stage_pixels(xs, x, soff, q0 - Wp - 1, P, Q, CIN);
        for (int e = threadIdx.x; e < (COUT / 8) * 128; e += blockDim.x) {
            const int c = e / 128, p = e - c * 128;
            const int q = q0 + p;
            unsigned char *d = gs + ((size_t)c * 128 + p) * 16;
            if (q < (H + 1) * Wp) cp16(d, dz + (soff + q) * COUT + c * 8);
            else *reinterpret_cast<uint4 *>(d) = make_uint4(0, 0, 0, 0);
        }
        cp_wait();
        proxy_fence();
        __syncthreads();
        tc_fence_after();
        if (threadIdx.x < COUT) {
            const __nv_bfloat16 *g = reinterpret_cast<const __nv_bfloat16 *>(gs);
            const int c = threadIdx.x / 8, k = threadIdx.x % 8;
            for (int p = 0; p < 128; p++) bsum += __bfloat162float(g[((size_t)c * 128 + p) * 8 + k]);
        }
        if (threadIdx.x == 0) {
            const uint32_t xa = smem_addr(xs), ga = smem_addr(gs);
#pragma unroll 1
            for (int t = 0; t < 9; t++) {
                const int off = (t / 3 - 1) * Wp + (t % 3 - 1);
#pragma unroll 1
                for (int ks = 0; ks < 8; ks++) {
                    // A: dz^T (M = co over 16 chunks of 8, K = 16 pixels), MN-major
                    const uint64_t a = mdesc(ga + (uint32_t)(ks * 16 * 16), 128, 128 * 16);
                    // B: x shifted by tap t (N = ci, K = 16 pixels), MN-major
                    const uint64_t bd = mdesc(xa + (uint32_t)((Wp + 1 + off + ks * 16) * 16), 128, (uint32_t)P * 16);
                    mma_bf16(tmem + (uint32_t)(t * CIN), a, bd, idesc, (first && ks == 0) ? 0u : 1u);
                }
            }
            mma_commit(mbar);
        }
        if (!mbar_wait(mbar, phase)) {
            if ((threadIdx.x & 31) == 0) atomicOr(err, 1u);
            ok = false;
        }
        phase ^= 1;
        first = false;
        tc_fence_before();
        ok = __syncthreads_and(ok);   // every thread leaves the loop together
    }
    tc_fence_after();
    if (threadIdx.x < COUT) atomicAdd(&db[threadIdx.x], bsum);
    // warp 0 holds rows co = lane of every accumulator
    if (!first && ok && threadIdx.x < 32) {
        const int co = threadIdx.x;
#pragma unroll 1
        for (int c0 = 0; c0 < 9 * CIN; c0 += 16) {
            float v[16];
            tmem_ld16(tmem + (uint32_t)c0, v);
            if (co < COUT)
#pragma unroll
                for (int k = 0; k < 16; k++) {
                    const int col = c0 + k, t = col / CIN, ci = col - t * CIN;
                    atomicAdd(&dw[((size_t)co * 9 + t) * CIN + ci], v[k]);
                }
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    tmem_free(tmem, NCOL);
}

// dz = dy * GELU'(pre) (or dy without activation), zero on the halo
template <int C>
__global__ void kc_act_bwd(const __nv_bfloat16 *__restrict__ dy, const __nv_bfloat16 *__restrict__ pre,
                           __nv_bfloat16 *__restrict__ dz, int B, int H, int W, int gelu_on) {
    const int Wp = W + 2, Q = (H + 2) * Wp;
    const long tot = (long)B * Q * C;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (long)gridDim.x * blockDim.x) {
        const long px = e / C;
        const int q = (int)(px % Q), yy = q / Wp, xx = q - yy * Wp;
        float g = 0.0f;
        if (yy >= 1 && yy <= H && xx >= 1 && xx <= W) {
            g = __bfloat162float(dy[e]);
            if (gelu_on) g *= gelu_grad(__bfloat162float(pre[e]));
        }
        dz[e] = __float2bfloat16_rn(g);
    }
}

// wt[ci][t'][co] = w[co][8 - t'][ci]: the input gradient as a forward convolution
__global__ void kc_flip(const __nv_bfloat16 *__restrict__ w, __nv_bfloat16 *__restrict__ wt, int cin, int cout) {
    const int tot = cin * 9 * cout;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += gridDim.x * blockDim.x) {
        const int ci = e / (9 * cout), r = e - ci * 9 * cout, t = r / cout, co = r - t * cout;
        wt[e] = w[((size_t)co * 9 + (8 - t)) * cin + ci];
    }
}

// Adam on FP32 master weights, BF16 copies for the kernels; `mask` (optional)
// zeroes the update of padded entries.
__global__ void kc_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                        float *__restrict__ v, __nv_bfloat16 *__restrict__ pb, const float *__restrict__ mask, int n,
                        float lr, float b1, float b2, float eps, float c1, float c2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        float step = lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        if (mask) step *= mask[i];
        const float pi = p[i] - step;
        p[i] = pi;
        if (pb) pb[i] = __float2bfloat16_rn(pi);
    }
}

// mean squared error over the valid sites and the first `nout` channels of
// out (padded, C channels) against target [B][H][W][nout] (FP32); writes the
// gradient into dout (padded, zero elsewhere) and adds the loss sum to *loss
template <int C>
__global__ void kc_mse(const __nv_bfloat16 *__restrict__ out, const float *__restrict__ target,
                       __nv_bfloat16 *__restrict__ dout, float *__restrict__ loss, int B, int H, int W, int nout,
                       float scale) {
    const int Wp = W + 2, Q = (H + 2) * Wp;
    const long tot = (long)B * Q * C;
    float acc = 0.0f;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (long)gridDim.x * blockDim.x) {
        const long px = e / C;
        const int ch = (int)(e - px * C);
        const int b = (int)(px / Q), q = (int)(px - (long)b * Q), yy = q / Wp, xx = q - yy * Wp;
        float g = 0.0f;
        if (ch < nout && yy >= 1 && yy <= H && xx >= 1 && xx <= W) {
            const float d = __bfloat162float(out[e]) - target[(((long)b * H + (yy - 1)) * W + (xx - 1)) * nout + ch];
            acc += d * d;
            g = 2.0f * d * scale;
        }
        dout[e] = __float2bfloat16_rn(g);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, acc);
}

// The corrector's input on each cell's FFT box [xc-z+1, xc+z-2]^2:
// x0[n][1+i][1+j] = (phi, rho, s_v vx, s_v vy, 0 ...) scaled, BF16, 16 channels
template <typename real>
__global__ void kc_gather(const real *__restrict__ phi, const real *__restrict__ rho, const real *__restrict__ vx,
                          const real *__restrict__ vy, const int *__restrict__ xc, const int *__restrict__ yc, int N,
                          int z, int M, float s_phi, float s_rho, float s_v, __nv_bfloat16 *__restrict__ x0) {
    const int n = blockIdx.y;
    const int bi = xc[n] - z + 1, bj = yc[n] - z + 1, Mp = M + 2;
    const size_t NN = (size_t)N * N;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < M * M; e += gridDim.x * blockDim.x) {
        const int i = e / M, j = e - i * M;
        const size_t s = (size_t)n * NN + (size_t)(bi + i) * N + bj + j;
        const size_t b = (size_t)n * M * M + e;
        __align__(16) __nv_bfloat16 v[16];
        v[0] = __float2bfloat16_rn((float)phi[s] * s_phi);
        v[1] = __float2bfloat16_rn((float)rho[s] * s_rho);
        v[2] = __float2bfloat16_rn(vx ? (float)vx[b] * s_v : 0.0f);
        v[3] = __float2bfloat16_rn(vy ? (float)vy[b] * s_v : 0.0f);
#pragma unroll
        for (int k = 4; k < 16; k++) v[k] = __float2bfloat16_rn(0.0f);
        uint4 *d = reinterpret_cast<uint4 *>(x0 + (((size_t)n * Mp + 1 + i) * Mp + 1 + j) * 16);
        d[0] = reinterpret_cast<const uint4 *>(v)[0];
        d[1] = reinterpret_cast<const uint4 *>(v)[1];
    }
}

// phi += s_phi out[..0], rho += s_rho out[..1] on each cell's FFT box
template <typename real>
__global__ void kc_apply(const __nv_bfloat16 *__restrict__ out, real *__restrict__ phi, real *__restrict__ rho,
                         const int *__restrict__ xc, const int *__restrict__ yc, int N, int z, int M, float s_phi,
                         float s_rho) {
    const int n = blockIdx.y;
    const int bi = xc[n] - z + 1, bj = yc[n] - z + 1, Mp = M + 2;
    const size_t NN = (size_t)N * N;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < M * M; e += gridDim.x * blockDim.x) {
        const int i = e / M, j = e - i * M;
        const size_t s = (size_t)n * NN + (size_t)(bi + i) * N + bj + j;
        const __nv_bfloat16 *o = out + (((size_t)n * Mp + 1 + i) * Mp + 1 + j) * 16;
        phi[s] = phi[s] + (real)(s_phi * __bfloat162float(o[0]));
        rho[s] = rho[s] + (real)(s_rho * __bfloat162float(o[1]));
    }
}

template <int CIN, int COUT, bool G>
int launch_fwd(const void *x, const void *w, const float *bias, void *y, void *pre, int B, int H, int W,
               unsigned *err, cudaStream_t s) {
    const int Wp = W + 2, P = 128 + 2 * Wp + 2;
    const size_t smem = (size_t)9 * CIN * COUT * 2 + (size_t)CIN / 8 * P * 16;
    if (smem > 200 * 1024) { pfag_set_error("conv: box width %d too large for the staged tile", W); return PFAG_E_ARG; }
    PFAG_CUDA_CHECK(cudaFuncSetAttribute(kc_conv_fwd<CIN, COUT, G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem));
    const long ntiles = (long)B * ((H * Wp + 127) / 128);
    const int grid = (int)std::min<long>(ntiles, 148L * 4);
    kc_conv_fwd<CIN, COUT, G><<<grid, KC_THREADS, smem, s>>>(
        (const __nv_bfloat16 *)x, (const __nv_bfloat16 *)w, bias, (__nv_bfloat16 *)y, (__nv_bfloat16 *)pre, B, H, W,
        err);
    PFAG_CUDA_CHECK(cudaGetLastError());
    return PFAG_OK;
}

template <int CIN, int COUT>
int launch_wgrad(const void *x, const void *dz, float *dw, float *db, int B, int H, int W, unsigned *err,
                 cudaStream_t s) {
    const int Wp = W + 2, P = 128 + 2 * Wp + 2;
    const size_t smem = (size_t)16 * 128 * 16 + (size_t)CIN / 8 * P * 16;
    if (smem > 200 * 1024) { pfag_set_error("conv: box width %d too large for the staged tile", W); return PFAG_E_ARG; }
    PFAG_CUDA_CHECK(cudaFuncSetAttribute(kc_conv_wgrad<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem));
    const long ntiles = (long)B * ((H * Wp + 127) / 128);
    // one CTA per SM at most (512 TMEM columns for CIN = 64), each over many tiles
    const int grid = (int)std::min<long>(ntiles, 148L);
    kc_conv_wgrad<CIN, COUT><<<grid, KC_THREADS, smem, s>>>((const __nv_bfloat16 *)x, (const __nv_bfloat16 *)dz, dw,
                                                             db, B, H, W, err);
    PFAG_CUDA_CHECK(cudaGetLastError());
    return PFAG_OK;
}

}  // namespace

// ---- C ABI ------------------------------------------------------------------
extern "C" int pfag_conv3x3(const void *x, const void *w, const float *bias, void *y, void *pre, int B, int H, int W,
                            int cin, int cout, int gelu_on, unsigned *err, void *stream) {
    if (!x || !w || !bias || !y || !err || B < 1 || H < 1 || W < 1) { pfag_set_error("pfag_conv3x3: bad arguments"); return PFAG_E_ARG; }
    cudaStream_t s = (cudaStream_t)stream;
#define KC_FWD(ci, co)                                                                                         \
    if (cin == ci && cout == co)                                                                               \
        return gelu_on ? launch_fwd<ci, co, true>(x, w, bias, y, pre, B, H, W, err, s)                         \
                       : launch_fwd<ci, co, false>(x, w, bias, y, pre, B, H, W, err, s);
    KC_FWD(16, 32) KC_FWD(32, 32) KC_FWD(32, 16) KC_FWD(16, 16)
#undef KC_FWD
    pfag_set_error("pfag_conv3x3: channel pair %d -> %d not built (16/32 -> 16/32)", cin, cout);
    return PFAG_E_UNSUPPORTED;
}

extern "C" int pfag_conv3x3_wgrad(const void *x, const void *dz, float *dw, float *db, int B, int H, int W, int cin,
                                  int cout, unsigned *err, void *stream) {
    if (!x || !dz || !dw || !db || !err || B < 1 || H < 1 || W < 1) { pfag_set_error("pfag_conv3x3_wgrad: bad arguments"); return PFAG_E_ARG; }
    cudaStream_t s = (cudaStream_t)stream;
#define KC_WG(ci, co) \
    if (cin == ci && cout == co) return launch_wgrad<ci, co>(x, dz, dw, db, B, H, W, err, s);
    KC_WG(16, 32) KC_WG(32, 32) KC_WG(32, 16) KC_WG(16, 16)
#undef KC_WG
    pfag_set_error("pfag_conv3x3_wgrad: channel pair %d -> %d not built", cin, cout);
    return PFAG_E_UNSUPPORTED;
}

extern "C" int pfag_conv_act_bwd(const void *dy, const void *pre, void *dz, int B, int H, int W, int c, int gelu_on,
                                 void *stream) {
    cudaStream_t s = (cudaStream_t)stream;
    if (c == 16) kc_act_bwd<16><<<592, 256, 0, s>>>((const __nv_bfloat16 *)dy, (const __nv_bfloat16 *)pre,
                                                    (__nv_bfloat16 *)dz, B, H, W, gelu_on);
    else if (c == 32) kc_act_bwd<32><<<592, 256, 0, s>>>((const __nv_bfloat16 *)dy, (const __nv_bfloat16 *)pre,
                                                         (__nv_bfloat16 *)dz, B, H, W, gelu_on);
    else { pfag_set_error("pfag_conv_act_bwd: %d channels", c); return PFAG_E_UNSUPPORTED; }
    PFAG_CUDA_CHECK(cudaGetLastError());
    return PFAG_OK;
}

extern "C" int pfag_conv_flip(const void *w, void *wt, int cin, int cout, void *stream) {
    kc_flip<<<64, 256, 0, (cudaStream_t)stream>>>((const __nv_bfloat16 *)w, (__nv_bfloat16 *)wt, cin, cout);
    PFAG_CUDA_CHECK(cudaGetLastError());
    return PFAG_OK;
}

extern "C" int pfag_adam(float *p, const float *g, float *m, float *v, void *pb, const float *mask, int n, float lr,
                         float b1, float b2, float eps, int t, void *stream) {
    if (t < 1) { pfag_set_error("pfag_adam: step t >= 1"); return PFAG_E_ARG; }
    const float c1 = 1.0f - powf(b1, (float)t), c2 = 1.0f - powf(b2, (float)t);
    kc_adam<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(p, g, m, v, (__nv_bfloat16 *)pb, mask, n, lr, b1, b2,
                                                               eps, c1, c2);
    PFAG_CUDA_CHECK(cudaGetLastError());
    return PFAG_OK;
}

extern "C" int pfag_conv_mse(const void *out, const float *target, void *dout, float *loss, int B, int H, int W,
                             int c, int nout, float scale, void *stream) {
    cudaStream_t s = (cudaStream_t)stream;
    if (c == 16) kc_mse<16><<<592, 256, 0, s>>>((const __nv_bfloat16 *)out, target, (__nv_bfloat16 *)dout, loss, B, H,
                                                W, nout, scale);
    else { pfag_set_error("pfag_conv_mse: %d channels", c); return PFAG_E_UNSUPPORTED; }
    PFAG_CUDA_CHECK(cudaGetLastError());
    return PFAG_OK;
}

extern "C" int pfag_corrector_gather(pfag_ctx *c, void *x0, float s_phi, float s_rho, float s_v) {
    if (!c || !x0) { pfag_set_error("pfag_corrector_gather: bad arguments"); return PFAG_E_ARG; }
    const dim3 g((c->M * c->M + 255) / 256, c->Ntot);
    if (c->prec == 64)
        kc_gather<double><<<g, 256, 0, c->stream>>>((const double *)c->phi, (const double *)c->rho,
                                                   (const double *)c->d_vx, (const double *)c->d_vy, c->d_xc, c->d_yc,
                                                   c->N, c->zone, c->M, s_phi, s_rho, s_v, (__nv_bfloat16 *)x0);
    else
        kc_gather<float><<<g, 256, 0, c->stream>>>((const float *)c->phi, (const float *)c->rho,
                                                  (const float *)c->d_vx, (const float *)c->d_vy, c->d_xc, c->d_yc,
                                                  c->N, c->zone, c->M, s_phi, s_rho, s_v, (__nv_bfloat16 *)x0);
    PFAG_CUDA_CHECK(cudaGetLastError());
    return PFAG_OK;
}

extern "C" int pfag_corrector_apply(pfag_ctx *c, const void *out, float s_phi, float s_rho) {
    if (!c || !out) { pfag_set_error("pfag_corrector_apply: bad arguments"); return PFAG_E_ARG; }
    if (c->path != PFAG_PATH_FUSED) { pfag_set_error("pfag_corrector_apply: fused path only"); return PFAG_E_UNSUPPORTED; }
    const dim3 g((c->M * c->M + 255) / 256, c->Ntot);
    if (c->prec == 64)
        kc_apply<double><<<g, 256, 0, c->stream>>>((const __nv_bfloat16 *)out, (double *)c->phi, (double *)c->rho,
                                                  c->d_xc, c->d_yc, c->N, c->zone, c->M, s_phi, s_rho);
    else
        kc_apply<float><<<g, 256, 0, c->stream>>>((const __nv_bfloat16 *)out, (float *)c->phi, (float *)c->rho,
                                                 c->d_xc, c->d_yc, c->N, c->zone, c->M, s_phi, s_rho);
    PFAG_CUDA_CHECK(cudaGetLastError());
    return pfag_fused_recentre(c);
}
