// Shared-memory FFT building blocks for the fused spectral solve.
//
// Power-of-two lengths M = 2^logm.  Sequences live in shared memory; the
// caller stores each input sequence in bit-reversed order, then
// fft_stages() runs in-place decimation-in-time radix-4 steps (one radix-2
// step first when logm is odd) and leaves the result in natural order.  Each
// radix-4 step is two radix-2 Cooley-Tukey merges done in registers:
//   merge of sub-transforms of size Q into 2Q with twiddle W_{2Q}^k, then of
//   2Q into L = 4Q with W_L^k and W_L^{k+Q}.
// Forward sign exp(-2 pi i k / M), inverse exp(+2 pi i k / M), unnormalised,
// matching the C2C transforms the reference's spectral solve uses.
#pragma once
#include <cuda_runtime.h>

template <typename T> struct CxOps;
template <> struct CxOps<double2> {
    typedef double real;
    static __device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }
};
template <> struct CxOps<float2> {
    typedef float real;
    static __device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }
};

template <typename T> __device__ __forceinline__ T cadd(T a, T b) { T r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename T> __device__ __forceinline__ T csub(T a, T b) { T r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <typename T> __device__ __forceinline__ T cmul(T a, T b) {
    T r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}
// FP32 complex add / subtract as sm_100 packed FP32 instructions (both
// components in one instruction, each rounded as the scalar operation is:
// a - b is fma(b, -1, a), exact product then one rounding), so the FFTs'
// butterflies take half the instructions and give the same bits
template <> __device__ __forceinline__ float2 cadd<float2>(float2 a, float2 b) { return __fadd2_rn(a, b); }
template <> __device__ __forceinline__ float2 csub<float2>(float2 a, float2 b) {
    return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a);
}
template <typename T> __device__ __forceinline__ T cconj(T a) { a.y = -a.y; return a; }

__device__ __forceinline__ int bitrev(int x, int logm) { return (int)(__brev((unsigned)x) >> (32 - logm)); }

// tw[k] = exp(-2 pi i k / M), k in [0, M)
template <typename T>
__device__ __forceinline__ void fft_twiddles(T *tw, int M) {
    typedef typename CxOps<T>::real real;
    for (int k = threadIdx.x; k < M; k += blockDim.x) {
        real s, c;
        if (sizeof(real) == 8) {
            double sd, cd;
            sincospi(-2.0 * (double)k / (double)M, &sd, &cd);
            s = (real)sd; c = (real)cd;
        } else {
            float sf, cf;
            sincospif(-2.0f * (float)k / (float)M, &sf, &cf);
            s = (real)sf; c = (real)cf;
        }
        tw[k] = CxOps<T>::mk(c, s);
    }
}

// In-place FFTs of `nseq` bit-reversed sequences; sequence s starts at
// base + s*sstride (complex elements, unit element stride).
template <typename T>
__device__ void fft_stages(T *base, int nseq, int sstride, int logm, const T *tw, bool inverse) {
    const int M = 1 << logm;
    int s = 0;
    if (logm & 1) {
        const int half = M >> 1;
        for (int w = threadIdx.x; w < nseq * half; w += blockDim.x) {
            const int q = w >> (logm - 1), b = w & (half - 1);
            T *a = base + (size_t)q * sstride + 2 * b;
            T u = a[0], v = a[1];
            a[0] = cadd(u, v);
            a[1] = csub(u, v);
        }
        s = 1;
        __syncthreads();
    }
    const int quarter = M >> 2;
    for (; s < logm; s += 2) {
        const int Q = 1 << s, L = Q << 2;
        const int strA = M / (2 * Q), strB = M / L;
        for (int w = threadIdx.x; w < nseq * quarter; w += blockDim.x) {
            const int q = w >> (logm - 2), r = w & (quarter - 1);
            const int grp = r >> s, k = r & (Q - 1);
            T *a = base + (size_t)q * sstride + grp * L + k;
            T x0 = a[0], x1 = a[Q], x2 = a[2 * Q], x3 = a[3 * Q];
            T wA = tw[k * strA], wB = tw[k * strB], wB2 = tw[(k + Q) * strB];
            if (inverse) { wA = cconj(wA); wB = cconj(wB); wB2 = cconj(wB2); }
            T t1 = cmul(wA, x1), t3 = cmul(wA, x3);
            T y0 = cadd(x0, t1), y1 = csub(x0, t1), y2 = cadd(x2, t3), y3 = csub(x2, t3);
            T t2 = cmul(wB, y2), t4 = cmul(wB2, y3);
            a[0] = cadd(y0, t2);
            a[2 * Q] = csub(y0, t2);
            a[Q] = cadd(y1, t4);
            a[3 * Q] = csub(y1, t4);
        }
        __syncthreads();
    }
}

// In-place bit-reversal permutation of `nseq` natural-order sequences.
template <typename T>
__device__ void bitrev_permute(T *base, int nseq, int sstride, int logm) {
    const int M = 1 << logm;
    for (int w = threadIdx.x; w < nseq * M; w += blockDim.x) {
        const int q = w >> logm, i = w & (M - 1);
        const int r = bitrev(i, logm);
        if (i < r) {
            T *a = base + (size_t)q * sstride;
            T t = a[i];
            a[i] = a[r];
            a[r] = t;
        }
    }
    __syncthreads();
}
