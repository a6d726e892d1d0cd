// Register-resident FFTs of power-of-two length M (32..1024) for the fused
// spectral solve (32..256 for the power-of-two boxes, 32..1024 as the inner
// transforms of the Bluestein passes of the other boxes).
//
// One transform is done by TT = M/E1 threads of a warp (a thread group), each
// holding E1 elements in registers.  With n = t + TT*n1 and k = k1 + E1*k2:
//   X[k1 + E1 k2] = sum_t W_TT^{t k2} W_M^{t k1} sum_n1 x[t + TT n1] W_E1^{n1 k1}
// so thread t first takes the E1-point DFT of its own elements, multiplies by
// W_M^{t k1}, the group exchanges these through shared memory (one
// __syncwarp), and each thread takes TT-point DFTs for E1/TT values of k1.
// The small DFTs are unrolled radix-2 decimation-in-frequency with constant
// twiddles (cosines of multiples of 2 pi/16, of 2 pi/32 for E1 = 32).  Input: thread t holds
// x[t + TT*n1] in v[n1].  Output: thread t holds X[t + TT*r + E1*k2] in
// v[r*TT + k2].  Forward sign exp(-2 pi i/M), inverse exp(+2 pi i/M),
// unnormalised.
#pragma once
#include "pfag_fft.cuh"

// cos(2 pi k / 16)
__host__ __device__ constexpr double cos16(int k) {
    return (k & 15) == 0 ? 1.0
         : (k & 15) == 1 ? 0.92387953251128675613
         : (k & 15) == 2 ? 0.70710678118654752440
         : (k & 15) == 3 ? 0.38268343236508977173
         : (k & 15) == 4 ? 0.0
         : (k & 15) == 5 ? -0.38268343236508977173
         : (k & 15) == 6 ? -0.70710678118654752440
         : (k & 15) == 7 ? -0.92387953251128675613
         : (k & 15) == 8 ? -1.0
         : (k & 15) == 9 ? -0.92387953251128675613
         : (k & 15) == 10 ? -0.70710678118654752440
         : (k & 15) == 11 ? -0.38268343236508977173
         : (k & 15) == 12 ? 0.0
         : (k & 15) == 13 ? 0.38268343236508977173
         : (k & 15) == 14 ? 0.70710678118654752440
         : 0.92387953251128675613;
}

// cos(2 pi k / 32): the odd k; the even ones are cos16(k / 2)
__host__ __device__ constexpr double cos32(int k) {
    return (k & 1) == 0 ? cos16((k & 31) >> 1)
         : (k & 31) == 1 ? 0.98078528040323044913
         : (k & 31) == 3 ? 0.83146961230254523708
         : (k & 31) == 5 ? 0.55557023301960222474
         : (k & 31) == 7 ? 0.19509032201612826785
         : (k & 31) == 9 ? -0.19509032201612826785
         : (k & 31) == 11 ? -0.55557023301960222474
         : (k & 31) == 13 ? -0.83146961230254523708
         : (k & 31) == 15 ? -0.98078528040323044913
         : (k & 31) == 17 ? -0.98078528040323044913
         : (k & 31) == 19 ? -0.83146961230254523708
         : (k & 31) == 21 ? -0.55557023301960222474
         : (k & 31) == 23 ? -0.19509032201612826785
         : (k & 31) == 25 ? 0.19509032201612826785
         : (k & 31) == 27 ? 0.55557023301960222474
         : (k & 31) == 29 ? 0.83146961230254523708
         : 0.98078528040323044913;
}

__host__ __device__ constexpr int brev_c(int x, int bits) {
    int r = 0;
    for (int b = 0; b < bits; b++) r |= ((x >> b) & 1) << (bits - 1 - b);
    return r;
}

__host__ __device__ constexpr int ilog2_c(int x) { return x <= 1 ? 0 : 1 + ilog2_c(x >> 1); }

// In-register 32-point DFT, as dft_dif below with twiddles in 32nds of a turn.
template <bool INV, typename T>
__device__ __forceinline__ void dft_dif32(T (&v)[32]) {
    typedef typename CxOps<T>::real real;
#pragma unroll
    for (int span = 16; span >= 1; span >>= 1) {
#pragma unroll
        for (int blk = 0; blk < 32; blk += 2 * span) {
#pragma unroll
            for (int j = 0; j < span; j++) {
                const T a = v[blk + j], b = v[blk + j + span];
                v[blk + j] = cadd(a, b);
                const T d = csub(a, b);
                const int m = j * (32 / (2 * span));   // twiddle W_{2span}^j = exp(-+ 2 pi i m / 32)
                T r;
                if (m == 0) {
                    r = d;
                } else if (m == 8) {
                    if (!INV) { r.x = d.y; r.y = -d.x; } else { r.x = -d.y; r.y = d.x; }
                } else {
                    const real c = (real)cos32(m), sn = (real)cos32(m - 8);
                    T w;
                    w.x = c;
                    w.y = INV ? sn : -sn;
                    r = cmul(d, w);
                }
                v[blk + j + span] = r;
            }
        }
    }
}

// In-register E-point DFT (E in {2,4,8,16,32}); output v[p] = X[bitrev(p)].
template <int E, bool INV, typename T>
__device__ __forceinline__ void dft_dif(T (&v)[E]) {
    typedef typename CxOps<T>::real real;
    if constexpr (E == 32) {
        dft_dif32<INV>(v);
    } else {
#pragma unroll
    for (int span = E / 2; span >= 1; span >>= 1) {
#pragma unroll
        for (int blk = 0; blk < E; blk += 2 * span) {
#pragma unroll
            for (int j = 0; j < span; j++) {
                const T a = v[blk + j], b = v[blk + j + span];
                v[blk + j] = cadd(a, b);
                const T d = csub(a, b);
                const int m = j * (16 / (2 * span));   // twiddle W_{2span}^j = exp(-+ 2 pi i m / 16)
                T r;
                if (m == 0) {
                    r = d;
                } else if (m == 4) {                    // -i (forward), +i (inverse)
                    if (!INV) { r.x = d.y; r.y = -d.x; } else { r.x = -d.y; r.y = d.x; }
                } else {
                    const real c = (real)cos16(m), s = (real)cos16(m - 4);   // sin = cos(x - pi/2)
                    T w;
                    w.x = c;
                    w.y = INV ? s : -s;
                    r = cmul(d, w);
                }
                v[blk + j + span] = r;
            }
        }
    }
    }
}

template <typename T, int M>
struct RegFFT {
    static constexpr int E1 = (M <= 64) ? 8 : (M <= 256 ? 16 : 32);
    static constexpr int TT = M / E1;       // threads per transform
    static constexpr int R2 = E1 / TT;      // second-stage transforms per thread
    static_assert(M >= 32 && M <= 1024 && (M & (M - 1)) == 0, "M must be a power of two in 32..1024");
    static_assert(E1 % TT == 0, "E1 must be a multiple of TT");

    // exchange layout: row k1 of TT entries, columns swizzled by k1
    static __device__ __forceinline__ int sidx(int k1, int t) { return k1 * TT + (t ^ (k1 & (TT - 1))); }

    // sm: M complex of shared memory private to the group; tw[k] = exp(-2 pi i k / M),
    // or with KT the same values laid out as [E1][TT]: tw[k1 TT + t] = exp(-2 pi i t k1 / M)
    // (a warp's twiddle loads then hit distinct banks whatever k1 is)
    template <bool INV, bool KT = false>
    static __device__ __forceinline__ void run(T (&v)[E1], int t, T *sm, const T *tw) {
        dft_dif<E1, INV>(v);
#pragma unroll
        for (int p = 0; p < E1; p++) {
            const int k1 = brev_c(p, ilog2_c(E1));
            T x = v[p];
            if (k1 != 0) {
                T w = KT ? tw[k1 * TT + t] : tw[(t * k1) & (M - 1)];
                if (INV) w = cconj(w);
                x = cmul(x, w);
            }
            sm[sidx(k1, t)] = x;
        }
        __syncwarp();
#pragma unroll
        for (int r = 0; r < R2; r++) {
            const int k1 = t + TT * r;
            T u[TT];
#pragma unroll
            for (int q = 0; q < TT; q++) u[q] = sm[sidx(k1, q)];
            dft_dif<TT, INV>(u);
#pragma unroll
            for (int p = 0; p < TT; p++) v[r * TT + brev_c(p, ilog2_c(TT))] = u[p];
        }
        __syncwarp();
    }

    // the twiddle table in the [E1][TT] layout of run<INV, true>, computed as
    // fft_twiddles computes the natural-order one (the same values)
    static __device__ __forceinline__ void twiddles_kt(T *tw) {
        typedef typename CxOps<T>::real real;
        for (int e = threadIdx.x; e < M; e += blockDim.x) {
            const int k1 = e / TT, t = e - k1 * TT, k = (t * k1) & (M - 1);
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
            tw[e] = CxOps<T>::mk(c, s);
        }
    }

    // natural index of the output held in v[r*TT + k2] by thread t
    static __device__ __forceinline__ int out_index(int t, int r, int k2) { return t + TT * r + E1 * k2; }
    // natural index of the input held in v[n1] by thread t
    static __device__ __forceinline__ int in_index(int t, int n1) { return t + TT * n1; }
};
