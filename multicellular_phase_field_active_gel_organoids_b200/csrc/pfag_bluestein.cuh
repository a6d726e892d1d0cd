// Spectral solve on boxes whose size M is not a power of two (the reference's
// default zone_size 200 gives M = 398 = 2 x 199), with hand-written
// transforms: Bluestein's algorithm over the register-resident power-of-two
// FFTs of pfag_regfft.cuh.
//
// Bluestein.  With nk = (n^2 + k^2 - (k-n)^2)/2 the length-M DFT
//   X_k = sum_n x_n exp(-+2 pi i nk/M)
//       = conj(c_k) sum_n (x_n conj(c_n)) c_{k-n},   c_m = exp(+i pi m^2/M)
// (forward; the inverse swaps c and conj(c)), a linear convolution of length
// 2M-1 done as a circular one of length L = next power of two >= 2M-1 (at
// least 32): FFT_L of the chirped input, times the spectrum of the chirp
// kernel (precomputed, 1/L folded in), inverse FFT_L, chirp again.  M <= 512
// (L <= 1024).
//
// Spectral derivatives.  update_fft_rho's divergence (rho_functions.cpp:
// 213-251) is separable (the transforms along the other axis cancel):
// dt kfac Re(IFFT_M(-i k' FFT_M(F)))/M along one axis, k' the wrapped
// wavenumber with the Nyquist bin zeroed (the Re() of the odd multiplier).
// That is a circular convolution of length M with the real, odd kernel
//   h_d = (dt kfac / M) 2 sum_{k=1}^{M/2-1} k sin(2 pi d k / M),
// done here as a circular convolution of length L (the same padding as
// above) with a precomputed spectrum: two FFT_L per sequence instead of the
// four of a forward and an inverse Bluestein transform.  Two real sequences
// share one complex one (z = a + i b: the kernel is real, so the results come
// back in the real and imaginary parts).
//
// Tables (per context, computed once on the device in FP64 with compensated
// sums, stored in the context's precision): tw[k] = exp(-2 pi i k/L),
// cw[n] = c_n (n^2 reduced mod 2M exactly), wf = FFT_L(c~)/L with c~ the
// symmetric chirp kernel, hdi = Im(FFT_L(h~))/L (the spectrum of the odd
// kernel is imaginary).
#pragma once
#include "pfag_regfft.cuh"

// Error-compensated FP64 accumulation (Neumaier): the tables' sums of up to
// 2M-1 terms keep their rounding near one ulp of the result.
struct KSum {
    double s = 0.0, c = 0.0;
    __device__ __forceinline__ void add(double x) {
        const double t = s + x;
        if (fabs(s) >= fabs(x)) c += (s - t) + x;
        else c += (x - t) + s;
        s = t;
    }
    __device__ __forceinline__ double get() const { return s + c; }
};

// pass 1: tw, cw and the derivative kernel h (length M)
template <typename cx>
__global__ void kbl_tables1(int M, int L, double dtk, cx *__restrict__ tw, cx *__restrict__ cw,
                            double *__restrict__ h) {
    typedef typename CxOps<cx>::real real;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < L) {
        double s, c;
        sincospi(-2.0 * (double)e / (double)L, &s, &c);
        tw[e] = CxOps<cx>::mk((real)c, (real)s);
    }
    if (e < M) {
        const long r = ((long)e * e) % (2L * M);
        double s, c;
        sincospi((double)r / (double)M, &s, &c);
        cw[e] = CxOps<cx>::mk((real)c, (real)s);
        KSum acc;
        for (int k = 1; k < M / 2; k++) acc.add((double)k * sinpi(2.0 * (double)(((long)e * k) % M) / (double)M));
        h[e] = 2.0 * dtk / (double)M * acc.get();
    }
}

// pass 2: wf and hdi (length L)
template <typename cx>
__global__ void kbl_tables2(int M, int L, const double *__restrict__ h, cx *__restrict__ wf,
                            typename CxOps<cx>::real *__restrict__ hdi) {
    typedef typename CxOps<cx>::real real;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= L) return;
    // wf[q] = (1/L) (c_0 + 2 sum_{m=1}^{M-1} c_m cos(2 pi m q / L))
    KSum re, im, hs;
    re.add(1.0);
    for (int m = 1; m < M; m++) {
        const long r = ((long)m * m) % (2L * M);
        double s, c;
        sincospi((double)r / (double)M, &s, &c);
        const double cq = 2.0 * cospi(2.0 * (double)(((long)m * q) % L) / (double)L);
        re.add(c * cq);
        im.add(s * cq);
        // hdi[q] = -(2/L) sum_{d=1}^{M-1} h_d sin(2 pi d q / L)
        hs.add(h[m] * sinpi(2.0 * (double)(((long)m * q) % L) / (double)L));
    }
    wf[q] = CxOps<cx>::mk((real)(re.get() / (double)L), (real)(im.get() / (double)L));
    hdi[q] = (real)(-2.0 * hs.get() / (double)L);
}

template <typename cx>
struct BlueTabs {
    const cx *tw, *cw, *wf;
    const typename CxOps<cx>::real *hdi;
};

template <typename cx, int L>
struct Blue {
    typedef RegFFT<cx, L> RF;
    typedef typename CxOps<cx>::real real;
    static constexpr int TT = RF::TT, E1 = RF::E1, R2 = RF::R2;

    // index held in register q of thread t (the register FFT's input order)
    static __device__ __forceinline__ int idx(int t, int q) { return t + TT * q; }

    // registers from the register FFT's output order (register r*TT + k2 holds
    // index t + TT (r + R2 k2)) to its input order
    static __device__ __forceinline__ void to_in(cx (&v)[E1]) {
        if constexpr (R2 > 1) {
            cx w[E1];
#pragma unroll
            for (int p = 0; p < E1; p++) w[(p / TT) + R2 * (p % TT)] = v[p];
#pragma unroll
            for (int p = 0; p < E1; p++) v[p] = w[p];
        }
    }

    // length-M DFT (forward exp(-2 pi i nk/M), INV exp(+...)), unnormalised, of
    // the sequence in v (input order; entries at index >= M are ignored);
    // the result in input order, valid below M.  sm: L complex of the
    // group's own shared memory; tw: the table in shared memory.
    template <bool INV>
    static __device__ __forceinline__ void dft(cx (&v)[E1], int t, int M, cx *sm, const cx *tw,
                                               const BlueTabs<cx> &tb) {
#pragma unroll
        for (int q = 0; q < E1; q++) {
            const int n = idx(t, q);
            if (n < M) {
                cx c = tb.cw[n];
                if (!INV) c = cconj(c);
                v[q] = cmul(v[q], c);
            } else {
                v[q] = CxOps<cx>::mk((real)0.0, (real)0.0);
            }
        }
        RF::template run<false, true>(v, t, sm, tw);
#pragma unroll
        for (int p = 0; p < E1; p++) {
            cx w = tb.wf[RF::out_index(t, p / TT, p % TT)];
            if (INV) w = cconj(w);
            v[p] = cmul(v[p], w);
        }
        to_in(v);
        RF::template run<true, true>(v, t, sm, tw);
        to_in(v);
#pragma unroll
        for (int q = 0; q < E1; q++) {
            const int n = idx(t, q);
            if (n < M) {
                cx c = tb.cw[n];
                if (!INV) c = cconj(c);
                v[q] = cmul(v[q], c);
            }
        }
    }

    // circular convolution of length M with the derivative kernel h (v in
    // input order, entries >= M ignored; result in input order, valid below M)
    static __device__ __forceinline__ void deriv(cx (&v)[E1], int t, int M, cx *sm, const cx *tw,
                                                 const BlueTabs<cx> &tb) {
#pragma unroll
        for (int q = 0; q < E1; q++)
            if (idx(t, q) >= M) v[q] = CxOps<cx>::mk((real)0.0, (real)0.0);
        RF::template run<false, true>(v, t, sm, tw);
#pragma unroll
        for (int p = 0; p < E1; p++) {
            const real hi = tb.hdi[RF::out_index(t, p / TT, p % TT)];   // times i hi
            const cx x = v[p];
            v[p] = CxOps<cx>::mk(-x.y * hi, x.x * hi);
        }
        to_in(v);
        RF::template run<true, true>(v, t, sm, tw);
        to_in(v);
    }
};

// launch geometry of the Bluestein passes for a transform length L
template <typename real, int L> struct BlueGeom {
    static constexpr int TT = RegFFT<float2, L>::TT;
    static constexpr int THREADS = (sizeof(real) == 8 && L >= 512) ? 128 : 256;
    static constexpr int GPB = THREADS / TT;     // thread groups per block
    // FP32: two blocks per SM (at most 128 registers a thread)
    static constexpr int MINB = sizeof(real) == 4 ? 2 : 1;
};

// global -> shared copy of one 8- or 16-byte element, asynchronous (cp.async);
// blue_cp_wait waits for the calling thread's copies
template <typename T>
__device__ __forceinline__ void blue_cp(T *dst, const T *src) {
    static_assert(sizeof(T) == 8 || sizeof(T) == 16, "element size");
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d), "l"(src), "n"(sizeof(T)) : "memory");
}
__device__ __forceinline__ void blue_cp_wait() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// the twiddles of the length-L register FFT in its [E1][TT] layout, from the
// natural-order table g[k] = exp(-2 pi i k / L)
template <typename cx, int L>
__device__ __forceinline__ void load_tw(cx *tw, const cx *__restrict__ g) {
    constexpr int TT = RegFFT<cx, L>::TT;
    for (int e = threadIdx.x; e < L; e += blockDim.x) {
        const int k1 = e / TT, t = e - k1 * TT;
        tw[e] = g[(t * k1) & (L - 1)];
    }
}

// The kernels' copy of the tables in shared memory at `base` (after the
// twiddles): the chirp (M) and its kernel's spectrum (L) when `chirp`, the
// derivative kernel's spectrum (L reals) when `deriv`; returns the table set
// the transforms read and the first byte after it.
template <typename cx, int L>
__device__ __forceinline__ BlueTabs<cx> stage_tabs(const BlueTabs<cx> &g, unsigned char *base, int M, bool chirp,
                                                   bool deriv, unsigned char **end) {
    typedef typename CxOps<cx>::real real;
    BlueTabs<cx> s = g;
    cx *p = reinterpret_cast<cx *>(base);
    if (chirp) {
        cx *wf = p, *cw = p + L;           // wf [L], then cw [M] (rounded up to even)
        for (int e = threadIdx.x; e < L; e += blockDim.x) {
            wf[e] = g.wf[e];
            if (e < M) cw[e] = g.cw[e];
        }
        s.wf = wf;
        s.cw = cw;
        p += L + ((M + 1) & ~1);
    }
    real *h = reinterpret_cast<real *>(p);
    if (deriv) {
        for (int e = threadIdx.x; e < L; e += blockDim.x) h[e] = g.hdi[e];
        s.hdi = h;
        h += L;
    }
    *end = reinterpret_cast<unsigned char *>(h);
    return s;
}

// bytes stage_tabs takes
template <typename cx, int L>
constexpr size_t tabs_bytes(int M, bool chirp, bool deriv) {
    return (chirp ? ((size_t)L + (size_t)((M + 1) & ~1)) * sizeof(cx) : 0) +
           (deriv ? (size_t)L * sizeof(typename CxOps<cx>::real) : 0);
}

// Pass A' (rows, forward): tasks [0, M) of a cell transform row i of Y1
// (pi_xx + i pi_yy) in place; tasks [M, 3M/2) transform rows 2p, 2p+1 of the
// real plane Y2r (pi_xy) packed as one complex row and split into the two
// rows' half spectra (k = 0 .. M/2, the layout [M][M/2+1] of Hs).
template <typename real, int L>
__global__ void __launch_bounds__(BlueGeom<real, L>::THREADS, BlueGeom<real, L>::MINB)
kbl_rowsA(typename Cplx<real>::type *__restrict__ Y1, const real *__restrict__ Y2r,
          typename Cplx<real>::type *__restrict__ Hs, int M, int Ntot, BlueTabs<typename Cplx<real>::type> tb) {
    typedef typename Cplx<real>::type cx;
    typedef Blue<cx, L> B;
    constexpr int TT = B::TT, E1 = B::E1, GPB = BlueGeom<real, L>::GPB;
    extern __shared__ unsigned char smraw[];
    cx *tw = (cx *)smraw;
    const int t = threadIdx.x % TT, g = threadIdx.x / TT;
    cx *sm = tw + L + (size_t)g * L;
    load_tw<cx, L>(tw, tb.tw);
    unsigned char *end;
    const BlueTabs<cx> st = stage_tabs<cx, L>(tb, reinterpret_cast<unsigned char *>(tw + L + (size_t)GPB * L), M,
                                              true, false, &end);
    __syncthreads();
    const int per = M + M / 2, H = M / 2 + 1;
    const long total = (long)Ntot * per;
    for (long base = (long)blockIdx.x * GPB; base < total; base += (long)gridDim.x * GPB) {
        const long task = base + g;
        const bool live = task < total;
        const int n = live ? (int)(task / per) : 0, w = live ? (int)(task % per) : 0;
        // every group of a warp runs the same sequence of warp barriers,
        // whichever kind of task it has
        const bool pair = w >= M;
        const int a = pair ? 2 * (w - M) : w;
        cx v[E1];
        if (!pair) {
            const cx *src = Y1 + ((size_t)n * M + a) * M;
#pragma unroll
            for (int q = 0; q < E1; q++) {
                const int j = B::idx(t, q);
                v[q] = (live && j < M) ? src[j] : CxOps<cx>::mk((real)0.0, (real)0.0);
            }
        } else {
            const real *ra = Y2r + ((size_t)n * M + a) * M;
#pragma unroll
            for (int q = 0; q < E1; q++) {
                const int j = B::idx(t, q);
                v[q] = (live && j < M) ? CxOps<cx>::mk(ra[j], ra[j + M]) : CxOps<cx>::mk((real)0.0, (real)0.0);
            }
        }
        B::template dft<false>(v, t, M, sm, tw, st);
        if (!pair) {
            if (live) {
                cx *dst = Y1 + ((size_t)n * M + a) * M;
#pragma unroll
                for (int q = 0; q < E1; q++) {
                    const int j = B::idx(t, q);
                    if (j < M) dst[j] = v[q];
                }
            }
        } else {
#pragma unroll
            for (int q = 0; q < E1; q++) {
                const int j = B::idx(t, q);
                if (j < M) sm[j] = v[q];
            }
        }
        __syncwarp();
        if (pair && live) {
            cx *ha = Hs + ((size_t)n * M + a) * H, *hb = ha + H;
#pragma unroll
            for (int q = 0; q < E1; q++) {
                const int k = B::idx(t, q);
                if (k < H) {
                    const cx zk = sm[k], zm = sm[(M - k) % M];
                    ha[k] = CxOps<cx>::mk((real)0.5 * (zk.x + zm.x), (real)0.5 * (zk.y - zm.y));
                    hb[k] = CxOps<cx>::mk((real)0.5 * (zk.y + zm.y), (real)0.5 * (zm.x - zk.x));
                }
            }
        }
        __syncwarp();
    }
}

// One set of columns for the column passes: cell n's columns are
// base + n * cell_stride + c (row stride `stride`), c < ncol.
template <typename cx>
struct ColSet {
    cx *base;
    long cell_stride;
    int stride, ncol, nblk;    // nblk: column blocks per cell
};

// Column transforms (forward, or inverse with INV) of up to two column sets;
// a block stages GPB columns of one cell in shared memory (one slot of L + 1
// complex per column, which is also the exchange scratch of its transform;
// all of a thread's copies in flight at once), transforms them and stores
// them back.
template <typename real, int L, bool INV>
__global__ void __launch_bounds__(BlueGeom<real, L>::THREADS, BlueGeom<real, L>::MINB)
kbl_cols(ColSet<typename Cplx<real>::type> s0, ColSet<typename Cplx<real>::type> s1, int M, int Ntot,
         BlueTabs<typename Cplx<real>::type> tb) {
    typedef typename Cplx<real>::type cx;
    typedef Blue<cx, L> B;
    constexpr int TT = B::TT, E1 = B::E1, GPB = BlueGeom<real, L>::GPB, S = L + 1;
    extern __shared__ unsigned char smraw[];
    cx *tw = (cx *)smraw;
    cx *Z = tw + L;                       // [GPB][S]
    const int t = threadIdx.x % TT, g = threadIdx.x / TT;
    load_tw<cx, L>(tw, tb.tw);
    unsigned char *end;
    const BlueTabs<cx> st = stage_tabs<cx, L>(tb, reinterpret_cast<unsigned char *>(Z + (size_t)GPB * S), M, true,
                                              false, &end);
    const long per = (long)s0.nblk + s1.nblk;
    const long total = (long)Ntot * per;
    for (long task = blockIdx.x; task < total; task += gridDim.x) {
        const int n = (int)(task / per), b = (int)(task % per);
        const ColSet<cx> &cs = (b < s0.nblk) ? s0 : s1;
        const int c0 = ((b < s0.nblk) ? b : b - s0.nblk) * GPB;
        const int nc = min(GPB, cs.ncol - c0);
        cx *src = cs.base + (size_t)n * cs.cell_stride + c0;
        __syncthreads();                  // the previous task's stores have read Z (and the tables are staged)
        for (int e = threadIdx.x; e < M * nc; e += blockDim.x) {
            const int i = e / nc, c = e - i * nc;
            blue_cp(Z + (size_t)c * S + i, src + (size_t)i * cs.stride + c);
        }
        blue_cp_wait();
        __syncthreads();
        {
            cx *col = Z + (size_t)g * S;
            cx v[E1];
#pragma unroll
            for (int q = 0; q < E1; q++) {
                const int i = B::idx(t, q);
                v[q] = (g < nc && i < M) ? col[i] : CxOps<cx>::mk((real)0.0, (real)0.0);
            }
            __syncwarp();
            B::template dft<INV>(v, t, M, col, tw, st);
#pragma unroll
            for (int q = 0; q < E1; q++) {
                const int i = B::idx(t, q);
                if (i < M) col[i] = v[q];
            }
        }
        __syncthreads();
        for (int e = threadIdx.x; e < M * nc; e += blockDim.x) {
            const int i = e / nc, c = e - i * nc;
            src[(size_t)i * cs.stride + c] = Z[(size_t)c * S + i];
        }
    }
}

// Pass D' (rows, inverse) in two kernels, so that each holds one transform's
// state (184 and 68 bytes of spills at 128 registers, against 592 for both
// transforms in one kernel): kbl_rowsD1 takes the inverse row transform of one
// row of Y1 (M^2 (vx + i vy)) and stores Fx = rho vx / M^2 into plane 0 and
// Fy = rho vy / M^2 into plane 1 of X (load_fft_rho_v, rho_functions.cpp:
// 213-284); kbl_rowsD2 differentiates Fy along the row, two rows as one
// complex sequence, and overwrites plane 1 with dt R + that row term (dt kfac
// folded in; the row half of update_fft_rho).
template <typename real, int L>
__global__ void __launch_bounds__(BlueGeom<real, L>::THREADS, BlueGeom<real, L>::MINB)
kbl_rowsD1(const typename Cplx<real>::type *__restrict__ Y1, real *__restrict__ X, const real *__restrict__ rho,
           const int *__restrict__ xc, const int *__restrict__ yc, int N, int z, int M, int Ntot,
           BlueTabs<typename Cplx<real>::type> tb, real *__restrict__ vdx, real *__restrict__ vdy) {
    typedef typename Cplx<real>::type cx;
    typedef Blue<cx, L> B;
    constexpr int TT = B::TT, E1 = B::E1, GPB = BlueGeom<real, L>::GPB;
    extern __shared__ unsigned char smraw[];
    cx *tw = (cx *)smraw;
    const int t = threadIdx.x % TT, g = threadIdx.x / TT;
    cx *sm = tw + L + (size_t)g * L;
    load_tw<cx, L>(tw, tb.tw);
    unsigned char *end;
    const BlueTabs<cx> st = stage_tabs<cx, L>(tb, reinterpret_cast<unsigned char *>(tw + L + (size_t)GPB * L), M,
                                              true, false, &end);
    __syncthreads();
    const long total = (long)Ntot * M;
    const real mm = (real)((double)M * (double)M);
    real *Fy = X + (size_t)Ntot * M * M;
    for (long base = (long)blockIdx.x * GPB; base < total; base += (long)gridDim.x * GPB) {
        const long task = base + g;
        const bool live = task < total;
        const int n = live ? (int)(task / M) : 0, i = live ? (int)(task % M) : 0;
        const int bi = xc[n] - z + 1, bj = yc[n] - z + 1;
        const size_t rowo = ((size_t)n * M + i) * M;
        cx v[E1];
#pragma unroll
        for (int q = 0; q < E1; q++) {
            const int j = B::idx(t, q);
            v[q] = (live && j < M) ? Y1[rowo + j] : CxOps<cx>::mk((real)0.0, (real)0.0);
        }
        B::template dft<true>(v, t, M, sm, tw, st);
        if (live) {
            const real *rh = rho + (size_t)n * N * N + (size_t)(bi + i) * N + bj;
#pragma unroll
            for (int q = 0; q < E1; q++) {
                const int j = B::idx(t, q);
                if (j < M) {
                    const real rr = rh[j];
                    X[rowo + j] = rr * v[q].x / mm;
                    Fy[rowo + j] = rr * v[q].y / mm;
                    if (vdx) { vdx[rowo + j] = v[q].x / mm; vdy[rowo + j] = v[q].y / mm; }
                }
            }
        }
    }
}

template <typename real, int L>
__global__ void __launch_bounds__(BlueGeom<real, L>::THREADS, BlueGeom<real, L>::MINB)
kbl_rowsD2(real *__restrict__ X, const real *__restrict__ Rb, double dt, int M, int Ntot,
           BlueTabs<typename Cplx<real>::type> tb) {
    typedef typename Cplx<real>::type cx;
    typedef Blue<cx, L> B;
    constexpr int TT = B::TT, E1 = B::E1, GPB = BlueGeom<real, L>::GPB;
    extern __shared__ unsigned char smraw[];
    cx *tw = (cx *)smraw;
    const int t = threadIdx.x % TT, g = threadIdx.x / TT;
    cx *sm = tw + L + (size_t)g * L;
    load_tw<cx, L>(tw, tb.tw);
    unsigned char *end;
    const BlueTabs<cx> st = stage_tabs<cx, L>(tb, reinterpret_cast<unsigned char *>(tw + L + (size_t)GPB * L), M,
                                              false, true, &end);
    __syncthreads();
    const int per = M / 2;
    const long total = (long)Ntot * per;
    const real dtr = (real)dt;
    for (long base = (long)blockIdx.x * GPB; base < total; base += (long)gridDim.x * GPB) {
        const long task = base + g;
        const bool live = task < total;
        const int n = live ? (int)(task / per) : 0, i0 = live ? 2 * (int)(task % per) : 0;
        real *d0 = X + (size_t)Ntot * M * M + ((size_t)n * M + i0) * M;     // Fy rows i0, i0 + 1
        cx v[E1];
#pragma unroll
        for (int q = 0; q < E1; q++) {
            const int j = B::idx(t, q);
            v[q] = (live && j < M) ? CxOps<cx>::mk(d0[j], d0[M + j]) : CxOps<cx>::mk((real)0.0, (real)0.0);
        }
        B::deriv(v, t, M, sm, tw, st);
        if (live) {
            const real *r0 = Rb + ((size_t)n * M + i0) * M;
#pragma unroll
            for (int q = 0; q < E1; q++) {
                const int j = B::idx(t, q);
                if (j < M) {
                    d0[j] = dtr * r0[j] + v[q].x;
                    d0[M + j] = dtr * r0[M + j] + v[q].y;
                }
            }
        }
    }
}

// Pass E' (columns): two real columns of Fx per complex sequence, the
// derivative along the column (dt kfac folded in) stored over Fx in plane 0.
template <typename real, int L>
__global__ void __launch_bounds__(BlueGeom<real, L>::THREADS, BlueGeom<real, L>::MINB)
kbl_colsE(real *__restrict__ X, int M, int Ntot, BlueTabs<typename Cplx<real>::type> tb) {
    typedef typename Cplx<real>::type cx;
    typedef Blue<cx, L> B;
    constexpr int TT = B::TT, E1 = B::E1, GPB = BlueGeom<real, L>::GPB, S = L + 1;
    extern __shared__ unsigned char smraw[];
    cx *tw = (cx *)smraw;
    cx *Z = tw + L;                       // [GPB][S]: column pairs
    const int t = threadIdx.x % TT, g = threadIdx.x / TT;
    load_tw<cx, L>(tw, tb.tw);
    unsigned char *end;
    const BlueTabs<cx> st = stage_tabs<cx, L>(tb, reinterpret_cast<unsigned char *>(Z + (size_t)GPB * S), M, false,
                                              true, &end);
    const int nblk = (M / 2 + GPB - 1) / GPB;
    const long total = (long)Ntot * nblk;
    for (long task = blockIdx.x; task < total; task += gridDim.x) {
        const int n = (int)(task / nblk), b = (int)(task % nblk);
        const int p0 = b * GPB, np = min(GPB, M / 2 - p0);     // column pairs 2p, 2p+1
        cx *fx = reinterpret_cast<cx *>(X + (size_t)n * M * M);  // row i, pair p at fx[i M/2 + p]
        __syncthreads();
        for (int e = threadIdx.x; e < M * np; e += blockDim.x) {
            const int i = e / np, p = e - i * np;
            blue_cp(Z + (size_t)p * S + i, fx + (size_t)i * (M / 2) + p0 + p);
        }
        blue_cp_wait();
        __syncthreads();
        {
            cx *col = Z + (size_t)g * S;
            cx v[E1];
#pragma unroll
            for (int q = 0; q < E1; q++) {
                const int i = B::idx(t, q);
                v[q] = (g < np && i < M) ? col[i] : CxOps<cx>::mk((real)0.0, (real)0.0);
            }
            __syncwarp();
            B::deriv(v, t, M, col, tw, st);
#pragma unroll
            for (int q = 0; q < E1; q++) {
                const int i = B::idx(t, q);
                if (i < M) col[i] = v[q];
            }
        }
        __syncthreads();
        for (int e = threadIdx.x; e < M * np; e += blockDim.x) {
            const int i = e / np, p = e - i * np;
            fx[(size_t)i * (M / 2) + p0 + p] = Z[(size_t)p * S + i];
        }
    }
}

// The new rho on every box: rho + (dt R + row term) + column term
// (update_fft_rho and copy_to_rhon, rho_functions.cpp:213-265, by linearity;
// planes 1 and 0 of X)
template <typename real>
__global__ void kbl_rho(const real *__restrict__ X, real *__restrict__ rho, const int *__restrict__ xc,
                        const int *__restrict__ yc, int N, int z, int M, int Ntot) {
    const int n = blockIdx.y;
    const int bi = xc[n] - z + 1, bj = yc[n] - z + 1;
    const real *dxc = X + (size_t)n * M * M, *q = X + (size_t)Ntot * M * M + (size_t)n * M * M;
    real *rc = rho + (size_t)n * N * N;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < M * M; e += gridDim.x * blockDim.x) {
        const int i = e / M, j = e - i * M;
        real &ro = rc[(size_t)(bi + i) * N + bj + j];
        ro = ro + (q[e] + dxc[e]);
    }
}
