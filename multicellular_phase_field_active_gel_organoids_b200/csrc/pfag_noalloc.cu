// Cell areas without any device allocation.
//
// Some callers cannot call cudaMalloc at all: a host program whose device
// memory is already owned by another allocator (an OpenACC data region like
// the reference's, a framework caching allocator, or a fixed pool reserved up
// front for the state arrays), or code on a latency-critical path where the
// implicit device synchronisation of cudaMalloc would stall the pipeline.
// pfag_areas_noalloc gives them the area reduction of sum_s_kernels without a
// context and without allocating: the per-block partial sums live in the
// file-scope array below, which every GPU that loads the library holds for the
// life of the process.
#include "pfag_internal.cuh"
#include <mutex>

namespace {

constexpr int NOALLOC_MAX_CELLS = 1024;   // largest Ntot accepted
constexpr int NOALLOC_BLOCKS = 128;       // partial sums per cell
constexpr int NOALLOC_THREADS = 256;
constexpr int NOALLOC_MAX_DEVICES = 64;

// 1024 cells x 128 partials x 8 bytes = 1 MiB per device.
static __device__ __align__(256) double g_area_partials[NOALLOC_MAX_CELLS * NOALLOC_BLOCKS];

// Device addresses of g_area_partials, resolved once per device (valid for
// the life of the device's primary context: a cudaDeviceReset reloads the
// module, and the entry point must not be called on that device again).
double *g_partials_addr[NOALLOC_MAX_DEVICES] = {};
std::mutex g_setup_mu;

__device__ __forceinline__ double noalloc_block_sum(double v) {
    __shared__ double sh[32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0)
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) r += sh[k];
    return r;
}

template <typename real>
__global__ void kn_area_partials(const real *__restrict__ h, size_t ng, double dx2, double *__restrict__ part) {
    const int n = blockIdx.y;
    const real *p = h + (size_t)n * ng;
    double acc = 0.0;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < ng; k += (size_t)gridDim.x * blockDim.x)
        acc += (double)p[k] * dx2;
    const double r = noalloc_block_sum(acc);
    if (threadIdx.x == 0) part[(size_t)n * gridDim.x + blockIdx.x] = r;
}

__global__ void kn_area_final(const double *__restrict__ part, int nblk, int ncells, double alpha, double s0,
                              double *__restrict__ s, double *__restrict__ f0) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= ncells) return;
    double a = 0.0;
    for (int b = 0; b < nblk; b++) a += part[(size_t)n * nblk + b];
    s[n] = a;
    f0[n] = alpha * (s0 - a);
}

// Resolve the scratch array's device address for the current device.
int partials_for_current_device(double **out) {
    int dev = 0;
    PFAG_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) {
        pfag_set_error("pfag_areas_noalloc: device index %d beyond %d", dev, NOALLOC_MAX_DEVICES);
        return PFAG_E_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_partials_addr[dev]) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_area_partials);
        if (e != cudaSuccess || !ptr) {
            pfag_set_error("pfag_areas_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
            return PFAG_E_CUDA;
        }
        g_partials_addr[dev] = (double *)ptr;
    }
    *out = g_partials_addr[dev];
    return PFAG_OK;
}

}  // namespace

extern "C" int pfag_areas_noalloc(const void *hfunc_cell, int precision, int Ntot, int N_s, double dx, double alpha,
                                  double s0, double *s, double *f0, void *stream) {
    if (!hfunc_cell || !s || !f0) { pfag_set_error("pfag_areas_noalloc: null pointer"); return PFAG_E_ARG; }
    if (precision != 32 && precision != 64) { pfag_set_error("pfag_areas_noalloc: precision must be 32 or 64"); return PFAG_E_ARG; }
    if (N_s < 1) { pfag_set_error("pfag_areas_noalloc: N_s must be positive"); return PFAG_E_ARG; }
    if (Ntot < 1 || Ntot > NOALLOC_MAX_CELLS) {
        pfag_set_error("pfag_areas_noalloc: Ntot=%d outside [1, %d], the size of its static scratch", Ntot,
                       NOALLOC_MAX_CELLS);
        return PFAG_E_ARG;
    }
    double *part = nullptr;
    PFAG_TRY(partials_for_current_device(&part));
    cudaStream_t st = (cudaStream_t)stream;
    const size_t ng = (size_t)N_s * N_s;
    const double dx2 = dx * dx;
    if (precision == 64)
        kn_area_partials<double><<<dim3(NOALLOC_BLOCKS, Ntot), NOALLOC_THREADS, 0, st>>>(
            (const double *)hfunc_cell, ng, dx2, part);
    else
        kn_area_partials<float><<<dim3(NOALLOC_BLOCKS, Ntot), NOALLOC_THREADS, 0, st>>>(
            (const float *)hfunc_cell, ng, dx2, part);
    PFAG_CUDA_CHECK(cudaGetLastError());
    kn_area_final<<<(Ntot + 127) / 128, 128, 0, st>>>(part, NOALLOC_BLOCKS, Ntot, alpha, s0, s, f0);
    PFAG_CUDA_CHECK(cudaGetLastError());
    return PFAG_OK;
}
