// Seeded synthetic organoids generated on the device, for workloads too large
// to build on the host (the batched sweep of many organoids up to 1024^2 with
// up to 128 cells each): the same fields as the host generator of the
// configurations, phi_n = 0.5 (1 - tanh((r_n - R)/2)) around each centre,
// rho_n = 1 where 0.05 < phi_n < 0.95 times (1 + 0.01 u), lumen 0 and ECM
// 0.5 (1 + tanh((r - r_env)/2)) about the centre of the cells, with u uniform
// in [-1, 1) from a counter-based hash of (seed, site) instead of the host
// generator's stream, then the set-up pfag_upload does.
#include "pfag_internal.cuh"

namespace {

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

template <typename real>
__global__ void ks_cells(real *__restrict__ phi, real *__restrict__ rho, const double2 *__restrict__ ctr, int Ntot,
                         int N, double R, unsigned long long seed) {
    const size_t tot = (size_t)Ntot * N * N;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
        const int n = (int)(e / ((size_t)N * N));
        const int rem = (int)(e - (size_t)n * N * N);
        const int i = rem / N, j = rem - i * N;
        const double di = (double)i - ctr[n].x, dj = (double)j - ctr[n].y;
        const double f = 0.5 * (1.0 - tanh((sqrt(di * di + dj * dj) - R) / 2.0));
        const unsigned long long h = splitmix64(seed * 0x100000001B3ull + (unsigned long long)e);
        const double u = 2.0 * ((double)(h >> 11) * 0x1.0p-53) - 1.0;
        phi[e] = (real)f;
        rho[e] = (real)((f > 0.05 && f < 0.95) ? 1.0 * (1.0 + 0.01 * u) : 0.0);
    }
}

template <typename real>
__global__ void ks_shared(real *__restrict__ lum, real *__restrict__ ecm, int N, double ci, double cj, double renv) {
    const size_t tot = (size_t)N * N;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(e / N), j = (int)(e - (size_t)i * N);
        const double di = (double)i - ci, dj = (double)j - cj;
        lum[e] = (real)0.0;
        ecm[e] = (real)(0.5 * (1.0 + tanh((sqrt(di * di + dj * dj) - renv) / 2.0)));
    }
}

}  // namespace

extern "C" int pfag_seed_organoid(pfag_ctx *c, const double *centres, double radius, double env_radius,
                                  unsigned long long seed) {
    if (!c || !centres || !(radius > 0.0) || !(env_radius > 0.0)) {
        pfag_set_error("pfag_seed_organoid: bad arguments");
        return PFAG_E_ARG;
    }
    double2 *d_ctr = nullptr;
    PFAG_CUDA_CHECK(cudaMalloc(&d_ctr, sizeof(double2) * c->Ntot));
    int rc = PFAG_OK;
    double ci = 0.0, cj = 0.0;
    for (int n = 0; n < c->Ntot; n++) { ci += centres[2 * n]; cj += centres[2 * n + 1]; }
    ci /= c->Ntot;
    cj /= c->Ntot;
    if (cudaMemcpyAsync(d_ctr, centres, sizeof(double2) * c->Ntot, cudaMemcpyHostToDevice, c->stream) != cudaSuccess) {
        pfag_set_error("pfag_seed_organoid: copy of the centres failed");
        rc = PFAG_E_CUDA;
    } else {
        if (c->prec == 64) {
            ks_cells<double><<<1184, 256, 0, c->stream>>>((double *)c->phi, (double *)c->rho, d_ctr, c->Ntot, c->N,
                                                           radius, seed);
            ks_shared<double><<<296, 256, 0, c->stream>>>((double *)c->lum, (double *)c->ecm, c->N, ci, cj,
                                                          env_radius);
        } else {
            ks_cells<float><<<1184, 256, 0, c->stream>>>((float *)c->phi, (float *)c->rho, d_ctr, c->Ntot, c->N,
                                                         radius, seed);
            ks_shared<float><<<296, 256, 0, c->stream>>>((float *)c->lum, (float *)c->ecm, c->N, ci, cj,
                                                         env_radius);
        }
        if (cudaGetLastError() != cudaSuccess) { pfag_set_error("pfag_seed_organoid: launch failed"); rc = PFAG_E_CUDA; }
    }
    if (rc == PFAG_OK) rc = pfag_after_upload(c);
    cudaStreamSynchronize(c->stream);
    cudaFree(d_ctr);
    return rc;
}
