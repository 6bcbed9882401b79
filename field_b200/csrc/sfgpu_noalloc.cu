// sfgpu_noalloc.cu -- chain propagation and composition for callers that
// cannot allocate device memory.
//
// Some hosts embed this library where cudaMalloc is not available to them: a
// solver running inside another application's memory pool or allocator, a
// process whose device memory is fully reserved up front, or a caller that
// must not change the device's allocation state while it works.  For them
// sfgpu_chain_phi_noalloc computes what the system path computes for one
// first-order chain molecule -- the forward propagators, the backward
// propagators with the Gf*Gb composition, CorrectDoubleCountG and lnGN -- but
// keeps every intermediate in one fixed array that lives in the library
// itself, so the call allocates nothing.
//
// The array is a file-scope __device__ array of SFGPU_NOALLOC_SCRATCH_DOUBLES
// doubles (16 MiB).  Every GPU that loads the library holds it until the
// process exits.  The caller passes the segment weighting factors and the
// output profiles; this file only ever writes into the scratch array and the
// caller's outputs.
#include <cstring>
#include <mutex>
#include <set>
#include <vector>
#include "sfgpu_kernels.cuh"
#include "sfgpu_system.h"

#define SFGPU_NOALLOC_SCRATCH_DOUBLES (2u * 1024u * 1024u)
#define SFGPU_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) double g_noalloc_scratch[SFGPU_NOALLOC_SCRATCH_DOUBLES];

// Host code cannot use the symbol g_noalloc_scratch as a device address: on
// the host it names a stand-in object, not GPU memory.  The device address
// is looked up once per device (with that device current) and cached here.
// The cache assumes the device's primary context lives as long as the
// process: after a cudaDeviceReset the cached address is stale, and calling
// this entry point again on that device is not supported.
static double *g_scratch_ptr[SFGPU_NOALLOC_MAX_DEVICES];
static std::mutex g_scratch_mu;

// Host copies of the lattice tables (lambda tables and lnGN weights), one per
// distinct table content, kept until the process exits.  The table copy of
// every call reads from here, so its host source outlives the call whatever
// the stream does with the copy later.  Grows by 8*(2*MX + M) bytes per
// distinct lattice a process uses.
static std::set<std::vector<double>> g_table_store;

static int scratch_for_current_device(double **out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) { sfgpu_set_error(e, "cudaGetDevice", __FILE__, __LINE__); return SFGPU_ERR_CUDA; }
    if (dev < 0 || dev >= SFGPU_NOALLOC_MAX_DEVICES) {
        sfgpu_set_error(cudaSuccess, "sfgpu_chain_phi_noalloc: device index beyond the 64 devices it caches",
                        __FILE__, __LINE__);
        return SFGPU_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            sfgpu_set_error(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
            return SFGPU_ERR_CUDA;
        }
        g_scratch_ptr[dev] = static_cast<double *>(p);
    }
    *out = g_scratch_ptr[dev];
    return SFGPU_OK;
}

namespace {

__global__ void noalloc_copy(int M, const double *__restrict__ g, double *__restrict__ out) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < M; r += gridDim.x * blockDim.x) out[r] = g[r];
}

__global__ void noalloc_zero(int M, double *__restrict__ p) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < M; r += gridDim.x * blockDim.x) p[r] = 0.0;
}

// CorrectDoubleCountG: phi /= G where G > 0, else 0 (Lat1DFlat1stO.cpp:294-300)
__global__ void noalloc_divide(int M, const double *__restrict__ G, double *__restrict__ phi) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < M; r += gridDim.x * blockDim.x) {
        double g = G[r];
        phi[r] = (g > 0) ? phi[r] / g : 0.0;
    }
}

__global__ void noalloc_lngn(int nblocks, const double *__restrict__ partial, double *__restrict__ out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double v = 0;
    for (int b = 0; b < nblocks; b++) v += partial[b];
    *out = log(v);
}

}  // namespace

// See include/sfgpu.h for the contract.
extern "C" int sfgpu_chain_phi_noalloc(const sfgpu_lattice_desc *lat, int N, const int *seg_of_s, int nseg,
                                       const double *const *G, double *const *phi, double *lngn, void *stream) {
    if (!lat || !seg_of_s || !G || !phi || !lngn || N < 2 || nseg < 1 || nseg > SFGPU_MAX_SEG)
        return SFGPU_ERR_INVALID;
    if (lat->order != 1) return SFGPU_ERR_UNSUPPORTED;
    for (int s = 0; s < N; s++)
        if (seg_of_s[s] < 0 || seg_of_s[s] >= nseg || !G[seg_of_s[s]] || !phi[seg_of_s[s]]) return SFGPU_ERR_INVALID;
    HostLat H;
    int rc = sfgpu_build_lattice(lat, &H);
    if (rc) return rc;
    const long long M = H.L.M, MX = H.L.Md[0];
    const long long nblocks = std::min<long long>(std::max<long long>((M + sfk::kBlock - 1) / sfk::kBlock, 1), 1024);
    // scratch layout (doubles): lam_m[MX] lam_p[MX] w_gn[M] partial[1024]
    // Gb0[M] Gb1[M] Gf[N*M]
    const long long need = 2 * MX + M + 1024 + 2 * M + (long long)N * M;
    if (need > (long long)SFGPU_NOALLOC_SCRATCH_DOUBLES) return SFGPU_ERR_INVALID;  // chain x lattice too large
    double *scr = nullptr;
    if ((rc = scratch_for_current_device(&scr))) return rc;
    double *lam_m = scr, *lam_p = lam_m + MX, *w_gn = lam_p + MX, *partial = w_gn + M;
    double *gb0 = partial + 1024, *gb1 = gb0 + M, *gf = gb1 + M;
    cudaStream_t st = (cudaStream_t)stream;
    // lattice tables: one plain copy into the scratch array (no allocation),
    // from the process-lifetime host store (lam_m, lam_p, w_gn are adjacent
    // in the scratch layout)
    const double *tables = nullptr;
    {
        std::vector<double> t;
        t.reserve(2 * MX + M);
        t.insert(t.end(), H.lam_m.begin(), H.lam_m.begin() + MX);
        t.insert(t.end(), H.lam_p.begin(), H.lam_p.begin() + MX);
        t.insert(t.end(), H.w_gn.begin(), H.w_gn.begin() + M);
        std::lock_guard<std::mutex> lock(g_scratch_mu);
        tables = g_table_store.insert(std::move(t)).first->data();
    }
    SFGPU_CUDA_TRY(cudaMemcpyAsync(lam_m, tables, sizeof(double) * (2 * MX + M), cudaMemcpyHostToDevice, st));
    DLat L = H.L;
    L.lam_m = lam_m;
    L.lam_p = lam_p;
    L.lamc_m = lam_m;   // contact tables are not read on this path
    L.lamc_p = lam_p;
    const int g = (int)nblocks;
    std::vector<int> used(nseg, 0);
    for (int s = 0; s < N; s++) used[seg_of_s[s]] = 1;
    for (int i = 0; i < nseg; i++)
        if (used[i]) noalloc_zero<<<g, sfk::kBlock, 0, st>>>((int)M, phi[i]);
    // forward: Gf(1) = G_seg(1), Gf(s) = G_seg(s) * stencil(Gf(s-1))
    noalloc_copy<<<g, sfk::kBlock, 0, st>>>((int)M, G[seg_of_s[0]], gf);
    for (int s = 1; s < N; s++)
        sfk::step1<<<g, sfk::kBlock, 0, st>>>(L, gf + (size_t)(s - 1) * M, G[seg_of_s[s]], gf + (size_t)s * M,
                                               nullptr, nullptr, sfk::COMP_NONE);
    // backward with composition (SF_Copol1stO.cpp:1215-1232)
    noalloc_copy<<<g, sfk::kBlock, 0, st>>>((int)M, G[seg_of_s[N - 1]], gb0);
    sfk::connect<<<g, sfk::kBlock, 0, st>>>((int)M, 1, gb0, gf + (size_t)(N - 1) * M, phi[seg_of_s[N - 1]]);
    double *cur = gb0, *nxt = gb1;
    for (int s = N - 2; s >= 0; s--) {
        sfk::step1<<<g, sfk::kBlock, 0, st>>>(L, cur, G[seg_of_s[s]], nxt, gf + (size_t)s * M, phi[seg_of_s[s]],
                                               sfk::COMP_ACC);
        double *t = cur; cur = nxt; nxt = t;
    }
    // lnGN of the end-point distribution, then phi /= G
    sfk::wsum_partial<<<g, sfk::kBlock, 0, st>>>((int)M, 1, cur, w_gn, partial);
    noalloc_lngn<<<1, 1, 0, st>>>(g, partial, lngn);
    for (int i = 0; i < nseg; i++)
        if (used[i]) noalloc_divide<<<g, sfk::kBlock, 0, st>>>((int)M, G[i], phi[i]);
    SFGPU_CUDA_TRY(cudaGetLastError());
    return SFGPU_OK;
}
