// sfgpu_adjoint.cu -- J(x)^T w for first-order systems by a reverse sweep
// (the transpose of the tangent in sfgpu_tangent.cu), and a limited-memory
// BFGS iteration on |f|^2 / 2 whose gradient J^T f comes from it.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#include "sfgpu_adjoint.cuh"
#include "sfgpu_system.h"

using namespace sfk;
using namespace sfa;

static int grid_a(long n) {
    long b = (n + kBlock - 1) / kBlock;
    return (int)std::max(1L, std::min(b, 148L * 16));
}
static int grid_rows_a(const DLat &L) {
    long threads = (L.grad == 1) ? (long)(L.Md[0] - 2) : 32L * lat_nrows(L);
    long b = (threads + kBlock - 1) / kBlock;
    return (int)std::max(1L, std::min(b, 148L * 32));
}

namespace {

// adjoint scalars per molecule
struct AdjScal {
    double cbar;        // cotangent of the normalisation C
    double phibbar;     // cotangent of phibulk (accumulated from bulk terms and the solvent)
    double lngnbar;     // cotangent of lnGN
    double qbar;        // cotangent of Q = exp(lnGN)
};

__global__ void adj_bulk(BulkParam b, ChiTable ct, const double *__restrict__ chibbar, AdjScal *__restrict__ as) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double phibbar_seg[SFGPU_MAX_SEG];
    for (int j = 0; j < b.nseg; j++) {
        double v = 0;
        for (int c = 0; c < b.nclass; c++) {
            double x = ct.chi[b.rep[c] * SFGPU_MAX_SEG + j];
            if (x != 0) v += chibbar[c] * x;
        }
        phibbar_seg[j] = v;
    }
    for (int m = 0; m < b.nmol; m++) {
        double v = 0;
        for (int j = 0; j < b.nseg; j++) v += phibbar_seg[j] * b.frac[j * SFGPU_MAX_SEG + m];
        as[m].phibbar = v;
        as[m].cbar = as[m].lngnbar = as[m].qbar = 0;
    }
}

// sum_z phibar . phi (normalised) of one molecule segment -> block partials
__global__ void adj_dot_partial(int M, const double *__restrict__ a, const double *__restrict__ b,
                                double *__restrict__ partial) {
    __shared__ double sh[kBlock];
    double acc = 0;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < M; r += gridDim.x * blockDim.x) acc += a[r] * b[r];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

// scalar adjoint of one molecule: phi = C * phi_cd, C from phibulk (free,
// solvent) or theta / GN (restricted); the solvent's phibulk = 1 - others'
__global__ void adj_mol_scalar(MolParam p, int nparts, const double *__restrict__ partial,
                               const MolScal *__restrict__ scal, AdjScal *__restrict__ as, int self) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double dot = 0;                      // sum phibar . phi
    for (int b = 0; b < nparts; b++) dot += partial[b];
    const MolScal s = scal[self];
    AdjScal a = as[self];
    a.cbar = (s.norm != 0) ? dot / s.norm : 0.0;
    double lngnbar = 0;
    if (p.freedom == SFGPU_MOL_RESTRICTED) {
        lngnbar += -a.cbar * s.norm;                                   // C = c0 exp(-lnGN)
        if (!p.pinned) lngnbar += -a.phibbar * (p.theta / exp(s.lngn));  // phibulk = theta exp(-lnGN)
    } else if (p.solvent) {
        double phib = s.phibulk;
        double pbar = a.phibbar + ((phib != 0) ? a.cbar * s.norm / phib : 0.0);
        for (int m = 0; m < p.nmol; m++)
            if (m != self) as[m].phibbar -= pbar;                       // phib_solv = 1 - sum others
    }
    a.lngnbar = lngnbar;
    a.qbar = lngnbar / exp(s.lngn);
    as[self] = a;
}

// phibar_raw = C phibar / G and Gbar -= phibar phi / G (CorrectDoubleCountG);
// monomers: phi = C G, Gbar += C phibar
__global__ void adj_phi_cd(DLat L, const double *__restrict__ phibar, const double *__restrict__ phi,
                           const double *__restrict__ G, const MolScal *__restrict__ scal, int mol, int monomer,
                           double *__restrict__ phibar_raw, double *__restrict__ gbar) {
    const double C = scal[mol].norm;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < L.M; r += gridDim.x * blockDim.x) {
        int c[3];
        lat_coords(L, r, c);
        if (!lat_interior(L, c)) { if (phibar_raw) phibar_raw[r] = 0; continue; }
        const double g = G[r];
        if (monomer) { gbar[r] += C * phibar[r]; continue; }
        if (g > 0) {
            phibar_raw[r] = C * phibar[r] / g;
            gbar[r] -= phibar[r] * phi[r] / g;
        } else {
            phibar_raw[r] = 0;
        }
    }
}

__global__ void adj_qbar_scale(const AdjScal *__restrict__ as, int mol, double *__restrict__ out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *out = as[mol].qbar;
}

// xbar(j, class) -= Gbar_full * G_full at the sites with iteration variables
struct SwfAdj {
    int nseg, nclass;
    int cls[SFGPU_MAX_SEG];
    int pinned[SFGPU_MAX_SEG];
    const double *gbar[SFGPU_MAX_SEG], *gfull[SFGPU_MAX_SEG], *range[SFGPU_MAX_SEG];
};
__global__ void adj_swf(int nsites, SwfAdj sa, const int *__restrict__ sites, double *__restrict__ xbar) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nsites; j += gridDim.x * blockDim.x) {
        const int z = sites[j];
        for (int i = 0; i < sa.nseg; i++) {
            if (sa.cls[i] < 0) continue;
            double gb = sa.gbar[i][z];
            if (sa.pinned[i] && !(sa.range[i][z] > 0)) gb = 0;
            xbar[(size_t)j * sa.nclass + sa.cls[i]] -= gb * sa.gfull[i][z];
        }
    }
}

}  // namespace

int sfgpu_system::ensure_adjoint() {
    if (a_ready) return SFGPU_OK;
    if (K != 1) return SFGPU_ERR_UNSUPPORTED;
    int rc;
    size_t store = 1;
    for (auto &o : mols) if (o.type != 0) store = std::max(store, (size_t)o.N * M);
    if ((rc = alloc_d(&a_gf, store)) || (rc = alloc_d(&a_gb, store))) return rc;
    SFGPU_CUDA_TRY(cudaMemset(a_gf, 0, sizeof(double) * store));
    SFGPU_CUDA_TRY(cudaMemset(a_gb, 0, sizeof(double) * store));
    a_phibar.assign(nseg, nullptr); a_gbar.assign(nseg, nullptr); a_phibar_raw.assign(nseg, nullptr);
    for (int i = 0; i < nseg; i++) {
        if ((rc = alloc_d(&a_phibar[i], M)) || (rc = alloc_d(&a_gbar[i], M)) || (rc = alloc_d(&a_phibar_raw[i], M)))
            return rc;
    }
    if ((rc = alloc_d(&a_cot[0], M)) || (rc = alloc_d(&a_cot[1], M))) return rc;
    if ((rc = alloc_d(&a_scal, 4 * (size_t)nmol)) || (rc = alloc_d(&a_chibbar, SFGPU_MAX_SEG)) ||
        (rc = alloc_d(&a_qbar, 1)))
        return rc;
    if ((rc = alloc_d(&a_w, nvar)) || (rc = alloc_d(&a_xbar, nvar))) return rc;
    a_ready = true;
    return SFGPU_OK;
}

// Gf and Gb of every position of molecule m's chain (full chains, also for
// symmetric homopolymers) into a_gf / a_gb; with compose, the backward sweep
// also accumulates Gf.Gb into the molecule's (zeroed) phi
int sfgpu_system::store_chains(int m, bool compose) {
    HMol &o = mols[m];
    const DLat &L = H.L;
    const int g = grid_a(M), gr = grid_rows_a(L);
    cudaStream_t s = stream;
    const int N = o.N;
    SFGPU_CUDA_TRY(cudaMemcpyAsync(a_gf, d_gseg[o.seg[0]], sizeof(double) * M, cudaMemcpyDeviceToDevice, s));
    for (int t = 1; t < N; t++)
        step1_rows<<<gr, kBlock, 0, s>>>(L, a_gf + (size_t)(t - 1) * M, d_gseg[o.seg[t]], a_gf + (size_t)t * M,
                                         nullptr, nullptr, COMP_NONE);
    SFGPU_CUDA_TRY(cudaMemcpyAsync(a_gb + (size_t)(N - 1) * M, d_gseg[o.seg[N - 1]], sizeof(double) * M,
                                   cudaMemcpyDeviceToDevice, s));
    if (compose)
        connect<<<g, kBlock, 0, s>>>(M, 1, a_gb + (size_t)(N - 1) * M, a_gf + (size_t)(N - 1) * M,
                                     o.d_phi[o.seg[N - 1]]);
    for (int t = N - 2; t >= 0; t--) {
        int sg = o.seg[t];
        step1_rows<<<gr, kBlock, 0, s>>>(L, a_gb + (size_t)(t + 1) * M, d_gseg[sg], a_gb + (size_t)t * M,
                                         compose ? a_gf + (size_t)t * M : nullptr, compose ? o.d_phi[sg] : nullptr,
                                         compose ? COMP_ACC : COMP_NONE);
    }
    return SFGPU_OK;
}

// primal evaluation of molecule m through store_chains
int sfgpu_system::molecule_phi_store(int m) {
    HMol &o = mols[m];
    const DLat &L = H.L;
    const int g = grid_a(M);
    cudaStream_t s = stream;
    MolParam p;
    p.N = o.N; p.type = o.type; p.freedom = o.freedom; p.sym = 0; p.K = 1;
    p.pinned = o.pinned; p.solvent = (m == solvent); p.nmol = nmol;
    p.phibulk_in = o.phibulk; p.theta = o.theta;
    MolScal *scal = (MolScal *)d_scal;
    if (o.type == 0) {
        int i = o.seg[0];
        wsum_partial<<<nblocks_red, kBlock, 0, s>>>(M, 1, d_gseg[i], d_wgn, d_partial);
        mol_scalars<<<1, 1, 0, s>>>(p, nblocks_red, d_partial, scal, m);
        finalize_phi<<<g, kBlock, 0, s>>>(M, d_gseg[i], o.d_phi[i], scal, m, 1);
        return SFGPU_OK;
    }
    for (int i : o.used) SFGPU_CUDA_TRY(cudaMemsetAsync(o.d_phi[i], 0, sizeof(double) * M, s));
    int rc = store_chains(m, true);
    if (rc) return rc;
    wsum_partial<<<nblocks_red, kBlock, 0, s>>>(M, 1, a_gb, d_wgn, d_partial);
    mol_scalars<<<1, 1, 0, s>>>(p, nblocks_red, d_partial, scal, m);
    for (int i : o.used) {
        finalize_phi<<<g, kBlock, 0, s>>>(M, d_gseg[i], o.d_phi[i], scal, m, 0);
        set_boundaries<<<g, kBlock, 0, s>>>(L, 1, o.d_phi[i]);
    }
    return SFGPU_OK;
}

// reverse sweep of one molecule; state phi cotangents in a_phibar
int sfgpu_system::molecule_adjoint(int m) {
    HMol &o = mols[m];
    const DLat &L = H.L;
    const int g = grid_a(M), gr = grid_rows_a(L);
    cudaStream_t s = stream;
    MolParam p;
    p.N = o.N; p.type = o.type; p.freedom = o.freedom; p.sym = 0; p.K = 1;
    p.pinned = o.pinned; p.solvent = (m == solvent); p.nmol = nmol;
    p.phibulk_in = o.phibulk; p.theta = o.theta;
    MolScal *scal = (MolScal *)d_scal;
    AdjScal *as = (AdjScal *)a_scal;
    // C-bar: sum over the molecule's segments of phibar . phi
    const int np = nblocks_red;
    for (size_t a = 0; a < o.used.size(); a++) {
        int i = o.used[a];
        adj_dot_partial<<<np, kBlock, 0, s>>>(M, a_phibar[i], o.d_phi[i], d_partial + a * np);
    }
    adj_mol_scalar<<<1, 1, 0, s>>>(p, np * (int)o.used.size(), d_partial, scal, as, m);
    for (int i : o.used)
        adj_phi_cd<<<g, kBlock, 0, s>>>(L, a_phibar[i], o.d_phi[i], d_gseg[i], scal, m, o.type == 0,
                                         a_phibar_raw[i], a_gbar[i]);
    if (o.type == 0) {
        // Q = sum w G enters restricted monomers: Gbar += qbar w
        adj_qbar_scale<<<1, 1, 0, s>>>(as, m, a_qbar);
        adj_axpy_interior<<<g, kBlock, 0, s>>>(L, d_wgn, a_qbar, a_gbar[o.seg[0]]);
        return SFGPU_OK;
    }
    const int N = o.N;
    double *cot = a_cot[0], *nxt = a_cot[1];
    // descending sweep over the forward recursion
    adj_init<<<g, kBlock, 0, s>>>(L, a_phibar_raw[o.seg[N - 1]], a_gb + (size_t)(N - 1) * M, cot);
    for (int t = N - 1; t >= 1; t--) {
        adj_init<<<g, kBlock, 0, s>>>(L, a_phibar_raw[o.seg[t - 1]], a_gb + (size_t)(t - 1) * M, nxt);
        adj_chain_step<<<gr, kBlock, 0, s>>>(L, cot, d_gseg[o.seg[t]], a_gf + (size_t)(t - 1) * M, a_gbar[o.seg[t]], nxt);
        std::swap(cot, nxt);
    }
    adj_add_interior<<<g, kBlock, 0, s>>>(L, cot, a_gbar[o.seg[0]]);
    // ascending sweep over the backward recursion (Q = sum w Gb(1) adds qbar * w)
    adj_init<<<g, kBlock, 0, s>>>(L, a_phibar_raw[o.seg[0]], a_gf, cot);
    adj_qbar_scale<<<1, 1, 0, s>>>(as, m, a_qbar);
    adj_axpy_interior<<<g, kBlock, 0, s>>>(L, d_wgn, a_qbar, cot);
    for (int t = 0; t < N - 1; t++) {
        adj_init<<<g, kBlock, 0, s>>>(L, a_phibar_raw[o.seg[t + 1]], a_gf + (size_t)(t + 1) * M, nxt);
        adj_chain_step<<<gr, kBlock, 0, s>>>(L, cot, d_gseg[o.seg[t]], a_gb + (size_t)(t + 1) * M, a_gbar[o.seg[t]], nxt);
        std::swap(cot, nxt);
    }
    adj_add_interior<<<g, kBlock, 0, s>>>(L, cot, a_gbar[o.seg[N - 1]]);
    return SFGPU_OK;
}

int sfgpu_system::vjp_async(const double *x, const double *w, double *f, double *xbar) {
    int rc = ensure_adjoint();
    if (rc) return rc;
    const DLat &L = H.L;
    const int g = grid_a(M);
    cudaStream_t s = stream;
    // primal with stored propagators
    for (int i = 0; i < nseg; i++) {
        if (freedom[i] == SFGPU_SEG_FROZEN) continue;
        swf_update<<<g, kBlock, 0, s>>>(L, x, d_jmap, nclass, class_of[i], d_range[i],
                                        freedom[i] == SFGPU_SEG_PINNED, d_gfull[i], d_gseg[i]);
    }
    for (int m = 0; m < nmol; m++) {
        if (m == solvent) continue;
        if ((rc = molecule_phi_store(m))) return rc;
    }
    if ((rc = molecule_phi_store(solvent))) return rc;
    for (int i = 0; i < nseg; i++) {
        if (freedom[i] == SFGPU_SEG_FROZEN) continue;
        PtrList pl;
        pl.n = 0;
        for (auto &o : mols) if (o.count[i]) pl.p[pl.n++] = o.d_phi[i];
        sum_profiles<<<g, kBlock, 0, s>>>(M, pl, d_phi[i]);
    }
    bulk_scalars<<<1, 1, 0, s>>>(bp, ct, (const MolScal *)d_scal, d_phib, d_chib);
    ResParam rp;
    memset(&rp, 0, sizeof(rp));
    rp.nsites = nsites; rp.nclass = nclass; rp.nseg = nseg;
    for (int c = 0; c < nclass; c++) { rp.rep[c] = rep_of_class[c]; rp.gfull[c] = d_gfull[rep_of_class[c]]; }
    for (int i = 0; i < nseg; i++) rp.phi[i] = d_phi[i];
    residual<<<grid_a(nsites), kBlock, 0, s>>>(L, rp, ct, d_sites, d_chib, f);
    if (!w) w = f;   // gradient of |f|^2 / 2
    // reverse
    for (int i = 0; i < nseg; i++) {
        SFGPU_CUDA_TRY(cudaMemsetAsync(a_phibar[i], 0, sizeof(double) * M, s));
        SFGPU_CUDA_TRY(cudaMemsetAsync(a_gbar[i], 0, sizeof(double) * M, s));
    }
    SFGPU_CUDA_TRY(cudaMemsetAsync(a_chibbar, 0, sizeof(double) * SFGPU_MAX_SEG, s));
    SFGPU_CUDA_TRY(cudaMemsetAsync(xbar, 0, sizeof(double) * nvar, s));
    AdjResParam ap;
    memset(&ap, 0, sizeof(ap));
    for (int i = 0; i < nseg; i++) ap.phibar[i] = a_phibar[i];
    ap.chibbar = a_chibbar;
    adj_residual<<<grid_a(nsites), kBlock, 0, s>>>(L, rp, ct, d_sites, w, ap, xbar);
    adj_bulk<<<1, 1, 0, s>>>(bp, ct, a_chibbar, (AdjScal *)a_scal);
    // molecules in reverse order of the primal (the solvent first).  The
    // chain storage holds one molecule: the last polymer the primal
    // propagated keeps its chains, every other polymer is propagated again.
    int held = (mols[solvent].type != 0) ? solvent : -1;
    if (held < 0)
        for (int m = nmol - 1; m >= 0 && held < 0; m--)
            if (m != solvent && mols[m].type != 0) held = m;
    if ((rc = molecule_adjoint(solvent))) return rc;
    for (int m = nmol - 1; m >= 0; m--) {
        if (m == solvent) continue;
        if (mols[m].type != 0 && m != held) {
            if ((rc = store_chains(m, false))) return rc;
            held = m;
        }
        if ((rc = molecule_adjoint(m))) return rc;
    }
    SwfAdj sa;
    memset(&sa, 0, sizeof(sa));
    sa.nseg = nseg; sa.nclass = nclass;
    for (int i = 0; i < nseg; i++) {
        sa.cls[i] = class_of[i];
        sa.pinned[i] = freedom[i] == SFGPU_SEG_PINNED;
        sa.gbar[i] = a_gbar[i];
        sa.gfull[i] = d_gfull[i];
        sa.range[i] = d_range[i];
    }
    adj_swf<<<grid_a(nsites), kBlock, 0, s>>>(nsites, sa, d_sites, xbar);
    SFGPU_CUDA_TRY(cudaGetLastError());
    return SFGPU_OK;
}

extern "C" int sfgpu_vjp(sfgpu_system *s, const double *x_dev, const double *w_dev, double *f_dev, double *xbar_dev) {
    if (!s) return SFGPU_ERR_INVALID;
    return s->vjp_async(x_dev, w_dev, f_dev, xbar_dev);
}

extern "C" int sfgpu_vjp_host(sfgpu_system *s, const double *x, const double *w, double *f, double *xbar) {
    if (!s || !x || !w) return SFGPU_ERR_INVALID;
    int rc = s->ensure_adjoint();
    if (rc) return rc;
    SFGPU_CUDA_TRY(cudaMemcpyAsync(s->d_x, x, sizeof(double) * s->nvar, cudaMemcpyHostToDevice, s->stream));
    SFGPU_CUDA_TRY(cudaMemcpyAsync(s->a_w, w, sizeof(double) * s->nvar, cudaMemcpyHostToDevice, s->stream));
    if ((rc = s->vjp_async(s->d_x, s->a_w, s->d_f, s->a_xbar))) return rc;
    if (f) SFGPU_CUDA_TRY(cudaMemcpyAsync(f, s->d_f, sizeof(double) * s->nvar, cudaMemcpyDeviceToHost, s->stream));
    if (xbar) SFGPU_CUDA_TRY(cudaMemcpyAsync(xbar, s->a_xbar, sizeof(double) * s->nvar, cudaMemcpyDeviceToHost, s->stream));
    SFGPU_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return SFGPU_OK;
}

// ---------------------------------------------------------------------------
// L-BFGS on Phi(x) = |f(x)|^2 / 2, gradient J^T f from the adjoint sweep
// ---------------------------------------------------------------------------
namespace {
__global__ void lb_axpy(size_t n, double a, const double *__restrict__ x, double *__restrict__ y) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        y[i] += a * x[i];
}
__global__ void lb_scale(size_t n, double a, const double *__restrict__ x, double *__restrict__ y) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        y[i] = a * x[i];
}
__global__ void lb_diff(size_t n, const double *__restrict__ a, const double *__restrict__ b, double *__restrict__ y) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        y[i] = a[i] - b[i];
}
__global__ void lb_lincomb(size_t n, const double *__restrict__ x, double a, const double *__restrict__ d,
                           double *__restrict__ y) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        y[i] = x[i] + a * d[i];
}
}  // namespace

extern "C" int sfgpu_solve_lbfgs(sfgpu_system *s, double *x_host, double tol, int maxit, int m,
                                 int *iterations, int *evaluations, double *final_error) {
    if (!s || !x_host || m < 1 || m > 64 || maxit < 0) return SFGPU_ERR_INVALID;
    int rc = s->ensure_adjoint();
    if (rc) return rc;
    const size_t n = s->nvar;
    cudaStream_t st = s->stream;
    std::vector<void *> mine;
    auto get = [&](double **p, size_t cnt) -> int {
        cudaError_t e = cudaMalloc((void **)p, sizeof(double) * (cnt ? cnt : 1));
        if (e != cudaSuccess) { sfgpu_set_error(e, "cudaMalloc", __FILE__, __LINE__); return SFGPU_ERR_NOMEM; }
        mine.push_back(*p);
        return SFGPU_OK;
    };
    auto cleanup = [&]() { for (void *p : mine) cudaFree(p); };
    const int gb = (int)std::max<size_t>(1, std::min<size_t>((n + kBlock - 1) / kBlock, 148 * 8));
    double *x, *f, *g, *xt, *ft, *gt, *d, *S, *Y, *partial, *sums;
    if ((rc = get(&x, n)) || (rc = get(&f, n)) || (rc = get(&g, n)) || (rc = get(&xt, n)) || (rc = get(&ft, n)) ||
        (rc = get(&gt, n)) || (rc = get(&d, n)) || (rc = get(&S, n * m)) || (rc = get(&Y, n * m)) ||
        (rc = get(&partial, (size_t)gb * 4)) || (rc = get(&sums, 4))) {
        cleanup();
        return rc;
    }
#define LBTRY(e) do { cudaError_t _e = (e); if (_e != cudaSuccess) { sfgpu_set_error(_e, #e, __FILE__, __LINE__); cleanup(); return SFGPU_ERR_CUDA; } } while (0)
#define LBRC(e) do { int _r = (e); if (_r) { cleanup(); return _r; } } while (0)
    auto dot = [&](const double *a, const double *b, double *out) -> int {
        DotList dl;
        dl.n = 1; dl.a[0] = a; dl.b[0] = b;
        dots_partial<<<gb, kBlock, 0, st>>>(n, dl, partial);
        finish_sums<<<1, 32, 0, st>>>(1, gb, partial, sums);
        cudaError_t e = cudaMemcpyAsync(out, sums, sizeof(double), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) { sfgpu_set_error(e, "dot", __FILE__, __LINE__); return SFGPU_ERR_CUDA; }
        return SFGPU_OK;
    };
    LBTRY(cudaMemcpyAsync(x, x_host, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    LBRC(s->vjp_async(x, nullptr, f, g));
    int nev = 1;
    double ff;
    LBRC(dot(f, f, &ff));
    double fn = sqrt(ff);
    std::vector<double> rho(m), alpha(m);
    int it = 0, stored = 0, head = 0;
    while (fn > tol && it < maxit && std::isfinite(fn)) {
        it++;
        // two-loop recursion: d = -H g
        LBTRY(cudaMemcpyAsync(d, g, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        for (int q = 0; q < stored; q++) {
            int k = (head - 1 - q + m) % m;
            double sd;
            LBRC(dot(S + (size_t)k * n, d, &sd));
            alpha[k] = rho[k] * sd;
            lb_axpy<<<gb, kBlock, 0, st>>>(n, -alpha[k], Y + (size_t)k * n, d);
        }
        if (stored > 0) {
            int k = (head - 1 + m) % m;
            double sy, yy;
            LBRC(dot(S + (size_t)k * n, Y + (size_t)k * n, &sy));
            LBRC(dot(Y + (size_t)k * n, Y + (size_t)k * n, &yy));
            lb_scale<<<gb, kBlock, 0, st>>>(n, sy / yy, d, d);
        } else {
            double gg;
            LBRC(dot(g, g, &gg));
            lb_scale<<<gb, kBlock, 0, st>>>(n, std::min(1.0, fn / sqrt(gg)), d, d);
        }
        for (int q = stored - 1; q >= 0; q--) {
            int k = (head - 1 - q + m) % m;
            double yd;
            LBRC(dot(Y + (size_t)k * n, d, &yd));
            double beta = rho[k] * yd;
            lb_axpy<<<gb, kBlock, 0, st>>>(n, alpha[k] - beta, S + (size_t)k * n, d);
        }
        lb_scale<<<gb, kBlock, 0, st>>>(n, -1.0, d, d);
        double gd;
        LBRC(dot(g, d, &gd));
        if (!(gd < 0)) {   // not a descent direction: restart from steepest descent
            stored = 0;
            lb_scale<<<gb, kBlock, 0, st>>>(n, -1.0, g, d);
            LBRC(dot(g, d, &gd));
        }
        // Armijo backtracking on Phi = |f|^2 / 2
        double a = 1.0, fft = 0;
        bool ok = false;
        for (int ls = 0; ls < 30; ls++) {
            lb_lincomb<<<gb, kBlock, 0, st>>>(n, x, a, d, xt);
            LBRC(s->vjp_async(xt, nullptr, ft, gt));
            nev++;
            LBRC(dot(ft, ft, &fft));
            if (std::isfinite(fft) && 0.5 * fft <= 0.5 * ff + 1e-4 * a * gd) { ok = true; break; }
            a *= 0.5;
        }
        if (!ok) break;
        // history: s = xt - x, y = gt - g
        lb_diff<<<gb, kBlock, 0, st>>>(n, xt, x, S + (size_t)head * n);
        lb_diff<<<gb, kBlock, 0, st>>>(n, gt, g, Y + (size_t)head * n);
        double ys;
        LBRC(dot(Y + (size_t)head * n, S + (size_t)head * n, &ys));
        if (ys > 1e-300) {
            rho[head] = 1.0 / ys;
            head = (head + 1) % m;
            stored = std::min(stored + 1, m);
        }
        std::swap(x, xt); std::swap(f, ft); std::swap(g, gt);
        ff = fft;
        fn = sqrt(ff);
    }
    LBTRY(cudaMemcpyAsync(x_host, x, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    LBTRY(cudaStreamSynchronize(st));
    LBRC(s->residual_async(x, f));
    LBTRY(cudaStreamSynchronize(st));
#undef LBTRY
#undef LBRC
    cleanup();
    if (iterations) *iterations = it;
    if (evaluations) *evaluations = nev;
    if (final_error) *final_error = fn;
    if (!std::isfinite(fn)) return SFGPU_ERR_NONFINITE;
    return (fn <= tol) ? SFGPU_OK : SFGPU_ERR_NOTCONVERGED;
}
