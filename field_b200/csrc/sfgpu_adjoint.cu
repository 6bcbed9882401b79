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
    double lncbar;      // cotangent of ln C (free energy)
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
        as[m].cbar = as[m].lngnbar = as[m].qbar = as[m].lncbar = 0;
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
        lngnbar += -a.lncbar;                                          // ln C = ln(theta [/N]) - lnGN
    } else if (p.solvent) {
        double phib = s.phibulk;
        double pbar = a.phibbar + ((phib != 0) ? (a.cbar * s.norm + a.lncbar) / phib : 0.0);  // ln C = ln(phib [/N])
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

// free-energy scalars: zero every molecule's cotangents, then
// lncbar of molecule m = invN sum_z wf p_m (block partials of its profiles)
__global__ void fe_zero_scal(int nmol, AdjScal *__restrict__ as) {
    if (threadIdx.x == 0 && blockIdx.x == 0)
        for (int m = 0; m < nmol; m++) as[m].cbar = as[m].phibbar = as[m].lngnbar = as[m].qbar = as[m].lncbar = 0;
}
__global__ void fe_set_lncbar(int nparts, const double *__restrict__ partial, double invN, AdjScal *__restrict__ as,
                              int mol) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double v = 0;
    for (int b = 0; b < nparts; b++) v += partial[b];
    as[mol].lncbar = invN * v;
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

// cotangent vectors and scalars of the reverse sweep (any lattice order)
int sfgpu_system::ensure_adjoint_misc() {
    int rc;
    if (!a_misc) {
        a_phibar.assign(nseg, nullptr); a_gbar.assign(nseg, nullptr); a_phibar_raw.assign(nseg, nullptr);
        for (int i = 0; i < nseg; i++) {
            if ((rc = alloc_d(&a_phibar[i], M)) || (rc = alloc_d(&a_gbar[i], M)) ||
                (rc = alloc_d(&a_phibar_raw[i], M)))
                return rc;
        }
        if ((rc = alloc_d(&a_cot[0], (size_t)K * M)) || (rc = alloc_d(&a_cot[1], (size_t)K * M))) return rc;
        if ((rc = alloc_d(&a_scal, sizeof(AdjScal) / sizeof(double) * (size_t)nmol)) || (rc = alloc_d(&a_chibbar, SFGPU_MAX_SEG)) ||
            (rc = alloc_d(&a_qbar, 1)))
            return rc;
        if ((rc = alloc_d(&a_w, nvar)) ||
            (rc = alloc_d(&a_xbar, std::max((size_t)nvar, (size_t)nseg * nseg))))
            return rc;
        a_misc = true;
    }
    return SFGPU_OK;
}

int sfgpu_system::ensure_adjoint() {
    if (logmode) return fail_unsupported("derivatives with overflow protection");
    if (charged) return fail_unsupported("derivatives of charged systems");
    for (auto &o : mols)
        if (o.dend) build_dend_tree(o);
    int rc = ensure_adjoint_misc();
    if (rc) return rc;
    // dendrimers run the tree recursion in the reverse sweep: 3N slices
    size_t dend_need = 0;
    for (auto &o : mols)
        if (o.dend) dend_need = std::max(dend_need, (size_t)3 * o.N * M);
    if (dend_need > a_dend_gi_doubles) {
        if (a_dend_gi) cudaFree(a_dend_gi);
        a_dend_gi = nullptr;
        a_dend_gi_doubles = 0;
        cudaError_t e = cudaMalloc((void **)&a_dend_gi, sizeof(double) * dend_need);
        if (e != cudaSuccess) {
            a_dend_gi = nullptr;
            sfgpu_set_error(e, "cudaMalloc (dendrimer tree slices)", __FILE__, __LINE__);
            return SFGPU_ERR_NOMEM;
        }
        a_dend_gi_doubles = dend_need;
    }
    // branched molecules: the cotangents of every U, Q, D slice and a pool
    // for the products a node's combinations pass through
    size_t tree_need = 0;
    for (auto &o : mols) {
        if (!o.tree && !o.dend) continue;
        size_t kmax = 1;
        for (auto &k : (o.dend ? o.tkids : o.kids)) kmax = std::max(kmax, k.size());
        tree_need = std::max(tree_need, (3 * (size_t)o.N + kmax + 3) * M);
    }
    if (tree_need > a_tree_doubles) {
        if (a_tree) cudaFree(a_tree);
        a_tree = nullptr;
        a_tree_doubles = 0;
        cudaError_t e = cudaMalloc((void **)&a_tree, sizeof(double) * tree_need);
        if (e != cudaSuccess) {
            a_tree = nullptr;
            sfgpu_set_error(e, "cudaMalloc (bond-tree cotangents)", __FILE__, __LINE__);
            return SFGPU_ERR_NOMEM;
        }
        a_tree_doubles = tree_need;
    }
    // rings: one set of walk levels per block of ring_phi_adj
    size_t ring_need = 0;
    for (auto &o : mols) {
        if (!o.ring) continue;
        const int Mmax = (o.N / 2 > M) ? 2 * M : M + o.N / 2;
        if ((size_t)3 * (Mmax + 1) * sizeof(double) > 200 * 1024)
            return fail_unsupported("the reverse mode of a ring walk larger than shared memory");
        ring_need = std::max(ring_need, (size_t)std::min(M, kRingAdjBlocks) * (o.N / 2) * (Mmax + 1));
    }
    if (ring_need > a_ring_doubles) {
        if (a_ring) cudaFree(a_ring);
        a_ring = nullptr;
        a_ring_doubles = 0;
        cudaError_t e = cudaMalloc((void **)&a_ring, sizeof(double) * ring_need);
        if (e != cudaSuccess) {
            a_ring = nullptr;
            sfgpu_set_error(e, "cudaMalloc (ring walk levels)", __FILE__, __LINE__);
            return SFGPU_ERR_NOMEM;
        }
        a_ring_doubles = ring_need;
    }
    if (!a_store) {
        int nmax = 1;
        for (auto &o : mols) if (o.type != 0) nmax = std::max(nmax, o.N);
        size_t slices;
        if (a_stride == 0) {
            slices = 2 * (size_t)nmax;
        } else {
            const size_t nq = (size_t)(nmax + a_stride - 1) / a_stride;
            slices = 2 * nq + 2 * (size_t)a_stride + 1;
        }
        const size_t KM = (size_t)K * M;
        cudaError_t e = cudaMalloc((void **)&a_store, sizeof(double) * slices * KM);
        if (e != cudaSuccess) {
            a_store = nullptr;
            sfgpu_set_error(e, "cudaMalloc (reverse-sweep chain storage)", __FILE__, __LINE__);
            return SFGPU_ERR_NOMEM;
        }
        // boundary entries of the slices are read only on surface layers, where
        // propagators are 0: start from zeros
        SFGPU_CUDA_TRY(cudaMemset(a_store, 0, sizeof(double) * slices * KM));
        if (a_stride == 0) {
            a_gf = a_store;
            a_gb = a_store + (size_t)nmax * KM;
        } else {
            const size_t nq = (size_t)(nmax + a_stride - 1) / a_stride;
            a_ckF = a_store;
            a_ckB = a_ckF + nq * KM;
            a_bufF = a_ckB + nq * KM;
            a_bufB = a_bufF + (size_t)a_stride * KM;   // a_stride + 1 slices: the last is the carry
            a_gf = a_gb = nullptr;
        }
        a_qseg = -1;
    }
    return SFGPU_OK;
}

int sfgpu_system::set_checkpoint(int stride) {
    if (stride < -1) return SFGPU_ERR_INVALID;
    if (stride == -1) {   // the memory-optimal stride for the longest chain
        int nmax = 1;
        for (auto &o : mols) if (o.type != 0) nmax = std::max(nmax, o.N);
        stride = std::max(1, (int)std::ceil(std::sqrt((double)nmax)));
    }
    if (stride == a_stride && a_store) return SFGPU_OK;
    SFGPU_CUDA_TRY(cudaStreamSynchronize(stream));
    if (a_store) SFGPU_CUDA_TRY(cudaFree(a_store));
    a_store = nullptr;
    a_stride = stride;
    return SFGPU_OK;
}

// Steps of molecule o's chain on K-component slices: the start slice (G in
// every component), forward step t (Gf(t) from Gf(t-1)), backward step t
// (Gb(t) from Gb(t+1), composing Gb(t).Gf(t) into phi when other != nullptr).
void sfgpu_system::adj_start(const double *G, double *dst) {
    const int g = grid_a(M);
    replicate<<<g, kBlock, 0, stream>>>(M, K, G, dst);
    if (K == 6) set_boundaries<<<g, kBlock, 0, stream>>>(H.L, 6, dst);
}
void sfgpu_system::adj_fstep(const HMol &o, int t, const double *src, double *dst) {
    const DLat &L = H.L;
    const int sg = o.seg[t];
    if (K == 1 && o.force != 0)   // SF_Copol1stO.cpp:1207-1211
        step1_force_rows<<<grid_rows_a(L), kBlock, 0, stream>>>(L, force_weights(L, o.force), src, d_gseg[sg], dst,
                                                                nullptr, nullptr, COMP_NONE);
    else if (K == 1)
        launch_step1(src, d_gseg[sg], dst, nullptr, nullptr, COMP_NONE);   // the residual's step (3D: x-marching)
    else if (K == 6 && L.stiff) {   // SF_Copol2ndO_stiff_range.cpp:211-217, the last step isotropic
        const bool last = (t == o.N - 1);
        step2_rows<<<grid_rows_a(L), kBlock, 0, stream>>>(L, src, d_gseg[sg],
                                                          last ? 0.2 : pf[o.seg[t - 1] * nseg + o.seg[t + 1]], dst,
                                                          nullptr, nullptr, COMP_NONE, 0,
                                                          last ? STEP2_ISO : STEP2_STIFF);
    } else if (K == 6)
        step2_rows<<<grid_rows_a(L), kBlock, 0, stream>>>(L, src, d_gseg[sg], pf[o.seg[t - 1] * nseg + sg], dst,
                                                          nullptr, nullptr, COMP_NONE, 0);
    else
        step2l_rows<<<grid_rows_a(L), kBlock, 0, stream>>>(L, src, d_gseg[sg], pf[o.seg[t - 1] * nseg + sg], dst,
                                                           nullptr, nullptr, COMP_NONE, 0);
}
void sfgpu_system::adj_bstep(const HMol &o, int t, const double *src, double *dst, const double *other,
                             double *phi) {
    const DLat &L = H.L;
    const int sg = o.seg[t];
    const int mode = other ? COMP_ACC : COMP_NONE;
    if (K == 1 && o.force != 0)   // SF_Copol1stO.cpp:1226-1230
        step1_force_rows<<<grid_rows_a(L), kBlock, 0, stream>>>(L, force_weights(L, -o.force), src, d_gseg[sg], dst,
                                                                other, phi, mode);
    else if (K == 1)
        launch_step1(src, d_gseg[sg], dst, other, phi, mode);
    else if (K == 6 && L.stiff) {   // :229-234, the first backward step isotropic
        const bool first = (t == o.N - 2);
        step2_rows<<<grid_rows_a(L), kBlock, 0, stream>>>(L, src, d_gseg[sg],
                                                          first ? 0.2 : pf[sg * nseg + o.seg[t + 2]], dst, other,
                                                          phi, mode, 1, first ? STEP2_ISO : STEP2_STIFF);
    } else if (K == 6)
        step2_rows<<<grid_rows_a(L), kBlock, 0, stream>>>(L, src, d_gseg[sg], pf[sg * nseg + o.seg[t + 1]], dst,
                                                          other, phi, mode, 1);
    else
        step2l_rows<<<grid_rows_a(L), kBlock, 0, stream>>>(L, src, d_gseg[sg], pf[sg * nseg + o.seg[t + 1]], dst,
                                                           other, phi, mode, 1);
}

// Gf and Gb of every position of molecule m's chain (full chains, also for
// symmetric homopolymers) into a_gf / a_gb; with compose, the backward sweep
// also accumulates Gf.Gb into the molecule's (zeroed) phi.  *gb0 = Gb(0).
int sfgpu_system::store_chains(int m, bool compose, const double **gb0) {
    if (a_stride > 0) return store_chains_ck(m, compose, gb0);
    HMol &o = mols[m];
    const int g = grid_a(M);
    cudaStream_t s = stream;
    const int N = o.N;
    const size_t KM = (size_t)K * M;
    adj_start(d_gseg[o.seg[0]], a_gf);
    for (int t = 1; t < N; t++) adj_fstep(o, t, a_gf + (size_t)(t - 1) * KM, a_gf + (size_t)t * KM);
    adj_start(d_gseg[o.seg[N - 1]], a_gb + (size_t)(N - 1) * KM);
    if (compose)
        connect<<<g, kBlock, 0, s>>>(M, K, a_gb + (size_t)(N - 1) * KM, a_gf + (size_t)(N - 1) * KM,
                                     o.d_phi[o.seg[N - 1]]);
    for (int t = N - 2; t >= 0; t--)
        adj_bstep(o, t, a_gb + (size_t)(t + 1) * KM, a_gb + (size_t)t * KM, compose ? a_gf + (size_t)t * KM : nullptr,
                  compose ? o.d_phi[o.seg[t]] : nullptr);
    if (gb0) *gb0 = a_gb;
    return SFGPU_OK;
}

// The same with checkpoints: Gf at the first and Gb at the last position of
// every segment of a_stride positions, each segment's slices recomputed by
// load_segment when a sweep needs them.  The backward sweep walks the
// segments downwards, recomputing each segment's Gf for the composition;
// a_bufB's last slice carries Gb from one segment to the next.
int sfgpu_system::store_chains_ck(int m, bool compose, const double **gb0) {
    HMol &o = mols[m];
    const int g = grid_a(M);
    cudaStream_t s = stream;
    const int N = o.N, k = a_stride, nq = (N + k - 1) / k;
    const size_t KM = (size_t)K * M, bytes = sizeof(double) * KM;
    auto F = [&](int j) { return a_bufF + (size_t)j * KM; };
    auto B = [&](int j) { return a_bufB + (size_t)j * KM; };
    double *carry = B(k);
    // forward: checkpoints at t = qk, the others in two alternating slices
    adj_start(d_gseg[o.seg[0]], a_ckF);
    const double *prev = a_ckF;
    for (int t = 1; t < N; t++) {
        double *dst = (t % k == 0) ? a_ckF + (size_t)(t / k) * KM : F(t & 1);
        adj_fstep(o, t, prev, dst);
        prev = dst;
    }
    a_qseg = -1;
    // backward, segments downwards
    for (int q = nq - 1; q >= 0; q--) {
        const int s0 = q * k, e = std::min(s0 + k, N) - 1;
        if (compose) {   // Gf of this segment
            SFGPU_CUDA_TRY(cudaMemcpyAsync(F(0), a_ckF + (size_t)q * KM, bytes, cudaMemcpyDeviceToDevice, s));
            for (int j = 1; j <= e - s0; j++) adj_fstep(o, s0 + j, F(j - 1), F(j));
        }
        for (int t = e; t >= s0; t--) {
            double *dst = B(t - s0);
            const int sg = o.seg[t];
            if (t == N - 1) {
                adj_start(d_gseg[sg], dst);
                if (compose) connect<<<g, kBlock, 0, s>>>(M, K, dst, F(t - s0), o.d_phi[sg]);
            } else {
                const double *src = (t == e) ? carry : B(t + 1 - s0);
                adj_bstep(o, t, src, dst, compose ? F(t - s0) : nullptr, compose ? o.d_phi[sg] : nullptr);
            }
            if (t == e)
                SFGPU_CUDA_TRY(cudaMemcpyAsync(a_ckB + (size_t)q * KM, dst, bytes, cudaMemcpyDeviceToDevice, s));
        }
        SFGPU_CUDA_TRY(cudaMemcpyAsync(carry, B(0), bytes, cudaMemcpyDeviceToDevice, s));
    }
    if (gb0) *gb0 = B(0);
    return SFGPU_OK;
}

// Gf and Gb of segment q (positions qk .. min(qk + k, N) - 1) of molecule m
// into a_bufF / a_bufB from its checkpoints
int sfgpu_system::load_segment(int m, int q) {
    if (a_stride == 0 || q == a_qseg) return SFGPU_OK;
    HMol &o = mols[m];
    cudaStream_t s = stream;
    const int N = o.N, k = a_stride;
    const int s0 = q * k, e = std::min(s0 + k, N) - 1;
    const size_t KM = (size_t)K * M, bytes = sizeof(double) * KM;
    auto F = [&](int j) { return a_bufF + (size_t)j * KM; };
    auto B = [&](int j) { return a_bufB + (size_t)j * KM; };
    SFGPU_CUDA_TRY(cudaMemcpyAsync(F(0), a_ckF + (size_t)q * KM, bytes, cudaMemcpyDeviceToDevice, s));
    for (int j = 1; j <= e - s0; j++) adj_fstep(o, s0 + j, F(j - 1), F(j));
    SFGPU_CUDA_TRY(cudaMemcpyAsync(B(e - s0), a_ckB + (size_t)q * KM, bytes, cudaMemcpyDeviceToDevice, s));
    for (int t = e - 1; t >= s0; t--) adj_bstep(o, t, B(t + 1 - s0), B(t - s0), nullptr, nullptr);
    a_qseg = q;
    return SFGPU_OK;
}

// primal evaluation of molecule m through store_chains
int sfgpu_system::molecule_phi_store(int m) {
    if (mols[m].dend) {   // the tree recursion on the dendrimer's tree form
        dend_view(mols[m], true);
        tree_gi = a_dend_gi;
        const int rc = molecule_phi_store(m);
        tree_gi = nullptr;
        dend_view(mols[m], false);
        return rc;
    }
    HMol &o = mols[m];
    const DLat &L = H.L;
    const int g = grid_a(M);
    cudaStream_t s = stream;
    MolParam p;
    p.N = o.N; p.type = o.type; p.freedom = o.freedom; p.sym = 0; p.K = K;
    p.pinned = o.pinned; p.solvent = (m == solvent); p.nmol = nmol;
    p.phibulk_in = o.phibulk; p.theta = o.theta;
    MolScal *scal = (MolScal *)d_scal;
    if (o.ring) return molecule_phi_ring(m);
    if (o.tree) return molecule_phi_tree(m);
    if (o.type == 0) {
        int i = o.seg[0];
        MolParam p1 = p;
        p1.K = 1;   // a monomer's end distribution is G itself
        wsum_partial<<<nblocks_red, kBlock, 0, s>>>(M, 1, d_gseg[i], d_wgn, d_partial);
        mol_scalars<<<1, 1, 0, s>>>(p1, nblocks_red, d_partial, scal, m);
        finalize_phi<<<g, kBlock, 0, s>>>(M, d_gseg[i], o.d_phi[i], scal, m, 1);
        return SFGPU_OK;
    }
    for (int i : o.used) SFGPU_CUDA_TRY(cudaMemsetAsync(o.d_phi[i], 0, sizeof(double) * M, s));
    const double *gb0 = nullptr;
    int rc = store_chains(m, true, &gb0);
    if (rc) return rc;
    wsum_partial<<<nblocks_red, kBlock, 0, s>>>(M, K, gb0, d_wgn, d_partial);
    mol_scalars<<<1, 1, 0, s>>>(p, nblocks_red, d_partial, scal, m);
    for (int i : o.used) {
        finalize_phi<<<g, kBlock, 0, s>>>(M, d_gseg[i], o.d_phi[i], scal, m, 0);
        set_boundaries<<<g, kBlock, 0, s>>>(L, 1, o.d_phi[i]);
    }
    return SFGPU_OK;
}

// reverse sweep of one molecule; state phi cotangents in a_phibar
int sfgpu_system::molecule_adjoint(int m, double *const *phibar_src) {
    if (mols[m].dend) {
        dend_view(mols[m], true);
        tree_gi = a_dend_gi;
        const int rc = molecule_adjoint(m, phibar_src);
        tree_gi = nullptr;
        dend_view(mols[m], false);
        return rc;
    }
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
    if (o.ring) {
        const int Mmax = (o.N / 2 > M) ? 2 * M : M + o.N / 2;
        const size_t shm = (size_t)3 * (Mmax + 1) * sizeof(double);
        if (shm > 48 * 1024)
            SFGPU_CUDA_TRY(cudaFuncSetAttribute(ring_phi_adj, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
        const int sg = o.seg[0];
        ring_phi_adj<<<std::min(M, kRingAdjBlocks), Mmax + 1 >= 256 ? 256 : 64, shm, s>>>(
            L, M, o.N, Mmax, d_gseg[sg], phibar_src[sg], o.phibulk, o.ring_norm0, a_ring, a_gbar[sg]);
        SFGPU_CUDA_TRY(cudaGetLastError());
        return SFGPU_OK;
    }
    // C-bar: sum over the molecule's segments of phibar . phi
    const int np = nblocks_red;
    for (size_t a = 0; a < o.used.size(); a++) {
        int i = o.used[a];
        adj_dot_partial<<<np, kBlock, 0, s>>>(M, phibar_src[i], o.d_phi[i], d_partial + a * np);
    }
    adj_mol_scalar<<<1, 1, 0, s>>>(p, np * (int)o.used.size(), d_partial, scal, as, m);
    for (int i : o.used)
        adj_phi_cd<<<g, kBlock, 0, s>>>(L, phibar_src[i], o.d_phi[i], d_gseg[i], scal, m, o.type == 0,
                                         a_phibar_raw[i], a_gbar[i]);
    if (o.type == 0) {
        // Q = sum w G enters restricted monomers: Gbar += qbar w
        adj_qbar_scale<<<1, 1, 0, s>>>(as, m, a_qbar);
        adj_axpy_interior<<<g, kBlock, 0, s>>>(L, 1, d_wgn, a_qbar, 1.0, a_gbar[o.seg[0]]);
        return SFGPU_OK;
    }
    if (o.tree) return molecule_adjoint_tree(m);
    const int N = o.N;
    double *cot = a_cot[0], *nxt = a_cot[1];
    // slices of position t: stored, or recomputed segment by segment
    a_qseg = -1;
    int rcs = SFGPU_OK;
    auto at = [&](int t) {
        if (a_stride == 0) return t;
        const int q = t / a_stride;
        if (!rcs) rcs = load_segment(m, q);
        return t - q * a_stride;
    };
    const size_t KM = (size_t)K * M;
    auto GF = [&](int j) -> const double * { return (a_stride ? a_bufF : a_gf) + (size_t)j * KM; };
    auto GB = [&](int j) -> const double * { return (a_stride ? a_bufB : a_gb) + (size_t)j * KM; };
    // one reverse step: gbar(seg t) += cot . A p; nxt += A^T (G_t cot)
    auto rstep = [&](int t, const double *p, double S, int backward) {
        const int sg = o.seg[t];
        if (K == 6 && L.stiff) {
            // the stiff-range chain's steps: forward into t with Pf(t-1, t+1),
            // backward into t with Pf(t, t+2), isotropic at the chain's end
            const bool iso = backward ? (t == N - 2) : (t == N - 1);
            const double Sv = iso ? 0.2 : (backward ? pf[sg * nseg + o.seg[t + 2]] : pf[o.seg[t - 1] * nseg + o.seg[t + 1]]);
            adj_step2v<<<gr, kBlock, 0, s>>>(L, cot, d_gseg[sg], p, Sv, backward, iso ? STEP2_ISO : STEP2_STIFF,
                                             a_gbar[sg], nxt);
            return;
        }
        if (K == 1 && o.force != 0)   // the forward recursion's +force, the backward one's -force
            adj_chain_step_force<<<gr, kBlock, 0, s>>>(L, force_weights(L, backward ? -o.force : o.force), cot,
                                                       d_gseg[sg], p, a_gbar[sg], nxt);
        else if (K == 1)
            adj_chain_step<<<gr, kBlock, 0, s>>>(L, cot, d_gseg[sg], p, a_gbar[sg], nxt);
        else if (K == 6)
            adj_step2<<<gr, kBlock, 0, s>>>(L, cot, d_gseg[sg], p, S, backward, a_gbar[sg], nxt);
        else
            adj_step2l<<<gr, kBlock, 0, s>>>(L, cot, d_gseg[sg], p, S, backward, a_gbar[sg], nxt);
    };
    // descending sweep over the forward recursion (step t used S(t-1, t))
    {
        const int j = at(N - 1);
        adj_init<<<g, kBlock, 0, s>>>(L, K, a_phibar_raw[o.seg[N - 1]], GB(j), cot);
    }
    for (int t = N - 1; t >= 1; t--) {
        const int j = at(t - 1);
        adj_init<<<g, kBlock, 0, s>>>(L, K, a_phibar_raw[o.seg[t - 1]], GB(j), nxt);
        rstep(t, GF(j), K > 1 ? pf[o.seg[t - 1] * nseg + o.seg[t]] : 0.0, 0);
        std::swap(cot, nxt);
    }
    adj_add_interior<<<g, kBlock, 0, s>>>(L, K, cot, a_gbar[o.seg[0]]);
    // ascending sweep over the backward recursion (step t used S(t, t+1));
    // lnGN = ln(sum w sum_k mu_k Gb_k(1) / 6) (mu_k the lumped multiplicities,
    // 1 in 3D; 1 and no division on first order) adds qbar mu_k / 6 * w
    {
        const int j = at(0);
        adj_init<<<g, kBlock, 0, s>>>(L, K, a_phibar_raw[o.seg[0]], GF(j), cot);
    }
    adj_qbar_scale<<<1, 1, 0, s>>>(as, m, a_qbar);
    adj_axpy_interior<<<g, kBlock, 0, s>>>(L, K, d_wgn, a_qbar, K > 1 ? 1.0 / 6.0 : 1.0, cot);
    for (int t = 0; t < N - 1; t++) {
        const int j = at(t + 1);
        adj_init<<<g, kBlock, 0, s>>>(L, K, a_phibar_raw[o.seg[t + 1]], GF(j), nxt);
        rstep(t, GB(j), K > 1 ? pf[o.seg[t] * nseg + o.seg[t + 1]] : 0.0, 1);
        std::swap(cot, nxt);
    }
    adj_add_interior<<<g, kBlock, 0, s>>>(L, K, cot, a_gbar[o.seg[N - 1]]);
    return rcs;
}

// Reverse sweep of a branched molecule (molecule_phi_tree's bond-tree
// recursion).  The primal's slices U(q), Q(q), D(q) are computed again into
// the chain scratch; the cotangents Ubar, Qbar, Dbar then run back through
// the outward pass (segments N-1 .. 0: the composition U D, every child's
// D(c) = step(D(q) prod_{siblings} Q / G_q, G_c)) and through the inward
// pass (segments 0 .. N-1: Q(q) = step(U(q), G_parent), U(q) = G_q at a leaf,
// Q of its only child, or the product of its children's Q over G_q).  The
// composition's cotangent phibar_raw and the lnGN term (qbar w into Ubar(0))
// are set up as for linear chains; every product a node's combinations pass
// through is formed again in a pool before it is reversed.
int sfgpu_system::molecule_adjoint_tree(int m) {
    HMol &o = mols[m];
    const DLat &L = H.L;
    const int g = grid_a(M), gr = grid_rows_a(L), N = o.N;
    cudaStream_t s = stream;
    const size_t bytes = sizeof(double) * M;
    int rc = molecule_phi_tree(m);   // U, Q, D of this molecule (the profiles come out unchanged)
    if (rc) return rc;
    double *const base = tree_gi ? tree_gi : d_gi;
    auto U = [&](int q) { return base + (size_t)q * M; };
    auto Q = [&](int q) { return base + (size_t)(N + q) * M; };
    auto D = [&](int q) { return base + (size_t)(2 * N + q) * M; };
    auto Ub = [&](int q) { return a_tree + (size_t)q * M; };
    auto Qb = [&](int q) { return a_tree + (size_t)(N + q) * M; };
    auto Db = [&](int q) { return a_tree + (size_t)(2 * N + q) * M; };
    size_t kmax = 1;
    for (auto &k : o.kids) kmax = std::max(kmax, k.size());
    double *pool = a_tree + (size_t)3 * N * M;            // kmax slices of products
    double *cb[2] = {pool + kmax * M, pool + (kmax + 1) * M};
    double *accbar = pool + (kmax + 2) * M;
    SFGPU_CUDA_TRY(cudaMemsetAsync(a_tree, 0, sizeof(double) * 3 * N * M, s));
    AdjScal *as = (AdjScal *)a_scal;
    adj_qbar_scale<<<1, 1, 0, s>>>(as, m, a_qbar);
    adj_axpy_interior<<<g, kBlock, 0, s>>>(L, 1, d_wgn, a_qbar, 1.0, Ub(0));
    // reverse a chain of combinations acc_j = acc_{j-1} b_j / Gq (j = 1..n,
    // acc_0 = first, the products in pool[0..n-1]) from the cotangent of
    // acc_n in cb[0]; returns the buffer with the cotangent of acc_0
    auto reverse_products = [&](const double *first, const std::vector<const double *> &bs,
                                const std::vector<double *> &bbars, const double *Gq, double *gbq) -> double * {
        const int n = (int)bs.size();
        // products again
        const double *acc = first;
        for (int j = 0; j < n; j++) {
            dend_combine<<<g, kBlock, 0, s>>>(M, acc, bs[j], Gq, pool + (size_t)j * M);
            acc = pool + (size_t)j * M;
        }
        int w = 0;
        for (int j = n - 1; j >= 0; j--) {
            const double *a = (j == 0) ? first : pool + (size_t)(j - 1) * M;
            tree_adj_combine<<<g, kBlock, 0, s>>>(L, cb[w], a, bs[j], Gq, pool + (size_t)j * M, cb[w ^ 1], bbars[j],
                                                  gbq);
            w ^= 1;
        }
        return cb[w];
    };
    // outward pass reversed
    for (int q = N - 1; q >= 0; q--) {
        const int sq = o.seg[q];
        const double *Gq = d_gseg[sq];
        tree_adj_connect<<<g, kBlock, 0, s>>>(L, a_phibar_raw[sq], U(q), D(q), Ub(q), Db(q));
        const std::vector<int> &kids = o.kids[q];
        for (int ci = (int)kids.size() - 1; ci >= 0; ci--) {
            const int c = kids[ci];
            std::vector<const double *> bs;
            std::vector<double *> bbars;
            for (int c2 : kids) if (c2 != c) { bs.push_back(Q(c2)); bbars.push_back(Qb(c2)); }
            // the step's input: D(q) times the siblings' Q over G_q
            const double *in = D(q);
            for (size_t j = 0; j < bs.size(); j++) {
                dend_combine<<<g, kBlock, 0, s>>>(M, in, bs[j], Gq, pool + j * M);
                in = pool + j * M;
            }
            SFGPU_CUDA_TRY(cudaMemsetAsync(accbar, 0, bytes, s));
            adj_chain_step<<<gr, kBlock, 0, s>>>(L, Db(c), d_gseg[o.seg[c]], in, a_gbar[o.seg[c]], accbar);
            if (bs.empty()) {
                adj_add_interior<<<g, kBlock, 0, s>>>(L, 1, accbar, Db(q));
            } else {
                SFGPU_CUDA_TRY(cudaMemcpyAsync(cb[0], accbar, bytes, cudaMemcpyDeviceToDevice, s));
                double *d0 = reverse_products(D(q), bs, bbars, Gq, a_gbar[sq]);
                adj_add_interior<<<g, kBlock, 0, s>>>(L, 1, d0, Db(q));
            }
        }
    }
    adj_add_interior<<<g, kBlock, 0, s>>>(L, 1, Db(0), a_gbar[o.seg[0]]);   // D(0) = G_0
    // inward pass reversed
    for (int q = 0; q < N; q++) {
        const int sq = o.seg[q];
        if (q > 0) {
            const int sp = o.seg[o.parent[q]];
            adj_chain_step<<<gr, kBlock, 0, s>>>(L, Qb(q), d_gseg[sp], U(q), a_gbar[sp], Ub(q));
        }
        const std::vector<int> &kids = o.kids[q];
        if (kids.empty()) {
            adj_add_interior<<<g, kBlock, 0, s>>>(L, 1, Ub(q), a_gbar[sq]);
        } else if (kids.size() == 1) {
            adj_add_interior<<<g, kBlock, 0, s>>>(L, 1, Ub(q), Qb(kids[0]));
        } else {
            std::vector<const double *> bs;
            std::vector<double *> bbars;
            for (size_t j = 1; j < kids.size(); j++) { bs.push_back(Q(kids[j])); bbars.push_back(Qb(kids[j])); }
            SFGPU_CUDA_TRY(cudaMemcpyAsync(cb[0], Ub(q), bytes, cudaMemcpyDeviceToDevice, s));
            double *q0 = reverse_products(Q(kids[0]), bs, bbars, d_gseg[sq], a_gbar[sq]);
            adj_add_interior<<<g, kBlock, 0, s>>>(L, 1, q0, Qb(kids[0]));
        }
    }
    SFGPU_CUDA_TRY(cudaGetLastError());
    return SFGPU_OK;
}

// primal residual evaluation that keeps what the reverse sweep reads:
// G of every state, every molecule's profiles and scalars, the state phi,
// the bulk terms, and the chains of the last polymer propagated
int sfgpu_system::primal_store(const double *x, double *f) {
    int rc;
    const DLat &L = H.L;
    const int g = grid_a(M);
    cudaStream_t s = stream;
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
    return SFGPU_OK;
}

int sfgpu_system::vjp_async(const double *x, const double *w, double *f, double *xbar) {
    int rc = ensure_adjoint();
    if (rc) return rc;
    const DLat &L = H.L;
    cudaStream_t s = stream;
    if ((rc = primal_store(x, f))) return rc;
    ResParam rp;
    memset(&rp, 0, sizeof(rp));
    rp.nsites = nsites; rp.nclass = nclass; rp.nseg = nseg;
    for (int c = 0; c < nclass; c++) { rp.rep[c] = rep_of_class[c]; rp.gfull[c] = d_gfull[rep_of_class[c]]; }
    for (int i = 0; i < nseg; i++) rp.phi[i] = d_phi[i];
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
    int held = (mols[solvent].type != 0 && !mols[solvent].ring && !mols[solvent].tree && !mols[solvent].dend) ? solvent : -1;
    if (held < 0)
        for (int m = nmol - 1; m >= 0 && held < 0; m--)
            if (m != solvent && mols[m].type != 0 && !mols[m].ring && !mols[m].tree && !mols[m].dend) held = m;
    if ((rc = molecule_adjoint(solvent, a_phibar.data()))) return rc;
    for (int m = nmol - 1; m >= 0; m--) {
        if (m == solvent) continue;
        if (mols[m].type != 0 && !mols[m].ring && !mols[m].tree && !mols[m].dend && m != held) {
            if ((rc = store_chains(m, false, nullptr))) return rc;
            held = m;
        }
        if ((rc = molecule_adjoint(m, a_phibar.data()))) return rc;
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

// F(x) and dF/dx by the reverse sweep: the free energy's direct
// cotangents (fe_contact_adj, fe_mol_phibar, fe_gbar, lncbar) feed the same
// molecule and SWF adjoints as the residual's.  x, xbar on the device.
int sfgpu_system::free_energy_grad(const double *x, double *F, double *xbar) {
    int rc = ensure_adjoint();
    if (rc) return rc;
    if (a_phibar_m.empty()) {
        a_phibar_m.assign(nseg, nullptr);
        for (int i = 0; i < nseg; i++)
            if ((rc = alloc_d(&a_phibar_m[i], M))) return rc;
    }
    const DLat &L = H.L;
    const int g = grid_a(M), np = nblocks_red;
    cudaStream_t s = stream;
    if ((rc = primal_store(x, d_f))) return rc;
    if ((rc = free_energy(F))) return rc;
    for (int i = 0; i < nseg; i++) {
        SFGPU_CUDA_TRY(cudaMemsetAsync(a_phibar[i], 0, sizeof(double) * M, s));
        SFGPU_CUDA_TRY(cudaMemsetAsync(a_gbar[i], 0, sizeof(double) * M, s));
    }
    FeAdjParam fp;
    memset(&fp, 0, sizeof(fp));
    fp.nseg = nseg;
    for (int i = 0; i < nseg; i++) { fp.phi[i] = d_phi[i]; fp.phibar[i] = a_phibar[i]; }
    fe_contact_adj<<<g, kBlock, 0, s>>>(L, fp, ct, d_wf);
    AdjScal *as = (AdjScal *)a_scal;
    const MolScal *scal = (const MolScal *)d_scal;
    fe_zero_scal<<<1, 1, 0, s>>>(nmol, as);
    for (int m = 0; m < nmol; m++) {
        HMol &o = mols[m];
        for (size_t a = 0; a < o.used.size(); a++)
            adj_dot_partial<<<np, kBlock, 0, s>>>(M, d_wf, o.d_phi[o.used[a]], d_partial + a * np);
        fe_set_lncbar<<<1, 1, 0, s>>>(np * (int)o.used.size(), d_partial, 1.0 / o.N, as, m);
        for (int i : o.used) fe_gbar<<<g, kBlock, 0, s>>>(M, o.d_phi[i], d_wf, d_gseg[i], a_gbar[i]);
    }
    auto mol_adj = [&](int m) -> int {
        HMol &o = mols[m];
        for (int i : o.used)
            fe_mol_phibar<<<g, kBlock, 0, s>>>(M, a_phibar[i], d_wf, d_gseg[i], 1.0 / o.N, log((double)o.N),
                                               o.chemintref, scal, m, a_phibar_m[i]);
        return molecule_adjoint(m, a_phibar_m.data());
    };
    int held = (mols[solvent].type != 0 && !mols[solvent].ring && !mols[solvent].tree && !mols[solvent].dend) ? solvent : -1;
    if (held < 0)
        for (int m = nmol - 1; m >= 0 && held < 0; m--)
            if (m != solvent && mols[m].type != 0 && !mols[m].ring && !mols[m].tree && !mols[m].dend) held = m;
    if ((rc = mol_adj(solvent))) return rc;
    for (int m = nmol - 1; m >= 0; m--) {
        if (m == solvent) continue;
        if (mols[m].type != 0 && !mols[m].ring && !mols[m].tree && !mols[m].dend && m != held) {
            if ((rc = store_chains(m, false, nullptr))) return rc;
            held = m;
        }
        if ((rc = mol_adj(m))) return rc;
    }
    SFGPU_CUDA_TRY(cudaMemsetAsync(xbar, 0, sizeof(double) * nvar, s));
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

// xbar = (d phi / dx)^T omega at fixed chi, for L = sum_i sum_z omega_i(z)
// phi_i(z) of the state profiles (omega: nseg device vectors of M)
int sfgpu_system::phi_vjp_async(const double *x, const double *const *omega, double *xbar) {
    int rc = ensure_adjoint();
    if (rc) return rc;
    cudaStream_t s = stream;
    if ((rc = primal_store(x, d_f))) return rc;
    for (int i = 0; i < nseg; i++) {
        SFGPU_CUDA_TRY(cudaMemcpyAsync(a_phibar[i], omega[i], sizeof(double) * M, cudaMemcpyDeviceToDevice, s));
        SFGPU_CUDA_TRY(cudaMemsetAsync(a_gbar[i], 0, sizeof(double) * M, s));
    }
    fe_zero_scal<<<1, 1, 0, s>>>(nmol, (AdjScal *)a_scal);
    int held = (mols[solvent].type != 0 && !mols[solvent].ring && !mols[solvent].tree && !mols[solvent].dend) ? solvent : -1;
    if (held < 0)
        for (int m = nmol - 1; m >= 0 && held < 0; m--)
            if (m != solvent && mols[m].type != 0 && !mols[m].ring && !mols[m].tree && !mols[m].dend) held = m;
    if ((rc = molecule_adjoint(solvent, a_phibar.data()))) return rc;
    for (int m = nmol - 1; m >= 0; m--) {
        if (m == solvent) continue;
        if (mols[m].type != 0 && !mols[m].ring && !mols[m].tree && !mols[m].dend && m != held) {
            if ((rc = store_chains(m, false, nullptr))) return rc;
            held = m;
        }
        if ((rc = molecule_adjoint(m, a_phibar.data()))) return rc;
    }
    SFGPU_CUDA_TRY(cudaMemsetAsync(xbar, 0, sizeof(double) * nvar, s));
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

// dchi = d (w . f(x)) / d chi at fixed x, nseg * nseg device values
int sfgpu_system::chi_vjp_async(const double *x, const double *w, double *dchi) {
    int rc = residual_async(x, d_f);
    if (rc) return rc;
    SFGPU_CUDA_TRY(cudaMemsetAsync(dchi, 0, sizeof(double) * (size_t)nseg * nseg, stream));
    ResParam rp;
    memset(&rp, 0, sizeof(rp));
    rp.nsites = nsites; rp.nclass = nclass; rp.nseg = nseg;
    for (int c = 0; c < nclass; c++) rp.rep[c] = rep_of_class[c];
    for (int i = 0; i < nseg; i++) rp.phi[i] = d_phi[i];
    adj_chi<<<grid_a(nsites), kBlock, 0, stream>>>(H.L, rp, d_sites, w, d_phib, dchi);
    SFGPU_CUDA_TRY(cudaGetLastError());
    return SFGPU_OK;
}

extern "C" int sfgpu_free_energy_grad(sfgpu_system *s, const double *x, double *F, double *xbar) {
    if (!s || !x || !F || !xbar) return SFGPU_ERR_INVALID;
    int rc = s->ensure_adjoint();
    if (rc) return rc;
    SFGPU_CUDA_TRY(cudaMemcpyAsync(s->d_x, x, sizeof(double) * s->nvar, cudaMemcpyHostToDevice, s->stream));
    if ((rc = s->free_energy_grad(s->d_x, F, s->a_xbar))) return rc;
    SFGPU_CUDA_TRY(cudaMemcpyAsync(xbar, s->a_xbar, sizeof(double) * s->nvar, cudaMemcpyDeviceToHost, s->stream));
    SFGPU_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return SFGPU_OK;
}

extern "C" int sfgpu_vjp(sfgpu_system *s, const double *x_dev, const double *w_dev, double *f_dev, double *xbar_dev) {
    if (!s) return SFGPU_ERR_INVALID;
    return s->vjp_async(x_dev, w_dev, f_dev, xbar_dev);
}

extern "C" int sfgpu_vjp_chi(sfgpu_system *s, const double *x, const double *w, double *dchi) {
    if (!s || !x || !w || !dchi) return SFGPU_ERR_INVALID;
    int rc = s->ensure_adjoint_misc();
    if (rc) return rc;
    cudaStream_t st = s->stream;
    const size_t nv = s->nvar;
    SFGPU_CUDA_TRY(cudaMemcpyAsync(s->d_x, x, sizeof(double) * nv, cudaMemcpyHostToDevice, st));
    SFGPU_CUDA_TRY(cudaMemcpyAsync(s->a_w, w, sizeof(double) * nv, cudaMemcpyHostToDevice, st));
    if ((rc = s->residual_async(s->d_x, s->d_f))) return rc;
    const int ns = s->nseg;
    SFGPU_CUDA_TRY(cudaMemsetAsync(s->a_xbar, 0, sizeof(double) * (size_t)ns * ns, st));
    ResParam rp;
    memset(&rp, 0, sizeof(rp));
    rp.nsites = s->nsites; rp.nclass = s->nclass; rp.nseg = ns;
    for (int c = 0; c < s->nclass; c++) rp.rep[c] = s->rep_of_class[c];
    for (int i = 0; i < ns; i++) rp.phi[i] = s->d_phi[i];
    adj_chi<<<grid_a(s->nsites), kBlock, 0, st>>>(s->H.L, rp, s->d_sites, s->a_w, s->d_phib, s->a_xbar);
    SFGPU_CUDA_TRY(cudaGetLastError());
    SFGPU_CUDA_TRY(cudaMemcpyAsync(dchi, s->a_xbar, sizeof(double) * (size_t)ns * ns, cudaMemcpyDeviceToHost, st));
    SFGPU_CUDA_TRY(cudaStreamSynchronize(st));
    return SFGPU_OK;
}

extern "C" int sfgpu_system_set_checkpoint(sfgpu_system *s, int stride) {
    if (!s) return SFGPU_ERR_INVALID;
    return s->set_checkpoint(stride);
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

// Checkpoint stride of the reverse sweep by measurement: every candidate
// (full storage; k = ceil(sqrt(N)) and k/2, 2k, N/4 of the longest chain)
// whose storage fits max_bytes (<= 0: no limit) is timed on `reps` reverse
// sweeps at x (host) with CUDA events on the system's stream after one
// untimed sweep; the fastest stays set.  Storage: 2N slices of K*M doubles
// in full, 2 ceil(N/k) + 2k + 1 with checkpoints.
extern "C" int sfgpu_system_autotune_checkpoint(sfgpu_system *s, const double *x, int reps, double max_bytes,
                                                int *stride, double *best_ms) {
    if (!s || !x || reps < 1) return SFGPU_ERR_INVALID;
    int nmax = 1;
    for (auto &o : s->mols) if (o.type != 0) nmax = std::max(nmax, o.N);
    const double slice = 8.0 * s->K * s->M;
    auto bytes = [&](int k) {
        if (k == 0) return 2.0 * nmax * slice;
        const double nq = (double)((nmax + k - 1) / k);
        return (2 * nq + 2.0 * k + 1) * slice;
    };
    const int r = std::max(1, (int)std::ceil(std::sqrt((double)nmax)));
    std::vector<int> cand = {0, r, std::max(1, r / 2), 2 * r, std::max(1, nmax / 4)};
    std::sort(cand.begin(), cand.end());
    cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
    cudaEvent_t e0, e1;
    SFGPU_CUDA_TRY(cudaEventCreate(&e0));
    SFGPU_CUDA_TRY(cudaEventCreate(&e1));
    int best = -1, rc = SFGPU_OK;
    double best_t = 0;
    for (int k : cand) {
        if (k >= nmax && k != 0) continue;
        if (max_bytes > 0 && bytes(k) > max_bytes) continue;
        if ((rc = s->set_checkpoint(k)) || (rc = s->ensure_adjoint())) break;
        if (cudaMemcpyAsync(s->d_x, x, sizeof(double) * s->nvar, cudaMemcpyHostToDevice, s->stream) != cudaSuccess) {
            rc = SFGPU_ERR_CUDA;
            break;
        }
        if ((rc = s->vjp_async(s->d_x, nullptr, s->d_f, s->a_xbar))) break;
        cudaEventRecord(e0, s->stream);
        for (int i = 0; i < reps && !rc; i++) rc = s->vjp_async(s->d_x, nullptr, s->d_f, s->a_xbar);
        cudaEventRecord(e1, s->stream);
        if (rc || cudaEventSynchronize(e1) != cudaSuccess) { if (!rc) rc = SFGPU_ERR_CUDA; break; }
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        const double t = ms / reps;
        if (best < 0 || t < best_t) { best = k; best_t = t; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    if (best < 0) { sfgpu_set_error(cudaErrorMemoryAllocation, "no checkpoint stride fits max_bytes", __FILE__, __LINE__); return SFGPU_ERR_NOMEM; }
    if ((rc = s->set_checkpoint(best))) return rc;
    if (stride) *stride = best;
    if (best_ms) *best_ms = best_t;
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
