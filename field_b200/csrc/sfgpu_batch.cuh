// sfgpu_batch.cuh -- one SF-SCF instance evaluated and iterated by ONE
// thread block.  The persistent batch kernel gives every block an instance
// from a work queue and the block runs the whole Pure_DIIS iteration
// (SFNewton::PlainLBFGSDIIS, sfnewton.cpp:566-664) on it: segment weighting
// factors, chain propagation with fused composition, normalisation, residual,
// Gram products and the DIIS combination, with __syncthreads between the
// propagator steps and no host round trip.  Uneven instances of a parameter
// sweep (Vary.cpp:127) therefore share the GPU without per-step launches.
#pragma once
#include <cuda_pipeline_primitives.h>
#include "sfgpu_kernels.cuh"

namespace sfb {

constexpr int kRing = 4;            // stored slices in flight in the shared-memory 1D path
constexpr int kMaxMol = SFGPU_MAX_SEG;
constexpr int kMaxHist = 16;        // DIIS memory m supported by the batch path

struct IMol {
    int N, type, sym, freedom, pinned, solvent, nused;
    int used[SFGPU_MAX_SEG];
    const int *seg;                 // device: segment of each chain position
    double *phi[SFGPU_MAX_SEG];     // per segment, nullptr when unused
    double phibulk, theta;
};

struct InstDesc {
    DLat L;
    int M, nseg, nmol, nclass, nsites, solvent;
    int gstage;                     // G of the running segment staged in shared memory
    int small1d;                    // 1D symmetric homopolymers: running slices, phi and a ring of
                                    // kRing stored slices in shared memory too
    long long nvar;
    int freedom[SFGPU_MAX_SEG];
    int class_of[SFGPU_MAX_SEG];
    int rep[SFGPU_MAX_SEG];
    ChiTable ct;
    double frac[SFGPU_MAX_SEG * SFGPU_MAX_SEG];     // [seg][mol] = count/N
    const int *jmap, *sites;
    const double *w_gn;
    const double *range[SFGPU_MAX_SEG];
    double *gfull[SFGPU_MAX_SEG], *gseg[SFGPU_MAX_SEG], *phi[SFGPU_MAX_SEG];
    IMol mol[kMaxMol];
    double *gi, *ginv0, *ginv1;
    // iteration work
    double *x, *x0, *g, *XR, *XX0;
    // mol : force (wide kernel): bit m of fmask marks molecule m, whose
    // forward and backward step weights are fw[2m], fw[2m + 1]
    int fmask;
    const sfk::ForceW *fw;
};

struct BlockShared {
    double red[32 * (kMaxHist + 2)];
    double val[kMaxHist + 2];
    sfk::MolScal scal[kMaxMol];
    double phib[SFGPU_MAX_SEG], chib[SFGPU_MAX_SEG];
    double gram[kMaxHist * kMaxHist];
    double A[kMaxHist * kMaxHist], Q[kMaxHist * kMaxHist];   // DIIS eigen-solve work
    double coef[kMaxHist];
    int pos[kMaxHist];
    int inst;
};

// Sum of per-thread values over the block in a fixed order (warp shuffle
// tree, then warps in index order): sh.val[slot[i]] = block sum of v[i] for
// every i < NMAX with slot[i] >= 0.  v is a register array, indexed only
// with compile-time constants so that it never goes to local memory.
template <int NMAX>
__device__ __forceinline__ void block_sums_slots(const double (&v)[NMAX], const int (&slot)[NMAX], BlockShared &sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    int nv = 0;
#pragma unroll
    for (int i = 0; i < NMAX; i++) {
        if (slot[i] < 0) continue;
        double a = v[i];
        for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
        if (lane == 0) sh.red[slot[i] * 32 + warp] = a;
        nv = max(nv, slot[i] + 1);
    }
    __syncthreads();
    if (threadIdx.x < nv) {
        double a = 0;
        for (int w = 0; w < nw; w++) a += sh.red[threadIdx.x * 32 + w];
        sh.val[threadIdx.x] = a;
    }
    __syncthreads();
}
// one value per thread: sh.val[0]
__device__ __forceinline__ void block_sum1(double v, BlockShared &sh) {
    const double a[1] = {v};
    const int sl[1] = {0};
    block_sums_slots<1>(a, sl, sh);
}

__device__ __forceinline__ void mol_scalars_block(const InstDesc &I, int m, double wsum, BlockShared &sh) {
    const IMol &o = I.mol[m];
    sfk::MolScal s;
    s.lngn = log(wsum);
    double phib = o.phibulk;
    if (o.solvent) {
        phib = 1.0;
        for (int q = 0; q < I.nmol; q++)
            if (q != m) phib -= sh.scal[q].phibulk;
    }
    const double N = (double)o.N;
    double gn = exp(s.lngn);
    if (o.freedom == SFGPU_MOL_RESTRICTED) {
        if (o.type == 0) { s.lnc = log(o.theta) - s.lngn; s.norm = o.theta / gn; }
        else {
            s.lnc = log(o.theta) - s.lngn - log(1.0 * o.N);
            s.norm = (o.sym ? 2 * o.theta / N : o.theta / N) / gn;
        }
        s.phibulk = o.theta / gn;
    } else {
        s.phibulk = phib;
        if (o.type == 0) { s.lnc = log(phib); s.norm = phib; }
        else { s.lnc = log(phib / N); s.norm = o.sym ? 2 * phib / N : phib / N; }
    }
    if (o.pinned) s.phibulk = 0;
    sh.scal[m] = s;
}

// lnGN sum, scalars and normalised phi of molecule m; cur = end-point
// distribution (Gi_inv after the backward pass)
__device__ __forceinline__ void finish_molecule(const InstDesc &I, int m, const double *cur, BlockShared &sh) {
    const IMol &o = I.mol[m];
    double acc = 0;
    for (int r = threadIdx.x; r < I.M; r += blockDim.x) {
        double w = I.w_gn[r];
        if (w != 0) acc += w * cur[r];
    }
    block_sum1(acc, sh);
    if (threadIdx.x == 0) mol_scalars_block(I, m, sh.val[0], sh);
    __syncthreads();
    const double norm = sh.scal[m].norm;
    for (int a = 0; a < o.nused; a++) {
        int i = o.used[a];
        const double *G = I.gseg[i];
        double *phi = o.phi[i];
        for (int r = threadIdx.x; r < I.M; r += blockDim.x) {
            double p;
            if (o.type == 0) p = G[r];
            else { double g = G[r]; p = (g > 0) ? phi[r] / g : 0.0; }
            phi[r] = p * norm;
        }
    }
    if (o.type == 0) return;
    // boundary entries of phi: copies of the mapped sites (row-wise steps
    // leave them untouched)
    __syncthreads();
    for (int a = 0; a < o.nused; a++) {
        double *phi = o.phi[o.used[a]];
        for (int r = threadIdx.x; r < I.M; r += blockDim.x) {
            int c[3];
            lat_coords(I.L, r, c);
            if (lat_interior(I.L, c)) continue;
            int t = lat_map(I.L, r);
            if (t != r) phi[r] = phi[t];
        }
    }
}

// SF_Homopol1stO::Matrix1 / SF_Copol1stO::Matrix1 / SF_Monomer1stO::Matrix1
// inside one block (first-order lattices)
//
// G of a run of equal segments is constant over the run's steps, so when the
// lattice fits (I.gstage) it is copied once per run into the block's dynamic
// shared memory and the steps read it there instead of streaming it from L2
// in every step.
// One step of a linear chain in the wide kernel: the constant-force step
// where the molecule has a force (forward +f, backward -f weights), else the
// first-order step of any lattice type.
__device__ __forceinline__ double chain_step_wide(const DLat &L, const InstDesc &I, int m, const RowInfo &R,
                                                  const double *src, const double *G, int k, int nlast, bool fwd) {
    if ((I.fmask >> m) & 1) return force_row(L, R, src, G, k, nlast, I.fw[2 * m + (fwd ? 0 : 1)]);
    return prop1_row<true>(L, R, src, G, k, nlast);
}

template <bool kWide>
__device__ inline void molecule_phi_block(const InstDesc &I, int m, BlockShared &sh) {
    extern __shared__ double g_stage[];
    const IMol &o = I.mol[m];
    const DLat &L = I.L;
    const int M = I.M;
    if (o.type == 0) { finish_molecule(I, m, I.gseg[o.seg[0]], sh); return; }
    int staged = -1;   // segment whose G is in g_stage (block-uniform)
    auto gof = [&](int sg) -> const double * {
        if (!I.gstage) return I.gseg[sg];
        if (sg != staged) {
            __syncthreads();
            const double *src = I.gseg[sg];
            for (int r = threadIdx.x; r < M; r += blockDim.x) g_stage[r] = src[r];
            __syncthreads();
            staged = sg;
        }
        return g_stage;
    };
    for (int a = 0; a < o.nused; a++) {
        double *phi = o.phi[o.used[a]];
        for (int r = threadIdx.x; r < M; r += blockDim.x) phi[r] = 0.0;
    }
    double *gi = I.gi;
    double *bufA = I.ginv0, *bufB = I.ginv1;
    if (o.sym && I.small1d && I.gstage) {
        // 1D lattices small enough to keep the whole step in shared memory:
        // the running propagator slice (two buffers) and the molecule's phi
        // sit next to the staged G, so a step reads only shared memory and
        // the stored half chain (gi), and writes gi; each step costs a
        // shared-memory round trip and a block barrier instead of an L2 one.
        // Same operands and operation order as the path below.
        const int sg = o.seg[0];
        const double *G = gof(sg);
        double *sa = g_stage + M, *sb = sa + M, *sphi = sb + M;
        const int N = o.N, half = N / 2;
        for (int r = threadIdx.x; r < M; r += blockDim.x) {
            const double gv = G[r];
            sa[r] = gv;
            gi[r] = gv;
            sb[r] = 0.0;
            sphi[r] = 0.0;
        }
        __syncthreads();
        for (int t = 1; t < half; t++) {
            double *dst = gi + (size_t)t * M;
            for_interior4(L, threadIdx.x, blockDim.x,
                [&](const RowInfo &R, int k, int nlast) { return prop1_row<false>(L, R, sa, G, k, nlast); },
                [&](const RowInfo &R, int k, double v) { sb[R.base + k] = v; dst[R.base + k] = v; });
            __syncthreads();
            double *tt = sa; sa = sb; sb = tt;
        }
        if (N % 2 == 1) {
            for_interior4(L, threadIdx.x, blockDim.x,
                [&](const RowInfo &R, int k, int nlast) { return prop1_row<false>(L, R, sa, G, k, nlast); },
                [&](const RowInfo &R, int k, double out) {
                    const int z = R.base + k;
                    sb[z] = out;
                    sphi[z] = (sphi[z] + out * out) * 0.5;
                });
            __syncthreads();
            double *tt = sa; sa = sb; sb = tt;
        }
        // backward sweep: the stored slice each step composes with streams
        // into a ring of kRing shared-memory slices by asynchronous copies
        // issued kRing steps ahead, so its L2 latency hides behind the steps
        // in between.  Every thread copies exactly the positions it later
        // reads, so the copy group's completion (no barrier) makes them
        // visible to it.
        double *ring = sphi + M;
        const int nlast = L.Md[0] - 2;
        const RowInfo R0 = lat_row(L, 0);
        const int sp0 = (N + 3) / 2, nsteps = N - sp0 + 1;
        auto issue = [&](int j) {
            if (j < nsteps) {
                const double *src = gi + (size_t)(N - sp0 - j) * M;
                double *dst = ring + (size_t)(j % kRing) * M;
                for (int k = threadIdx.x + 1; k <= nlast; k += blockDim.x)
                    __pipeline_memcpy_async(dst + k, src + k, sizeof(double));
            }
            __pipeline_commit();
        };
        for (int j = 0; j < kRing; j++) issue(j);
        for (int j = 0; j < nsteps; j++) {
            __pipeline_wait_prior(kRing - 1);
            const double *ot = ring + (size_t)(j % kRing) * M;
            for (int k = threadIdx.x + 1; k <= nlast; k += blockDim.x) {
                const double ph = sphi[k], o2 = ot[k];
                const double out = prop1_row<false>(L, R0, sa, G, k, nlast);
                sb[k] = out;
                sphi[k] = ph + out * o2;
            }
            __syncthreads();
            issue(j + kRing);
            double *tt = sa; sa = sb; sb = tt;
        }
        __pipeline_wait_prior(0);
        double *phi = o.phi[sg];
        for (int r = threadIdx.x; r < M; r += blockDim.x) phi[r] = sphi[r];
        __syncthreads();
        finish_molecule(I, m, sa, sh);
        __syncthreads();
        return;
    }
    if (o.sym) {
        const int sg = o.seg[0];
        const double *G = gof(sg);
        double *phi = o.phi[sg];
        const int N = o.N, half = N / 2;
        for (int r = threadIdx.x; r < M; r += blockDim.x) gi[r] = G[r];
        __syncthreads();
        for (int t = 1; t < half; t++) {
            const double *src = gi + (size_t)(t - 1) * M;
            double *dst = gi + (size_t)t * M;
            for_interior4(L, threadIdx.x, blockDim.x,
                [&](const RowInfo &R, int k, int nlast) { return prop1_row<kWide>(L, R, src, G, k, nlast); },
                [&](const RowInfo &R, int k, double v) { dst[R.base + k] = v; });
            __syncthreads();
        }
        const double *cur = gi + (size_t)(half - 1) * M;
        if (N % 2 == 1) {
            double *dst = bufA;
            for_interior4(L, threadIdx.x, blockDim.x,
                [&](const RowInfo &R, int k, int nlast) { return prop1_row<kWide>(L, R, cur, G, k, nlast); },
                [&](const RowInfo &R, int k, double out) {
                    const int z = R.base + k;
                    dst[z] = out;
                    phi[z] = (phi[z] + out * out) * 0.5;
                });
            __syncthreads();
            cur = bufA; double *t = bufA; bufA = bufB; bufB = t;
        }
        for (int sp = (N + 3) / 2; sp <= N; sp++) {
            const double *other = gi + (size_t)(N - sp) * M;
            double *dst = bufA;
            for_interior4_acc(L, threadIdx.x, blockDim.x, phi, other,
                [&](const RowInfo &R, int k, int nlast) { return prop1_row<kWide>(L, R, cur, G, k, nlast); },
                [&](const RowInfo &R, int k, double out, double ph, double ot) {
                    const int z = R.base + k;
                    dst[z] = out;
                    phi[z] = ph + out * ot;
                });
            __syncthreads();
            cur = bufA; double *t = bufA; bufA = bufB; bufB = t;
        }
        finish_molecule(I, m, cur, sh);
        return;
    }
    const int N = o.N;
    {
        const double *G1 = I.gseg[o.seg[0]];
        for (int r = threadIdx.x; r < M; r += blockDim.x) gi[r] = G1[r];
        __syncthreads();
    }
    for (int t = 1; t < N; t++) {
        const double *src = gi + (size_t)(t - 1) * M;
        double *dst = gi + (size_t)t * M;
        const double *G = gof(o.seg[t]);
        for_interior4(L, threadIdx.x, blockDim.x,
            [&](const RowInfo &R, int k, int nlast) {
                if constexpr (kWide) return chain_step_wide(L, I, m, R, src, G, k, nlast, true);
                else return prop1_row<false>(L, R, src, G, k, nlast);
            },
            [&](const RowInfo &R, int k, double v) { dst[R.base + k] = v; });
        __syncthreads();
    }
    {
        const int sN = o.seg[N - 1];
        const double *GN = I.gseg[sN];
        const double *gf = gi + (size_t)(N - 1) * M;
        double *phi = o.phi[sN];
        for (int r = threadIdx.x; r < M; r += blockDim.x) {
            double g = GN[r];
            bufA[r] = g;
            phi[r] += g * gf[r];
        }
        __syncthreads();
    }
    const double *cur = bufA;
    { double *t = bufA; bufA = bufB; bufB = t; }
    for (int t = N - 2; t >= 0; t--) {
        const int sg = o.seg[t];
        const double *G = gof(sg);
        const double *gf = gi + (size_t)t * M;
        double *phi = o.phi[sg];
        double *dst = bufA;
        for_interior4_acc(L, threadIdx.x, blockDim.x, phi, gf,
            [&](const RowInfo &R, int k, int nlast) {
                if constexpr (kWide) return chain_step_wide(L, I, m, R, cur, G, k, nlast, false);
                else return prop1_row<false>(L, R, cur, G, k, nlast);
            },
            [&](const RowInfo &R, int k, double out, double ph, double ot) {
                const int z = R.base + k;
                dst[z] = out;
                phi[z] = ph + out * ot;
            });
        __syncthreads();
        cur = bufA; double *tt = bufA; bufA = bufB; bufB = tt;
    }
    finish_molecule(I, m, cur, sh);
}

// f at iteration site j (lattice site z) of SF_Solve::GetResiduals
// (SF_Solve.cpp:527-591) once phi and the bulk terms (sh.chib) are known.
// Segment types and classes are bounded by kResMax so that the per-site
// contact averages and potentials stay in registers; the sums run in the
// same order as the single-system kernel.
constexpr int kResMax = 8;
template <bool kWide>
__device__ __forceinline__ void site_residual(const InstDesc &I, const BlockShared &sh, int j, double *f) {
    const DLat &L = I.L;
    const int z = I.sites[j];
    const int nseg = I.nseg, ncl = I.nclass;
    double phit = 0;
    double rho[kResMax];
#pragma unroll
    for (int i = 0; i < kResMax; i++) {
        rho[i] = 0;
        if (i < nseg) phit += I.phi[i][z];
    }
#pragma unroll
    for (int i = 0; i < kResMax; i++) {
        if (i >= nseg) continue;
        bool need = false;
        for (int c = 0; c < ncl; c++) need |= I.ct.chi[I.rep[c] * SFGPU_MAX_SEG + i] != 0;
        if (need) rho[i] = side_fraction<kWide>(L, I.phi[i], z);
    }
    double u[kResMax];
    double av = 0;
#pragma unroll
    for (int c = 0; c < kResMax; c++) {
        u[c] = 0;
        if (c >= ncl) continue;
        const int st = I.rep[c];
        double v = -log(I.gfull[st][z]);
        double ci = 0;
#pragma unroll
        for (int i = 0; i < kResMax; i++) {
            if (i >= nseg) continue;
            const double xx = I.ct.chi[st * SFGPU_MAX_SEG + i];
            if (xx != 0) ci += xx * rho[i];
        }
        v -= ci / phit;
        v += sh.chib[c];
        u[c] = v;
        av += v;
    }
    av /= ncl;
#pragma unroll
    for (int c = 0; c < kResMax; c++)
        if (c < ncl) f[(size_t)j * ncl + c] = -1.0 + 1.0 / phit + u[c] - av;
}

// x -> f for one instance (SF_Solve::residuals, SF_Solve.cpp:647-651)
template <bool kWide>
__device__ inline void residual_block(const InstDesc &I, const double *x, double *f, BlockShared &sh) {
    const DLat &L = I.L;
    const int M = I.M;
    for (int i = 0; i < I.nseg; i++) {
        if (I.freedom[i] == SFGPU_SEG_FROZEN) continue;
        const int cls = I.class_of[i];
        const bool pinned = I.freedom[i] == SFGPU_SEG_PINNED;
        double *gf = I.gfull[i], *gs = I.gseg[i];
        const double *range = I.range[i];
        for (int r = threadIdx.x; r < M; r += blockDim.x) {
            int t = lat_map(L, r);
            int j = I.jmap[t];
            double v = (j >= 0) ? exp(-x[(size_t)j * I.nclass + cls]) : 0.0;
            gf[r] = v;
            gs[r] = pinned ? (range[t] > 0 ? v : 0.0) : v;
        }
    }
    __syncthreads();
    for (int m = 0; m < I.nmol; m++) {
        if (m == I.solvent) continue;
        molecule_phi_block<kWide>(I, m, sh);
        __syncthreads();
    }
    molecule_phi_block<kWide>(I, I.solvent, sh);
    __syncthreads();
    for (int i = 0; i < I.nseg; i++) {
        if (I.freedom[i] == SFGPU_SEG_FROZEN) continue;
        double *p = I.phi[i];
        for (int r = threadIdx.x; r < M; r += blockDim.x) {
            double acc = 0;
            for (int m = 0; m < I.nmol; m++) {
                const double *q = I.mol[m].phi[i];
                if (q) acc += q[r];
            }
            p[r] = acc;
        }
    }
    if (threadIdx.x == 0) {
        for (int i = 0; i < I.nseg; i++) {
            double v = 0;
            for (int m = 0; m < I.nmol; m++) v += sh.scal[m].phibulk * I.frac[i * SFGPU_MAX_SEG + m];
            sh.phib[i] = v;
        }
        for (int c = 0; c < I.nclass; c++) {
            int st = I.rep[c];
            double v = 0;
            for (int j = 0; j < I.nseg; j++) {
                double xx = I.ct.chi[st * SFGPU_MAX_SEG + j];
                if (xx != 0) v += xx * sh.phib[j];
            }
            sh.chib[c] = v;
        }
    }
    __syncthreads();
    for (int j = threadIdx.x; j < I.nsites; j += blockDim.x) site_residual<kWide>(I, sh, j, f);
    __syncthreads();
}

// DIIS coefficients c = A^-1 1 through the eigen-decomposition of the
// symmetric Gram matrix by cyclic Jacobi (the oracle's jacobi_eig: same
// rotation order, same per-element expressions), run by one warp on A and Q
// in shared memory: lane k owns row / column k of each rotation, lane 0 takes
// the convergence sums in the serial order, so the result is bit-identical
// to the serial form (n <= kMaxHist <= 32).
__device__ __forceinline__ void diis_coeff_warp(int n, double *A, double *Q, double *c) {
    const int lane = threadIdx.x & 31;
    const unsigned full = 0xffffffffu;
    for (int i = lane; i < n * n; i += 32) Q[i] = (i / n == i % n);
    __syncwarp();
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0, tot = 0;
        if (lane == 0) {
            for (int i = 0; i < n; i++)
                for (int j = 0; j < n; j++) {
                    tot += A[i * n + j] * A[i * n + j];
                    if (i != j) off += A[i * n + j] * A[i * n + j];
                }
        }
        off = __shfl_sync(full, off, 0);
        tot = __shfl_sync(full, tot, 0);
        if (off <= 1e-30 * tot || off == 0) break;
        for (int p = 0; p < n; p++)
            for (int q = p + 1; q < n; q++) {
                const double apq = A[p * n + q];
                if (apq == 0) continue;
                const double theta = (A[q * n + q] - A[p * n + p]) / (2 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1));
                const double cs = 1 / sqrt(t * t + 1), sn = t * cs;
                __syncwarp();
                if (lane < n) {
                    const int k = lane;
                    const double akp = A[k * n + p], akq = A[k * n + q];
                    A[k * n + p] = cs * akp - sn * akq; A[k * n + q] = sn * akp + cs * akq;
                    const double qkp = Q[k * n + p], qkq = Q[k * n + q];
                    Q[k * n + p] = cs * qkp - sn * qkq; Q[k * n + q] = sn * qkp + cs * qkq;
                }
                __syncwarp();
                if (lane < n) {
                    const int k = lane;
                    const double apk = A[p * n + k], aqk = A[q * n + k];
                    A[p * n + k] = cs * apk - sn * aqk; A[q * n + k] = sn * apk + cs * aqk;
                }
                __syncwarp();
            }
    }
    if (lane < n) {
        const int i = lane;
        double ci = 0;
        for (int k = 0; k < n; k++) {
            double proj = 0;
            for (int j = 0; j < n; j++) proj += Q[j * n + k];
            const double t = proj / A[k * n + k];
            ci += Q[i * n + k] * t;
        }
        c[i] = ci;
    }
    __syncwarp();
}

}  // namespace sfb
