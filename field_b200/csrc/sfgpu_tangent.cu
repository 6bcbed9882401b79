// sfgpu_tangent.cu -- exact Jacobian-vector products of the residual
// (forward-mode tangent of SF_Solve::residuals) and a Newton-Krylov iteration
// built on them (GMRES with exact J*v in place of the finite-difference
// products of SFNewton's truncated Newton, sfnewton.cpp:1662-1688).
#include <algorithm>
#include <functional>
#include <cmath>
#include <cstring>
#include <vector>
#include "sfgpu_tangent.cuh"
#include "sfgpu_system.h"

using namespace sfk;
using namespace sft;

static int grid_n(long n) {
    long b = (n + kBlock - 1) / kBlock;
    return (int)std::max(1L, std::min(b, 148L * 16));
}
static int grid_rows_t(const DLat &L) {
    long threads = (L.grad == 1) ? (long)(L.Md[0] - 2) : 32L * lat_nrows(L);
    long b = (threads + kBlock - 1) / kBlock;
    return (int)std::max(1L, std::min(b, 148L * 32));
}

int sfgpu_system::ensure_tangent() {
    if (logmode) return fail_unsupported("derivatives with overflow protection");
    if (charged) return fail_unsupported("derivatives of charged systems");
    for (auto &o : mols)
        if (o.dend) build_dend_tree(o);
    if (t_ready) return SFGPU_OK;
    int rc;
    dgfull.assign(nseg, nullptr); dgseg.assign(nseg, nullptr); dphi.assign(nseg, nullptr);
    for (int i = 0; i < nseg; i++) {
        if ((rc = alloc_d(&dphi[i], M))) return rc;
        SFGPU_CUDA_TRY(cudaMemset(dphi[i], 0, sizeof(double) * M));   // frozen states: 0
        if (freedom[i] == SFGPU_SEG_FROZEN) continue;
        if ((rc = alloc_d(&dgfull[i], M))) return rc;
        if ((rc = alloc_d(&dgseg[i], M))) return rc;
    }
    for (auto &o : mols) {
        o.d_dphi.assign(nseg, nullptr);
        for (int i : o.used) if ((rc = alloc_d(&o.d_dphi[i], M))) return rc;
    }
    size_t store = 0;
    for (auto &o : mols) {
        size_t need = (o.type == 0 || o.ring) ? 0
                      : (size_t)((o.tree || o.dend) ? 3 * o.N : o.sym ? std::max(1, o.N / 2) : o.N) * K * M;
        store = std::max(store, need);
    }
    if ((rc = alloc_d(&d_dgi, store))) return rc;
    // checkpointed primal storage holds fewer slices than the tangent sweeps write
    // (and a dendrimer's primal keeps one path, its tree three slices per segment)
    bool ck = false;
    for (auto &o : mols) ck |= primal_checkpointed(o) || o.dend;
    t_gi = d_gi;
    if (ck) {
        if ((rc = alloc_d(&t_gi, store))) return rc;
        SFGPU_CUDA_TRY(cudaMemset(t_gi, 0, sizeof(double) * std::max<size_t>(store, 1)));
    }
    if ((rc = alloc_d(&t_w[0], (size_t)K * M)) || (rc = alloc_d(&t_w[1], (size_t)K * M))) return rc;
    SFGPU_CUDA_TRY(cudaMemset(t_w[0], 0, sizeof(double) * K * M));
    SFGPU_CUDA_TRY(cudaMemset(t_w[1], 0, sizeof(double) * K * M));
    if ((rc = alloc_d(&d_dginv[0], (size_t)K * M)) || (rc = alloc_d(&d_dginv[1], (size_t)K * M))) return rc;
    SFGPU_CUDA_TRY(cudaMemset(d_dgi, 0, sizeof(double) * std::max<size_t>(store, 1)));
    SFGPU_CUDA_TRY(cudaMemset(d_dginv[0], 0, sizeof(double) * K * M));
    SFGPU_CUDA_TRY(cudaMemset(d_dginv[1], 0, sizeof(double) * K * M));
    if ((rc = alloc_d(&d_tscal, 4 * (size_t)nmol))) return rc;
    SFGPU_CUDA_TRY(cudaMemset(d_tscal, 0, sizeof(MolScalT) * nmol));
    if ((rc = alloc_d(&d_dpartial, (size_t)std::max(nblocks_red, 64) * 64))) return rc;
    if ((rc = alloc_d(&d_dphib, nseg)) || (rc = alloc_d(&d_dchib, nclass))) return rc;
    if ((rc = alloc_d(&d_v, nvar)) || (rc = alloc_d(&d_jv, nvar))) return rc;
    t_ready = true;
    return SFGPU_OK;
}

int sfgpu_system::molecule_phi_t(int m) {
    if (mols[m].dend) {
        // a dendrimer's derivatives: the bond-tree recursion on its tree form
        build_dend_tree(mols[m]);
        dend_view(mols[m], true);
        const int rc = molecule_phi_t(m);
        dend_view(mols[m], false);
        return rc;
    }
    HMol &o = mols[m];
    const DLat &L = H.L;
    const int g = grid_n(M), gr = grid_rows_t(L);
    cudaStream_t s = stream;
    MolParam p;
    p.N = o.N; p.type = o.type; p.freedom = o.freedom; p.sym = o.sym; p.K = K;
    p.pinned = o.pinned; p.solvent = (m == solvent); p.nmol = nmol;
    p.phibulk_in = o.phibulk; p.theta = o.theta;
    MolScal *scal = (MolScal *)d_scal;
    MolScalT *tscal = (MolScalT *)d_tscal;
    const size_t KM = (size_t)K * M;
    if (o.type == 0) {
        int i = o.seg[0];
        MolParam p1 = p; p1.K = 1;
        wsum_partial<<<nblocks_red, kBlock, 0, s>>>(M, 1, d_gseg[i], d_wgn, d_partial);
        wsum_partial<<<nblocks_red, kBlock, 0, s>>>(M, 1, dgseg[i], d_wgn, d_dpartial);
        mol_scalars<<<1, 1, 0, s>>>(p1, nblocks_red, d_partial, scal, m);
        mol_scalars_t<<<1, 1, 0, s>>>(p1, nblocks_red, d_dpartial, scal, tscal, m);
        finalize_phi_t<<<g, kBlock, 0, s>>>(M, d_gseg[i], dgseg[i], o.d_phi[i], o.d_dphi[i], scal, tscal, m, 1);
        return SFGPU_OK;
    }
    if (o.ring) {
        // the ring's walk with its tangent; lnGN, ln C and phibulk are
        // constants of the ring (ring_scalars), their tangents 0
        const int Mmax = (o.N / 2 > M) ? 2 * M : M + o.N / 2;
        const size_t shm = (size_t)4 * (Mmax + 1) * sizeof(double);
        if (shm > 200 * 1024) return fail_unsupported("the tangent of a ring walk larger than shared memory");
        if (shm > 48 * 1024)
            SFGPU_CUDA_TRY(cudaFuncSetAttribute(ring_phi_t, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
        const int sg = o.seg[0];
        ring_phi_t<<<std::min(M, 148 * 8), Mmax + 1 >= 256 ? 256 : 64, shm, s>>>(
            M, o.N, Mmax, d_gseg[sg], dgseg[sg], o.phibulk, o.ring_norm0, o.d_phi[sg], o.d_dphi[sg]);
        SFGPU_CUDA_TRY(cudaGetLastError());
        set_boundaries<<<g, kBlock, 0, s>>>(L, 1, o.d_phi[sg]);
        set_boundaries<<<g, kBlock, 0, s>>>(L, 1, o.d_dphi[sg]);
        ring_scalars<<<1, 1, 0, s>>>(o.N, o.phibulk, scal, m);
        SFGPU_CUDA_TRY(cudaMemsetAsync(tscal + m, 0, sizeof(MolScalT), s));
        return SFGPU_OK;
    }
    const double *cur = nullptr, *dcur = nullptr;
    if (o.tree) {
        // the bond-tree recursion of molecule_phi_tree with tangents: steps
        // by step1_rows_t, products by combine_t, compositions by connect_t
        const int N = o.N;
        auto U = [&](int q) { return t_gi + (size_t)q * M; };
        auto Q = [&](int q) { return t_gi + (size_t)(N + q) * M; };
        auto D = [&](int q) { return t_gi + (size_t)(2 * N + q) * M; };
        auto dU = [&](int q) { return d_dgi + (size_t)q * M; };
        auto dQ = [&](int q) { return d_dgi + (size_t)(N + q) * M; };
        auto dD = [&](int q) { return d_dgi + (size_t)(2 * N + q) * M; };
        const size_t bytes = sizeof(double) * M;
        for (int i : o.used) {
            SFGPU_CUDA_TRY(cudaMemsetAsync(o.d_phi[i], 0, bytes, s));
            SFGPU_CUDA_TRY(cudaMemsetAsync(o.d_dphi[i], 0, bytes, s));
        }
        auto stepT = [&](const double *in, const double *din, int sgq, double *out, double *dout) {
            step1_rows_t<<<gr, kBlock, 0, s>>>(L, in, din, d_gseg[sgq], dgseg[sgq], out, dout, nullptr, nullptr,
                                               nullptr, nullptr, COMP_NONE);
        };
        for (int q = N - 1; q >= 0; q--) {
            const int sq = o.seg[q];
            const std::vector<int> &kids = o.kids[q];
            if (kids.empty()) {
                SFGPU_CUDA_TRY(cudaMemcpyAsync(U(q), d_gseg[sq], bytes, cudaMemcpyDeviceToDevice, s));
                SFGPU_CUDA_TRY(cudaMemcpyAsync(dU(q), dgseg[sq], bytes, cudaMemcpyDeviceToDevice, s));
            } else if (kids.size() == 1) {
                SFGPU_CUDA_TRY(cudaMemcpyAsync(U(q), Q(kids[0]), bytes, cudaMemcpyDeviceToDevice, s));
                SFGPU_CUDA_TRY(cudaMemcpyAsync(dU(q), dQ(kids[0]), bytes, cudaMemcpyDeviceToDevice, s));
            } else {
                const double *acc = Q(kids[0]), *dacc = dQ(kids[0]);
                int w = 0;
                for (size_t c = 1; c < kids.size(); c++) {
                    const bool last = c + 1 == kids.size();
                    double *dst = last ? U(q) : d_ginv[w], *ddst = last ? dU(q) : d_dginv[w];
                    combine_t<<<g, kBlock, 0, s>>>(M, acc, dacc, Q(kids[c]), dQ(kids[c]), d_gseg[sq], dgseg[sq], dst,
                                                   ddst);
                    acc = dst; dacc = ddst;
                    w ^= 1;
                }
            }
            if (q > 0) stepT(U(q), dU(q), o.seg[o.parent[q]], Q(q), dQ(q));
        }
        SFGPU_CUDA_TRY(cudaMemcpyAsync(D(0), d_gseg[o.seg[0]], bytes, cudaMemcpyDeviceToDevice, s));
        SFGPU_CUDA_TRY(cudaMemcpyAsync(dD(0), dgseg[o.seg[0]], bytes, cudaMemcpyDeviceToDevice, s));
        for (int q = 0; q < N; q++) {
            const int sq = o.seg[q];
            connect_t<<<g, kBlock, 0, s>>>(M, 1, U(q), dU(q), D(q), dD(q), o.d_phi[sq], o.d_dphi[sq]);
            const std::vector<int> &kids = o.kids[q];
            for (int c : kids) {
                const double *acc = D(q), *dacc = dD(q);
                int w = 0;
                for (int c2 : kids) {
                    if (c2 == c) continue;
                    combine_t<<<g, kBlock, 0, s>>>(M, acc, dacc, Q(c2), dQ(c2), d_gseg[sq], dgseg[sq], d_ginv[w],
                                                   d_dginv[w]);
                    acc = d_ginv[w]; dacc = d_dginv[w];
                    w ^= 1;
                }
                stepT(acc, dacc, o.seg[c], D(c), dD(c));
            }
        }
        cur = U(0);
        dcur = dU(0);
    } else {
    for (int i : o.used) {
        SFGPU_CUDA_TRY(cudaMemsetAsync(o.d_phi[i], 0, sizeof(double) * M, s));
        SFGPU_CUDA_TRY(cudaMemsetAsync(o.d_dphi[i], 0, sizeof(double) * M, s));
    }
    double *ginv = d_ginv[0], *tmp = d_ginv[1], *dginv = d_dginv[0], *dtmp = d_dginv[1];
    if (o.sym) {
        const int i = o.seg[0];
        const double *G = d_gseg[i], *dG = dgseg[i];
        const int N = o.N, half = N / 2;
        double *phi = o.d_phi[i], *dph = o.d_dphi[i];
        SFGPU_CUDA_TRY(cudaMemcpyAsync(t_gi, G, sizeof(double) * M, cudaMemcpyDeviceToDevice, s));
        SFGPU_CUDA_TRY(cudaMemcpyAsync(d_dgi, dG, sizeof(double) * M, cudaMemcpyDeviceToDevice, s));
        for (int t = 1; t < half; t++)
            step1_rows_t<<<gr, kBlock, 0, s>>>(L, t_gi + (size_t)(t - 1) * M, d_dgi + (size_t)(t - 1) * M, G, dG,
                                               t_gi + (size_t)t * M, d_dgi + (size_t)t * M, nullptr, nullptr,
                                               nullptr, nullptr, COMP_NONE);
        cur = t_gi + (size_t)(half - 1) * M;
        dcur = d_dgi + (size_t)(half - 1) * M;
        if (N % 2 == 1) {
            step1_rows_t<<<gr, kBlock, 0, s>>>(L, cur, dcur, G, dG, ginv, dginv, nullptr, nullptr, phi, dph, COMP_CENTRE);
            cur = ginv; dcur = dginv;
            std::swap(ginv, tmp); std::swap(dginv, dtmp);
        }
        for (int sp = (N + 3) / 2; sp <= N; sp++) {
            int sinv = N - sp + 1;
            step1_rows_t<<<gr, kBlock, 0, s>>>(L, cur, dcur, G, dG, ginv, dginv, t_gi + (size_t)(sinv - 1) * M,
                                               d_dgi + (size_t)(sinv - 1) * M, phi, dph, COMP_ACC);
            cur = ginv; dcur = dginv;
            std::swap(ginv, tmp); std::swap(dginv, dtmp);
        }
    } else {
        const int N = o.N;
        // lumped second-order lattices and stiff ranges: a step is bilinear
        // in (propagator, G), so its tangent is step(d in, G) + step(in, dG),
        // two more launches of the primal step with the primal's parameters
        // (molecule_phi: SF_Copol2ndO_stiff_range.cpp:211-234 for the stiff
        // range's Pf(s-1, s+1) and isotropic end steps)
        const bool pair = (K == 3 || K == 5) || (K == 6 && L.stiff);
        auto prim = [&](int t, bool backward, const double *in, const double *G, double *out) {
            const int sg = o.seg[t];
            if (K == 6) {
                const bool iso = backward ? (t == N - 2) : (t == N - 1);
                const double Sv = iso ? 0.2 : (backward ? pf[sg * nseg + o.seg[t + 2]] : pf[o.seg[t - 1] * nseg + o.seg[t + 1]]);
                step2_rows<<<gr, kBlock, 0, s>>>(L, in, G, Sv, out, nullptr, nullptr, COMP_NONE, backward ? 1 : 0,
                                                 iso ? STEP2_ISO : STEP2_STIFF);
            } else {
                const double Sv = backward ? pf[sg * nseg + o.seg[t + 1]] : pf[o.seg[t - 1] * nseg + sg];
                step2l_rows<<<gr, kBlock, 0, s>>>(L, in, G, Sv, out, nullptr, nullptr, COMP_NONE, backward ? 1 : 0);
            }
        };
        auto pair_step = [&](int t, bool backward, const double *in, const double *din, double *out, double *dout) {
            const int sg = o.seg[t];
            prim(t, backward, in, d_gseg[sg], out);
            prim(t, backward, din, d_gseg[sg], t_w[0]);
            prim(t, backward, in, dgseg[sg], t_w[1]);
            sum2<<<g, kBlock, 0, s>>>(KM, t_w[0], t_w[1], dout);
        };
        replicate<<<g, kBlock, 0, s>>>(M, K, d_gseg[o.seg[0]], t_gi);
        replicate<<<g, kBlock, 0, s>>>(M, K, dgseg[o.seg[0]], d_dgi);
        for (int t = 1; t < N; t++) {
            int sg = o.seg[t];
            const double *src = t_gi + (size_t)(t - 1) * KM, *dsrc = d_dgi + (size_t)(t - 1) * KM;
            double *dst = t_gi + (size_t)t * KM, *ddst = d_dgi + (size_t)t * KM;
            if (pair)
                pair_step(t, false, src, dsrc, dst, ddst);
            else if (K == 1 && o.force != 0)   // forward steps with +force
                step1_force_rows_t<<<gr, kBlock, 0, s>>>(L, force_weights(L, o.force), src, dsrc, d_gseg[sg], dgseg[sg],
                                                         dst, ddst, nullptr, nullptr, nullptr, nullptr, COMP_NONE);
            else if (K == 1)
                step1_rows_t<<<gr, kBlock, 0, s>>>(L, src, dsrc, d_gseg[sg], dgseg[sg], dst, ddst, nullptr, nullptr,
                                                   nullptr, nullptr, COMP_NONE);
            else
                step2_rows_t<<<gr, kBlock, 0, s>>>(L, src, dsrc, d_gseg[sg], dgseg[sg], pf[o.seg[t - 1] * nseg + sg],
                                                   dst, ddst, nullptr, nullptr, nullptr, nullptr, COMP_NONE, 0);
        }
        replicate<<<g, kBlock, 0, s>>>(M, K, d_gseg[o.seg[N - 1]], ginv);
        replicate<<<g, kBlock, 0, s>>>(M, K, dgseg[o.seg[N - 1]], dginv);
        connect_t<<<g, kBlock, 0, s>>>(M, K, ginv, dginv, t_gi + (size_t)(N - 1) * KM, d_dgi + (size_t)(N - 1) * KM,
                                       o.d_phi[o.seg[N - 1]], o.d_dphi[o.seg[N - 1]]);
        cur = ginv; dcur = dginv;
        std::swap(ginv, tmp); std::swap(dginv, dtmp);
        for (int t = N - 2; t >= 0; t--) {
            int sg = o.seg[t];
            if (pair) {
                pair_step(t, true, cur, dcur, ginv, dginv);
                compose2_t<<<g, kBlock, 0, s>>>(L, K, ginv, dginv, t_gi + (size_t)t * KM, d_dgi + (size_t)t * KM,
                                                o.d_phi[sg], o.d_dphi[sg]);
            } else if (K == 1 && o.force != 0)   // backward steps with -force
                step1_force_rows_t<<<gr, kBlock, 0, s>>>(L, force_weights(L, -o.force), cur, dcur, d_gseg[sg],
                                                         dgseg[sg], ginv, dginv, t_gi + (size_t)t * KM,
                                                         d_dgi + (size_t)t * KM, o.d_phi[sg], o.d_dphi[sg], COMP_ACC);
            else if (K == 1)
                step1_rows_t<<<gr, kBlock, 0, s>>>(L, cur, dcur, d_gseg[sg], dgseg[sg], ginv, dginv,
                                                   t_gi + (size_t)t * KM, d_dgi + (size_t)t * KM, o.d_phi[sg],
                                                   o.d_dphi[sg], COMP_ACC);
            else
                step2_rows_t<<<gr, kBlock, 0, s>>>(L, cur, dcur, d_gseg[sg], dgseg[sg], pf[sg * nseg + o.seg[t + 1]],
                                                   ginv, dginv, t_gi + (size_t)t * KM, d_dgi + (size_t)t * KM,
                                                   o.d_phi[sg], o.d_dphi[sg], COMP_ACC, 1);
            cur = ginv; dcur = dginv;
            std::swap(ginv, tmp); std::swap(dginv, dtmp);
        }
    }
    }
    wsum_partial<<<nblocks_red, kBlock, 0, s>>>(M, K, cur, d_wgn, d_partial);
    wsum_partial<<<nblocks_red, kBlock, 0, s>>>(M, K, dcur, d_wgn, d_dpartial);
    mol_scalars<<<1, 1, 0, s>>>(p, nblocks_red, d_partial, scal, m);
    mol_scalars_t<<<1, 1, 0, s>>>(p, nblocks_red, d_dpartial, scal, tscal, m);
    for (int i : o.used) {
        finalize_phi_t<<<g, kBlock, 0, s>>>(M, d_gseg[i], dgseg[i], o.d_phi[i], o.d_dphi[i], scal, tscal, m, 0);
        set_boundaries<<<g, kBlock, 0, s>>>(L, 1, o.d_phi[i]);
        set_boundaries<<<g, kBlock, 0, s>>>(L, 1, o.d_dphi[i]);
    }
    return SFGPU_OK;
}

// f = F(x) and jv = J(x) v, both on the device, asynchronous
int sfgpu_system::jvp_async(const double *x, const double *v, double *f, double *jv) {
    int rc = ensure_tangent();
    if (rc) return rc;
    const DLat &L = H.L;
    const int g = grid_n(M);
    cudaStream_t s = stream;
    for (int i = 0; i < nseg; i++) {
        if (freedom[i] == SFGPU_SEG_FROZEN) continue;
        swf_update_t<<<g, kBlock, 0, s>>>(L, x, v, d_jmap, nclass, class_of[i], d_range[i],
                                          freedom[i] == SFGPU_SEG_PINNED, d_gfull[i], d_gseg[i], dgfull[i], dgseg[i]);
    }
    for (int m = 0; m < nmol; m++) {
        if (m == solvent) continue;
        if ((rc = molecule_phi_t(m))) return rc;
    }
    if ((rc = molecule_phi_t(solvent))) return rc;
    for (int i = 0; i < nseg; i++) {
        if (freedom[i] == SFGPU_SEG_FROZEN) continue;
        PtrList pl, dl;
        pl.n = dl.n = 0;
        for (auto &o : mols)
            if (o.count[i]) { pl.p[pl.n++] = o.d_phi[i]; dl.p[dl.n++] = o.d_dphi[i]; }
        sum_profiles<<<g, kBlock, 0, s>>>(M, pl, d_phi[i]);
        sum_profiles<<<g, kBlock, 0, s>>>(M, dl, dphi[i]);
    }
    bulk_scalars<<<1, 1, 0, s>>>(bp, ct, (const MolScal *)d_scal, d_phib, d_chib);
    bulk_scalars_t<<<1, 1, 0, s>>>(bp, ct, (const MolScalT *)d_tscal, d_dphib, d_dchib);
    ResParam rp;
    ResParamT tp;
    memset(&rp, 0, sizeof(rp));
    memset(&tp, 0, sizeof(tp));
    rp.nsites = nsites; rp.nclass = nclass; rp.nseg = nseg;
    for (int c = 0; c < nclass; c++) {
        rp.rep[c] = rep_of_class[c];
        rp.gfull[c] = d_gfull[rep_of_class[c]];
        tp.dgfull[c] = dgfull[rep_of_class[c]];
    }
    for (int i = 0; i < nseg; i++) { rp.phi[i] = d_phi[i]; tp.dphi[i] = dphi[i]; }
    residual_t<<<grid_n(nsites), kBlock, 0, s>>>(L, rp, tp, ct, d_sites, d_chib, d_dchib, f, jv);
    SFGPU_CUDA_TRY(cudaGetLastError());
    return SFGPU_OK;
}

extern "C" int sfgpu_jvp(sfgpu_system *s, const double *x_dev, const double *v_dev, double *f_dev, double *jv_dev) {
    if (!s) return SFGPU_ERR_INVALID;
    return s->jvp_async(x_dev, v_dev, f_dev, jv_dev);
}

extern "C" int sfgpu_jvp_host(sfgpu_system *s, const double *x, const double *v, double *f, double *jv) {
    if (!s || !x || !v) return SFGPU_ERR_INVALID;
    int rc = s->ensure_tangent();
    if (rc) return rc;
    SFGPU_CUDA_TRY(cudaMemcpyAsync(s->d_x, x, sizeof(double) * s->nvar, cudaMemcpyHostToDevice, s->stream));
    SFGPU_CUDA_TRY(cudaMemcpyAsync(s->d_v, v, sizeof(double) * s->nvar, cudaMemcpyHostToDevice, s->stream));
    if ((rc = s->jvp_async(s->d_x, s->d_v, s->d_f, s->d_jv))) return rc;
    if (f) SFGPU_CUDA_TRY(cudaMemcpyAsync(f, s->d_f, sizeof(double) * s->nvar, cudaMemcpyDeviceToHost, s->stream));
    if (jv) SFGPU_CUDA_TRY(cudaMemcpyAsync(jv, s->d_jv, sizeof(double) * s->nvar, cudaMemcpyDeviceToHost, s->stream));
    SFGPU_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return SFGPU_OK;
}

// ---------------------------------------------------------------------------
// Newton-Krylov: x <- x + alpha d with J d = -f solved by restarted GMRES
// (Saad & Schultz 1986) to the forcing tolerance of Eisenstat & Walker (1996,
// choice 2), classical Gram-Schmidt with one re-orthogonalisation, and a
// backtracking line search on |f|.
// ---------------------------------------------------------------------------
namespace {

__global__ void k_scale_copy(size_t n, double a, const double *__restrict__ x, double *__restrict__ y) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        y[i] = a * x[i];
}
__global__ void k_lincomb(size_t n, const double *__restrict__ x0, double a, const double *__restrict__ d,
                          double *__restrict__ y) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        y[i] = x0[i] + a * d[i];
}
// w -= sum_j h_j V_j
struct HCoef { double h[64]; int n; };
__global__ void k_subtract_basis(size_t n, HCoef c, const double *__restrict__ V, double *__restrict__ w) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        double acc = w[i];
        for (int j = 0; j < c.n; j++) acc -= c.h[j] * V[(size_t)j * n + i];
        w[i] = acc;
    }
}
__global__ void k_add_basis(size_t n, HCoef c, const double *__restrict__ V, double *__restrict__ x) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        double acc = 0;
        for (int j = 0; j < c.n; j++) acc += c.h[j] * V[(size_t)j * n + i];
        x[i] += acc;
    }
}

}  // namespace

struct NKWork {
    sfgpu_system *s;
    size_t n;
    int gb;
    double *partial = nullptr, *sums = nullptr;
    std::vector<double> hsum;
    int dots(int cnt, const double *const *a, const double *const *b, double *out) {
        cudaStream_t st = s->stream;
        for (int c0 = 0; c0 < cnt; c0 += 16) {
            DotList dl;
            dl.n = std::min(16, cnt - c0);
            for (int i = 0; i < dl.n; i++) { dl.a[i] = a[c0 + i]; dl.b[i] = b[c0 + i]; }
            dots_partial<<<gb, kBlock, 0, st>>>(n, dl, partial + (size_t)c0 * gb);
        }
        finish_sums<<<1, 128, 0, st>>>(cnt, gb, partial, sums);
        SFGPU_CUDA_TRY(cudaMemcpyAsync(out, sums, sizeof(double) * cnt, cudaMemcpyDeviceToHost, st));
        SFGPU_CUDA_TRY(cudaStreamSynchronize(st));
        return SFGPU_OK;
    }
    int norm(const double *a, double *out) {
        const double *pa[1] = {a};
        double v;
        int rc = dots(1, pa, pa, &v);
        *out = sqrt(v);
        return rc;
    }
};

extern "C" int sfgpu_solve_nk(sfgpu_system *s, double *x_host, double tol, int maxit, int krylov,
                              int *iterations, int *jvps, double *final_error) {
    if (!s || !x_host || krylov < 1 || krylov > 60 || maxit < 0) return SFGPU_ERR_INVALID;
    int rc = s->ensure_tangent();
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
    NKWork W;
    W.s = s;
    W.n = n;
    W.gb = (int)std::max<size_t>(1, std::min<size_t>((n + kBlock - 1) / kBlock, 148 * 8));
    double *x, *f, *xt, *ft, *d, *V, *w, *scratch;
    if ((rc = get(&x, n)) || (rc = get(&f, n)) || (rc = get(&xt, n)) || (rc = get(&ft, n)) || (rc = get(&d, n)) ||
        (rc = get(&V, n * (krylov + 1))) || (rc = get(&w, n)) || (rc = get(&scratch, n)) ||
        (rc = get(&W.partial, (size_t)W.gb * 64)) || (rc = get(&W.sums, 64))) {
        cleanup();
        return rc;
    }
    const int gv = W.gb;
#define NKTRY(e) do { cudaError_t _e = (e); if (_e != cudaSuccess) { sfgpu_set_error(_e, #e, __FILE__, __LINE__); cleanup(); return SFGPU_ERR_CUDA; } } while (0)
#define NKRC(e) do { int _r = (e); if (_r) { cleanup(); return _r; } } while (0)
    NKTRY(cudaMemcpyAsync(x, x_host, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    NKRC(s->residual_async(x, f));
    double fn;
    NKRC(W.norm(f, &fn));
    int it = 0, nj = 0;
    double fn_prev = fn, eta = 0.5;
    std::vector<double> H((size_t)(krylov + 1) * krylov), cs(krylov), sn(krylov), gvec(krylov + 1), y(krylov);
    while (fn > tol && it < maxit && std::isfinite(fn)) {
        it++;
        if (it > 1) {   // Eisenstat-Walker choice 2, safeguarded
            double e2 = 0.9 * (fn / fn_prev) * (fn / fn_prev);
            double sfg = 0.9 * eta * eta;
            eta = std::min(0.5, std::max(e2, sfg > 0.1 ? sfg : 0.0));
            eta = std::max(eta, 0.5 * tol / fn);
        }
        // GMRES(krylov) from d = 0 on J d = -f, one cycle
        NKTRY(cudaMemsetAsync(d, 0, sizeof(double) * n, st));
        const double beta = fn;
        k_scale_copy<<<gv, kBlock, 0, st>>>(n, -1.0 / beta, f, V);
        std::fill(gvec.begin(), gvec.end(), 0.0);
        gvec[0] = beta;
        int kdim = 0;
        for (int j = 0; j < krylov; j++) {
            NKRC(s->jvp_async(x, V + (size_t)j * n, scratch, w));
            nj++;
            // CGS2
            std::vector<const double *> va(j + 1), wb(j + 1, w);
            for (int i = 0; i <= j; i++) va[i] = V + (size_t)i * n;
            std::vector<double> h1(j + 1), h2(j + 1);
            NKRC(W.dots(j + 1, va.data(), wb.data(), h1.data()));
            HCoef c;
            c.n = j + 1;
            for (int i = 0; i <= j; i++) c.h[i] = h1[i];
            k_subtract_basis<<<gv, kBlock, 0, st>>>(n, c, V, w);
            NKRC(W.dots(j + 1, va.data(), wb.data(), h2.data()));
            for (int i = 0; i <= j; i++) c.h[i] = h2[i];
            k_subtract_basis<<<gv, kBlock, 0, st>>>(n, c, V, w);
            double hn;
            NKRC(W.norm(w, &hn));
            for (int i = 0; i <= j; i++) H[(size_t)i * krylov + j] = h1[i] + h2[i];
            H[(size_t)(j + 1) * krylov + j] = hn;
            // apply previous rotations, then a new one
            for (int i = 0; i < j; i++) {
                double a = H[(size_t)i * krylov + j], b = H[(size_t)(i + 1) * krylov + j];
                H[(size_t)i * krylov + j] = cs[i] * a + sn[i] * b;
                H[(size_t)(i + 1) * krylov + j] = -sn[i] * a + cs[i] * b;
            }
            double a = H[(size_t)j * krylov + j], b = H[(size_t)(j + 1) * krylov + j];
            double r = sqrt(a * a + b * b);
            cs[j] = (r > 0) ? a / r : 1.0;
            sn[j] = (r > 0) ? b / r : 0.0;
            H[(size_t)j * krylov + j] = r;
            H[(size_t)(j + 1) * krylov + j] = 0;
            gvec[j + 1] = -sn[j] * gvec[j];
            gvec[j] = cs[j] * gvec[j];
            kdim = j + 1;
            if (hn > 0 && j + 1 < krylov + 1)
                k_scale_copy<<<gv, kBlock, 0, st>>>(n, 1.0 / hn, w, V + (size_t)(j + 1) * n);
            if (fabs(gvec[j + 1]) <= eta * beta || !(hn > 0)) break;
        }
        // back substitution y = H^-1 g, d = V y
        for (int i = kdim - 1; i >= 0; i--) {
            double acc = gvec[i];
            for (int k = i + 1; k < kdim; k++) acc -= H[(size_t)i * krylov + k] * y[k];
            y[i] = acc / H[(size_t)i * krylov + i];
        }
        HCoef c;
        c.n = kdim;
        for (int i = 0; i < kdim; i++) c.h[i] = y[i];
        k_add_basis<<<gv, kBlock, 0, st>>>(n, c, V, d);
        // backtracking line search on |f|
        double alpha = 1.0, fn_new = 0;
        bool accepted = false;
        for (int ls = 0; ls < 12; ls++) {
            k_lincomb<<<gv, kBlock, 0, st>>>(n, x, alpha, d, xt);
            NKRC(s->residual_async(xt, ft));
            NKRC(W.norm(ft, &fn_new));
            if (std::isfinite(fn_new) && fn_new <= (1.0 - 1e-4 * alpha) * fn) { accepted = true; break; }
            alpha *= 0.5;
        }
        if (!accepted) break;
        std::swap(x, xt);
        std::swap(f, ft);
        fn_prev = fn;
        fn = fn_new;
    }
    NKTRY(cudaMemcpyAsync(x_host, x, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    NKTRY(cudaStreamSynchronize(st));
    // leave the profiles of the returned iterate in the system
    NKRC(s->residual_async(x, f));
    NKTRY(cudaStreamSynchronize(st));
#undef NKTRY
#undef NKRC
    cleanup();
    if (iterations) *iterations = it;
    if (jvps) *jvps = nj;
    if (final_error) *final_error = fn;
    if (!std::isfinite(fn)) return SFGPU_ERR_NONFINITE;
    return (fn <= tol) ? SFGPU_OK : SFGPU_ERR_NOTCONVERGED;
}

// Restarted GMRES(krylov) on A y = b from y = 0, A applied by op (CGS2
// orthogonalisation, Givens rotations), until |b - A y| <= rtol |b| or
// maxcycles restarts.  V: n (krylov + 1) doubles; w, r: n doubles.
static int gmres_solve(NKWork &W, const std::function<int(const double *, double *)> &op, const double *b,
                       double *y, double rtol, int krylov, int maxcycles, double *V, double *w, double *r,
                       double *relres, int *nops) {
    sfgpu_system *s = W.s;
    const size_t n = W.n;
    const int gv = W.gb;
    cudaStream_t st = s->stream;
    int rc;
    double bn;
    if ((rc = W.norm(b, &bn))) return rc;
    SFGPU_CUDA_TRY(cudaMemsetAsync(y, 0, sizeof(double) * n, st));
    SFGPU_CUDA_TRY(cudaMemcpyAsync(r, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    std::vector<double> H((size_t)(krylov + 1) * krylov), cs(krylov), sn(krylov), g(krylov + 1), yk(krylov);
    double rn = bn;
    *nops = 0;
    for (int cycle = 0; cycle < maxcycles && rn > rtol * bn && bn > 0; cycle++) {
        const double beta = rn;
        k_scale_copy<<<gv, kBlock, 0, st>>>(n, 1.0 / beta, r, V);
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        int kdim = 0;
        for (int j = 0; j < krylov; j++) {
            if ((rc = op(V + (size_t)j * n, w))) return rc;
            (*nops)++;
            std::vector<const double *> va(j + 1), wb(j + 1, w);
            for (int i = 0; i <= j; i++) va[i] = V + (size_t)i * n;
            std::vector<double> h1(j + 1), h2(j + 1);
            if ((rc = W.dots(j + 1, va.data(), wb.data(), h1.data()))) return rc;
            HCoef c;
            c.n = j + 1;
            for (int i = 0; i <= j; i++) c.h[i] = h1[i];
            k_subtract_basis<<<gv, kBlock, 0, st>>>(n, c, V, w);
            if ((rc = W.dots(j + 1, va.data(), wb.data(), h2.data()))) return rc;
            for (int i = 0; i <= j; i++) c.h[i] = h2[i];
            k_subtract_basis<<<gv, kBlock, 0, st>>>(n, c, V, w);
            double hn;
            if ((rc = W.norm(w, &hn))) return rc;
            for (int i = 0; i <= j; i++) H[(size_t)i * krylov + j] = h1[i] + h2[i];
            H[(size_t)(j + 1) * krylov + j] = hn;
            for (int i = 0; i < j; i++) {
                const double a = H[(size_t)i * krylov + j], bb = H[(size_t)(i + 1) * krylov + j];
                H[(size_t)i * krylov + j] = cs[i] * a + sn[i] * bb;
                H[(size_t)(i + 1) * krylov + j] = -sn[i] * a + cs[i] * bb;
            }
            const double a = H[(size_t)j * krylov + j], bb = H[(size_t)(j + 1) * krylov + j];
            const double rr = sqrt(a * a + bb * bb);
            cs[j] = (rr > 0) ? a / rr : 1.0;
            sn[j] = (rr > 0) ? bb / rr : 0.0;
            H[(size_t)j * krylov + j] = rr;
            H[(size_t)(j + 1) * krylov + j] = 0;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            kdim = j + 1;
            if (hn > 0) k_scale_copy<<<gv, kBlock, 0, st>>>(n, 1.0 / hn, w, V + (size_t)(j + 1) * n);
            if (fabs(g[j + 1]) <= rtol * bn || !(hn > 0)) break;
        }
        for (int i = kdim - 1; i >= 0; i--) {
            double acc = g[i];
            for (int k = i + 1; k < kdim; k++) acc -= H[(size_t)i * krylov + k] * yk[k];
            yk[i] = acc / H[(size_t)i * krylov + i];
        }
        HCoef c;
        c.n = kdim;
        for (int i = 0; i < kdim; i++) c.h[i] = yk[i];
        k_add_basis<<<gv, kBlock, 0, st>>>(n, c, V, y);
        // true residual r = b - A y
        if ((rc = op(y, w))) return rc;
        (*nops)++;
        k_lincomb<<<gv, kBlock, 0, st>>>(n, b, -1.0, w, r);
        if ((rc = W.norm(r, &rn))) return rc;
    }
    *relres = (bn > 0) ? rn / bn : 0.0;
    return SFGPU_OK;
}

extern "C" int sfgpu_phi_sensitivity_chi(sfgpu_system *s, const double *x_host, const double *omega_host,
                                         double *dchi_host, double rtol, int krylov, int maxcycles,
                                         double *relres) {
    if (!s || !x_host || !omega_host || !dchi_host || krylov < 1 || krylov > 60 || maxcycles < 1 || !(rtol > 0))
        return SFGPU_ERR_INVALID;
    int rc = s->ensure_adjoint();
    if (rc) return rc;
    const size_t n = s->nvar, M = s->M;
    const int ns = s->nseg;
    cudaStream_t st = s->stream;
    std::vector<void *> mine;
    auto get = [&](double **p, size_t cnt) -> int {
        cudaError_t e = cudaMalloc((void **)p, sizeof(double) * (cnt ? cnt : 1));
        if (e != cudaSuccess) { sfgpu_set_error(e, "cudaMalloc", __FILE__, __LINE__); return SFGPU_ERR_NOMEM; }
        mine.push_back(*p);
        return SFGPU_OK;
    };
    auto cleanup = [&]() { for (void *p : mine) cudaFree(p); };
    NKWork W;
    W.s = s;
    W.n = n;
    W.gb = (int)std::max<size_t>(1, std::min<size_t>((n + kBlock - 1) / kBlock, 148 * 8));
    double *x, *b, *lam, *V, *w, *r, *om, *dchi;
    if ((rc = get(&x, n)) || (rc = get(&b, n)) || (rc = get(&lam, n)) || (rc = get(&V, n * (krylov + 1))) ||
        (rc = get(&w, n)) || (rc = get(&r, n)) || (rc = get(&om, (size_t)ns * M)) ||
        (rc = get(&dchi, (size_t)ns * ns)) || (rc = get(&W.partial, (size_t)W.gb * 64)) || (rc = get(&W.sums, 64))) {
        cleanup();
        return rc;
    }
#define SCTRY(e) do { cudaError_t _e = (e); if (_e != cudaSuccess) { sfgpu_set_error(_e, #e, __FILE__, __LINE__); cleanup(); return SFGPU_ERR_CUDA; } } while (0)
#define SCRC(e) do { int _r = (e); if (_r) { cleanup(); return _r; } } while (0)
    SCTRY(cudaMemcpyAsync(x, x_host, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    SCTRY(cudaMemcpyAsync(om, omega_host, sizeof(double) * ns * M, cudaMemcpyHostToDevice, st));
    std::vector<const double *> omp(ns);
    for (int i = 0; i < ns; i++) omp[i] = om + (size_t)i * M;
    SCRC(s->phi_vjp_async(x, omp.data(), b));   // b = dL/dx at fixed chi
    int nops = 0;
    double rr = 0;
    // J^T lam = b
    SCRC(gmres_solve(W, [&](const double *v, double *out) { return s->vjp_async(x, v, s->d_f, out); }, b, lam,
                     rtol, krylov, maxcycles, V, w, r, &rr, &nops));
    SCRC(s->chi_vjp_async(x, lam, dchi));
    std::vector<double> h((size_t)ns * ns);
    SCTRY(cudaMemcpyAsync(h.data(), dchi, sizeof(double) * ns * ns, cudaMemcpyDeviceToHost, st));
    SCTRY(cudaStreamSynchronize(st));
    for (int i = 0; i < ns * ns; i++) dchi_host[i] = -h[i];
    if (relres) *relres = rr;
    cleanup();
#undef SCTRY
#undef SCRC
    return SFGPU_OK;
}
