// sfgpu_batch.cu -- persistent batched solver: many independent SF-SCF
// instances (a Vary-style sweep, Vary.cpp:127 / SF_Box.cpp:145-177) solved by
// Pure_DIIS in ONE kernel launch.  Blocks take instances from an atomic work
// queue, so uneven instances (different lattices and chain lengths) balance
// across the SMs; each block iterates its instance to convergence on device.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#include "sfgpu_batch_kernel.cuh"
#include "sfgpu_system.h"

using namespace sfb;

struct sfgpu_batch {
    std::vector<sfgpu_system *> sys;
    std::vector<InstDesc> desc_h;
    InstDesc *d_desc = nullptr;
    int *d_queue = nullptr, *d_status = nullptr, *d_iters = nullptr;
    double *d_err = nullptr, *d_xall = nullptr;
    std::vector<long long> offset;      // start of each instance in the concatenated x
    long long total = 0;
    int m = 10, block = 256;
    size_t stage_bytes = 0;         // dynamic shared memory per block (staged G)
    bool wide = false;              // some instance needs batch_diis_kernel_t<true>
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<void *> allocs;
    ~sfgpu_batch() {
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        for (void *p : allocs) cudaFree(p);
        for (auto *s : sys) delete s;
        if (own_stream && stream) cudaStreamDestroy(stream);
    }
};

static int balloc(sfgpu_batch *b, void **p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes ? bytes : 8);
    if (e != cudaSuccess) { sfgpu_set_error(e, "cudaMalloc", __FILE__, __LINE__); return SFGPU_ERR_NOMEM; }
    b->allocs.push_back(*p);
    return SFGPU_OK;
}

// ---------------------------------------------------------------------------
// Shared-memory staging of each instance: G of the running segment where
// the lattice fits next to the kernel's static shared memory, and on 1D
// symmetric homopolymers also the running slices, phi and the ring of
// stored slices.  allow = false stages nothing (more blocks per SM).
static BatchKernel batch_kernel(const sfgpu_batch *b) {
    return b->wide ? batch_kernel_wide() : batch_diis_kernel_t<false>;
}

static int configure_stage(sfgpu_batch *b, bool allow) {
    int dev = 0, optin = 0;
    cudaFuncAttributes fa;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
        cudaFuncGetAttributes(&fa, batch_kernel(b)) != cudaSuccess)
        return SFGPU_ERR_CUDA;
    const size_t fixed = fa.sharedSizeBytes + 1024;   // 1 KB the system reserves per block
    const size_t room = (size_t)optin > fixed ? (size_t)optin - fixed : 0;
    size_t need = 0;
    const int n = (int)b->sys.size();
    for (int i = 0; i < n; i++) {
        const size_t bytes = sizeof(double) * (size_t)b->sys[i]->M;
        b->desc_h[i].gstage = (allow && bytes <= room) ? 1 : 0;
        if (b->desc_h[i].gstage) need = std::max(need, bytes);
        // 1D symmetric homopolymers: G, two running slices, phi and the
        // ring of stored slices, when these 4 + kRing lattice vectors fit
        // in 48 KB (M <= 768), a budget that keeps several blocks
        // resident per SM
        const auto *sy = b->sys[i];
        bool sym1d = allow && sy->H.L.grad == 1;
        bool any_sym = false;
        for (const auto &o : sy->mols) any_sym |= o.sym != 0;
        const size_t vecs = (4 + sfb::kRing) * bytes;
        sym1d = sym1d && any_sym && vecs <= 48 * 1024 && vecs <= room;
        b->desc_h[i].small1d = sym1d ? 1 : 0;
        if (sym1d) need = std::max(need, vecs);
    }
    if (cudaMemcpy(b->d_desc, b->desc_h.data(), sizeof(InstDesc) * n, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaFuncSetAttribute(batch_kernel(b), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need) !=
            cudaSuccess)
        return SFGPU_ERR_CUDA;
    b->stage_bytes = need;
    return SFGPU_OK;
}

extern "C" int sfgpu_batch_create(int n, const sfgpu_system_desc *descs, int m, sfgpu_batch **out) {
    if (!out || !descs || n < 1) return SFGPU_ERR_INVALID;
    *out = nullptr;
    if (m < 1 || m > kMaxHist) return SFGPU_ERR_INVALID;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); return SFGPU_ERR_NODEVICE; }
    sfgpu_batch *b = new sfgpu_batch();
    b->m = m;
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) { delete b; return SFGPU_ERR_CUDA; }
    b->own_stream = true;
    int rc = SFGPU_OK;
    int maxM = 1;
    b->offset.resize(n);
    for (int i = 0; i < n && !rc; i++) {
        if (descs[i].lattice.order != 1) { rc = fail_unsupported("batched second-order lattices"); break; }
        if (descs[i].overflow_protection) { rc = fail_unsupported("batched systems with overflow protection"); break; }
        for (int q = 0; q < descs[i].n_segments && !rc; q++)
            if (descs[i].segments[q].valence != 0) rc = fail_unsupported("batched charged systems");
        if (rc) break;
        for (int q = 0; q < descs[i].n_molecules && !rc; q++) {
            if (descs[i].molecules[q].n_generations > 0 || descs[i].molecules[q].bond_parent ||
                descs[i].molecules[q].ring)
                rc = fail_unsupported("batched dendrimers, branched molecules and rings");
            if (descs[i].molecules[q].force != 0) b->wide = true;
        }
        if (rc) break;
        if (descs[i].lattice.gradients == 3 && descs[i].lattice.lattice_type != SFGPU_LATTICE_STANDARD) b->wide = true;
        sfgpu_system *s = new sfgpu_system();
        s->stream = b->stream;
        rc = s->setup(&descs[i]);
        if (!rc && (s->nseg > kResMax || s->nclass > kResMax)) rc = SFGPU_ERR_UNSUPPORTED;   // site_residual registers
        if (rc) { delete s; break; }
        b->sys.push_back(s);
        b->offset[i] = b->total;
        b->total += (long long)s->nvar;
        maxM = std::max(maxM, s->M);
    }
    if (rc) { delete b; return rc; }
    // concatenated iteration variables and per-instance DIIS work
    if ((rc = balloc(b, (void **)&b->d_xall, sizeof(double) * b->total))) { delete b; return rc; }
    b->desc_h.resize(n);
    for (int i = 0; i < n && !rc; i++) {
        sfgpu_system *s = b->sys[i];
        InstDesc &I = b->desc_h[i];
        memset(&I, 0, sizeof(I));
        I.L = s->H.L;
        I.M = s->M; I.nseg = s->nseg; I.nmol = s->nmol; I.nclass = s->nclass; I.nsites = s->nsites;
        I.solvent = s->solvent; I.nvar = (long long)s->nvar;
        for (int q = 0; q < s->nseg; q++) {
            I.freedom[q] = s->freedom[q];
            I.class_of[q] = s->class_of[q];
            I.range[q] = s->d_range[q];
            I.gfull[q] = s->d_gfull[q]; I.gseg[q] = s->d_gseg[q]; I.phi[q] = s->d_phi[q];
        }
        for (int c = 0; c < s->nclass; c++) I.rep[c] = s->rep_of_class[c];
        I.ct = s->ct;
        memcpy(I.frac, s->bp.frac, sizeof(I.frac));
        I.jmap = s->d_jmap; I.sites = s->d_sites; I.w_gn = s->d_wgn;
        for (int q = 0; q < s->nmol; q++) {
            const HMol &o = s->mols[q];
            IMol &im = I.mol[q];
            im.N = o.N; im.type = o.type; im.sym = o.sym; im.freedom = o.freedom; im.pinned = o.pinned;
            im.solvent = (q == s->solvent); im.phibulk = o.phibulk; im.theta = o.theta;
            im.nused = (int)o.used.size();
            for (int a = 0; a < im.nused; a++) im.used[a] = o.used[a];
            for (int a = 0; a < s->nseg; a++) im.phi[a] = o.d_phi[a];
            int *dseg = nullptr;
            if ((rc = balloc(b, (void **)&dseg, sizeof(int) * o.N))) break;
            if (cudaMemcpy(dseg, o.seg.data(), sizeof(int) * o.N, cudaMemcpyHostToDevice) != cudaSuccess) { rc = SFGPU_ERR_CUDA; break; }
            im.seg = dseg;
        }
        if (rc) break;
        {   // force ensembles: step weights per molecule
            std::vector<sfk::ForceW> fw(2 * s->nmol);
            I.fmask = 0;
            for (int q = 0; q < s->nmol; q++)
                if (s->mols[q].force != 0) {
                    I.fmask |= 1 << q;
                    fw[2 * q] = force_weights(s->H.L, s->mols[q].force);
                    fw[2 * q + 1] = force_weights(s->H.L, -s->mols[q].force);
                }
            sfk::ForceW *dfw = nullptr;
            if (I.fmask) {
                if ((rc = balloc(b, (void **)&dfw, sizeof(sfk::ForceW) * fw.size()))) break;
                if (cudaMemcpy(dfw, fw.data(), sizeof(sfk::ForceW) * fw.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
                    rc = SFGPU_ERR_CUDA;
                    break;
                }
            }
            I.fw = dfw;
        }
        I.gi = s->d_gi; I.ginv0 = s->d_ginv[0]; I.ginv1 = s->d_ginv[1];
        const size_t iv = s->nvar;
        I.x = b->d_xall + b->offset[i];
        if ((rc = balloc(b, (void **)&I.x0, sizeof(double) * iv)) || (rc = balloc(b, (void **)&I.g, sizeof(double) * iv)) ||
            (rc = balloc(b, (void **)&I.XR, sizeof(double) * iv * m)) || (rc = balloc(b, (void **)&I.XX0, sizeof(double) * iv * m)))
            break;
    }
    if (!rc) rc = balloc(b, (void **)&b->d_desc, sizeof(InstDesc) * n);
    if (!rc && cudaMemcpy(b->d_desc, b->desc_h.data(), sizeof(InstDesc) * n, cudaMemcpyHostToDevice) != cudaSuccess) rc = SFGPU_ERR_CUDA;
    if (!rc) rc = balloc(b, (void **)&b->d_queue, sizeof(int));
    if (!rc) rc = balloc(b, (void **)&b->d_status, sizeof(int) * n);
    if (!rc) rc = balloc(b, (void **)&b->d_iters, sizeof(int) * n);
    if (!rc) rc = balloc(b, (void **)&b->d_err, sizeof(double) * n);
    if (rc) { delete b; return rc; }
    // threads per block by the largest lattice (timed on the 2D cylinder and
    // on the uneven 1D sweep, where 384 beat 256 by 4.5 % and 32..128 lost)
    b->block = maxM >= 4096 ? 1024 : (maxM >= 1024 ? 512 : (maxM >= 384 ? 384 : 256));
    if ((rc = configure_stage(b, true))) { delete b; return rc; }
    *out = b;
    return SFGPU_OK;
}

extern "C" int sfgpu_batch_destroy(sfgpu_batch *b) {
    if (!b) return SFGPU_OK;
    cudaStreamSynchronize(b->stream);
    delete b;
    return SFGPU_OK;
}

extern "C" int sfgpu_batch_info(sfgpu_batch *b, int *n, long long *total_nvar, long long *offsets) {
    if (!b) return SFGPU_ERR_INVALID;
    if (n) *n = (int)b->sys.size();
    if (total_nvar) *total_nvar = b->total;
    if (offsets) for (size_t i = 0; i < b->sys.size(); i++) offsets[i] = b->offset[i];
    return SFGPU_OK;
}

extern "C" int sfgpu_batch_set_stream(sfgpu_batch *b, void *stream) {
    if (!b) return SFGPU_ERR_INVALID;
    SFGPU_CUDA_TRY(cudaStreamSynchronize(b->stream));
    if (b->own_stream) cudaStreamDestroy(b->stream);
    b->own_stream = false;
    b->stream = (cudaStream_t)stream;
    for (auto *s : b->sys) s->stream = b->stream;
    return SFGPU_OK;
}

// Launch shape of the persistent kernel: threads per block (32..1024, a
// multiple of 32) and whether instances stage G (and the 1D slices) in
// shared memory.  By default 1024/512/256 threads by lattice size and
// staging on.
extern "C" int sfgpu_batch_set_launch(sfgpu_batch *b, int threads, int stage) {
    if (!b || threads < 32 || threads > 1024 || threads % 32) return SFGPU_ERR_INVALID;
    SFGPU_CUDA_TRY(cudaStreamSynchronize(b->stream));
    b->block = threads;
    return configure_stage(b, stage != 0);
}

// Load the concatenated initial guesses (host) into the device iterate.
extern "C" int sfgpu_batch_load(sfgpu_batch *b, const double *x) {
    if (!b || !x) return SFGPU_ERR_INVALID;
    SFGPU_CUDA_TRY(cudaMemcpyAsync(b->d_xall, x, sizeof(double) * b->total, cudaMemcpyHostToDevice, b->stream));
    SFGPU_CUDA_TRY(cudaStreamSynchronize(b->stream));
    return SFGPU_OK;
}

// Solve every instance by Pure_DIIS starting from the device-resident
// iterate: one persistent kernel launch, queued asynchronously on the batch
// stream and bracketed by CUDA events (sfgpu_batch_kernel_ms).
extern "C" int sfgpu_batch_solve_resident(sfgpu_batch *b, double tol, int maxit, double eta) {
    if (!b || maxit < 0 || !(eta > 0)) return SFGPU_ERR_INVALID;
    const int n = (int)b->sys.size();
    cudaStream_t st = b->stream;
    SFGPU_CUDA_TRY(cudaMemsetAsync(b->d_queue, 0, sizeof(int), st));
    int dev = 0, nsm = 148;
    SFGPU_CUDA_TRY(cudaGetDevice(&dev));
    SFGPU_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    int per_sm = 1;
    SFGPU_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel(b), b->block, b->stage_bytes));
    int grid = std::max(1, std::min(n, nsm * std::max(1, per_sm)));
    if (!b->ev0) {
        SFGPU_CUDA_TRY(cudaEventCreate(&b->ev0));
        SFGPU_CUDA_TRY(cudaEventCreate(&b->ev1));
    }
    SFGPU_CUDA_TRY(cudaEventRecord(b->ev0, st));
    batch_kernel(b)<<<grid, b->block, b->stage_bytes, st>>>(b->d_desc, n, b->d_queue, b->m, eta, tol, maxit,
                                                  b->d_status, b->d_iters, b->d_err);
    SFGPU_CUDA_TRY(cudaGetLastError());
    SFGPU_CUDA_TRY(cudaEventRecord(b->ev1, st));
    return SFGPU_OK;
}

// Copy out the per-instance results (and the iterates when x != NULL).
extern "C" int sfgpu_batch_results(sfgpu_batch *b, double *x, int *status, int *iterations, double *errors) {
    if (!b) return SFGPU_ERR_INVALID;
    const int n = (int)b->sys.size();
    cudaStream_t st = b->stream;
    if (x) SFGPU_CUDA_TRY(cudaMemcpyAsync(x, b->d_xall, sizeof(double) * b->total, cudaMemcpyDeviceToHost, st));
    std::vector<int> s_h(n), it_h(n);
    std::vector<double> e_h(n);
    SFGPU_CUDA_TRY(cudaMemcpyAsync(s_h.data(), b->d_status, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
    SFGPU_CUDA_TRY(cudaMemcpyAsync(it_h.data(), b->d_iters, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
    SFGPU_CUDA_TRY(cudaMemcpyAsync(e_h.data(), b->d_err, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    SFGPU_CUDA_TRY(cudaStreamSynchronize(st));
    for (int i = 0; i < n; i++) {
        if (status) status[i] = s_h[i];
        if (iterations) iterations[i] = it_h[i];
        if (errors) errors[i] = e_h[i];
    }
    return SFGPU_OK;
}

extern "C" int sfgpu_batch_kernel_ms(sfgpu_batch *b, double *ms) {
    if (!b || !b->ev0) return SFGPU_ERR_INVALID;
    SFGPU_CUDA_TRY(cudaEventSynchronize(b->ev1));
    float v = 0;
    SFGPU_CUDA_TRY(cudaEventElapsedTime(&v, b->ev0, b->ev1));
    *ms = v;
    return SFGPU_OK;
}

// Host convenience: load guesses x_in, solve, read back the iterates into
// x_out (may be NULL) and the per-instance results.
extern "C" int sfgpu_batch_solve(sfgpu_batch *b, const double *x_in, double *x_out, double tol, int maxit,
                                 double eta, int *status, int *iterations, double *errors) {
    if (!b || !x_in) return SFGPU_ERR_INVALID;
    cudaStream_t st = b->stream;
    SFGPU_CUDA_TRY(cudaMemcpyAsync(b->d_xall, x_in, sizeof(double) * b->total, cudaMemcpyHostToDevice, st));
    int rc = sfgpu_batch_solve_resident(b, tol, maxit, eta);
    if (rc) return rc;
    return sfgpu_batch_results(b, x_out, status, iterations, errors);
}

// results of instance i after a solve (its last residual evaluation)
extern "C" int sfgpu_batch_get_phi(sfgpu_batch *b, int inst, int seg, double *phi) {
    if (!b || inst < 0 || inst >= (int)b->sys.size()) return SFGPU_ERR_INVALID;
    sfgpu_system *s = b->sys[inst];
    if (seg < 0 || seg >= s->nseg) return SFGPU_ERR_INVALID;
    SFGPU_CUDA_TRY(cudaMemcpyAsync(phi, s->d_phi[seg], sizeof(double) * s->M, cudaMemcpyDeviceToHost, b->stream));
    SFGPU_CUDA_TRY(cudaStreamSynchronize(b->stream));
    return SFGPU_OK;
}
