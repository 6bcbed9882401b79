// sfgpu_solve.cu -- host-driven Pure_DIIS iteration on one system (the plain
// GPU form): SFNewton::PlainLBFGSDIIS (sfnewton.cpp:566-664) with the DIIS
// coefficients of SFNewton::Ax (sfnewton.cpp:531-557).  Residuals, vector
// updates and Gram dot products run on the device; the k x k coefficient
// solve (k <= 64) runs on the host after one small device-to-host copy per
// iteration.
#include <cmath>
#include <cstring>
#include <vector>
#include <algorithm>
#include "sfgpu_system.h"

using namespace sfk;

// cyclic Jacobi eigen-decomposition of a symmetric k x k matrix (Golub & Van
// Loan, Matrix Computations 4th ed., sec. 8.5); for the symmetric Gram matrix
// the SVD pseudo-inverse of SFNewton::Ax equals Q diag(1/ev) Q^T.
void sfgpu_diis_coefficients(int n, const double *A_in, double *c) {
    std::vector<double> A(A_in, A_in + (size_t)n * n), Q((size_t)n * n, 0.0), ev(n);
    for (int i = 0; i < n; i++) Q[i * n + i] = 1;
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0, tot = 0;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                tot += A[i * n + j] * A[i * n + j];
                if (i != j) off += A[i * n + j] * A[i * n + j];
            }
        if (off <= 1e-30 * tot || off == 0) break;
        for (int p = 0; p < n; p++)
            for (int q = p + 1; q < n; q++) {
                double apq = A[p * n + q];
                if (apq == 0) continue;
                double theta = (A[q * n + q] - A[p * n + p]) / (2 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1));
                double cs = 1 / sqrt(t * t + 1), sn = t * cs;
                for (int k = 0; k < n; k++) {
                    double akp = A[k * n + p], akq = A[k * n + q];
                    A[k * n + p] = cs * akp - sn * akq; A[k * n + q] = sn * akp + cs * akq;
                }
                for (int k = 0; k < n; k++) {
                    double apk = A[p * n + k], aqk = A[q * n + k];
                    A[p * n + k] = cs * apk - sn * aqk; A[q * n + k] = sn * apk + cs * aqk;
                }
                for (int k = 0; k < n; k++) {
                    double qkp = Q[k * n + p], qkq = Q[k * n + q];
                    Q[k * n + p] = cs * qkp - sn * qkq; Q[k * n + q] = sn * qkp + cs * qkq;
                }
            }
    }
    for (int i = 0; i < n; i++) ev[i] = A[i * n + i];
    for (int i = 0; i < n; i++) c[i] = 0;
    for (int k = 0; k < n; k++) {
        double proj = 0;
        for (int i = 0; i < n; i++) proj += Q[i * n + k];
        double t = proj / ev[k];
        for (int i = 0; i < n; i++) c[i] += Q[i * n + k] * t;
    }
}

static int grid_len(size_t n) {
    size_t b = (n + kBlock - 1) / kBlock;
    if (b > 148 * 8) b = 148 * 8;
    return (int)(b ? b : 1);
}

struct DiisWork {
    double *x = nullptr, *x0 = nullptr, *g = nullptr, *XR = nullptr, *XX0 = nullptr, *partial = nullptr, *sums = nullptr;
};

extern "C" int sfgpu_solve_diis(sfgpu_system *s, double *x_host, double tol, int maxit, int m,
                                double eta, int *iterations, double *final_error) {
    if (!s || !x_host) return SFGPU_ERR_INVALID;
    if (m < 1 || m > 64 || !(eta > 0) || maxit < 0) return SFGPU_ERR_INVALID;
    const size_t iv = s->nvar;
    cudaStream_t st = s->stream;
    DiisWork w;
    const int gb = grid_len(iv);
    std::vector<void *> mine;
    auto get = [&](double **p, size_t n) -> int {
        cudaError_t e = cudaMalloc((void **)p, sizeof(double) * (n ? n : 1));
        if (e != cudaSuccess) { sfgpu_set_error(e, "cudaMalloc", __FILE__, __LINE__); return SFGPU_ERR_NOMEM; }
        mine.push_back(*p);
        return SFGPU_OK;
    };
    int rc = SFGPU_OK;
    auto cleanup = [&]() { for (void *p : mine) cudaFree(p); };
    if ((rc = get(&w.x, iv)) || (rc = get(&w.x0, iv)) || (rc = get(&w.g, iv)) || (rc = get(&w.XR, iv * m)) ||
        (rc = get(&w.XX0, iv * m)) || (rc = get(&w.partial, (size_t)gb * (m + 1))) || (rc = get(&w.sums, m + 1))) {
        cleanup();
        return rc;
    }
    std::vector<double> Aij((size_t)m * m, 0.0), Ap((size_t)m * m), C(m), sums(m + 1);
    int k = 0, it = 0, kd = 1;
    double err = 0;
#define TRY(e) do { cudaError_t _e = (e); if (_e != cudaSuccess) { sfgpu_set_error(_e, #e, __FILE__, __LINE__); cleanup(); return SFGPU_ERR_CUDA; } } while (0)
    TRY(cudaMemcpyAsync(w.x, x_host, sizeof(double) * iv, cudaMemcpyHostToDevice, st));
    if ((rc = s->residual_async(w.x, w.g))) { cleanup(); return rc; }
    TRY(cudaMemcpyAsync(w.x0, w.x, sizeof(double) * iv, cudaMemcpyDeviceToDevice, st));
    // x = -eta*g (the first step of PlainLBFGSDIIS discards x, sfnewton.cpp:582)
    TRY(cudaMemsetAsync(w.x, 0, sizeof(double) * iv, st));
    diis_step<<<gb, kBlock, 0, st>>>(iv, eta, w.x, w.x0, w.g, w.XR, w.XX0);
    {
        DotList dl; dl.n = 1; dl.a[0] = w.g; dl.b[0] = w.g;
        dots_partial<<<gb, kBlock, 0, st>>>(iv, dl, w.partial);
        finish_sums<<<1, 32, 0, st>>>(1, gb, w.partial, w.sums);
        TRY(cudaMemcpyAsync(sums.data(), w.sums, sizeof(double), cudaMemcpyDeviceToHost, st));
        TRY(cudaStreamSynchronize(st));
        err = sqrt(sums[0]);
    }
    // the first diis_step also computed XX0[0] = x - x0 with x = -eta*g
    // against x0 = x_initial; SFbox forms X_X0 = x - x0 the same way.
    while (tol < err && it < maxit) {
        it++;
        TRY(cudaMemcpyAsync(w.x0, w.x, sizeof(double) * iv, cudaMemcpyDeviceToDevice, st));
        if ((rc = s->residual_async(w.x, w.g))) { cleanup(); return rc; }
        k = it % m;
        kd++;
        diis_step<<<gb, kBlock, 0, st>>>(iv, eta, w.x, w.x0, w.g, w.XR + (size_t)k * iv, w.XX0 + (size_t)k * iv);
        if (kd > m) {
            kd = m;
            for (int i = 1; i < m; i++)
                for (int j = 1; j < m; j++) Aij[m * (i - 1) + j - 1] = Aij[m * i + j];
        }
        // Gram row <XX0[pos_i], XX0[k]> for the kd stored steps and |g|^2,
        // in chunks of 16 pairs per launch
        std::vector<int> pos(kd);
        std::vector<const double *> pa(kd + 1), pb(kd + 1);
        for (int i = 0; i < kd; i++) {
            int posi = k - kd + 1 + i;
            if (posi < 0) posi += m;
            pos[i] = posi;
            pa[i] = w.XX0 + (size_t)posi * iv;
            pb[i] = w.XX0 + (size_t)k * iv;
        }
        pa[kd] = w.g; pb[kd] = w.g;
        for (int c0 = 0; c0 <= kd; c0 += 16) {
            DotList dl;
            dl.n = std::min(16, kd + 1 - c0);
            for (int i = 0; i < dl.n; i++) { dl.a[i] = pa[c0 + i]; dl.b[i] = pb[c0 + i]; }
            dots_partial<<<gb, kBlock, 0, st>>>(iv, dl, w.partial + (size_t)c0 * gb);
        }
        finish_sums<<<1, 128, 0, st>>>(kd + 1, gb, w.partial, w.sums);
        TRY(cudaMemcpyAsync(sums.data(), w.sums, sizeof(double) * (kd + 1), cudaMemcpyDeviceToHost, st));
        TRY(cudaStreamSynchronize(st));
        for (int i = 0; i < kd; i++) Aij[i + m * (kd - 1)] = Aij[kd - 1 + m * i] = sums[i];
        for (int i = 0; i < kd; i++)
            for (int j = 0; j < kd; j++) Ap[j + kd * i] = Aij[j + m * i];
        sfgpu_diis_coefficients(kd, Ap.data(), C.data());
        double nc = 0;
        for (int i = 0; i < kd; i++) nc += C[i];
        Coef cf;
        cf.n = kd;
        for (int i = 0; i < kd; i++) { cf.c[i] = C[i] / nc; cf.pos[i] = pos[i]; }
        diis_combine<<<gb, kBlock, 0, st>>>(iv, cf, w.XR, iv, w.x);
        err = sqrt(sums[kd]);
        if (!std::isfinite(err)) { rc = SFGPU_ERR_NONFINITE; break; }
    }
    TRY(cudaMemcpyAsync(x_host, w.x, sizeof(double) * iv, cudaMemcpyDeviceToHost, st));
    TRY(cudaStreamSynchronize(st));
#undef TRY
    cleanup();
    if (iterations) *iterations = it;
    if (final_error) *final_error = err;
    if (rc == SFGPU_OK && !(err <= tol)) rc = SFGPU_ERR_NOTCONVERGED;
    return rc;
}

// Many systems solved concurrently: each by sfgpu_solve_diis on its own
// stream, driven by its own host thread, so the device interleaves the
// systems' kernels and each system's per-iteration host round trip hides
// behind the others' work.  For instances large enough to fill the GPU one
// step at a time (3D second order), where a block per instance would leave
// most SMs idle.
#include <atomic>
#include <thread>

extern "C" int sfgpu_solve_diis_many(int n, sfgpu_system *const *systems, double *const *x, double tol, int maxit,
                                     int m, double eta, int threads, int *status, int *iterations, double *errors) {
    if (n < 1 || !systems || !x || !status) return SFGPU_ERR_INVALID;
    for (int i = 0; i < n; i++)
        if (!systems[i] || !x[i]) return SFGPU_ERR_INVALID;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) { sfgpu_set_error(e, "cudaGetDevice", __FILE__, __LINE__); return SFGPU_ERR_CUDA; }
    const int nt = std::max(1, std::min(threads > 0 ? threads : n, n));
    std::atomic<int> next(0);
    auto worker = [&]() {
        cudaSetDevice(dev);
        for (int i = next++; i < n; i = next++) {
            int it = 0;
            double err = 0;
            status[i] = sfgpu_solve_diis(systems[i], x[i], tol, maxit, m, eta, &it, &err);
            if (iterations) iterations[i] = it;
            if (errors) errors[i] = err;
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; t++) pool.emplace_back(worker);
    worker();
    for (auto &t : pool) t.join();
    for (int i = 0; i < n; i++)
        if (status[i] != SFGPU_OK && status[i] != SFGPU_ERR_NOTCONVERGED && status[i] != SFGPU_ERR_NONFINITE)
            return status[i];
    return SFGPU_OK;
}
