// sfgpu_batch_kernel.cuh -- the persistent batched Pure_DIIS kernel
// (SFNewton::PlainLBFGSDIIS, sfnewton.cpp:566-664, one instance per thread
// block).  kWide = false compiles the six-neighbour lattices only (every
// configuration of the bench) and is instantiated in sfgpu_batch.cu;
// kWide = true also compiles the FCC, HEX and stencils lattice types and the
// force ensemble and is instantiated alone in sfgpu_batch_wide.cu, so that
// neither instantiation changes the other's register allocation.
#pragma once
#include "sfgpu_batch.cuh"

using namespace sfb;

// status codes written per instance
enum { ST_CONVERGED = 0, ST_NOTCONVERGED = SFGPU_ERR_NOTCONVERGED, ST_NONFINITE = SFGPU_ERR_NONFINITE };

template <bool kWide>
__global__ void __launch_bounds__(1024) batch_diis_kernel_t(const InstDesc *__restrict__ descs, int n,
                                                          int *queue, int m, double eta, double tol,
                                                          int maxit, int *status, int *iters, double *errs) {
    __shared__ InstDesc I;
    __shared__ BlockShared sh;
    for (;;) {
        if (threadIdx.x == 0) sh.inst = atomicAdd(queue, 1);
        __syncthreads();
        const int inst = sh.inst;
        if (inst >= n) return;
        {   // copy the descriptor into shared memory
            const int *src = reinterpret_cast<const int *>(descs + inst);
            int *dst = reinterpret_cast<int *>(&I);
            for (int i = threadIdx.x; i < (int)(sizeof(InstDesc) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
        }
        __syncthreads();
        const long long iv = I.nvar;
        double *x = I.x, *x0 = I.x0, *g = I.g, *XR = I.XR, *XX0 = I.XX0;
        // first step: x = -eta * g(x_initial)  (sfnewton.cpp:578-584)
        residual_block<kWide>(I, x, g, sh);
        double acc = 0;
        for (long long r = threadIdx.x; r < iv; r += blockDim.x) {
            double xi = x[r];
            double v = 0.0 - g[r] * eta;
            x0[r] = xi;
            x[r] = v;
            XR[r] = v;
            XX0[r] = v - xi;
            acc += g[r] * g[r];
        }
        block_sum1(acc, sh);
        double err = sqrt(sh.val[0]);
        int k = 0, it = 0, kd = 1, st = ST_CONVERGED;
        if (threadIdx.x == 0)
            for (int i = 0; i < kMaxHist * kMaxHist; i++) sh.gram[i] = 0;
        __syncthreads();
        while (tol < err && it < maxit) {
            it++;
            for (long long r = threadIdx.x; r < iv; r += blockDim.x) x0[r] = x[r];
            __syncthreads();
            residual_block<kWide>(I, x, g, sh);
            k = it % m;
            kd++;
            if (kd > m) kd = m;
            double *xr = XR + (size_t)k * iv, *xx = XX0 + (size_t)k * iv;
            // x -= eta*g; XR[k] = x; XX0[k] = x - x0; Gram row and |g|^2 in one pass
            double part[kMaxHist + 1];
            int slot[kMaxHist + 1];
#pragma unroll
            for (int i = 0; i <= kMaxHist; i++) {
                part[i] = 0;
                slot[i] = (i < kd) ? i : (i == kMaxHist ? kd : -1);
            }
            for (long long r = threadIdx.x; r < iv; r += blockDim.x) {
                const double v = x[r] - g[r] * eta;
                const double d = v - x0[r];
                x[r] = v; xr[r] = v; xx[r] = d;
                part[kMaxHist] += g[r] * g[r];
#pragma unroll
                for (int i = 0; i < kMaxHist; i++) {
                    if (i >= kd) continue;
                    int posi = k - kd + 1 + i;
                    if (posi < 0) posi += m;
                    part[i] += XX0[(size_t)posi * iv + r] * d;
                }
            }
            block_sums_slots<kMaxHist + 1>(part, slot, sh);
            if (threadIdx.x == 0) {
                // shift out the oldest row/column when the memory is full
                // (sfnewton.cpp:624-628), then write the new row
                if (it >= m) {
                    for (int i = 1; i < m; i++)
                        for (int j = 1; j < m; j++) sh.gram[m * (i - 1) + j - 1] = sh.gram[m * i + j];
                }
                for (int i = 0; i < kd; i++) sh.gram[i + m * (kd - 1)] = sh.gram[kd - 1 + m * i] = sh.val[i];
            }
            __syncthreads();
            if (threadIdx.x < 32) {
                for (int e = threadIdx.x; e < kd * kd; e += 32) sh.A[e] = sh.gram[(e % kd) + m * (e / kd)];
                __syncwarp();
                diis_coeff_warp(kd, sh.A, sh.Q, sh.coef);
                if (threadIdx.x == 0) {
                    double nc = 0;
                    for (int i = 0; i < kd; i++) nc += sh.coef[i];
                    for (int i = 0; i < kd; i++) {
                        sh.coef[i] = sh.coef[i] / nc;
                        int posi = k - kd + 1 + i;
                        if (posi < 0) posi += m;
                        sh.pos[i] = posi;
                    }
                }
            }
            __syncthreads();
            for (long long r = threadIdx.x; r < iv; r += blockDim.x) {
                double v = sh.coef[0] * XR[(size_t)sh.pos[0] * iv + r];
                for (int i = 1; i < kd; i++) v += sh.coef[i] * XR[(size_t)sh.pos[i] * iv + r];
                x[r] = v;
            }
            err = sqrt(sh.val[kd]);
            if (!isfinite(err)) { st = ST_NONFINITE; break; }
            __syncthreads();
        }
        if (st == ST_CONVERGED && !(err <= tol)) st = ST_NOTCONVERGED;
        if (threadIdx.x == 0) {
            status[inst] = st;
            iters[inst] = it;
            errs[inst] = err;
        }
        __syncthreads();
    }
}


// the kernel of a batch, by width
using BatchKernel = void (*)(const InstDesc *, int, int *, int, double, double, int, int *, int *, double *);
BatchKernel batch_kernel_wide();
