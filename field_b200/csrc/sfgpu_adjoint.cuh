// sfgpu_adjoint.cuh -- reverse-mode (adjoint) kernels of the residual for
// first-order lattices: given a cotangent w on f = residuals(x) they produce
// J(x)^T w.  The chain part is the adjoint of the propagator recursions:
// with Gf(s) = G_s * A Gf(s-1) and Gb(s) = G_s * A Gb(s+1),
//   Fbar(s-1) = phibar_raw . Gb(s-1) + A^T (G_s * Fbar(s)),   Gbar_s += Fbar(s) * A Gf(s-1)
//   Bbar(s+1) = phibar_raw . Gf(s+1) + A^T (G_s * Bbar(s)),   Gbar_s += Bbar(s) * A Gb(s+1)
// run as a descending and an ascending sweep over stored Gf and Gb.  A^T is
// applied by scattering every interior value to the (mapped) sites its
// stencil reads, with FP64 atomics.
#pragma once
#include "sfgpu_tangent.cuh"

namespace sfa {
using namespace sfk;
using namespace sft;

// out[map(n)] += c_n * y[t] for every site n the first-order stencil at
// interior t reads (the transpose of the un-weighted stencil, raw1_row)
__device__ __forceinline__ void scatter1(const DLat &L, const RowInfo &R, int k, int nlast, double y,
                                         double *__restrict__ out) {
    const int d = L.grad - 1;
    const int t = R.base + k;
    const int km = R.base + ((k == 1) ? L.map_lo[d] : k - 1);
    const int kp = R.base + ((k == nlast) ? L.map_hi[d] : k + 1);
    if (L.grad == 1) {
        atomicAdd(out + t, (1.0 - 2.0 * L.l1) * y);
        atomicAdd(out + km, L.l1 * y);
        atomicAdd(out + kp, L.l1 * y);
        return;
    }
    if (L.grad == 2) {
        double lm = L.l1, lp = L.l1, l0 = 1 - 4 * L.l1;
        if (L.cyl) { lm = L.lam_m[R.x]; lp = L.lam_p[R.x]; l0 = 1 - lm - lp - 2 * L.l1; }
        atomicAdd(out + t, l0 * y);
        atomicAdd(out + t + R.up, lm * y);
        atomicAdd(out + t + R.dn, lp * y);
        atomicAdd(out + km, L.l1 * y);
        atomicAdd(out + kp, L.l1 * y);
        return;
    }
    const double c = y * (1.0 / 6.0);
    atomicAdd(out + t + R.up, c);
    atomicAdd(out + t + R.dn, c);
    atomicAdd(out + t + R.up2, c);
    atomicAdd(out + t + R.dn2, c);
    atomicAdd(out + km, c);
    atomicAdd(out + kp, c);
}

// one reverse chain step: Gbar[t] += cot[t] * A p (p = the neighbouring
// propagator slice), and out += A^T (G * cot)
static __global__ void adj_chain_step(DLat L, const double *__restrict__ cot, const double *__restrict__ G,
                                      const double *__restrict__ p, double *__restrict__ gbar,
                                      double *__restrict__ out) {
    const int worker = blockIdx.x * blockDim.x + threadIdx.x;
    for_interior(L, worker, gridDim.x * blockDim.x, [&](const RowInfo &R, int k, int nlast) {
        const int t = R.base + k;
        const double c = cot[t];
        if (c == 0.0) return;
        gbar[t] += c * raw1_row(L, R, p, k, nlast);
        scatter1(L, R, k, nlast, G[t] * c, out);
    });
}

// out[t] = phibar_raw[t] * q[t] on interior sites (0 elsewhere)
static __global__ void adj_init(DLat L, const double *__restrict__ phibar_raw, const double *__restrict__ q,
                                double *__restrict__ out) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < L.M; r += gridDim.x * blockDim.x) {
        int c[3];
        lat_coords(L, r, c);
        out[r] = lat_interior(L, c) ? phibar_raw[r] * q[r] : 0.0;
    }
}

// gbar[t] += cot[t] on interior sites (slice 1 / slice N equal G itself)
static __global__ void adj_add_interior(DLat L, const double *__restrict__ cot, double *__restrict__ gbar) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < L.M; r += gridDim.x * blockDim.x) {
        int c[3];
        lat_coords(L, r, c);
        if (lat_interior(L, c)) gbar[r] += cot[r];
    }
}

// out[t] += s * w[t] (interior)
static __global__ void adj_axpy_interior(DLat L, const double *__restrict__ w, const double *__restrict__ sptr,
                                         double *__restrict__ out) {
    const double s = *sptr;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < L.M; r += gridDim.x * blockDim.x) {
        int c[3];
        lat_coords(L, r, c);
        if (lat_interior(L, c)) out[r] += s * w[r];
    }
}

// residual adjoint: x-direct terms, phi-state cotangents (with the
// transpose of SideFraction scattered to mapped sites) and the bulk
// contact-term cotangents per class
struct AdjResParam {
    double *phibar[SFGPU_MAX_SEG];   // state phi cotangents (M each, zeroed)
    double *chibbar;                 // per class, zeroed
};
__device__ __forceinline__ void side_scatter(const DLat &L, int z, double y, double *__restrict__ out) {
    // transpose of side_fraction at an interior site (1D/2D: the contact
    // stencil with lambda_chi; 3D: the six neighbours at 1/6)
    int c[3];
    lat_coords(L, z, c);
    auto at = [&](int cx, int cy, int cz) {
        int cc[3] = {cx, cy, cz};
        for (int d = 0; d < L.grad; d++) cc[d] = lat_mapc(L, d, cc[d]);
        return cc[0] * L.st[0] + cc[1] * L.st[1] + cc[2] * L.st[2];
    };
    if (L.grad == 3) {
        const double q = y * (1.0 / 6.0);
        atomicAdd(out + at(c[0] + 1, c[1], c[2]), q);
        atomicAdd(out + at(c[0] - 1, c[1], c[2]), q);
        atomicAdd(out + at(c[0], c[1] + 1, c[2]), q);
        atomicAdd(out + at(c[0], c[1] - 1, c[2]), q);
        atomicAdd(out + at(c[0], c[1], c[2] + 1), q);
        atomicAdd(out + at(c[0], c[1], c[2] - 1), q);
        return;
    }
    const double l = L.l1chi;
    if (L.grad == 1) {
        atomicAdd(out + z, (1.0 - 2.0 * l) * y);
        atomicAdd(out + at(c[0] - 1, 0, 0), l * y);
        atomicAdd(out + at(c[0] + 1, 0, 0), l * y);
        return;
    }
    double lm = l, lp = l, l0 = 1 - 4 * l;
    if (L.cyl) { lm = L.lam_m[c[0]]; lp = L.lam_p[c[0]]; l0 = 1 - lm - lp - 2 * l; }
    atomicAdd(out + z, l0 * y);
    atomicAdd(out + at(c[0] - 1, c[1], 0), lm * y);
    atomicAdd(out + at(c[0] + 1, c[1], 0), lp * y);
    atomicAdd(out + at(c[0], c[1] - 1, 0), l * y);
    atomicAdd(out + at(c[0], c[1] + 1, 0), l * y);
}

static __global__ void adj_residual(DLat L, ResParam rp, ChiTable ct, const int *__restrict__ sites,
                                    const double *__restrict__ w, AdjResParam ap, double *__restrict__ xbar) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < rp.nsites; j += gridDim.x * blockDim.x) {
        const int z = sites[j];
        double phit = 0;
        double rho[SFGPU_MAX_SEG];
        for (int i = 0; i < rp.nseg; i++) { phit += rp.phi[i][z]; rho[i] = 0; }
        for (int i = 0; i < rp.nseg; i++) {
            bool need = false;
            for (int c = 0; c < rp.nclass; c++) need |= ct.chi[rp.rep[c] * SFGPU_MAX_SEG + i] != 0;
            if (need) rho[i] = side_fraction(L, rp.phi[i], z);
        }
        double fb[SFGPU_MAX_SEG], ub[SFGPU_MAX_SEG];
        double mean = 0;
        for (int c = 0; c < rp.nclass; c++) { fb[c] = w[(size_t)j * rp.nclass + c]; mean += fb[c]; }
        mean /= rp.nclass;
        double phitbar = 0;
        double rhobar[SFGPU_MAX_SEG];
        for (int i = 0; i < rp.nseg; i++) rhobar[i] = 0;
        for (int c = 0; c < rp.nclass; c++) {
            ub[c] = fb[c] - mean;               // u'_c enters f_c and the class average
            phitbar -= fb[c] / (phit * phit);   // from 1/phi_T
            const int st = rp.rep[c];
            double ci = 0;
            for (int i = 0; i < rp.nseg; i++) {
                double x = ct.chi[st * SFGPU_MAX_SEG + i];
                if (x != 0) { ci += x * rho[i]; rhobar[i] -= ub[c] * x / phit; }
            }
            phitbar += ub[c] * ci / (phit * phit);
            xbar[(size_t)j * rp.nclass + c] += ub[c];     // u' contains -ln G = x
            atomicAdd(ap.chibbar + c, ub[c]);
        }
        for (int i = 0; i < rp.nseg; i++) {
            atomicAdd(ap.phibar[i] + z, phitbar);
            if (rhobar[i] != 0) side_scatter(L, z, rhobar[i], ap.phibar[i]);
        }
    }
}

}  // namespace sfa
