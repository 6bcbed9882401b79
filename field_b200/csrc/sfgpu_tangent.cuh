// sfgpu_tangent.cuh -- forward-mode derivative (tangent) kernels: for a
// direction v in iteration-variable space they carry dG/dx*v through the
// segment weighting factors, both propagator sweeps, the composition, the
// normalisations (lnGN, restricted and solvent bulk volume fractions), the
// contact averages and the residual, giving the exact Jacobian-vector product
// J(x) v of SF_Solve::residuals in one pass beside the primal values.  SFbox
// only forms J*v by finite differences (SFNewton::Hp, sfnewton.cpp:1662-1688).
#pragma once
#include "sfgpu_kernels.cuh"

namespace sft {
using namespace sfk;

struct MolScalT {           // tangents of the molecule scalars
    double dlngn, dphibulk, dnorm, pad;
};

static __global__ void swf_update_t(DLat L, const double *__restrict__ x, const double *__restrict__ v,
                                    const int *__restrict__ jmap, int nclass, int cls,
                                    const double *__restrict__ range, int pinned,
                                    double *__restrict__ gfull, double *__restrict__ gseg,
                                    double *__restrict__ dgfull, double *__restrict__ dgseg) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < L.M; r += gridDim.x * blockDim.x) {
        int t = lat_map(L, r);
        int j = jmap[t];
        double g = 0, dg = 0;
        if (j >= 0) {
            size_t q = (size_t)j * nclass + cls;
            g = exp(-x[q]);
            dg = -g * v[q];
        }
        gfull[r] = g;
        dgfull[r] = dg;
        bool keep = !pinned || range[t] > 0;
        gseg[r] = keep ? g : 0.0;
        dgseg[r] = keep ? dg : 0.0;
    }
}

// un-weighted first-order stencil at interior position k of row R (the value
// G multiplies)
__device__ __forceinline__ double raw1_row(const DLat &L, const RowInfo &R, const double *__restrict__ p, int k,
                                           int nlast) {
    const int d = L.grad - 1;
    const int t = R.base + k;
    const int km = (k == 1) ? L.map_lo[d] : k - 1;
    const int kp = (k == nlast) ? L.map_hi[d] : k + 1;
    const double a = p[R.base + km], b = p[t], c = p[R.base + kp];
    if (L.grad == 1) {
        if (L.cyl) return b + L.lam_m[t] * (a - b) + L.lam_p[t] * (c - b);
        return b + L.l1 * (a - b - b + c);
    }
    if (L.grad == 2) {
        const double u = p[t + R.up], dd = p[t + R.dn];
        if (L.cyl) return b + L.lam_m[R.x] * (u - b) + L.lam_p[R.x] * (dd - b) + L.l1 * (a + c - b - b);
        double l0 = 1 - 4 * L.l1;
        return l0 * b + L.l1 * (a + c) + L.l1 * (u + dd);
    }
    if (lat_twelve(L)) {
        // FCC / HEX: the twelve neighbours of step12 at weight 1/12, mapped
        // per coordinate as prop1_row maps them
        return step12(L.ltype, 1.0, [&](int dx, int dy, int dz) {
            const int xo = dx < 0 ? R.up : (dx > 0 ? R.dn : 0);
            const int yo = dy < 0 ? R.up2 : (dy > 0 ? R.dn2 : 0);
            const int kk = dz < 0 ? km : (dz > 0 ? kp : k);
            return p[R.base + kk + xo + yo];
        });
    }
    return (p[t + R.up] + p[t + R.dn] + p[t + R.up2] + p[t + R.dn2] + a + c) * (1.0 / 6.0);
}

// primal step (same rounding as step1_rows) plus its tangent
static __global__ void step1_rows_t(DLat L, const double *__restrict__ gin, const double *__restrict__ dgin,
                                    const double *__restrict__ G, const double *__restrict__ dG,
                                    double *__restrict__ gout, double *__restrict__ dgout,
                                    const double *__restrict__ other, const double *__restrict__ dother,
                                    double *__restrict__ phi, double *__restrict__ dphi, int mode) {
    const int worker = blockIdx.x * blockDim.x + threadIdx.x;
    for_interior(L, worker, gridDim.x * blockDim.x, [&](const RowInfo &R, int k, int nlast) {
        const int t = R.base + k;
        const double out = prop1_row(L, R, gin, G, k, nlast);
        const double dout = dG[t] * raw1_row(L, R, gin, k, nlast) + G[t] * raw1_row(L, R, dgin, k, nlast);
        gout[t] = out;
        dgout[t] = dout;
        if (mode == COMP_ACC) {
            phi[t] += out * other[t];
            dphi[t] += dout * other[t] + out * dother[t];
        } else if (mode == COMP_CENTRE) {
            phi[t] = (phi[t] + out * out) * 0.5;
            dphi[t] = (dphi[t] + 2.0 * out * dout) * 0.5;
        }
    });
}

// primal constant-force step (as step1_force_rows) plus its tangent: the
// step is linear in gin with the weights of force_row, so d(out) =
// dG * stencil(gin) + G * stencil(dgin) with the bare (g = 1) stencil
static __global__ void step1_force_rows_t(DLat L, ForceW w, const double *__restrict__ gin,
                                          const double *__restrict__ dgin, const double *__restrict__ G,
                                          const double *__restrict__ dG, double *__restrict__ gout,
                                          double *__restrict__ dgout, const double *__restrict__ other,
                                          const double *__restrict__ dother, double *__restrict__ phi,
                                          double *__restrict__ dphi, int mode) {
    const int worker = blockIdx.x * blockDim.x + threadIdx.x;
    for_interior(L, worker, gridDim.x * blockDim.x, [&](const RowInfo &R, int k, int nlast) {
        const int t = R.base + k;
        const double out = force_row(L, R, gin, G, k, nlast, w);
        const double dout = dG[t] * force_row_g(L, R, gin, 1.0, k, nlast, w) +
                            G[t] * force_row_g(L, R, dgin, 1.0, k, nlast, w);
        gout[t] = out;
        dgout[t] = dout;
        if (mode == COMP_ACC) {
            phi[t] += out * other[t];
            dphi[t] += dout * other[t] + out * dother[t];
        }
    });
}

// primal second-order step (as step2_rows) plus its tangent
static __global__ void step2_rows_t(DLat L, const double *__restrict__ gin, const double *__restrict__ dgin,
                                    const double *__restrict__ G, const double *__restrict__ dG, double S,
                                    double *__restrict__ gout, double *__restrict__ dgout,
                                    const double *__restrict__ other, const double *__restrict__ dother,
                                    double *__restrict__ phi, double *__restrict__ dphi, int mode, int backward) {
    const int M = L.M;
    const double Lw = (1.0 - S) / 4.0;
    const int nx = L.Md[0] - 2, ny = L.Md[1] - 2;
    const int worker = blockIdx.x * blockDim.x + threadIdx.x;
    for_interior(L, worker, gridDim.x * blockDim.x, [&](const RowInfo &R, int k, int nlast) {
        const int t = R.base + k;
        const int zm = (k == 1) ? L.map_lo[2] : k - 1;
        const int zp = (k == nlast) ? L.map_hi[2] : k + 1;
        const int off[6] = {R.up, R.dn, R.up2, R.dn2, zm - k, zp - k};
        const bool sw[6] = {R.x == 1 && is_mirror(L.bc_lo[0]), R.x == nx && is_mirror(L.bc_hi[0]),
                            R.y == 1 && is_mirror(L.bc_lo[1]), R.y == ny && is_mirror(L.bc_hi[1]),
                            k == 1 && is_mirror(L.bc_lo[2]), k == nlast && is_mirror(L.bc_hi[2])};
        const double g = G[t], dg = dG[t];
        const double gS = g * S, gL = g * Lw, dgS = dg * S, dgL = dg * Lw;
        double out[6], dout[6];
        if (!backward) {
            const int dir_of[6] = {0, 2, 4, 5, 3, 1};
#pragma unroll
            for (int kk = 0; kk < 6; kk++) {
                const int dd = dir_of[kk];
                const int src = t + off[dd];
                const int axis = dd >> 1;
                const bool s = sw[dd];
                double acc = 0, dacc = 0;
                bool first = true;
#pragma unroll
                for (int kp = 0; kp < 6; kp++) {
                    if (kp == 5 - kk) continue;
                    int c = kp;
                    if (s) {
                        if (axis == 0 && (kp == 0 || kp == 5)) c = 5 - kp;
                        if (axis == 1 && (kp == 1 || kp == 4)) c = 5 - kp;
                        if (axis == 2 && (kp == 2 || kp == 3)) c = 5 - kp;
                    }
                    const double w = (kp == kk ? gS : gL), dw = (kp == kk ? dgS : dgL);
                    const double p = gin[(size_t)c * M + src], dp = dgin[(size_t)c * M + src];
                    double vv = p * w;
                    if (first) { acc = vv; first = false; } else acc += vv;
                    dacc += dp * w + p * dw;
                }
                out[kk] = acc;
                dout[kk] = dacc;
            }
        } else {
            const int dir_of[6] = {1, 3, 5, 4, 2, 0};
            double v[6], dv[6];
#pragma unroll
            for (int kk = 0; kk < 6; kk++) {
                const int dd = dir_of[kk];
                const int c = sw[dd] ? 5 - kk : kk;
                v[kk] = gin[(size_t)c * M + t + off[dd]];
                dv[kk] = dgin[(size_t)c * M + t + off[dd]];
            }
#pragma unroll
            for (int kq = 0; kq < 6; kq++) {
                double acc = 0, dacc = 0;
                bool first = true;
#pragma unroll
                for (int kp = 5; kp >= 0; kp--) {
                    if (kp == 5 - kq) continue;
                    const double w = (kp == kq ? gS : gL), dw = (kp == kq ? dgS : dgL);
                    double vv = v[kp] * w;
                    if (first) { acc = vv; first = false; } else acc += vv;
                    dacc += dv[kp] * w + v[kp] * dw;
                }
                out[kq] = acc;
                dout[kq] = dacc;
            }
        }
#pragma unroll
        for (int kk = 0; kk < 6; kk++) {
            gout[(size_t)kk * M + t] = out[kk];
            dgout[(size_t)kk * M + t] = dout[kk];
        }
        if (mode == COMP_ACC) {
            double p = phi[t], dp = dphi[t];
#pragma unroll
            for (int kk = 0; kk < 6; kk++) {
                p += out[kk] * other[(size_t)kk * M + t];
                dp += dout[kk] * other[(size_t)kk * M + t] + out[kk] * dother[(size_t)kk * M + t];
            }
            phi[t] = p;
            dphi[t] = dp;
        }
    });
}

// composition of a second-order backward step on interior sites, phi +=
// sum_k mu_k out_k gf_k with the lumped multiplicities, and its tangent
static __global__ void compose2_t(DLat L, int K, const double *__restrict__ out, const double *__restrict__ dout,
                                  const double *__restrict__ gf, const double *__restrict__ dgf,
                                  double *__restrict__ phi, double *__restrict__ dphi) {
    const int M = L.M;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < M; r += gridDim.x * blockDim.x) {
        int c[3];
        lat_coords(L, r, c);
        if (!lat_interior(L, c)) continue;
        double p = phi[r], dp = dphi[r];
        for (int k = 0; k < K; k++) {
            const size_t q = (size_t)k * M + r;
            const double mu = comp_mult(K, k);
            const double a = out[q] * gf[q], da = dout[q] * gf[q] + out[q] * dgf[q];
            p += (mu == 1.0) ? a : a * mu;
            dp += (mu == 1.0) ? da : da * mu;
        }
        phi[r] = p;
        dphi[r] = dp;
    }
}

// a b / G where G > 0, else 0 (dend_combine) and its tangent
static __global__ void combine_t(int M, const double *__restrict__ a, const double *__restrict__ da,
                                 const double *__restrict__ b, const double *__restrict__ db,
                                 const double *__restrict__ G, const double *__restrict__ dG,
                                 double *__restrict__ out, double *__restrict__ dout) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < M; r += gridDim.x * blockDim.x) {
        const double g = G[r];
        if (g > 0) {
            const double o = (a[r] * b[r]) / g;
            out[r] = o;
            dout[r] = (da[r] * b[r] + a[r] * db[r]) / g - o * dG[r] / g;
        } else {
            out[r] = 0;
            dout[r] = 0;
        }
    }
}

// the ring's return walk (ring_phi, SF_HomoRing1stO.cpp:110-160) carrying
// the walk's tangent dY beside Y: phi(k) = phib sum Y^2 / norm0, dphi(k) =
// phib 2 sum Y dY / norm0; four shared-memory buffers of Mmax + 1 values
static __global__ void ring_phi_t(int M, int N, int Mmax, const double *__restrict__ G, const double *__restrict__ dG,
                                  double phibulk, double norm0, double *__restrict__ phi, double *__restrict__ dphi) {
    extern __shared__ double ring_t_sh[];
    __shared__ double red[32], dred[32];
    double *Y = ring_t_sh, *Yn = Y + (Mmax + 1), *dY = Yn + (Mmax + 1), *dYn = dY + (Mmax + 1);
    for (int k = blockIdx.x + 1; k <= M; k += gridDim.x) {
        for (int z = threadIdx.x; z <= Mmax; z += blockDim.x) {
            Y[z] = (z == k) ? G[k - 1] : 0.0;
            dY[z] = (z == k) ? dG[k - 1] : 0.0;
        }
        __syncthreads();
        for (int st = 1; st < N / 2; st++) {
            const int zmin = max(k - st, 1), zmax = min(k + st, Mmax);
            const double ytop = Y[Mmax - 1], dytop = dY[Mmax - 1];
            for (int z = threadIdx.x; z <= Mmax; z += blockDim.x) {
                double v = (z == Mmax) ? ytop : Y[z], dv = (z == Mmax) ? dytop : dY[z];
                if (z >= zmin && z < zmax) {
                    const double a = Y[z - 1], b = Y[z], c = (z + 1 == Mmax) ? ytop : Y[z + 1];
                    const double da = dY[z - 1], db = dY[z], dc = (z + 1 == Mmax) ? dytop : dY[z + 1];
                    const double gz = (z <= M) ? G[z - 1] / 6.0 : 1.0 / 6.0;
                    const double dgz = (z <= M) ? dG[z - 1] / 6.0 : 0.0;
                    v = gz * (a + 4 * b + c);
                    dv = dgz * (a + 4 * b + c) + gz * (da + 4 * db + dc);
                }
                Yn[z] = v;
                dYn[z] = dv;
            }
            __syncthreads();
            double *t = Y; Y = Yn; Yn = t;
            t = dY; dY = dYn; dYn = t;
        }
        double acc = 0, dacc = 0;
        for (int z = threadIdx.x + 1; z <= Mmax; z += blockDim.x) { acc += Y[z] * Y[z]; dacc += 2 * Y[z] * dY[z]; }
        for (int o = 16; o > 0; o >>= 1) {
            acc += __shfl_down_sync(0xffffffffu, acc, o);
            dacc += __shfl_down_sync(0xffffffffu, dacc, o);
        }
        if ((threadIdx.x & 31) == 0) { red[threadIdx.x >> 5] = acc; dred[threadIdx.x >> 5] = dacc; }
        __syncthreads();
        if (threadIdx.x == 0) {
            double v = 0, dv = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) { v += red[w]; dv += dred[w]; }
            phi[k - 1] = v / norm0 * phibulk;
            dphi[k - 1] = dv / norm0 * phibulk;
        }
        __syncthreads();
    }
}

// out = a + b
static __global__ void sum2(size_t n, const double *__restrict__ a, const double *__restrict__ b,
                            double *__restrict__ out) {
    for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < n; r += (size_t)gridDim.x * blockDim.x)
        out[r] = a[r] + b[r];
}

static __global__ void connect_t(int M, int K, const double *__restrict__ a, const double *__restrict__ da,
                                 const double *__restrict__ b, const double *__restrict__ db,
                                 double *__restrict__ phi, double *__restrict__ dphi) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < M; r += gridDim.x * blockDim.x) {
        double p = phi[r], dp = dphi[r];
        for (int k = 0; k < K; k++) {
            size_t q = (size_t)k * M + r;
            const double mu = comp_mult(K, k);   // lumped multiplicities (1 otherwise)
            const double v = a[q] * b[q], dv = da[q] * b[q] + a[q] * db[q];
            p += (mu == 1.0) ? v : v * mu;
            dp += (mu == 1.0) ? dv : dv * mu;
        }
        phi[r] = p;
        dphi[r] = dp;
    }
}

// tangents of lnGN, phibulk and the normalisation (after mol_scalars ran)
static __global__ void mol_scalars_t(MolParam p, int nblocks, const double *__restrict__ dpartial,
                                     const MolScal *__restrict__ scal, MolScalT *__restrict__ tscal, int self) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double dv = 0;
    for (int b = 0; b < nblocks; b++) dv += dpartial[b];
    if (p.K > 1) dv /= 6.0;   // six bond directions, lumped or not (as mol_scalars)
    const MolScal s = scal[self];
    MolScalT t;
    t.pad = 0;
    t.dlngn = dv / exp(s.lngn);
    if (p.freedom == SFGPU_MOL_RESTRICTED) {
        t.dnorm = -s.norm * t.dlngn;
        t.dphibulk = p.pinned ? 0.0 : -(p.theta / exp(s.lngn)) * t.dlngn;
    } else if (p.solvent) {
        double dphib = 0;
        for (int m = 0; m < p.nmol; m++)
            if (m != self) dphib -= tscal[m].dphibulk;
        double phib = s.phibulk;
        t.dphibulk = p.pinned ? 0.0 : dphib;
        t.dnorm = (phib != 0) ? s.norm / phib * dphib : 0.0;
    } else {
        t.dphibulk = 0;
        t.dnorm = 0;
    }
    tscal[self] = t;
}

// CorrectDoubleCountG + normalisation, primal and tangent
static __global__ void finalize_phi_t(int M, const double *__restrict__ G, const double *__restrict__ dG,
                                      double *__restrict__ phi, double *__restrict__ dphi,
                                      const MolScal *__restrict__ scal, const MolScalT *__restrict__ tscal,
                                      int mol, int monomer) {
    const double norm = scal[mol].norm, dnorm = tscal[mol].dnorm;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < M; r += gridDim.x * blockDim.x) {
        double p, dp;
        if (monomer) { p = G[r]; dp = dG[r]; }
        else {
            double g = G[r];
            if (g > 0) { p = phi[r] / g; dp = (dphi[r] - p * dG[r]) / g; }
            else { p = 0; dp = 0; }
        }
        phi[r] = p * norm;
        dphi[r] = dp * norm + p * dnorm;
    }
}

static __global__ void bulk_scalars_t(BulkParam b, ChiTable ct, const MolScalT *__restrict__ tscal,
                                      double *__restrict__ dphib, double *__restrict__ dchib) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int i = 0; i < b.nseg; i++) {
        double v = 0;
        for (int m = 0; m < b.nmol; m++) v += tscal[m].dphibulk * b.frac[i * SFGPU_MAX_SEG + m];
        dphib[i] = v;
    }
    for (int c = 0; c < b.nclass; c++) {
        int st = b.rep[c];
        double v = 0;
        for (int j = 0; j < b.nseg; j++) {
            double x = ct.chi[st * SFGPU_MAX_SEG + j];
            if (x != 0) v += x * dphib[j];
        }
        dchib[c] = v;
    }
}

struct ResParamT {
    const double *dphi[SFGPU_MAX_SEG];     // state phi tangents
    const double *dgfull[SFGPU_MAX_SEG];   // tangent of the representative G, by class
};

static __global__ void residual_t(DLat L, ResParam rp, ResParamT tp, ChiTable ct, const int *__restrict__ sites,
                                  const double *__restrict__ chib, const double *__restrict__ dchib,
                                  double *__restrict__ f, double *__restrict__ df) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < rp.nsites; j += gridDim.x * blockDim.x) {
        int z = sites[j];
        double phit = 0, dphit = 0;
        double rho[SFGPU_MAX_SEG], drho[SFGPU_MAX_SEG];
        for (int i = 0; i < rp.nseg; i++) {
            phit += rp.phi[i][z];
            dphit += tp.dphi[i][z];
            rho[i] = 0;
            drho[i] = 0;
        }
        for (int i = 0; i < rp.nseg; i++) {
            bool need = false;
            for (int c = 0; c < rp.nclass; c++) need |= ct.chi[rp.rep[c] * SFGPU_MAX_SEG + i] != 0;
            if (need) {
                rho[i] = side_fraction(L, rp.phi[i], z);
                drho[i] = side_fraction(L, tp.dphi[i], z);
            }
        }
        double u[SFGPU_MAX_SEG], du[SFGPU_MAX_SEG];
        double av = 0, dav = 0;
        for (int c = 0; c < rp.nclass; c++) {
            int st = rp.rep[c];
            double g = rp.gfull[c][z];
            double v = -log(g);
            double dv = -tp.dgfull[c][z] / g;
            double ci = 0, dci = 0;
            for (int i = 0; i < rp.nseg; i++) {
                double x = ct.chi[st * SFGPU_MAX_SEG + i];
                if (x != 0) { ci += x * rho[i]; dci += x * drho[i]; }
            }
            v -= ci / phit;
            dv += -dci / phit + ci * dphit / (phit * phit);
            v += chib[c];
            dv += dchib[c];
            u[c] = v;
            du[c] = dv;
            av += v;
            dav += dv;
        }
        av /= rp.nclass;
        dav /= rp.nclass;
        for (int c = 0; c < rp.nclass; c++) {
            f[(size_t)j * rp.nclass + c] = -1.0 + 1.0 / phit + u[c] - av;
            df[(size_t)j * rp.nclass + c] = -dphit / (phit * phit) + du[c] - dav;
        }
    }
}

}  // namespace sft
