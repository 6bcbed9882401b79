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

// neighbour i (0..11) of the twelve-neighbour steps, in step12's order
__device__ __forceinline__ void twelve_offset(int ltype, int i, int &dx, int &dy, int &dz) {
    // FCC (Lat3DFCC1stO.cpp:79-91) and HEX (Lat3DHEX1stO.cpp:79-91) bond sets
    const signed char fcc[12][3] = {{-1, -1, 0}, {1, 1, 0},  {-1, 1, 0},  {1, -1, 0}, {0, -1, -1}, {0, 1, 1},
                                    {0, -1, 1},  {0, 1, -1}, {-1, 0, -1}, {1, 0, 1},  {-1, 0, 1},  {1, 0, -1}};
    const signed char hex[12][3] = {{-1, 0, 0}, {1, 0, 0},  {-1, 1, 0}, {0, 1, 0},  {0, -1, 0}, {1, -1, 0},
                                    {0, 1, -1}, {0, 0, -1}, {1, 0, -1}, {-1, 0, 1}, {0, 0, 1},  {0, -1, 1}};
    const signed char *o = (ltype == SFGPU_LATTICE_FCC) ? fcc[i] : hex[i];
    dx = o[0];
    dy = o[1];
    dz = o[2];
}

// contact neighbour i (0..11) of the HEX lattice (side_fraction's set,
// Lat3D.cpp:1733-1752)
__device__ __forceinline__ void hex_side_offset(int i, int &dx, int &dy, int &dz) {
    const signed char o[12][3] = {{1, 0, 0},  {-1, 0, 0}, {1, -1, 0}, {0, -1, 0}, {0, 1, 0},  {-1, 1, 0},
                                  {0, -1, 1}, {0, 0, 1},  {-1, 0, 1}, {1, 0, -1}, {0, 0, -1}, {0, 1, -1}};
    dx = o[i][0];
    dy = o[i][1];
    dz = o[i][2];
}

// out[map(n)] += c_n * y[t] for every site n the first-order stencil at
// interior t reads (the transpose of the un-weighted stencil, raw1_row)
__device__ __forceinline__ void scatter1(const DLat &L, const RowInfo &R, int k, int nlast, double y,
                                         double *__restrict__ out) {
    const int d = L.grad - 1;
    const int t = R.base + k;
    const int km = R.base + ((k == 1) ? L.map_lo[d] : k - 1);
    const int kp = R.base + ((k == nlast) ? L.map_hi[d] : k + 1);
    if (L.grad == 1) {
        if (L.cyl) {
            const double lm = L.lam_m[t], lp = L.lam_p[t];
            atomicAdd(out + t, (1.0 - lm - lp) * y);
            atomicAdd(out + km, lm * y);
            atomicAdd(out + kp, lp * y);
            return;
        }
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
    if (lat_twelve(L)) {
        // transpose of the twelve-neighbour step (step12): 1/12 to each
        // (mapped) neighbour it read
        const double c12 = y * (1.0 / 12.0);
        for (int i = 0; i < 12; i++) {
            int dx, dy, dz;
            twelve_offset(L.ltype, i, dx, dy, dz);
            const int xo = dx < 0 ? R.up : (dx > 0 ? R.dn : 0);
            const int yo = dy < 0 ? R.up2 : (dy > 0 ? R.dn2 : 0);
            const int kk = dz < 0 ? km : (dz > 0 ? kp : t);
            atomicAdd(out + kk + xo + yo, c12);
        }
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

// transpose of the bare constant-force stencil (force_row_g with g = 1):
// y spread to the sites the step read with their weights
__device__ __forceinline__ void scatter_force(const DLat &L, const RowInfo &R, int k, int nlast, double y,
                                              const ForceW &w, double *__restrict__ out) {
    const int d = L.grad - 1;
    const int t = R.base + k;
    const int km = R.base + ((k == 1) ? L.map_lo[d] : k - 1);
    const int kp = R.base + ((k == nlast) ? L.map_hi[d] : k + 1);
    if (L.grad == 1 && !L.cyl) {   // b + a1 (a - b) + a2 (c - b)
        atomicAdd(out + t, (1.0 - w.a1 - w.a2) * y);
        atomicAdd(out + km, w.a1 * y);
        atomicAdd(out + kp, w.a2 * y);
        return;
    }
    if (L.grad == 1) {             // f-1 a + f0 b + f1 c
        atomicAdd(out + km, L.lam_m[t] * w.a2 * y);
        atomicAdd(out + t, (1 - L.lam_p[t] - L.lam_m[t]) / w.a3 * y);
        atomicAdd(out + kp, L.lam_p[t] * w.a1 * y);
        return;
    }
    if (L.grad == 2) {             // (b + lm (u - b) + lp (d - b) + l1 (a a1 + c a2 - 2 b)) / a3
        const double lm = L.lam_m[R.x], lp = L.lam_p[R.x], yy = y / w.a3;
        atomicAdd(out + t, (1.0 - lm - lp - 2.0 * L.l1) * yy);
        atomicAdd(out + t + R.up, lm * yy);
        atomicAdd(out + t + R.dn, lp * yy);
        atomicAdd(out + km, L.l1 * w.a1 * yy);
        atomicAdd(out + kp, L.l1 * w.a2 * yy);
        return;
    }
    const double c = y * w.a3;     // (x-, x+, y-, y+, z- a1, z+ a2) a3
    atomicAdd(out + t + R.up, c);
    atomicAdd(out + t + R.dn, c);
    atomicAdd(out + t + R.up2, c);
    atomicAdd(out + t + R.dn2, c);
    atomicAdd(out + km, c * w.a1);
    atomicAdd(out + kp, c * w.a2);
}

// one reverse constant-force step: Gbar[t] += cot[t] * A_f p and
// out += A_f^T (G * cot)
static __global__ void adj_chain_step_force(DLat L, ForceW w, const double *__restrict__ cot,
                                            const double *__restrict__ G, const double *__restrict__ p,
                                            double *__restrict__ gbar, double *__restrict__ out) {
    const int worker = blockIdx.x * blockDim.x + threadIdx.x;
    for_interior(L, worker, gridDim.x * blockDim.x, [&](const RowInfo &R, int k, int nlast) {
        const int t = R.base + k;
        const double c = cot[t];
        if (c == 0.0) return;
        gbar[t] += c * force_row_g(L, R, p, 1.0, k, nlast, w);
        scatter_force(L, R, k, nlast, G[t] * c, w, out);
    });
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

// out[k][t] = phibar_raw[t] * q[k][t] on interior sites (0 elsewhere), K components
static __global__ void adj_init(DLat L, int K, const double *__restrict__ phibar_raw, const double *__restrict__ q,
                                double *__restrict__ out) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < L.M; r += gridDim.x * blockDim.x) {
        int c[3];
        lat_coords(L, r, c);
        const bool in = lat_interior(L, c);
        for (int k = 0; k < K; k++) {
            // lumped components carry their multiplicity in the composition
            const double mu = comp_mult(K, k), v = phibar_raw[r] * q[(size_t)k * L.M + r];
            out[(size_t)k * L.M + r] = in ? ((mu == 1.0) ? v : v * mu) : 0.0;
        }
    }
}

// gbar[t] += sum_k cot[k][t] on interior sites (slice 1 / slice N hold G in
// every component)
static __global__ void adj_add_interior(DLat L, int K, const double *__restrict__ cot, double *__restrict__ gbar) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < L.M; r += gridDim.x * blockDim.x) {
        int c[3];
        lat_coords(L, r, c);
        if (!lat_interior(L, c)) continue;
        double a = 0;
        for (int k = 0; k < K; k++) a += cot[(size_t)k * L.M + r];
        gbar[r] += a;
    }
}

// out[k][t] += s * w[t] (interior, every component); s = *sptr * scale
static __global__ void adj_axpy_interior(DLat L, int K, const double *__restrict__ w,
                                         const double *__restrict__ sptr, double scale, double *__restrict__ out) {
    const double s = *sptr * scale;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < L.M; r += gridDim.x * blockDim.x) {
        int c[3];
        lat_coords(L, r, c);
        if (!lat_interior(L, c)) continue;
        for (int k = 0; k < K; k++) {
            const double mu = comp_mult(K, k), v = s * w[r];   // lumped: the lnGN sum weighs components
            out[(size_t)k * L.M + r] += (mu == 1.0) ? v : v * mu;
        }
    }
}

// One reverse step of the 3D second-order stiff-range steps (the transpose
// of step2_rows with STEP2_STIFF or STEP2_ISO): every read of the forward
// step (the mapped, component-swapped source) scattered with its weight --
// per site S inside the range and 0.2 outside, taken at the index the
// forward step takes it, or G/6 for the isotropic steps (whose forward -y
// component reads +z twice and -y never) -- and G's cotangent from the
// unweighted sums.
static __global__ void adj_step2v(DLat L, const double *__restrict__ cot, const double *__restrict__ G,
                                  const double *__restrict__ p, double S, int backward, int wmode,
                                  double *__restrict__ gbar, double *__restrict__ out) {
    const int M = L.M;
    const int nx = L.Md[0] - 2, ny = L.Md[1] - 2;
    const int worker = blockIdx.x * blockDim.x + threadIdx.x;
    for_interior(L, worker, gridDim.x * blockDim.x, [&](const RowInfo &R, int k, int nlast) {
        const int t = R.base + k;
        double c[6];
        bool any = false;
#pragma unroll
        for (int kk = 0; kk < 6; kk++) {
            c[kk] = cot[(size_t)kk * M + t];
            any |= c[kk] != 0.0;
        }
        if (!any) return;
        const int zm = (k == 1) ? L.map_lo[2] : k - 1;
        const int zp = (k == nlast) ? L.map_hi[2] : k + 1;
        const int off[6] = {R.up, R.dn, R.up2, R.dn2, zm - k, zp - k};
        const bool sw[6] = {R.x == 1 && is_mirror(L.bc_lo[0]), R.x == nx && is_mirror(L.bc_hi[0]),
                            R.y == 1 && is_mirror(L.bc_lo[1]), R.y == ny && is_mirror(L.bc_hi[1]),
                            k == 1 && is_mirror(L.bc_lo[2]), k == nlast && is_mirror(L.bc_hi[2])};
        const int raw[6] = {L.st[0], L.st[1], 1, 1, L.st[1], L.st[0]};
        auto ps_at = [&](int i) { return (L.stiff[i] != 0) ? S : 0.2; };
        const double g = G[t];
        double gb = 0;
        if (!backward) {
            const int dir_of[6] = {0, 2, 4, 5, 3, 1};
            for (int kk = 0; kk < 6; kk++) {
                const int dd = dir_of[kk];
                const int src = t + off[dd];
                const int axis = dd >> 1;
                const bool sflag = sw[dd];
                auto cidx = [&](int kp) {
                    int cc = kp;
                    if (sflag) {
                        if (axis == 0 && (kp == 0 || kp == 5)) cc = 5 - kp;
                        if (axis == 1 && (kp == 1 || kp == 4)) cc = 5 - kp;
                        if (axis == 2 && (kp == 2 || kp == 3)) cc = 5 - kp;
                    }
                    return cc;
                };
                double acc = 0;
                if (wmode == STEP2_ISO) {
                    const int seq4[6] = {0, 2, 2, 3, 4, 5};
                    for (int q = 0; q < 6; q++) {
                        const int cc = cidx(kk == 4 ? seq4[q] : q);
                        acc += p[(size_t)cc * M + src] * (1.0 / 6.0);
                        atomicAdd(out + (size_t)cc * M + src, c[kk] * g * (1.0 / 6.0));
                    }
                } else {
                    const int pi = (kk < 3) ? t - raw[kk] : t;
                    const double ps = ps_at(pi), pl = (1.0 - ps) / 4.0;
                    for (int kp = 0; kp < 6; kp++) {
                        if (kp == 5 - kk) continue;
                        const double w = (kp == kk) ? ps : pl;
                        const int cc = cidx(kp);
                        acc += p[(size_t)cc * M + src] * w;
                        atomicAdd(out + (size_t)cc * M + src, c[kk] * g * w);
                    }
                }
                gb += c[kk] * acc;
            }
        } else {
            const int dir_of[6] = {1, 3, 5, 4, 2, 0};
            for (int kp = 0; kp < 6; kp++) {
                const int dd = dir_of[kp];
                const int cc = sw[dd] ? 5 - kp : kp;
                const int src = t + off[dd];
                const double v = p[(size_t)cc * M + src];
                double wc = 0;   // sum_kq w(kq, kp) cot[kq], w without G
                for (int kq = 0; kq < 6; kq++) {
                    double w;
                    if (wmode == STEP2_ISO) {
                        w = 1.0 / 6.0;
                    } else {
                        if (kp == 5 - kq) continue;
                        const int pi = (kp >= 3) ? t - raw[kp] : t;
                        const double ps = ps_at(pi), pl = (1.0 - ps) / 4.0;
                        w = (kp == kq) ? ps : pl;
                    }
                    wc += w * c[kq];
                }
                atomicAdd(out + (size_t)cc * M + src, g * wc);
                gb += wc * v;
            }
        }
        gbar[t] += gb;
    });
}

// One reverse step of the lumped 1D/2D second-order lattices (the transpose
// of step2l_rows, flat and curved): gbar[t] += sum_k cot[k][t] (A p)[k][t]
// and out += A^T (G cot), every read of the forward step (its mapped site,
// its component after boundary swaps, the curved lattices' mixture
// f read + (1 - f) reflected component at t) scattered with its weight.
static __global__ void adj_step2l(DLat L, const double *__restrict__ cot, const double *__restrict__ G,
                                  const double *__restrict__ p, double S, int backward, double *__restrict__ gbar,
                                  double *__restrict__ out) {
    const int M = L.M;
    const Lump2 q = lump2_of(L.grad);
    const double Lw = (1.0 - S) / 4.0;
    const int worker = blockIdx.x * blockDim.x + threadIdx.x;
    for_interior(L, worker, gridDim.x * blockDim.x, [&](const RowInfo &R, int k, int nlast) {
        const int t = R.base + k;
        const int x = (L.grad == 1) ? k : R.x, y = (L.grad == 1) ? 0 : k;
        double c[5];
        bool any = false;
        for (int kk = 0; kk < q.K; kk++) {
            c[kk] = cot[(size_t)kk * M + t];
            any |= c[kk] != 0.0;
        }
        if (!any) return;
        const double g = G[t];
        double gb = 0;
        if (!backward) {
            for (int kk = 0; kk < q.K; kk++) {
                int src = t, sm = 0;
                if (q.axis[kk] >= 0) src = lump2_nb(L, x, y, q.axis[kk], -q.sgn[kk], sm);
                const bool mix = L.cyl && q.axis[kk] == 0;
                const double f = mix ? 6 * ((-q.sgn[kk] > 0) ? L.lam_p[x] : L.lam_m[x]) : 1.0;
                const double y0 = g * c[kk];
                double acc = 0;
                for (int kp = 0; kp < q.K; kp++) {
                    const double w = lump2_w(q, kk, kp, S, Lw);
                    if (w == 0.0) continue;
                    const int ci = lump2_read(q, kp, q.axis[kk], sm);
                    double r = p[(size_t)ci * M + src];
                    if (mix) {
                        const int refl = lump2_read(q, kp, 0, 1);
                        r = f * r + (1.0 - f) * p[(size_t)refl * M + t];
                        atomicAdd(out + (size_t)ci * M + src, y0 * w * f);
                        atomicAdd(out + (size_t)refl * M + t, y0 * w * (1.0 - f));
                    } else {
                        atomicAdd(out + (size_t)ci * M + src, y0 * w);
                    }
                    acc += w * r;
                }
                gb += c[kk] * acc;
            }
        } else {
            for (int kp = 0; kp < q.K; kp++) {
                int src = t, sm = 0;
                if (q.axis[kp] >= 0) src = lump2_nb(L, x, y, q.axis[kp], q.sgn[kp], sm);
                const int ci = lump2_read(q, kp, q.axis[kp], sm);
                const bool mixed = L.cyl && q.axis[kp] == 0 && (L.grad == 1 || q.sgn[kp] < 0);
                const double f = mixed ? 6 * ((q.sgn[kp] > 0) ? L.lam_p[x] : L.lam_m[x]) : 1.0;
                double v = p[(size_t)ci * M + src];
                if (mixed) v = f * v + (1.0 - f) * p[(size_t)lump2_swap(q, kp) * M + t];
                double wc = 0;   // sum_kq w(kq, kp) cot[kq]
                for (int kq = 0; kq < q.K; kq++) {
                    const double w = lump2_w(q, kq, kp, S, Lw);
                    if (w != 0.0) wc += w * c[kq];
                }
                const double vb = g * wc;
                if (mixed) {
                    atomicAdd(out + (size_t)ci * M + src, vb * f);
                    atomicAdd(out + (size_t)lump2_swap(q, kp) * M + t, vb * (1.0 - f));
                } else {
                    atomicAdd(out + (size_t)ci * M + src, vb);
                }
                gb += wc * v;
            }
        }
        gbar[t] += gb;
    });
}

// One reverse second-order step (the transpose of step2_rows): with
// new = G * A(S) p, gbar[t] += sum_k cot[k][t] * (A(S) p)[k][t] and
// out += A(S)^T (G * cot), scattered with FP64 atomics to the (mapped,
// component-swapped) sources each output component read.
static __global__ void adj_step2(DLat L, const double *__restrict__ cot, const double *__restrict__ G,
                                 const double *__restrict__ p, double S, int backward, double *__restrict__ gbar,
                                 double *__restrict__ out) {
    const int M = L.M;
    const double Lw = (1.0 - S) / 4.0;
    const int nx = L.Md[0] - 2, ny = L.Md[1] - 2;
    const int worker = blockIdx.x * blockDim.x + threadIdx.x;
    for_interior(L, worker, gridDim.x * blockDim.x, [&](const RowInfo &R, int k, int nlast) {
        const int t = R.base + k;
        double c[6];
        bool any = false;
#pragma unroll
        for (int kk = 0; kk < 6; kk++) {
            c[kk] = cot[(size_t)kk * M + t];
            any |= c[kk] != 0.0;
        }
        if (!any) return;
        const int zm = (k == 1) ? L.map_lo[2] : k - 1;
        const int zp = (k == nlast) ? L.map_hi[2] : k + 1;
        const int off[6] = {R.up, R.dn, R.up2, R.dn2, zm - k, zp - k};
        const bool sw[6] = {R.x == 1 && is_mirror(L.bc_lo[0]), R.x == nx && is_mirror(L.bc_hi[0]),
                            R.y == 1 && is_mirror(L.bc_lo[1]), R.y == ny && is_mirror(L.bc_hi[1]),
                            k == 1 && is_mirror(L.bc_lo[2]), k == nlast && is_mirror(L.bc_hi[2])};
        const double g = G[t];
        double raw[6];
        if (!backward) {
            const int dir_of[6] = {0, 2, 4, 5, 3, 1};
#pragma unroll
            for (int kk = 0; kk < 6; kk++) {
                const int dd = dir_of[kk];
                const int src = t + off[dd];
                const int axis = dd >> 1;
                const bool s = sw[dd];
                const double y = g * c[kk];
                double acc = 0;
#pragma unroll
                for (int kp = 0; kp < 6; kp++) {
                    if (kp == 5 - kk) continue;
                    int cc = kp;
                    if (s) {
                        if (axis == 0 && (kp == 0 || kp == 5)) cc = 5 - kp;
                        if (axis == 1 && (kp == 1 || kp == 4)) cc = 5 - kp;
                        if (axis == 2 && (kp == 2 || kp == 3)) cc = 5 - kp;
                    }
                    const double wgt = (kp == kk) ? S : Lw;
                    acc += p[(size_t)cc * M + src] * wgt;
                    if (y != 0.0) atomicAdd(out + (size_t)cc * M + src, y * wgt);
                }
                raw[kk] = acc;
            }
        } else {
            const int dir_of[6] = {1, 3, 5, 4, 2, 0};
            double v[6], vbar[6];
            size_t at[6];
#pragma unroll
            for (int kk = 0; kk < 6; kk++) {
                const int dd = dir_of[kk];
                const int cc = sw[dd] ? 5 - kk : kk;
                at[kk] = (size_t)cc * M + t + off[dd];
                v[kk] = p[at[kk]];
                vbar[kk] = 0.0;
            }
#pragma unroll
            for (int kq = 0; kq < 6; kq++) {
                const double y = g * c[kq];
                double acc = 0;
#pragma unroll
                for (int kp = 0; kp < 6; kp++) {
                    if (kp == 5 - kq) continue;
                    const double wgt = (kp == kq) ? S : Lw;
                    acc += v[kp] * wgt;
                    vbar[kp] += y * wgt;
                }
                raw[kq] = acc;
            }
#pragma unroll
            for (int kp = 0; kp < 6; kp++)
                if (vbar[kp] != 0.0) atomicAdd(out + at[kp], vbar[kp]);
        }
        double gb = 0;
#pragma unroll
        for (int kk = 0; kk < 6; kk++) gb += c[kk] * raw[kk];
        gbar[t] += gb;
    });
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
    // stencil with lambda_chi; 3D: the contact set of the lattice type)
    int c[3];
    lat_coords(L, z, c);
    auto at = [&](int cx, int cy, int cz) {
        int cc[3] = {cx, cy, cz};
        for (int d = 0; d < L.grad; d++) cc[d] = lat_mapc(L, d, cc[d]);
        return cc[0] * L.st[0] + cc[1] * L.st[1] + cc[2] * L.st[2];
    };
    if (L.grad == 3) {
        if (L.ltype == SFGPU_LATTICE_STANDARD) {
            const double q = y * (1.0 / 6.0);
            atomicAdd(out + at(c[0] + 1, c[1], c[2]), q);
            atomicAdd(out + at(c[0] - 1, c[1], c[2]), q);
            atomicAdd(out + at(c[0], c[1] + 1, c[2]), q);
            atomicAdd(out + at(c[0], c[1] - 1, c[2]), q);
            atomicAdd(out + at(c[0], c[1], c[2] + 1), q);
            atomicAdd(out + at(c[0], c[1], c[2] - 1), q);
            return;
        }
        if (L.ltype == SFGPU_LATTICE_HEX) {
            // the twelve HEX contact neighbours at 1/12 (side_fraction's set)
            const double q = y * (1.0 / 12.0);
            for (int i = 0; i < 12; i++) {
                int dx, dy, dz;
                hex_side_offset(i, dx, dy, dz);
                atomicAdd(out + at(c[0] + dx, c[1] + dy, c[2] + dz), q);
            }
            return;
        }
        // FCC and stencils: the 27-site cube, weight by the offset's class
        // (centre, face, edge, corner)
        for (int dx = -1; dx <= 1; dx++)
            for (int dy = -1; dy <= 1; dy++)
                for (int dz = -1; dz <= 1; dz++) {
                    const double wgt = L.sl[abs(dx) + abs(dy) + abs(dz)];
                    if (wgt != 0.0) atomicAdd(out + at(c[0] + dx, c[1] + dy, c[2] + dz), wgt * y);
                }
        return;
    }
    const double l = L.l1chi;
    if (L.grad == 1 && L.cyl) {
        const double lm = L.lamc_m[z], lp = L.lamc_p[z];
        atomicAdd(out + z, (1.0 - lp - lm) * y);
        atomicAdd(out + at(c[0] + 1, 0, 0), lp * y);
        atomicAdd(out + at(c[0] - 1, 0, 0), lm * y);
        return;
    }
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

// d(w . f)/d chi at fixed x: chi enters f only through the contact averages
// and the bulk terms of u' (SF_Solve.cpp:527-591), so for class c with
// representative state a = rep(c), d f_c' / d chi(a, i) = (delta_cc' - 1/n_class)
// (phib_i - <phi_i>/phi_T).  dchi[a * nseg + i] accumulates over sites.
static __global__ void adj_chi(DLat L, ResParam rp, const int *__restrict__ sites, const double *__restrict__ w,
                               const double *__restrict__ phib, double *__restrict__ dchi) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < rp.nsites; j += gridDim.x * blockDim.x) {
        const int z = sites[j];
        double phit = 0;
        for (int i = 0; i < rp.nseg; i++) phit += rp.phi[i][z];
        double mean = 0;
        for (int c = 0; c < rp.nclass; c++) mean += w[(size_t)j * rp.nclass + c];
        mean /= rp.nclass;
        for (int i = 0; i < rp.nseg; i++) {
            const double term = phib[i] - side_fraction(L, rp.phi[i], z) / phit;
            for (int c = 0; c < rp.nclass; c++) {
                const double ub = w[(size_t)j * rp.nclass + c] - mean;
                atomicAdd(dchi + rp.rep[c] * rp.nseg + i, ub * term);
            }
        }
    }
}

// out[idx] += v for a value side_fraction read at idx: a boundary entry that
// holds a copy of another site (SetBoundaries) passes v on to that site;
// surface layers keep it
__device__ __forceinline__ void side_put(const DLat &L, int idx, double v, double *__restrict__ out) {
    atomicAdd(out + lat_map(L, idx), v);
}

// Transpose of side_fraction(L, p, z) at any site z (surface layers
// included): out += y * d<p>(z)/dp, branch by branch as side_fraction reads.
__device__ inline void side_fraction_adj(const DLat &L, int z, double y, double *__restrict__ out) {
    if (y == 0.0) return;
    int c[3];
    lat_coords(L, z, c);
    if (L.grad == 3) {
        if (lat_interior(L, c)) side_scatter(L, z, y, out);   // every 3D lattice type
        return;
    }
    const double l = L.l1chi;
    if (L.grad == 1 && L.cyl) {
        int zz = z;
        if (z == 0) {
            if (L.bc_lo[0] == SFGPU_BOUND_SURFACE) {
                const double lp = L.lamc_p[0];
                side_put(L, 0, (1.0 - 2.0 * lp) * y, out);
                side_put(L, 1, lp * y, out);
                return;
            }
            zz = L.map_lo[0];
        } else if (z == L.M - 1) {
            if (L.bc_hi[0] == SFGPU_BOUND_SURFACE) {
                const double lm = L.lamc_m[z];
                side_put(L, z, (1.0 - 2.0 * lm) * y, out);
                side_put(L, z - 1, lm * y, out);
                return;
            }
            zz = L.map_hi[0];
        }
        const double lm = L.lamc_m[zz], lp = L.lamc_p[zz];
        side_put(L, zz, (1.0 - lp - lm) * y, out);
        side_put(L, zz + 1, lp * y, out);
        side_put(L, zz - 1, lm * y, out);
        return;
    }
    if (L.grad == 1) {
        int zz = z;
        if (z == 0) {
            if (L.bc_lo[0] == SFGPU_BOUND_SURFACE) {
                side_put(L, 0, (1.0 - 2.0 * l) * y, out);
                side_put(L, 1, l * y, out);
                return;
            }
            zz = L.map_lo[0];
        } else if (z == L.M - 1) {
            if (L.bc_hi[0] == SFGPU_BOUND_SURFACE) {
                side_put(L, z, (1.0 - 2.0 * l) * y, out);
                side_put(L, z - 1, l * y, out);
                return;
            }
            zz = L.map_hi[0];
        }
        side_put(L, zz, (1.0 - 2.0 * l) * y, out);
        side_put(L, zz - 1, l * y, out);
        side_put(L, zz + 1, l * y, out);
        return;
    }
    const int MX = L.Md[0], MY = L.Md[1];
    const bool onsurf = (c[0] == 0 && L.bc_lo[0] == SFGPU_BOUND_SURFACE) ||
                        (c[0] == MX - 1 && L.bc_hi[0] == SFGPU_BOUND_SURFACE) ||
                        (c[1] == 0 && L.bc_lo[1] == SFGPU_BOUND_SURFACE) ||
                        (c[1] == MY - 1 && L.bc_hi[1] == SFGPU_BOUND_SURFACE);
    int x = c[0], zz = z;
    if (!onsurf) { zz = lat_map(L, z); x = zz / MY; }
    const double lm = L.cyl ? L.lam_m[x] : l, lp = L.cyl ? L.lam_p[x] : l;
    if (!onsurf) {
        if (L.cyl) {
            side_put(L, zz, (1.0 - lp - lm - 2.0 * l) * y, out);
            side_put(L, zz + MY, lp * y, out);
            side_put(L, zz - MY, lm * y, out);
        } else {
            side_put(L, zz, (1.0 - 2.0 * l - lm - lp) * y, out);
            side_put(L, zz - MY, l * y, out);
            side_put(L, zz + MY, l * y, out);
        }
        side_put(L, zz - 1, l * y, out);
        side_put(L, zz + 1, l * y, out);
        return;
    }
    side_put(L, z, (1.0 - 2.0 * l - lm - lp) * y, out);
    if (c[0] > 0) side_put(L, z - MY, lm * y, out);
    if (c[0] < MX - 1) side_put(L, z + MY, lp * y, out);
    if (c[1] > 0) side_put(L, z - 1, l * y, out);
    if (c[1] < MY - 1) side_put(L, z + 1, l * y, out);
}

// Free energy F = sum_z wf [sum_m p_m (ln(N_m) + lnC_m)/N_m - p_m chemintref_m
// + sum_(m,i) q_mi ln G_i + 1/2 sum_(i,j) chi_ij phi_i <phi_j>] (the form of
// free_energy_partial).  Contact part of the state cotangents:
// phibar_i += 1/2 wf sum_j chi_ij <phi_j> directly and, through the
// averages, the transpose of SideFraction applied to 1/2 wf sum_i chi_ij phi_i.
struct FeAdjParam {
    int nseg;
    const double *phi[SFGPU_MAX_SEG];
    double *phibar[SFGPU_MAX_SEG];
};
static __global__ void fe_contact_adj(DLat L, FeAdjParam fp, ChiTable ct, const double *__restrict__ wf) {
    for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < L.M; z += gridDim.x * blockDim.x) {
        const double w = wf[z];
        if (w == 0) continue;
        for (int i = 0; i < fp.nseg; i++) {
            double ci = 0;
            for (int j = 0; j < fp.nseg; j++) {
                const double x = ct.chi[i * SFGPU_MAX_SEG + j];
                if (x != 0) ci += x * side_fraction(L, fp.phi[j], z);
            }
            if (ci != 0) atomicAdd(fp.phibar[i] + z, 0.5 * w * ci);
        }
        for (int j = 0; j < fp.nseg; j++) {
            double yj = 0;
            for (int i = 0; i < fp.nseg; i++) {
                const double x = ct.chi[i * SFGPU_MAX_SEG + j];
                if (x != 0) yj += x * fp.phi[i][z];
            }
            side_fraction_adj(L, z, 0.5 * w * yj, fp.phibar[j]);
        }
    }
}

// cotangent of molecule m's profile of segment i: the state part plus
// wf ((ln N + lnC)/N - chemintref + ln G_i)
static __global__ void fe_mol_phibar(int M, const double *__restrict__ state_bar, const double *__restrict__ wf,
                                     const double *__restrict__ G, double invN, double lnN, double chemintref,
                                     const MolScal *__restrict__ scal, int mol, double *__restrict__ out) {
    const double a = invN * (lnN + scal[mol].lnc) - chemintref;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < M; r += gridDim.x * blockDim.x) {
        const double w = wf[r];
        double v = state_bar[r];
        if (w != 0) {
            const double g = G[r];
            v += w * (a + (g > 0 ? log(g) : 0.0));
        }
        out[r] = v;
    }
}

// Gbar_i += wf q_mi / G_i where G_i > 0 (the q ln G term), for one molecule profile
static __global__ void fe_gbar(int M, const double *__restrict__ q, const double *__restrict__ wf,
                               const double *__restrict__ G, double *__restrict__ gbar) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < M; r += gridDim.x * blockDim.x) {
        const double w = wf[r], g = G[r];
        if (w != 0 && g > 0) gbar[r] += w * q[r] / g;
    }
}

// Reverse sweep of the ring's return walk (ring_phi, SF_HomoRing1stO.cpp:
// 110-160): for every interior site k the walk is run forward again with its
// levels Y_0 .. Y_{N/2-1} kept in `levels` (Mmax + 1 values each, one set per
// block), then walked back with the cotangent Ybar, from
// Ybar = 2 Y phibar(k) phib / norm0 (phi(k) = phib sum_z Y(z)^2 / norm0).  A
// step maps Y to Y'(z) = g_z (Y(z-1) + 4 Y(z) + Y(z+1)) on the window
// zmin <= z < zmax (g_z = G(z-1) / 6 up to M, 1/6 beyond), copies Y(Mmax-1)
// into Y(Mmax) before it, and keeps Y elsewhere; its transpose gathers, for
// every j, the window's three terms, the untouched value, and at Mmax - 1
// the copy.  G's cotangent collects Ybar'(z) (Y(z-1) + 4 Y(z) + Y(z+1)) / 6
// per step and Ybar_0(k) at the start in shared memory, then goes to Gbar
// with one atomic add per site; a boundary layer's share goes to the site it
// copies (a surface layer's G is a constant).  The ring's scalars (lnGN 0,
// its phibulk the input's) carry no cotangent.  Boundary sites' profiles
// are copies whose cotangents arrive folded into their mapped sites.
// Reverse of the bond tree's composition phi_raw += U D (connect, K = 1) on
// interior sites: Ubar += pr D, Dbar += pr U
static __global__ void tree_adj_connect(DLat L, const double *__restrict__ pr, const double *__restrict__ U,
                                        const double *__restrict__ D, double *__restrict__ Ubar,
                                        double *__restrict__ Dbar) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < L.M; r += gridDim.x * blockDim.x) {
        int c[3];
        lat_coords(L, r, c);
        if (!lat_interior(L, c)) continue;
        const double v = pr[r];
        Ubar[r] += v * D[r];
        Dbar[r] += v * U[r];
    }
}

// Reverse of dst = a b / G (dend_combine; 0 where G <= 0) on interior sites:
// abar = dstbar b / G (written), bbar += dstbar a / G, Gbar -= dstbar dst / G
static __global__ void tree_adj_combine(DLat L, const double *__restrict__ dstbar, const double *__restrict__ a,
                                        const double *__restrict__ b, const double *__restrict__ G,
                                        const double *__restrict__ dst, double *__restrict__ abar,
                                        double *__restrict__ bbar, double *__restrict__ gbar) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < L.M; r += gridDim.x * blockDim.x) {
        int c[3];
        lat_coords(L, r, c);
        const double g = G[r];
        if (!lat_interior(L, c) || !(g > 0)) { abar[r] = 0.0; continue; }
        const double v = dstbar[r];
        abar[r] = v * b[r] / g;
        bbar[r] += v * a[r] / g;
        gbar[r] -= v * dst[r] / g;
    }
}

constexpr int kRingAdjBlocks = 148 * 4;   // blocks of ring_phi_adj (each keeps one set of levels)
static __global__ void ring_phi_adj(DLat L, int M, int N, int Mmax, const double *__restrict__ G,
                                    const double *__restrict__ phibar, double phibulk, double norm0,
                                    double *__restrict__ levels, double *__restrict__ gbar) {
    extern __shared__ double ring_a_sh[];
    double *Yb = ring_a_sh, *Ybn = Yb + (Mmax + 1), *gacc = Ybn + (Mmax + 1);
    const int W = Mmax + 1, nlev = N / 2;
    double *lev = levels + (size_t)blockIdx.x * nlev * W;
    for (int k = blockIdx.x + 1; k <= M; k += gridDim.x) {
        int ck[3];
        lat_coords(L, k - 1, ck);
        if (!lat_interior(L, ck)) continue;   // block-uniform
        const double pb = phibar[k - 1];
        if (pb == 0.0) continue;               // block-uniform
        // forward walk, every level kept
        for (int z = threadIdx.x; z <= Mmax; z += blockDim.x) {
            lev[z] = (z == k) ? G[k - 1] : 0.0;
            gacc[z] = 0.0;
        }
        __syncthreads();
        for (int st = 1; st < nlev; st++) {
            const double *Y = lev + (size_t)(st - 1) * W;
            double *Yn = lev + (size_t)st * W;
            const int zmin = max(k - st, 1), zmax = min(k + st, Mmax);
            const double ytop = Y[Mmax - 1];
            for (int z = threadIdx.x; z <= Mmax; z += blockDim.x) {
                double v = (z == Mmax) ? ytop : Y[z];
                if (z >= zmin && z < zmax) {
                    const double a = Y[z - 1], b = Y[z], c = (z + 1 == Mmax) ? ytop : Y[z + 1];
                    const double gz = (z <= M) ? G[z - 1] / 6.0 : 1.0 / 6.0;
                    v = gz * (a + 4 * b + c);
                }
                Yn[z] = v;
            }
            __syncthreads();
        }
        // cotangent of the last level
        const double *Yl = lev + (size_t)(nlev - 1) * W;
        const double sc = 2.0 * pb * phibulk / norm0;
        for (int z = threadIdx.x; z <= Mmax; z += blockDim.x) Yb[z] = (z >= 1) ? sc * Yl[z] : 0.0;
        __syncthreads();
        for (int st = nlev - 1; st >= 1; st--) {
            const double *Y = lev + (size_t)(st - 1) * W;   // the step's input
            const int zmin = max(k - st, 1), zmax = min(k + st, Mmax);
            const double ytop = Y[Mmax - 1];
            auto in_win = [&](int z) { return z >= zmin && z < zmax; };
            auto gz = [&](int z) { return (z <= M) ? G[z - 1] / 6.0 : 1.0 / 6.0; };
            for (int j = threadIdx.x; j <= Mmax; j += blockDim.x) {
                double v = 0.0;
                if (j >= 1 && j < Mmax) {
                    if (!in_win(j)) v += Yb[j];
                    if (in_win(j + 1)) v += gz(j + 1) * Yb[j + 1];
                    if (in_win(j)) v += 4.0 * gz(j) * Yb[j];
                    if (j - 1 >= 1 && in_win(j - 1)) v += gz(j - 1) * Yb[j - 1];
                    if (j == Mmax - 1) {
                        v += Yb[Mmax];
                        if (in_win(Mmax - 1)) v += gz(Mmax - 1) * Yb[Mmax - 1];
                    }
                }
                Ybn[j] = v;
                if (in_win(j) && j <= M) {
                    const double a = Y[j - 1], b = Y[j], c = (j + 1 == Mmax) ? ytop : Y[j + 1];
                    gacc[j] += Yb[j] * ((a + 4 * b + c) / 6.0);
                }
            }
            __syncthreads();
            double *t = Yb; Yb = Ybn; Ybn = t;
        }
        if (threadIdx.x == 0) gacc[k] += Yb[k];   // Y_0(k) = G(k - 1)
        __syncthreads();
        for (int z = threadIdx.x + 1; z <= M; z += blockDim.x) {
            const double v = gacc[z];
            if (v == 0.0) continue;
            int c[3];
            lat_coords(L, z - 1, c);
            int t = z - 1;
            if (!lat_interior(L, c)) {
                t = lat_map(L, z - 1);
                if (t == z - 1) continue;      // surface layer: G there is a constant
            }
            atomicAdd(gbar + t, v);
        }
        __syncthreads();
    }
}

}  // namespace sfa
