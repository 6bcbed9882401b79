// sfgpu_internal.cuh -- device-side lattice descriptor and the per-site
// stencils of the SFbox hot path, shared by all kernels of libsfgpu.
//
// Layout in HBM: every profile is a full lattice vector of M doubles
// including SFbox's boundary layers, last gradient fastest (Lat3D.cpp:59-68).
// Boundary entries always hold SetBoundaries copies (Lat3D.cpp:1510-1562),
// so stencils on interior sites read their neighbours directly.  Second-order
// propagators stack the six direction components k*M + z
// (k: 0=+x 1=+y 2=+z 3=-z 4=-y 5=-x, Lat3D2ndO.cpp:70-82).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include "../../include/sfgpu.h"

#ifndef SFGPU_MAX_SEG
#define SFGPU_MAX_SEG 8          // segment types per system (chi held in kernel params)
#endif

struct DLat {
    int grad, cyl, order;
    int M;
    int Md[3];                 // layers incl. boundaries (1 for unused gradients)
    int st[3];                 // strides
    int bc_lo[3], bc_hi[3];    // SFGPU_BOUND_*
    int map_lo[3], map_hi[3];  // coordinate copied into 0 / Md-1
    double l1, l1chi;
    // curved lattices (2D cylinder; 1D cylinder and sphere): step
    // probabilities to the inner / outer neighbour by radial coordinate x,
    // for propagators (lam_*) and contact averages (lamc_*, lambda_chi)
    const double *lam_m, *lam_p;
    const double *lamc_m, *lamc_p;
    // second order: direction components (6 in 3D; 1D and 2D lump the
    // directions along the homogeneous gradients: 3 and 5), and whether a
    // step that reads across the lower / upper boundary of gradient d swaps
    // the +d and -d components
    int K;
    int sw_lo[3], sw_hi[3];
    // 3D lattice type (SFGPU_LATTICE_*) and the contact weights of the
    // 27-site cube (centre, face, edge, corner) for STANDARD, STENCILS, FCC
    int ltype;
    double sl[4];
    // 3D second order: nonzero inside 'lat : stiff_range' (M values), or null
    const double *stiff;
};

struct ChiTable {              // passed by value: small interaction tables
    int nseg;
    double chi[SFGPU_MAX_SEG * SFGPU_MAX_SEG];
};

__host__ __device__ inline void lat_coords(const DLat &L, int z, int c[3]) {
    if (L.grad == 1) { c[0] = z; c[1] = 0; c[2] = 0; return; }
    if (L.grad == 2) { c[0] = z / L.st[0]; c[1] = z - c[0] * L.st[0]; c[2] = 0; return; }
    c[0] = z / L.st[0];
    int r = z - c[0] * L.st[0];
    c[1] = r / L.st[1];
    c[2] = r - c[1] * L.st[1];
}

__host__ __device__ inline bool lat_interior(const DLat &L, const int c[3]) {
    for (int d = 0; d < L.grad; d++)
        if (c[d] == 0 || c[d] == L.Md[d] - 1) return false;
    return true;
}

// Site whose value boundary site z copies (z itself for interior sites and for
// surface layers); *swap gets one bit per mirrored gradient.
__host__ __device__ inline int lat_map(const DLat &L, int z, int *swap = nullptr) {
    int c[3];
    lat_coords(L, z, c);
    int m = 0;
    bool bnd = false;
    for (int d = 0; d < L.grad; d++) {
        if (c[d] == 0) {
            bnd = true; c[d] = L.map_lo[d];
            if (L.bc_lo[d] == SFGPU_BOUND_MIRROR1 || L.bc_lo[d] == SFGPU_BOUND_MIRROR2) m |= 1 << d;
        } else if (c[d] == L.Md[d] - 1) {
            bnd = true; c[d] = L.map_hi[d];
            if (L.bc_hi[d] == SFGPU_BOUND_MIRROR1 || L.bc_hi[d] == SFGPU_BOUND_MIRROR2) m |= 1 << d;
        }
    }
    if (swap) *swap = m;
    if (!bnd) return z;
    return c[0] * L.st[0] + c[1] * L.st[1] + c[2] * L.st[2];
}

__device__ inline int swap_dir(int k, int sw) {
    if (sw & 1) { if (k == 0) k = 5; else if (k == 5) k = 0; }
    if (sw & 2) { if (k == 1) k = 4; else if (k == 4) k = 1; }
    if (sw & 4) { if (k == 2) k = 3; else if (k == 3) k = 2; }
    return k;
}

// First-order step of the twelve-neighbour 3D lattices, g * sum / 12 with
// the neighbours (dx, dy, dz) in the reference's summation order; v(dx, dy,
// dz) returns the input value at that offset.
//   FCC (Lat3DFCC1stO.cpp:79-91): -x-y, +x+y, -x+y, +x-y, -y-z, +y+z, -y+z,
//       +y-z, -x-z, +x+z, -x+z, +x-z
//   HEX (Lat3DHEX1stO.cpp:79-91): -x, +x, -x+y, +y, -y, +x-y, +y-z, -z, +x-z,
//       -x+z, +z, -y+z
template <class V>
__device__ __forceinline__ double step12(int ltype, double g, V &&v) {
    double acc;
    if (ltype == SFGPU_LATTICE_FCC) {
        acc = v(-1, -1, 0) * g;
        acc += v(1, 1, 0) * g;
        acc += v(-1, 1, 0) * g;
        acc += v(1, -1, 0) * g;
        acc += v(0, -1, -1) * g;
        acc += v(0, 1, 1) * g;
        acc += v(0, -1, 1) * g;
        acc += v(0, 1, -1) * g;
        acc += v(-1, 0, -1) * g;
        acc += v(1, 0, 1) * g;
        acc += v(-1, 0, 1) * g;
        acc += v(1, 0, -1) * g;
    } else {
        acc = v(-1, 0, 0) * g;
        acc += v(1, 0, 0) * g;
        acc += v(-1, 1, 0) * g;
        acc += v(0, 1, 0) * g;
        acc += v(0, -1, 0) * g;
        acc += v(1, -1, 0) * g;
        acc += v(0, 1, -1) * g;
        acc += v(0, 0, -1) * g;
        acc += v(1, 0, -1) * g;
        acc += v(-1, 0, 1) * g;
        acc += v(0, 0, 1) * g;
        acc += v(0, -1, 1) * g;
    }
    return acc * (1.0 / 12.0);
}

__host__ __device__ inline bool lat_twelve(const DLat &L) {
    return L.grad == 3 && (L.ltype == SFGPU_LATTICE_FCC || L.ltype == SFGPU_LATTICE_HEX);
}

// First-order step at interior site t: G(t) * stencil(gin) in SFbox's
// operation order (Lat1DFlat1stO.cpp:44-47, Lat2DFlat1stO.cpp:40-46,
// Lat2DCyl1stO.cpp:24-33, Lat3D1stO.cpp:151-157).  The library is compiled
// without FMA contraction so the rounding sequence matches the CPU code.
__device__ __forceinline__ double stencil1(const DLat &L, const double *__restrict__ gin, double g, int t) {
    if (L.grad == 1) {
        double a = gin[t - 1], b = gin[t], c = gin[t + 1];
        if (L.cyl) return g * (b + L.lam_m[t] * (a - b) + L.lam_p[t] * (c - b));   // Lat1DCyl1stO.cpp:21-22
        return g * (b + L.l1 * (a - b - b + c));
    } else if (L.grad == 2) {
        int MY = L.st[0];
        double a = gin[t - 1], b = gin[t], c = gin[t + 1];
        double u = gin[t - MY], d = gin[t + MY];
        if (L.cyl) {
            int x = t / MY;
            return g * (b + L.lam_m[x] * (u - b) + L.lam_p[x] * (d - b) + L.l1 * (a + c - b - b));
        }
        double l0 = 1 - 4 * L.l1;
        return g * (l0 * b + L.l1 * (a + c) + L.l1 * (u + d));
    } else {
        int jx = L.st[0], jy = L.st[1];
        if (lat_twelve(L))
            return step12(L.ltype, g, [&](int dx, int dy, int dz) { return gin[t + dx * jx + dy * jy + dz]; });
        double acc = gin[t - jx] * g;
        acc += gin[t + jx] * g;
        acc += gin[t - jy] * g;
        acc += gin[t + jy] * g;
        acc += gin[t - 1] * g;
        acc += gin[t + 1] * g;
        return acc * (1.0 / 6.0);
    }
}

// Value of site r after one first-order step: interior sites by the stencil;
// boundary sites copy their mapped site (UpdateBoundaries), and a site on a
// surface layer (or a corner reached through one) keeps its value.
__device__ __forceinline__ double prop1_site(const DLat &L, const double *__restrict__ gin,
                                             const double *__restrict__ G, int r) {
    int c[3];
    lat_coords(L, r, c);
    if (lat_interior(L, c)) return stencil1(L, gin, G[r], r);
    int t = lat_map(L, r);
    int ct[3];
    lat_coords(L, t, ct);
    return lat_interior(L, ct) ? stencil1(L, gin, G[t], t) : gin[t];
}

// ---------------------------------------------------------------------------
// Row-wise first-order steps.  The interior of the lattice is walked as rows
// along the fastest gradient; a row knows the (mapped) offsets of its
// neighbour rows, and only the two ends of a row need the mapped left/right
// neighbour, so no per-site division or branch remains.  Boundary entries
// of the output are not written: every neighbour read goes to the site a
// boundary entry would copy (SetBoundaries), and surface layers (which keep
// their value, always 0 for a propagator) are read in place.
// ---------------------------------------------------------------------------
__host__ __device__ inline int lat_mapc(const DLat &L, int d, int c) {
    if (c == 0) return L.map_lo[d];
    if (c == L.Md[d] - 1) return L.map_hi[d];
    return c;
}

__host__ __device__ inline int lat_nrows(const DLat &L) {
    if (L.grad == 1) return 1;
    if (L.grad == 2) return L.Md[0] - 2;
    return (L.Md[0] - 2) * (L.Md[1] - 2);
}

struct RowInfo {
    int base;        // site index of the row's element 0 (boundary position)
    int up, dn;      // offsets of the first-gradient neighbour rows (2D/3D)
    int up2, dn2;    // offsets of the second-gradient neighbour rows (3D)
    int x, y;        // coordinates of the row (x: cylinder tables)
};

__device__ __forceinline__ RowInfo lat_row(const DLat &L, int row) {
    RowInfo R;
    R.up = R.dn = R.up2 = R.dn2 = 0;
    R.y = 0;
    if (L.grad == 1) { R.base = 0; R.x = 0; return R; }
    if (L.grad == 2) {
        int x = row + 1;
        R.x = x;
        R.base = x * L.st[0];
        R.up = (lat_mapc(L, 0, x - 1) - x) * L.st[0];
        R.dn = (lat_mapc(L, 0, x + 1) - x) * L.st[0];
        return R;
    }
    int ny = L.Md[1] - 2;
    int x = row / ny + 1, y = row - (x - 1) * ny + 1;
    R.x = x;
    R.y = y;
    R.base = x * L.st[0] + y * L.st[1];
    R.up = (lat_mapc(L, 0, x - 1) - x) * L.st[0];
    R.dn = (lat_mapc(L, 0, x + 1) - x) * L.st[0];
    R.up2 = (lat_mapc(L, 1, y - 1) - y) * L.st[1];
    R.dn2 = (lat_mapc(L, 1, y + 1) - y) * L.st[1];
    return R;
}

// new value at interior position k (1..n_last) of row R, same operation
// order as stencil1.  kTypes = false compiles the six-neighbour 3D step only
// (callers that accept the standard 3D lattice type alone and must not carry
// the registers of the twelve-neighbour steps).
template <bool kTypes = true>
__device__ __forceinline__ double prop1_row(const DLat &L, const RowInfo &R, const double *__restrict__ gin,
                                            const double *__restrict__ G, int k, int nlast) {
    const int d = L.grad - 1;
    const int t = R.base + k;
    const int km = (k == 1) ? L.map_lo[d] : k - 1;
    const int kp = (k == nlast) ? L.map_hi[d] : k + 1;
    const double g = G[t];
    const double a = gin[R.base + km], b = gin[t], c = gin[R.base + kp];
    if (L.grad == 1) {
        if (L.cyl) return g * (b + L.lam_m[t] * (a - b) + L.lam_p[t] * (c - b));
        return g * (b + L.l1 * (a - b - b + c));
    }
    if (L.grad == 2) {
        const double u = gin[t + R.up], dd = gin[t + R.dn];
        if (L.cyl) return g * (b + L.lam_m[R.x] * (u - b) + L.lam_p[R.x] * (dd - b) + L.l1 * (a + c - b - b));
        double l0 = 1 - 4 * L.l1;
        return g * (l0 * b + L.l1 * (a + c) + L.l1 * (u + dd));
    }
    if (kTypes && lat_twelve(L)) {
        // diagonal neighbours: the x and y row offsets add (each coordinate
        // maps across its own boundary, as SetBoundaries' plane copies do)
        return step12(L.ltype, g, [&](int dx, int dy, int dz) {
            const int xo = dx < 0 ? R.up : (dx > 0 ? R.dn : 0);
            const int yo = dy < 0 ? R.up2 : (dy > 0 ? R.dn2 : 0);
            const int kk = dz < 0 ? km : (dz > 0 ? kp : k);
            return gin[R.base + kk + xo + yo];
        });
    }
    double acc = gin[t + R.up] * g;
    acc += gin[t + R.dn] * g;
    acc += gin[t + R.up2] * g;
    acc += gin[t + R.dn2] * g;
    acc += a * g;
    acc += c * g;
    return acc * (1.0 / 6.0);
}

// Visit the interior sites assigned to this thread: for 1 gradient threads
// stride over the single row; otherwise warps take rows and lanes take the
// positions along the row.  worker = thread index among nworkers threads.
template <class F>
__device__ __forceinline__ void for_interior(const DLat &L, int worker, int nworkers, F &&f) {
    const int d = L.grad - 1;
    const int nlast = L.Md[d] - 2;
    if (L.grad == 1) {
        RowInfo R = lat_row(L, 0);
        for (int k = worker + 1; k <= nlast; k += nworkers) f(R, k, nlast);
        return;
    }
    const int lane = worker & 31, warp = worker >> 5, nw = nworkers >> 5;
    const int nrows = lat_nrows(L);
    for (int row = warp; row < nrows; row += nw) {
        RowInfo R = lat_row(L, row);
        for (int k = lane + 1; k <= nlast; k += 32) f(R, k, nlast);
    }
}

// The walk of for_interior4 for a step fused with a composition
// phi += out * other: the two operands of the four positions are loaded first,
// with the stencils' loads, so that no load waits behind a store of an earlier
// position (phi and other may alias nothing the compiler can see past).
// compute(R, k, nlast) -> double, store(R, k, value, phi_value, other_value).
template <class C, class S>
__device__ __forceinline__ void for_interior4_acc(const DLat &L, int worker, int nworkers,
                                                  const double *__restrict__ pphi, const double *__restrict__ pother,
                                                  C &&compute, S &&store) {
    const int d = L.grad - 1;
    const int nlast = L.Md[d] - 2;
    if (L.grad == 1) {
        RowInfo R = lat_row(L, 0);
        for (int k0 = worker + 1; k0 <= nlast; k0 += 4 * nworkers) {
            double v[4], a[4], b[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int k = k0 + u * nworkers;
                a[u] = (k <= nlast) ? pphi[R.base + k] : 0.0;
                b[u] = (k <= nlast) ? pother[R.base + k] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int k = k0 + u * nworkers;
                v[u] = (k <= nlast) ? compute(R, k, nlast) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int k = k0 + u * nworkers;
                if (k <= nlast) store(R, k, v[u], a[u], b[u]);
            }
        }
        return;
    }
    const int lane = worker & 31, warp = worker >> 5, nw = nworkers >> 5;
    const int nrows = lat_nrows(L);
    for (int row = warp; row < nrows; row += nw) {
        RowInfo R = lat_row(L, row);
        for (int k0 = lane + 1; k0 <= nlast; k0 += 128) {
            double v[4], a[4], b[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int k = k0 + 32 * u;
                a[u] = (k <= nlast) ? pphi[R.base + k] : 0.0;
                b[u] = (k <= nlast) ? pother[R.base + k] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int k = k0 + 32 * u;
                v[u] = (k <= nlast) ? compute(R, k, nlast) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int k = k0 + 32 * u;
                if (k <= nlast) store(R, k, v[u], a[u], b[u]);
            }
        }
    }
}

// Same walk, four positions per lane at a time: all four stencils are
// computed (every load issued) before any result is stored, so one thread
// keeps four rows' worth of loads in flight instead of waiting on each.
// compute(R, k, nlast) -> double, store(R, k, value).
template <class C, class S>
__device__ __forceinline__ void for_interior4(const DLat &L, int worker, int nworkers, C &&compute, S &&store) {
    const int d = L.grad - 1;
    const int nlast = L.Md[d] - 2;
    if (L.grad == 1) {
        RowInfo R = lat_row(L, 0);
        for (int k0 = worker + 1; k0 <= nlast; k0 += 4 * nworkers) {
            double v[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                int k = k0 + u * nworkers;
                v[u] = (k <= nlast) ? compute(R, k, nlast) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                int k = k0 + u * nworkers;
                if (k <= nlast) store(R, k, v[u]);
            }
        }
        return;
    }
    const int lane = worker & 31, warp = worker >> 5, nw = nworkers >> 5;
    const int nrows = lat_nrows(L);
    for (int row = warp; row < nrows; row += nw) {
        RowInfo R = lat_row(L, row);
        for (int k0 = lane + 1; k0 <= nlast; k0 += 128) {
            double v[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                int k = k0 + 32 * u;
                v[u] = (k <= nlast) ? compute(R, k, nlast) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                int k = k0 + 32 * u;
                if (k <= nlast) store(R, k, v[u]);
            }
        }
    }
}

// Contact average <phi>(z) at any site (SideFraction, Lat1DFlat.cpp:511-524,
// Lat2DFlat.cpp:996-1109, Lat2DCylinder.cpp:205-320; Sides with removed
// boundaries in 3D, Lat3D.cpp:1729-1785).  p must carry boundary copies.
// kTypes = false: the standard 3D lattice type only (see prop1_row).
template <bool kTypes = true>
__device__ inline double side_fraction(const DLat &L, const double *__restrict__ p, int z) {
    int c[3];
    lat_coords(L, z, c);
    if (L.grad == 3) {
        if (!lat_interior(L, c)) return 0.0;
        int jx = L.st[0], jy = L.st[1];
        if (!kTypes || L.ltype == SFGPU_LATTICE_STANDARD) {
            const double l1 = 1.0 / 6.0;
            double acc = 0 * p[z];
            acc += l1 * p[z + jx]; acc += l1 * p[z - jx];
            acc += l1 * p[z + jy]; acc += l1 * p[z - jy];
            acc += l1 * p[z + 1];  acc += l1 * p[z - 1];
            return acc;
        }
        auto q = [&](int dx, int dy, int dz) { return p[z + dx * jx + dy * jy + dz]; };
        if (L.ltype == SFGPU_LATTICE_HEX) {
            // the twelve HEX neighbours, 1/12 each (Lat3D.cpp:1733-1752)
            const double l = 1.0 / 12.0;
            double acc = q(1, 0, 0) * l;
            acc += q(-1, 0, 0) * l; acc += q(1, -1, 0) * l; acc += q(0, -1, 0) * l;
            acc += q(0, 1, 0) * l;  acc += q(-1, 1, 0) * l; acc += q(0, -1, 1) * l;
            acc += q(0, 0, 1) * l;  acc += q(-1, 0, 1) * l; acc += q(1, 0, -1) * l;
            acc += q(0, 0, -1) * l; acc += q(0, 1, -1) * l;
            return acc;
        }
        // the 27-site cube: centre, faces, edges, corners (Lat3D.cpp:1765-1778)
        const double l0 = L.sl[0], l1 = L.sl[1], l2 = L.sl[2], l3 = L.sl[3];
        double acc = q(0, 0, 0) * l0;
        acc += q(1, 0, 0) * l1;   acc += q(-1, 0, 0) * l1;
        acc += q(0, 1, 0) * l1;   acc += q(0, -1, 0) * l1;
        acc += q(0, 0, 1) * l1;   acc += q(0, 0, -1) * l1;
        acc += q(1, 1, 0) * l2;   acc += q(1, -1, 0) * l2;
        acc += q(-1, 1, 0) * l2;  acc += q(-1, -1, 0) * l2;
        acc += q(1, 0, 1) * l2;   acc += q(1, 0, -1) * l2;
        acc += q(-1, 0, 1) * l2;  acc += q(-1, 0, -1) * l2;
        acc += q(0, 1, 1) * l2;   acc += q(0, 1, -1) * l2;
        acc += q(0, -1, 1) * l2;  acc += q(0, -1, -1) * l2;
        acc += q(1, 1, 1) * l3;   acc += q(1, 1, -1) * l3;
        acc += q(1, -1, 1) * l3;  acc += q(1, -1, -1) * l3;
        acc += q(-1, 1, 1) * l3;  acc += q(-1, 1, -1) * l3;
        acc += q(-1, -1, 1) * l3; acc += q(-1, -1, -1) * l3;
        return acc;
    }
    double l = L.l1chi;
    if (L.grad == 1 && L.cyl) {
        // Lat1DCylinder::SideFraction (Lat1DCylinder.cpp:159-171)
        int zz = z;
        if (z == 0) {
            if (L.bc_lo[0] == SFGPU_BOUND_SURFACE) return p[0] + L.lamc_p[0] * (-p[0] - p[0] + p[1]);
            zz = L.map_lo[0];
        } else if (z == L.M - 1) {
            if (L.bc_hi[0] == SFGPU_BOUND_SURFACE) return p[z] + L.lamc_m[z] * (-p[z] - p[z] + p[z - 1]);
            zz = L.map_hi[0];
        }
        return p[zz] + L.lamc_p[zz] * (p[zz + 1] - p[zz]) + L.lamc_m[zz] * (p[zz - 1] - p[zz]);
    }
    if (L.grad == 1) {
        int zz = z;
        if (z == 0) {
            if (L.bc_lo[0] == SFGPU_BOUND_SURFACE) return p[0] + l * (-p[0] - p[0] + p[1]);
            zz = L.map_lo[0];
        } else if (z == L.M - 1) {
            if (L.bc_hi[0] == SFGPU_BOUND_SURFACE) return p[z] + l * (-p[z] - p[z] + p[z - 1]);
            zz = L.map_hi[0];
        }
        return p[zz] + l * (p[zz - 1] - p[zz] - p[zz] + p[zz + 1]);
    }
    int MX = L.Md[0], MY = L.Md[1];
    bool onsurf = (c[0] == 0 && L.bc_lo[0] == SFGPU_BOUND_SURFACE) ||
                  (c[0] == MX - 1 && L.bc_hi[0] == SFGPU_BOUND_SURFACE) ||
                  (c[1] == 0 && L.bc_lo[1] == SFGPU_BOUND_SURFACE) ||
                  (c[1] == MY - 1 && L.bc_hi[1] == SFGPU_BOUND_SURFACE);
    int x = c[0], zz = z;
    if (!onsurf) { zz = lat_map(L, z); x = zz / MY; }
    double lm = L.cyl ? L.lam_m[x] : l, lp = L.cyl ? L.lam_p[x] : l;
    if (!onsurf) {
        if (L.cyl)
            return p[zz] + lp * (p[zz + MY] - p[zz]) + lm * (p[zz - MY] - p[zz]) + l * (p[zz - 1] + p[zz + 1] - p[zz] - p[zz]);
        double l0 = 1 - 2 * l - lm - lp;
        return l0 * p[zz] + l * (p[zz - MY] + p[zz + MY]) + l * (p[zz - 1] + p[zz + 1]);
    }
    double l0 = 1 - 2 * l - lm - lp;
    double acc = l0 * p[z];
    if (c[0] > 0) acc += lm * p[z - MY];
    if (c[0] < MX - 1) acc += lp * p[z + MY];
    if (c[1] > 0) acc += l * p[z - 1];
    if (c[1] < MY - 1) acc += l * p[z + 1];
    return acc;
}

#define SFGPU_CUDA_TRY(expr)                                          \
    do {                                                              \
        cudaError_t _e = (expr);                                      \
        if (_e != cudaSuccess) { sfgpu_set_error(_e, #expr, __FILE__, __LINE__); return SFGPU_ERR_CUDA; } \
    } while (0)

void sfgpu_set_error(cudaError_t e, const char *what, const char *file, int line);
int fail_unsupported(const char *what);   // records the message, returns SFGPU_ERR_UNSUPPORTED
