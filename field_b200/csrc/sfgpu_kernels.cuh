// sfgpu_kernels.cuh -- streaming kernels of the single-system path.
// Every kernel is grid-stride over lattice sites; all scalars that one
// residual evaluation needs (lnGN, bulk volume fractions, normalisations)
// stay in device memory so a whole evaluation is one asynchronous launch
// sequence that can be captured in a CUDA graph.
#pragma once
#include "sfgpu_internal.cuh"

namespace sfk {

// Programmatic dependent launch (PTX griddepcontrol, sm_90+): a step launched
// with programmatic stream serialization may be scheduled while the step
// before it drains; it waits here for that step's completion and memory
// before touching global memory, then lets the next step be scheduled.  In
// a launch without the attribute both are no-ops.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}


constexpr int kBlock = 256;

struct MolScal {            // per-molecule device scalars
    double lngn, phibulk, lnc, norm;
};

// SF_Solve::UpdateSWF (SF_Solve.cpp:794-852), SF_State/SF_MolState::UpdateSWF
// (SF_State.cpp:281-287, SF_MolState.cpp:147-151) and the SetBoundaries of the
// molecule drivers (SF_Homopol1stO.cpp:105-106): G = exp(-x) on sites with
// iteration variables, 0 elsewhere, pinned segments masked to their range.
static __global__ void swf_update(DLat L, const double *__restrict__ x, const int *__restrict__ jmap,
                           int nclass, int cls, const double *__restrict__ range, int pinned,
                           double *__restrict__ gfull, double *__restrict__ gseg) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < L.M; r += gridDim.x * blockDim.x) {
        int t = lat_map(L, r);
        int j = jmap[t];
        double v = (j >= 0) ? exp(-x[(size_t)j * nclass + cls]) : 0.0;
        gfull[r] = v;
        gseg[r] = pinned ? (range[t] > 0 ? v : 0.0) : v;
    }
}

// composition modes of a propagator step
enum { COMP_NONE = 0, COMP_ACC = 1, COMP_CENTRE = 2 };

// One first-order step gout = G * stencil(gin), boundaries written as the
// copies SFbox's UpdateBoundaries makes (surface layers keep their value),
// fused with the composition phi += gout * other (ConnectG,
// Lat1DFlat1stO.cpp:259-265) or, for the centre segment of an odd
// homopolymer, phi = (phi + gout^2) * 0.5 (SF_Homopol1stO.cpp:580-587).
static __global__ void step1(DLat L, const double *__restrict__ gin, const double *__restrict__ G,
                      double *__restrict__ gout, const double *__restrict__ other,
                      double *__restrict__ phi, int mode) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < L.M; r += gridDim.x * blockDim.x) {
        double out = prop1_site(L, gin, G, r);
        gout[r] = out;
        if (mode == COMP_ACC) phi[r] += out * other[r];
        else if (mode == COMP_CENTRE) phi[r] = (phi[r] + out * out) * 0.5;
    }
}

// The same step over interior sites only (row-wise, see for_interior); the
// path used inside residual evaluations.  Boundary entries of gout and phi
// are left untouched.
static __global__ void step1_rows(DLat L, const double *__restrict__ gin, const double *__restrict__ G,
                                  double *__restrict__ gout, const double *__restrict__ other,
                                  double *__restrict__ phi, int mode) {
    pdl_enter();
    const int worker = blockIdx.x * blockDim.x + threadIdx.x;
    if (mode == COMP_ACC) {
        for_interior4_acc(L, worker, gridDim.x * blockDim.x, phi, other,
            [&](const RowInfo &R, int k, int nlast) { return prop1_row(L, R, gin, G, k, nlast); },
            [&](const RowInfo &R, int k, double out, double ph, double ot) {
                const int t = R.base + k;
                gout[t] = out;
                phi[t] = ph + out * ot;
            });
        return;
    }
    for_interior4(L, worker, gridDim.x * blockDim.x,
        [&](const RowInfo &R, int k, int nlast) { return prop1_row(L, R, gin, G, k, nlast); },
        [&](const RowInfo &R, int k, double out) {
            const int t = R.base + k;
            gout[t] = out;
            if (mode == COMP_CENTRE) phi[t] = (phi[t] + out * out) * 0.5;
        });
}

// First-order step on a 3D lattice, x-marching: a block owns a 32 (z) x 8
// (y) tile of columns and walks `xc` consecutive x planes.  The x-1/x/x+1
// values of a column stay in registers, the y/z neighbours come from the
// current plane staged in shared memory, so every value of gin is read from
// L2/HBM about once (plus a 1-plane overlap per chunk and the tile halos).
// Neighbour coordinates 0 and n+1 read the site their boundary entry would
// copy; boundary entries are neither read nor written.  Operation order as
// stencil1 (Lat3D1stO.cpp:151-157).
constexpr int kTZ = 32, kTY = 8;
static __global__ void __launch_bounds__(kTZ * kTY)
step3d_march(DLat L, const double *__restrict__ gin, const double *__restrict__ G,
             double *__restrict__ gout, const double *__restrict__ other, double *__restrict__ phi,
             int mode, int xc) {
    __shared__ double tile[kTY + 2][kTZ + 2];
    pdl_enter();
    const int nx = L.Md[0] - 2, ny = L.Md[1] - 2, nz = L.Md[2] - 2;
    const int jx = L.st[0], jy = L.st[1];
    const int tz = threadIdx.x % kTZ, ty = threadIdx.x / kTZ;
    const int z = blockIdx.x * kTZ + tz + 1;
    const int y = blockIdx.y * kTY + ty + 1;
    const int x0 = blockIdx.z * xc + 1;
    if (x0 > nx) return;
    const int x1 = min(x0 + xc - 1, nx);
    const bool act = (z <= nz) && (y <= ny);
    const int zm = lat_mapc(L, 2, z - 1), zp = lat_mapc(L, 2, z + 1);
    const int ym = lat_mapc(L, 1, y - 1), yp = lat_mapc(L, 1, y + 1);
    const bool hz0 = (tz == 0), hz1 = (tz == kTZ - 1) || (z == nz);
    const bool hy0 = (ty == 0), hy1 = (ty == kTY - 1) || (y == ny);
    const int col = y * jy + z;
    double vprev = 0, vcur = 0;
    if (act) {
        vprev = gin[lat_mapc(L, 0, x0 - 1) * jx + col];
        vcur = gin[x0 * jx + col];
    }
    for (int x = x0; x <= x1; x++) {
        double vnext = 0, g = 0, hz_lo = 0, hz_hi = 0, hy_lo = 0, hy_hi = 0;
        const int base = x * jx;
        if (act) {
            vnext = gin[lat_mapc(L, 0, x + 1) * jx + col];
            g = G[base + col];
            if (hz0) hz_lo = gin[base + y * jy + zm];
            if (hz1) hz_hi = gin[base + y * jy + zp];
            if (hy0) hy_lo = gin[base + ym * jy + z];
            if (hy1) hy_hi = gin[base + yp * jy + z];
        }
        __syncthreads();
        if (act) {
            // only active columns write their own slot: in a partial tile the
            // slot right of the last column is that column's halo
            tile[ty + 1][tz + 1] = vcur;
            if (hz0) tile[ty + 1][0] = hz_lo;
            if (hz1) tile[ty + 1][tz + 2] = hz_hi;
            if (hy0) tile[0][tz + 1] = hy_lo;
            if (hy1) tile[ty + 2][tz + 1] = hy_hi;
        }
        __syncthreads();
        if (act) {
            double acc = vprev * g;
            acc += vnext * g;
            acc += tile[ty][tz + 1] * g;
            acc += tile[ty + 2][tz + 1] * g;
            acc += tile[ty + 1][tz] * g;
            acc += tile[ty + 1][tz + 2] * g;
            const double out = acc * (1.0 / 6.0);
            const int t = base + col;
            gout[t] = out;
            if (mode == COMP_ACC) phi[t] += out * other[t];
            else if (mode == COMP_CENTRE) phi[t] = (phi[t] + out * out) * 0.5;
        }
        vprev = vcur;
        vcur = vnext;
    }
}

// The same x-marching step software-pipelined: the loads of plane x+1 (the
// column value two planes ahead, G, and for a composition phi and the other
// propagator) are issued before plane x is computed, so every thread keeps a
// plane's worth of loads in flight across the barrier, and the (z, y) tile is
// double-buffered so one barrier per plane suffices (a thread writes buffer
// b^1 for plane x+1 only after every thread passed plane x's barrier, i.e.
// finished reading b^1 for plane x-1).  Same operands and operation order as
// step3d_march, so the results are bit-identical.
// kCompose = false compiles the composition-free (forward) step alone, whose
// registers then leave room for more resident blocks.
template <bool kCompose>
static __global__ void __launch_bounds__(kTZ * kTY, kCompose ? 4 : 6)
step3d_march_pf(DLat L, const double *__restrict__ gin, const double *__restrict__ G,
                double *__restrict__ gout, const double *__restrict__ other, double *__restrict__ phi,
                int mode, int xc) {
    __shared__ double tile[2][kTY + 2][kTZ + 2];
    pdl_enter();
    const int nx = L.Md[0] - 2, ny = L.Md[1] - 2, nz = L.Md[2] - 2;
    const int jx = L.st[0], jy = L.st[1];
    const int tz = threadIdx.x % kTZ, ty = threadIdx.x / kTZ;
    const int z = blockIdx.x * kTZ + tz + 1;
    const int y = blockIdx.y * kTY + ty + 1;
    const int x0 = blockIdx.z * xc + 1;
    if (x0 > nx) return;
    const int x1 = min(x0 + xc - 1, nx);
    const bool act = (z <= nz) && (y <= ny);
    const int zm = lat_mapc(L, 2, z - 1), zp = lat_mapc(L, 2, z + 1);
    const int ym = lat_mapc(L, 1, y - 1), yp = lat_mapc(L, 1, y + 1);
    const bool hz0 = (tz == 0), hz1 = (tz == kTZ - 1) || (z == nz);
    const bool hy0 = (ty == 0), hy1 = (ty == kTY - 1) || (y == ny);
    const int col = y * jy + z;
    const bool acc_mode = kCompose && (mode == COMP_ACC), centre = kCompose && (mode == COMP_CENTRE);
    // registers: column values of planes x-1, x, x+1; plane x's G, halos and
    // composition operands
    double vprev = 0, vcur = 0, vnext = 0, g = 0, hzl = 0, hzh = 0, hyl = 0, hyh = 0, ot = 0, ph = 0;
    if (act) {
        const int base = x0 * jx;
        vprev = gin[lat_mapc(L, 0, x0 - 1) * jx + col];
        vcur = gin[base + col];
        vnext = gin[lat_mapc(L, 0, x0 + 1) * jx + col];
        g = G[base + col];
        if (hz0) hzl = gin[base + y * jy + zm];
        if (hz1) hzh = gin[base + y * jy + zp];
        if (hy0) hyl = gin[base + ym * jy + z];
        if (hy1) hyh = gin[base + yp * jy + z];
        if (acc_mode) { ot = other[base + col]; ph = phi[base + col]; }
        else if (centre) ph = phi[base + col];
    }
    int b = 0;
    for (int x = x0; x <= x1; x++) {
        // loads of plane x+1, in flight while plane x is computed
        double vn2 = 0, gn = 0, nzl = 0, nzh = 0, nyl = 0, nyh = 0, otn = 0, phn = 0;
        const bool more = x < x1;
        if (act && more) {
            const int nb = (x + 1) * jx;
            vn2 = gin[lat_mapc(L, 0, x + 2) * jx + col];
            gn = G[nb + col];
            if (hz0) nzl = gin[nb + y * jy + zm];
            if (hz1) nzh = gin[nb + y * jy + zp];
            if (hy0) nyl = gin[nb + ym * jy + z];
            if (hy1) nyh = gin[nb + yp * jy + z];
            if (acc_mode) { otn = other[nb + col]; phn = phi[nb + col]; }
            else if (centre) phn = phi[nb + col];
        }
        if (act) {
            tile[b][ty + 1][tz + 1] = vcur;
            if (hz0) tile[b][ty + 1][0] = hzl;
            if (hz1) tile[b][ty + 1][tz + 2] = hzh;
            if (hy0) tile[b][0][tz + 1] = hyl;
            if (hy1) tile[b][ty + 2][tz + 1] = hyh;
        }
        __syncthreads();
        if (act) {
            double acc = vprev * g;
            acc += vnext * g;
            acc += tile[b][ty][tz + 1] * g;
            acc += tile[b][ty + 2][tz + 1] * g;
            acc += tile[b][ty + 1][tz] * g;
            acc += tile[b][ty + 1][tz + 2] * g;
            const double out = acc * (1.0 / 6.0);
            const int t = x * jx + col;
            gout[t] = out;
            if (acc_mode) phi[t] = ph + out * ot;
            else if (centre) phi[t] = (ph + out * out) * 0.5;
        }
        vprev = vcur; vcur = vnext; vnext = vn2;
        g = gn; hzl = nzl; hzh = nzh; hyl = nyl; hyh = nyh; ot = otn; ph = phn;
        b ^= 1;
    }
}

// The composition-free (forward) step of step3d_march_pf with two y rows
// per thread: a block owns a 32 (z) x 16 (y) tile, thread (tz, ty) the
// columns y and y + 8, so every thread keeps two columns' loads of plane x+1
// in flight (the forward step moves half the bytes of a composing one, and
// one column per thread leaves its reads latency-bound).  Same operands and
// operation order, bit-identical results.
constexpr int kTY2 = 2 * kTY;
static __global__ void __launch_bounds__(kTZ * kTY, 3)
step3d_march_pf2(DLat L, const double *__restrict__ gin, const double *__restrict__ G, double *__restrict__ gout,
                 int xc) {
    __shared__ double tile[2][kTY2 + 2][kTZ + 2];
    pdl_enter();
    const int nx = L.Md[0] - 2, ny = L.Md[1] - 2, nz = L.Md[2] - 2;
    const int jx = L.st[0], jy = L.st[1];
    const int tz = threadIdx.x % kTZ, ty = threadIdx.x / kTZ;
    const int z = blockIdx.x * kTZ + tz + 1;
    const int x0 = blockIdx.z * xc + 1;
    if (x0 > nx) return;
    const int x1 = min(x0 + xc - 1, nx);
    const int zm = lat_mapc(L, 2, z - 1), zp = lat_mapc(L, 2, z + 1);
    const bool hz0 = (tz == 0), hz1 = (tz == kTZ - 1) || (z == nz);
    int yr[2], ymr[2], ypr[2], colr[2];
    bool act[2], hy0[2], hy1[2];
#pragma unroll
    for (int r = 0; r < 2; r++) {
        yr[r] = blockIdx.y * kTY2 + ty + kTY * r + 1;
        act[r] = (z <= nz) && (yr[r] <= ny);
        ymr[r] = lat_mapc(L, 1, yr[r] - 1);
        ypr[r] = lat_mapc(L, 1, yr[r] + 1);
        colr[r] = yr[r] * jy + z;
        hy0[r] = (r == 0) && (ty == 0);
        hy1[r] = (r == 1 && ty == kTY - 1) || (yr[r] == ny);
    }
    double vprev[2], vcur[2], vnext[2], g[2], hzl[2], hzh[2], hyl[2], hyh[2];
#pragma unroll
    for (int r = 0; r < 2; r++) {
        vprev[r] = vcur[r] = vnext[r] = g[r] = hzl[r] = hzh[r] = hyl[r] = hyh[r] = 0;
        if (act[r]) {
            const int base = x0 * jx;
            vprev[r] = gin[lat_mapc(L, 0, x0 - 1) * jx + colr[r]];
            vcur[r] = gin[base + colr[r]];
            vnext[r] = gin[lat_mapc(L, 0, x0 + 1) * jx + colr[r]];
            g[r] = G[base + colr[r]];
            if (hz0) hzl[r] = gin[base + yr[r] * jy + zm];
            if (hz1) hzh[r] = gin[base + yr[r] * jy + zp];
            if (hy0[r]) hyl[r] = gin[base + ymr[r] * jy + z];
            if (hy1[r]) hyh[r] = gin[base + ypr[r] * jy + z];
        }
    }
    int b = 0;
    for (int x = x0; x <= x1; x++) {
        double vn2[2], gn[2], nzl[2], nzh[2], nyl[2], nyh[2];
        const bool more = x < x1;
#pragma unroll
        for (int r = 0; r < 2; r++) {
            vn2[r] = gn[r] = nzl[r] = nzh[r] = nyl[r] = nyh[r] = 0;
            if (act[r] && more) {
                const int nb = (x + 1) * jx;
                vn2[r] = gin[lat_mapc(L, 0, x + 2) * jx + colr[r]];
                gn[r] = G[nb + colr[r]];
                if (hz0) nzl[r] = gin[nb + yr[r] * jy + zm];
                if (hz1) nzh[r] = gin[nb + yr[r] * jy + zp];
                if (hy0[r]) nyl[r] = gin[nb + ymr[r] * jy + z];
                if (hy1[r]) nyh[r] = gin[nb + ypr[r] * jy + z];
            }
        }
#pragma unroll
        for (int r = 0; r < 2; r++) {
            if (!act[r]) continue;
            const int tr = ty + kTY * r + 1;
            tile[b][tr][tz + 1] = vcur[r];
            if (hz0) tile[b][tr][0] = hzl[r];
            if (hz1) tile[b][tr][tz + 2] = hzh[r];
            if (hy0[r]) tile[b][0][tz + 1] = hyl[r];
            if (hy1[r]) tile[b][tr + 1][tz + 1] = hyh[r];
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < 2; r++) {
            if (!act[r]) continue;
            const int tr = ty + kTY * r + 1;
            double acc = vprev[r] * g[r];
            acc += vnext[r] * g[r];
            acc += tile[b][tr - 1][tz + 1] * g[r];
            acc += tile[b][tr + 1][tz + 1] * g[r];
            acc += tile[b][tr][tz] * g[r];
            acc += tile[b][tr][tz + 2] * g[r];
            gout[x * jx + colr[r]] = acc * (1.0 / 6.0);
        }
#pragma unroll
        for (int r = 0; r < 2; r++) {
            vprev[r] = vcur[r]; vcur[r] = vnext[r]; vnext[r] = vn2[r];
            g[r] = gn[r]; hzl[r] = nzl[r]; hzh[r] = nzh[r]; hyl[r] = nyl[r]; hyh[r] = nyh[r];
        }
        b ^= 1;
    }
}

// One second-order step (Lat3D2ndO::PropagateF, Lat3D2ndO.cpp:65-152, and
// PropagateB, :597-678) for the six direction components, with boundary
// components swapped at mirrors (SetBx1(gz0,gz5)..., Lat3D2ndO.cpp:84-89) and
// fused composition phi += sum_k gout_k * other_k (ConnectG, :895-902).
__device__ __forceinline__ double comp2(const DLat &L, const double *__restrict__ gin, double gS,
                                        double gL, int t, int k, bool backward) {
    const int M = L.M;
    const int jx = L.st[0], jy = L.st[1];
    const int e[6] = {jx, jy, 1, -1, -jy, -jx};
    const int opp = 5 - k;
    double acc = 0;
    bool first = true;
    if (!backward) {
        int src = t - e[k];
#pragma unroll
        for (int kp = 0; kp < 6; kp++) {
            if (kp == opp) continue;
            double v = gin[(size_t)kp * M + src] * (kp == k ? gS : gL);
            if (first) { acc = v; first = false; } else acc += v;
        }
    } else {
#pragma unroll
        for (int kp = 5; kp >= 0; kp--) {
            if (kp == opp) continue;
            double v = gin[(size_t)kp * M + t + e[kp]] * (kp == k ? gS : gL);
            if (first) { acc = v; first = false; } else acc += v;
        }
    }
    return acc;
}

static __global__ void step2(DLat L, const double *__restrict__ gin, const double *__restrict__ G, double S,
                      double *__restrict__ gout, const double *__restrict__ other,
                      double *__restrict__ phi, int mode, int backward) {
    const int M = L.M;
    const double Lw = (1.0 - S) / 4.0;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < M; r += gridDim.x * blockDim.x) {
        int sw = 0;
        int t = lat_map(L, r, &sw);
        double gS = G[t] * S, gL = G[t] * Lw;
        double out[6];
#pragma unroll
        for (int k = 0; k < 6; k++) {
            out[k] = comp2(L, gin, gS, gL, t, swap_dir(k, sw), backward != 0);
            gout[(size_t)k * M + r] = out[k];
        }
        if (mode == COMP_ACC) {
            double p = phi[r];
#pragma unroll
            for (int k = 0; k < 6; k++) p += out[k] * other[(size_t)k * M + r];
            phi[r] = p;
        }
    }
}

// Second-order steps over interior sites only (row-wise).  A neighbour on a
// boundary plane is read at its mapped site, with the x/y/z direction pair
// swapped when that boundary is a mirror (the SetBx1(gz0,gz5) ... copies of
// Lat3D2ndO.cpp:84-89).  Forward: component k at t collects the five allowed
// components at t - e_k (Lat3D2ndO.cpp:109-143); backward: component k' at t
// collects component k at t + e_k (:634-668).  Same weights and summation
// order as comp2.
__device__ __forceinline__ bool is_mirror(int bc) {
    return bc == SFGPU_BOUND_MIRROR1 || bc == SFGPU_BOUND_MIRROR2;
}
// wmode: STEP2_PLAIN weights S and (1-S)/4 (PropagateF/B(..., S),
// Lat3D2ndO.cpp:65-152, :597-678); STEP2_STIFF the stiff_range steps
// (:155-247, :680-764): per site S inside the range and 0.2 outside, the
// weight taken at the unshifted index of the reference's array operation --
// the source site for the +x/+y/+z components forward and for reads from the
// lower neighbour backward, the target site otherwise -- and multiplied
// after G; STEP2_ISO the isotropic steps with G/6 for all six components
// (:250-344, :765-850), whose forward -y component reads +z twice and -y
// never (Lat3D2ndO.cpp:308-313).
enum { STEP2_PLAIN = 0, STEP2_STIFF = 1, STEP2_ISO = 2 };
static __global__ void __launch_bounds__(kBlock, 4)
step2_rows(DLat L, const double *__restrict__ gin, const double *__restrict__ G, double S,
           double *__restrict__ gout, const double *__restrict__ other,
           double *__restrict__ phi, int mode, int backward, int wmode = STEP2_PLAIN) {
    pdl_enter();
    const int M = L.M;
    const double Lw = (1.0 - S) / 4.0;
    const int nx = L.Md[0] - 2, ny = L.Md[1] - 2;
    const int worker = blockIdx.x * blockDim.x + threadIdx.x;
    for_interior(L, worker, gridDim.x * blockDim.x, [&](const RowInfo &R, int k, int nlast) {
        const int t = R.base + k;
        // neighbour offsets and mirror swaps by direction: [0]=-x [1]=+x [2]=-y [3]=+y [4]=-z [5]=+z
        const int zm = (k == 1) ? L.map_lo[2] : k - 1;
        const int zp = (k == nlast) ? L.map_hi[2] : k + 1;
        const int off[6] = {R.up, R.dn, R.up2, R.dn2, zm - k, zp - k};
        const bool sw[6] = {R.x == 1 && is_mirror(L.bc_lo[0]), R.x == nx && is_mirror(L.bc_hi[0]),
                            R.y == 1 && is_mirror(L.bc_lo[1]), R.y == ny && is_mirror(L.bc_hi[1]),
                            k == 1 && is_mirror(L.bc_lo[2]), k == nlast && is_mirror(L.bc_hi[2])};
        const double g = G[t];
        const double gS = g * S, gL = g * Lw;
        double out[6];
        if (wmode != STEP2_PLAIN) {
            const int raw[6] = {L.st[0], L.st[1], 1, 1, L.st[1], L.st[0]};   // axis stride by component
            const double gI = g * (1.0 / 6.0);
            auto ps_at = [&](int i) { return (L.stiff[i] != 0) ? S : 0.2; };
            if (!backward) {
                const int dir_of[6] = {0, 2, 4, 5, 3, 1};
#pragma unroll
                for (int kk = 0; kk < 6; kk++) {
                    const int dd = dir_of[kk];
                    const int src = t + off[dd];
                    const int axis = dd >> 1;
                    const bool sflag = sw[dd];
                    auto comp = [&](int kp) {
                        int c = kp;
                        if (sflag) {
                            if (axis == 0 && (kp == 0 || kp == 5)) c = 5 - kp;
                            if (axis == 1 && (kp == 1 || kp == 4)) c = 5 - kp;
                            if (axis == 2 && (kp == 2 || kp == 3)) c = 5 - kp;
                        }
                        return gin[(size_t)c * M + src];
                    };
                    double acc;
                    if (wmode == STEP2_ISO) {
                        const int seq4[6] = {0, 2, 2, 3, 4, 5};
                        acc = comp(kk == 4 ? seq4[0] : 0) * gI;
                        for (int q = 1; q < 6; q++) acc += comp(kk == 4 ? seq4[q] : q) * gI;
                    } else {
                        const int pi = (kk < 3) ? t - raw[kk] : t;
                        const double ps = ps_at(pi), pl = (1.0 - ps) / 4.0;
                        bool first = true;
                        acc = 0;
                        for (int kp = 0; kp < 6; kp++) {
                            if (kp == 5 - kk) continue;
                            const double v = comp(kp) * g * (kp == kk ? ps : pl);
                            if (first) { acc = v; first = false; } else acc += v;
                        }
                    }
                    out[kk] = acc;
                }
            } else {
                const int dir_of[6] = {1, 3, 5, 4, 2, 0};
                double v[6];
#pragma unroll
                for (int kk = 0; kk < 6; kk++) {
                    const int dd = dir_of[kk];
                    const int c = sw[dd] ? 5 - kk : kk;
                    v[kk] = gin[(size_t)c * M + t + off[dd]];
                }
#pragma unroll
                for (int kq = 0; kq < 6; kq++) {
                    double acc = 0;
                    bool first = true;
                    for (int kp = 5; kp >= 0; kp--) {
                        double w;
                        if (wmode == STEP2_ISO) {
                            w = v[kp] * gI;
                        } else {
                            if (kp == 5 - kq) continue;
                            const int pi = (kp >= 3) ? t - raw[kp] : t;
                            const double ps = ps_at(pi), pl = (1.0 - ps) / 4.0;
                            w = v[kp] * g * (kp == kq ? ps : pl);
                        }
                        if (first) { acc = w; first = false; } else acc += w;
                    }
                    out[kq] = acc;
                }
            }
        } else if (!backward) {
            // source of component kk is t - e_kk: kk=0 -> -x, 5 -> +x, 1 -> -y, 4 -> +y, 2 -> -z, 3 -> +z
            const int dir_of[6] = {0, 2, 4, 5, 3, 1};
#pragma unroll
            for (int kk = 0; kk < 6; kk++) {
                const int dd = dir_of[kk];
                const int src = t + off[dd];
                const int axis = dd >> 1;
                const bool s = sw[dd];
                double acc = 0;
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
                    double v = gin[(size_t)c * M + src] * (kp == kk ? gS : gL);
                    if (first) { acc = v; first = false; } else acc += v;
                }
                out[kk] = acc;
            }
        } else {
            // component k is read at t + e_k: 0 -> +x, 5 -> -x, 1 -> +y, 4 -> -y, 2 -> +z, 3 -> -z
            const int dir_of[6] = {1, 3, 5, 4, 2, 0};
            double v[6];
#pragma unroll
            for (int kk = 0; kk < 6; kk++) {
                const int dd = dir_of[kk];
                const int c = sw[dd] ? 5 - kk : kk;
                v[kk] = gin[(size_t)c * M + t + off[dd]];
            }
#pragma unroll
            for (int kq = 0; kq < 6; kq++) {
                double acc = 0;
                bool first = true;
#pragma unroll
                for (int kp = 5; kp >= 0; kp--) {
                    if (kp == 5 - kq) continue;
                    double w = v[kp] * (kp == kq ? gS : gL);
                    if (first) { acc = w; first = false; } else acc += w;
                }
                out[kq] = acc;
            }
        }
#pragma unroll
        for (int kk = 0; kk < 6; kk++) gout[(size_t)kk * M + t] = out[kk];
        if (mode == COMP_ACC) {
            double p = phi[t];
#pragma unroll
            for (int kk = 0; kk < 6; kk++) p += out[kk] * other[(size_t)kk * M + t];
            phi[t] = p;
        }
    });
}

// Second-order steps of the flat 1D and 2D lattices, whose homogeneous
// gradients lump their bond directions into one component each (Lat1D2ndO:
// +x, lateral x4, -x, Lat1D2ndO.cpp:33-147; Lat2D2ndO: +x, +y, z x2, -y, -x,
// Lat2D2ndO.cpp:32-230).  W[kk][kp] = the weight of a bond in direction kk
// after one in kp summed over kp's group: S for the same direction (plus
// 2L for the 1D lateral group's two perpendicular members), 0 for the
// opposite direction, mult[kp] L otherwise.  The forward step reads every
// component at t - e_kk, the backward step reads component kp at t + e_kp;
// a read across a boundary goes to the mapped site and, where the lattice
// swaps there (sw_lo / sw_hi), takes the opposite component of that axis
// (at a surface, the site itself, only the + component does).
struct Lump2 {
    int K;
    int axis[5], sgn[5];
    double mult[5];
};
__host__ __device__ inline Lump2 lump2_of(int grad) {
    Lump2 q;
    if (grad == 1) {
        q.K = 3;
        const int ax[3] = {0, -1, 0}, sg[3] = {1, 0, -1};
        const double mu[3] = {1, 4, 1};
        for (int k = 0; k < 3; k++) { q.axis[k] = ax[k]; q.sgn[k] = sg[k]; q.mult[k] = mu[k]; }
        q.axis[3] = q.axis[4] = -1; q.sgn[3] = q.sgn[4] = 0; q.mult[3] = q.mult[4] = 0;
    } else {
        q.K = 5;
        const int ax[5] = {0, 1, -1, 1, 0}, sg[5] = {1, 1, 0, -1, -1};
        const double mu[5] = {1, 1, 2, 1, 1};
        for (int k = 0; k < 5; k++) { q.axis[k] = ax[k]; q.sgn[k] = sg[k]; q.mult[k] = mu[k]; }
    }
    return q;
}
__host__ __device__ inline double lump2_w(const Lump2 &q, int kk, int kp, double S, double Lw) {
    if (kk == kp) return (q.K == 3 && kk == 1) ? S + 2 * Lw : S;
    if (q.axis[kk] >= 0 && q.axis[kk] == q.axis[kp] && q.sgn[kk] == -q.sgn[kp]) return 0.0;
    return q.mult[kp] * Lw;
}
// the component of the opposite direction along kp's axis (kp itself for a lumped one)
__host__ __device__ inline int lump2_swap(const Lump2 &q, int kp) {
    if (q.axis[kp] < 0) return kp;
    for (int k = 0; k < q.K; k++)
        if (q.axis[k] == q.axis[kp] && q.sgn[k] == -q.sgn[kp]) return k;
    return kp;
}

// site and swap mode (0 none, 1 swap, 2 surface) of a read one step from
// interior site (x, y) along axis a in direction d (+1 / -1); 1D: x is the
// position, y = 0
__device__ __forceinline__ int lump2_nb(const DLat &L, int x, int y, int a, int d, int &sm) {
    int c[2] = {x, y};
    int v = c[a] + d;
    sm = 0;
    if (v == 0) { sm = L.sw_lo[a]; v = L.map_lo[a]; }
    else if (v == L.Md[a] - 1) { sm = L.sw_hi[a]; v = L.map_hi[a]; }
    c[a] = v;
    return (L.grad == 1) ? c[0] : c[0] * L.st[0] + c[1];
}
// the component read for kp across a boundary of axis a with swap mode sm:
// components of other axes are plain copies; a swap reads the opposite
// direction; at a surface only the + direction reads the - one
__host__ __device__ inline int lump2_read(const Lump2 &q, int kp, int a, int sm) {
    if (sm == 0 || q.axis[kp] != a) return kp;
    if (sm == 1 || q.sgn[kp] > 0) return lump2_swap(q, kp);
    return kp;
}

// Curved lumped lattices (Lat1DCyl2ndO.cpp:52-95, :149-186; Lat1DSphere2ndO
// alike; Lat2DCyl2ndO.cpp:45-115, :180-249): a radial read of component kp
// one layer away becomes f * g_kp(neighbour) + (1 - f) * g_refl(kp)(t)
// (LReflect / UReflect), refl swapping +x and -x, with f = 6 lambda_-(x) for
// a read from the inner layer and 6 lambda_+(x) from the outer one.  Forward
// steps mix every radial read.  The 2D cylinder's backward step mixes only
// the reads of -x (SFbox computes the +x mixture there and does not use it,
// Lat2DCyl2ndO.cpp:203-207); the 1D backward step mixes both.
__device__ __forceinline__ double lump2_mix(const DLat &L, const double *__restrict__ gin, int M, double v, int refl,
                                            int t, int x, int dir) {
    const double f = 6 * ((dir > 0) ? L.lam_p[x] : L.lam_m[x]);
    const double fc = 1.0 - f;
    return f * v + fc * gin[(size_t)refl * M + t];
}

static __global__ void step2l_rows(DLat L, const double *__restrict__ gin, const double *__restrict__ G, double S,
                                   double *__restrict__ gout, const double *__restrict__ other,
                                   double *__restrict__ phi, int mode, int backward) {
    const int M = L.M;
    const Lump2 q = lump2_of(L.grad);
    const double Lw = (1.0 - S) / 4.0;
    const int worker = blockIdx.x * blockDim.x + threadIdx.x;
    for_interior(L, worker, gridDim.x * blockDim.x, [&](const RowInfo &R, int k, int nlast) {
        const int t = R.base + k;
        const int x = (L.grad == 1) ? k : R.x, y = (L.grad == 1) ? 0 : k;
        const double g = G[t];
        double out[5];
        if (!backward) {
            for (int kk = 0; kk < q.K; kk++) {
                int src = t;
                int sm = 0;
                if (q.axis[kk] >= 0) src = lump2_nb(L, x, y, q.axis[kk], -q.sgn[kk], sm);
                const bool mix = L.cyl && q.axis[kk] == 0;
                double acc = 0;
                bool first = true;
                for (int kp = 0; kp < q.K; kp++) {
                    const double w = lump2_w(q, kk, kp, S, Lw);
                    if (w == 0.0) continue;
                    const int c = lump2_read(q, kp, q.axis[kk], sm);
                    double r = gin[(size_t)c * M + src];
                    if (mix) r = lump2_mix(L, gin, M, r, lump2_read(q, kp, 0, 1), t, x, -q.sgn[kk]);
                    const double v = w * r;
                    if (first) { acc = v; first = false; } else acc += v;
                }
                out[kk] = acc * g;
            }
        } else {
            double v[5];
            for (int kp = 0; kp < q.K; kp++) {
                int src = t;
                int sm = 0;
                if (q.axis[kp] >= 0) src = lump2_nb(L, x, y, q.axis[kp], q.sgn[kp], sm);
                const int c = lump2_read(q, kp, q.axis[kp], sm);
                v[kp] = gin[(size_t)c * M + src];
                if (L.cyl && q.axis[kp] == 0 && (L.grad == 1 || q.sgn[kp] < 0))
                    v[kp] = lump2_mix(L, gin, M, v[kp], lump2_swap(q, kp), t, x, q.sgn[kp]);
            }
            for (int kq = 0; kq < q.K; kq++) {
                double acc = 0;
                bool first = true;
                for (int kp = 0; kp < q.K; kp++) {
                    const double w = lump2_w(q, kq, kp, S, Lw);
                    if (w == 0.0) continue;
                    const double u = w * v[kp];
                    if (first) { acc = u; first = false; } else acc += u;
                }
                out[kq] = acc * g;
            }
        }
        for (int kk = 0; kk < q.K; kk++) gout[(size_t)kk * M + t] = out[kk];
        if (mode == COMP_ACC) {
            double p = phi[t];
            for (int kk = 0; kk < q.K; kk++) {
                const double a = out[kk] * other[(size_t)kk * M + t];
                p += (q.mult[kk] == 1.0) ? a : a * q.mult[kk];
            }
            phi[t] = p;
        }
    });
}

// multiplicity of direction component k of a K-component slice
__host__ __device__ inline double comp_mult(int K, int k) {
    if (K == 3 && k == 1) return 4.0;
    if (K == 5 && k == 2) return 2.0;
    return 1.0;
}

// phi += a * b over all K*M entries summed per site (copolymer end segment,
// SF_Copol1stO.cpp:1218-1222; Lat3D2ndO::ConnectG over six components)
static __global__ void connect(int M, int K, const double *__restrict__ a, const double *__restrict__ b,
                        double *__restrict__ phi) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < M; r += gridDim.x * blockDim.x) {
        double p = phi[r];
        for (int k = 0; k < K; k++) {
            const double v = a[(size_t)k * M + r] * b[(size_t)k * M + r];
            const double mu = comp_mult(K, k);
            p += (mu == 1.0) ? v : v * mu;
        }
        phi[r] = p;
    }
}

// Bond-orientation composition, the OUT/PHI argument of the second-order
// ConnectG (Lat3D2ndO.cpp:905-918, Lat2D2ndO.cpp:285-304,
// Lat1D2ndO.cpp:215-227): the product of component k of the two propagators
// is added to the slot of k's bond axis.  3D: +-x -> 0, +-y -> 1, +-z -> 2.
// 1D: +-x -> 0, the lateral group (times 4) -> 1.  2D follows SFbox's slot
// selection as written: k = 3 (-y) keeps the slot of k = 2 and k = 4 (-x)
// goes to slot 1, and the z group's product is added to slot 2 a second
// time after the loop.  Interior sites only; boundary entries stay 0.
__host__ __device__ inline int orient_slot(int K, int k) {
    if (K == 6) { const int s6[6] = {0, 1, 2, 2, 1, 0}; return s6[k]; }
    if (K == 5) { const int s5[5] = {0, 1, 2, 2, 1}; return s5[k]; }
    return (k == 1) ? 1 : 0;
}
static __global__ void orient_acc(DLat L, const double *__restrict__ a, const double *__restrict__ b,
                                  double *__restrict__ out) {
    const int M = L.M, K = L.K;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < M; r += gridDim.x * blockDim.x) {
        int c[3];
        lat_coords(L, r, c);
        if (!lat_interior(L, c)) continue;
        for (int k = 0; k < K; k++) {
            double v = a[(size_t)k * M + r] * b[(size_t)k * M + r];
            if (K == 3 && k == 1) v = v * 4.0;
            out[(size_t)orient_slot(K, k) * M + r] += v;
        }
        if (K == 5) out[2 * (size_t)M + r] += a[2 * (size_t)M + r] * b[2 * (size_t)M + r];
    }
}

// copy a full lattice vector into K components (Gi[.][1] = G, Gi_inv = G)
static __global__ void replicate(int M, int K, const double *__restrict__ g, double *__restrict__ out) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < M; r += gridDim.x * blockDim.x)
        for (int k = 0; k < K; k++) out[(size_t)k * M + r] = g[r];
}

// Block partial sums of sum_k sum_z w(z) g_k(z) (the lnGN sums) in a fixed
// order; the last pass is done by mol_scalars.
static __global__ void wsum_partial(int M, int K, const double *__restrict__ g, const double *__restrict__ w,
                             double *__restrict__ partial) {
    __shared__ double sh[kBlock];
    double acc = 0;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < M; r += gridDim.x * blockDim.x) {
        double wr = w[r];
        if (wr != 0)
            for (int k = 0; k < K; k++) {
                const double mu = comp_mult(K, k);
                acc += (mu == 1.0) ? wr * g[(size_t)k * M + r] : wr * (g[(size_t)k * M + r] * mu);
            }
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

// Molecule scalars after a propagation: lnGN, bulk volume fraction and the
// normalisation of phi (SF_Homopol1stO.cpp:597-619, SF_Copol1stO.cpp:1234-1280,
// SF_Monomer1stO.cpp:106-126, SF_Homopol2ndO.cpp:186-204).  The solvent takes
// phibulk = 1 - sum of the others (SF_MolList1stO.cpp:278-291).
struct MolParam {
    int N, type, freedom, sym, K, pinned, solvent, nmol;
    double phibulk_in, theta;
    const double *phib_dev = nullptr;   // device bulk fraction (a neutralizer's), else phibulk_in
};
static __global__ void mol_scalars(MolParam p, int nblocks, const double *__restrict__ partial,
                            MolScal *__restrict__ scal, int self) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double v = 0;
    for (int b = 0; b < nblocks; b++) v += partial[b];
    if (p.K > 1) v /= 6.0;   // six bond directions (lumped or not)
    MolScal s;
    s.lngn = log(v);
    double phib = p.phib_dev ? *p.phib_dev : p.phibulk_in;
    if (p.solvent) {
        phib = 1.0;
        for (int m = 0; m < p.nmol; m++)
            if (m != self) phib -= scal[m].phibulk;
    }
    const double N = (double)p.N;
    double gn = exp(s.lngn);
    if (p.freedom == SFGPU_MOL_RESTRICTED) {
        if (p.type == 0) {
            s.lnc = log(p.theta) - s.lngn;
            s.norm = p.theta / gn;
        } else {
            s.lnc = log(p.theta) - s.lngn - log(1.0 * p.N);
            double c = (p.sym ? 2 * p.theta / N : p.theta / N);
            s.norm = (p.K > 1) ? c / (6.0 * gn) : c / gn;
        }
        s.phibulk = p.theta / gn;
    } else {
        s.phibulk = phib;
        if (p.type == 0) {
            s.lnc = log(phib);
            s.norm = phib;
        } else {
            s.lnc = log(phib / N);
            s.norm = p.sym ? 2 * phib / N : (p.K > 1 ? phib / (6 * N) : phib / N);
        }
    }
    if (p.pinned) s.phibulk = 0;   // SF_Homopol1stO.cpp:124-125
    scal[self] = s;
}

// CorrectDoubleCountG + NormPhi (Lat1DFlat1stO.cpp:294-300, :317-322);
// monomers start from phi = G (SF_Monomer1stO.cpp:103-106)
static __global__ void finalize_phi(int M, const double *__restrict__ G, double *__restrict__ phi,
                             const MolScal *__restrict__ scal, int mol, int monomer) {
    const double norm = scal[mol].norm;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < M; r += gridDim.x * blockDim.x) {
        double p;
        if (monomer) p = G[r];
        else { double g = G[r]; p = (g > 0) ? phi[r] / g : 0.0; }
        phi[r] = p * norm;
    }
}

// Constant-force steps (mol : force) of the first-order lattices, with the
// weights the host computes as the reference does:
//  1D flat   (Lat1DFlat1stO.cpp:116-130): g (b + a1 (a - b) + a2 (c - b)),
//            a1 = l1 e^f / n, a2 = l1 e^-f / n, n = l1 (e^-f + e^f - 2) + 1
//  1D curved (Lat1DCyl1stO.cpp:112-133): g (l-(z) a2 a + (1 - l+ - l-)/a3 b
//            + l+(z) a1 c), a1 = e^-f / a3, a2 = e^f / a3, a3 = (4 + e^-f + e^f)/6
//  2D cyl    (Lat2DCyl1stO.cpp:100-126): g (b + l-(x)(u - b) + l+(x)(d - b)
//            + l1 (a a1 + c a2 - b - b)) / a3, a1 = e^f, a2 = e^-f,
//            a3 = l1 (e^-f + e^f - 2) + 1, along y
//  3D        (Lat3D1stO.cpp:94-130): (x-, x+, y-, y+ times g, z- g a1, z+ g a2) a3,
//            a1 = e^f, a2 = e^-f, a3 = 1 / (4 + e^f + e^-f)
struct ForceW { double a1, a2, a3; };
// the step with the weight g of the target site given (force_row: g = G[t];
// the derivative kernels take g = 1 for the bare stencil)
__device__ __forceinline__ double force_row_g(const DLat &L, const RowInfo &R, const double *__restrict__ gin,
                                              double g, int k, int nlast, const ForceW &w) {
    const int d = L.grad - 1;
    const int t = R.base + k;
    const int km = (k == 1) ? L.map_lo[d] : k - 1;
    const int kp = (k == nlast) ? L.map_hi[d] : k + 1;
    const double a = gin[R.base + km], b = gin[t], c = gin[R.base + kp];
    if (L.grad == 1 && !L.cyl) return g * (b + w.a1 * (a - b) + w.a2 * (c - b));
    if (L.grad == 1) {
        const double f1z = L.lam_p[t] * w.a1, f_1z = L.lam_m[t] * w.a2;
        const double f0z = (1 - L.lam_p[t] - L.lam_m[t]) / w.a3;
        return g * (f_1z * a + f0z * b + f1z * c);
    }
    if (L.grad == 2)
        return g * (b + L.lam_m[R.x] * (gin[t + R.up] - b) + L.lam_p[R.x] * (gin[t + R.dn] - b) +
                    L.l1 * (a * w.a1 + c * w.a2 - b - b)) / w.a3;
    double acc = gin[t + R.up] * g;
    acc += gin[t + R.dn] * g;
    acc += gin[t + R.up2] * g;
    acc += gin[t + R.dn2] * g;
    acc += a * g * w.a1;
    acc += c * g * w.a2;
    return acc * w.a3;
}
__device__ __forceinline__ double force_row(const DLat &L, const RowInfo &R, const double *__restrict__ gin,
                                            const double *__restrict__ G, int k, int nlast, const ForceW &w) {
    return force_row_g(L, R, gin, G[R.base + k], k, nlast, w);
}

static __global__ void step1_force_rows(DLat L, ForceW w, const double *__restrict__ gin, const double *__restrict__ G,
                                        double *__restrict__ gout, const double *__restrict__ other,
                                        double *__restrict__ phi, int mode) {
    const int worker = blockIdx.x * blockDim.x + threadIdx.x;
    for_interior(L, worker, gridDim.x * blockDim.x, [&](const RowInfo &R, int k, int nlast) {
        const int t = R.base + k;
        const double out = force_row(L, R, gin, G, k, nlast, w);
        gout[t] = out;
        if (mode == COMP_ACC) phi[t] += out * other[t];
    });
}

// SF_HomoRing1stO::Matrix1 (SF_HomoRing1stO.cpp:110-160), the ring's
// profile as a return weight: for every lattice site k (1-based) a walk
// starts at k with weight G(k) and takes N/2 - 1 steps over the sites
// 1 .. Mmax (beyond the lattice G = 1; site 0 stays 0), step s updating the
// window [max(k - s, 1), min(k + s, Mmax)) from the previous values as
// (a + 4 b + c) G / 6 after the top site has copied its lower neighbour;
// phi(k) = phibulk sum_z Y(z)^2 / norm0.  One block per site, the walk in
// two shared-memory buffers of Mmax + 1 values.
static __global__ void ring_phi(int M, int N, int Mmax, const double *__restrict__ G, double phibulk,
                                double norm0, double *__restrict__ phi) {
    extern __shared__ double ring_sh[];
    __shared__ double red[32];
    double *Y = ring_sh, *Yn = ring_sh + (Mmax + 1);
    for (int k = blockIdx.x + 1; k <= M; k += gridDim.x) {
        for (int z = threadIdx.x; z <= Mmax; z += blockDim.x) Y[z] = (z == k) ? G[k - 1] : 0.0;
        __syncthreads();
        for (int st = 1; st < N / 2; st++) {
            const int zmin = max(k - st, 1), zmax = min(k + st, Mmax);
            const double ytop = Y[Mmax - 1];
            for (int z = threadIdx.x; z <= Mmax; z += blockDim.x) {
                double v = (z == Mmax) ? ytop : Y[z];
                if (z >= zmin && z < zmax) {
                    const double a = Y[z - 1], b = Y[z];
                    const double c = (z + 1 == Mmax) ? ytop : Y[z + 1];
                    const double gz = (z <= M) ? G[z - 1] / 6.0 : 1.0 / 6.0;
                    v = gz * (a + 4 * b + c);
                }
                Yn[z] = v;
            }
            __syncthreads();
            double *t = Y; Y = Yn; Yn = t;
        }
        double acc = 0;
        for (int z = threadIdx.x + 1; z <= Mmax; z += blockDim.x) acc += Y[z] * Y[z];
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
        __syncthreads();
        if (threadIdx.x == 0) {
            double v = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += red[w];
            phi[k - 1] = v / norm0 * phibulk;
        }
        __syncthreads();
    }
}

// a ring's molecule scalars: SF_HomoRing1stO::Matrix1 leaves lnGN and
// ln Cb at their initial 0 (SF_Molecule.cpp:269), which the free energy
// reads; the bulk fraction is the input's
static __global__ void ring_scalars(int N, double phibulk, MolScal *__restrict__ scal, int self) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    MolScal v;
    v.lngn = 0;
    v.phibulk = phibulk;
    v.lnc = 0;
    v.norm = phibulk / N;
    scal[self] = v;
}

// Dendrimer branch points (SF_Dend1stO.cpp:199-214, :245-253): out = a b / G
// where G > 0, else 0 -- ConnectG into a zero vector, then CorrectDoubleCountG
static __global__ void dend_combine(int M, const double *__restrict__ a, const double *__restrict__ b,
                                    const double *__restrict__ G, double *__restrict__ out) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < M; r += gridDim.x * blockDim.x) {
        const double g = G[r];
        out[r] = (g > 0) ? (a[r] * b[r]) / g : 0.0;
    }
}

// NormPhiFree(Gi_inv, nr); ConnectG(Gi_inv, Gi, s, phi); NormPhiFree(Gi_inv,
// 1/nr) of SF_Dend1stO.cpp:254-262 in one pass, with the same roundings
static __global__ void dend_connect(int M, double *__restrict__ ginv, const double *__restrict__ gf,
                                    double *__restrict__ phi, double nr, double inv_nr) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < M; r += gridDim.x * blockDim.x) {
        const double t = ginv[r] * nr;
        phi[r] += t * gf[r];
        ginv[r] = t * inv_nr;
    }
}

// state phi = sum of the molecule contributions (SF_State::GetPhi, SF_State.cpp:302-320)
struct PtrList { const double *p[SFGPU_MAX_SEG]; int n; };
static __global__ void sum_profiles(int M, PtrList src, double *__restrict__ out) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < M; r += gridDim.x * blockDim.x) {
        double acc = 0;
        for (int i = 0; i < src.n; i++) acc += src.p[i][r];
        out[r] = acc;
    }
}

// bulk values per state and the bulk contact terms per class
// (SF_Segment::UpdatePhiBulk, SF_Segment.cpp:443-456; ChemIntBulk, SF_SegmentList.cpp:610-623)
struct BulkParam {
    int nseg, nmol, nclass;
    int rep[SFGPU_MAX_SEG];
    double frac[SFGPU_MAX_SEG * SFGPU_MAX_SEG];   // [seg][mol] = count/N
};
static __global__ void bulk_scalars(BulkParam b, ChiTable ct, const MolScal *__restrict__ scal,
                             double *__restrict__ phib, double *__restrict__ chib) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int i = 0; i < b.nseg; i++) {
        double v = 0;
        for (int m = 0; m < b.nmol; m++) v += scal[m].phibulk * b.frac[i * SFGPU_MAX_SEG + m];
        phib[i] = v;
    }
    for (int c = 0; c < b.nclass; c++) {
        int st = b.rep[c];
        double v = 0;
        for (int j = 0; j < b.nseg; j++) {
            double x = ct.chi[st * SFGPU_MAX_SEG + j];
            if (x != 0) v += x * phib[j];
        }
        chib[c] = v;
    }
}

// residual of SF_Solve::GetResiduals (SF_Solve.cpp:527-591) on every site
// carrying iteration variables
struct ResParam {
    int nsites, nclass, nseg;
    int rep[SFGPU_MAX_SEG];
    const double *phi[SFGPU_MAX_SEG];     // state phi, by segment
    const double *gfull[SFGPU_MAX_SEG];   // G of the representative state, by class
};
static __global__ void residual(DLat L, ResParam rp, ChiTable ct, const int *__restrict__ sites,
                         const double *__restrict__ chib, double *__restrict__ f) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < rp.nsites; j += gridDim.x * blockDim.x) {
        int z = sites[j];
        double phit = 0;
        double rho[SFGPU_MAX_SEG];
        for (int i = 0; i < rp.nseg; i++) {
            phit += rp.phi[i][z];
            rho[i] = 0;
        }
        for (int i = 0; i < rp.nseg; i++) {
            bool need = false;
            for (int c = 0; c < rp.nclass; c++) need |= ct.chi[rp.rep[c] * SFGPU_MAX_SEG + i] != 0;
            if (need) rho[i] = side_fraction(L, rp.phi[i], z);
        }
        double u[SFGPU_MAX_SEG];
        double av = 0;
        for (int c = 0; c < rp.nclass; c++) {
            int st = rp.rep[c];
            double v = -log(rp.gfull[c][z]);
            double ci = 0;
            for (int i = 0; i < rp.nseg; i++) {
                double x = ct.chi[st * SFGPU_MAX_SEG + i];
                if (x != 0) ci += x * rho[i];
            }
            v -= ci / phit;
            v += chib[c];
            u[c] = v;
            av += v;
        }
        av /= rp.nclass;
        for (int c = 0; c < rp.nclass; c++) f[(size_t)j * rp.nclass + c] = -1.0 + 1.0 / phit + u[c] - av;
    }
}

// free-energy density (SF_MolList1stO.cpp:815-940) weighted by the lattice
// sites, block partial sums
struct FreeParam {
    int nseg, nmol;
    const double *phi[SFGPU_MAX_SEG];                        // state phi
    const double *mphi[SFGPU_MAX_SEG * SFGPU_MAX_SEG];       // [mol][seg] or null
    const double *gseg[SFGPU_MAX_SEG];                       // segment G
    double invN[SFGPU_MAX_SEG], lnN[SFGPU_MAX_SEG], chemintref[SFGPU_MAX_SEG];
};
static __global__ void free_energy_partial(DLat L, FreeParam fp, ChiTable ct, const double *__restrict__ wf,
                                    const MolScal *__restrict__ scal, double *__restrict__ partial,
                                    const double *__restrict__ el = nullptr) {
    __shared__ double sh[kBlock];
    double acc = 0;
    for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < L.M; z += gridDim.x * blockDim.x) {
        double w = wf[z];
        if (w == 0) continue;
        double entropy = 0, contact = 0;
        for (int m = 0; m < fp.nmol; m++) {
            double pm = 0;
            for (int i = 0; i < fp.nseg; i++) {
                const double *q = fp.mphi[m * SFGPU_MAX_SEG + i];
                if (q) pm += q[z];
            }
            entropy -= (pm * fp.invN[m]) * (fp.lnN[m] + scal[m].lnc);
            contact -= pm * fp.chemintref[m];
        }
        for (int m = 0; m < fp.nmol; m++)
            for (int i = 0; i < fp.nseg; i++) {
                const double *q = fp.mphi[m * SFGPU_MAX_SEG + i];
                if (!q) continue;
                double G = fp.gseg[i][z];
                if (G > 0) entropy -= q[z] * log(G);
            }
        for (int i = 0; i < fp.nseg; i++) {
            double ci = 0;
            for (int j = 0; j < fp.nseg; j++) {
                double x = ct.chi[i * SFGPU_MAX_SEG + j];
                if (x != 0) ci += x * side_fraction(L, fp.phi[j], z);
            }
            contact += 0.5 * fp.phi[i][z] * ci;
        }
        if (el) acc += w * (-entropy + contact + el[z]);   // charged: + electrostatic profile
        else acc += w * (-entropy + contact);
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

// Free-energy and grand-potential densities per site, each multiplied by the
// SubtractBoundaries factor, and their sums weighted with the lattice sites
// (two block partials per block: F, Omega).  Densities as free_energy_partial
// and SF_MolList1stO::GetGrandPotentialProfile (SF_MolList1stO.cpp:1001-1101;
// the same in SF_MolList2ndO): the molecules' (phi - phib)/N, u' phi of every
// liquid state (u' = -ln G - ChemInt + ChemIntBulk where G > 0), and the
// contact pairs of liquid states, in that order.  No charges, external
// potentials or grafted chains on this path.  fe / gp may be null.
struct ThermoParam {
    int nseg, nmol;
    const double *phi[SFGPU_MAX_SEG];
    const double *mphi[SFGPU_MAX_SEG * SFGPU_MAX_SEG];
    const double *gseg[SFGPU_MAX_SEG], *gfull[SFGPU_MAX_SEG];
    int frozen[SFGPU_MAX_SEG];
    double invN[SFGPU_MAX_SEG], N[SFGPU_MAX_SEG], lnN[SFGPU_MAX_SEG], chemintref[SFGPU_MAX_SEG];
    // charged systems (null el otherwise): the electrostatic profile, the
    // potential psi, valences, e / kT and the layers of frozen segments
    const double *el, *psi, *surf;
    double val[SFGPU_MAX_SEG], ech, kT;
};
static __global__ void thermo_partial(DLat L, ThermoParam tp, ChiTable ct, const double *__restrict__ wf,
                                      const double *__restrict__ sb, const MolScal *__restrict__ scal,
                                      const double *__restrict__ phib, double *__restrict__ fe,
                                      double *__restrict__ gp, double *__restrict__ partial) {
    __shared__ double shF[kBlock], shO[kBlock];
    double accF = 0, accO = 0;
    for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < L.M; z += gridDim.x * blockDim.x) {
        double entropy = 0, contact = 0, omega = 0;
        for (int m = 0; m < tp.nmol; m++) {
            double pm = 0;
            for (int i = 0; i < tp.nseg; i++) {
                const double *q = tp.mphi[m * SFGPU_MAX_SEG + i];
                if (q) pm += q[z];
            }
            entropy -= (pm * tp.invN[m]) * (tp.lnN[m] + scal[m].lnc);
            contact -= pm * tp.chemintref[m];
        }
        for (int m = 0; m < tp.nmol; m++)
            for (int i = 0; i < tp.nseg; i++) {
                const double *q = tp.mphi[m * SFGPU_MAX_SEG + i];
                if (!q) continue;
                double G = tp.gseg[i][z];
                if (G > 0) entropy -= q[z] * log(G);
            }
        double rho[SFGPU_MAX_SEG];
#pragma unroll
        for (int j = 0; j < SFGPU_MAX_SEG; j++) rho[j] = (j < tp.nseg) ? side_fraction(L, tp.phi[j], z) : 0.0;
        for (int i = 0; i < tp.nseg; i++) {
            double ci = 0;
#pragma unroll
            for (int j = 0; j < SFGPU_MAX_SEG; j++) {
                if (j >= tp.nseg) continue;
                double x = ct.chi[i * SFGPU_MAX_SEG + j];
                if (x != 0) ci += x * rho[j];
            }
            contact += 0.5 * tp.phi[i][z] * ci;
        }
        for (int m = 0; m < tp.nmol; m++) {
            double pm = 0;
            for (int i = 0; i < tp.nseg; i++) {
                const double *q = tp.mphi[m * SFGPU_MAX_SEG + i];
                if (q) pm += q[z];
            }
            if (pm > 0) omega -= (pm - scal[m].phibulk) / tp.N[m];
        }
        for (int i = 0; i < tp.nseg; i++) {
            if (tp.frozen[i]) continue;
            const double G = tp.gfull[i][z];
            double up = 0;
            if (G > 0) {
                double ci = 0, cb = 0;
#pragma unroll
                for (int j = 0; j < SFGPU_MAX_SEG; j++) {
                    if (j >= tp.nseg) continue;
                    double x = ct.chi[i * SFGPU_MAX_SEG + j];
                    if (x != 0) { ci += x * rho[j]; cb += x * phib[j]; }
                }
                up = -log(G);
                up -= ci;
                up += cb;
                if (tp.el) up -= tp.val[i] * tp.psi[z] * tp.ech / tp.kT;
            }
            omega -= up * tp.phi[i][z];
        }
        for (int i = 0; i < tp.nseg; i++) {
            if (tp.frozen[i]) continue;
            const double p1 = tp.phi[i][z];
#pragma unroll
            for (int j = 0; j < SFGPU_MAX_SEG; j++) {
                if (j >= tp.nseg || tp.frozen[j]) continue;
                const double x = ct.chi[i * SFGPU_MAX_SEG + j];
                omega -= 0.5 * x * p1 * rho[j];
                if (p1 > 0) omega += 0.5 * x * phib[i] * phib[j];
            }
        }
        if (tp.el) {
            // SF_MolList1stO.cpp:1074-1096: added on frozen segments' layers,
            // subtracted elsewhere, boundaries subtracted twice
            omega += tp.surf[z] != 0 ? tp.el[z] * sb[z] : -tp.el[z] * sb[z];
        }
        const double f = tp.el ? -entropy + contact + tp.el[z] : -entropy + contact;
        const double w = wf[z];
        accF += w * f;
        accO += w * omega;
        if (fe) fe[z] = f * sb[z];
        if (gp) gp[z] = omega * sb[z];
    }
    shF[threadIdx.x] = accF;
    shO[threadIdx.x] = accO;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) { shF[threadIdx.x] += shF[threadIdx.x + s]; shO[threadIdx.x] += shO[threadIdx.x + s]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) { partial[blockIdx.x] = shF[0]; partial[gridDim.x + blockIdx.x] = shO[0]; }
}

// per-site contact average of one profile (for the Lattice-level API)
static __global__ void side_kernel(DLat L, const double *__restrict__ p, double *__restrict__ rho) {
    for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < L.M; z += gridDim.x * blockDim.x)
        rho[z] = side_fraction(L, p, z);
}

// SetBoundaries on a profile of K components: 6 swap at mirrors (3D); the
// lumped 1D/2D components swap where the lattice's sw_lo / sw_hi say so
static __global__ void set_boundaries(DLat L, int K, double *__restrict__ p) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < L.M; r += gridDim.x * blockDim.x) {
        int c[3];
        lat_coords(L, r, c);
        if (lat_interior(L, c)) continue;
        int sw = 0;
        int t = lat_map(L, r, &sw);
        if (t == r) {
            // a surface site of a lumped lattice: the + component of each
            // surface axis takes the - one's value (SetBx1(P,Q) with the
            // boundary as its own copy layer)
            if (K == 3 || K == 5) {
                const Lump2 q = lump2_of(L.grad);
                for (int k = 0; k < K; k++) {
                    const int a = q.axis[k];
                    if (a < 0 || q.sgn[k] < 0) continue;
                    const int sm = (c[a] == 0) ? L.sw_lo[a] : (c[a] == L.Md[a] - 1 ? L.sw_hi[a] : 0);
                    if (sm == 2) p[(size_t)k * L.M + r] = p[(size_t)lump2_swap(q, k) * L.M + r];
                }
            }
            continue;
        }
        int swl = 0;   // axes whose boundary this site lies on and swaps, lumped lattices
        if (K == 3 || K == 5)
            for (int d = 0; d < L.grad; d++) {
                if (c[d] == 0 && L.sw_lo[d]) swl |= 1 << d;
                if (c[d] == L.Md[d] - 1 && L.sw_hi[d]) swl |= 1 << d;
            }
        for (int k = 0; k < K; k++) {
            int ks = k;
            if (K == 6) ks = swap_dir(k, sw);
            else if (K == 3 || K == 5) {
                const Lump2 q = lump2_of(L.grad);
                if (q.axis[k] >= 0 && (swl >> q.axis[k]) & 1) ks = lump2_swap(q, k);
            }
            p[(size_t)k * L.M + r] = p[(size_t)ks * L.M + t];
        }
    }
}

// ---- vector helpers for the host-driven iterations ----------------------
// partial dot products a_i . b_i of up to 16 vector pairs, one partial per
// block in a fixed order: partial[i * gridDim.x + block]
struct DotList { const double *a[16]; const double *b[16]; int n; };
static __global__ void dots_partial(size_t len, DotList dl, double *__restrict__ partial) {
    __shared__ double sh[kBlock];
    for (int i = 0; i < dl.n; i++) {
        const double *a = dl.a[i], *b = dl.b[i];
        double acc = 0;
        for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < len; r += (size_t)gridDim.x * blockDim.x)
            acc += a[r] * b[r];
        sh[threadIdx.x] = acc;
        __syncthreads();
        for (int s = blockDim.x / 2; s > 0; s >>= 1) {
            if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x == 0) partial[(size_t)i * gridDim.x + blockIdx.x] = sh[0];
        __syncthreads();
    }
}

static __global__ void finish_sums(int n, int nblocks, const double *__restrict__ partial, double *__restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double acc = 0;
    for (int b = 0; b < nblocks; b++) acc += partial[(size_t)i * nblocks + b];
    out[i] = acc;
}

// DIIS step pieces (SFNewton::PlainLBFGSDIIS, sfnewton.cpp:602-661)
// x -= eta*g; XR[k] = x; XX0[k] = x - x0
static __global__ void diis_step(size_t len, double eta, double *__restrict__ x, const double *__restrict__ x0,
                          const double *__restrict__ g, double *__restrict__ xr, double *__restrict__ xx0) {
    for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < len; r += (size_t)gridDim.x * blockDim.x) {
        double v = x[r] - g[r] * eta;
        x[r] = v;
        xr[r] = v;
        xx0[r] = v - x0[r];
    }
}

struct Coef { double c[64]; int pos[64]; int n; };
// x = sum_i c_i XR[pos_i] (in SFbox's accumulation order)
static __global__ void diis_combine(size_t len, Coef cf, const double *__restrict__ XR, size_t ld, double *__restrict__ x) {
    for (size_t r = blockIdx.x * (size_t)blockDim.x + threadIdx.x; r < len; r += (size_t)gridDim.x * blockDim.x) {
        double v = cf.c[0] * XR[(size_t)cf.pos[0] * ld + r];
        for (int i = 1; i < cf.n; i++) v += cf.c[i] * XR[(size_t)cf.pos[i] * ld + r];
        x[r] = v;
    }
}

}  // namespace sfk
