// sfgpu_kernels.cuh -- streaming kernels of the single-system path.
// Every kernel is grid-stride over lattice sites; all scalars that one
// residual evaluation needs (lnGN, bulk volume fractions, normalisations)
// stay in device memory so a whole evaluation is one asynchronous launch
// sequence that can be captured in a CUDA graph.
#pragma once
#include "sfgpu_internal.cuh"

namespace sfk {

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
    const int worker = blockIdx.x * blockDim.x + threadIdx.x;
    for_interior(L, worker, gridDim.x * blockDim.x, [&](const RowInfo &R, int k, int nlast) {
        const double out = prop1_row(L, R, gin, G, k, nlast);
        const int t = R.base + k;
        gout[t] = out;
        if (mode == COMP_ACC) phi[t] += out * other[t];
        else if (mode == COMP_CENTRE) phi[t] = (phi[t] + out * out) * 0.5;
    });
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

// phi += a * b over all K*M entries summed per site (copolymer end segment,
// SF_Copol1stO.cpp:1218-1222; Lat3D2ndO::ConnectG over six components)
static __global__ void connect(int M, int K, const double *__restrict__ a, const double *__restrict__ b,
                        double *__restrict__ phi) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < M; r += gridDim.x * blockDim.x) {
        double p = phi[r];
        for (int k = 0; k < K; k++) p += a[(size_t)k * M + r] * b[(size_t)k * M + r];
        phi[r] = p;
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
            for (int k = 0; k < K; k++) acc += wr * g[(size_t)k * M + r];
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
};
static __global__ void mol_scalars(MolParam p, int nblocks, const double *__restrict__ partial,
                            MolScal *__restrict__ scal, int self) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double v = 0;
    for (int b = 0; b < nblocks; b++) v += partial[b];
    if (p.K == 6) v /= 6.0;
    MolScal s;
    s.lngn = log(v);
    double phib = p.phibulk_in;
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
            s.norm = (p.K == 6) ? c / (6.0 * gn) : c / gn;
        }
        s.phibulk = p.theta / gn;
    } else {
        s.phibulk = phib;
        if (p.type == 0) {
            s.lnc = log(phib);
            s.norm = phib;
        } else {
            s.lnc = log(phib / N);
            s.norm = p.sym ? 2 * phib / N : (p.K == 6 ? phib / (6 * N) : phib / N);
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
                                    const MolScal *__restrict__ scal, double *__restrict__ partial) {
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
        acc += w * (-entropy + contact);
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

// per-site contact average of one profile (for the Lattice-level API)
static __global__ void side_kernel(DLat L, const double *__restrict__ p, double *__restrict__ rho) {
    for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < L.M; z += gridDim.x * blockDim.x)
        rho[z] = side_fraction(L, p, z);
}

// SetBoundaries on a profile (K components, with mirror swaps when K == 6)
static __global__ void set_boundaries(DLat L, int K, double *__restrict__ p) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < L.M; r += gridDim.x * blockDim.x) {
        int c[3];
        lat_coords(L, r, c);
        if (lat_interior(L, c)) continue;
        int sw = 0;
        int t = lat_map(L, r, &sw);
        if (t == r) continue;
        for (int k = 0; k < K; k++) {
            int ks = (K == 6) ? swap_dir(k, sw) : k;
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
