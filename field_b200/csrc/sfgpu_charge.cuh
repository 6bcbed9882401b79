// sfgpu_charge.cuh -- charged systems on the first-order 1D lattices (flat,
// cylinder, sphere):
// the electrostatic potential psi as iteration variables next to the
// segment potentials (SF_Solve.cpp:164-177, :794-852), its Poisson sweep
// (Lat1DFlat::ElectricPotential, Lat1DFlat.cpp:526-549) and field
// (Lat1DFlat::ElectricFieldSquared, :551-570), the layer charge and
// dielectric constant (SF_SegmentList.cpp:759-799), the residual rows of
// psi and the electrostatic terms of u' (SF_Solve.cpp:527-591), and the
// electrostatic free-energy profile (SF_MolList1stO.cpp:942-952); the
// curved lattices' sweeps and fields (Lat1DCylinder.cpp:178-240,
// Lat1DSphere.cpp:76-131).  All
// arithmetic keeps the reference's operation order; every kernel walks the
// M sites of the lattice.
#pragma once
#include "sfgpu_kernels.cuh"

namespace sfk {

// physical constants of SF_Box.h:37-43
constexpr double kBoltzmann = 1.38065812e-23;
constexpr double kEps0 = 8.85418785e-12;
constexpr double kElemCharge = 1.6021773349e-19;
constexpr double kPi = 3.141592653589793;   // PI = 4 atan(1) of SF_Box.h:35, as the host computes it

struct QParam {
    int diffeps;                      // dielectric constants differ among liquid states
    int surf_lo, surf_hi;             // surface bounds (their layers take their own charge)
    int map_lo, map_hi;               // sites the other bound layers copy
    double kT;                        // BOLTZMANN * TEMPERATURE
    double pf_esq;                    // EPS0 * bondlength / kT (ElectricFieldSquared's preFactor)
    double pf_psi;                    // (ELEM_CHARGE / EPS0) / bondlength (ElectricPotential's)
    double val[SFGPU_MAX_SEG], eps[SFGPU_MAX_SEG];
    const int *xu, *xp;               // per site: offset of its first u / of its psi in x, -1 if none
    const double *lsites;             // lattice sites per layer (MultiplyWithLatticeSites)
    int curved, sph;                  // 1D cylinder / sphere
    double off1, ladj;                // offset_first_layer, layer adjustment
    double *psi0, *psi, *esq, *epsav, *charge;
};

// psi0 from x on the sites that carry it; boundary layers copy their mapped
// site (SetBoundaries), a surface layer keeps its own value
static __global__ void q_psi0(DLat L, QParam q, const double *__restrict__ x) {
    for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < L.M; z += gridDim.x * blockDim.x) {
        const int t = lat_map(L, z);
        q.psi0[z] = (q.xp[t] >= 0) ? x[q.xp[t]] : 0.0;
    }
}

// E^2 of Lat1DFlat::ElectricFieldSquared: pf ((psi(z-1) - psi(z))^2 +
// (psi(z) - psi(z+1))^2), surface layers one term
static __global__ void q_esq(DLat L, QParam q) {
    const int M = L.M;
    const double pf = q.pf_esq / 2;
    for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < M; z += gridDim.x * blockDim.x) {
        const double *p = q.psi0;
        if (z == 0) {
            if (q.surf_lo) { double e = p[0] - p[1]; e *= e; q.esq[0] = pf * e; }
        } else if (z == M - 1) {
            if (q.surf_hi) { double e = p[M - 2] - p[M - 1]; e *= e; q.esq[M - 1] = pf * e; }
        } else {
            double emin = p[z - 1] - p[z];
            emin *= emin;
            double eplus = p[z] - p[z + 1];
            eplus *= eplus;
            q.esq[z] = pf * (emin + eplus);
        }
    }
}

// segment weighting factor of a state on a charged lattice: exp(-x) times
// exp(-v psi0 e / kT) and, when the liquid states' dielectric constants
// differ, exp(eps E^2 / 2) (SF_Solve.cpp:808, :819-834); boundary layers copy
static __global__ void swf_update_q(DLat L, QParam q, const double *__restrict__ x, int cls, int seg,
                                    const double *__restrict__ range, int pinned, double *__restrict__ gfull,
                                    double *__restrict__ gseg) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < L.M; r += gridDim.x * blockDim.x) {
        const int t = lat_map(L, r);
        const int o = q.xu[t];
        double v = 0.0;
        if (o >= 0) {
            v = exp(-x[o + cls] - 0.0);
            v *= exp(-q.val[seg] * q.psi0[t] * kElemCharge / q.kT);
            if (q.diffeps) v *= exp(0.5 * q.eps[seg] * q.esq[t]);
        }
        gfull[r] = v;
        gseg[r] = pinned ? (range[t] > 0 ? v : 0.0) : v;
    }
}

// radius of layer z's outer edge in the curved sweeps: the reference starts
// from z0 and adds 1 per layer (Z++), the same additions here
__device__ __forceinline__ double q_radius(double z0, int z) {
    double Z = z0;
    for (int k = 0; k < z; k++) Z++;
    return Z;
}

// E^2 on the 1D cylinder (Lat1DCylinder.cpp:211-240) and sphere
// (Lat1DSphere.cpp:108-131), per layer from its two differences
static __global__ void q_esq_curved(DLat L, QParam q) {
    const int M = L.M;
    const double *p = q.psi0;
    for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < M; z += gridDim.x * blockDim.x) {
        if (q.sph) {
            const double pf = q.pf_esq * kPi * 2, z0 = q.off1 + q.ladj - 1;
            auto ep = [&](int k) { double e = q_radius(z0, k) * (p[k] - p[k + 1]); e *= e; return e; };
            if (z == 0) { if (q.surf_lo) q.esq[0] = pf * ep(0) / q.lsites[0]; }
            else if (z == M - 1) { if (q.surf_hi) q.esq[M - 1] = pf * ep(M - 2) / q.lsites[M - 1]; }
            else q.esq[z] = pf * (ep(z - 1) + ep(z)) / q.lsites[z];
            continue;
        }
        const double pf = q.pf_esq / 2, z0 = q.off1 + q.ladj - 1.5;
        auto ep = [&](int k) { double e = p[k] - p[k + 1]; e *= (q_radius(z0, k) + 0.5) * e; return e; };
        if (z == 0) {
            if (q.off1 > 0 && q.surf_lo) q.esq[0] = pf * ep(0) / q_radius(z0, 0);
        } else if (z == M - 1) {
            if (q.surf_hi) q.esq[M - 1] = pf * ep(M - 2) / q_radius(z0, M - 2);
        } else if (z == 1 && q.off1 <= 0) {
            q.esq[1] = pf * ep(1) / q_radius(z0, 1);
        } else {
            q.esq[z] = pf * (ep(z - 1) + ep(z)) / q_radius(z0, z);
        }
    }
}

// layer dielectric constant sum_i phi_i eps_i and charge sum_i phi_i v_i /
// phi_T times the layer's lattice sites, states in order
static __global__ void q_eps_charge(int M, int nseg, PtrList phi, QParam q) {
    for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < M; z += gridDim.x * blockDim.x) {
        double e = 0, c = 0, pt = 0;
        for (int i = 0; i < nseg; i++) {
            const double p = phi.p[i][z];
            e += p * q.eps[i];
            c += p * q.val[i];
            pt += p;
        }
        c /= pt;
        c *= q.lsites[z];
        q.epsav[z] = e;
        q.charge[z] = c;
    }
}

// one Jacobi sweep of the Poisson equation (Lat1DFlat::ElectricPotential)
static __global__ void q_poisson(DLat L, QParam q) {
    const int M = L.M;
    const double pf = 2 * q.pf_psi;
    const double *e = q.epsav, *p0 = q.psi0;
    for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < M; z += gridDim.x * blockDim.x) {
        if (z == M - 1) {
            q.psi[z] = q.surf_hi ? p0[M - 2] + pf * q.charge[M - 1] / (e[M - 2] + e[M - 1]) : p0[q.map_hi];
        } else if (z == 0) {
            q.psi[0] = q.surf_lo ? p0[1] + pf * q.charge[0] / (e[0] + e[1]) : p0[q.map_lo];
        } else {
            const double epsmin = e[z - 1] + e[z], epsplus = e[z] + e[z + 1];
            q.psi[z] = (epsmin * p0[z - 1] + pf * q.charge[z] + epsplus * p0[z + 1]) / (epsmin + epsplus);
        }
    }
}

// the Poisson sweep on the 1D cylinder (Lat1DCylinder.cpp:178-210) and
// sphere (Lat1DSphere.cpp:76-107): the dielectric sums weighted by the
// radius (squared on the sphere) of each layer's outer edge; without an
// offset the first interior layer takes only its outer neighbour; entries
// the reference leaves unset keep their value
static __global__ void q_poisson_curved(DLat L, QParam q) {
    const int M = L.M;
    const double pf = q.sph ? q.pf_psi / 2 / kPi : q.pf_psi / kPi;
    const double z0 = q.off1 + q.ladj - 1;
    const double *e = q.epsav, *p0 = q.psi0;
    auto W = [&](int k) {
        const double Z = q_radius(z0, k);
        return (q.sph ? Z * Z : Z) * (e[k] + e[k + 1]);
    };
    for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < M; z += gridDim.x * blockDim.x) {
        if (z == 0) {
            if (q.off1 > 0 && q.surf_lo) q.psi[0] = p0[1] + pf * q.charge[0] / W(0);
        } else if (z == M - 1) {
            if (q.surf_hi) q.psi[M - 1] = p0[M - 2] + pf * q.charge[M - 1] / W(M - 2);
        } else if (z == 1 && q.off1 <= 0) {
            q.psi[1] = p0[2] + pf * q.charge[1] / W(1);
        } else {
            const double epsmin = W(z - 1), epsplus = W(z);
            q.psi[z] = (pf * q.charge[z] + p0[z - 1] * epsmin + p0[z + 1] * epsplus) / (epsmin + epsplus);
        }
    }
}

// SF_Solve::GetResiduals on a charged lattice: psi0 - psi on the sites of
// psi, and u' with -v psi0 e / kT (+ eps E^2 / 2) of the class's last state
static __global__ void residual_q(DLat L, ResParam rp, ChiTable ct, QParam q, const double *__restrict__ chib,
                                  double *__restrict__ f) {
    for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < L.M; z += gridDim.x * blockDim.x) {
        if (q.xp[z] >= 0) f[q.xp[z]] = q.psi0[z] - q.psi[z];
        const int o = q.xu[z];
        if (o < 0) continue;
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
            const int st = rp.rep[c];
            double v = -log(rp.gfull[c][z]);
            double ci = 0;
            for (int i = 0; i < rp.nseg; i++) {
                const double x = ct.chi[st * SFGPU_MAX_SEG + i];
                if (x != 0) ci += x * rho[i];
            }
            v -= ci / phit;
            v += chib[c];
            v -= q.val[st] * q.psi0[z] * kElemCharge / q.kT;
            if (q.diffeps) v += 0.5 * q.eps[st] * q.esq[z];
            u[c] = v;
            av += v;
        }
        av /= rp.nclass;
        for (int c = 0; c < rp.nclass; c++) f[o + c] = -1.0 + 1.0 / phit + u[c] - av;
    }
}

// electrostatic free-energy profile 1/2 psi q e / kT with q the layer charge
// divided by the layer's lattice sites (GetElectricInteractionsProfile)
static __global__ void q_elec(int M, QParam q, double *__restrict__ el) {
    for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < M; z += gridDim.x * blockDim.x) {
        double c = q.charge[z];
        if (!q.curved || c != 0) c /= q.lsites[z];   // DivideByLatticeSites (curved: nonzero only)
        el[z] = 0.5 * q.psi[z] * c * kElemCharge / q.kT;
    }
}

// the neutralizer's bulk fraction, -(sum of the other molecules' bulk
// charge) N / Q (SF_MolList1stO.cpp:250-266)
struct NeutParam {
    int nmol, solvent, self;
    double q[SFGPU_MAX_SEG], n[SFGPU_MAX_SEG];   // bulk charge and length per molecule
};
static __global__ void q_neutralizer(NeutParam np, const MolScal *__restrict__ scal, double *__restrict__ out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double bc = 0;
    for (int m = 0; m < np.nmol; m++) {
        if (m == np.solvent || m == np.self) continue;
        bc += np.q[m] * scal[m].phibulk / np.n[m];
    }
    *out = -bc * np.n[np.self] / np.q[np.self];
}

}  // namespace sfk
