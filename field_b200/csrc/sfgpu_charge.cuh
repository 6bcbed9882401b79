// sfgpu_charge.cuh -- charged systems on every lattice (1D flat,
// cylinder, sphere; 2D flat and cylinder; 3D; first or second order):
// the electrostatic potential psi as iteration variables next to the
// segment potentials (SF_Solve.cpp:164-177, :794-852), its Poisson sweep
// (Lat1DFlat::ElectricPotential, Lat1DFlat.cpp:526-549) and field
// (Lat1DFlat::ElectricFieldSquared, :551-570), the layer charge and
// dielectric constant (SF_SegmentList.cpp:759-799), the residual rows of
// psi and the electrostatic terms of u' (SF_Solve.cpp:527-591), and the
// electrostatic free-energy profile (SF_MolList1stO.cpp:942-952); the
// curved lattices' sweeps and fields (Lat1DCylinder.cpp:178-240,
// Lat1DSphere.cpp:76-131), and those of the 2D and 3D lattices
// (Lat2DFlat.cpp:1116-1272, Lat2DCylinder.cpp:323-541, Lat3D.cpp:1937-2005).  All
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
    int surf_ylo, surf_yhi;           // 2D: surface bounds of the second gradient
    int cyl2;                         // 2D cylinder
    double z0c;                       // 2D cylinder: radius to the centre of layer 1, L[3]/2/PI - 2
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

// ---------------------------------------------------------------------------
// 2D sweeps and fields, one thread per site.  The reference walks the
// lattice row by row and carries the dielectric sum and the squared
// difference of the previous site along a row; here every site forms the
// same operands itself (two-term sums commute exactly) and combines them in
// the reference's order.  1-based site k of the reference is index k - 1;
// x1, y1 are the 1-based row and column.  A boundary row or column is
// computed only where its bound is a surface, as in the reference, which
// also keeps the charge of site 1 for the upper y corner of the lower x row
// and the dielectric sum eps[M-MY] + eps[M] for the upper corner of the
// upper x row.
// ---------------------------------------------------------------------------
struct Q2 {
    const double *e, *p, *q;
    __device__ double E(int k) const { return e[k - 1]; }
    __device__ double P(int k) const { return p[k - 1]; }
    __device__ double C(int k) const { return q[k - 1]; }
};

// Lat2DFlat::ElectricPotential (Lat2DFlat.cpp:1116-1207)
__device__ __forceinline__ bool q_poisson_2dflat_site(const QParam &q, const Q2 &a, int MX, int MY, int x1, int y1,
                                                      double &out) {
    const int M = MX * MY, z = (x1 - 1) * MY + y1;
    const double pf = 2 * q.pf_psi;
    if (x1 == 1) {
        if (!q.surf_lo) return false;
        if (y1 == 1) {
            if (!q.surf_ylo) return false;
            const double ex = a.E(1) + a.E(MY + 1), ey = a.E(1) + a.E(2);
            out = (pf * a.C(1) + ex * a.P(MY + 1) + ey * a.P(2)) / (ex + ey);
        } else if (y1 == MY) {
            if (!q.surf_yhi) return false;
            const double ex = a.E(MY) + a.E(MY + MY), ey = a.E(2) + a.E(3);
            out = (pf * a.C(1) + ex * a.P(MY + MY) + ey * a.P(MY - 1)) / (ex + ey);
        } else {
            const double eym = (y1 == MY - 1) ? a.E(1) + a.E(2) : a.E(z + 1) + a.E(z + 2);
            const double ex = a.E(z) + a.E(z + MY), eyp = a.E(z) + a.E(z + 1);
            out = (pf * a.C(z) + ex * a.P(z + MY) + eym * a.P(z - 1) + eyp * a.P(z + 1)) / (ex + eym + eyp);
        }
        return true;
    }
    if (x1 == MX) {
        if (!q.surf_hi) return false;
        if (y1 == 1) {
            if (!q.surf_ylo) return false;
            const double ey = a.E(M - MY + 1) + a.E(M - MY + 2), exm = a.E(M - MY + 1) + a.E(M - MY - MY + 1);
            out = (pf * a.C(M - MY + 1) + exm * a.P(M - MY - MY + 1) + ey * a.P(M - MY + 2)) / (exm + ey);
        } else if (y1 == MY) {
            if (!q.surf_yhi) return false;
            const double exm = a.E(M - MY) + a.E(M), ey = a.E(M - 1) + a.E(M);
            out = (pf * a.C(M) + exm * a.P(M - MY) + ey * a.P(M - 1)) / (exm + ey);
        } else {
            const double eym = a.E(z - 1) + a.E(z), exm = a.E(z) + a.E(z - MY), eyp = a.E(z) + a.E(z + 1);
            out = (pf * a.C(z) + exm * a.P(z - MY) + eym * a.P(z - 1) + eyp * a.P(z + 1)) / (exm + eym + eyp);
        }
        return true;
    }
    const double exm = a.E(z) + a.E(z - MY), exp_ = a.E(z) + a.E(z + MY);
    if (y1 == 1) {
        if (!q.surf_ylo) return false;
        const double eyp = a.E(z) + a.E(z + 1);
        out = (pf * a.C(z) + exm * a.P(z - MY) + exp_ * a.P(z + MY) + eyp * a.P(z + 1)) / (exm + exp_ + eyp);
    } else if (y1 == MY) {
        if (!q.surf_yhi) return false;
        const double eyp = a.E(z - 1) + a.E(z);
        out = (pf * a.C(z) + exm * a.P(z - MY) + exp_ * a.P(z + MY) + eyp * a.P(z - 1)) / (exm + exp_ + eyp);
    } else {
        const double eym = a.E(z - 1) + a.E(z), eyp = a.E(z) + a.E(z + 1);
        out = (pf * a.C(z) + exm * a.P(z - MY) + exp_ * a.P(z + MY) + eym * a.P(z - 1) + eyp * a.P(z + 1)) /
              (exm + exp_ + eym + eyp);
    }
    return true;
}

// Lat2DCylinder::ElectricPotential (Lat2DCylinder.cpp:323-450): row x1 has
// the radius Z = z0c + 1 + ... + 1 (x1 - 1 additions), the charge term the
// factor 1/(PI Z), the terms across rows 1 -+ 1/(2Z); without an offset the
// first interior row has no inner neighbour (and row 1 is not computed)
__device__ __forceinline__ bool q_poisson_2dcyl_site(const QParam &q, const Q2 &a, int MX, int MY, int x1, int y1,
                                                     double &out) {
    const int M = MX * MY, z = (x1 - 1) * MY + y1;
    const double Z = q_radius(q.z0c, x1 - 1);
    const double pf = q.pf_psi / kPi / Z;
    const double xm = 1 - 0.5 / Z, xp = 1 + 0.5 / Z;
    const bool axis = q.off1 <= 0;
    if ((axis && x1 == 2) || (!axis && x1 == 1)) {
        // walked from y = MY down; no inner neighbour
        if (x1 == 1 && !q.surf_lo) return false;
        const int zr = (x1 - 1) * MY;   // site before the row's first
        if (y1 == MY) {
            if (!q.surf_yhi) return false;
            const double eym = a.E(z) + a.E(z - 1), ex = xp * (a.E(z) + a.E(z + MY));
            out = (pf * a.C(z) + eym * a.P(z - 1) + ex * a.P(z + MY)) / (eym + ex);
        } else if (y1 == 1) {
            if (!q.surf_ylo) return false;
            const double ex = xp * (a.E(z) + a.E(z + MY)), eym = a.E(zr + 2) + a.E(zr + 1);
            out = (pf * a.C(z) + ex * a.P(z + MY) + eym * a.P(z + 1)) / (ex + eym);
        } else {
            const double eyp = a.E(z + 1) + a.E(z), eym = a.E(z) + a.E(z - 1), ex = xp * (a.E(z) + a.E(z + MY));
            out = (pf * a.C(z) + ex * a.P(z + MY) + eym * a.P(z - 1) + eyp * a.P(z + 1)) / (ex + eym + eyp);
        }
        return true;
    }
    if (x1 == 1) return false;   // axis: the boundary row is not computed
    if (x1 == MX) {
        if (!q.surf_hi) return false;
        if (y1 == 1) {
            if (!q.surf_ylo) return false;
            const double ey = a.E(M - MY + 1) + a.E(M - MY + 2), exm = xm * (a.E(M - MY - MY + 1) + a.E(M - MY + 1));
            out = (pf * a.C(M - MY + 1) + exm * a.P(M - MY - MY + 1) + ey * a.P(M - MY + 2)) / (exm + ey);
        } else if (y1 == MY) {
            if (!q.surf_yhi) return false;
            const double exm = xm * (a.E(M) + a.E(M - MY)), ey = a.E(M - 1) + a.E(M);
            out = (pf * a.C(M) + exm * a.P(M - MY) + ey * a.P(M - 1)) / (exm + ey);
        } else {
            const double eym = a.E(z - 1) + a.E(z), eyp = a.E(z) + a.E(z + 1), exm = xm * (a.E(z - MY) + a.E(z));
            out = (pf * a.C(z) + exm * a.P(z - MY) + eym * a.P(z - 1) + eyp * a.P(z + 1)) / (exm + eym + eyp);
        }
        return true;
    }
    const double exm = xm * (a.E(z - MY) + a.E(z)), exp_ = xp * (a.E(z) + a.E(z + MY));
    if (y1 == 1) {
        if (!q.surf_ylo) return false;
        const double eyp = a.E(z) + a.E(z + 1);
        out = (pf * a.C(z) + exm * a.P(z - MY) + exp_ * a.P(z + MY) + eyp * a.P(z + 1)) / (exm + exp_ + eyp);
    } else if (y1 == MY) {
        if (!q.surf_yhi) return false;
        const double eyp = a.E(z - 1) + a.E(z);
        out = (pf * a.C(z) + exm * a.P(z - MY) + exp_ * a.P(z + MY) + eyp * a.P(z - 1)) / (exm + exp_ + eyp);
    } else {
        const double eym = a.E(z - 1) + a.E(z), eyp = a.E(z) + a.E(z + 1);
        out = (pf * a.C(z) + exm * a.P(z - MY) + exp_ * a.P(z + MY) + eym * a.P(z - 1) + eyp * a.P(z + 1)) /
              (exm + exp_ + eym + eyp);
    }
    return true;
}

static __global__ void q_poisson_2d(DLat L, QParam q) {
    const int MX = L.Md[0], MY = L.Md[1];
    const Q2 a{q.epsav, q.psi0, q.charge};
    for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < L.M; z += gridDim.x * blockDim.x) {
        const int x1 = z / MY + 1, y1 = z - (x1 - 1) * MY + 1;
        double v;
        const bool set = q.cyl2 ? q_poisson_2dcyl_site(q, a, MX, MY, x1, y1, v)
                                : q_poisson_2dflat_site(q, a, MX, MY, x1, y1, v);
        if (set) q.psi[z] = v;
    }
}

__device__ __forceinline__ double q_sq(double v) { return v * v; }

// Lat2DFlat::ElectricFieldSquared (Lat2DFlat.cpp:1209-1272) and
// Lat2DCylinder::ElectricFieldSquared (Lat2DCylinder.cpp:452-541), whose
// squared differences across rows carry 1 -+ 1/(2Z)
static __global__ void q_esq_2d(DLat L, QParam q) {
    const int MX = L.Md[0], MY = L.Md[1];
    const Q2 a{q.epsav, q.psi0, q.charge};
    const double pf = q.pf_esq / 2;
    for (int z0 = blockIdx.x * blockDim.x + threadIdx.x; z0 < L.M; z0 += gridDim.x * blockDim.x) {
        const int x1 = z0 / MY + 1, y1 = z0 - (x1 - 1) * MY + 1, z = z0 + 1;
        double xm = 1, xp = 1;
        if (q.cyl2) {
            const double Z = q_radius(q.z0c, x1 - 1);
            xm = 1 - 0.5 / Z;
            xp = 1 + 0.5 / Z;
        }
        // squared difference to the row below / above, weighted on the cylinder
        auto dxm = [&]() { double d = a.P(z) - a.P(z - MY); return q.cyl2 ? d * (xm * d) : d * d; };
        auto dxp = [&]() { double d = a.P(z) - a.P(z + MY); return q.cyl2 ? d * (xp * d) : d * d; };
        const bool first = q.cyl2 ? ((q.off1 <= 0 && x1 == 2) || (q.off1 > 0 && x1 == 1 && q.surf_lo))
                                  : (x1 == 1 && q.surf_lo);
        if (first) {
            // walked from y = MY - 1 down, no inner row
            if (y1 < 2 || y1 > MY - 1) continue;
            const double eyp = q_sq(a.P(z) - a.P(z + 1)), eym = q_sq(a.P(z) - a.P(z - 1));
            q.esq[z0] = pf * (dxp() + eym + eyp);
            continue;
        }
        if (x1 == 1) continue;
        if (x1 == MX) {
            if (!q.surf_hi || y1 < 2 || y1 > MY - 1) continue;
            const double eym = q_sq(a.P(z - 1) - a.P(z)), eyp = q_sq(a.P(z) - a.P(z + 1));
            q.esq[z0] = pf * (dxm() + eym + eyp);
            continue;
        }
        if (y1 == 1) {
            if (!q.surf_ylo) continue;
            const double eyp = q_sq(a.P(z) - a.P(z + 1));
            q.esq[z0] = pf * (dxm() + dxp() + eyp);
        } else if (y1 == MY) {
            if (!q.surf_yhi) continue;
            const double eym = q_sq(a.P(z - 1) - a.P(z));
            q.esq[z0] = pf * (dxm() + dxp() + eym);
        } else {
            const double eym = q_sq(a.P(z - 1) - a.P(z)), eyp = q_sq(a.P(z) - a.P(z + 1));
            q.esq[z0] = pf * (dxm() + dxp() + eym + eyp);
        }
    }
}

// Lat3D::ElectricPotential (Lat3D.cpp:1937-1969) on the interior sites: the
// six neighbour terms -x, +x, -y, +y, -z, +z (dielectric profile and psi0
// with boundary copies), the charge term, the division by the summed
// dielectric weights (0 where not positive); boundary entries copy their
// mapped site afterwards (q_copy_boundaries)
static __global__ void q_poisson_3d(DLat L, QParam q) {
    const int jx = L.st[0], jy = L.st[1];
    const double *e = q.epsav, *p0 = q.psi0;
    for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < L.M; z += gridDim.x * blockDim.x) {
        int c[3];
        lat_coords(L, z, c);
        if (!lat_interior(L, c)) continue;
        const int nb[6] = {z - jx, z + jx, z - jy, z + jy, z - 1, z + 1};
        const double ez = e[z];
        double w = e[lat_map(L, nb[0])] + ez;
        double tot = w, acc = w * p0[nb[0]];
#pragma unroll
        for (int k = 1; k < 6; k++) {
            w = e[lat_map(L, nb[k])] + ez;
            tot += w;
            acc += w * p0[nb[k]];
        }
        acc += q.charge[z] * (2 * q.pf_psi);
        q.psi[z] = (tot > 0) ? acc / tot : 0.0;
    }
}

// Lat3D::ElectricFieldSquared (Lat3D.cpp:1979-2003) on the interior sites
static __global__ void q_esq_3d(DLat L, QParam q) {
    const int jx = L.st[0], jy = L.st[1];
    const double *p = q.psi0;
    const double pf = q.pf_esq / 2;
    for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < L.M; z += gridDim.x * blockDim.x) {
        int c[3];
        lat_coords(L, z, c);
        if (!lat_interior(L, c)) continue;
        double v = q_sq(p[z] - p[z - jx]);
        v += q_sq(p[z] - p[z + jx]);
        v += q_sq(p[z] - p[z - jy]);
        v += q_sq(p[z] - p[z + jy]);
        v += q_sq(p[z] - p[z - 1]);
        v += q_sq(p[z] - p[z + 1]);
        q.esq[z] = v * pf;
    }
}

// boundary entries of a profile from their mapped sites (SetBoundaries)
static __global__ void q_copy_boundaries(DLat L, double *__restrict__ v) {
    for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < L.M; z += gridDim.x * blockDim.x) {
        const int t = lat_map(L, z);
        if (t != z) v[z] = v[t];
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
        // DivideByLatticeSites: the 1D curved lattices skip zero entries, the
        // 2D cylinder rows without sites
        if (q.cyl2) { if (q.lsites[z] != 0) c /= q.lsites[z]; }
        else if (!q.curved || c != 0) c /= q.lsites[z];
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
