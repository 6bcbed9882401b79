// sfgpu_logspace.cuh -- overflow-protected chain statistics (sys :
// overflow_protection : true): the first-order 1D and 2D lattices of SFbox's
// *1stOS family (Lat1DFlat1stOS, Lat1DCyl1stOS, Lat1DSphere1stOS,
// Lat2DFlat1stOS, Lat2DCyl1stOS) keep every propagator, composition and
// lnGN sum as a natural logarithm, so that chains whose statistical weights
// leave the range of a double stay finite.  0 is represented by LOGZERO =
// -DBL_MAX/2 (SF_Box.h:31-53); segment weights enter through MakeSafe and
// the volume fractions leave through RestoreFromSafe (Lat1DFlat1stOS.cpp:21-56).
#pragma once
#include <cfloat>
#include "sfgpu_kernels.cuh"

namespace sfk {

#define SFGPU_LOGZERO (-DBL_MAX / 2)

// SF_Box.h:31-53: LOGMAXDOUBLE = log(DBL_MAX), LOGCUTOFF = 100,
// LOGTOLERANCE = 50, LOGMAXPREFACTOR = LOGMAXDOUBLE - LOGCUTOFF - LOGTOLERANCE,
// CUTOFF = exp(LOGCUTOFF); filled on the host
struct LogConst {
    double lmax, logcutoff, cutoff, prefactor;
};

// per-lattice constants of the log-space step
enum { LOG_FLAT1 = 0, LOG_CURVED1 = 1, LOG_FLAT2 = 2, LOG_CYL2 = 3 };
struct LogLat {
    int kind;
    double logl0, logl1, logl1l0;   // flat: log(l0), log(l1), log(l1/l0) with l0 = 1 - 2 l1 (1D), 1 - 4 l1 (2D)
    double nl_centre;               // 2D cylinder: the centre weight its step uses, 1 - 4 l1
    const double *logl0x, *loglmx, *loglpx;   // 2D cylinder: log of lambda0, lambda-, lambda+ by x (0 where <= 0)
};

// MakeSafe (Lat1DFlat1stOS.cpp:21-38)
static __global__ void make_safe(int M, LogConst c, const double *__restrict__ a, double *__restrict__ out) {
    for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < M; z += gridDim.x * blockDim.x) {
        const double v = a[z];
        double r;
        if (v > 0) {
            if (v > c.cutoff) {
                const double y = (log(v) - c.logcutoff) / c.prefactor;
                r = c.logcutoff + 0.5 * c.prefactor * log((1 + y) / (1 - y));
            } else {
                r = log(v);
            }
        } else {
            r = SFGPU_LOGZERO;
        }
        out[z] = r;
    }
}

__device__ __forceinline__ double restore_from_safe(const LogConst &c, double v) {
    // RestoreFromSafe (Lat1DFlat1stOS.cpp:39-55)
    if (v > SFGPU_LOGZERO) {
        if (v > c.logcutoff) return exp(c.logcutoff + c.prefactor * tanh((v - c.logcutoff) / c.prefactor));
        return exp(v);
    }
    return 0.0;
}

static __global__ void fill_value(int n, double v, double *__restrict__ p) {
    for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < n; z += gridDim.x * blockDim.x) p[z] = v;
}

// log(e^out + e^(a + b)) for a, b > LOGZERO, in ConnectG's form
// (Lat1DFlat1stOS.cpp:344-360): the sum replaces out when out is LOGZERO or
// when the new term exceeds it by more than the range of a double
__device__ __forceinline__ double log_connect(const LogConst &c, double out, double a, double b) {
    if (a > SFGPU_LOGZERO && b > SFGPU_LOGZERO) {
        const double x = a + b - out;
        if (x > c.lmax - 1 || out == SFGPU_LOGZERO) return a + b;
        return out + log1p(exp(x));
    }
    return out;
}

// One log-space step at interior position k of row R: lg = log G (site),
// neighbours read from gin (logs).  Surface layers hold LOGZERO.
//  1D flat   Lat1DFlat1stOS.cpp:120-145 (centre first when l1 < 1/2)
//  1D curved Lat1DCyl1stOS.cpp:45-74 (also Lat1DSphere1stOS)
//  2D flat   Lat2DFlat1stOS.cpp:140-169 with getNewGi (:335-362); neighbours
//            y-1, y+1, x-1, x+1
//  2D cyl    Lat2DCyl1stOS.cpp:173-228: neighbours y-1, centre, y+1, x-1,
//            x+1 with weights l1, 1 - 4 l1, l1, lambda-(x), lambda+(x); the
//            first non-zero neighbour is the pivot
__device__ __forceinline__ double log_step_row(const DLat &L, const LogLat &Q, const RowInfo &R,
                                               const double *__restrict__ gin, double lg, int k, int nlast) {
    const double LZ = SFGPU_LOGZERO;
    if (lg == LZ) return LZ;
    const int d = L.grad - 1;
    const int t = R.base + k;
    const double b = gin[t];
    const double a = (k == 1 && L.bc_lo[d] == SFGPU_BOUND_SURFACE) ? LZ
                     : gin[R.base + ((k == 1) ? L.map_lo[d] : k - 1)];
    const double c = (k == nlast && L.bc_hi[d] == SFGPU_BOUND_SURFACE) ? LZ
                     : gin[R.base + ((k == nlast) ? L.map_hi[d] : k + 1)];
    if (Q.kind == LOG_FLAT1) {
        if (b > LZ && L.l1 < 0.5) return lg + Q.logl0 + b + log1p(exp(Q.logl1l0 + a - b) + exp(Q.logl1l0 + c - b));
        if (a > LZ) return lg + Q.logl1 + a + log1p(exp(c - a));
        if (c > LZ) return lg + Q.logl1 + c;
        return LZ;
    }
    if (Q.kind == LOG_CURVED1) {
        const double lm = L.lam_m[t], lp = L.lam_p[t];
        const double l0 = 1 - lp - lm;
        if (b > LZ && l0 > 0) return lg + log(l0) + b + log1p((lm / l0) * exp(a - b) + (lp / l0) * exp(c - b));
        if (a > LZ) return lg + log(lm) + a + log1p((lp / lm) * exp(c - a));
        if (c > LZ) return lg + log(lp) + c;
        return LZ;
    }
    const int x = R.x;
    const double u = (x == 1 && L.bc_lo[0] == SFGPU_BOUND_SURFACE) ? LZ : gin[t + R.up];
    const double dn = (x == L.Md[0] - 2 && L.bc_hi[0] == SFGPU_BOUND_SURFACE) ? LZ : gin[t + R.dn];
    if (Q.kind == LOG_FLAT2) {
        const double n[4] = {a, c, u, dn};
        if (b != LZ && L.l1 < 0.25) {
            double lnterm = 0;
#pragma unroll
            for (int i = 0; i < 4; i++)
                if (n[i] != LZ) lnterm += exp(Q.logl1l0 + n[i] - b);
            return lg + Q.logl0 + b + log1p(lnterm);
        }
        int i = 0;
        while (i < 4 && n[i] == LZ) i++;
        if (i == 4) return LZ;
        double lnterm = 0;
        for (int j = i + 1; j < 4; j++)
            if (n[j] != LZ) lnterm += exp(n[j] - n[i]);
        return lg + Q.logl1 + n[i] + log1p(lnterm);
    }
    // LOG_CYL2
    const double ng[5] = {a, b, c, u, dn};
    const double nl[5] = {L.l1, Q.nl_centre, L.l1, L.lam_m[x], L.lam_p[x]};
    const double lognl[5] = {Q.logl1, Q.logl0x[x], Q.logl1, Q.loglmx[x], Q.loglpx[x]};
    int i = 0;
    while (i < 5 && (ng[i] == LZ || nl[i] <= 0)) i++;
    if (i == 5) return LZ;
    double lnterm = 0;
    for (int j = 0; j < 5; j++)
        if (j != i && ng[j] != LZ) lnterm += nl[j] * exp(ng[j] - ng[i]);
    return lg + lognl[i] + ng[i] + log1p(lnterm / nl[i]);
}

// One log-space propagator step over the interior, with the composition of
// the molecule drivers fused: COMP_ACC phi = log(e^phi + e^(out + other))
// (ConnectG); COMP_CENTRE phi = log(e^phi + e^(2 out)) + log(1/2) (the odd
// centre of a symmetric chain, ConnectG(Gi_inv, Gi_inv) then NormPhiFree(0.5),
// SF_Homopol1stO.cpp:583-585).
static __global__ void step1_log_rows(DLat L, LogLat Q, LogConst lc, const double *__restrict__ gin,
                                      const double *__restrict__ lG, double *__restrict__ gout,
                                      const double *__restrict__ other, double *__restrict__ phi, int mode) {
    const int worker = blockIdx.x * blockDim.x + threadIdx.x, nworkers = gridDim.x * blockDim.x;
    for_interior(L, worker, nworkers, [&](const RowInfo &R, int k, int nlast) {
        const int t = R.base + k;
        const double out = log_step_row(L, Q, R, gin, lG[t], k, nlast);
        gout[t] = out;
        if (mode == COMP_ACC) {
            phi[t] = log_connect(lc, phi[t], out, other[t]);
        } else if (mode == COMP_CENTRE) {
            double p = log_connect(lc, phi[t], out, out);
            if (p > SFGPU_LOGZERO) p += log(0.5);
            phi[t] = p;
        }
    });
}

// phi = log(e^phi + e^(a + b)) on every site (ConnectG of the chain end)
static __global__ void connect_log(int M, LogConst lc, const double *__restrict__ a, const double *__restrict__ b,
                                   double *__restrict__ phi) {
    for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < M; z += gridDim.x * blockDim.x)
        phi[z] = log_connect(lc, phi[z], a[z], b[z]);
}

// lnGN = log sum_z w(z) e^(v(z)) over the sites with w > 0 and v > LOGZERO,
// shifted by the largest term (one block; the weights carry the lattice's
// own ComputeLnGN terms, see the builder).  LOGZERO when no term is left.
static __global__ void lse_weighted(int M, const double *__restrict__ v, const double *__restrict__ w,
                                    double *__restrict__ out) {
    __shared__ double red[32];
    double mx = -DBL_MAX;
    for (int z = threadIdx.x; z < M; z += blockDim.x)
        if (w[z] > 0 && v[z] > SFGPU_LOGZERO) mx = fmax(mx, v[z] + log(w[z]));
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x < 32) {
        double m2 = (threadIdx.x < (blockDim.x + 31) / 32) ? red[threadIdx.x] : -DBL_MAX;
        for (int o = 16; o > 0; o >>= 1) m2 = fmax(m2, __shfl_xor_sync(0xffffffffu, m2, o));
        if (threadIdx.x == 0) red[0] = m2;
    }
    __syncthreads();
    mx = red[0];
    __syncthreads();
    double s = 0;
    if (mx > -DBL_MAX)
        for (int z = threadIdx.x; z < M; z += blockDim.x)
            if (w[z] > 0 && v[z] > SFGPU_LOGZERO) s += w[z] * exp(v[z] - mx);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0;
        for (int i = 0; i < (int)((blockDim.x + 31) / 32); i++) tot += red[i];
        *out = (mx > -DBL_MAX && tot > 0) ? mx + log(tot) : SFGPU_LOGZERO;
    }
}

// The scalars of mol_scalars from a lnGN computed in log space: the partial
// sum is replaced by lnGN itself (phibulk, ln C and the linear norm as
// there; the log of the norm is taken where it is applied).
static __global__ void mol_scalars_log(MolParam p, const double *__restrict__ lngn, MolScal *__restrict__ scal,
                                       int self) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    MolScal s;
    s.lngn = *lngn;
    double phib = p.phib_dev ? *p.phib_dev : p.phibulk_in;   // a neutralizer's from the device
    if (p.solvent) {
        phib = 1.0;
        for (int m = 0; m < p.nmol; m++)
            if (m != self) phib -= scal[m].phibulk;
    }
    const double N = (double)p.N;
    if (p.freedom == SFGPU_MOL_RESTRICTED) {
        s.lnc = (p.type == 0) ? log(p.theta) - s.lngn : log(p.theta) - s.lngn - log(N);
        s.norm = 0;   // applied as log(numerator) - lnGN
        s.phibulk = p.theta / exp(s.lngn);
    } else {
        s.phibulk = phib;
        if (p.type == 0) { s.lnc = log(phib); s.norm = phib; }
        else { s.lnc = log(phib / N); s.norm = p.sym ? 2 * phib / N : phib / N; }
    }
    if (p.pinned) s.phibulk = 0;
    scal[self] = s;
}

// CorrectDoubleCountG, NormPhiFree / NormPhiRestr and RestoreFromSafe of a
// log-space profile, in place (Lat1DFlat1stOS.cpp:289-298, :340-358).
// restricted: log norm = log_num - lnGN; free: log of the molecule's norm.
static __global__ void finalize_phi_log(int M, LogConst lc, const double *__restrict__ lG, double *__restrict__ phi,
                                        const MolScal *__restrict__ scal, int mol, int monomer, int restricted,
                                        double log_num) {
    const double lognorm = restricted ? log_num - scal[mol].lngn : log(scal[mol].norm);
    for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < M; z += gridDim.x * blockDim.x) {
        double p;
        if (monomer) p = lG[z];
        else {
            const double g = lG[z], v = phi[z];
            p = (g > SFGPU_LOGZERO && v > SFGPU_LOGZERO) ? v - g : SFGPU_LOGZERO;
        }
        if (p > SFGPU_LOGZERO) p += lognorm;
        phi[z] = restore_from_safe(lc, p);
    }
}

}  // namespace sfk
