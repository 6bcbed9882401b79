/*
 * sfbox_oracle.c -- TEST INFRASTRUCTURE ONLY: the checker for the CUDA
 * library, never linked into it, never the thing measured or shipped.
 *
 * A plain-C restatement of the SFbox 2.1 SF-SCF hot path (lattice
 * propagators, Gf*Gb/G composition, normalisation, segment-potential update,
 * residual, free energy and the Pure_DIIS iteration).  Every function cites
 * the reference lines it follows.  Arrays are 0-based; SFbox's 1-based site
 * z corresponds to index z-1 here.
 *
 * Pinned against SFbox itself: SFbox ships no tests or golden files for this
 * path, so oracle/refbuild builds the reference's own C++ sources (with
 * stand-ins for its absent 'fenk' container library and CLAPACK) and
 * tests/golden/reference_cases.npz holds that build's outputs on one system
 * per lattice family; this file meets them to 1e-13 per evaluation and to
 * 1e-10 (phi) / 1e-9 (F) at convergence.  Known-answer tests derived from the
 * equations check it further.
 *
 * Where SFbox leaves boundary-site values unspecified (3D propagator slices
 * keep stale scratch values on the boundary planes, Lat3D1stO.cpp:151-157;
 * contact averages on mirror boundary rows, Lat2DCylinder.cpp:205-320), this
 * file writes the SetBoundaries copy instead.  Those values never reach an
 * interior residual, lnGN or the free energy.
 */
#include "sfbox_oracle.h"
#include <math.h>
#include <float.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>

/* ------------------------------------------------------------------------ */
/* lattice                                                                   */
/* ------------------------------------------------------------------------ */
typedef struct {
    int grad, cyl, order;
    int n[3];          /* interior layers */
    int Md[3];         /* layers incl. the two boundary layers (1 if unused) */
    int M;
    int st[3];         /* strides, last gradient fastest */
    int bc_lo[3], bc_hi[3];     /* SFGPU_BOUND_* */
    int map_lo[3], map_hi[3];   /* coordinate copied into 0 / Md-1 */
    double l1, l1chi, ladj;
    int sph;           /* 1D curved: spherical (else cylindrical) */
    double off1;       /* 1D curved: offset_first_layer */
    double *lam_m, *lam_p, *Lx; /* curved-lattice tables by 0-based x (0..MX-1) */
    double *lamc_m, *lamc_p;    /* 1D curved: contact tables with lambda_chi */
    double *w_gn;      /* weights of interior sites in lnGN sums */
    double *w_f;       /* weights in the free-energy sum (surfaces included) */
    double *sb;        /* SubtractBoundaries factors: 0 on removed boundary layers, 1/2 on mirror2 layers */
    int K;             /* 2nd-order direction components: 3 (1D), 5 (2D), 6 (3D); 1 first order */
    int sw_lo[3], sw_hi[3];   /* 2nd order: +/- components swap at a boundary copy */
    int ltype;         /* 3D lattice type, SFGPU_LATTICE_* */
    double sl[4];      /* contact weights of the 27-site cube: centre, face, edge, corner */
    /* overflow protection (*1stOS lattices): constants of the log-space steps */
    double *stiff;     /* 'lat : stiff_range' mask (3D second order), NULL if none */
    int logmode;
    double LogL0, LogL1, LogL1L0;          /* flat 1D / 2D */
    double *logl0x, *loglmx, *loglpx;      /* 2D cylinder, by x (0 where lambda <= 0) */
    double logl1, nl_centre;               /* 2D cylinder */
} olat;

static int map_lo_of(int bc, int n) {
    /* Lat1DFlat.cpp:81-88, Lat2DFlat.cpp:140-145, Lat3D.cpp:205-210 */
    switch (bc) {
        case SFGPU_BOUND_SURFACE: return 0;
        case SFGPU_BOUND_MIRROR1: return 1;
        case SFGPU_BOUND_MIRROR2: return 2;
        case SFGPU_BOUND_PERIODIC: return n;
    }
    return -1;
}
static int map_hi_of(int bc, int n) {
    switch (bc) {
        case SFGPU_BOUND_SURFACE: return n + 1;
        case SFGPU_BOUND_MIRROR1: return n;
        case SFGPU_BOUND_MIRROR2: return n - 1;
        case SFGPU_BOUND_PERIODIC: return 1;
    }
    return -1;
}

static void coords(const olat *L, int z, int c[3]) {
    c[0] = c[1] = c[2] = 0;
    if (L->grad == 1) { c[0] = z; return; }
    if (L->grad == 2) { c[0] = z / L->Md[1]; c[1] = z % L->Md[1]; return; }
    c[0] = z / L->st[0]; c[1] = (z % L->st[0]) / L->st[1]; c[2] = z % L->st[1];
}
static int site(const olat *L, const int c[3]) {
    return c[0] * L->st[0] + c[1] * L->st[1] + c[2] * L->st[2];
}
static int is_interior(const olat *L, int z) {
    int c[3]; coords(L, z, c);
    for (int d = 0; d < L->grad; d++) if (c[d] == 0 || c[d] == L->Md[d] - 1) return 0;
    return 1;
}
/* site whose value a boundary site copies (the site itself if interior or on
   a surface); swapmask gets one bit per mirrored gradient */
static int mapped_site(const olat *L, int z, int *swapmask) {
    int c[3]; coords(L, z, c);
    int m = 0;
    for (int d = 0; d < L->grad; d++) {
        if (c[d] == 0) {
            c[d] = L->map_lo[d];
            if (L->bc_lo[d] == SFGPU_BOUND_MIRROR1 || L->bc_lo[d] == SFGPU_BOUND_MIRROR2) m |= 1 << d;
        } else if (c[d] == L->Md[d] - 1) {
            c[d] = L->map_hi[d];
            if (L->bc_hi[d] == SFGPU_BOUND_MIRROR1 || L->bc_hi[d] == SFGPU_BOUND_MIRROR2) m |= 1 << d;
        }
    }
    if (swapmask) *swapmask = m;
    return site(L, c);
}

/* SetBoundaries: Lat1DFlat.cpp:396-399, Lat2DFlat.cpp:619-666, Lat3D.cpp:1510-1562 */
static void olat_set_boundaries(const olat *L, double *P) {
    for (int z = 0; z < L->M; z++) {
        if (is_interior(L, z)) continue;
        int m = mapped_site(L, z, NULL);
        if (m != z) P[z] = P[m];
    }
}

/* direction swap of the 2nd-order components at mirror boundaries,
   Lat3D2ndO.cpp:84-89 with Lat3D.cpp:1276-1290 (k: 0=+x 1=+y 2=+z 3=-z 4=-y 5=-x) */
static void olat_set_boundaries6(const olat *L, double *P) {
    for (int z = 0; z < L->M; z++) {
        if (is_interior(L, z)) continue;
        int sw;
        int m = mapped_site(L, z, &sw);
        if (m == z) continue;
        for (int k = 0; k < 6; k++) {
            int kk = k;
            if (sw & 1) { if (kk == 0) kk = 5; else if (kk == 5) kk = 0; }
            if (sw & 2) { if (kk == 1) kk = 4; else if (kk == 4) kk = 1; }
            if (sw & 4) { if (kk == 2) kk = 3; else if (kk == 3) kk = 2; }
            P[k * L->M + z] = P[kk * L->M + m];
        }
    }
}

static int olat_init(olat *L, const sfgpu_lattice_desc *d) {
    memset(L, 0, sizeof(*L));
    L->grad = d->gradients;
    L->order = d->order;
    /* curved: Lat2DCylinder, Lat1DCylinder, Lat1DSphere (SF_System.cpp:434-519) */
    L->cyl = (d->geometry == SFGPU_GEOM_CYLINDRICAL && (d->gradients == 1 || d->gradients == 2)) ||
             (d->geometry == SFGPU_GEOM_SPHERICAL && d->gradients == 1);
    if (L->grad < 1 || L->grad > 3) return SFGPU_ERR_INVALID;
    if (d->geometry < SFGPU_GEOM_FLAT || d->geometry > SFGPU_GEOM_SPHERICAL) return SFGPU_ERR_INVALID;
    if (d->geometry != SFGPU_GEOM_FLAT && !L->cyl) return SFGPU_ERR_UNSUPPORTED;
    for (int k = 0; k < 3; k++) { L->Md[k] = 1; }
    for (int k = 0; k < L->grad; k++) {
        L->n[k] = d->n_layers[k];
        if (L->n[k] < 1) return SFGPU_ERR_INVALID;
        L->Md[k] = L->n[k] + 2;
        int lo = d->bound_lo[k], hi = d->bound_hi[k];
        if (lo < 1 || lo > 4 || hi < 1 || hi > 4) return SFGPU_ERR_INVALID;
        if ((lo == SFGPU_BOUND_PERIODIC) != (hi == SFGPU_BOUND_PERIODIC)) return SFGPU_ERR_INVALID;
        if (L->grad == 3 && (lo == SFGPU_BOUND_SURFACE || hi == SFGPU_BOUND_SURFACE)) return SFGPU_ERR_INVALID;
        if ((lo == SFGPU_BOUND_MIRROR2 || hi == SFGPU_BOUND_MIRROR2) && L->n[k] < 2) return SFGPU_ERR_INVALID;
        L->bc_lo[k] = lo; L->bc_hi[k] = hi;
        L->map_lo[k] = map_lo_of(lo, L->n[k]);
        L->map_hi[k] = map_hi_of(hi, L->n[k]);
        /* SetBx1(P,Q) / SetBxm(P,Q) swap the two components of an axis when
           the 1-based copy layer is <= 2 (lower side) or >= n - 1 (upper
           side): Lat3D.cpp:1276-1289 (codes mirror1 1, mirror2 2);
           Lat1DFlat.cpp:33-58 and :658-680, Lat2DFlat.cpp:1343-1413 (lower:
           surface 1, mirror1 2, mirror2 3, periodic M-1; upper: M - code + 1,
           periodic 2), i.e. the 0-based copy index map_lo <= 1 or
           map_hi >= n - 2 */
        if (L->grad == 3) {
            L->sw_lo[k] = (lo == SFGPU_BOUND_MIRROR1 || lo == SFGPU_BOUND_MIRROR2);
            L->sw_hi[k] = (hi == SFGPU_BOUND_MIRROR1 || hi == SFGPU_BOUND_MIRROR2);
        } else {
            L->sw_lo[k] = L->map_lo[k] <= 1;
            L->sw_hi[k] = L->map_hi[k] >= L->n[k] - 2;
        }
    }
    L->K = (L->order == 2) ? (L->grad == 1 ? 3 : (L->grad == 2 ? 5 : 6)) : 1;
    L->M = L->Md[0] * L->Md[1] * L->Md[2];
    /* lat : stiff_range, Lat3D.cpp:265-268 (used by second-order copolymers) */
    if (d->stiff_range) {
        if (L->grad != 3) return SFGPU_ERR_INVALID;
        if (L->order == 2) {
            L->stiff = malloc(sizeof(double) * L->M);
            memcpy(L->stiff, d->stiff_range, sizeof(double) * L->M);
        }
    }
    L->st[2] = 1; L->st[1] = L->Md[2]; L->st[0] = L->Md[1] * L->Md[2];
    if (L->grad == 1) { L->st[0] = 1; L->st[1] = L->st[2] = 0; }
    if (L->grad == 2) { L->st[0] = L->Md[1]; L->st[1] = 1; L->st[2] = 0; }
    L->l1 = (L->grad == 3) ? 1.0 / 6.0 : d->lambda;   /* Lat3D.cpp:231-236 */
    /* lattice type and contact weights, Lat3D.cpp:212-259: standard ("BCC")
       l1 = 1/6 and the rest 0, FCC 1/27 everywhere, stencils from the input
       with lambda3 recomputed from the other three */
    L->ltype = d->lattice_type;
    if (L->ltype < SFGPU_LATTICE_STANDARD || L->ltype > SFGPU_LATTICE_HEX) return SFGPU_ERR_INVALID;
    if (L->ltype != SFGPU_LATTICE_STANDARD && L->grad != 3) return SFGPU_ERR_UNSUPPORTED;
    L->sl[0] = 0; L->sl[1] = 1.0 / 6.0; L->sl[2] = 0; L->sl[3] = 0;
    if (L->ltype == SFGPU_LATTICE_FCC) L->sl[0] = L->sl[1] = L->sl[2] = L->sl[3] = 1.0 / 27.0;
    if (L->ltype == SFGPU_LATTICE_STENCILS) {
        double dev;
        for (int k = 0; k < 4; k++) {
            L->sl[k] = d->lambda_3d[k];
            if (!(L->sl[k] >= 0 && L->sl[k] <= 0.5)) return SFGPU_ERR_INVALID;
        }
        dev = fabs(L->sl[0] + 6.0 * L->sl[1] + 12.0 * L->sl[2] + 8.0 * L->sl[3] - 1.0);
        if (dev > DBL_EPSILON) return SFGPU_ERR_INVALID;
        L->sl[3] = (1.0 - L->sl[0] - 6.0 * L->sl[1] - 12.0 * L->sl[2]) / 8.0;
    }
    L->l1chi = (d->lambda_chi >= 0 && L->grad == 1) ? d->lambda_chi : L->l1;
    L->ladj = (L->grad == 1 && d->layer_adjustment > 0) ? d->layer_adjustment : 1.0;

    int MX = L->Md[0];
    if (L->cyl && L->grad == 1) {
        /* Lat1DCylinder::calculateLambdas (Lat1DCylinder.cpp:375-415) and
           Lat1DSphere::calculateLambdas (Lat1DSphere.cpp:240-286), tables
           indexed 1..M there, 0..M-1 here; adjustOuterLayer holds whenever
           layer_adjustment differs from 1 (Lat1DFlat.cpp:139-148) */
        const double PI_ = 4.0 * atan(1.0);
        int sph = d->geometry == SFGPU_GEOM_SPHERICAL;
        double off = d->offset_first_layer;
        L->sph = sph;
        L->off1 = off;
        if (off <= 0 && d->bound_lo[0] == SFGPU_BOUND_SURFACE) return SFGPU_ERR_INVALID;   /* Lat1DCylinder.cpp:50-53 */
        double dim = d->dimensions > 0 ? d->dimensions : 3.0;
        double D = sph ? dim : dim - 1;
        double *V = calloc(MX + 1, sizeof(double)), *S = calloc(MX + 1, sizeof(double));
        double *LL = calloc(MX + 1, sizeof(double));
        double *lm = calloc(MX + 1, sizeof(double)), *lp = calloc(MX + 1, sizeof(double));
        double *lcm = calloc(MX + 1, sizeof(double)), *lcp = calloc(MX + 1, sizeof(double));
        if (sph) { S[1] = off * off * PI_ * 4; V[1] = (4.0 / 3.0) * pow(off, 3) * PI_; }
        else { S[1] = off * PI_ * 2; V[1] = off * off * PI_; }
        LL[1] = V[1];
        for (int z = 2; z <= MX; z++) {
            double x = z + off - 2 + L->ladj;
            if (z == MX - 1 && L->ladj != 1.0) x += -L->ladj + 1;
            V[z] = (PI_ * pow(2, (D - 1)) / D) * pow(x, D);
            LL[z] = V[z] - V[z - 1];
            S[z] = pow(2, (D - 1)) * PI_ * pow(x, (D - 1));
            lm[z] = L->l1 * S[z - 1] / LL[z];
            lp[z] = L->l1 * S[z] / LL[z];
            lcm[z] = L->l1chi * S[z - 1] / LL[z];
            lcp[z] = L->l1chi * S[z] / LL[z];
        }
        if (sph) { if (LL[1] > 4.0 * PI_ / 3.0) LL[1] = V[1] - pow((off - 1), 3) * PI_ * 4.0 / 3.0; }
        else if (LL[1] > PI_) LL[1] = V[1] - (off - 1) * (off - 1) * PI_;
        if (LL[1] > 0) { lp[1] = LL[2] * lm[2] / LL[1]; lcp[1] = LL[2] * lcm[2] / LL[1]; }
        L->lam_m = calloc(MX, sizeof(double)); L->lam_p = calloc(MX, sizeof(double));
        L->lamc_m = calloc(MX, sizeof(double)); L->lamc_p = calloc(MX, sizeof(double));
        L->Lx = calloc(MX, sizeof(double));
        for (int x = 0; x < MX; x++) {
            L->lam_m[x] = lm[x + 1]; L->lam_p[x] = lp[x + 1]; L->Lx[x] = LL[x + 1];
            L->lamc_m[x] = lcm[x + 1]; L->lamc_p[x] = lcp[x + 1];
        }
        free(V); free(S); free(LL); free(lm); free(lp); free(lcm); free(lcp);
    } else if (L->cyl) {
        /* Lat2DCylinder.cpp:7-55 (tables indexed 1..MX there, 0..MX-1 here) */
        const double PI_ = 4.0 * atan(1.0);
        double off = d->offset_first_layer;
        double D = (d->dimensions > 0 ? d->dimensions : 3.0) - 1;
        double ladj = 1.0;
        L->off1 = off;
        double *V = calloc(MX + 1, sizeof(double)), *S = calloc(MX + 1, sizeof(double));
        double *lm = calloc(MX + 1, sizeof(double)), *lp = calloc(MX + 1, sizeof(double));
        double *LL = calloc(MX + 1, sizeof(double));
        S[1] = off * PI_ * 2; V[1] = off * off * PI_; LL[1] = V[1];
        for (int z = 2; z <= MX; z++) {
            double x = z + off - 2 + ladj;
            V[z] = (PI_ * pow(2, (D - 1)) / D) * pow(x, D);
            LL[z] = V[z] - V[z - 1];
            S[z] = pow(2, (D - 1)) * PI_ * pow(x, (D - 1));
            lm[z] = L->l1 * S[z - 1] / LL[z];
            lp[z] = L->l1 * S[z] / LL[z];
        }
        lp[MX] = 0;
        if (LL[1] > PI_) LL[1] = V[1] - (off - 1) * (off - 1) * PI_;
        if (LL[1] > 0) lp[1] = LL[2] * lm[2] / LL[1];
        L->lam_m = calloc(MX, sizeof(double)); L->lam_p = calloc(MX, sizeof(double));
        L->Lx = calloc(MX, sizeof(double));
        for (int x = 0; x < MX; x++) { L->lam_m[x] = lm[x + 1]; L->lam_p[x] = lp[x + 1]; L->Lx[x] = LL[x + 1]; }
        free(V); free(S); free(lm); free(lp); free(LL);
    }

    /* site weights: SubtractBoundaries + MultiplyWithLatticeSites
       (Lat1DFlat.cpp:266-269,410-415; Lat2DFlat.cpp:716-731; Lat2DCylinder.cpp:156-164;
        Lat3D.cpp:1591-1633) */
    L->w_gn = calloc(L->M, sizeof(double));
    L->w_f = calloc(L->M, sizeof(double));
    L->sb = calloc(L->M, sizeof(double));
    /* Lat2DFlat1stO::ComputeLnGN and Lat2DCyl1stO::ComputeLnGN halve the
       1-based column y = MY-2 for an upper mirror2 in y, one layer inside the
       last interior one that SubtractBoundaries halves (Lat2DFlat1stO.cpp:
       321-326, :333-341; Lat2DCyl1stO.cpp:415-437); the lnGN weights follow
       them, the free-energy weights do not */
    const int gn_y_shift = (L->grad == 2 && L->order == 1) ? 1 : 0;
    for (int z = 0; z < L->M; z++) {
        int c[3]; coords(L, z, c);
        double w = 1.0, wg = 1.0; int keep = 1, interior = 1;
        for (int k = 0; k < L->grad; k++) {
            int last = L->Md[k] - 1;
            if (c[k] == 0) { interior = 0; if (L->bc_lo[k] != SFGPU_BOUND_SURFACE) keep = 0; }
            else if (c[k] == last) { interior = 0; if (L->bc_hi[k] != SFGPU_BOUND_SURFACE) keep = 0; }
            else {
                if (c[k] == 1 && L->bc_lo[k] == SFGPU_BOUND_MIRROR2) w *= 0.5;
                else if (c[k] == last - 1 && L->bc_hi[k] == SFGPU_BOUND_MIRROR2) w *= 0.5;
                int hi_gn = last - 1 - (k == 1 ? gn_y_shift : 0);
                if (c[k] == 1 && L->bc_lo[k] == SFGPU_BOUND_MIRROR2) wg *= 0.5;
                else if (c[k] == hi_gn && L->bc_hi[k] == SFGPU_BOUND_MIRROR2) wg *= 0.5;
            }
        }
        L->sb[z] = keep ? w : 0.0;
        if (L->cyl) { w *= L->Lx[c[0]]; wg *= L->Lx[c[0]]; }
        if (L->grad == 1 && !L->cyl) {   /* flat: Lat1DFlat.cpp:266-269 */
            if (z == 1) { w *= L->ladj; wg *= L->ladj; }
            if (z == L->M - 2 && L->M > 3) { w *= (2 - L->ladj); wg *= (2 - L->ladj); }
        }
        L->w_f[z] = keep ? w : 0.0;
        L->w_gn[z] = interior ? wg : 0.0;
        /* Lat1D2ndO::ComputeLnGN: interior sum without mirror2 halves or layer
           adjustment (Lat1D2ndO.cpp:275-285) */
        if (L->order == 2 && L->grad == 1 && !L->cyl) L->w_gn[z] = interior ? 1.0 : 0.0;
    }
    return SFGPU_OK;
}

static void olat_free(olat *L) {
    free(L->lam_m); free(L->lam_p); free(L->lamc_m); free(L->lamc_p); free(L->Lx); free(L->w_gn); free(L->w_f); free(L->sb);
    free(L->logl0x); free(L->loglmx); free(L->loglpx); free(L->stiff);
}

/* one first-order step gout = G * stencil(gin); gin must carry valid
   boundary copies.  Op order as in Lat1DFlat1stO.cpp:37-50,
   Lat2DFlat1stO.cpp:32-53, Lat2DCyl1stO.cpp:17-39, Lat3D1stO.cpp:134-163 */
static void olat_prop1(const olat *L, const double *gin, const double *G, double *gout) {
    int M = L->M;
    for (int z = 0; z < M; z++) {
        if (!is_interior(L, z)) continue;
        double g = G[z], r;
        if (L->grad == 1) {
            double a = gin[z - 1], b = gin[z], c = gin[z + 1];
            if (L->cyl) r = g * (b + L->lam_m[z] * (a - b) + L->lam_p[z] * (c - b));   /* Lat1DCyl1stO.cpp:14-27 */
            else r = g * (b + L->l1 * (a - b - b + c));
        } else if (L->grad == 2) {
            int MY = L->Md[1];
            double a = gin[z - 1], b = gin[z], c = gin[z + 1];
            double u = gin[z - MY], dn = gin[z + MY];
            if (L->cyl) {
                int x = z / MY;
                r = g * (b + L->lam_m[x] * (u - b) + L->lam_p[x] * (dn - b) + L->l1 * (a + c - b - b));
            } else {
                double l0 = 1 - 4 * L->l1;
                r = g * (l0 * b + L->l1 * (a + c) + L->l1 * (u + dn));
            }
        } else if (L->ltype == SFGPU_LATTICE_FCC || L->ltype == SFGPU_LATTICE_HEX) {
            /* Lat3DFCC1stO.cpp:79-92 / Lat3DHEX1stO.cpp:79-92: twelve
               neighbours (dx, dy, dz) summed in this order, then times 1/12 */
            static const int fcc[12][3] = {{-1, -1, 0}, {1, 1, 0}, {-1, 1, 0}, {1, -1, 0},
                                           {0, -1, -1}, {0, 1, 1}, {0, -1, 1}, {0, 1, -1},
                                           {-1, 0, -1}, {1, 0, 1}, {-1, 0, 1}, {1, 0, -1}};
            static const int hex[12][3] = {{-1, 0, 0}, {1, 0, 0}, {-1, 1, 0}, {0, 1, 0},
                                           {0, -1, 0}, {1, -1, 0}, {0, 1, -1}, {0, 0, -1},
                                           {1, 0, -1}, {-1, 0, 1}, {0, 0, 1}, {0, -1, 1}};
            const int (*nb)[3] = (L->ltype == SFGPU_LATTICE_FCC) ? fcc : hex;
            int jx = L->st[0], jy = L->st[1];
            double acc = gin[z + nb[0][0] * jx + nb[0][1] * jy + nb[0][2]] * g;
            for (int k = 1; k < 12; k++) acc += gin[z + nb[k][0] * jx + nb[k][1] * jy + nb[k][2]] * g;
            r = acc * (1.0 / 12.0);
        } else {
            int jx = L->st[0], jy = L->st[1];
            double acc = gin[z - jx] * g;
            acc += gin[z + jx] * g;
            acc += gin[z - jy] * g;
            acc += gin[z + jy] * g;
            acc += gin[z - 1] * g;
            acc += gin[z + 1] * g;
            r = acc * (1.0 / 6.0);
        }
        gout[z] = r;
    }
    /* boundary: copy of the mapped site; surface layers keep their value */
    for (int z = 0; z < M; z++) {
        if (is_interior(L, z)) continue;
        int m = mapped_site(L, z, NULL);
        gout[z] = is_interior(L, m) ? gout[m] : gin[m];
    }
}

/* second-order steps, Lat3D2ndO.cpp:65-152 (forward) and :597-678 (backward) */
static const int OPP[6] = {5, 4, 3, 2, 1, 0};
static void olat_prop2(const olat *L, const double *gin, const double *G, double S,
                       double *gout, int backward) {
    int M = L->M, jx = L->st[0], jy = L->st[1];
    int e[6] = {jx, jy, 1, -1, -jy, -jx};
    double Lw = (1.0 - S) / 4.0;
    for (int z = 0; z < M; z++) {
        if (!is_interior(L, z)) continue;
        double gS = G[z] * S, gL = G[z] * Lw;
        for (int k = 0; k < 6; k++) {
            double acc = 0; int first = 1;
            if (!backward) {
                int src = z - e[k];
                for (int kp = 0; kp < 6; kp++) {
                    if (kp == OPP[k]) continue;
                    double t = gin[kp * M + src] * (kp == k ? gS : gL);
                    if (first) { acc = t; first = 0; } else acc += t;
                }
            } else {
                for (int kp = 5; kp >= 0; kp--) {
                    if (kp == OPP[k]) continue;
                    double t = gin[kp * M + z + e[kp]] * (kp == k ? gS : gL);
                    if (first) { acc = t; first = 0; } else acc += t;
                }
            }
            gout[k * M + z] = acc;
        }
    }
    olat_set_boundaries6(L, gout);
}

/* one constant-force step (mol : force), Lat1DFlat1stO.cpp:116-130,
   Lat1DCyl1stO.cpp:112-133 (the sphere inherits it), Lat2DCyl1stO.cpp:100-126,
   Lat3D1stO.cpp:94-130; gin carries boundary copies */
static void olat_prop1_force(const olat *L, const double *gin, const double *G, double *gout, double f) {
    int M = L->M;
    double l1 = L->l1;
    for (int z = 0; z < M; z++) {
        if (!is_interior(L, z)) continue;
        double g = G[z], r;
        if (L->grad == 1 && !L->cyl) {
            double norm = l1 * (exp(-f) + exp(f) - 2) + 1;
            double f_1 = l1 * exp(-f) / norm, f1 = l1 * exp(f) / norm;
            double a = gin[z - 1], b = gin[z], c = gin[z + 1];
            r = g * (b + f1 * (a - b) + f_1 * (c - b));
        } else if (L->grad == 1) {
            double f_1 = exp(f), f1 = exp(-f);
            double fnorm = (4.0 + f1 + f_1) / 6.0;
            f1 = f1 / fnorm; f_1 = f_1 / fnorm;
            double f1z = L->lam_p[z] * f1, f_1z = L->lam_m[z] * f_1, f0z = (1 - L->lam_p[z] - L->lam_m[z]) / fnorm;
            r = g * (f_1z * gin[z - 1] + f0z * gin[z] + f1z * gin[z + 1]);
        } else if (L->grad == 2) {
            int MY = L->Md[1], x = z / MY;
            double f_1 = exp(-f), f1 = exp(f), norm = l1 * (f_1 + f1 - 2) + 1;
            double a = gin[z - 1], b = gin[z], c = gin[z + 1];
            r = g * (b + L->lam_m[x] * (gin[z - MY] - b) + L->lam_p[x] * (gin[z + MY] - b) + l1 * (a * f1 + c * f_1 - b - b)) / norm;
        } else {
            int jx = L->st[0], jy = L->st[1];
            double f1 = exp(f), f_1 = exp(-f), fnorm = 1.0 / (4.0 + exp(f) + exp(-f));
            double acc = gin[z - jx] * g;
            acc += gin[z + jx] * g;
            acc += gin[z - jy] * g;
            acc += gin[z + jy] * g;
            acc += gin[z - 1] * g * f1;
            acc += gin[z + 1] * g * f_1;
            r = acc * fnorm;
        }
        gout[z] = r;
    }
    for (int z = 0; z < M; z++) {
        if (is_interior(L, z)) continue;
        int m = mapped_site(L, z, NULL);
        gout[z] = is_interior(L, m) ? gout[m] : gin[m];
    }
}

/* the stiff_range and isotropic 3D second-order steps of
   SF_Copol2ndO_stiff_range: PropagateF/B(..., S, stiff) (Lat3D2ndO.cpp:155-247,
   :680-764) weigh with ps = S inside the range and 0.2 outside, pl = (1-ps)/4,
   taken at the unshifted index of each array operation (the source site for
   the + components forward and for reads of the - components backward, the
   target site otherwise), as (Gi * G) * p; PropagateF/B(Gi, G) (:250-344,
   :765-850) weigh all six components with G/6, the forward -y component
   reading +z twice and -y not at all (:308-313). */
static void olat_prop2_var(const olat *L, const double *gin, const double *G, double S,
                           double *gout, int backward, int iso) {
    int M = L->M, jx = L->st[0], jy = L->st[1];
    int e[6] = {jx, jy, 1, -1, -jy, -jx};
    static const int seq[6] = {0, 1, 2, 3, 4, 5}, seq4[6] = {0, 2, 2, 3, 4, 5};
    for (int z = 0; z < M; z++) {
        if (!is_interior(L, z)) continue;
        double gI = G[z] * (1.0 / 6.0);
        for (int k = 0; k < 6; k++) {
            double acc = 0; int first = 1;
            if (!backward) {
                int src = z - e[k];
                if (iso) {
                    const int *q = (k == 4) ? seq4 : seq;
                    for (int i = 0; i < 6; i++) {
                        double t = gin[q[i] * M + src] * gI;
                        if (first) { acc = t; first = 0; } else acc += t;
                    }
                } else {
                    int pi = (k < 3) ? src : z;
                    double ps = (L->stiff[pi] != 0) ? S : 0.2, pl = (1.0 - ps) / 4.0;
                    for (int kp = 0; kp < 6; kp++) {
                        if (kp == OPP[k]) continue;
                        double t = gin[kp * M + src] * G[z] * (kp == k ? ps : pl);
                        if (first) { acc = t; first = 0; } else acc += t;
                    }
                }
            } else {
                for (int kp = 5; kp >= 0; kp--) {
                    double t;
                    if (iso) t = gin[kp * M + z + e[kp]] * gI;
                    else {
                        if (kp == OPP[k]) continue;
                        int pi = (kp >= 3) ? z + e[kp] : z;
                        double ps = (L->stiff[pi] != 0) ? S : 0.2, pl = (1.0 - ps) / 4.0;
                        t = gin[kp * M + z + e[kp]] * G[z] * (kp == k ? ps : pl);
                    }
                    if (first) { acc = t; first = 0; } else acc += t;
                }
            }
            gout[k * M + z] = acc;
        }
    }
    olat_set_boundaries6(L, gout);
}

/* 2nd-order steps of the flat 1D and 2D lattices, whose homogeneous
   gradients lump their bond directions: Lat1D2ndO (k: 0 = +x, 1 = lateral x4,
   2 = -x), Lat1D2ndO.cpp:33-147; Lat2D2ndO (0 = +x, 1 = +y, 2 = z x2, 3 = -y,
   4 = -x), Lat2D2ndO.cpp:32-230.  Boundary copies first (SetBx1/SetBxm/
   SetBy1/SetBym on the input, swapping the two components of an axis where
   the lattice does), then gx[kk](z) = sum_kp W[kk][kp] gin[kp](z - e_kk)
   forward, gx[kq](z) = sum_kp W[kq][kp] gin[kp](z + e_kp) backward, times
   G(z).  W: S for the same direction (+2L for the 1D lateral group), 0 for
   the opposite one, mult[kp] L otherwise. */
static const int LUMP_AXIS[2][5] = {{0, -1, 0, -1, -1}, {0, 1, -1, 1, 0}};
static const int LUMP_SGN[2][5] = {{1, 0, -1, 0, 0}, {1, 1, 0, -1, -1}};
static const double LUMP_MULT[2][5] = {{1, 4, 1, 0, 0}, {1, 1, 2, 1, 1}};
static double lump_w(int g, int kk, int kp, double S, double Lw) {
    if (kk == kp) return (g == 0 && kk == 1) ? S + 2 * Lw : S;
    if (LUMP_AXIS[g][kk] >= 0 && LUMP_AXIS[g][kk] == LUMP_AXIS[g][kp] && LUMP_SGN[g][kk] == -LUMP_SGN[g][kp]) return 0.0;
    return LUMP_MULT[g][kp] * Lw;
}
/* one SetBx1 / SetBxm / SetBy1 / SetBym call (Lat1DFlat.cpp:654-681,
   Lat2DFlat.cpp:1336-1413) on the boundary line of axis a (upper side when
   hi): every entry of P (and Q) on the line copies the copy layer's; where
   the side swaps, P = Q' then Q = P' site by site, so at a surface (the
   boundary is its own copy layer) both end with Q's value */
static void lump_setb(const olat *L, double *P, double *Q, int a, int hi) {
    int b = hi ? L->Md[a] - 1 : 0;
    int src = hi ? L->map_hi[a] : L->map_lo[a];
    int sw = hi ? L->sw_hi[a] : L->sw_lo[a];
    for (int z = 0; z < L->M; z++) {
        int c[3]; coords(L, z, c);
        if (c[a] != b) continue;
        c[a] = src;
        int zs = site(L, c);
        if (Q && sw) { P[z] = Q[zs]; Q[z] = P[zs]; }
        else { P[z] = P[zs]; if (Q) Q[z] = Q[zs]; }
    }
}
/* the boundary calls of Lat1D2ndO::PropagateF/B (Lat1D2ndO.cpp:43-44):
   SetBx1(g0,g2) SetBx1(g1) SetBxm(g0,g2) SetBxm(g1); of Lat2D2ndO
   (Lat2D2ndO.cpp:48-51): x below on (g0,g4) then g1..g3, y below on (g1,g3)
   then g0, g2, g4, x above, y above */
static void olat_set_boundaries_lumped(const olat *L, double *P) {
    size_t M = (size_t)L->M;
    double *g[5];
    for (int k = 0; k < L->K; k++) g[k] = P + k * M;
    for (int hi = 0; hi < 2; hi++) {
        if (L->grad == 1) {
            lump_setb(L, g[0], g[2], 0, hi);
            lump_setb(L, g[1], NULL, 0, hi);
        } else {
            lump_setb(L, g[0], g[4], 0, hi);
            for (int k = 1; k <= 3; k++) lump_setb(L, g[k], NULL, 0, hi);
            lump_setb(L, g[1], g[3], 1, hi);
            lump_setb(L, g[0], NULL, 1, hi);
            lump_setb(L, g[2], NULL, 1, hi);
            lump_setb(L, g[4], NULL, 1, hi);
        }
    }
}
/* the opposite radial direction of component kp (kp itself off the radial axis) */
static int lump_refl(int g, int kp) {
    if (LUMP_AXIS[g][kp] != 0) return kp;
    return (LUMP_SGN[g][kp] > 0) ? (g == 0 ? 2 : 4) : 0;
}
/* Curved lattices (Lat1DCyl2ndO.cpp:52-95 and :149-186, Lat1DSphere2ndO the
   same with spherical tables, Lat2DCyl2ndO.cpp:45-115 and :180-249): a
   radial read of component kp one layer away is the mixture
   f * g_kp(neighbour) + (1 - f) * g_refl(kp)(z) (LReflect / UReflect), with
   f = 6 lambda_-(x) for a read from the inner layer and 6 lambda_+(x) for
   one from the outer layer.  Forward steps mix every radial read; the 2D
   cylinder's backward step mixes only the reads of -x (its UReflect of +x is
   computed and not used, Lat2DCyl2ndO.cpp:203-207), the 1D backward both. */
static void olat_prop2l(const olat *L, const double *gin_, const double *G, double S, double *gout, int backward) {
    int g = L->grad - 1, K = L->K, M = L->M;
    int e[2] = {L->st[0], L->grad == 2 ? L->st[1] : 0};
    double Lw = (1.0 - S) / 4.0;
    double *gin = malloc(sizeof(double) * K * M);
    memcpy(gin, gin_, sizeof(double) * K * M);
    olat_set_boundaries_lumped(L, gin);
    for (int z = 0; z < M; z++) {
        if (!is_interior(L, z)) continue;
        int x = z / L->st[0];   /* radial coordinate */
        for (int kk = 0; kk < K; kk++) {
            double acc = 0; int first = 1;
            for (int kp = 0; kp < K; kp++) {
                double w = lump_w(g, kk, kp, S, Lw);
                if (w == 0.0) continue;
                int src, dir;   /* dir: +1 read from the outer layer, -1 from the inner, 0 no radial mixing */
                if (!backward) {
                    src = (LUMP_AXIS[g][kk] >= 0) ? z - LUMP_SGN[g][kk] * e[LUMP_AXIS[g][kk]] : z;
                    dir = (LUMP_AXIS[g][kk] == 0) ? -LUMP_SGN[g][kk] : 0;
                } else {
                    src = (LUMP_AXIS[g][kp] >= 0) ? z + LUMP_SGN[g][kp] * e[LUMP_AXIS[g][kp]] : z;
                    dir = (LUMP_AXIS[g][kp] == 0 && (g == 0 || LUMP_SGN[g][kp] < 0)) ? LUMP_SGN[g][kp] : 0;
                }
                double v = gin[(size_t)kp * M + src];
                if (L->cyl && dir != 0) {
                    double f = 6 * ((dir > 0) ? L->lam_p[x] : L->lam_m[x]);
                    double fc = 1.0 - f;
                    v = f * v + fc * gin[(size_t)lump_refl(g, kp) * M + z];
                }
                double t = w * v;
                if (first) { acc = t; first = 0; } else acc += t;
            }
            gout[(size_t)kk * M + z] = acc * G[z];
        }
    }
    /* boundary entries: surface layers keep their (boundary-set) value, 0
       for a propagator; the others copy as the next step's SetB calls do */
    for (int z = 0; z < M; z++)
        if (!is_interior(L, z) && mapped_site(L, z, NULL) == z)
            for (int k = 0; k < K; k++) gout[(size_t)k * M + z] = gin[(size_t)k * M + z];
    olat_set_boundaries_lumped(L, gout);
    free(gin);
}
static double comp_mult(int K, int k) {
    if (K == 3 && k == 1) return 4.0;
    if (K == 5 && k == 2) return 2.0;
    return 1.0;
}

/* lnGN of an end-point distribution: Lat1DFlat1stO.cpp:301-316,
   Lat2DFlat1stO.cpp:293-342, Lat2DCyl1stO.cpp:388-438, Lat3D1stO.cpp:344-370,
   Lat3D2ndO.cpp:995-1025 (sum of the six components over 6) */
static double olat_lngn(const olat *L, const double *G) {
    double v = 0;
    int K = L->K;
    for (int k = 0; k < K; k++) {
        double mu = comp_mult(K, k);
        for (int z = 0; z < L->M; z++)
            v += (mu == 1.0) ? L->w_gn[z] * G[k * L->M + z] : L->w_gn[z] * (G[k * L->M + z] * mu);
    }
    if (K > 1) v /= 6.0;   /* six bond directions, lumped or not */
    return log(v);
}

/* contact average <phi>: Lat1DFlat.cpp:511-524, Lat2DFlat.cpp:996-1109,
   Lat2DCylinder.cpp:205-320 (surface rows drop the missing neighbour),
   Lat3D.cpp:1729-1785 (Sides, boundary values removed) */
static void olat_side(const olat *L, const double *phi_in, double *rho) {
    int M = L->M;
    double *p = malloc(sizeof(double) * M);
    memcpy(p, phi_in, sizeof(double) * M);
    olat_set_boundaries(L, p);   /* SF_SegmentList.cpp:524-525 */
    double l = L->l1chi;
    for (int z = 0; z < M; z++) {
        int c[3]; coords(L, z, c);
        if (L->grad == 3) {
            if (!is_interior(L, z)) { rho[z] = 0; continue; }
            int jx = L->st[0], jy = L->st[1];
            if (L->ltype == SFGPU_LATTICE_HEX) {
                /* Lat3D.cpp:1733-1752: the twelve HEX neighbours, 1/12 each
                   (boundary values, which no sum reads, set to 0 here) */
                static const int hx[12][3] = {{1, 0, 0}, {-1, 0, 0}, {1, -1, 0}, {0, -1, 0},
                                              {0, 1, 0}, {-1, 1, 0}, {0, -1, 1}, {0, 0, 1},
                                              {-1, 0, 1}, {1, 0, -1}, {0, 0, -1}, {0, 1, -1}};
                double l = 1.0 / 12.0, acc = p[z + hx[0][0] * jx + hx[0][1] * jy + hx[0][2]] * l;
                for (int k = 1; k < 12; k++) acc += p[z + hx[k][0] * jx + hx[k][1] * jy + hx[k][2]] * l;
                rho[z] = acc;
                continue;
            }
            /* Lat3D.cpp:1765-1778: the 27-site cube in the order centre,
               faces, edges, corners (standard: only the faces weigh) */
            static const int cube[27][4] = {
                {0, 0, 0, 0},
                {1, 0, 0, 1}, {-1, 0, 0, 1}, {0, 1, 0, 1}, {0, -1, 0, 1}, {0, 0, 1, 1}, {0, 0, -1, 1},
                {1, 1, 0, 2}, {1, -1, 0, 2}, {-1, 1, 0, 2}, {-1, -1, 0, 2},
                {1, 0, 1, 2}, {1, 0, -1, 2}, {-1, 0, 1, 2}, {-1, 0, -1, 2},
                {0, 1, 1, 2}, {0, 1, -1, 2}, {0, -1, 1, 2}, {0, -1, -1, 2},
                {1, 1, 1, 3}, {1, 1, -1, 3}, {1, -1, 1, 3}, {1, -1, -1, 3},
                {-1, 1, 1, 3}, {-1, 1, -1, 3}, {-1, -1, 1, 3}, {-1, -1, -1, 3}};
            double acc = p[z] * L->sl[0];
            for (int k = 1; k < 27; k++) {
                double w = L->sl[cube[k][3]];
                if (w == 0) continue;   /* adding +0 products changes no sum */
                acc += p[z + cube[k][0] * jx + cube[k][1] * jy + cube[k][2]] * w;
            }
            rho[z] = acc;
            continue;
        }
        if (L->grad == 1 && L->cyl) {
            /* Lat1DCylinder::SideFraction (Lat1DCylinder.cpp:159-171) */
            int zz = z;
            if (z == 0) {
                if (L->bc_lo[0] == SFGPU_BOUND_SURFACE) { rho[z] = p[0] + L->lamc_p[0] * (-p[0] - p[0] + p[1]); continue; }
                zz = L->map_lo[0];
            } else if (z == M - 1) {
                if (L->bc_hi[0] == SFGPU_BOUND_SURFACE) { rho[z] = p[z] + L->lamc_m[z] * (-p[z] - p[z] + p[z - 1]); continue; }
                zz = L->map_hi[0];
            }
            rho[z] = p[zz] + L->lamc_p[zz] * (p[zz + 1] - p[zz]) + L->lamc_m[zz] * (p[zz - 1] - p[zz]);
            continue;
        }
        if (L->grad == 1) {
            int zz = z;
            if (z == 0) {
                if (L->bc_lo[0] == SFGPU_BOUND_SURFACE) { rho[z] = p[0] + l * (-p[0] - p[0] + p[1]); continue; }
                zz = L->map_lo[0];
            } else if (z == M - 1) {
                if (L->bc_hi[0] == SFGPU_BOUND_SURFACE) { rho[z] = p[z] + l * (-p[z] - p[z] + p[z - 1]); continue; }
                zz = L->map_hi[0];
            }
            rho[z] = p[zz] + l * (p[zz - 1] - p[zz] - p[zz] + p[zz + 1]);
            continue;
        }
        /* 2 gradients */
        int MX = L->Md[0], MY = L->Md[1];
        int onsurf = 0;
        if ((c[0] == 0 && L->bc_lo[0] == SFGPU_BOUND_SURFACE) || (c[0] == MX - 1 && L->bc_hi[0] == SFGPU_BOUND_SURFACE) ||
            (c[1] == 0 && L->bc_lo[1] == SFGPU_BOUND_SURFACE) || (c[1] == MY - 1 && L->bc_hi[1] == SFGPU_BOUND_SURFACE))
            onsurf = 1;
        int x = c[0], zz = z;
        if (!onsurf) zz = mapped_site(L, z, NULL), x = zz / MY;
        double lm = L->cyl ? L->lam_m[x] : l, lp = L->cyl ? L->lam_p[x] : l;
        double l0 = 1 - 2 * l - lm - lp;
        if (!onsurf) {
            if (L->cyl)
                rho[z] = p[zz] + lp * (p[zz + MY] - p[zz]) + lm * (p[zz - MY] - p[zz]) + l * (p[zz - 1] + p[zz + 1] - p[zz] - p[zz]);
            else
                rho[z] = l0 * p[zz] + l * (p[zz - MY] + p[zz + MY]) + l * (p[zz - 1] + p[zz + 1]);
        } else {
            double acc = l0 * p[z];
            if (c[0] > 0) acc += lm * p[z - MY];
            if (c[0] < MX - 1) acc += lp * p[z + MY];
            if (c[1] > 0) acc += l * p[z - 1];
            if (c[1] < MY - 1) acc += l * p[z + 1];
            rho[z] = acc;
        }
    }
    free(p);
}

/* ------------------------------------------------------------------------ */
/* system                                                                    */
/* ------------------------------------------------------------------------ */
typedef struct {
    int N, type;          /* type: 0 monomer, 1 homopolymer, 2 copolymer */
    int *seg;             /* segment of each chain position, N entries */
    int freedom;
    double phibulk, theta;
    int nseg_used;        /* number of distinct segments */
    int *used;            /* list of distinct segments */
    int *count;           /* per segment (n_segments): occurrences */
    int pinned;
    double lngn, lnc, chemintref;
    double *phi;          /* n_segments * M (only used ones nonzero) */
    double *ori;          /* 2nd order: n_segments * 3 * M bond-orientation slots */
    /* symmetric dendrimer: generations (segments of each position, first =
       branch point) and functionalities; nshort positions centre to end */
    int ngen, nshort;
    int *gen_len, *gen_rep, *gen_seg;   /* gen_seg: positions of all generations in order */
    double force;         /* mol : force, constant-force ensemble */
    /* branched molecule: parent of every segment (parent[0] = -1) */
    int tree;
    int *parent;
    /* homopolymer ring (SF_HomoRing1stO) and its free return weight NORM[0] */
    int ring;
    double ring_norm0;
} omol;

struct orc_system {
    olat L;
    int nseg;
    int *freedom;
    double *range;        /* nseg*M (zeros for free) */
    double *chi, *pf;
    int nmol, solvent;
    omol *mol;
    /* iteration variables, SF_Solve.cpp:37-163 */
    int nliq, nclass;
    int *stateQ;          /* liquid states in SFbox's reordered order */
    int *class_of;        /* per segment, -1 for frozen */
    int *rep_of_class;    /* last state of each class (SF_Solve.cpp:563-564) */
    int nsites; int *sites;
    int nvar;
    /* work */
    double *swf_full;     /* nseg*M, state level G = exp(-x) */
    double *swf;          /* nseg*M, segment level (pinned mask) */
    double *phi;          /* nseg*M, state phi */
    double *rho;          /* nseg*M */
    double *phib;         /* nseg */
    int evaluated;
    /* charges (SF_Solve.cpp:164-177, :527-591, :794-852): valence and
       relative dielectric constant per segment; psi joins the iteration
       variables on the sites of PotItVar (SF_Solve.cpp:1761-1776) */
    int charged, diffeps, neutralizer;
    double *val, *eps;
    double bondlength, sitedist, temperature;
    int *xu, *xp;         /* per site: offset of its first u / of its psi in x, -1 if none */
    double *psi0, *psi, *esq, *lsites;
};

/* physical constants of SF_Box.h:37-43 */
#define ORC_BOLTZMANN 1.38065812e-23
#define ORC_EPS0 8.85418785e-12
#define ORC_ELEM_CHARGE 1.6021773349e-19

static int chi_rows_equal(const orc_system *s, int a, int b) {
    for (int i = 0; i < s->nseg; i++)
        if (s->chi[i * s->nseg + a] != s->chi[i * s->nseg + b]) return 0;
    return 1;
}

static int olat_init_log(olat *L);

int orc_create(const sfgpu_system_desc *d, orc_system **out) {
    *out = NULL;
    orc_system *s = calloc(1, sizeof(orc_system));
    int rc = olat_init(&s->L, &d->lattice);
    if (rc) { free(s); return rc; }
    if (d->overflow_protection && (rc = olat_init_log(&s->L))) { olat_free(&s->L); free(s); return rc; }
    int M = s->L.M, ns = d->n_segments;
    s->nseg = ns;
    s->freedom = calloc(ns, sizeof(int));
    s->range = calloc((size_t)ns * M, sizeof(double));
    s->chi = calloc((size_t)ns * ns, sizeof(double));
    s->pf = calloc((size_t)ns * ns, sizeof(double));
    s->val = calloc(ns, sizeof(double));
    s->eps = calloc(ns, sizeof(double));
    s->neutralizer = -1;
    for (int i = 0; i < ns; i++) {
        s->freedom[i] = d->segments[i].freedom;
        if (s->freedom[i] != SFGPU_SEG_FREE && d->segments[i].range)
            memcpy(s->range + (size_t)i * M, d->segments[i].range, sizeof(double) * M);
        s->val[i] = d->segments[i].valence;
        s->eps[i] = d->segments[i].epsilon != 0 ? d->segments[i].epsilon : 80.0;   /* SF_Segment.cpp:170 */
        if (s->val[i] != 0) s->charged = 1;
        for (int j = 0; j < ns; j++) {
            s->chi[i * ns + j] = d->chi ? d->chi[i * ns + j] : 0.0;
            s->pf[i * ns + j] = d->pf ? d->pf[i * ns + j] : 0.2;
        }
    }
    s->bondlength = d->lattice.bondlength > 0 ? d->lattice.bondlength : 3e-10;   /* Lat1DFlat.cpp:128 */
    {   /* the site distance: bondlength / sqrt(2 dimensions lambda) on the 1D and
           2D lattices (Lat1DFlat.cpp:129, Lat2DFlat.cpp:209), the bondlength in
           3D (Lat3D.cpp:263) */
        const double dims = d->lattice.dimensions > 0 ? d->lattice.dimensions : 3.0;
        s->sitedist = s->L.grad == 3 ? s->bondlength : s->bondlength / sqrt(2 * dims * s->L.l1);
    }
    s->temperature = d->temperature > 0 ? d->temperature : 298.15;              /* SF_System.cpp:68 */
    for (int i = 0; i < ns; i++)   /* epsilon differs among liquid states (SF_Solve.cpp:154-162) */
        for (int j = 0; j < ns; j++)
            if (s->charged && s->freedom[i] != SFGPU_SEG_FROZEN && s->freedom[j] != SFGPU_SEG_FROZEN &&
                s->eps[i] != s->eps[j]) s->diffeps = 1;
    /* molecules */
    s->nmol = d->n_molecules;
    s->mol = calloc(s->nmol, sizeof(omol));
    s->solvent = -1;
    for (int m = 0; m < s->nmol; m++) {
        const sfgpu_molecule_desc *md = &d->molecules[m];
        omol *o = &s->mol[m];
        int N = 0;
        for (int b = 0; b < md->n_blocks; b++) N += md->block_length[b];
        if (N < 1) { orc_destroy(s); return SFGPU_ERR_INVALID; }
        o->N = N; o->seg = calloc(N, sizeof(int)); o->count = calloc(ns, sizeof(int));
        int p = 0;
        for (int b = 0; b < md->n_blocks; b++)
            for (int q = 0; q < md->block_length[b]; q++) o->seg[p++] = md->block_segment[b];
        for (int q = 0; q < N; q++) {
            if (o->seg[q] < 0 || o->seg[q] >= ns || s->freedom[o->seg[q]] == SFGPU_SEG_FROZEN) {
                orc_destroy(s); return SFGPU_ERR_INVALID;
            }
            o->count[o->seg[q]]++;
        }
        o->used = calloc(ns, sizeof(int));
        for (int i = 0; i < ns; i++) if (o->count[i]) {
            o->used[o->nseg_used++] = i;
            if (s->freedom[i] == SFGPU_SEG_PINNED) o->pinned = 1;
        }
        if (md->n_generations > 0) {
            /* symmetric dendrimer, SF_MolStructure.cpp:348-359, :552-595, :847-877 */
            int G = md->n_generations, b = 0, pos = 0;
            if (s->L.order != 1) { orc_destroy(s); return SFGPU_ERR_UNSUPPORTED; }
            o->ngen = G;
            o->gen_len = calloc(G, sizeof(int)); o->gen_rep = calloc(G, sizeof(int));
            o->gen_seg = calloc(N, sizeof(int));
            for (int i = 0; i < G; i++) {
                int nb = md->generation_blocks[i];
                if (nb < 1 || b + nb > md->n_blocks || md->generation_repeat[i] < 1) { orc_destroy(s); return SFGPU_ERR_INVALID; }
                for (int q = b; q < b + nb; q++)
                    for (int r = 0; r < md->block_length[q]; r++) { o->gen_seg[pos++] = md->block_segment[q]; o->gen_len[i]++; }
                b += nb;
                o->gen_rep[i] = md->generation_repeat[i];
            }
            if (b != md->n_blocks) { orc_destroy(s); return SFGPU_ERR_INVALID; }
            o->nshort = pos;
            long long Lm = 0;
            for (int i = G - 1; i >= 0; i--) Lm = (Lm + o->gen_len[i] - 1) * o->gen_rep[i] + 1;
            int off[64];
            if (G > 64) { orc_destroy(s); return SFGPU_ERR_INVALID; }
            off[0] = 0;
            for (int i = 1; i < G; i++) off[i] = off[i - 1] + o->gen_len[i - 1];
            for (int sg = 0; sg < ns; sg++) {
                long long num = 0;
                for (int i = G - 1; i >= 0; i--) {
                    long long n = 0;
                    for (int q = 0; q < o->gen_len[i]; q++) n += (o->gen_seg[off[i] + q] == sg);
                    num = (o->gen_seg[off[i]] == sg) ? (num + n - 1) * o->gen_rep[i] + 1 : (num + n) * o->gen_rep[i];
                }
                o->count[sg] = (int)num;
            }
            N = (int)Lm;
            o->N = N;
            if (N == 1) o->ngen = 0;
        }
        if (md->bond_parent) {
            /* branched: SF_ParserBranched::FillLinks (SF_ParserBranched.cpp:43-60) as a
               parent per segment */
            if (o->ngen || s->L.order != 1 || s->L.logmode) { orc_destroy(s); return SFGPU_ERR_UNSUPPORTED; }
            if (md->bond_parent[0] != -1) { orc_destroy(s); return SFGPU_ERR_INVALID; }
            o->parent = calloc(N, sizeof(int));
            o->parent[0] = -1;
            for (int q = 1; q < N; q++) {
                if (md->bond_parent[q] < 0 || md->bond_parent[q] >= q) { orc_destroy(s); return SFGPU_ERR_INVALID; }
                o->parent[q] = md->bond_parent[q];
            }
            o->tree = (N > 1);
        }
        o->type = (N == 1) ? 0 : (o->nseg_used == 1 && !o->ngen && !o->tree ? 1 : 2);
        o->freedom = md->freedom; o->phibulk = md->phibulk; o->theta = md->theta;
        if (md->ring) {
            /* SF_MolList1stO.cpp:28-38; SF_HomoRing1stO.cpp:110-160 on the 1D flat
               lattice, free rings of even length */
            if (o->type != 1 || N % 2 || s->L.order != 1 || s->L.grad != 1 || s->L.cyl || s->L.logmode ||
                o->freedom != SFGPU_MOL_FREE || o->pinned) { orc_destroy(s); return SFGPU_ERR_UNSUPPORTED; }
            int h = N / 2;
            double *X = calloc(2 * h + 1, sizeof(double));
            #define XAT(z) X[(z) + h]
            XAT(0) = 1;
            for (int st = 1; st < h; st++) {
                double a = 0, b = XAT(-st - 1), c = XAT(-st);
                for (int z = -st; z < st; z++) { a = b; b = c; c = XAT(z + 1); XAT(z) = (a + 4.0 * b + c) / 6.0; }
            }
            double n0 = 0;
            for (int z = -h; z < h; z++) n0 += XAT(z) * XAT(z);
            #undef XAT
            free(X);
            o->ring_norm0 = n0;
            o->ring = 1;
        }
        o->force = (o->type == 0) ? 0.0 : md->force;
        if (o->force != 0) {
            /* copolymers only (SF_Homopol1stO.cpp:24-27, SF_Dend1stO.cpp:11-14);
               no step on the 2D flat lattice (Lat2DFlat1stO.cpp:115-117) */
            if (s->L.order != 1 || o->type != 2 || o->ngen || o->tree || (s->L.grad == 2 && !s->L.cyl) ||
                s->L.ltype != SFGPU_LATTICE_STANDARD || s->L.logmode) { orc_destroy(s); return SFGPU_ERR_UNSUPPORTED; }
        }
        if (o->freedom == SFGPU_MOL_SOLVENT) {
            if (s->solvent >= 0) { orc_destroy(s); return SFGPU_ERR_INVALID; }
            s->solvent = m;
        }
        if (o->freedom == SFGPU_MOL_NEUTRALIZER) {
            /* SF_Molecule.cpp:110-126; SF_MolList1stO.cpp:250-266 */
            if (s->neutralizer >= 0 || !s->charged) { orc_destroy(s); return SFGPU_ERR_INVALID; }
            s->neutralizer = m;
        }
        /* chemIntRef, SF_MolStructure.cpp:411-423 */
        double cr = 0;
        for (int a = 0; a < o->nseg_used; a++) {
            int i = o->used[a];
            double inner = 0;
            for (int bb = 0; bb < o->nseg_used; bb++) {
                int j = o->used[bb];
                inner += s->chi[i * ns + j] * ((double)o->count[j] / N);
            }
            cr += ((double)o->count[i] / N) * inner;
        }
        o->chemintref = cr / 2;
        o->phi = calloc((size_t)ns * M, sizeof(double));
        o->ori = calloc((size_t)ns * 3 * M, sizeof(double));
    }
    if (s->solvent < 0) { orc_destroy(s); return SFGPU_ERR_INVALID; }
    if (s->L.stiff)   /* SF_MolList2ndO.cpp:39: only copolymers take a stiff range */
        for (int m = 0; m < s->nmol; m++) {
            if (s->mol[m].type == 1) { orc_destroy(s); return SFGPU_ERR_UNSUPPORTED; }
            /* palindromic copolymers take SF_Copol2ndO_stiff_range::SymMatrix1
               (SF_Copol2ndO_stiff_range.cpp:97-99, :407-452): not restated */
            const omol *o = &s->mol[m];
            int pal = o->type == 2 && o->ngen == 0;
            for (int q = 0; pal && q < o->N / 2; q++) pal = o->seg[q] == o->seg[o->N - 1 - q];
            if (pal) { orc_destroy(s); return SFGPU_ERR_UNSUPPORTED; }
        }

    /* liquid states and their classes, SF_Solve.cpp:37-86 */
    s->stateQ = calloc(ns, sizeof(int));
    s->class_of = calloc(ns, sizeof(int));
    s->rep_of_class = calloc(ns, sizeof(int));
    for (int i = 0; i < ns; i++) if (s->freedom[i] != SFGPU_SEG_FROZEN) s->stateQ[s->nliq++] = i;
    for (int i = 0; i < s->nliq; i++) {
        int s1 = s->stateQ[i];
        for (int j = i + 1; j < s->nliq; j++) {
            if (chi_rows_equal(s, s1, s->stateQ[j])) {
                if (j != i + 1) { int t = s->stateQ[i + 1]; s->stateQ[i + 1] = s->stateQ[j]; s->stateQ[j] = t; }
                i++;
            }
        }
    }
    for (int i = 0; i < ns; i++) s->class_of[i] = -1;
    s->nclass = 0;
    for (int i = 0; i < s->nliq; i++) {
        int s1 = s->stateQ[i];
        int c = s->nclass++;
        s->class_of[s1] = c; s->rep_of_class[c] = s1;
        for (int j = i + 1; j < s->nliq; j++) {
            if (chi_rows_equal(s, s1, s->stateQ[j])) {
                i++; s->class_of[s->stateQ[i]] = c; s->rep_of_class[c] = s->stateQ[i];
            }
        }
    }
    /* itvar sites, SF_Solve.cpp:129-150 */
    s->sites = calloc(M, sizeof(int));
    for (int z = 0; z < M; z++) {
        if (!is_interior(&s->L, z)) continue;
        int ok = 1;
        for (int i = 0; i < ns; i++)
            if (s->freedom[i] == SFGPU_SEG_FROZEN && s->range[(size_t)i * M + z] > 0.999) ok = 0;
        if (ok) s->sites[s->nsites++] = z;
    }
    s->nvar = s->nsites * s->nclass;
    /* charges: psi at every interior site and every site of a frozen
       segment's range (PotItVar, SF_Solve.cpp:1761-1776), interleaved with
       the u of the site in x (UpdateSWF, SF_Solve.cpp:797-810) */
    s->xu = malloc(sizeof(int) * M);
    s->xp = malloc(sizeof(int) * M);
    for (int z = 0; z < M; z++) s->xu[z] = s->xp[z] = -1;
    if (s->charged) {
        int k = 0, j = 0;
        for (int z = 0; z < M; z++) {
            int pot = is_interior(&s->L, z);
            for (int i = 0; i < ns; i++)
                if (s->freedom[i] == SFGPU_SEG_FROZEN && s->range[(size_t)i * M + z] > 0) pot = 1;
            if (pot) s->xp[z] = k++;
            if (j < s->nsites && s->sites[j] == z) { s->xu[z] = k; k += s->nclass; j++; }
            /* the 3D sweep leaves boundary layers to SetBoundaries: a psi
               there would be a copy, not a variable */
            if (pot && s->L.grad == 3 && !is_interior(&s->L, z)) { orc_destroy(s); return SFGPU_ERR_UNSUPPORTED; }
        }
        s->nvar = k;
    } else {
        for (int j = 0; j < s->nsites; j++) s->xu[s->sites[j]] = j * s->nclass;
    }
    s->psi0 = calloc(M, sizeof(double));
    s->psi = calloc(M, sizeof(double));
    s->esq = calloc(M, sizeof(double));
    /* lattice sites per layer (MultiplyWithLatticeSites, Lat1DFlat.cpp:266-269) */
    s->lsites = malloc(sizeof(double) * M);
    for (int z = 0; z < M; z++) {   /* curved: Lat1DCylinder.cpp:127-132, Lat2DCylinder.cpp:156-164 */
        int c[3]; coords(&s->L, z, c);
        s->lsites[z] = s->L.cyl ? s->L.Lx[c[0]] : 1.0;
    }
    if (s->L.grad == 1 && !s->L.cyl && M > 3) { s->lsites[1] *= s->L.ladj; s->lsites[M - 2] *= 2 - s->L.ladj; }
    s->swf_full = calloc((size_t)ns * M, sizeof(double));
    s->swf = calloc((size_t)ns * M, sizeof(double));
    s->phi = calloc((size_t)ns * M, sizeof(double));
    s->rho = calloc((size_t)ns * M, sizeof(double));
    s->phib = calloc(ns, sizeof(double));
    *out = s;
    return SFGPU_OK;
}

void orc_destroy(orc_system *s) {
    if (!s) return;
    olat_free(&s->L);
    for (int m = 0; m < s->nmol; m++) {
        free(s->mol[m].seg); free(s->mol[m].count); free(s->mol[m].used); free(s->mol[m].phi); free(s->mol[m].ori);
        free(s->mol[m].gen_len); free(s->mol[m].gen_rep); free(s->mol[m].gen_seg); free(s->mol[m].parent);
    }
    free(s->val); free(s->eps); free(s->xu); free(s->xp); free(s->psi0); free(s->psi); free(s->esq); free(s->lsites);
    free(s->mol); free(s->freedom); free(s->range); free(s->chi); free(s->pf);
    free(s->stateQ); free(s->class_of); free(s->rep_of_class); free(s->sites);
    free(s->swf_full); free(s->swf); free(s->phi); free(s->rho); free(s->phib);
    free(s);
}

int orc_num_sites(const orc_system *s) { return s->L.M; }
int orc_num_itvar(const orc_system *s) { return s->nvar; }
int orc_num_classes(const orc_system *s) { return s->nclass; }
int orc_itvar_sites(const orc_system *s, int *sites) { memcpy(sites, s->sites, sizeof(int) * s->nsites); return s->nsites; }
int orc_class_of_segment(const orc_system *s, int seg) { return s->class_of[seg]; }

/* SF_Solve::UpdateSWF (SF_Solve.cpp:794-852) + SF_State/SF_MolState::UpdateSWF
   (SF_State.cpp:281-287, SF_MolState.cpp:147-151) */
/* Lat1DFlat::ElectricPotential (Lat1DFlat.cpp:526-549): one Jacobi sweep of
   the Poisson equation with the layer-averaged dielectric constant, 0-based;
   a surface layer takes its own charge, other boundary layers copy */
static void olat_poisson_flat(const olat *L, const double *psi0, const double *eps, const double *charge,
                              double preFactor, double *psi) {
    int M = L->M;
    double pf = 2 * preFactor, epsmin, epsplus;
    if (L->bc_hi[0] == SFGPU_BOUND_SURFACE) {
        epsmin = eps[M - 2] + eps[M - 1];
        psi[M - 1] = psi0[M - 2] + pf * charge[M - 1] / epsmin;
    } else {
        psi[M - 1] = psi0[mapped_site(L, M - 1, NULL)];
    }
    epsplus = eps[0] + eps[1];
    if (L->bc_lo[0] == SFGPU_BOUND_SURFACE) psi[0] = psi0[1] + pf * charge[0] / epsplus;
    else psi[0] = psi0[mapped_site(L, 0, NULL)];
    for (int z = 1; z < M - 1; z++) {
        epsmin = epsplus;
        epsplus = eps[z] + eps[z + 1];
        psi[z] = (epsmin * psi0[z - 1] + pf * charge[z] + epsplus * psi0[z + 1]) / (epsmin + epsplus);
    }
}

/* Lat1DFlat::ElectricFieldSquared (Lat1DFlat.cpp:551-570) */
static void olat_esq_flat(const olat *L, const double *psi, double preFactor, double *esq) {
    int M = L->M;
    double pf = preFactor / 2, emin, eplus = psi[0] - psi[1];
    eplus *= eplus;
    if (L->bc_lo[0] == SFGPU_BOUND_SURFACE) esq[0] = pf * eplus;
    for (int z = 1; z < M - 1; z++) {
        emin = eplus;
        eplus = psi[z] - psi[z + 1];
        eplus *= eplus;
        esq[z] = pf * (emin + eplus);
    }
    if (L->bc_hi[0] == SFGPU_BOUND_SURFACE) esq[M - 1] = pf * eplus;
}

/* Lat1DCylinder::ElectricPotential (Lat1DCylinder.cpp:178-210) and
   Lat1DSphere::ElectricPotential (Lat1DSphere.cpp:76-107), 0-based: the
   sweep weighted by the radius (cylinder) or its square (sphere) of the
   outer edge of each layer; without an offset the first interior layer
   takes only its outer neighbour.  Entries the reference leaves unset keep
   their previous value.  The cylinder sets psi0's boundaries first. */
static void olat_poisson_curved(const olat *L, double *psi0, const double *eps, const double *charge,
                                double preFactor, double *psi) {
    const double PI_ = 4.0 * atan(1.0);
    int M = L->M, z;
    double Z, pf, epsmin, epsplus;
    if (!L->sph) olat_set_boundaries(L, psi0);
    pf = L->sph ? preFactor / 2 / PI_ : preFactor / PI_;
    Z = L->off1 + L->ladj - 1;
    #define RW(Z) (L->sph ? (Z) * (Z) : (Z))
    if (L->off1 <= 0) {
        Z++;
        epsplus = RW(Z) * (eps[1] + eps[2]);
        psi[1] = psi0[2] + pf * charge[1] / epsplus;
        z = 2;
    } else {
        epsplus = RW(Z) * (eps[0] + eps[1]);
        if (L->bc_lo[0] == SFGPU_BOUND_SURFACE) psi[0] = psi0[1] + pf * charge[0] / epsplus;
        z = 1;
    }
    for (; z < M - 1; z++) {
        Z++;
        epsmin = epsplus;
        epsplus = RW(Z) * (eps[z] + eps[z + 1]);
        psi[z] = (pf * charge[z] + psi0[z - 1] * epsmin + psi0[z + 1] * epsplus) / (epsmin + epsplus);
    }
    #undef RW
    if (L->bc_hi[0] == SFGPU_BOUND_SURFACE) psi[M - 1] = psi0[M - 2] + pf * charge[M - 1] / epsplus;
}

/* Lat1DCylinder::ElectricFieldSquared (Lat1DCylinder.cpp:211-240) and
   Lat1DSphere::ElectricFieldSquared (Lat1DSphere.cpp:108-131), 0-based */
static void olat_esq_curved(const olat *L, const double *psi, double preFactor, double *esq) {
    const double PI_ = 4.0 * atan(1.0);
    int M = L->M, z;
    double Z, pf, emin, eplus;
    if (L->sph) {
        pf = preFactor * PI_ * 2;
        Z = L->off1 + L->ladj - 1;
        eplus = Z * (psi[0] - psi[1]);
        eplus *= eplus;
        if (L->bc_lo[0] == SFGPU_BOUND_SURFACE) esq[0] = pf * eplus / L->Lx[0];
        for (z = 1; z < M - 1; z++) {
            Z++;
            emin = eplus;
            eplus = Z * (psi[z] - psi[z + 1]);
            eplus *= eplus;
            esq[z] = pf * (emin + eplus) / L->Lx[z];
        }
        if (L->bc_hi[0] == SFGPU_BOUND_SURFACE) esq[M - 1] = pf * eplus / L->Lx[M - 1];
        return;
    }
    pf = preFactor / 2;
    Z = L->off1 + L->ladj - 1.5;
    if (L->off1 <= 0) {
        Z++;
        eplus = psi[1] - psi[2];
        eplus *= (Z + 0.5) * eplus;
        esq[1] = pf * eplus / Z;
        z = 2;
    } else {
        eplus = psi[0] - psi[1];
        eplus *= (Z + 0.5) * eplus;
        if (L->bc_lo[0] == SFGPU_BOUND_SURFACE) esq[0] = pf * eplus / Z;
        z = 1;
    }
    for (; z < M - 1; z++) {
        Z++;
        emin = eplus;
        eplus = psi[z] - psi[z + 1];
        eplus *= (Z + 0.5) * eplus;
        esq[z] = pf * (emin + eplus) / Z;
    }
    if (L->bc_hi[0] == SFGPU_BOUND_SURFACE) esq[M - 1] = pf * eplus / Z;
}

/* The 2D sweeps and fields below walk the lattice as the reference does,
   1-based (site k of the reference is index k - 1 here; MY sites per row x):
   the lower x row first, then the rows x = 2..MX-1 from y = 1 to MY, then the
   upper x row.  A boundary row or column is updated only where its bound is
   a surface; the other entries keep their previous value.  Two-term sums are
   exact under commutation, so only longer sums keep the reference's order,
   and the reference's own choices are kept where they look like slips (the
   first site of the lower x row takes the running y-sum of the corner, the
   upper y corner of the lower row the charge of site 1, the upper corner of
   the upper row the dielectric sum eps[M-MY] + eps[M]). */
#define R1(a, k) (a)[(k) - 1]

/* Lat2DFlat::ElectricPotential (Lat2DFlat.cpp:1116-1207) */
static void olat_poisson_2dflat(const olat *L, double *psi0, const double *eps, const double *charge,
                                double preFactor, double *psi) {
    const int MX = L->Md[0], MY = L->Md[1], M = MX * MY;
    const int sx1 = L->bc_lo[0] == SFGPU_BOUND_SURFACE, sx2 = L->bc_hi[0] == SFGPU_BOUND_SURFACE;
    const int sy1 = L->bc_lo[1] == SFGPU_BOUND_SURFACE, sy2 = L->bc_hi[1] == SFGPU_BOUND_SURFACE;
    const double pf = 2 * preFactor;
    double exm, exp_, eym = 0, eyp;
    int z;
    olat_set_boundaries(L, psi0);
    if (sx1) {
        eyp = R1(eps, 1) + R1(eps, 2);
        if (sy1) {
            exp_ = R1(eps, 1) + R1(eps, MY + 1);
            R1(psi, 1) = (pf * R1(charge, 1) + exp_ * R1(psi0, MY + 1) + eyp * R1(psi0, 2)) / (exp_ + eyp);
        }
        for (z = MY - 1; z > 1; z--) {
            eym = eyp;
            exp_ = R1(eps, z) + R1(eps, z + MY);
            eyp = R1(eps, z) + R1(eps, z + 1);
            R1(psi, z) = (pf * R1(charge, z) + exp_ * R1(psi0, z + MY) + eym * R1(psi0, z - 1) + eyp * R1(psi0, z + 1)) /
                         (exp_ + eym + eyp);
        }
        if (sy2) {
            exp_ = R1(eps, MY) + R1(eps, MY + MY);
            R1(psi, MY) = (pf * R1(charge, z) + exp_ * R1(psi0, MY + MY) + eyp * R1(psi0, MY - 1)) / (exp_ + eyp);
        }
    }
    z = MY + 1;
    for (int x = 2; x < MX; x++) {
        eyp = R1(eps, z) + R1(eps, z + 1);
        if (sy1) {
            exm = R1(eps, z) + R1(eps, z - MY);
            exp_ = R1(eps, z) + R1(eps, z + MY);
            R1(psi, z) = (pf * R1(charge, z) + exm * R1(psi0, z - MY) + exp_ * R1(psi0, z + MY) + eyp * R1(psi0, z + 1)) /
                         (exm + exp_ + eyp);
        }
        z++;
        for (int y = 2; y < MY; y++, z++) {
            eym = eyp;
            exm = R1(eps, z) + R1(eps, z - MY);
            exp_ = R1(eps, z) + R1(eps, z + MY);
            eyp = R1(eps, z) + R1(eps, z + 1);
            R1(psi, z) = (pf * R1(charge, z) + exm * R1(psi0, z - MY) + exp_ * R1(psi0, z + MY) + eym * R1(psi0, z - 1) +
                          eyp * R1(psi0, z + 1)) / (exm + exp_ + eym + eyp);
        }
        if (sy2) {
            exm = R1(eps, z) + R1(eps, z - MY);
            exp_ = R1(eps, z) + R1(eps, z + MY);
            R1(psi, z) = (pf * R1(charge, z) + exm * R1(psi0, z - MY) + exp_ * R1(psi0, z + MY) + eyp * R1(psi0, z - 1)) /
                         (exm + exp_ + eyp);
        }
        z++;
    }
    if (sx2) {
        eyp = R1(eps, M - MY + 1) + R1(eps, M - MY + 2);
        if (sy1) {
            exm = R1(eps, M - MY + 1) + R1(eps, M - MY - MY + 1);
            R1(psi, M - MY + 1) = (pf * R1(charge, M - MY + 1) + exm * R1(psi0, M - MY - MY + 1) + eyp * R1(psi0, M - MY + 2)) /
                                  (exm + eyp);
        }
        for (z = M - MY + 2; z < M; z++) {
            eym = eyp;
            exm = R1(eps, z) + R1(eps, z - MY);
            eyp = R1(eps, z) + R1(eps, z + 1);
            R1(psi, z) = (pf * R1(charge, z) + exm * R1(psi0, z - MY) + eym * R1(psi0, z - 1) + eyp * R1(psi0, z + 1)) /
                         (exm + eym + eyp);
        }
        if (sy2) {
            exm = R1(eps, M - MY) + R1(eps, M);
            R1(psi, M) = (pf * R1(charge, M) + exm * R1(psi0, M - MY) + eyp * R1(psi0, M - 1)) / (exm + eyp);
        }
    }
}

/* Lat2DFlat::ElectricFieldSquared (Lat2DFlat.cpp:1209-1272) */
static void olat_esq_2dflat(const olat *L, const double *psi, double preFactor, double *esq) {
    const int MX = L->Md[0], MY = L->Md[1], M = MX * MY;
    const int sx1 = L->bc_lo[0] == SFGPU_BOUND_SURFACE, sx2 = L->bc_hi[0] == SFGPU_BOUND_SURFACE;
    const int sy1 = L->bc_lo[1] == SFGPU_BOUND_SURFACE, sy2 = L->bc_hi[1] == SFGPU_BOUND_SURFACE;
    const double pf = preFactor / 2;
    double exm, exp_, eym, eyp;
    int z;
    #define SQ(v) ((v) * (v))
    if (sx1) {
        eym = SQ(R1(psi, MY - 1) - R1(psi, MY));
        for (z = MY - 1; z > 1; z--) {
            eyp = eym;
            eym = SQ(R1(psi, z) - R1(psi, z - 1));
            exp_ = SQ(R1(psi, z) - R1(psi, z + MY));
            R1(esq, z) = pf * (exp_ + eym + eyp);
        }
    }
    z = MY + 1;
    for (int x = 2; x < MX; x++) {
        eyp = SQ(R1(psi, z) - R1(psi, z + 1));
        if (sy1) {
            exm = SQ(R1(psi, z) - R1(psi, z - MY));
            exp_ = SQ(R1(psi, z) - R1(psi, z + MY));
            R1(esq, z) = pf * (exm + exp_ + eyp);
        }
        z++;
        for (int y = 2; y < MY; y++, z++) {
            eym = eyp;
            eyp = SQ(R1(psi, z) - R1(psi, z + 1));
            exm = SQ(R1(psi, z) - R1(psi, z - MY));
            exp_ = SQ(R1(psi, z) - R1(psi, z + MY));
            R1(esq, z) = pf * (exm + exp_ + eym + eyp);
        }
        if (sy2) {
            exm = SQ(R1(psi, z) - R1(psi, z - MY));
            exp_ = SQ(R1(psi, z) - R1(psi, z + MY));
            R1(esq, z) = pf * (exm + exp_ + eyp);
        }
        z++;
    }
    if (sx2) {
        eyp = SQ(R1(psi, M - MY + 2) - R1(psi, M - MY + 1));
        for (z = M - MY + 2; z < M; z++) {
            eym = eyp;
            eyp = SQ(R1(psi, z) - R1(psi, z + 1));
            exm = SQ(R1(psi, z) - R1(psi, z - MY));
            R1(esq, z) = pf * (exm + eym + eyp);
        }
    }
}

/* radius to the centre of the first layer of the 2D cylinder, L[3]/2/PI - 2
   (Lat2DCylinder.cpp:337) */
static double cyl2d_z0(const olat *L) {
    const double PI_ = 4.0 * atan(1.0);
    return L->Lx[2] / 2 / PI_ - 2;
}

/* Lat2DCylinder::ElectricPotential (Lat2DCylinder.cpp:323-450): the
   dielectric sums across rows weighted by 1 -+ 1/(2Z), the charge term by
   1/(PI Z); without an offset the first interior row has no inner
   neighbour and is walked from y = MY down */
static void olat_poisson_2dcyl(const olat *L, double *psi0, const double *eps, const double *charge,
                               double preFactor, double *psi) {
    const double PI_ = 4.0 * atan(1.0);
    const int MX = L->Md[0], MY = L->Md[1], M = MX * MY;
    const int sx1 = L->bc_lo[0] == SFGPU_BOUND_SURFACE, sx2 = L->bc_hi[0] == SFGPU_BOUND_SURFACE;
    const int sy1 = L->bc_lo[1] == SFGPU_BOUND_SURFACE, sy2 = L->bc_hi[1] == SFGPU_BOUND_SURFACE;
    double Z = cyl2d_z0(L), pf, xm, xp, exm, exp_, eym, eyp = 0;
    int x, z;
    olat_set_boundaries(L, psi0);
    if (L->off1 <= 0) {
        Z++;
        pf = preFactor / PI_ / Z;
        xp = 1 + 0.5 / Z;
        z = MY + MY;
        eym = R1(eps, z) + R1(eps, z - 1);
        if (sy2) {
            exp_ = xp * (R1(eps, z) + R1(eps, z + MY));
            R1(psi, z) = (pf * R1(charge, z) + eym * R1(psi0, z - 1) + exp_ * R1(psi0, z + MY)) / (eym + exp_);
        }
        for (z = 2 * MY - 1; z > MY + 1; z--) {
            eyp = eym;
            eym = R1(eps, z) + R1(eps, z - 1);
            exp_ = xp * (R1(eps, z) + R1(eps, z + MY));
            R1(psi, z) = (pf * R1(charge, z) + exp_ * R1(psi0, z + MY) + eym * R1(psi0, z - 1) + eyp * R1(psi0, z + 1)) /
                         (exp_ + eym + eyp);
        }
        if (sy1) {
            exp_ = xp * (R1(eps, z) + R1(eps, z + MY));
            R1(psi, z) = (pf * R1(charge, z) + exp_ * R1(psi0, z + MY) + eym * R1(psi0, z + 1)) / (exp_ + eym);
        }
        x = 3;
        z = MY + MY + 1;
    } else {
        if (sx1) {
            pf = preFactor / PI_ / Z;
            xp = 1 + 0.5 / Z;
            eym = R1(eps, MY) + R1(eps, MY - 1);
            if (sy2) {
                exp_ = xp * (R1(eps, MY) + R1(eps, MY + MY));
                R1(psi, MY) = (pf * R1(charge, MY) + eym * R1(psi0, MY - 1) + exp_ * R1(psi0, MY + MY)) / (eym + exp_);
            }
            for (z = MY - 1; z > 1; z--) {
                eyp = eym;
                eym = R1(eps, z) + R1(eps, z - 1);
                exp_ = xp * (R1(eps, z) + R1(eps, z + MY));
                R1(psi, z) = (pf * R1(charge, z) + exp_ * R1(psi0, z + MY) + eym * R1(psi0, z - 1) + eyp * R1(psi0, z + 1)) /
                             (exp_ + eym + eyp);
            }
            if (sy1) {
                exp_ = xp * (R1(eps, 1) + R1(eps, MY + 1));
                R1(psi, 1) = (pf * R1(charge, 1) + exp_ * R1(psi0, MY + 1) + eym * R1(psi0, 2)) / (exp_ + eym);
            }
        }
        x = 2;
        z = MY + 1;
    }
    for (; x < MX; x++) {
        Z++;
        pf = preFactor / PI_ / Z;
        xm = 1 - 0.5 / Z;
        xp = 1 + 0.5 / Z;
        eyp = R1(eps, z) + R1(eps, z + 1);
        if (sy1) {
            exm = xm * (R1(eps, z - MY) + R1(eps, z));
            exp_ = xp * (R1(eps, z) + R1(eps, z + MY));
            R1(psi, z) = (pf * R1(charge, z) + exm * R1(psi0, z - MY) + exp_ * R1(psi0, z + MY) + eyp * R1(psi0, z + 1)) /
                         (exm + exp_ + eyp);
        }
        z++;
        for (int y = 2; y < MY; y++, z++) {
            eym = eyp;
            eyp = R1(eps, z) + R1(eps, z + 1);
            exm = xm * (R1(eps, z - MY) + R1(eps, z));
            exp_ = xp * (R1(eps, z) + R1(eps, z + MY));
            R1(psi, z) = (pf * R1(charge, z) + exm * R1(psi0, z - MY) + exp_ * R1(psi0, z + MY) + eym * R1(psi0, z - 1) +
                          eyp * R1(psi0, z + 1)) / (exm + exp_ + eym + eyp);
        }
        if (sy2) {
            exm = xm * (R1(eps, z - MY) + R1(eps, z));
            exp_ = xp * (R1(eps, z) + R1(eps, z + MY));
            R1(psi, z) = (pf * R1(charge, z) + exm * R1(psi0, z - MY) + exp_ * R1(psi0, z + MY) + eyp * R1(psi0, z - 1)) /
                         (exm + exp_ + eyp);
        }
        z++;
    }
    if (sx2) {
        Z++;
        pf = preFactor / PI_ / Z;
        xm = 1 - 0.5 / Z;
        eyp = R1(eps, M - MY + 1) + R1(eps, M - MY + 2);
        if (sy1) {
            exm = xm * (R1(eps, M - MY - MY + 1) + R1(eps, M - MY + 1));
            R1(psi, M - MY + 1) = (pf * R1(charge, M - MY + 1) + exm * R1(psi0, M - MY - MY + 1) + eyp * R1(psi0, M - MY + 2)) /
                                  (exm + eyp);
        }
        for (z = M - MY + 2; z < M; z++) {
            eym = eyp;
            eyp = R1(eps, z) + R1(eps, z + 1);
            exm = xm * (R1(eps, z - MY) + R1(eps, z));
            R1(psi, z) = (pf * R1(charge, z) + exm * R1(psi0, z - MY) + eym * R1(psi0, z - 1) + eyp * R1(psi0, z + 1)) /
                         (exm + eym + eyp);
        }
        if (sy2) {
            exm = xm * (R1(eps, M) + R1(eps, M - MY));
            R1(psi, M) = (pf * R1(charge, M) + exm * R1(psi0, M - MY) + eyp * R1(psi0, M - 1)) / (exm + eyp);
        }
    }
}

/* Lat2DCylinder::ElectricFieldSquared (Lat2DCylinder.cpp:452-541) */
static void olat_esq_2dcyl(const olat *L, const double *psi, double preFactor, double *esq) {
    const int MX = L->Md[0], MY = L->Md[1], M = MX * MY;
    const int sx1 = L->bc_lo[0] == SFGPU_BOUND_SURFACE, sx2 = L->bc_hi[0] == SFGPU_BOUND_SURFACE;
    const int sy1 = L->bc_lo[1] == SFGPU_BOUND_SURFACE, sy2 = L->bc_hi[1] == SFGPU_BOUND_SURFACE;
    const double pf = preFactor / 2;
    double Z = cyl2d_z0(L), xm, xp, exm, exp_, eym, eyp;
    int x, z;
    if (L->off1 <= 0) {
        Z++;
        xp = 1 + 0.5 / Z;
        eym = SQ(R1(psi, MY + MY) - R1(psi, MY + MY - 1));
        for (z = 2 * MY - 1; z > MY + 1; z--) {
            eyp = eym;
            eym = SQ(R1(psi, z) - R1(psi, z - 1));
            exp_ = R1(psi, z) - R1(psi, z + MY);
            exp_ *= xp * exp_;
            R1(esq, z) = pf * (exp_ + eym + eyp);
        }
        x = 3;
        z = MY + MY + 1;
    } else {
        if (sx1) {
            xp = 1 + 0.5 / Z;
            eym = SQ(R1(psi, MY) - R1(psi, MY - 1));
            for (z = MY - 1; z > 1; z--) {
                eyp = eym;
                eym = SQ(R1(psi, z) - R1(psi, z - 1));
                exp_ = R1(psi, z) - R1(psi, z + MY);
                exp_ *= xp * exp_;
                R1(esq, z) = pf * (exp_ + eym + eyp);
            }
        }
        x = 2;
        z = MY + 1;
    }
    for (; x < MX; x++) {
        Z++;
        xm = 1 - 0.5 / Z;
        xp = 1 + 0.5 / Z;
        eyp = SQ(R1(psi, z) - R1(psi, z + 1));
        if (sy1) {
            exm = R1(psi, z) - R1(psi, z - MY);
            exm *= xm * exm;
            exp_ = R1(psi, z) - R1(psi, z + MY);
            exp_ *= xp * exp_;
            R1(esq, z) = pf * (exm + exp_ + eyp);
        }
        z++;
        for (int y = 2; y < MY; y++, z++) {
            eym = eyp;
            eyp = SQ(R1(psi, z) - R1(psi, z + 1));
            exm = R1(psi, z) - R1(psi, z - MY);
            exm *= xm * exm;
            exp_ = R1(psi, z) - R1(psi, z + MY);
            exp_ *= xp * exp_;
            R1(esq, z) = pf * (exm + exp_ + eym + eyp);
        }
        if (sy2) {
            exm = R1(psi, z) - R1(psi, z - MY);
            exm *= xm * exm;
            exp_ = R1(psi, z) - R1(psi, z + MY);
            exp_ *= xp * exp_;
            R1(esq, z) = pf * (exm + exp_ + eyp);
        }
        z++;
    }
    if (sx2) {
        Z++;
        xm = 1 - 0.5 / Z;
        eyp = SQ(R1(psi, M - MY + 2) - R1(psi, M - MY + 1));
        for (z = M - MY + 2; z < M; z++) {
            eym = eyp;
            eyp = SQ(R1(psi, z) - R1(psi, z + 1));
            exm = R1(psi, z) - R1(psi, z - MY);
            exm *= xm * exm;
            R1(esq, z) = pf * (exm + eym + eyp);
        }
    }
    (void)sy1; (void)sy2;
}

/* Lat3D::ElectricPotential (Lat3D.cpp:1937-1969): boundaries of psi0 and
   of the dielectric profile first, then per site the six neighbour terms in
   the order -x, +x, -y, +y, -z, +z, the charge term, the division by the
   summed dielectric weights (0 where they are not positive), and the
   boundaries of psi.  Only interior sites are computed here: the
   reference's shifted vector operations leave boundary entries to
   SetBoundaries (no psi site lies on a boundary layer of a 3D lattice). */
static void olat_poisson_3d(const olat *L, double *psi0, const double *eps_in, const double *charge,
                            double preFactor, double *psi) {
    const int M = L->M, jx = L->st[0], jy = L->st[1];
    double *eps = malloc(sizeof(double) * M);
    memcpy(eps, eps_in, sizeof(double) * M);
    olat_set_boundaries(L, psi0);
    olat_set_boundaries(L, eps);
    const int off[6] = {-jx, jx, -jy, jy, -1, 1};
    for (int z = 0; z < M; z++) {
        if (!is_interior(L, z)) continue;
        double tot = 0, acc = 0;
        for (int k = 0; k < 6; k++) {
            const double w = eps[z + off[k]] + eps[z];
            if (k == 0) { tot = w; acc = w * psi0[z + off[k]]; }
            else { tot += w; acc += w * psi0[z + off[k]]; }
        }
        acc += charge[z] * (2 * preFactor);
        psi[z] = (tot > 0) ? acc / tot : 0.0;
    }
    olat_set_boundaries(L, psi);
    free(eps);
}

/* Lat3D::ElectricFieldSquared (Lat3D.cpp:1979-2005): the six squared
   differences in the same order, times preFactor / 2 */
static void olat_esq_3d(const olat *L, double *psi, double preFactor, double *esq) {
    const int M = L->M, jx = L->st[0], jy = L->st[1];
    const int off[6] = {-jx, jx, -jy, jy, -1, 1};
    olat_set_boundaries(L, psi);
    const double pf = preFactor / 2;
    for (int z = 0; z < M; z++) {
        if (!is_interior(L, z)) continue;
        double e = SQ(psi[z] - psi[z + off[0]]);
        for (int k = 1; k < 6; k++) e += SQ(psi[z] - psi[z + off[k]]);
        esq[z] = e * pf;
    }
    olat_set_boundaries(L, esq);
}
#undef SQ
#undef R1

/* SF_SegmentList::GetCharge (SF_SegmentList.cpp:759-784): sum phi valence /
   phi_T per layer, times the lattice sites of the layer */
static void state_charge(const orc_system *s, double *charge) {
    int M = s->L.M;
    double *pt = calloc(M, sizeof(double));
    for (int z = 0; z < M; z++) charge[z] = 0;
    for (int i = 0; i < s->nseg; i++) {
        const double *p = s->phi + (size_t)i * M;
        for (int z = 0; z < M; z++) { charge[z] += p[z] * s->val[i]; pt[z] += p[z]; }
    }
    for (int z = 0; z < M; z++) charge[z] /= pt[z];
    for (int z = 0; z < M; z++) charge[z] *= s->lsites[z];
    free(pt);
}

static void update_swf(orc_system *s, const double *x) {
    int M = s->L.M, nc = s->nclass;
    const double kT = ORC_BOLTZMANN * s->temperature;
    if (s->charged) {
        /* psi0 from x, its boundary copies and E^2 (SF_Solve.cpp:797-818) */
        for (int z = 0; z < M; z++) if (s->xp[z] >= 0) s->psi0[z] = x[s->xp[z]];
        olat_set_boundaries(&s->L, s->psi0);
        const double pfe = (ORC_EPS0 * s->sitedist) / kT;
        if (s->L.grad == 3) olat_esq_3d(&s->L, s->psi0, pfe, s->esq);
        else if (s->L.grad == 2 && s->L.cyl) olat_esq_2dcyl(&s->L, s->psi0, pfe, s->esq);
        else if (s->L.grad == 2) olat_esq_2dflat(&s->L, s->psi0, pfe, s->esq);
        else if (s->L.cyl) olat_esq_curved(&s->L, s->psi0, pfe, s->esq);
        else olat_esq_flat(&s->L, s->psi0, pfe, s->esq);
    }
    for (int i = 0; i < s->nseg; i++) {
        double *gf = s->swf_full + (size_t)i * M;
        memset(gf, 0, sizeof(double) * M);
        int c = s->class_of[i];
        if (c < 0) continue;
        if (s->charged) {
            /* exp(-x) times the electrostatic factors of the state
               (SF_Solve.cpp:808, :819-834) */
            for (int j = 0; j < s->nsites; j++) {
                int z = s->sites[j];
                gf[z] = exp(-x[s->xu[z] + c] - 0.0);
                gf[z] *= exp(-s->val[i] * s->psi0[z] * ORC_ELEM_CHARGE / kT);
                if (s->diffeps) gf[z] *= exp(0.5 * s->eps[i] * s->esq[z]);
            }
        } else {
            for (int j = 0; j < s->nsites; j++) gf[s->sites[j]] = exp(-x[j * nc + c]);
        }
        olat_set_boundaries(&s->L, gf);
        double *g = s->swf + (size_t)i * M;
        if (s->freedom[i] == SFGPU_SEG_PINNED) {
            const double *r = s->range + (size_t)i * M;
            for (int z = 0; z < M; z++) g[z] = (r[z] > 0) ? gf[z] : 0.0;
            olat_set_boundaries(&s->L, g);   /* SF_Homopol1stO.cpp:105-106, SF_Copol1stO.cpp:123-127 */
        } else {
            memcpy(g, gf, sizeof(double) * M);
        }
    }
}

static void propagate_any(const orc_system *s, const double *gin, const double *G, double S, double *gout, int backward) {
    if (s->L.order == 2 && s->L.grad == 3) olat_prop2(&s->L, gin, G, S, gout, backward);
    else if (s->L.order == 2) olat_prop2l(&s->L, gin, G, S, gout, backward);
    else olat_prop1(&s->L, gin, G, gout);
}

/* bond-orientation composition, Lat2ndO::ConnectG(..., PHI):
   Lat3D2ndO.cpp:905-918 (+-x -> 0, +-y -> 1, +-z -> 2), Lat1D2ndO.cpp:215-227
   (+-x -> 0, lateral group times 4 -> 1), Lat2D2ndO.cpp:285-304 (slot kk of
   k = 0..4 is 0, 1, 2, then 2 again for k = 3 since kk is not reassigned, and
   1 for k = 4; the z group is added to slot 2 once more after the loop).
   Interior sites only (Lat1D2ndO::ConnectG removes the boundaries first). */
static void orient_acc(const olat *L, const double *a, const double *b, double *out) {
    static const int s6[6] = {0, 1, 2, 2, 1, 0}, s5[5] = {0, 1, 2, 2, 1}, s3[3] = {0, 1, 0};
    int M = L->M, K = L->K;
    const int *sl = (K == 6) ? s6 : (K == 5) ? s5 : s3;
    for (int k = 0; k < K; k++)
        for (int z = 0; z < M; z++) {
            if (!is_interior(L, z)) continue;
            double v = a[(size_t)k * M + z] * b[(size_t)k * M + z];
            if (K == 3 && k == 1) v = v * 4.0;
            out[(size_t)sl[k] * M + z] += v;
        }
    if (K == 5)
        for (int z = 0; z < M; z++)
            if (is_interior(L, z)) out[2 * (size_t)M + z] += a[2 * (size_t)M + z] * b[2 * (size_t)M + z];
}

/* ------------------------------------------------------------------------ */
/* Overflow protection: the *1stOS lattices in natural logarithms            */
/* ------------------------------------------------------------------------ */
#define LOGZERO (-DBL_MAX / 2)          /* SF_Box.h:51 */
#define LOGCUTOFF 100.0                 /* SF_Box.h:45 */
#define LOGTOLERANCE 50.0               /* SF_Box.h:47 */
static double logmaxdouble(void) { return log(DBL_MAX); }                         /* SF_Box.h:31 */
static double logmaxprefactor(void) { return logmaxdouble() - LOGCUTOFF - LOGTOLERANCE; }   /* SF_Box.h:49 */

/* Lat1DFlat1stOS.cpp:3-9, Lat2DFlat1stOS.cpp:8-13, Lat2DCyl1stOS.cpp:3-25 */
static int olat_init_log(olat *L) {
    if (L->order != 1 || L->grad > 2) return SFGPU_ERR_UNSUPPORTED;   /* SF_System.cpp:395, :478-481 */
    L->logmode = 1;
    double l1 = L->l1;
    if (!L->cyl) {
        double l0 = (L->grad == 1) ? 1 - 2 * l1 : 1 - 4 * l1;
        L->LogL1L0 = log(l1 / l0);
        L->LogL0 = log(l0);
        L->LogL1 = log(l1);
    }
    if (L->cyl && L->grad == 2) {
        int MX = L->Md[0];
        L->logl0x = calloc(MX, sizeof(double));
        L->loglmx = calloc(MX, sizeof(double));
        L->loglpx = calloc(MX, sizeof(double));
        for (int x = 1; x < MX - 1; x++) {
            double lm = L->lam_m[x], lp = L->lam_p[x];
            L->loglpx[x] = (lp > 0) ? log(lp) : 0;
            L->loglmx[x] = (lm > 0) ? log(lm) : 0;
            double l0 = 1.0 - lm - lp - 2 * l1;
            L->logl0x[x] = (l0 > 0) ? log(l0) : 0;
        }
        L->logl1 = (l1 > 0) ? log(l1) : 0;
        L->nl_centre = 1.0 - l1 - l1 - l1 - l1;   /* nl[1], Lat2DCyl1stOS.cpp:191 */
    }
    return SFGPU_OK;
}

/* MakeSafe / RestoreFromSafe, Lat1DFlat1stOS.cpp:21-56 */
static void make_safe(int M, double *A) {
    for (int z = 0; z < M; z++) {
        if (A[z] > 0) {
            if (A[z] > exp(LOGCUTOFF)) {
                double y = (log(A[z]) - LOGCUTOFF) / logmaxprefactor();
                A[z] = LOGCUTOFF + 0.5 * logmaxprefactor() * log((1 + y) / (1 - y));
            } else {
                A[z] = log(A[z]);
            }
        } else {
            A[z] = LOGZERO;
        }
    }
}
static void restore_from_safe(int M, double *A) {
    for (int z = 0; z < M; z++) {
        if (A[z] > LOGZERO) {
            if (A[z] > LOGCUTOFF) A[z] = exp(LOGCUTOFF + logmaxprefactor() * tanh((A[z] - LOGCUTOFF) / logmaxprefactor()));
            else A[z] = exp(A[z]);
        } else {
            A[z] = 0;
        }
    }
}

/* boundary values of a log-space vector: LOGZERO on surfaces, copies
   elsewhere (Gout[1] = LOGZERO; Gout[1] = Gout[bound1], Lat1DFlat1stOS.cpp:140-143;
   UpdateBoundaries, Lat2DFlat1stOS.cpp:538-573) */
static void olat_log_boundaries(const olat *L, double *p) {
    for (int z = 0; z < L->M; z++) {
        if (is_interior(L, z)) continue;
        int c[3]; coords(L, z, c);
        for (int k = 0; k < L->grad; k++)
            if ((c[k] == 0 && L->bc_lo[k] == SFGPU_BOUND_SURFACE) || (c[k] == L->Md[k] - 1 && L->bc_hi[k] == SFGPU_BOUND_SURFACE))
                p[z] = LOGZERO;
    }
    for (int z = 0; z < L->M; z++) {
        if (is_interior(L, z)) continue;
        int m = mapped_site(L, z, NULL);
        if (m != z && is_interior(L, m)) p[z] = p[m];
    }
}

/* one log-space step; gin carries its boundary values.  Lat1DFlat1stOS.cpp:120-145,
   Lat1DCyl1stOS.cpp:45-74 (also the sphere), Lat2DFlat1stOS.cpp:140-169 with
   getNewGi (:335-362), Lat2DCyl1stOS.cpp:173-228 */
static void olat_prop1_log(const olat *L, const double *gin, const double *G, double *gout) {
    int M = L->M;
    for (int z = 0; z < M; z++) {
        if (!is_interior(L, z)) continue;
        if (G[z] == LOGZERO) { gout[z] = LOGZERO; continue; }
        double r;
        if (L->grad == 1) {
            double a = gin[z - 1], b = gin[z], c = gin[z + 1];
            if (!L->cyl) {
                if (b > LOGZERO && L->l1 < 0.5) r = G[z] + L->LogL0 + b + log1p(exp(L->LogL1L0 + a - b) + exp(L->LogL1L0 + c - b));
                else if (a > LOGZERO) r = G[z] + L->LogL1 + a + log1p(exp(c - a));
                else if (c > LOGZERO) r = G[z] + L->LogL1 + c;
                else r = LOGZERO;
            } else {
                double lp = L->lam_p[z], lm = L->lam_m[z];
                double lambda0 = 1 - lp - lm;
                if (b > LOGZERO && lambda0 > 0) r = G[z] + log(lambda0) + b + log1p((lm / lambda0) * exp(a - b) + (lp / lambda0) * exp(c - b));
                else if (a > LOGZERO) r = G[z] + log(lm) + a + log1p((lp / lm) * exp(c - a));
                else if (c > LOGZERO) r = G[z] + log(lp) + c;
                else r = LOGZERO;
            }
        } else {
            int MY = L->Md[1], x = z / MY;
            double b = gin[z];
            if (!L->cyl) {
                double n[4] = {gin[z - 1], gin[z + 1], gin[z - MY], gin[z + MY]};
                double lnterm = 0;
                if (b != LOGZERO && L->l1 < 0.25) {
                    for (int i = 0; i < 4; i++) if (n[i] != LOGZERO) lnterm += exp(L->LogL1L0 + n[i] - b);
                    r = G[z] + L->LogL0 + b + log1p(lnterm);
                } else {
                    int i = 0;
                    while (i < 4 && n[i] == LOGZERO) i++;
                    if (i == 4) r = LOGZERO;
                    else {
                        for (int j = i + 1; j < 4; j++) if (n[j] != LOGZERO) lnterm += exp(n[j] - n[i]);
                        r = G[z] + L->LogL1 + n[i] + log1p(lnterm);
                    }
                }
            } else {
                double ng[5] = {gin[z - 1], b, gin[z + 1], gin[z - MY], gin[z + MY]};
                double nl[5] = {L->l1, L->nl_centre, L->l1, L->lam_m[x], L->lam_p[x]};
                double lognl[5] = {L->logl1, L->logl0x[x], L->logl1, L->loglmx[x], L->loglpx[x]};
                int i = 0;
                while (i < 5 && (ng[i] == LOGZERO || nl[i] <= 0)) i++;
                if (i == 5) r = LOGZERO;
                else {
                    double lnterm = 0;
                    for (int j = 0; j < 5; j++) if (j != i && ng[j] != LOGZERO) lnterm += nl[j] * exp(ng[j] - ng[i]);
                    r = G[z] + lognl[i] + ng[i] + log1p(lnterm / nl[i]);
                }
            }
        }
        gout[z] = r;
    }
    olat_log_boundaries(L, gout);
}

/* copy layer indices of the reference (1-based): lower surface 1, mirror1 2,
   mirror2 3, periodic M-1; upper M, M-1, M-2, periodic 2 */
static int copy_lo1(const olat *L, int k) { return L->bc_lo[k] == SFGPU_BOUND_PERIODIC ? L->Md[k] - 1 : L->bc_lo[k]; }
static int copy_hi1(const olat *L, int k) { return L->bc_hi[k] == SFGPU_BOUND_PERIODIC ? 2 : L->Md[k] - L->bc_hi[k] + 1; }

/* addLntoLn, Lat2DFlat1stOS.cpp:430-447 */
static void add_ln_to_ln(double v1, double v2, double *v, int add) {
    if (v1 != LOGZERO && v2 != LOGZERO) {
        if (*v == LOGZERO) *v = v1 + v2;
        else {
            double sum = v1 + v2 - *v;
            if (sum > logmaxdouble() - 1) *v = v1 + v2;
            else { sum = add ? exp(sum) : -exp(sum); *v += log1p(sum); }
        }
    }
}

/* ComputeLnGN of the log-space lattices, in the reference's own sequence:
   Lat1DFlat1stOS.cpp:441-478, Lat1DCyl1stOS.cpp:242-281,
   Lat2DFlat1stOS.cpp:449-505, Lat2DCyl1stOS.cpp:471-540 */
static double olat_lngn_log(const olat *L, const double *Gi) {
    double value = LOGZERO, lmax = logmaxdouble();
    if (L->grad == 1) {
        int M = L->M;   /* the reference's 1-based layer z is z - 1 here */
        #define LNL(z) (L->cyl ? log(L->Lx[z]) : 0.0)
        if (Gi[1] > LOGZERO) {
            value = L->cyl ? LNL(1) + Gi[1] : Gi[1];
            if (copy_lo1(L, 0) == 3) value -= log(2.0);
        }
        for (int z = 2; z <= M - 3; z++) {
            if (Gi[z] > LOGZERO) {
                double t = L->cyl ? LNL(z) + Gi[z] : Gi[z];
                double x = t - value;
                if (x > lmax - 1 || value == LOGZERO) value = t;
                else value += log1p(exp(x));
            }
        }
        if (copy_hi1(L, 0) == M - 2 && Gi[M - 2] > LOGZERO) {
            double x = L->cyl ? LNL(M - 2) + Gi[M - 2] - value - log(2.0) : Gi[M - 2] - log(2.0) - value;
            if (x > lmax - 1 || value == LOGZERO) value = L->cyl ? LNL(M - 2) + Gi[M - 2] - log(2.0) : Gi[M - 2] - log(2.0);
            else value += log1p(exp(x));
        } else if (M > 3) {
            if (Gi[M - 2] > LOGZERO) {
                double t = L->cyl ? LNL(M - 2) + Gi[M - 2] : Gi[M - 2];
                double x = t - value;
                if (x > lmax - 1 || value == LOGZERO) value = t;
                else value += log1p(exp(x));
            }
        }
        #undef LNL
        return value;
    }
    int MX = L->Md[0], MY = L->Md[1];
    double log2 = log(2.0), log4 = log(4.0);
    #define AT(x, y) Gi[(x) * MY + (y)]
    #define LX(x) (L->cyl ? log(L->Lx[x]) : 0.0)
    for (int x = 1; x < MX - 1; x++)
        for (int y = 1; y < MY - 1; y++) add_ln_to_ln(AT(x, y), LX(x), &value, 1);
    if (copy_lo1(L, 0) == 3)
        for (int y = 1; y < MY - 1; y++) add_ln_to_ln(AT(1, y), LX(1) - log2, &value, 0);
    if (copy_hi1(L, 0) == MX - 2)
        for (int y = 1; y < MY - 1; y++) add_ln_to_ln(AT(MX - 2, y), LX(MX - 2) - log2, &value, 0);
    if (copy_lo1(L, 1) == 3)
        for (int x = 1; x < MX - 1; x++) add_ln_to_ln(AT(x, 1), LX(x) - log2, &value, 0);
    /* the upper y column is taken at 1-based y = MY-2, 0-based MY-3 */
    if (copy_hi1(L, 1) == MY - 2)
        for (int x = 1; x < MX - 1; x++) add_ln_to_ln(AT(x, MY - 3), LX(x) - log2, &value, 0);
    {
        /* corners back: flat -log 4, cylinder log L + log 4 */
        double c1 = L->cyl ? LX(1) + log4 : -log4, c2 = L->cyl ? LX(MX - 2) + log4 : -log4;
        int X1 = copy_lo1(L, 0) == 3, X2 = copy_hi1(L, 0) == MX - 2;
        int Y1 = copy_lo1(L, 1) == 3, Y2 = copy_hi1(L, 1) == MY - 2;
        if (X1 && Y1) add_ln_to_ln(AT(1, 1), c1, &value, 1);
        if (X1 && Y2) add_ln_to_ln(AT(1, MY - 3), c1, &value, 1);
        if (X2 && Y1) add_ln_to_ln(AT(MX - 2, 1), c2, &value, 1);
        if (X2 && Y2) add_ln_to_ln(AT(MX - 2, MY - 3), c2, &value, 1);
    }
    #undef AT
    #undef LX
    return value;
}

/* ConnectG of the log-space lattices, Lat1DFlat1stOS.cpp:344-375, on every site */
static void connect_log(int M, const double *a, const double *b, double *out) {
    for (int z = 0; z < M; z++) {
        if (a[z] > LOGZERO && b[z] > LOGZERO) {
            double x = a[z] + b[z] - out[z];
            if (x > logmaxdouble() - 1 || out[z] == LOGZERO) out[z] = a[z] + b[z];
            else out[z] += log1p(exp(x));
        }
    }
}
/* CorrectDoubleCountG, Lat1DFlat1stOS.cpp:289-298 */
static void correct_double_count_log(int M, double *phi, const double *G) {
    for (int z = 0; z < M; z++) {
        if (G[z] > LOGZERO && phi[z] > LOGZERO) phi[z] -= G[z];
        else phi[z] = LOGZERO;
    }
}
/* NormPhiFree, Lat1DFlat1stOS.cpp:340-347 and Lat2DFlat1stOS.cpp:507-522 */
static void norm_phi_log(const olat *L, int M, double *phi, double lognorm, int norm_is_zero) {
    if (norm_is_zero && L->grad == 2) { for (int z = 0; z < M; z++) phi[z] = LOGZERO; return; }
    for (int z = 0; z < M; z++) if (phi[z] > LOGZERO) phi[z] += lognorm;
}

/* molecule_phi with overflow protection: SF_Monomer1stO.cpp:101-133,
   SF_Homopol1stO.cpp:553-622, SF_Copol1stO.cpp:1187-1281 on the log-space
   lattice functions above; the segment weights enter through MakeSafe and
   the volume fractions leave through RestoreFromSafe */
static void molecule_phi_log(orc_system *s, omol *o) {
    olat *L = &s->L;
    int M = L->M, N = o->N;
    double *lG = malloc(sizeof(double) * M * (size_t)s->nseg);
    for (int a = 0; a < o->nseg_used; a++) {
        int i = o->used[a];
        memcpy(lG + (size_t)i * M, s->swf + (size_t)i * M, sizeof(double) * M);
        make_safe(M, lG + (size_t)i * M);
        for (int z = 0; z < M; z++) o->phi[(size_t)i * M + z] = LOGZERO;
    }
    if (o->type == 0) {
        int i = o->seg[0];
        double *phi = o->phi + (size_t)i * M;
        const double *G = lG + (size_t)i * M;
        memcpy(phi, G, sizeof(double) * M);
        o->lngn = olat_lngn_log(L, G);
        if (o->freedom == SFGPU_MOL_RESTRICTED) {
            o->lnc = log(o->theta) - o->lngn;
            norm_phi_log(L, M, phi, log(o->theta) - olat_lngn_log(L, G), 0);
            o->phibulk = o->theta / exp(o->lngn);
        } else {
            o->lnc = log(o->phibulk);
            norm_phi_log(L, M, phi, log(o->phibulk), o->phibulk == 0);
        }
        restore_from_safe(M, phi);
        free(lG);
        return;
    }
    double *Ginv = malloc(sizeof(double) * M), *tmp = malloc(sizeof(double) * M);
    if (o->type == 1) {
        int i = o->seg[0], half = N / 2;
        const double *G = lG + (size_t)i * M;
        double *phi = o->phi + (size_t)i * M;
        double *Gi = malloc(sizeof(double) * M * (size_t)half);
        memcpy(Gi, G, sizeof(double) * M);
        for (int t = 1; t < half; t++) olat_prop1_log(L, Gi + (size_t)(t - 1) * M, G, Gi + (size_t)t * M);
        memcpy(Ginv, Gi + (size_t)(half - 1) * M, sizeof(double) * M);
        if (N % 2 == 1) {
            olat_prop1_log(L, Ginv, G, tmp); memcpy(Ginv, tmp, sizeof(double) * M);
            connect_log(M, Ginv, Ginv, phi);
            norm_phi_log(L, M, phi, log(0.5), 0);
        }
        for (int sp = (N + 3) / 2; sp <= N; sp++) {
            int sinv = N - sp + 1;
            olat_prop1_log(L, Ginv, G, tmp); memcpy(Ginv, tmp, sizeof(double) * M);
            connect_log(M, Ginv, Gi + (size_t)(sinv - 1) * M, phi);
        }
        correct_double_count_log(M, phi, G);
        o->lngn = olat_lngn_log(L, Ginv);
        if (o->freedom == SFGPU_MOL_RESTRICTED) {
            o->lnc = log(o->theta) - o->lngn - log(1.0 * N);
            norm_phi_log(L, M, phi, log(2 * o->theta / N) - olat_lngn_log(L, Ginv), 0);
            o->phibulk = o->theta / exp(o->lngn);
        } else {
            norm_phi_log(L, M, phi, log(2 * o->phibulk / N), o->phibulk == 0);
            o->lnc = log(o->phibulk / N);
        }
        restore_from_safe(M, phi);
        free(Gi);
    } else {
        double *Gi = malloc(sizeof(double) * M * (size_t)N);
        memcpy(Gi, lG + (size_t)o->seg[0] * M, sizeof(double) * M);
        for (int t = 1; t < N; t++)
            olat_prop1_log(L, Gi + (size_t)(t - 1) * M, lG + (size_t)o->seg[t] * M, Gi + (size_t)t * M);
        memcpy(Ginv, lG + (size_t)o->seg[N - 1] * M, sizeof(double) * M);
        connect_log(M, Ginv, Gi + (size_t)(N - 1) * M, o->phi + (size_t)o->seg[N - 1] * M);
        for (int t = N - 2; t >= 0; t--) {
            int sg = o->seg[t];
            olat_prop1_log(L, Ginv, lG + (size_t)sg * M, tmp); memcpy(Ginv, tmp, sizeof(double) * M);
            connect_log(M, Ginv, Gi + (size_t)t * M, o->phi + (size_t)sg * M);
        }
        o->lngn = olat_lngn_log(L, Ginv);
        for (int a = 0; a < o->nseg_used; a++)
            correct_double_count_log(M, o->phi + (size_t)o->used[a] * M, lG + (size_t)o->used[a] * M);
        double lognorm;
        int zero = 0;
        if (o->freedom == SFGPU_MOL_RESTRICTED) {
            o->lnc = log(o->theta) - o->lngn - log(1.0 * N);
            o->phibulk = o->theta / exp(o->lngn);
            lognorm = log(o->theta / N) - olat_lngn_log(L, Ginv);
        } else {
            o->lnc = log(o->phibulk / N);
            lognorm = log(o->phibulk / N);
            zero = (o->phibulk == 0);
        }
        for (int a = 0; a < o->nseg_used; a++) {
            double *phi = o->phi + (size_t)o->used[a] * M;
            norm_phi_log(L, M, phi, lognorm, zero);
            restore_from_safe(M, phi);
        }
        free(Gi);
    }
    free(Ginv); free(tmp); free(lG);
}

/* one molecule: SF_Monomer1stO::Matrix1 (SF_Monomer1stO.cpp:99-130),
   SF_Homopol1stO::Matrix1 (SF_Homopol1stO.cpp:553-622),
   SF_Copol1stO::Matrix1 (SF_Copol1stO.cpp:1187-1281),
   SF_Homopol2ndO::Matrix1 (SF_Homopol2ndO.cpp:153-207),
   SF_Copol2ndO::Matrix1 (SF_Copol2ndO.cpp:250-356) */
/* SF_Dend1stO::Matrix1 (SF_Dend1stO.cpp:163-312) with the plain first-order
   lattice functions: ends inwards along one end-to-centre path, f copies
   combined at each branch point (ConnectG into zero, CorrectDoubleCountG),
   then centre outwards with NormPhiFree(Gi_inv, NormRepeat) around ConnectG */
static void molecule_phi_dend(orc_system *s, omol *o) {
    olat *L = &s->L;
    int M = L->M, G = o->ngen, NS = o->nshort, N = o->N;
    double *Gi = calloc((size_t)M * NS, sizeof(double));
    double *Ginv = malloc(sizeof(double) * M), *tmp = malloc(sizeof(double) * M);
    double *add = malloc(sizeof(double) * M), *gt = malloc(sizeof(double) * M);
    int off[64];
    off[0] = 0;
    for (int i = 1; i < G; i++) off[i] = off[i - 1] + o->gen_len[i - 1];
    #define SEGAT(i, j) (o->gen_seg[off[i] + (j) - 1])
    #define SLICE(sp) (Gi + (size_t)((sp) - 1) * M)
    int sp = 0;
    const double *Gold = NULL;
    for (int i = G - 1; i >= 0; i--) {
        for (int j = o->gen_len[i]; j >= 1; j--) {
            const double *Gc = s->swf + (size_t)SEGAT(i, j) * M;
            sp++;
            if (sp == 1) memcpy(SLICE(1), Gc, sizeof(double) * M);
            else if (j == o->gen_len[i] && i + 1 < G && o->gen_rep[i + 1] > 1) {
                memcpy(gt, SLICE(sp - 1), sizeof(double) * M);
                for (int k = 1; k <= o->gen_rep[i + 1] - 1; k++) {
                    for (int z = 0; z < M; z++) add[z] = 0 + SLICE(sp - 1)[z] * gt[z];
                    for (int z = 0; z < M; z++) add[z] = (Gold[z] > 0) ? add[z] / Gold[z] : 0;
                    memcpy(gt, add, sizeof(double) * M);
                }
                olat_prop1(L, add, Gc, SLICE(sp));
            } else {
                olat_prop1(L, SLICE(sp - 1), Gc, SLICE(sp));
            }
            Gold = Gc;
        }
    }
    sp = NS;
    double nr = 1;
    for (int i = 0; i < G; i++) {
        int rep = o->gen_rep[i];
        for (int j = 1; j <= o->gen_len[i]; j++) {
            int sg = SEGAT(i, j);
            const double *Gc = s->swf + (size_t)sg * M;
            if (sp == NS) memcpy(Ginv, Gc, sizeof(double) * M);
            else { olat_prop1(L, Ginv, Gc, tmp); memcpy(Ginv, tmp, sizeof(double) * M); }
            double *phi = o->phi + (size_t)sg * M;
            if (j == 1)
                for (int k = 1; k <= rep - 1; k++) {
                    for (int z = 0; z < M; z++) add[z] = 0 + Ginv[z] * SLICE(sp)[z];
                    for (int z = 0; z < M; z++) Ginv[z] = (Gc[z] > 0) ? add[z] / Gc[z] : 0;
                }
            for (int z = 0; z < M; z++) Ginv[z] *= nr;
            for (int z = 0; z < M; z++) phi[z] += Ginv[z] * SLICE(sp)[z];
            double inv = 1.0 / nr;
            for (int z = 0; z < M; z++) Ginv[z] *= inv;
            if (j == 1) nr *= rep;
            sp--;
        }
    }
    #undef SEGAT
    #undef SLICE
    o->lngn = olat_lngn(L, Ginv);
    for (int a = 0; a < o->nseg_used; a++) {
        double *phi = o->phi + (size_t)o->used[a] * M;
        const double *G1 = s->swf + (size_t)o->used[a] * M;
        for (int z = 0; z < M; z++) { if (G1[z] > 0) phi[z] /= G1[z]; else phi[z] = 0; }
    }
    double norm;
    if (o->freedom == SFGPU_MOL_RESTRICTED) {
        o->lnc = log(o->theta) - o->lngn - log(1.0 * N);
        o->phibulk = o->theta / exp(o->lngn);
        norm = (o->theta / N) / exp(o->lngn);
    } else {
        o->lnc = log(o->phibulk / N);
        norm = o->phibulk / N;
    }
    for (int a = 0; a < o->nseg_used; a++) {
        double *phi = o->phi + (size_t)o->used[a] * M;
        for (int z = 0; z < M; z++) phi[z] *= norm;
    }
    free(Gi); free(Ginv); free(tmp); free(add); free(gt);
}

/* Branched molecules (SF_Branched1stO::Matrix1, SF_Branched1stO.cpp:1240-1310)
   on the bond tree rooted at segment 0: U(s) = G_s prod_c A U(c) from the ends
   inwards, Q(c) = G_parent A U(c), D(0) = G_0, D(c) = G_c A [D(p) prod_(c' != c)
   Q(c')], each product of factors that carry G_s once divided by G_s where
   G > 0 (ConnectG then CorrectDoubleCountG); phi += U D before the division by
   G; lnGN from U(0) (SF_Branched1stO.cpp:1269). */
static void molecule_phi_tree(orc_system *s, omol *o) {
    olat *L = &s->L;
    int M = L->M, N = o->N;
    double *U = calloc((size_t)M * N, sizeof(double)), *Q = calloc((size_t)M * N, sizeof(double));
    double *D = calloc((size_t)M * N, sizeof(double)), *acc = malloc(sizeof(double) * M);
    #define SL(A, q) ((A) + (size_t)(q) * M)
    #define GOF(q) (s->swf + (size_t)o->seg[q] * M)
    for (int q = N - 1; q >= 0; q--) {
        const double *Gq = GOF(q);
        int first = 1;
        for (int c = q + 1; c < N; c++) {
            if (o->parent[c] != q) continue;
            if (first) { memcpy(SL(U, q), SL(Q, c), sizeof(double) * M); first = 0; continue; }
            for (int z = 0; z < M; z++) SL(U, q)[z] = (Gq[z] > 0) ? (SL(U, q)[z] * SL(Q, c)[z]) / Gq[z] : 0;
        }
        if (first) memcpy(SL(U, q), Gq, sizeof(double) * M);
        if (q > 0) olat_prop1(L, SL(U, q), GOF(o->parent[q]), SL(Q, q));
    }
    memcpy(SL(D, 0), GOF(0), sizeof(double) * M);
    for (int q = 0; q < N; q++) {
        const double *Gq = GOF(q);
        double *phi = o->phi + (size_t)o->seg[q] * M;
        for (int z = 0; z < M; z++) phi[z] += SL(U, q)[z] * SL(D, q)[z];
        for (int c = q + 1; c < N; c++) {
            if (o->parent[c] != q) continue;
            memcpy(acc, SL(D, q), sizeof(double) * M);
            for (int c2 = q + 1; c2 < N; c2++) {
                if (o->parent[c2] != q || c2 == c) continue;
                for (int z = 0; z < M; z++) acc[z] = (Gq[z] > 0) ? (acc[z] * SL(Q, c2)[z]) / Gq[z] : 0;
            }
            olat_prop1(L, acc, GOF(c), SL(D, c));
        }
    }
    o->lngn = olat_lngn(L, SL(U, 0));
    #undef SL
    #undef GOF
    for (int a = 0; a < o->nseg_used; a++) {
        double *phi = o->phi + (size_t)o->used[a] * M;
        const double *G1 = s->swf + (size_t)o->used[a] * M;
        for (int z = 0; z < M; z++) { if (G1[z] > 0) phi[z] /= G1[z]; else phi[z] = 0; }
    }
    double norm;
    if (o->freedom == SFGPU_MOL_RESTRICTED) {
        o->lnc = log(o->theta) - o->lngn - log(1.0 * N);
        o->phibulk = o->theta / exp(o->lngn);
        norm = (o->theta / N) / exp(o->lngn);
    } else {
        o->lnc = log(o->phibulk / N);
        norm = o->phibulk / N;
    }
    for (int a = 0; a < o->nseg_used; a++) {
        double *phi = o->phi + (size_t)o->used[a] * M;
        for (int z = 0; z < M; z++) phi[z] *= norm;
        olat_set_boundaries(L, phi);
    }
    free(U); free(Q); free(D); free(acc);
}

/* SF_HomoRing1stO::Matrix1 (SF_HomoRing1stO.cpp:110-160) as the reference
   loops it, 1-based: per site k a walk from k over sites 1 .. Mmax (G = 1
   beyond the lattice, site 0 absorbing), phi(k) = NORM[k] / NORM[0] phibulk.
   lnGN and ln Cb keep their initial 0 there (SF_Molecule.cpp:269), which the
   free energy's entropy term then reads. */
static void molecule_phi_ring(orc_system *s, omol *o) {
    int M = s->L.M, N = o->N;
    int Mmax = (N / 2 > M) ? 2 * M : M + N / 2;
    const double *G0 = s->swf + (size_t)o->seg[0] * M;   /* 0-based */
    double *phi = o->phi + (size_t)o->seg[0] * M;
    double *Y = calloc(Mmax + 1, sizeof(double));
    for (int k = 1; k <= M; k++) {
        for (int z = 1; z <= Mmax; z++) Y[z] = (z == k) ? G0[z - 1] : 0;
        for (int st = 1; st < N / 2; st++) {
            int zmin = k - st; if (zmin < 1) zmin = 1;
            int zmax = k + st; if (zmax > Mmax) zmax = Mmax;
            double a, b = Y[zmin - 1], c = Y[zmin];
            Y[Mmax] = Y[Mmax - 1];
            for (int z = zmin; z < zmax; z++) {
                a = b; b = c; c = Y[z + 1];
                double gz = (z <= M) ? G0[z - 1] / 6.0 : 1.0 / 6.0;
                Y[z] = gz * (a + 4 * b + c);
            }
        }
        double nk = 0;
        for (int z = 1; z <= Mmax; z++) nk += Y[z] * Y[z];
        phi[k - 1] = nk / o->ring_norm0 * o->phibulk;
    }
    olat_set_boundaries(&s->L, phi);   /* SF_SegmentList.cpp:524-525, as the contact averages read it */
    free(Y);
    o->lngn = 0;
    o->lnc = 0;
}

static void molecule_phi(orc_system *s, omol *o) {
    if (s->L.logmode) { molecule_phi_log(s, o); return; }
    if (o->tree || o->ring) {
        for (int a = 0; a < o->nseg_used; a++) memset(o->phi + (size_t)o->used[a] * s->L.M, 0, sizeof(double) * s->L.M);
        if (o->tree) molecule_phi_tree(s, o); else molecule_phi_ring(s, o);
        return;
    }
    if (o->ngen) { for (int a = 0; a < o->nseg_used; a++) memset(o->phi + (size_t)o->used[a] * s->L.M, 0, sizeof(double) * s->L.M);
                   molecule_phi_dend(s, o); return; }
    olat *L = &s->L;
    int M = L->M, N = o->N, K = L->K;
    size_t KM = (size_t)K * M;
    for (int a = 0; a < o->nseg_used; a++) memset(o->phi + (size_t)o->used[a] * M, 0, sizeof(double) * M);
    if (o->type == 0) {
        int i = o->seg[0];
        const double *G = s->swf + (size_t)i * M;
        double *phi = o->phi + (size_t)i * M;
        memcpy(phi, G, sizeof(double) * M);
        double *Gk = malloc(sizeof(double) * KM);
        for (int k = 0; k < K; k++) memcpy(Gk + (size_t)k * M, G, sizeof(double) * M);
        o->lngn = olat_lngn(L, Gk);
        free(Gk);
        if (o->freedom == SFGPU_MOL_RESTRICTED) {
            o->lnc = log(o->theta) - o->lngn;
            double norm = o->theta / exp(o->lngn);
            for (int z = 0; z < M; z++) phi[z] *= norm;
            o->phibulk = o->theta / exp(o->lngn);
        } else {
            o->lnc = log(o->phibulk);
            for (int z = 0; z < M; z++) phi[z] *= o->phibulk;
        }
        return;
    }
    if (o->type == 1 && K == 1) {
        /* symmetric half chain */
        int i = o->seg[0];
        const double *G = s->swf + (size_t)i * M;
        double *phi = o->phi + (size_t)i * M;
        int half = N / 2;
        double *Gi = malloc(sizeof(double) * M * (size_t)half);
        double *Ginv = malloc(sizeof(double) * M), *tmp = malloc(sizeof(double) * M);
        memcpy(Gi, G, sizeof(double) * M);
        for (int t = 1; t < half; t++) olat_prop1(L, Gi + (size_t)(t - 1) * M, G, Gi + (size_t)t * M);
        memcpy(Ginv, Gi + (size_t)(half - 1) * M, sizeof(double) * M);
        if (N % 2 == 1) {
            olat_prop1(L, Ginv, G, tmp); memcpy(Ginv, tmp, sizeof(double) * M);
            for (int z = 0; z < M; z++) phi[z] += Ginv[z] * Ginv[z];
            for (int z = 0; z < M; z++) phi[z] *= 0.5;
        }
        for (int sp = (N + 3) / 2; sp <= N; sp++) {
            int sinv = N - sp + 1;
            olat_prop1(L, Ginv, G, tmp); memcpy(Ginv, tmp, sizeof(double) * M);
            const double *Gb = Gi + (size_t)(sinv - 1) * M;
            for (int z = 0; z < M; z++) phi[z] += Ginv[z] * Gb[z];
        }
        for (int z = 0; z < M; z++) { if (G[z] > 0) phi[z] /= G[z]; else phi[z] = 0; }
        o->lngn = olat_lngn(L, Ginv);
        if (o->freedom == SFGPU_MOL_RESTRICTED) {
            o->lnc = log(o->theta) - o->lngn - log(1.0 * N);
            double norm = (2 * o->theta / N) / exp(olat_lngn(L, Ginv));
            for (int z = 0; z < M; z++) phi[z] *= norm;
            o->phibulk = o->theta / exp(o->lngn);
        } else {
            double norm = 2 * o->phibulk / N;
            for (int z = 0; z < M; z++) phi[z] *= norm;
            o->lnc = log(o->phibulk / N);
        }
        free(Gi); free(Ginv); free(tmp);
        return;
    }
    /* copolymer (1st order) and every 2nd-order chain: full storage */
    double *Gi = malloc(sizeof(double) * KM * (size_t)N);
    double *Ginv = malloc(sizeof(double) * KM), *tmp = malloc(sizeof(double) * KM);
    const double *G1 = s->swf + (size_t)o->seg[0] * M;
    for (int k = 0; k < K; k++) memcpy(Gi + (size_t)k * M, G1, sizeof(double) * M);
    if (K == 6) olat_set_boundaries6(L, Gi);
    for (int t = 1; t < N; t++) {
        int sg = o->seg[t];
        double S = s->pf[o->seg[t - 1] * s->nseg + sg];
        if (o->force != 0) {   /* SF_Copol1stO.cpp:1207-1211: PropagateG(Gi, G, s, force) */
            olat_prop1_force(L, Gi + (size_t)(t - 1) * KM, s->swf + (size_t)sg * M, Gi + (size_t)t * KM, o->force);
        } else if (L->stiff && K == 6) {
            /* SF_Copol2ndO_stiff_range::Matrix1, SF_Copol2ndO_stiff_range.cpp:211-217:
               Pf(s-1, s+1) (1-based s), the last step isotropic */
            int last = (t == N - 1);
            S = last ? 0.2 : s->pf[o->seg[t - 1] * s->nseg + o->seg[t + 1]];
            olat_prop2_var(L, Gi + (size_t)(t - 1) * KM, s->swf + (size_t)sg * M, S, Gi + (size_t)t * KM, 0, last);
        } else
            propagate_any(s, Gi + (size_t)(t - 1) * KM, s->swf + (size_t)sg * M, S, Gi + (size_t)t * KM, 0);
    }
    const double *GN = s->swf + (size_t)o->seg[N - 1] * M;
    for (int k = 0; k < K; k++) memcpy(Ginv + (size_t)k * M, GN, sizeof(double) * M);
    if (K == 6) olat_set_boundaries6(L, Ginv);
    if (K > 1) {
        for (int a = 0; a < o->nseg_used; a++) memset(o->ori + (size_t)o->used[a] * 3 * M, 0, sizeof(double) * 3 * M);
        orient_acc(L, Ginv, Gi + (size_t)(N - 1) * KM, o->ori + (size_t)o->seg[N - 1] * 3 * M);
    }
    {
        double *phi = o->phi + (size_t)o->seg[N - 1] * M;
        const double *Gf = Gi + (size_t)(N - 1) * KM;
        for (int k = 0; k < K; k++) {
            double mu = comp_mult(K, k);
            for (int z = 0; z < M; z++) {
                double v = Ginv[(size_t)k * M + z] * Gf[(size_t)k * M + z];
                phi[z] += (mu == 1.0) ? v : v * mu;
            }
        }
    }
    for (int t = N - 2; t >= 0; t--) {
        int sg = o->seg[t];
        double S = s->pf[sg * s->nseg + o->seg[t + 1]];
        if (o->force != 0) {   /* backward with -force, SF_Copol1stO.cpp:1226-1230 */
            olat_prop1_force(L, Ginv, s->swf + (size_t)sg * M, tmp, -o->force);
        } else if (L->stiff && K == 6) {
            /* backward: Pf(s, s+2), the first step (s = N-1) isotropic,
               SF_Copol2ndO_stiff_range.cpp:229-234 */
            int firstb = (t == N - 2);
            S = firstb ? 0.2 : s->pf[sg * s->nseg + o->seg[t + 2]];
            olat_prop2_var(L, Ginv, s->swf + (size_t)sg * M, S, tmp, 1, firstb);
        } else
            propagate_any(s, Ginv, s->swf + (size_t)sg * M, S, tmp, 1);
        memcpy(Ginv, tmp, sizeof(double) * KM);
        if (K > 1) orient_acc(L, Ginv, Gi + (size_t)t * KM, o->ori + (size_t)sg * 3 * M);
        double *phi = o->phi + (size_t)sg * M;
        const double *Gf = Gi + (size_t)t * KM;
        for (int k = 0; k < K; k++) {
            double mu = comp_mult(K, k);
            for (int z = 0; z < M; z++) {
                double v = Ginv[(size_t)k * M + z] * Gf[(size_t)k * M + z];
                phi[z] += (mu == 1.0) ? v : v * mu;
            }
        }
    }
    o->lngn = olat_lngn(L, Ginv);
    for (int a = 0; a < o->nseg_used; a++) {
        int i = o->used[a];
        double *phi = o->phi + (size_t)i * M;
        const double *G = s->swf + (size_t)i * M;
        for (int z = 0; z < M; z++) { if (G[z] > 0) phi[z] /= G[z]; else phi[z] = 0; }
    }
    double norm;
    if (o->freedom == SFGPU_MOL_RESTRICTED) {
        o->lnc = log(o->theta) - o->lngn - log(1.0 * N);
        o->phibulk = o->theta / exp(o->lngn);
        norm = (o->theta / N) / (K > 1 ? 6.0 * exp(o->lngn) : exp(o->lngn));
    } else {
        o->lnc = log(o->phibulk / N);
        norm = o->phibulk / (K > 1 ? 6.0 * N : (double)N);
    }
    for (int a = 0; a < o->nseg_used; a++) {
        double *phi = o->phi + (size_t)o->used[a] * M;
        for (int z = 0; z < M; z++) phi[z] *= norm;
    }
    /* CorrectDoubleCountG / NormPhi* on the orientation slots
       (Lat3D2ndO.cpp:986-993, :1031-1046; Lat1D2ndO.cpp:281-289, :309-327) */
    if (K > 1)
        for (int a = 0; a < o->nseg_used; a++) {
            const double *G = s->swf + (size_t)o->used[a] * M;
            double *ori = o->ori + (size_t)o->used[a] * 3 * M;
            for (int sl = 0; sl < 3; sl++)
                for (int z = 0; z < M; z++) {
                    double v = ori[(size_t)sl * M + z];
                    ori[(size_t)sl * M + z] = ((G[z] > 0) ? v / G[z] : 0.0) * norm;
                }
        }
    free(Gi); free(Ginv); free(tmp);
}

/* SF_MolList1stO::ComputePhi (SF_MolList1stO.cpp:246-295) */
/* SF_Molecule::GetBulkCharge (SF_Molecule.cpp:803-818): valence times the
   number of each segment in one molecule */
static double mol_bulk_charge(const orc_system *s, const omol *o) {
    double q = 0;
    for (int a = 0; a < o->nseg_used; a++) q += 1.0 * s->val[o->used[a]] * o->count[o->used[a]];
    return q;
}

static void compute_phi(orc_system *s) {
    int M = s->L.M;
    double phib_solv = 1.0;
    double bulkcharge = 0;
    for (int m = 0; m < s->nmol; m++) {
        if (m == s->solvent || m == s->neutralizer) continue;
        omol *o = &s->mol[m];
        molecule_phi(s, o);
        if (o->pinned) o->phibulk = 0;   /* SF_Homopol1stO.cpp:124-125 */
        bulkcharge += mol_bulk_charge(s, o) * o->phibulk / o->N;
    }
    if (s->neutralizer >= 0) {
        /* SF_MolList1stO.cpp:250-266 */
        omol *o = &s->mol[s->neutralizer];
        o->phibulk = -bulkcharge * o->N / mol_bulk_charge(s, o);
        molecule_phi(s, o);
    }
    for (int m = 0; m < s->nmol; m++)
        if (m != s->solvent) phib_solv -= s->mol[m].phibulk;
    s->mol[s->solvent].phibulk = phib_solv;
    molecule_phi(s, &s->mol[s->solvent]);
    /* state phi and bulk values */
    for (int i = 0; i < s->nseg; i++) {
        double *p = s->phi + (size_t)i * M;
        s->phib[i] = 0;
        if (s->freedom[i] == SFGPU_SEG_FROZEN) {
            memcpy(p, s->range + (size_t)i * M, sizeof(double) * M);
            olat_set_boundaries(&s->L, p);   /* SF_Segment.cpp:428-433 */
            continue;
        }
        memset(p, 0, sizeof(double) * M);
        for (int m = 0; m < s->nmol; m++) {
            omol *o = &s->mol[m];
            if (!o->count[i]) continue;
            const double *q = o->phi + (size_t)i * M;
            for (int z = 0; z < M; z++) p[z] += q[z];
            s->phib[i] += o->phibulk * ((double)o->count[i] / o->N);
        }
    }
}

/* SF_Solve::GetResiduals (SF_Solve.cpp:527-591) with PutSides/ChemInt/
   ChemIntBulk/GetPhiTotal (SF_SegmentList.cpp:512-744) */
static void get_residuals(orc_system *s, double *f) {
    int M = s->L.M, ns = s->nseg, nc = s->nclass;
    if (s->charged) {
        /* SF_SegmentList::ComputeElectricPotential(psi0) (SF_SegmentList.cpp:
           839-860) before PutSides, with the layer-averaged epsilon
           (GetAverageEpsilon, :785-799) */
        double *epsav = calloc(M, sizeof(double)), *charge = malloc(sizeof(double) * M);
        for (int i = 0; i < ns; i++)
            for (int z = 0; z < M; z++) epsav[z] += s->phi[(size_t)i * M + z] * s->eps[i];
        state_charge(s, charge);
        const double pfp = (ORC_ELEM_CHARGE / ORC_EPS0) / s->sitedist;
        if (s->L.grad == 3) olat_poisson_3d(&s->L, s->psi0, epsav, charge, pfp, s->psi);
        else if (s->L.grad == 2 && s->L.cyl) olat_poisson_2dcyl(&s->L, s->psi0, epsav, charge, pfp, s->psi);
        else if (s->L.grad == 2) olat_poisson_2dflat(&s->L, s->psi0, epsav, charge, pfp, s->psi);
        else if (s->L.cyl) olat_poisson_curved(&s->L, s->psi0, epsav, charge, pfp, s->psi);
        else olat_poisson_flat(&s->L, s->psi0, epsav, charge, pfp, s->psi);
        free(epsav); free(charge);
    }
    for (int i = 0; i < ns; i++) olat_side(&s->L, s->phi + (size_t)i * M, s->rho + (size_t)i * M);
    double *upr = malloc(sizeof(double) * nc);
    if (s->charged) {
        const double kT = ORC_BOLTZMANN * s->temperature;
        for (int z = 0; z < M; z++) {
            if (s->xp[z] >= 0) f[s->xp[z]] = s->psi0[z] - s->psi[z];
            if (s->xu[z] < 0) continue;
            double phit = 0;
            for (int i = 0; i < ns; i++) phit += s->phi[(size_t)i * M + z];
            double av = 0;
            for (int c = 0; c < nc; c++) {
                int st = s->rep_of_class[c];
                double u = -log(s->swf_full[(size_t)st * M + z]);
                double ci = 0, cb = 0;
                for (int i = 0; i < ns; i++) {
                    double x = s->chi[st * ns + i];
                    if (x != 0) { ci += x * s->rho[(size_t)i * M + z]; cb += x * s->phib[i]; }
                }
                u -= ci / phit;
                u += cb;
                u -= s->val[st] * s->psi0[z] * ORC_ELEM_CHARGE / kT;
                if (s->diffeps) u += 0.5 * s->eps[st] * s->esq[z];
                upr[c] = u; av += u;
            }
            av /= nc;
            for (int c = 0; c < nc; c++) f[s->xu[z] + c] = -1.0 + 1.0 / phit + upr[c] - av;
        }
        free(upr);
        return;
    }
    for (int j = 0; j < s->nsites; j++) {
        int z = s->sites[j];
        double phit = 0;
        for (int i = 0; i < ns; i++) phit += s->phi[(size_t)i * M + z];
        double av = 0;
        for (int c = 0; c < nc; c++) {
            int st = s->rep_of_class[c];
            double u = -log(s->swf_full[(size_t)st * M + z]);
            double ci = 0, cb = 0;
            for (int i = 0; i < ns; i++) {
                double x = s->chi[st * ns + i];
                if (x != 0) { ci += x * s->rho[(size_t)i * M + z]; cb += x * s->phib[i]; }
            }
            u -= ci / phit;
            u += cb;
            upr[c] = u; av += u;
        }
        av /= nc;
        for (int c = 0; c < nc; c++) f[j * nc + c] = -1.0 + 1.0 / phit + upr[c] - av;
    }
    free(upr);
}

int orc_residual(orc_system *s, const double *x, double *f) {
    update_swf(s, x);
    compute_phi(s);
    get_residuals(s, f);
    s->evaluated = 1;
    return SFGPU_OK;
}

int orc_get_phi(const orc_system *s, int seg, double *phi) {
    if (seg < 0 || seg >= s->nseg) return SFGPU_ERR_INVALID;
    memcpy(phi, s->phi + (size_t)seg * s->L.M, sizeof(double) * s->L.M);
    return SFGPU_OK;
}
int orc_get_mol_phi(const orc_system *s, int mol, int seg, double *phi) {
    if (mol < 0 || mol >= s->nmol || seg < 0 || seg >= s->nseg) return SFGPU_ERR_INVALID;
    memcpy(phi, s->mol[mol].phi + (size_t)seg * s->L.M, sizeof(double) * s->L.M);
    return SFGPU_OK;
}
double orc_get_lngn(const orc_system *s, int mol) { return s->mol[mol].lngn; }
double orc_get_phibulk(const orc_system *s, int mol) { return s->mol[mol].phibulk; }
int orc_get_swf(const orc_system *s, int seg, double *g) {
    memcpy(g, s->swf + (size_t)seg * s->L.M, sizeof(double) * s->L.M);
    return SFGPU_OK;
}

/* SF_MolList1stO::GetFreeEnergy (SF_MolList1stO.cpp:606-635) with
   GetEntropyProfile (:827-911) and GetContactInteractionsProfile (:914-940) */
/* SF_MolList1stO::GetElectricInteractionsProfile (SF_MolList1stO.cpp:942-952):
   1/2 psi q e / kT per layer, q = GetCharge / lattice sites, psi the
   potential of the last Poisson sweep; NULL when the system has no charges */
static double *elec_profile(const orc_system *s) {
    if (!s->charged) return NULL;
    int M = s->L.M;
    double *q = malloc(sizeof(double) * M);
    state_charge(s, q);
    for (int z = 0; z < M; z++) {   /* DivideByLatticeSites: the 1D curved lattices skip zero
                                       entries, the 2D cylinder rows without sites */
        if (s->L.grad == 2 && s->L.cyl) { if (s->lsites[z] != 0) q[z] /= s->lsites[z]; }
        else if (!s->L.cyl || q[z] != 0) q[z] /= s->lsites[z];
    }
    const double kT = ORC_BOLTZMANN * s->temperature;
    for (int z = 0; z < M; z++) q[z] = 0.5 * s->psi[z] * q[z] * ORC_ELEM_CHARGE / kT;
    return q;
}

double orc_free_energy(orc_system *s) {
    if (!s->evaluated) return NAN;
    int M = s->L.M, ns = s->nseg;
    double F = 0;
    double *el = elec_profile(s);
    for (int z = 0; z < M; z++) {
        double w = s->L.w_f[z];
        if (w == 0) continue;
        double entropy = 0, contact = 0;
        for (int m = 0; m < s->nmol; m++) {
            omol *o = &s->mol[m];
            double phim = 0;
            for (int a = 0; a < o->nseg_used; a++) phim += o->phi[(size_t)o->used[a] * M + z];
            entropy -= (phim / o->N) * (log((double)o->N) + o->lnc);
            contact -= phim * o->chemintref;
        }
        for (int m = 0; m < s->nmol; m++) {
            omol *o = &s->mol[m];
            for (int a = 0; a < o->nseg_used; a++) {
                int i = o->used[a];
                double G = s->swf[(size_t)i * M + z];
                if (G > 0) entropy -= o->phi[(size_t)i * M + z] * log(G);
            }
        }
        for (int i = 0; i < ns; i++) {
            double ci = 0;
            for (int j = 0; j < ns; j++) {
                double x = s->chi[i * ns + j];
                if (x != 0) ci += x * s->rho[(size_t)j * M + z];
            }
            contact += 0.5 * s->phi[(size_t)i * M + z] * ci;
        }
        F += w * (-entropy + contact + (el ? el[z] : 0.0));
    }
    free(el);
    return F;
}

/* The free-energy density (SF_MolList1stO::GetFreeEnergyProfile,
   SF_MolList1stO.cpp:815-826) and the grand-potential density
   (GetGrandPotentialProfile, :1001-1101; the same in SF_MolList2ndO.cpp)
   without charges, external potentials or grafted chains, both after
   SubtractBoundaries; F and Omega = sum_z L(z) density(z)
   (GetFreeEnergy :606-635, GetGrandPotential :636-646). */
int orc_thermo(orc_system *s, double *F, double *Omega, double *fe, double *gp) {
    if (!s->evaluated) return SFGPU_ERR_INVALID;
    int M = s->L.M, ns = s->nseg;
    double Ft = 0, Ot = 0;
    double *el = elec_profile(s);
    const double kT = ORC_BOLTZMANN * s->temperature;
    for (int z = 0; z < M; z++) {
        double entropy = 0, contact = 0, omega = 0;
        for (int m = 0; m < s->nmol; m++) {
            omol *o = &s->mol[m];
            double phim = 0;
            for (int a = 0; a < o->nseg_used; a++) phim += o->phi[(size_t)o->used[a] * M + z];
            entropy -= (phim / o->N) * (log((double)o->N) + o->lnc);
            contact -= phim * o->chemintref;
        }
        for (int m = 0; m < s->nmol; m++) {
            omol *o = &s->mol[m];
            for (int a = 0; a < o->nseg_used; a++) {
                int i = o->used[a];
                double G = s->swf[(size_t)i * M + z];
                if (G > 0) entropy -= o->phi[(size_t)i * M + z] * log(G);
            }
        }
        for (int i = 0; i < ns; i++) {
            double ci = 0;
            for (int j = 0; j < ns; j++) {
                double x = s->chi[i * ns + j];
                if (x != 0) ci += x * s->rho[(size_t)j * M + z];
            }
            contact += 0.5 * s->phi[(size_t)i * M + z] * ci;
        }
        /* grand potential: molecules, then u' of every liquid state, then the
           contact pairs of liquid states, in the reference's order */
        for (int m = 0; m < s->nmol; m++) {
            omol *o = &s->mol[m];
            double phim = 0;
            for (int a = 0; a < o->nseg_used; a++) phim += o->phi[(size_t)o->used[a] * M + z];
            if (phim > 0) omega -= (phim - o->phibulk) / o->N;
        }
        for (int i = 0; i < ns; i++) {
            if (s->freedom[i] == SFGPU_SEG_FROZEN) continue;
            double G = s->swf_full[(size_t)i * M + z], up = 0;
            if (G > 0) {
                double ci = 0, cb = 0;
                for (int j = 0; j < ns; j++) {
                    double x = s->chi[i * ns + j];
                    if (x != 0) { ci += x * s->rho[(size_t)j * M + z]; cb += x * s->phib[j]; }
                }
                up = -log(G);
                up -= ci;
                up += cb;
                if (s->charged) up -= s->val[i] * s->psi[z] * ORC_ELEM_CHARGE / kT;
            }
            omega -= up * s->phi[(size_t)i * M + z];
        }
        for (int i = 0; i < ns; i++) {
            if (s->freedom[i] == SFGPU_SEG_FROZEN) continue;
            double p1 = s->phi[(size_t)i * M + z];
            for (int j = 0; j < ns; j++) {
                if (s->freedom[j] == SFGPU_SEG_FROZEN) continue;
                double x = s->chi[i * ns + j];
                omega -= 0.5 * x * p1 * s->rho[(size_t)j * M + z];
                if (p1 > 0) omega += 0.5 * x * s->phib[i] * s->phib[j];
            }
        }
        if (el) {
            /* SF_MolList1stO.cpp:1074-1096: added on a frozen segment's
               layers, subtracted elsewhere */
            int surface = 0;
            for (int i = 0; i < ns; i++)
                if (s->freedom[i] == SFGPU_SEG_FROZEN && s->range[(size_t)i * M + z] > 0) surface = 1;
            /* the electric profile arrives with its boundaries already
               subtracted and the sum is subtracted once more (SF_MolList1stO.cpp:
               952, :1098): mirror2 layers take it at 1/4 */
            omega += surface ? el[z] * s->L.sb[z] : -el[z] * s->L.sb[z];
        }
        double f = -entropy + contact + (el ? el[z] : 0.0);
        Ft += s->L.w_f[z] * f;
        Ot += s->L.w_f[z] * omega;
        if (fe) fe[z] = f * s->L.sb[z];
        if (gp) gp[z] = omega * s->L.sb[z];
    }
    if (F) *F = Ft;
    if (Omega) *Omega = Ot;
    free(el);
    return SFGPU_OK;
}

int orc_propagate(const orc_system *s, const double *gin, const double *g, double *gout, double S, int backward) {
    int M = s->L.M, K = s->L.K;
    double *tmp = malloc(sizeof(double) * K * M);
    memcpy(tmp, gin, sizeof(double) * K * M);
    if (s->L.logmode) {   /* the *1stOS step on logarithms */
        olat_log_boundaries(&s->L, tmp);
        olat_prop1_log(&s->L, tmp, g, gout);
        free(tmp);
        return SFGPU_OK;
    }
    if (K == 6) olat_set_boundaries6(&s->L, tmp);
    else if (K > 1) olat_set_boundaries_lumped(&s->L, tmp);
    else olat_set_boundaries(&s->L, tmp);
    propagate_any(s, tmp, g, S, gout, backward);
    free(tmp);
    return SFGPU_OK;
}
/* one stiff_range (iso = 0) or isotropic (iso = 1) 3D second-order step,
   6*M values, with the lattice's stiff_range mask */
int orc_propagate_stiff(const orc_system *s, const double *gin, const double *g, double *gout, double S,
                        int backward, int iso) {
    int M = s->L.M;
    if (s->L.K != 6 || (!iso && !s->L.stiff)) return SFGPU_ERR_INVALID;
    double *tmp = malloc(sizeof(double) * 6 * M);
    memcpy(tmp, gin, sizeof(double) * 6 * M);
    olat_set_boundaries6(&s->L, tmp);
    olat_prop2_var(&s->L, tmp, g, S, gout, backward, iso);
    free(tmp);
    return SFGPU_OK;
}

/* lnGN of a propagator at the lattice level: ComputeLnGN (on logarithms
   with overflow protection) */
int orc_lat_lngn(const orc_system *s, const double *g, double *lngn) {
    *lngn = s->L.logmode ? olat_lngn_log(&s->L, g) : olat_lngn(&s->L, g);
    return SFGPU_OK;
}
int orc_side(const orc_system *s, const double *phi, double *rho) { olat_side(&s->L, phi, rho); return SFGPU_OK; }
int orc_site_weights(const orc_system *s, double *w) { memcpy(w, s->L.w_gn, sizeof(double) * s->L.M); return SFGPU_OK; }
int orc_set_boundaries(const orc_system *s, double *p) { olat_set_boundaries(&s->L, p); return SFGPU_OK; }

/* ------------------------------------------------------------------------ */
/* Pure_DIIS                                                                 */
/* ------------------------------------------------------------------------ */
/* cyclic Jacobi eigen-decomposition of a small symmetric matrix (Golub and
   Van Loan, Matrix Computations, 4th ed., sec. 8.5): A = Q diag(ev) Q^T */
static void jacobi_eig(int n, double *A, double *Q, double *ev) {
    for (int i = 0; i < n; i++) for (int j = 0; j < n; j++) Q[i * n + j] = (i == j);
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0, tot = 0;
        for (int i = 0; i < n; i++) for (int j = 0; j < n; j++) {
            tot += A[i * n + j] * A[i * n + j];
            if (i != j) off += A[i * n + j] * A[i * n + j];
        }
        if (off <= 1e-30 * tot || off == 0) break;
        for (int p = 0; p < n; p++) for (int q = p + 1; q < n; q++) {
            double apq = A[p * n + q];
            if (apq == 0) continue;
            double theta = (A[q * n + q] - A[p * n + p]) / (2 * apq);
            double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1));
            double c = 1 / sqrt(t * t + 1), sn = t * c;
            for (int k = 0; k < n; k++) {
                double akp = A[k * n + p], akq = A[k * n + q];
                A[k * n + p] = c * akp - sn * akq; A[k * n + q] = sn * akp + c * akq;
            }
            for (int k = 0; k < n; k++) {
                double apk = A[p * n + k], aqk = A[q * n + k];
                A[p * n + k] = c * apk - sn * aqk; A[q * n + k] = sn * apk + c * aqk;
            }
            for (int k = 0; k < n; k++) {
                double qkp = Q[k * n + p], qkq = Q[k * n + q];
                Q[k * n + p] = c * qkp - sn * qkq; Q[k * n + q] = sn * qkp + c * qkq;
            }
        }
    }
    for (int i = 0; i < n; i++) ev[i] = A[i * n + i];
}

/* coefficients c = A^-1 * 1 of the DIIS Gram matrix (SFNewton::Ax,
   sfnewton.cpp:531-557, which forms V S^-1 U^T 1 from an SVD) */
static void diis_coeff(int n, const double *A, double *c) {
    double *B = malloc(sizeof(double) * n * n), *Q = malloc(sizeof(double) * n * n), *ev = malloc(sizeof(double) * n);
    memcpy(B, A, sizeof(double) * n * n);
    jacobi_eig(n, B, Q, ev);
    for (int i = 0; i < n; i++) c[i] = 0;
    for (int k = 0; k < n; k++) {
        double proj = 0;
        for (int i = 0; i < n; i++) proj += Q[i * n + k];
        double t = proj / ev[k];
        for (int i = 0; i < n; i++) c[i] += Q[i * n + k] * t;
    }
    free(B); free(Q); free(ev);
}

static double dot(const double *a, const double *b, int n) {
    double r = 0; for (int i = 0; i < n; i++) r += a[i] * b[i]; return r;
}

/* SFNewton::PlainLBFGSDIIS, sfnewton.cpp:566-664 */
int orc_solve_diis(orc_system *s, double *x, double tol, int maxit, int m, double eta,
                   int *iterations, double *final_error) {
    int iv = s->nvar;
    double *g = malloc(sizeof(double) * iv), *x0 = malloc(sizeof(double) * iv);
    double *XR = malloc(sizeof(double) * iv * (size_t)m), *XX0 = malloc(sizeof(double) * iv * (size_t)m);
    double *Aij = calloc((size_t)m * m, sizeof(double)), *Ap = calloc((size_t)m * m, sizeof(double));
    double *C = calloc(m, sizeof(double));
    int k = 0, it = 0, kd = 1, rc = SFGPU_OK;
    orc_residual(s, x, g);
    memcpy(x0, x, sizeof(double) * iv);
    for (int i = 0; i < iv; i++) x[i] = -eta * g[i];
    for (int i = 0; i < iv; i++) XX0[i] = x[i] - x0[i];
    memcpy(XR, x, sizeof(double) * iv);
    double err = sqrt(dot(g, g, iv));
    while (tol < err && it < maxit) {
        it++;
        memcpy(x0, x, sizeof(double) * iv);
        orc_residual(s, x, g);
        for (int i = 0; i < iv; i++) x[i] -= g[i] * eta;
        k = it % m; kd++;
        memcpy(XR + (size_t)k * iv, x, sizeof(double) * iv);
        for (int i = 0; i < iv; i++) XX0[(size_t)k * iv + i] = x[i] - x0[i];
        if (kd > m) {
            kd = m;
            for (int i = 1; i < m; i++) for (int j = 1; j < m; j++) Aij[m * (i - 1) + j - 1] = Aij[m * i + j];
        }
        for (int i = 0; i < kd; i++) {
            int posi = k - kd + 1 + i; if (posi < 0) posi += m;
            Aij[i + m * (kd - 1)] = Aij[kd - 1 + m * i] = dot(XX0 + (size_t)posi * iv, XX0 + (size_t)k * iv, iv);
        }
        for (int i = 0; i < kd; i++) for (int j = 0; j < kd; j++) Ap[j + kd * i] = Aij[j + m * i];
        diis_coeff(kd, Ap, C);
        double nc = 0;
        for (int i = 0; i < kd; i++) nc += C[i];
        for (int i = 0; i < kd; i++) C[i] /= nc;
        int posi = k - kd + 1; if (posi < 0) posi += m;
        for (int i = 0; i < iv; i++) x[i] = C[0] * XR[(size_t)posi * iv + i];
        for (int q = 1; q < kd; q++) {
            posi = k - kd + 1 + q; if (posi < 0) posi += m;
            for (int i = 0; i < iv; i++) x[i] += C[q] * XR[(size_t)posi * iv + i];
        }
        err = sqrt(dot(g, g, iv));
        if (!isfinite(err)) { rc = SFGPU_ERR_NONFINITE; break; }
    }
    if (rc == SFGPU_OK && err > tol) rc = SFGPU_ERR_NOTCONVERGED;
    if (iterations) *iterations = it;
    if (final_error) *final_error = err;
    free(g); free(x0); free(XR); free(XX0); free(Aij); free(Ap); free(C);
    return rc;
}

/* SF_Homopol2ndO::GetBondOrientation (SF_Homopol2ndO.cpp:82-90) and
   SF_Copol2ndO::GetBondOrientation (SF_Copol2ndO.cpp:108-116): slot axis of
   the molecule, summed over its segment types */
int orc_bond_orientation(const orc_system *s, int mol, int axis, double *out) {
    if (s->L.K == 1 || mol < 0 || mol >= s->nmol) return SFGPU_ERR_INVALID;
    if (axis < 0 || axis >= (s->L.K == 3 ? 2 : 3)) return SFGPU_ERR_INVALID;
    const omol *o = &s->mol[mol];
    int M = s->L.M;
    for (int z = 0; z < M; z++) out[z] = 0;
    if (o->type == 0) return SFGPU_OK;
    for (int a = 0; a < o->nseg_used; a++) {
        const double *src = o->ori + ((size_t)o->used[a] * 3 + axis) * M;
        for (int z = 0; z < M; z++) out[z] += src[z];
    }
    return SFGPU_OK;
}
