// sfgpu_system.cu -- one SF-SCF system on one GPU: set-up of the lattice and
// molecules, the residual evaluation x -> f (SF_Solve::residuals,
// SF_Solve.cpp:647-651), free energy, the Lattice-level entry points and the
// host-driven Pure_DIIS iteration (the plain GPU form).
#include <cmath>
#include <cfloat>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>
#include "sfgpu_kernels.cuh"
#include "sfgpu_system.h"

static thread_local char g_errmsg[512] = "";

void sfgpu_set_error(cudaError_t e, const char *what, const char *file, int line) {
    snprintf(g_errmsg, sizeof(g_errmsg), "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
}
static int fail(int code, const char *msg) {
    snprintf(g_errmsg, sizeof(g_errmsg), "%s", msg);
    return code;
}

int fail_unsupported(const char *what) {
    snprintf(g_errmsg, sizeof(g_errmsg), "not implemented: %s", what);
    return SFGPU_ERR_UNSUPPORTED;
}

extern "C" const char *sfgpu_last_error(void) { return g_errmsg; }

using namespace sfk;

static int grid_for(long n) {
    long b = (n + kBlock - 1) / kBlock;
    return (int)std::max(1L, std::min(b, 148L * 16));
}

// blocks for a row-wise kernel: one warp per interior row (1D: one thread
// per interior site)
static int grid_rows(const DLat &L) {
    long threads = (L.grad == 1) ? (long)(L.Md[0] - 2) : 32L * lat_nrows(L);
    long b = (threads + kBlock - 1) / kBlock;
    return (int)std::max(1L, std::min(b, 148L * 32));
}

// a step launch with programmatic stream serialization: the kernel may be
// scheduled while the previous one drains and waits for it in pdl_enter()
template <class... KArgs, class... Args>
static cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// first-order step inside a residual evaluation: x-marching tiles on the
// six-neighbour 3D lattices (launched as programmatic dependents of the
// step before), row-wise otherwise
int sfgpu_system::launch_step1(const double *gin, const double *G, double *gout, const double *other, double *phi,
                               int mode) {
    const DLat &L = H.L;
    if (L.grad == 3 && !lat_twelve(L)) {
        const bool composing = mode != COMP_NONE;
        const int xc = composing ? tile_xc_bwd : tile_xc;
        dim3 grid((L.Md[2] - 2 + kTZ - 1) / kTZ, (L.Md[1] - 2 + kTY - 1) / kTY, (L.Md[0] - 2 + xc - 1) / xc);
        const dim3 block(kTZ * kTY);
        cudaError_t e;
        if (!composing && tile_pipelined == 2) {
            grid.y = (L.Md[1] - 2 + kTY2 - 1) / kTY2;
            e = launch_pdl(step3d_march_pf2, grid, block, stream, L, gin, G, gout, xc);
        } else if (composing && tile_pipelined_bwd) {
            e = launch_pdl(step3d_march_pf<true>, grid, block, stream, L, gin, G, gout, other, phi, mode, xc);
        } else if (!composing && tile_pipelined) {
            e = launch_pdl(step3d_march_pf<false>, grid, block, stream, L, gin, G, gout, other, phi, mode, xc);
        } else {
            e = launch_pdl(step3d_march, grid, block, stream, L, gin, G, gout, other, phi, mode, xc);
        }
        if (e != cudaSuccess) { sfgpu_set_error(e, "cudaLaunchKernelEx", __FILE__, __LINE__); return SFGPU_ERR_CUDA; }
    } else {
        const cudaError_t e = launch_pdl(step1_rows, dim3(grid_rows(L)), dim3(kBlock), stream, L, gin, G, gout, other, phi,
                                         mode);
        if (e != cudaSuccess) { sfgpu_set_error(e, "cudaLaunchKernelEx", __FILE__, __LINE__); return SFGPU_ERR_CUDA; }
    }
    return SFGPU_OK;
}

// ---------------------------------------------------------------------------
// lattice set-up (Lat1DFlat.cpp:4-149, Lat2DFlat.cpp:35-220,
// Lat2DCylinder.cpp:7-55, Lat3D.cpp:44-236)
// ---------------------------------------------------------------------------
static int map_lo_of(int bc, int n) {
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

int sfgpu_build_lattice(const sfgpu_lattice_desc *d, HostLat *H) {
    DLat &L = H->L;
    memset(&L, 0, sizeof(L));
    L.grad = d->gradients;
    L.order = d->order;
    // curved lattices: Lat2DCylinder, Lat1DCylinder, Lat1DSphere (the radial
    // coordinate is the first gradient); SF_System.cpp:434-519
    L.cyl = (d->geometry == SFGPU_GEOM_CYLINDRICAL && (d->gradients == 1 || d->gradients == 2)) ||
            (d->geometry == SFGPU_GEOM_SPHERICAL && d->gradients == 1);
    if (L.grad < 1 || L.grad > 3) return fail(SFGPU_ERR_INVALID, "gradients must be 1, 2 or 3");
    if (d->geometry < SFGPU_GEOM_FLAT || d->geometry > SFGPU_GEOM_SPHERICAL) return fail(SFGPU_ERR_INVALID, "unknown geometry");
    if (d->geometry != SFGPU_GEOM_FLAT && !L.cyl)
        return fail(SFGPU_ERR_UNSUPPORTED, "cylindrical geometry needs 1 or 2 gradients, spherical 1");
    if (L.order != 1 && L.order != 2) return fail(SFGPU_ERR_INVALID, "order must be 1 or 2");
    for (int k = 0; k < 3; k++) L.Md[k] = 1;
    for (int k = 0; k < L.grad; k++) {
        int n = d->n_layers[k];
        if (n < 1) return fail(SFGPU_ERR_INVALID, "n_layers must be positive");
        if (L.grad == 3 && n < 3) return fail(SFGPU_ERR_INVALID, "3D lattices need at least 3 layers per gradient");
        int lo = d->bound_lo[k], hi = d->bound_hi[k];
        if (lo < 1 || lo > 4 || hi < 1 || hi > 4) return fail(SFGPU_ERR_INVALID, "unknown boundary condition");
        if ((lo == SFGPU_BOUND_PERIODIC) != (hi == SFGPU_BOUND_PERIODIC))
            return fail(SFGPU_ERR_INVALID, "periodic boundaries must be periodic on both sides");
        if ((lo == SFGPU_BOUND_MIRROR2 || hi == SFGPU_BOUND_MIRROR2) && n < 2)
            return fail(SFGPU_ERR_INVALID, "mirror2 needs at least 2 layers");
        if (L.grad == 3 && (lo == SFGPU_BOUND_SURFACE || hi == SFGPU_BOUND_SURFACE))
            return fail(SFGPU_ERR_INVALID, "the 3D lattice has no surface boundary");
        L.Md[k] = n + 2;
        L.bc_lo[k] = lo; L.bc_hi[k] = hi;
        L.map_lo[k] = map_lo_of(lo, n);
        L.map_hi[k] = map_hi_of(hi, n);
        // component swaps of second-order steps across a boundary: 3D swaps
        // at both mirror kinds (Lat3D::SetBx1(P,Q), Lat3D.cpp:1276-1289).  The
        // flat 1D/2D lattices swap where the 1-based copy layer (surface 1 /
        // n+2, mirror1 2 / n+1, mirror2 3 / n, periodic n+1 / 2) is <= 2 below
        // (Lat1DFlat.cpp:658-666, Lat2DFlat.cpp:1382-1393) or >= n - 1 above
        // (Lat1DFlat.cpp:673-680, Lat2DFlat.cpp:1401-1413), assigning P = Q',
        // Q = P' in that order; at a surface the copy layer is the boundary
        // itself, so the + component takes the - one's value and the - one
        // keeps its own (swap mode 2)
        if (L.grad == 3) {
            L.sw_lo[k] = (lo == SFGPU_BOUND_MIRROR1 || lo == SFGPU_BOUND_MIRROR2);
            L.sw_hi[k] = (hi == SFGPU_BOUND_MIRROR1 || hi == SFGPU_BOUND_MIRROR2);
        } else {
            const int copy_lo = (lo == SFGPU_BOUND_PERIODIC) ? n + 1 : lo;
            const int copy_hi = (hi == SFGPU_BOUND_PERIODIC) ? 2 : (n + 2) - hi + 1;
            L.sw_lo[k] = (copy_lo <= 2) ? (lo == SFGPU_BOUND_SURFACE ? 2 : 1) : 0;
            L.sw_hi[k] = (copy_hi >= n - 1) ? (hi == SFGPU_BOUND_SURFACE ? 2 : 1) : 0;
        }
    }
    L.K = (L.order == 2) ? (L.grad == 1 ? 3 : (L.grad == 2 ? 5 : 6)) : 1;
    L.M = L.Md[0] * L.Md[1] * L.Md[2];
    // lat : stiff_range (Lat3D.cpp:265-268): read by the 3D lattices, used by
    // the second-order copolymers (SF_MolList2ndO.cpp:22-47)
    H->stiff.clear();
    L.stiff = nullptr;
    if (d->stiff_range) {
        if (L.grad != 3) return fail(SFGPU_ERR_INVALID, "stiff_range is a 3D lattice parameter");
        if (L.order == 2) H->stiff.assign(d->stiff_range, d->stiff_range + L.M);
    }
    if (L.grad == 1) { L.st[0] = 1; L.st[1] = 0; L.st[2] = 0; }
    else if (L.grad == 2) { L.st[0] = L.Md[1]; L.st[1] = 1; L.st[2] = 0; }
    else { L.st[0] = L.Md[1] * L.Md[2]; L.st[1] = L.Md[2]; L.st[2] = 1; }
    L.l1 = (L.grad == 3) ? 1.0 / 6.0 : d->lambda;
    // 3D lattice type and its contact weights (Lat3D.cpp:212-259)
    L.ltype = d->lattice_type;
    if (L.ltype < SFGPU_LATTICE_STANDARD || L.ltype > SFGPU_LATTICE_HEX)
        return fail(SFGPU_ERR_INVALID, "unknown lattice_type");
    if (L.ltype != SFGPU_LATTICE_STANDARD && L.grad != 3)
        return fail(SFGPU_ERR_UNSUPPORTED, "lattice types other than standard are built for 3 gradients");
    L.sl[0] = 0; L.sl[1] = 1.0 / 6.0; L.sl[2] = 0; L.sl[3] = 0;
    if (L.ltype == SFGPU_LATTICE_FCC) L.sl[0] = L.sl[1] = L.sl[2] = L.sl[3] = 1.0 / 27.0;
    if (L.ltype == SFGPU_LATTICE_STENCILS) {
        for (int k = 0; k < 4; k++) {
            L.sl[k] = d->lambda_3d[k];
            if (!(L.sl[k] >= 0 && L.sl[k] <= 0.5)) return fail(SFGPU_ERR_INVALID, "lambda0..lambda3 must be in [0, 0.5]");
        }
        double dev = L.sl[0] + 6.0 * L.sl[1] + 12.0 * L.sl[2] + 8.0 * L.sl[3] - 1.0;
        if ((dev < 0 ? -dev : dev) > DBL_EPSILON) return fail(SFGPU_ERR_INVALID, "sum of the lambdas is not 1");
        L.sl[3] = (1.0 - L.sl[0] - 6.0 * L.sl[1] - 12.0 * L.sl[2]) / 8.0;
    }
    if (L.grad != 3 && !(d->lambda > 0 && d->lambda <= 0.5)) return fail(SFGPU_ERR_INVALID, "lambda must be in (0, 0.5]");
    L.l1chi = (L.grad == 1 && d->lambda_chi >= 0) ? d->lambda_chi : L.l1;
    double ladj = (L.grad == 1 && d->layer_adjustment > 0) ? d->layer_adjustment : 1.0;

    int MX = L.Md[0];
    H->lam_m.assign(MX, 0.0); H->lam_p.assign(MX, 0.0); H->Lx.assign(MX, 1.0);
    if (L.cyl && L.grad == 1) {
        // Lat1DCylinder::calculateLambdas (Lat1DCylinder.cpp:375-415; D =
        // dimensions - 1) and Lat1DSphere::calculateLambdas
        // (Lat1DSphere.cpp:240-286; D = dimensions), with layer_adjustment in
        // the radius of the first layer and removed again from the last one
        // (adjustOuterLayer), and separate contact tables for lambda_chi
        const double PI_ = 4.0 * atan(1.0);
        const bool sph = d->geometry == SFGPU_GEOM_SPHERICAL;
        const double off = d->offset_first_layer;
        if (off <= 0 && d->bound_lo[0] == SFGPU_BOUND_SURFACE)
            return fail(SFGPU_ERR_INVALID, "a surface at the lower bound of a curved lattice needs offset_first_layer");
        const double dim = d->dimensions > 0 ? d->dimensions : 3.0;
        const double D = sph ? dim : dim - 1;
        std::vector<double> V(MX + 1, 0), S(MX + 1, 0), LL(MX + 1, 0);
        std::vector<double> lm(MX + 1, 0), lp(MX + 1, 0), lcm(MX + 1, 0), lcp(MX + 1, 0);
        if (sph) { S[1] = off * off * PI_ * 4; V[1] = (4.0 / 3.0) * pow(off, 3) * PI_; }
        else { S[1] = off * PI_ * 2; V[1] = off * off * PI_; }
        LL[1] = V[1];
        for (int z = 2; z <= MX; z++) {
            double x = z + off - 2 + ladj;
            if (z == MX - 1 && ladj != 1.0) x += -ladj + 1;
            V[z] = (PI_ * pow(2, (D - 1)) / D) * pow(x, D);
            LL[z] = V[z] - V[z - 1];
            S[z] = pow(2, (D - 1)) * PI_ * pow(x, (D - 1));
            lm[z] = L.l1 * S[z - 1] / LL[z];
            lp[z] = L.l1 * S[z] / LL[z];
            lcm[z] = L.l1chi * S[z - 1] / LL[z];
            lcp[z] = L.l1chi * S[z] / LL[z];
        }
        if (sph) { if (LL[1] > 4.0 * PI_ / 3.0) LL[1] = V[1] - pow((off - 1), 3) * PI_ * 4.0 / 3.0; }
        else if (LL[1] > PI_) LL[1] = V[1] - (off - 1) * (off - 1) * PI_;
        if (LL[1] > 0) { lp[1] = LL[2] * lm[2] / LL[1]; lcp[1] = LL[2] * lcm[2] / LL[1]; }
        H->lamc_m.assign(MX, 0.0); H->lamc_p.assign(MX, 0.0);
        for (int x = 0; x < MX; x++) {
            H->lam_m[x] = lm[x + 1]; H->lam_p[x] = lp[x + 1]; H->Lx[x] = LL[x + 1];
            H->lamc_m[x] = lcm[x + 1]; H->lamc_p[x] = lcp[x + 1];
        }
    } else if (L.cyl) {
        const double PI_ = 4.0 * atan(1.0);
        double off = d->offset_first_layer;
        double D = (d->dimensions > 0 ? d->dimensions : 3.0) - 1;
        std::vector<double> V(MX + 1, 0), S(MX + 1, 0), lm(MX + 1, 0), lp(MX + 1, 0), LL(MX + 1, 0);
        S[1] = off * PI_ * 2; V[1] = off * off * PI_; LL[1] = V[1];
        for (int z = 2; z <= MX; z++) {
            double x = z + off - 2 + 1.0;
            V[z] = (PI_ * pow(2, (D - 1)) / D) * pow(x, D);
            LL[z] = V[z] - V[z - 1];
            S[z] = pow(2, (D - 1)) * PI_ * pow(x, (D - 1));
            lm[z] = L.l1 * S[z - 1] / LL[z];
            lp[z] = L.l1 * S[z] / LL[z];
        }
        lp[MX] = 0;
        if (LL[1] > PI_) LL[1] = V[1] - (off - 1) * (off - 1) * PI_;
        if (LL[1] > 0) lp[1] = LL[2] * lm[2] / LL[1];
        for (int x = 0; x < MX; x++) { H->lam_m[x] = lm[x + 1]; H->lam_p[x] = lp[x + 1]; H->Lx[x] = LL[x + 1]; }
    }
    // weights of lnGN sums and of the free energy (SubtractBoundaries +
    // MultiplyWithLatticeSites)
    H->w_gn.assign(L.M, 0.0); H->w_f.assign(L.M, 0.0); H->sb.assign(L.M, 0.0);
    // Lat2DFlat1stO::ComputeLnGN and Lat2DCyl1stO::ComputeLnGN halve the
    // 1-based column y = MY-2 for an upper mirror2 in y, one layer inside the
    // last interior one that SubtractBoundaries halves (Lat2DFlat1stO.cpp:
    // 321-326, :333-341; Lat2DCyl1stO.cpp:415-437): the lnGN weights follow
    // them, the free-energy weights do not
    const int gn_y_shift = (L.grad == 2 && L.order == 1) ? 1 : 0;
    for (int z = 0; z < L.M; z++) {
        int c[3];
        lat_coords(L, z, c);
        double w = 1.0, wg = 1.0;
        bool keep = true, interior = true;
        for (int k = 0; k < L.grad; k++) {
            int last = L.Md[k] - 1;
            if (c[k] == 0) { interior = false; if (L.bc_lo[k] != SFGPU_BOUND_SURFACE) keep = false; }
            else if (c[k] == last) { interior = false; if (L.bc_hi[k] != SFGPU_BOUND_SURFACE) keep = false; }
            else {
                if (c[k] == 1 && L.bc_lo[k] == SFGPU_BOUND_MIRROR2) w *= 0.5;
                else if (c[k] == last - 1 && L.bc_hi[k] == SFGPU_BOUND_MIRROR2) w *= 0.5;
                const int hi_gn = last - 1 - (k == 1 ? gn_y_shift : 0);
                if (c[k] == 1 && L.bc_lo[k] == SFGPU_BOUND_MIRROR2) wg *= 0.5;
                else if (c[k] == hi_gn && L.bc_hi[k] == SFGPU_BOUND_MIRROR2) wg *= 0.5;
            }
        }
        H->sb[z] = keep ? w : 0.0;
        if (L.cyl) { w *= H->Lx[c[0]]; wg *= H->Lx[c[0]]; }
        if (L.grad == 1 && !L.cyl) {   // flat MultiplyWithLatticeSites, Lat1DFlat.cpp:266-269
            if (z == 1) { w *= ladj; wg *= ladj; }
            if (z == L.M - 2 && L.M > 3) { w *= (2 - ladj); wg *= (2 - ladj); }
        }
        H->w_f[z] = keep ? w : 0.0;
        H->w_gn[z] = interior ? wg : 0.0;
        // Lat1D2ndO::ComputeLnGN sums the interior without mirror2 halves or
        // layer adjustment (Lat1D2ndO.cpp:291-300); the curved second-order
        // lattices keep L(z) and the mirror2 halves (Lat1DCyl2ndO.cpp:318-330,
        // Lat2DCyl2ndO.cpp:420-469)
        if (L.order == 2 && L.grad == 1 && !L.cyl) H->w_gn[z] = interior ? 1.0 : 0.0;
    }
    return SFGPU_OK;
}

// ---------------------------------------------------------------------------
// system
// ---------------------------------------------------------------------------
template <class T> static int dalloc(T **p, size_t n) {
    *p = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc((void **)p, n * sizeof(T));
    if (e != cudaSuccess) { sfgpu_set_error(e, "cudaMalloc", __FILE__, __LINE__); return SFGPU_ERR_NOMEM; }
    return SFGPU_OK;
}

static bool chi_cols_equal(const std::vector<double> &chi, int ns, int a, int b) {
    for (int i = 0; i < ns; i++)
        if (chi[i * ns + a] != chi[i * ns + b]) return false;
    return true;
}

sfgpu_system::~sfgpu_system() {
    if (a_store) cudaFree(a_store);
    if (a_ring) cudaFree(a_ring);
    if (a_tree) cudaFree(a_tree);
    if (a_dend_gi) cudaFree(a_dend_gi);
    for (void *p : allocs) cudaFree(p);
    if (own_stream && stream) cudaStreamDestroy(stream);
}

int sfgpu_system::alloc_d(double **p, size_t n) {
    int rc = dalloc(p, n);
    if (rc == SFGPU_OK) allocs.push_back(*p);
    return rc;
}
int sfgpu_system::alloc_i(int **p, size_t n) {
    int rc = dalloc(p, n);
    if (rc == SFGPU_OK) allocs.push_back(*p);
    return rc;
}

int sfgpu_system::setup(const sfgpu_system_desc *d) {
    int rc = sfgpu_build_lattice(&d->lattice, &H);
    if (rc) return rc;
    DLat &L = H.L;
    M = L.M;
    K = L.K;
    nseg = d->n_segments;
    if (nseg < 1 || nseg > SFGPU_MAX_SEG) return fail(SFGPU_ERR_UNSUPPORTED, "1 to 8 segment types are supported");
    nmol = d->n_molecules;
    if (nmol < 1 || nmol > SFGPU_MAX_SEG) return fail(SFGPU_ERR_UNSUPPORTED, "1 to 8 molecules are supported");
    chi.assign(nseg * nseg, 0.0);
    pf.assign(nseg * nseg, 0.2);
    freedom.resize(nseg);
    range_h.assign((size_t)nseg * M, 0.0);
    for (int i = 0; i < nseg; i++) {
        freedom[i] = d->segments[i].freedom;
        if (freedom[i] < SFGPU_SEG_FREE || freedom[i] > SFGPU_SEG_PINNED) return fail(SFGPU_ERR_UNSUPPORTED, "segment freedom");
        if (freedom[i] != SFGPU_SEG_FREE) {
            if (!d->segments[i].range) return fail(SFGPU_ERR_INVALID, "frozen/pinned segment without range");
            memcpy(&range_h[(size_t)i * M], d->segments[i].range, sizeof(double) * M);
        }
        for (int j = 0; j < nseg; j++) {
            chi[i * nseg + j] = d->chi ? d->chi[i * nseg + j] : 0.0;
            pf[i * nseg + j] = d->pf ? d->pf[i * nseg + j] : 0.2;
        }
    }
    for (int i = 0; i < nseg; i++)
        for (int j = 0; j < nseg; j++)
            if (chi[i * nseg + j] != chi[j * nseg + i]) return fail(SFGPU_ERR_INVALID, "chi must be symmetric");
    memset(&ct, 0, sizeof(ct));
    ct.nseg = nseg;
    for (int i = 0; i < nseg; i++)
        for (int j = 0; j < nseg; j++) ct.chi[i * SFGPU_MAX_SEG + j] = chi[i * nseg + j];

    // molecules
    mols.resize(nmol);
    solvent = -1;
    for (int m = 0; m < nmol; m++) {
        const sfgpu_molecule_desc &md = d->molecules[m];
        HMol &o = mols[m];
        o.seg.clear();
        if (md.n_blocks < 1) return fail(SFGPU_ERR_INVALID, "molecule without blocks");
        for (int b = 0; b < md.n_blocks; b++) {
            if (md.block_length[b] < 1) return fail(SFGPU_ERR_INVALID, "block length must be positive");
            for (int q = 0; q < md.block_length[b]; q++) o.seg.push_back(md.block_segment[b]);
        }
        o.N = (int)o.seg.size();
        o.count.assign(nseg, 0);
        for (int sg : o.seg) {
            if (sg < 0 || sg >= nseg) return fail(SFGPU_ERR_INVALID, "segment index out of range");
            if (freedom[sg] == SFGPU_SEG_FROZEN) return fail(SFGPU_ERR_INVALID, "frozen segment inside a molecule");
            o.count[sg]++;
        }
        o.dend = 0;
        if (md.n_generations > 0) {
            // symmetric dendrimer: generations of consecutive blocks, the
            // chain length and segment numbers of SF_MolStructure::SetMolLength
            // and GetAvNumSegments (SF_MolStructure.cpp:552-595, :847-877)
            if (!md.generation_blocks || !md.generation_repeat) return fail(SFGPU_ERR_INVALID, "dendrimer without generations");
            if (K != 1) return fail(SFGPU_ERR_UNSUPPORTED, "dendrimers on second-order lattices");
            const int G = md.n_generations;
            o.gen_seg.assign(G, {});
            o.gen_rep.assign(G, 0);
            int b = 0;
            for (int i = 0; i < G; i++) {
                const int nb = md.generation_blocks[i];
                if (nb < 1 || b + nb > md.n_blocks) return fail(SFGPU_ERR_INVALID, "dendrimer generation blocks");
                for (int q = b; q < b + nb; q++)
                    for (int r = 0; r < md.block_length[q]; r++) o.gen_seg[i].push_back(md.block_segment[q]);
                b += nb;
                o.gen_rep[i] = md.generation_repeat[i];
                if (o.gen_rep[i] < 1) return fail(SFGPU_ERR_INVALID, "dendrimer functionality must be positive");
            }
            if (b != md.n_blocks) return fail(SFGPU_ERR_INVALID, "dendrimer generations must cover the blocks");
            long long L = 0;
            o.nshort = 0;
            for (int i = G - 1; i >= 0; i--) L = (L + (long long)o.gen_seg[i].size() - 1) * o.gen_rep[i] + 1;
            for (int i = 0; i < G; i++) o.nshort += (int)o.gen_seg[i].size();
            if (L > (1LL << 30)) return fail(SFGPU_ERR_INVALID, "dendrimer too large");
            for (int sg = 0; sg < nseg; sg++) {
                long long num = 0;
                for (int i = G - 1; i >= 0; i--) {
                    long long n = 0;
                    for (int q : o.gen_seg[i]) n += (q == sg);
                    num = (o.gen_seg[i][0] == sg) ? (num + n - 1) * o.gen_rep[i] + 1 : (num + n) * o.gen_rep[i];
                }
                o.count[sg] = (int)num;
            }
            o.N = (int)L;
            o.dend = (L > 1);
        }
        // branched molecules: the bond tree of the segments (SF_ParserBranched::
        // FillLinks, SF_ParserBranched.cpp:43-60: every block's first segment
        // bonds to the last segment of the nearest preceding block of lower
        // or equal rank)
        o.tree = 0;
        o.parent.clear();
        o.kids.clear();
        if (md.bond_parent) {
            if (o.dend) return fail(SFGPU_ERR_INVALID, "a molecule is either a dendrimer or branched");
            if (K != 1) return fail(SFGPU_ERR_UNSUPPORTED, "branched molecules on second-order lattices");
            if (md.bond_parent[0] != -1) return fail(SFGPU_ERR_INVALID, "bond_parent[0] must be -1");
            o.parent.assign(md.bond_parent, md.bond_parent + o.N);
            o.kids.assign(o.N, {});
            for (int q = 1; q < o.N; q++) {
                if (o.parent[q] < 0 || o.parent[q] >= q) return fail(SFGPU_ERR_INVALID, "bond_parent[s] must lie in [0, s)");
                o.kids[o.parent[q]].push_back(q);
            }
            o.tree = (o.N > 1);
        }
        o.used.clear();
        o.pinned = 0;
        for (int i = 0; i < nseg; i++)
            if (o.count[i]) { o.used.push_back(i); if (freedom[i] == SFGPU_SEG_PINNED) o.pinned = 1; }
        o.type = (o.N == 1) ? 0 : (o.used.size() == 1 && !o.dend && !o.tree ? 1 : 2);
        o.sym = (o.type == 1 && K == 1);
        o.freedom = md.freedom;
        o.phibulk = md.phibulk;
        o.theta = md.theta;
        // mol : force: first-order copolymers on the lattices with a force
        // step (Lat2DFlat1stO.cpp:115-117 and the homopolymer and dendrimer
        // drivers stop with an error; the monomer has no step)
        o.force = (o.type == 0) ? 0.0 : md.force;
        if (o.force != 0) {
            if (!(o.force >= -1000.0 && o.force <= 1000.0)) return fail(SFGPU_ERR_INVALID, "force must lie in [-1000, 1000]");
            if (K != 1 || o.type != 2 || o.dend || o.tree)
                return fail(SFGPU_ERR_UNSUPPORTED, "the force ensemble takes first-order linear copolymers");
            if (L.grad == 2 && !L.cyl) return fail(SFGPU_ERR_UNSUPPORTED, "no force ensemble on the 2D flat lattice");
            if (L.ltype != SFGPU_LATTICE_STANDARD) return fail(SFGPU_ERR_UNSUPPORTED, "force ensemble on FCC, HEX or stencils lattices");
        }
        if (o.freedom == SFGPU_MOL_SOLVENT) {
            if (solvent >= 0) return fail(SFGPU_ERR_INVALID, "more than one solvent molecule");
            solvent = m;
        } else if (o.freedom == SFGPU_MOL_RESTRICTED) {
            if (!(o.theta > 0)) return fail(SFGPU_ERR_INVALID, "restricted molecule needs theta > 0");
        } else if (o.freedom == SFGPU_MOL_FREE) {
            if (!(o.phibulk > 0 && o.phibulk < 1)) return fail(SFGPU_ERR_INVALID, "free molecule needs 0 < phibulk < 1");
        } else if (o.freedom != SFGPU_MOL_NEUTRALIZER) {   // checked with the charges
            return fail(SFGPU_ERR_UNSUPPORTED, "molecule freedom");
        }
        // homopolymer ring (SF_MolList1stO.cpp:28-38, SF_HomoRing1stO::Matrix1)
        o.ring = 0;
        if (md.ring) {
            if (o.type != 1 || o.tree) return fail(SFGPU_ERR_INVALID, "only linear homopolymers form rings (SF_MolList1stO.cpp:29-30)");
            if (o.N % 2 != 0) return fail(SFGPU_ERR_INVALID, "rings have an even length (SF_HomoRing1stO.cpp:120)");
            if (K != 1 || L.grad != 1 || L.cyl) return fail(SFGPU_ERR_UNSUPPORTED, "rings on lattices other than the 1D flat one");
            if (o.freedom != SFGPU_MOL_FREE) return fail(SFGPU_ERR_UNSUPPORTED, "rings other than free ones (phibulk)");
            if (o.pinned) return fail(SFGPU_ERR_UNSUPPORTED, "rings of pinned segments");
            const int Mmax = (o.N / 2 > M) ? 2 * M : M + o.N / 2;
            if ((size_t)2 * (Mmax + 1) * sizeof(double) > 200 * 1024) return fail(SFGPU_ERR_UNSUPPORTED, "ring walk larger than shared memory");
            // NORM[0]: the free ring's return weight, the reference's own loop
            // (SF_HomoRing1stO.cpp:123-135) on the host
            const int h = o.N / 2;
            std::vector<double> X(2 * h + 1, 0.0);
            auto at = [&](int z) -> double & { return X[z + h]; };
            at(0) = 1;
            for (int st = 1; st < h; st++) {
                double a = 0, b = at(-st - 1), c = at(-st);
                for (int z = -st; z < st; z++) {
                    a = b; b = c; c = at(z + 1);
                    at(z) = (a + 4.0 * b + c) / 6.0;
                }
            }
            double n0 = 0;
            for (int z = -h; z < h; z++) n0 += at(z) * at(z);
            o.ring_norm0 = n0;
            o.ring = 1;
        }
        double cr = 0;   // SF_MolStructure.cpp:411-423
        for (int a : o.used) {
            double inner = 0;
            for (int b : o.used) inner += chi[a * nseg + b] * ((double)o.count[b] / o.N);
            cr += ((double)o.count[a] / o.N) * inner;
        }
        o.chemintref = cr / 2;
    }
    if (solvent < 0) return fail(SFGPU_ERR_INVALID, "a solvent molecule is required");

    // classes of liquid states (SF_Solve.cpp:37-86)
    std::vector<int> q;
    for (int i = 0; i < nseg; i++) if (freedom[i] != SFGPU_SEG_FROZEN) q.push_back(i);
    int nl = (int)q.size();
    if (nl == 0) return fail(SFGPU_ERR_INVALID, "no liquid segments");
    for (int i = 0; i < nl; i++) {
        int s1 = q[i];
        for (int j = i + 1; j < nl; j++)
            if (chi_cols_equal(chi, nseg, s1, q[j])) {
                if (j != i + 1) std::swap(q[i + 1], q[j]);
                i++;
            }
    }
    class_of.assign(nseg, -1);
    rep_of_class.clear();
    for (int i = 0; i < nl; i++) {
        int s1 = q[i];
        int c = (int)rep_of_class.size();
        class_of[s1] = c;
        rep_of_class.push_back(s1);
        for (int j = i + 1; j < nl; j++)
            if (chi_cols_equal(chi, nseg, s1, q[j])) { i++; class_of[q[i]] = c; rep_of_class[c] = q[i]; }
    }
    nclass = (int)rep_of_class.size();
    // sites with iteration variables (SF_Solve.cpp:129-150)
    std::vector<int> jmap(M, -1);
    sites_h.clear();
    for (int z = 0; z < M; z++) {
        int c[3];
        lat_coords(L, z, c);
        if (!lat_interior(L, c)) continue;
        bool ok = true;
        for (int i = 0; i < nseg; i++)
            if (freedom[i] == SFGPU_SEG_FROZEN && range_h[(size_t)i * M + z] > 0.999) ok = false;
        if (ok) { jmap[z] = (int)sites_h.size(); sites_h.push_back(z); }
    }
    nsites = (int)sites_h.size();
    nvar = (size_t)nsites * nclass;
    if (nsites == 0) return fail(SFGPU_ERR_INVALID, "no sites carry iteration variables");
    if ((rc = setup_charges(d, jmap))) return rc;

    // device buffers
    if ((rc = alloc_d(&d_lam_m, M > 0 ? L.Md[0] : 1))) return rc;
    if ((rc = alloc_d(&d_lam_p, L.Md[0]))) return rc;
    SFGPU_CUDA_TRY(cudaMemcpy(d_lam_m, H.lam_m.data(), sizeof(double) * L.Md[0], cudaMemcpyHostToDevice));
    SFGPU_CUDA_TRY(cudaMemcpy(d_lam_p, H.lam_p.data(), sizeof(double) * L.Md[0], cudaMemcpyHostToDevice));
    L.lam_m = d_lam_m; L.lam_p = d_lam_p;
    // contact tables: their own on 1D curved lattices (lambda_chi), else the step tables
    const std::vector<double> &tcm = H.lamc_m.empty() ? H.lam_m : H.lamc_m;
    const std::vector<double> &tcp = H.lamc_p.empty() ? H.lam_p : H.lamc_p;
    if ((rc = alloc_d(&d_lamc_m, L.Md[0])) || (rc = alloc_d(&d_lamc_p, L.Md[0]))) return rc;
    SFGPU_CUDA_TRY(cudaMemcpy(d_lamc_m, tcm.data(), sizeof(double) * L.Md[0], cudaMemcpyHostToDevice));
    SFGPU_CUDA_TRY(cudaMemcpy(d_lamc_p, tcp.data(), sizeof(double) * L.Md[0], cudaMemcpyHostToDevice));
    L.lamc_m = d_lamc_m; L.lamc_p = d_lamc_p;
    if ((rc = alloc_d(&d_wgn, M)) || (rc = alloc_d(&d_wf, M)) || (rc = alloc_d(&d_sb, M))) return rc;
    if (!H.stiff.empty()) {
        for (auto &o : mols) {
            if (o.type == 1) return fail(SFGPU_ERR_UNSUPPORTED, "a stiff range with homopolymers (SFbox: only copolymers)");
            // a palindromic copolymer takes SF_Copol2ndO_stiff_range::SymMatrix1
            // (SF_Copol2ndO_stiff_range.cpp:97-99, :407-452), whose half-chain
            // route has no isotropic end steps and other Pf indices: not built
            bool pal = o.type == 2 && !o.dend;
            for (int s = 0; pal && s < o.N / 2; s++) pal = o.seg[s] == o.seg[o.N - 1 - s];
            if (pal) return fail(SFGPU_ERR_UNSUPPORTED, "a palindromic copolymer on a stiff range (SFbox's SymMatrix1)");
        }
        if ((rc = alloc_d(&d_stiff, M))) return rc;
        SFGPU_CUDA_TRY(cudaMemcpy(d_stiff, H.stiff.data(), sizeof(double) * M, cudaMemcpyHostToDevice));
        L.stiff = d_stiff;
    }
    SFGPU_CUDA_TRY(cudaMemcpy(d_sb, H.sb.data(), sizeof(double) * M, cudaMemcpyHostToDevice));
    SFGPU_CUDA_TRY(cudaMemcpy(d_wgn, H.w_gn.data(), sizeof(double) * M, cudaMemcpyHostToDevice));
    SFGPU_CUDA_TRY(cudaMemcpy(d_wf, H.w_f.data(), sizeof(double) * M, cudaMemcpyHostToDevice));
    if ((rc = alloc_i(&d_jmap, M)) || (rc = alloc_i(&d_sites, nsites))) return rc;
    SFGPU_CUDA_TRY(cudaMemcpy(d_jmap, jmap.data(), sizeof(int) * M, cudaMemcpyHostToDevice));
    SFGPU_CUDA_TRY(cudaMemcpy(d_sites, sites_h.data(), sizeof(int) * nsites, cudaMemcpyHostToDevice));
    d_range.assign(nseg, nullptr); d_gfull.assign(nseg, nullptr); d_gseg.assign(nseg, nullptr); d_phi.assign(nseg, nullptr);
    for (int i = 0; i < nseg; i++) {
        if ((rc = alloc_d(&d_phi[i], M))) return rc;
        if (freedom[i] != SFGPU_SEG_FREE) {
            if ((rc = alloc_d(&d_range[i], M))) return rc;
            SFGPU_CUDA_TRY(cudaMemcpy(d_range[i], &range_h[(size_t)i * M], sizeof(double) * M, cudaMemcpyHostToDevice));
        }
        if (freedom[i] == SFGPU_SEG_FROZEN) {
            // phi of a frozen state: its range values with boundary copies (SF_Segment.cpp:428-433)
            std::vector<double> p(range_h.begin() + (size_t)i * M, range_h.begin() + (size_t)(i + 1) * M);
            for (int z = 0; z < M; z++) { int t = lat_map(L, z); if (t != z) p[z] = range_h[(size_t)i * M + t]; }
            SFGPU_CUDA_TRY(cudaMemcpy(d_phi[i], p.data(), sizeof(double) * M, cudaMemcpyHostToDevice));
            continue;
        }
        if ((rc = alloc_d(&d_gfull[i], M))) return rc;
        if (freedom[i] == SFGPU_SEG_PINNED) { if ((rc = alloc_d(&d_gseg[i], M))) return rc; }
        else d_gseg[i] = d_gfull[i];
    }
    size_t store = 0;
    for (auto &o : mols) {
        o.d_phi.assign(nseg, nullptr);
        for (int i : o.used) if ((rc = alloc_d(&o.d_phi[i], M))) return rc;
        size_t need = (o.type == 0 || o.ring) ? 0
                      : (size_t)(o.tree ? 3 * o.N : o.dend ? o.nshort : o.sym ? std::max(1, o.N / 2) : o.N) * K * M;
        if (primal_checkpointed(o)) {
            const int k = primal_stride;
            need = (size_t)((o.N + k - 1) / k + k) * K * M;   // checkpoints + one segment
        }
        store = std::max(store, need);
    }
    if ((rc = alloc_d(&d_gi, store))) return rc;
    if ((rc = alloc_d(&d_ginv[0], (size_t)K * M)) || (rc = alloc_d(&d_ginv[1], (size_t)K * M))) return rc;
    // row-wise steps never write boundary entries; surface layers are read
    // in place and must hold the propagator's value there, 0
    SFGPU_CUDA_TRY(cudaMemset(d_gi, 0, sizeof(double) * std::max<size_t>(store, 1)));
    SFGPU_CUDA_TRY(cudaMemset(d_ginv[0], 0, sizeof(double) * K * M));
    SFGPU_CUDA_TRY(cudaMemset(d_ginv[1], 0, sizeof(double) * K * M));
    nblocks_red = grid_for(M);
    if ((rc = alloc_d(&d_partial, (size_t)std::max(nblocks_red, 64) * 64))) return rc;
    if ((rc = alloc_d((double **)&d_scal, 4 * (size_t)nmol))) return rc;
    if ((rc = alloc_d(&d_phib, nseg)) || (rc = alloc_d(&d_chib, nclass)) || (rc = alloc_d(&d_misc, 64))) return rc;
    if ((rc = alloc_d(&d_x, nvar)) || (rc = alloc_d(&d_f, nvar))) return rc;
    SFGPU_CUDA_TRY(cudaMemset(d_scal, 0, sizeof(MolScal) * nmol));

    // bulk parameters
    memset(&bp, 0, sizeof(bp));
    bp.nseg = nseg; bp.nmol = nmol; bp.nclass = nclass;
    for (int c = 0; c < nclass; c++) bp.rep[c] = rep_of_class[c];
    for (int i = 0; i < nseg; i++)
        for (int m = 0; m < nmol; m++) bp.frac[i * SFGPU_MAX_SEG + m] = (double)mols[m].count[i] / mols[m].N;
    if (d->overflow_protection) return setup_logspace();
    return SFGPU_OK;
}

// Overflow protection (sys : overflow_protection, SF_System.cpp:67, :445-519):
// the *1stOS lattice constants (Lat1DFlat1stOS.cpp:3-9, Lat2DFlat1stOS.cpp:8-13,
// Lat2DCyl1stOS.cpp:3-25), the weights of their ComputeLnGN and the log-space
// buffers.
int sfgpu_system::setup_logspace() {
    const DLat &L = H.L;
    if (L.order != 1 || L.grad > 2)
        return fail(SFGPU_ERR_UNSUPPORTED, "overflow protection needs a first-order 1D or 2D lattice");
    for (auto &o : mols) {
        if (o.dend) return fail(SFGPU_ERR_UNSUPPORTED, "dendrimers with overflow protection");
        if (o.tree || o.ring) return fail(SFGPU_ERR_UNSUPPORTED, "branched molecules and rings with overflow protection");
        if (o.force != 0) return fail(SFGPU_ERR_UNSUPPORTED, "the force ensemble with overflow protection");
    }
    logmode = true;
    logc.lmax = log(DBL_MAX);
    logc.logcutoff = 100.0;
    logc.cutoff = exp(logc.logcutoff);
    logc.prefactor = logc.lmax - logc.logcutoff - 50.0;
    memset(&logq, 0, sizeof(logq));
    const double l1 = L.l1;
    logq.kind = (L.grad == 1) ? (L.cyl ? LOG_CURVED1 : LOG_FLAT1) : (L.cyl ? LOG_CYL2 : LOG_FLAT2);
    if (logq.kind == LOG_FLAT1 || logq.kind == LOG_FLAT2) {
        const double l0 = (logq.kind == LOG_FLAT1) ? 1 - 2 * l1 : 1 - 4 * l1;
        logq.logl1l0 = log(l1 / l0);
        logq.logl0 = log(l0);
        logq.logl1 = log(l1);
    }
    int rc;
    const int MX = L.Md[0];
    if (logq.kind == LOG_CYL2) {
        std::vector<double> a(MX, 0.0), b(MX, 0.0), c(MX, 0.0);
        for (int x = 1; x < MX - 1; x++) {
            const double lm = H.lam_m[x], lp = H.lam_p[x];
            b[x] = lm > 0 ? log(lm) : 0;
            c[x] = lp > 0 ? log(lp) : 0;
            const double l0 = 1.0 - lm - lp - 2 * l1;
            a[x] = l0 > 0 ? log(l0) : 0;
        }
        logq.logl1 = l1 > 0 ? log(l1) : 0;
        logq.nl_centre = 1.0 - l1 - l1 - l1 - l1;
        if ((rc = alloc_d(&d_logl0x, MX)) || (rc = alloc_d(&d_loglmx, MX)) || (rc = alloc_d(&d_loglpx, MX))) return rc;
        SFGPU_CUDA_TRY(cudaMemcpy(d_logl0x, a.data(), sizeof(double) * MX, cudaMemcpyHostToDevice));
        SFGPU_CUDA_TRY(cudaMemcpy(d_loglmx, b.data(), sizeof(double) * MX, cudaMemcpyHostToDevice));
        SFGPU_CUDA_TRY(cudaMemcpy(d_loglpx, c.data(), sizeof(double) * MX, cudaMemcpyHostToDevice));
        logq.logl0x = d_logl0x; logq.loglmx = d_loglmx; logq.loglpx = d_loglpx;
    }
    // ComputeLnGN of the log-space lattices as weights: 1D
    // (Lat1DFlat1stOS.cpp:441-478, Lat1DCyl1stOS.cpp:242-281) weighs the
    // first interior layer 1/2 when the lower copy layer is 3, the last one
    // 1/2 when the upper copy layer is M-2 (1-based; mirror2), and takes no
    // layer adjustment; curved layers also weigh L(z).  2D
    // (Lat2DFlat1stOS.cpp:449-505, Lat2DCyl1stOS.cpp:471-540) adds every
    // interior site (times L(x) on the cylinder), takes half of the x rows
    // and y columns next to a mirror2, the upper one in y being the column
    // y = MY-2 (1-based), and adds the four corners back with 1/4 (flat) or
    // 4 L(x) (cylinder).
    w_os.assign(M, 0.0);
    auto copy_lo = [&](int k) { return L.bc_lo[k] == SFGPU_BOUND_PERIODIC ? L.Md[k] - 1 : L.bc_lo[k]; };
    auto copy_hi = [&](int k) { return L.bc_hi[k] == SFGPU_BOUND_PERIODIC ? 2 : L.Md[k] - L.bc_hi[k] + 1; };
    auto Lx = [&](int x) { return L.cyl ? H.Lx[x] : 1.0; };
    if (L.grad == 1) {
        const int Mz = L.Md[0];
        w_os[1] = Lx(1) * (copy_lo(0) == 3 ? 0.5 : 1.0);
        for (int z = 2; z <= Mz - 3; z++) w_os[z] = Lx(z);
        // the last term is added on top of the first one when both are the
        // same layer (one interior layer)
        if (copy_hi(0) == Mz - 2) w_os[Mz - 2] += 0.5 * Lx(Mz - 2);
        else if (Mz > 3) w_os[Mz - 2] = Lx(Mz - 2);
    } else {
        const int MY = L.Md[1], nx = MX - 2, ny = MY - 2;
        auto at = [&](int x, int y) -> double & { return w_os[(size_t)x * MY + y]; };
        for (int x = 1; x <= nx; x++)
            for (int y = 1; y <= ny; y++) at(x, y) = Lx(x);
        const bool X1 = copy_lo(0) == 3, X2 = copy_hi(0) == MX - 2;
        const bool Y1 = copy_lo(1) == 3, Y2 = copy_hi(1) == MY - 2;
        if (X1) for (int y = 1; y <= ny; y++) at(1, y) -= 0.5 * Lx(1);
        if (X2) for (int y = 1; y <= ny; y++) at(nx, y) -= 0.5 * Lx(nx);
        if (Y1) for (int x = 1; x <= nx; x++) at(x, 1) -= 0.5 * Lx(x);
        if (Y2) for (int x = 1; x <= nx; x++) at(x, ny - 1) -= 0.5 * Lx(x);
        const double f1 = L.cyl ? 4.0 * Lx(1) : 0.25, f2 = L.cyl ? 4.0 * Lx(nx) : 0.25;
        if (X1 && Y1) at(1, 1) += f1;
        if (X1 && Y2) at(1, ny - 1) += f1;
        if (X2 && Y1) at(nx, 1) += f2;
        if (X2 && Y2) at(nx, ny - 1) += f2;
    }
    if ((rc = alloc_d(&d_wos, M)) || (rc = alloc_d(&d_lse, nmol))) return rc;
    SFGPU_CUDA_TRY(cudaMemcpy(d_wos, w_os.data(), sizeof(double) * M, cudaMemcpyHostToDevice));
    d_lgseg.assign(nseg, nullptr);
    for (int i = 0; i < nseg; i++)
        if (freedom[i] != SFGPU_SEG_FROZEN && (rc = alloc_d(&d_lgseg[i], M))) return rc;
    return SFGPU_OK;
}

// propagation of one molecule (SF_Monomer1stO::Matrix1, SF_Homopol1stO::Matrix1,
// SF_Copol1stO::Matrix1, SF_Homopol2ndO::Matrix1, SF_Copol2ndO::Matrix1)
// molecule_phi in logarithms, for overflow protection: the same chain walks
// with the *1stOS steps, ConnectG, CorrectDoubleCountG, ComputeLnGN and
// NormPhi* of Lat1DFlat1stOS.cpp:289-358 (and the 1D curved and 2D ones),
// between MakeSafe(G) and RestoreFromSafe(phi) as in SF_Monomer1stO.cpp:105-132,
// SF_Homopol1stO.cpp:562-621 and SF_Copol1stO.cpp:1196-1281.
int sfgpu_system::molecule_phi_log(int m) {
    HMol &o = mols[m];
    const DLat &L = H.L;
    const int g = grid_for(M), gr = grid_rows(L);
    cudaStream_t s = stream;
    MolParam p;
    p.N = o.N; p.type = o.type; p.freedom = o.freedom; p.sym = o.sym; p.K = 1;
    p.pinned = o.pinned; p.solvent = (m == solvent); p.nmol = nmol;
    p.phibulk_in = o.phibulk; p.theta = o.theta;
    if (m == neutralizer) { p.freedom = SFGPU_MOL_FREE; p.phib_dev = d_neut_phib; }
    MolScal *scal = (MolScal *)d_scal;
    const int restr = (o.freedom == SFGPU_MOL_RESTRICTED);
    const double N = (double)o.N;
    const double LZ = SFGPU_LOGZERO;
    if (o.type == 0) {
        const int i = o.seg[0];
        lse_weighted<<<1, 1024, 0, s>>>(M, d_lgseg[i], d_wos, d_lse + m);
        mol_scalars_log<<<1, 1, 0, s>>>(p, d_lse + m, scal, m);
        finalize_phi_log<<<g, kBlock, 0, s>>>(M, logc, d_lgseg[i], o.d_phi[i], scal, m, 1, restr,
                                              restr ? log(o.theta) : 0.0);
        return SFGPU_OK;
    }
    for (int i : o.used) fill_value<<<g, kBlock, 0, s>>>(M, LZ, o.d_phi[i]);
    double *ginv = d_ginv[0], *tmp = d_ginv[1];
    const double *cur;
    if (o.sym) {
        const int i = o.seg[0], half = o.N / 2;
        const double *lG = d_lgseg[i];
        double *phi = o.d_phi[i];
        SFGPU_CUDA_TRY(cudaMemcpyAsync(d_gi, lG, sizeof(double) * M, cudaMemcpyDeviceToDevice, s));
        for (int t = 1; t < half; t++)
            step1_log_rows<<<gr, kBlock, 0, s>>>(L, logq, logc, d_gi + (size_t)(t - 1) * M, lG, d_gi + (size_t)t * M,
                                                 nullptr, nullptr, COMP_NONE);
        cur = d_gi + (size_t)(half - 1) * M;
        if (o.N % 2 == 1) {
            step1_log_rows<<<gr, kBlock, 0, s>>>(L, logq, logc, cur, lG, ginv, nullptr, phi, COMP_CENTRE);
            cur = ginv; std::swap(ginv, tmp);
        }
        for (int sp = (o.N + 3) / 2; sp <= o.N; sp++) {
            const int sinv = o.N - sp + 1;
            step1_log_rows<<<gr, kBlock, 0, s>>>(L, logq, logc, cur, lG, ginv, d_gi + (size_t)(sinv - 1) * M, phi,
                                                 COMP_ACC);
            cur = ginv; std::swap(ginv, tmp);
        }
        lse_weighted<<<1, 1024, 0, s>>>(M, cur, d_wos, d_lse + m);
        mol_scalars_log<<<1, 1, 0, s>>>(p, d_lse + m, scal, m);
        finalize_phi_log<<<g, kBlock, 0, s>>>(M, logc, lG, phi, scal, m, 0, restr, restr ? log(2 * o.theta / N) : 0.0);
        set_boundaries<<<g, kBlock, 0, s>>>(L, 1, phi);
        return SFGPU_OK;
    }
    SFGPU_CUDA_TRY(cudaMemcpyAsync(d_gi, d_lgseg[o.seg[0]], sizeof(double) * M, cudaMemcpyDeviceToDevice, s));
    for (int t = 1; t < o.N; t++)
        step1_log_rows<<<gr, kBlock, 0, s>>>(L, logq, logc, d_gi + (size_t)(t - 1) * M, d_lgseg[o.seg[t]],
                                             d_gi + (size_t)t * M, nullptr, nullptr, COMP_NONE);
    SFGPU_CUDA_TRY(cudaMemcpyAsync(ginv, d_lgseg[o.seg[o.N - 1]], sizeof(double) * M, cudaMemcpyDeviceToDevice, s));
    connect_log<<<g, kBlock, 0, s>>>(M, logc, ginv, d_gi + (size_t)(o.N - 1) * M, o.d_phi[o.seg[o.N - 1]]);
    cur = ginv; std::swap(ginv, tmp);
    for (int t = o.N - 2; t >= 0; t--) {
        const int sg = o.seg[t];
        step1_log_rows<<<gr, kBlock, 0, s>>>(L, logq, logc, cur, d_lgseg[sg], ginv, d_gi + (size_t)t * M, o.d_phi[sg],
                                             COMP_ACC);
        cur = ginv; std::swap(ginv, tmp);
    }
    lse_weighted<<<1, 1024, 0, s>>>(M, cur, d_wos, d_lse + m);
    mol_scalars_log<<<1, 1, 0, s>>>(p, d_lse + m, scal, m);
    for (int i : o.used) {
        finalize_phi_log<<<g, kBlock, 0, s>>>(M, logc, d_lgseg[i], o.d_phi[i], scal, m, 0, restr,
                                              restr ? log(o.theta / N) : 0.0);
        set_boundaries<<<g, kBlock, 0, s>>>(L, 1, o.d_phi[i]);
    }
    return SFGPU_OK;
}

// weights of a constant-force step with force f (see force_row)
ForceW force_weights(const DLat &L, double f) {
    ForceW w;
    const double l1 = L.l1;
    if (L.grad == 1 && !L.cyl) {
        const double norm = l1 * (exp(-f) + exp(f) - 2) + 1;
        w.a2 = l1 * exp(-f) / norm;
        w.a1 = l1 * exp(f) / norm;
        w.a3 = norm;
    } else if (L.grad == 1) {
        double f_1 = exp(f), f1 = exp(-f);
        const double fnorm = (4.0 + f1 + f_1) / 6.0;
        w.a1 = f1 / fnorm;
        w.a2 = f_1 / fnorm;
        w.a3 = fnorm;
    } else if (L.grad == 2) {
        const double f_1 = exp(-f), f1 = exp(f);
        w.a1 = f1; w.a2 = f_1;
        w.a3 = l1 * (f_1 + f1 - 2) + 1;
    } else {
        w.a1 = exp(f); w.a2 = exp(-f);
        w.a3 = 1.0 / (4.0 + exp(f) + exp(-f));
    }
    return w;
}

// SF_Dend1stO::Matrix1 (SF_Dend1stO.cpp:163-312): the propagator from the
// ends inwards along one path from an end to the centre (nshort positions,
// stored), the branch points combining f copies of the arriving propagator
// (product divided by the branch point's G f-1 times), then from the centre
// outwards with the composition weighted by the number of equivalent copies.
int sfgpu_system::molecule_phi_dend(int m) {
    HMol &o = mols[m];
    const DLat &L = H.L;
    const int g = grid_for(M);
    cudaStream_t s = stream;
    const int G = (int)o.gen_seg.size(), NS = o.nshort;
    auto slice = [&](int sp) { return d_gi + (size_t)(sp - 1) * M; };   // position sp = 1..NS
    for (int i : o.used) SFGPU_CUDA_TRY(cudaMemsetAsync(o.d_phi[i], 0, sizeof(double) * M, s));
    double *ginv = d_ginv[0], *tmp = d_ginv[1];
    // ends inwards
    int sp = 0;
    const double *Gold = nullptr;
    for (int i = G - 1; i >= 0; i--) {
        const int len = (int)o.gen_seg[i].size();
        for (int j = len; j >= 1; j--) {
            const double *Gc = d_gseg[o.gen_seg[i][j - 1]];
            sp++;
            if (sp == 1) {
                SFGPU_CUDA_TRY(cudaMemcpyAsync(slice(1), Gc, sizeof(double) * M, cudaMemcpyDeviceToDevice, s));
            } else if (j == len && i + 1 < G && o.gen_rep[i + 1] > 1) {
                // the node: f copies of the branch arriving at the outer
                // generation's first segment (Gold)
                const double *arr = slice(sp - 1);
                const double *acc = arr;
                for (int k = 1; k <= o.gen_rep[i + 1] - 1; k++) {
                    dend_combine<<<g, kBlock, 0, s>>>(M, arr, acc, Gold, ginv);
                    acc = ginv; std::swap(ginv, tmp);
                }
                launch_step1(acc, Gc, slice(sp), nullptr, nullptr, COMP_NONE);
            } else {
                launch_step1(slice(sp - 1), Gc, slice(sp), nullptr, nullptr, COMP_NONE);
            }
            Gold = Gc;
        }
    }
    // centre outwards
    sp = NS;
    double nr = 1.0;
    const double *cur = nullptr;
    for (int i = 0; i < G; i++) {
        const int len = (int)o.gen_seg[i].size(), rep = o.gen_rep[i];
        for (int j = 1; j <= len; j++) {
            const int sg = o.gen_seg[i][j - 1];
            const double *Gc = d_gseg[sg];
            if (sp == NS) SFGPU_CUDA_TRY(cudaMemcpyAsync(ginv, Gc, sizeof(double) * M, cudaMemcpyDeviceToDevice, s));
            else launch_step1(cur, Gc, ginv, nullptr, nullptr, COMP_NONE);
            cur = ginv; std::swap(ginv, tmp);
            if (j == 1)
                for (int k = 1; k <= rep - 1; k++) {
                    dend_combine<<<g, kBlock, 0, s>>>(M, cur, slice(sp), Gc, ginv);
                    cur = ginv; std::swap(ginv, tmp);
                }
            dend_connect<<<g, kBlock, 0, s>>>(M, const_cast<double *>(cur), slice(sp), o.d_phi[sg], nr, 1.0 / nr);
            if (j == 1) nr *= rep;
            sp--;
        }
    }
    MolParam p;
    p.N = o.N; p.type = o.type; p.freedom = o.freedom; p.sym = 0; p.K = 1;
    p.pinned = o.pinned; p.solvent = (m == solvent); p.nmol = nmol;
    p.phibulk_in = o.phibulk; p.theta = o.theta;
    wsum_partial<<<nblocks_red, kBlock, 0, s>>>(M, 1, cur, d_wgn, d_partial);
    mol_scalars<<<1, 1, 0, s>>>(p, nblocks_red, d_partial, (MolScal *)d_scal, m);
    for (int i : o.used) {
        finalize_phi<<<g, kBlock, 0, s>>>(M, d_gseg[i], o.d_phi[i], (const MolScal *)d_scal, m, 0);
        set_boundaries<<<g, kBlock, 0, s>>>(L, 1, o.d_phi[i]);
    }
    return SFGPU_OK;
}

// Branched molecules (SF_Branched1stO::Matrix1, SF_Branched1stO.cpp:1240-1310;
// combs, SF_Comb1stO): for the bond tree rooted at segment 0,
//   U(s) = G_s prod_(children c) A U(c)      (the subtree hanging from s,
//                                             ends inwards, U(leaf) = G),
//   Q(c) = G_p . A U(c)                       (child c's subtree seen from its
//                                             parent p),
//   D(0) = G_0,  D(c) = G_c . A [D(p) prod_(siblings c' != c) Q(c')]
//                                             (the rest of the molecule seen
//                                             from c),
// every product over factors that each carry G_s once divided by G_s (where
// G > 0, the reference's ConnectG + CorrectDoubleCountG pairs), and
// phi += U(s) D(s) per segment before the division by G of finalize_phi.
// lnGN comes from U(0), the whole molecule's propagator at its first
// segment (Gzs[1][1], SF_Branched1stO.cpp:1269).  U, Q and D take 3 N
// slices of the chain storage.
// A symmetric dendrimer as its bond tree, in the order SF_Dend1stO's
// generations nest (SF_MolStructure.cpp:552-595): generation i is a branch
// point (its first segment) with f_i copies of the rest of its segments,
// each continued by generation i + 1; segment 0 is the centre and every
// parent precedes its children.
void sfgpu_system::build_dend_tree(HMol &o) {
    if (!o.tseg.empty()) return;
    const int G = (int)o.gen_seg.size();
    std::vector<int> seg, par;
    // iterative expansion: (generation, parent index) work items
    std::vector<std::pair<int, int>> todo{{0, -1}};
    while (!todo.empty()) {
        const auto [i, p] = todo.back();
        todo.pop_back();
        const int root = (int)seg.size();
        seg.push_back(o.gen_seg[i][0]);
        par.push_back(p);
        for (int r = 0; r < o.gen_rep[i]; r++) {
            int prev = root;
            for (size_t j = 1; j < o.gen_seg[i].size(); j++) {
                seg.push_back(o.gen_seg[i][j]);
                par.push_back(prev);
                prev = (int)seg.size() - 1;
            }
            if (i + 1 < G) todo.push_back({i + 1, prev});
        }
    }
    o.tseg = seg;
    o.tparent = par;
    o.tkids.assign(seg.size(), {});
    for (size_t q = 1; q < seg.size(); q++) o.tkids[par[q]].push_back((int)q);
}

// swap a dendrimer's tree form in (on) or out: the tree recursion then reads
// seg, parent, kids and tree as for a branched molecule; N is the same
void sfgpu_system::dend_view(HMol &o, bool on) {
    std::swap(o.seg, o.tseg);
    std::swap(o.parent, o.tparent);
    std::swap(o.kids, o.tkids);
    o.tree = on ? 1 : 0;
    o.dend = on ? 0 : 1;
}

int sfgpu_system::molecule_phi_tree(int m) {
    HMol &o = mols[m];
    const DLat &L = H.L;
    const int g = grid_for(M), N = o.N;
    cudaStream_t s = stream;
    double *const base = tree_gi ? tree_gi : d_gi;
    auto U = [&](int q) { return base + (size_t)q * M; };
    auto Q = [&](int q) { return base + (size_t)(N + q) * M; };
    auto D = [&](int q) { return base + (size_t)(2 * N + q) * M; };
    const size_t bytes = sizeof(double) * M;
    for (int i : o.used) SFGPU_CUDA_TRY(cudaMemsetAsync(o.d_phi[i], 0, bytes, s));
    // ends inwards
    for (int q = N - 1; q >= 0; q--) {
        const double *Gq = d_gseg[o.seg[q]];
        const std::vector<int> &kids = o.kids[q];
        if (kids.empty()) {
            SFGPU_CUDA_TRY(cudaMemcpyAsync(U(q), Gq, bytes, cudaMemcpyDeviceToDevice, s));
        } else if (kids.size() == 1) {
            SFGPU_CUDA_TRY(cudaMemcpyAsync(U(q), Q(kids[0]), bytes, cudaMemcpyDeviceToDevice, s));
        } else {
            // the last product lands in U(q), earlier ones alternate between
            // the two work slices (no kernel reads and writes one array)
            const double *acc = Q(kids[0]);
            int w = 0;
            for (size_t c = 1; c < kids.size(); c++) {
                double *dst = (c + 1 == kids.size()) ? U(q) : d_ginv[w];
                dend_combine<<<g, kBlock, 0, s>>>(M, acc, Q(kids[c]), Gq, dst);
                acc = dst;
                w ^= 1;
            }
        }
        if (q > 0) launch_step1(U(q), d_gseg[o.seg[o.parent[q]]], Q(q), nullptr, nullptr, COMP_NONE);
    }
    // from segment 0 outwards, composing every segment
    SFGPU_CUDA_TRY(cudaMemcpyAsync(D(0), d_gseg[o.seg[0]], bytes, cudaMemcpyDeviceToDevice, s));
    double *const tmp[2] = {d_ginv[0], d_ginv[1]};
    for (int q = 0; q < N; q++) {
        const double *Gq = d_gseg[o.seg[q]];
        connect<<<g, kBlock, 0, s>>>(M, 1, U(q), D(q), o.d_phi[o.seg[q]]);
        const std::vector<int> &kids = o.kids[q];
        for (int c : kids) {
            const double *acc = D(q);
            int w = 0;
            for (int c2 : kids) {
                if (c2 == c) continue;
                dend_combine<<<g, kBlock, 0, s>>>(M, acc, Q(c2), Gq, tmp[w]);
                acc = tmp[w];
                w ^= 1;
            }
            launch_step1(acc, d_gseg[o.seg[c]], D(c), nullptr, nullptr, COMP_NONE);
        }
    }
    MolParam p;
    p.N = o.N; p.type = o.type; p.freedom = o.freedom; p.sym = 0; p.K = 1;
    p.pinned = o.pinned; p.solvent = (m == solvent); p.nmol = nmol;
    p.phibulk_in = o.phibulk; p.theta = o.theta;
    wsum_partial<<<nblocks_red, kBlock, 0, s>>>(M, 1, U(0), d_wgn, d_partial);
    mol_scalars<<<1, 1, 0, s>>>(p, nblocks_red, d_partial, (MolScal *)d_scal, m);
    for (int i : o.used) {
        finalize_phi<<<g, kBlock, 0, s>>>(M, d_gseg[i], o.d_phi[i], (const MolScal *)d_scal, m, 0);
        set_boundaries<<<g, kBlock, 0, s>>>(L, 1, o.d_phi[i]);
    }
    return SFGPU_OK;
}

// homopolymer ring (SF_HomoRing1stO::Matrix1): the profile of every site
// from its own walk (ring_phi); the boundary layers then hold copies, as the
// state profile has them once SF_SegmentList::PutSides has run
// SetBoundaries on it (SF_SegmentList.cpp:524-525)
int sfgpu_system::molecule_phi_ring(int m) {
    HMol &o = mols[m];
    cudaStream_t s = stream;
    const int Mmax = (o.N / 2 > M) ? 2 * M : M + o.N / 2;
    const size_t shm = (size_t)2 * (Mmax + 1) * sizeof(double);
    if (shm > 48 * 1024)
        SFGPU_CUDA_TRY(cudaFuncSetAttribute(ring_phi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
    const int threads = Mmax + 1 >= 256 ? 256 : 64;
    ring_phi<<<std::min(M, 148 * 8), threads, shm, s>>>(M, o.N, Mmax, d_gseg[o.seg[0]], o.phibulk, o.ring_norm0,
                                                       o.d_phi[o.seg[0]]);
    SFGPU_CUDA_TRY(cudaGetLastError());
    set_boundaries<<<grid_for(M), kBlock, 0, s>>>(H.L, 1, o.d_phi[o.seg[0]]);
    ring_scalars<<<1, 1, 0, s>>>(o.N, o.phibulk, (MolScal *)d_scal, m);
    return SFGPU_OK;
}

int sfgpu_system::molecule_phi(int m) {
    if (logmode) return molecule_phi_log(m);
    if (mols[m].dend) return molecule_phi_dend(m);
    if (mols[m].tree) return molecule_phi_tree(m);
    if (mols[m].ring) return molecule_phi_ring(m);
    HMol &o = mols[m];
    const DLat &L = H.L;
    const int g = grid_for(M);
    cudaStream_t s = stream;
    MolParam p;
    p.N = o.N; p.type = o.type; p.freedom = o.freedom; p.sym = o.sym; p.K = K;
    p.pinned = o.pinned; p.solvent = (m == solvent); p.nmol = nmol;
    p.phibulk_in = o.phibulk; p.theta = o.theta;
    if (m == neutralizer) { p.freedom = SFGPU_MOL_FREE; p.phib_dev = d_neut_phib; }
    MolScal *scal = (MolScal *)d_scal;
    const size_t KM = (size_t)K * M;
    if (o.type == 0) {
        int i = o.seg[0];
        // lnGN of the end-point distribution G itself (all K components equal)
        wsum_partial<<<nblocks_red, kBlock, 0, s>>>(M, 1, d_gseg[i], d_wgn, d_partial);
        MolParam p1 = p; p1.K = 1;
        mol_scalars<<<1, 1, 0, s>>>(p1, nblocks_red, d_partial, scal, m);
        finalize_phi<<<g, kBlock, 0, s>>>(M, d_gseg[i], o.d_phi[i], scal, m, 1);
        return SFGPU_OK;
    }
    for (int i : o.used) SFGPU_CUDA_TRY(cudaMemsetAsync(o.d_phi[i], 0, sizeof(double) * M, s));
    double *ginv = d_ginv[0], *tmp = d_ginv[1];
    if (o.sym) {
        const int i = o.seg[0];
        const double *G = d_gseg[i];
        const int N = o.N, half = N / 2;
        double *phi = o.d_phi[i];
        SFGPU_CUDA_TRY(cudaMemcpyAsync(d_gi, G, sizeof(double) * M, cudaMemcpyDeviceToDevice, s));
        for (int t = 1; t < half; t++)
            launch_step1(d_gi + (size_t)(t - 1) * M, G, d_gi + (size_t)t * M, nullptr, nullptr, COMP_NONE);
        const double *cur = d_gi + (size_t)(half - 1) * M;
        if (N % 2 == 1) {
            launch_step1(cur, G, ginv, nullptr, phi, COMP_CENTRE);
            cur = ginv; std::swap(ginv, tmp);
        }
        for (int sp = (N + 3) / 2; sp <= N; sp++) {
            int sinv = N - sp + 1;
            launch_step1(cur, G, ginv, d_gi + (size_t)(sinv - 1) * M, phi, COMP_ACC);
            cur = ginv; std::swap(ginv, tmp);
        }
        wsum_partial<<<nblocks_red, kBlock, 0, s>>>(M, 1, cur, d_wgn, d_partial);
        mol_scalars<<<1, 1, 0, s>>>(p, nblocks_red, d_partial, scal, m);
        finalize_phi<<<g, kBlock, 0, s>>>(M, G, phi, scal, m, 0);
        set_boundaries<<<g, kBlock, 0, s>>>(L, 1, phi);
        return SFGPU_OK;
    }
    // full storage: copolymers and all second-order chains
    const int N = o.N;
    // forward step into position t (SF_Copol1stO::Matrix1 / SF_Copol2ndO::Matrix1)
    auto fwd = [&](int t, const double *in, double *out) {
        int sg = o.seg[t];
        if (K == 1 && o.force != 0)   // SF_Copol1stO.cpp:1207-1211: PropagateG(Gi, G, s, force)
            step1_force_rows<<<grid_rows(L), kBlock, 0, s>>>(L, force_weights(L, o.force), in, d_gseg[sg], out,
                                                             nullptr, nullptr, COMP_NONE);
        else if (K == 1)
            launch_step1(in, d_gseg[sg], out, nullptr, nullptr, COMP_NONE);
        else if (K == 6 && L.stiff) {
            // SF_Copol2ndO_stiff_range::Matrix1 (SF_Copol2ndO_stiff_range.cpp:211-217):
            // step s (1-based) takes Pf(s-1, s+1); the last one is isotropic
            const bool last = (t == N - 1);
            const double Sv = last ? 0.2 : pf[o.seg[t - 1] * nseg + o.seg[t + 1]];
            launch_pdl(step2_rows, dim3(grid_rows(L)), dim3(kBlock), s, L, in, (const double *)d_gseg[sg], Sv, out,
                       (const double *)nullptr, (double *)nullptr, (int)COMP_NONE, 0,
                       (int)(last ? STEP2_ISO : STEP2_STIFF));
        } else if (K == 6)
            launch_pdl(step2_rows, dim3(grid_rows(L)), dim3(kBlock), s, L, in, (const double *)d_gseg[sg],
                       pf[o.seg[t - 1] * nseg + sg], out, (const double *)nullptr, (double *)nullptr, (int)COMP_NONE, 0,
                       (int)STEP2_PLAIN);
        else
            step2l_rows<<<grid_rows(L), kBlock, 0, s>>>(L, in, d_gseg[sg], pf[o.seg[t - 1] * nseg + sg], out,
                                        nullptr, nullptr, COMP_NONE, 0);
    };
    // backward step into position t with the composition phi += Gb(t) Gf(t)
    auto bwd = [&](int t, const double *in, double *out, const double *gf) {
        int sg = o.seg[t];
        if (K == 1 && o.force != 0)   // backward steps with -force (SF_Copol1stO.cpp:1226-1230)
            step1_force_rows<<<grid_rows(L), kBlock, 0, s>>>(L, force_weights(L, -o.force), in, d_gseg[sg], out, gf,
                                                             o.d_phi[sg], COMP_ACC);
        else if (K == 1)
            launch_step1(in, d_gseg[sg], out, gf, o.d_phi[sg], COMP_ACC);
        else if (K == 6 && L.stiff) {
            // backward step s (1-based) takes Pf(s, s+2); the first one
            // (s = N-1) is isotropic (SF_Copol2ndO_stiff_range.cpp:229-234)
            const bool first = (t == N - 2);
            const double Sv = first ? 0.2 : pf[sg * nseg + o.seg[t + 2]];
            launch_pdl(step2_rows, dim3(grid_rows(L)), dim3(kBlock), s, L, in, (const double *)d_gseg[sg], Sv, out, gf,
                       o.d_phi[sg], (int)COMP_ACC, 1, (int)(first ? STEP2_ISO : STEP2_STIFF));
        } else if (K == 6)
            launch_pdl(step2_rows, dim3(grid_rows(L)), dim3(kBlock), s, L, in, (const double *)d_gseg[sg],
                       pf[sg * nseg + o.seg[t + 1]], out, gf, o.d_phi[sg], (int)COMP_ACC, 1, (int)STEP2_PLAIN);
        else
            step2l_rows<<<grid_rows(L), kBlock, 0, s>>>(L, in, d_gseg[sg], pf[sg * nseg + o.seg[t + 1]], out, gf,
                                        o.d_phi[sg], COMP_ACC, 1);
    };
    const bool ori = orient && K > 1;
    // storage: every slice, or checkpoints ck[q] = Gf(qk) plus one segment
    // of slices seg[j] = Gf(qk + j), j = 1..k-1 (the forward sweep leaves the
    // last segment there; the others are recomputed from their checkpoint)
    const bool ckpt = primal_checkpointed(o);
    const int kst = ckpt ? primal_stride : N;
    const int nck = ckpt ? (N + kst - 1) / kst : 0;
    double *segbuf = ckpt ? d_gi + (size_t)nck * KM : nullptr;
    auto slot = [&](int t) -> double * {
        if (!ckpt) return d_gi + (size_t)t * KM;
        return (t % kst == 0) ? d_gi + (size_t)(t / kst) * KM : segbuf + (size_t)(t % kst) * KM;
    };
    replicate<<<g, kBlock, 0, s>>>(M, K, d_gseg[o.seg[0]], slot(0));
    if (K == 6) set_boundaries<<<g, kBlock, 0, s>>>(L, 6, slot(0));
    for (int t = 1; t < N; t++) fwd(t, slot(t - 1), slot(t));
    replicate<<<g, kBlock, 0, s>>>(M, K, d_gseg[o.seg[N - 1]], ginv);
    if (K == 6) set_boundaries<<<g, kBlock, 0, s>>>(L, 6, ginv);
    connect<<<g, kBlock, 0, s>>>(M, K, ginv, slot(N - 1), o.d_phi[o.seg[N - 1]]);
    if (ori) {
        for (int i : o.used) SFGPU_CUDA_TRY(cudaMemsetAsync(o.d_ori[i], 0, sizeof(double) * mphi() * M, s));
        orient_acc<<<g, kBlock, 0, s>>>(L, ginv, slot(N - 1), o.d_ori[o.seg[N - 1]]);
    }
    const double *cur = ginv;
    std::swap(ginv, tmp);
    int seg_held = ckpt ? (N - 1) / kst : -1;   // segment whose slices segbuf holds
    for (int t = N - 2; t >= 0; t--) {
        if (ckpt && t % kst != 0 && t / kst != seg_held) {
            const int q = t / kst;   // recompute Gf(qk+1 .. qk+k-1) from ck[q]
            for (int u = q * kst + 1; u <= std::min(q * kst + kst - 1, N - 1); u++) fwd(u, slot(u - 1), slot(u));
            seg_held = q;
        }
        bwd(t, cur, ginv, slot(t));
        if (ori) orient_acc<<<g, kBlock, 0, s>>>(L, ginv, slot(t), o.d_ori[o.seg[t]]);
        cur = ginv; std::swap(ginv, tmp);
    }
    wsum_partial<<<nblocks_red, kBlock, 0, s>>>(M, K, cur, d_wgn, d_partial);
    mol_scalars<<<1, 1, 0, s>>>(p, nblocks_red, d_partial, scal, m);
    for (int i : o.used) {
        finalize_phi<<<g, kBlock, 0, s>>>(M, d_gseg[i], o.d_phi[i], scal, m, 0);
        set_boundaries<<<g, kBlock, 0, s>>>(L, 1, o.d_phi[i]);
        // CorrectDoubleCountG / NormPhi* on the orientation slots
        // (Lat3D2ndO.cpp:986-993, :1031-1046)
        if (ori)
            for (int a = 0; a < mphi(); a++)
                finalize_phi<<<g, kBlock, 0, s>>>(M, d_gseg[i], o.d_ori[i] + (size_t)a * M, scal, m, 0);
    }
    return SFGPU_OK;
}

// Bond-orientation profiles (SF_Homopol2ndO::GetBondOrientation,
// SF_Homopol2ndO.cpp:82-90; SF_Copol2ndO.cpp:108-116): per molecule and
// segment type mphi profiles, filled by the residual evaluations that follow.
int sfgpu_system::set_orientation(int enable) {
    if (K == 1) return fail(SFGPU_ERR_UNSUPPORTED, "bond orientation needs a second-order lattice");
    if (H.L.stiff) return fail(SFGPU_ERR_UNSUPPORTED, "bond orientation with a stiff range");
    if (enable && !d_ori_sum) {
        int rc = alloc_d(&d_ori_sum, M);
        if (rc) return rc;
        for (auto &o : mols) {
            o.d_ori.assign(nseg, nullptr);
            for (int i : o.used) {
                if ((rc = alloc_d(&o.d_ori[i], (size_t)mphi() * M))) return rc;
                SFGPU_CUDA_TRY(cudaMemsetAsync(o.d_ori[i], 0, sizeof(double) * mphi() * M, stream));
            }
        }
    }
    orient = enable != 0;
    return SFGPU_OK;
}

int sfgpu_system::residual_async(const double *x, double *f) {
    const DLat &L = H.L;
    const int g = grid_for(M);
    cudaStream_t s = stream;
    // segment weighting factors; on a charged lattice psi0 and E^2 first
    if (charged) {
        q_psi0<<<g, kBlock, 0, s>>>(L, qp, x);
        if (L.grad == 3) {
            q_esq_3d<<<g, kBlock, 0, s>>>(L, qp);
            q_copy_boundaries<<<g, kBlock, 0, s>>>(L, qp.esq);
        } else if (L.grad == 2) {
            q_esq_2d<<<g, kBlock, 0, s>>>(L, qp);
        } else if (qp.curved) {
            q_esq_curved<<<g, kBlock, 0, s>>>(L, qp);
        } else {
            q_esq<<<g, kBlock, 0, s>>>(L, qp);
        }
    }
    for (int i = 0; i < nseg; i++) {
        if (freedom[i] == SFGPU_SEG_FROZEN) continue;
        if (charged)
            swf_update_q<<<g, kBlock, 0, s>>>(L, qp, x, class_of[i], i, d_range[i], freedom[i] == SFGPU_SEG_PINNED,
                                              d_gfull[i], d_gseg[i]);
        else
            swf_update<<<g, kBlock, 0, s>>>(L, x, d_jmap, nclass, class_of[i], d_range[i],
                                            freedom[i] == SFGPU_SEG_PINNED, d_gfull[i], d_gseg[i]);
        if (logmode) make_safe<<<g, kBlock, 0, s>>>(M, logc, d_gseg[i], d_lgseg[i]);
    }
    // molecules, the neutralizer after the others, solvent last
    // (SF_MolList1stO.cpp:246-295)
    for (int m = 0; m < nmol; m++) {
        if (m == solvent || m == neutralizer) continue;
        int rc = molecule_phi(m);
        if (rc) return rc;
    }
    if (neutralizer >= 0) {
        NeutParam np;
        np.nmol = nmol; np.solvent = solvent; np.self = neutralizer;
        for (int m = 0; m < nmol; m++) {
            double q = 0;
            for (int i : mols[m].used) q += 1.0 * valence[i] * mols[m].count[i];
            np.q[m] = q;
            np.n[m] = mols[m].N;
        }
        q_neutralizer<<<1, 1, 0, s>>>(np, (const MolScal *)d_scal, d_neut_phib);
        int rc = molecule_phi(neutralizer);
        if (rc) return rc;
    }
    int rc = molecule_phi(solvent);
    if (rc) return rc;
    // state profiles
    for (int i = 0; i < nseg; i++) {
        if (freedom[i] == SFGPU_SEG_FROZEN) continue;
        PtrList pl; pl.n = 0;
        for (auto &o : mols) if (o.count[i]) pl.p[pl.n++] = o.d_phi[i];
        sum_profiles<<<g, kBlock, 0, s>>>(M, pl, d_phi[i]);
    }
    bulk_scalars<<<1, 1, 0, s>>>(bp, ct, (const MolScal *)d_scal, d_phib, d_chib);
    ResParam rp;
    memset(&rp, 0, sizeof(rp));
    rp.nsites = nsites; rp.nclass = nclass; rp.nseg = nseg;
    for (int c = 0; c < nclass; c++) { rp.rep[c] = rep_of_class[c]; rp.gfull[c] = d_gfull[rep_of_class[c]]; }
    for (int i = 0; i < nseg; i++) rp.phi[i] = d_phi[i];
    if (charged) {
        // the Poisson sweep from psi0 before the contact averages
        // (SF_SegmentList::ComputeElectricPotential, SF_SegmentList.cpp:839-860)
        PtrList all;
        all.n = nseg;
        for (int i = 0; i < nseg; i++) all.p[i] = d_phi[i];
        q_eps_charge<<<g, kBlock, 0, s>>>(M, nseg, all, qp);
        if (L.grad == 3) {
            q_poisson_3d<<<g, kBlock, 0, s>>>(L, qp);
            q_copy_boundaries<<<g, kBlock, 0, s>>>(L, qp.psi);
        } else if (L.grad == 2) {
            q_poisson_2d<<<g, kBlock, 0, s>>>(L, qp);
        } else if (qp.curved) {
            q_poisson_curved<<<g, kBlock, 0, s>>>(L, qp);
        } else {
            q_poisson<<<g, kBlock, 0, s>>>(L, qp);
        }
        residual_q<<<g, kBlock, 0, s>>>(L, rp, ct, qp, d_chib, f);
    } else {
        residual<<<grid_for(nsites), kBlock, 0, s>>>(L, rp, ct, d_sites, d_chib, f);
    }
    SFGPU_CUDA_TRY(cudaGetLastError());
    return SFGPU_OK;
}

// Charges (SF_Solve.cpp:93-177; SF_Segment.cpp:170-217): valences and
// dielectric constants, the neutralizer, and the iteration layout of SFbox
// (per site its psi, then its class potentials: UpdateSWF, SF_Solve.cpp:
// 797-810).  psi is an iteration variable on the interior sites and on
// every site of a frozen segment's range (PotItVar, SF_Solve.cpp:1761-1776).
int sfgpu_system::setup_charges(const sfgpu_system_desc *d, const std::vector<int> &jmap) {
    const DLat &L = H.L;
    int rc;
    valence.assign(nseg, 0.0);
    epsilon.assign(nseg, 80.0);
    charged = false;
    for (int i = 0; i < nseg; i++) {
        valence[i] = d->segments[i].valence;
        if (d->segments[i].epsilon != 0) epsilon[i] = d->segments[i].epsilon;
        if (!std::isfinite(valence[i]) || !std::isfinite(epsilon[i])) return fail(SFGPU_ERR_INVALID, "valence and epsilon must be finite");
        if (valence[i] != 0) charged = true;
    }
    neutralizer = -1;
    for (int m = 0; m < nmol; m++)
        if (mols[m].freedom == SFGPU_MOL_NEUTRALIZER) {
            if (neutralizer >= 0) return fail(SFGPU_ERR_INVALID, "more than one neutralizer");
            neutralizer = m;
        }
    if (!charged) {
        if (neutralizer >= 0) return fail(SFGPU_ERR_INVALID, "a neutralizer needs charged segments");
        return SFGPU_OK;
    }
    auto bulk_charge = [&](const HMol &o) {
        double q = 0;
        for (int i : o.used) q += 1.0 * valence[i] * o.count[i];
        return q;
    };
    if (neutralizer >= 0) {
        const HMol &o = mols[neutralizer];
        if (o.dend || o.tree || o.ring) return fail(SFGPU_ERR_UNSUPPORTED, "a branched neutralizer");
        if (bulk_charge(o) == 0) return fail(SFGPU_ERR_INVALID, "the neutralizer carries no charge");
    } else {
        for (const auto &o : mols)   // SF_Solve.cpp:100-107
            if (o.freedom == SFGPU_MOL_FREE && bulk_charge(o) != 0)
                return fail(SFGPU_ERR_INVALID, "charged free molecules need a neutralizer molecule");
    }
    int diffeps = 0;   // SF_Solve.cpp:154-162
    for (int i = 0; i < nseg; i++)
        for (int j = 0; j < nseg; j++)
            if (freedom[i] != SFGPU_SEG_FROZEN && freedom[j] != SFGPU_SEG_FROZEN && epsilon[i] != epsilon[j]) diffeps = 1;
    // layout
    std::vector<int> xu(M, -1), xp(M, -1);
    std::vector<double> surf(M, 0.0);
    long long k = 0;
    for (int z = 0; z < M; z++) {
        int c[3];
        lat_coords(L, z, c);
        bool pot = lat_interior(L, c);
        for (int i = 0; i < nseg; i++)
            if (freedom[i] == SFGPU_SEG_FROZEN && range_h[(size_t)i * M + z] > 0) { pot = true; surf[z] = 1.0; }
        if (pot) xp[z] = (int)k++;
        if (jmap[z] >= 0) { xu[z] = (int)k; k += nclass; }
        // the 3D sweep leaves boundary layers to SetBoundaries (Lat3D.cpp:1966):
        // a psi there would be a copy, not a variable
        if (pot && L.grad == 3 && !lat_interior(L, c))
            return fail(SFGPU_ERR_UNSUPPORTED, "3D charges with frozen segments on a boundary layer");
    }
    nvar = (size_t)k;
    // lattice sites per layer (Lat1DFlat::MultiplyWithLatticeSites, Lat1DFlat.cpp:266-269)
    const double ladj = d->lattice.layer_adjustment > 0 ? d->lattice.layer_adjustment : 1.0;
    std::vector<double> ls(M, 1.0);
    if (L.cyl) {   // Lat1DCylinder.cpp:127-132, Lat2DCylinder.cpp:156-164: the sites of the row
        for (int z = 0; z < M; z++) {
            int c[3];
            lat_coords(L, z, c);
            ls[z] = H.Lx[c[0]];
        }
    } else if (L.grad == 1 && M > 3) {
        ls[1] *= ladj;
        ls[M - 2] *= 2 - ladj;
    }
    memset(&qp, 0, sizeof(qp));
    qp.diffeps = diffeps;
    qp.surf_lo = L.bc_lo[0] == SFGPU_BOUND_SURFACE;
    qp.surf_hi = L.bc_hi[0] == SFGPU_BOUND_SURFACE;
    qp.map_lo = lat_map(L, 0);
    qp.map_hi = lat_map(L, M - 1);
    qp.curved = L.cyl && L.grad == 1;
    qp.cyl2 = L.cyl && L.grad == 2;
    if (L.grad >= 2) {
        qp.surf_ylo = L.bc_lo[1] == SFGPU_BOUND_SURFACE;
        qp.surf_yhi = L.bc_hi[1] == SFGPU_BOUND_SURFACE;
    }
    if (qp.cyl2) qp.z0c = H.Lx[2] / 2 / sfk::kPi - 2;   // Lat2DCylinder.cpp:337
    qp.sph = d->lattice.geometry == SFGPU_GEOM_SPHERICAL;
    qp.off1 = d->lattice.offset_first_layer;
    qp.ladj = ladj;
    const double T = d->temperature > 0 ? d->temperature : 298.15;                      // SF_System.cpp:68
    const double bl = d->lattice.bondlength > 0 ? d->lattice.bondlength : 3e-10;       // Lat1DFlat.cpp:128
    // the site distance: bondlength / sqrt(2 dimensions lambda) on the 1D and 2D
    // lattices (Lat1DFlat.cpp:129, Lat2DFlat.cpp:209), the bondlength in 3D (Lat3D.cpp:263)
    const double dims = d->lattice.dimensions > 0 ? d->lattice.dimensions : 3.0;
    const double sd = L.grad == 3 ? bl : bl / sqrt(2 * dims * L.l1);
    qp.kT = sfk::kBoltzmann * T;
    qp.pf_esq = (sfk::kEps0 * sd) / qp.kT;
    qp.pf_psi = (sfk::kElemCharge / sfk::kEps0) / sd;
    for (int i = 0; i < nseg; i++) { qp.val[i] = valence[i]; qp.eps[i] = epsilon[i]; }
    int *dxu, *dxp;
    double *dls;
    if ((rc = alloc_i(&dxu, M)) || (rc = alloc_i(&dxp, M)) || (rc = alloc_d(&dls, M))) return rc;
    if ((rc = alloc_d(&qp.psi0, M)) || (rc = alloc_d(&qp.psi, M)) || (rc = alloc_d(&qp.esq, M)) ||
        (rc = alloc_d(&qp.epsav, M)) || (rc = alloc_d(&qp.charge, M)) || (rc = alloc_d(&d_el, M)) ||
        (rc = alloc_d(&d_surf, M)) || (rc = alloc_d(&d_neut_phib, 1)))
        return rc;
    SFGPU_CUDA_TRY(cudaMemcpy(dxu, xu.data(), sizeof(int) * M, cudaMemcpyHostToDevice));
    SFGPU_CUDA_TRY(cudaMemcpy(dxp, xp.data(), sizeof(int) * M, cudaMemcpyHostToDevice));
    SFGPU_CUDA_TRY(cudaMemcpy(dls, ls.data(), sizeof(double) * M, cudaMemcpyHostToDevice));
    SFGPU_CUDA_TRY(cudaMemcpy(d_surf, surf.data(), sizeof(double) * M, cudaMemcpyHostToDevice));
    for (double *p : {qp.psi0, qp.psi, qp.esq, qp.epsav, qp.charge, d_el, d_neut_phib})
        SFGPU_CUDA_TRY(cudaMemset(p, 0, sizeof(double) * (p == d_neut_phib ? 1 : M)));
    qp.xu = dxu;
    qp.xp = dxp;
    qp.lsites = dls;
    return SFGPU_OK;
}

int sfgpu_system::free_energy(double *F) {
    FreeParam fp;
    memset(&fp, 0, sizeof(fp));
    fp.nseg = nseg; fp.nmol = nmol;
    for (int i = 0; i < nseg; i++) { fp.phi[i] = d_phi[i]; fp.gseg[i] = d_gseg[i] ? d_gseg[i] : d_phi[i]; }
    for (int m = 0; m < nmol; m++) {
        fp.invN[m] = 1.0 / mols[m].N;
        fp.lnN[m] = log((double)mols[m].N);
        fp.chemintref[m] = mols[m].chemintref;
        for (int i : mols[m].used) fp.mphi[m * SFGPU_MAX_SEG + i] = mols[m].d_phi[i];
    }
    if (charged) q_elec<<<grid_for(M), kBlock, 0, stream>>>(M, qp, d_el);
    free_energy_partial<<<nblocks_red, kBlock, 0, stream>>>(H.L, fp, ct, d_wf, (const MolScal *)d_scal, d_partial,
                                                            charged ? d_el : nullptr);
    finish_sums<<<1, 32, 0, stream>>>(1, nblocks_red, d_partial, d_misc);
    SFGPU_CUDA_TRY(cudaMemcpyAsync(F, d_misc, sizeof(double), cudaMemcpyDeviceToHost, stream));
    SFGPU_CUDA_TRY(cudaStreamSynchronize(stream));
    return SFGPU_OK;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
#define CHECK_SYS(s) do { if (!(s)) return fail(SFGPU_ERR_INVALID, "null system"); } while (0)

extern "C" int sfgpu_device_count(int *count) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) { *count = 0; cudaGetLastError(); return SFGPU_ERR_NODEVICE; }
    *count = n;
    return n > 0 ? SFGPU_OK : SFGPU_ERR_NODEVICE;
}

// the full-storage chains (copolymers, second-order chains; not dendrimers,
// not symmetric homopolymers, which store half a chain) when a stride is set
bool sfgpu_system::primal_checkpointed(const HMol &o) const {
    return primal_stride > 0 && primal_stride < o.N && o.type != 0 && !o.dend && !o.sym && !o.tree && !o.ring &&
           !logmode;
}

static int create_system(const sfgpu_system_desc *desc, int stride, sfgpu_system **out) {
    if (!desc || !out) return fail(SFGPU_ERR_INVALID, "null argument");
    if (stride < 0) return fail(SFGPU_ERR_INVALID, "checkpoint stride must be >= 0");
    *out = nullptr;
    int n = 0;
    if (sfgpu_device_count(&n) != SFGPU_OK) return fail(SFGPU_ERR_NODEVICE, "no CUDA device");
    sfgpu_system *s = new sfgpu_system();
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { delete s; sfgpu_set_error(e, "cudaStreamCreate", __FILE__, __LINE__); return SFGPU_ERR_CUDA; }
    s->own_stream = true;
    // the log-space chains (overflow protection) keep every slice
    s->primal_stride = desc->overflow_protection ? 0 : stride;
    int rc = s->setup(desc);
    if (rc) { delete s; return rc; }
    *out = s;
    return SFGPU_OK;
}

extern "C" int sfgpu_system_create(const sfgpu_system_desc *desc, sfgpu_system **out) {
    return create_system(desc, 0, out);
}

extern "C" int sfgpu_system_create_checkpointed(const sfgpu_system_desc *desc, int stride, sfgpu_system **out) {
    return create_system(desc, stride, out);
}

extern "C" int sfgpu_system_destroy(sfgpu_system *s) {
    if (!s) return SFGPU_OK;
    cudaStreamSynchronize(s->stream);
    delete s;
    return SFGPU_OK;
}

extern "C" int sfgpu_system_info(sfgpu_system *s, int *M, int *nvar, int *nclass, int *nsites) {
    CHECK_SYS(s);
    if (M) *M = s->M;
    if (nvar) *nvar = (int)s->nvar;
    if (nclass) *nclass = s->nclass;
    if (nsites) *nsites = s->nsites;
    return SFGPU_OK;
}

extern "C" int sfgpu_system_stream(sfgpu_system *s, void **stream) {
    CHECK_SYS(s);
    *stream = (void *)s->stream;
    return SFGPU_OK;
}

extern "C" int sfgpu_residual(sfgpu_system *s, const double *x_dev, double *f_dev) {
    CHECK_SYS(s);
    return s->residual_async(x_dev, f_dev);
}

extern "C" int sfgpu_residual_host(sfgpu_system *s, const double *x, double *f) {
    CHECK_SYS(s);
    SFGPU_CUDA_TRY(cudaMemcpyAsync(s->d_x, x, sizeof(double) * s->nvar, cudaMemcpyHostToDevice, s->stream));
    int rc = s->residual_async(s->d_x, s->d_f);
    if (rc) return rc;
    SFGPU_CUDA_TRY(cudaMemcpyAsync(f, s->d_f, sizeof(double) * s->nvar, cudaMemcpyDeviceToHost, s->stream));
    SFGPU_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return SFGPU_OK;
}

extern "C" int sfgpu_system_set_stream(sfgpu_system *s, void *stream) {
    CHECK_SYS(s);
    SFGPU_CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
    s->own_stream = false;
    s->stream = (cudaStream_t)stream;
    return SFGPU_OK;
}

extern "C" int sfgpu_synchronize(sfgpu_system *s) {
    CHECK_SYS(s);
    SFGPU_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return SFGPU_OK;
}

extern "C" int sfgpu_get_phi(sfgpu_system *s, int seg, double *phi) {
    CHECK_SYS(s);
    if (seg < 0 || seg >= s->nseg) return fail(SFGPU_ERR_INVALID, "segment index");
    SFGPU_CUDA_TRY(cudaMemcpyAsync(phi, s->d_phi[seg], sizeof(double) * s->M, cudaMemcpyDeviceToHost, s->stream));
    SFGPU_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return SFGPU_OK;
}

extern "C" int sfgpu_get_mol_phi(sfgpu_system *s, int mol, int seg, double *phi) {
    CHECK_SYS(s);
    if (mol < 0 || mol >= s->nmol || seg < 0 || seg >= s->nseg) return fail(SFGPU_ERR_INVALID, "index");
    const double *p = s->mols[mol].d_phi[seg];
    if (!p) { memset(phi, 0, sizeof(double) * s->M); return SFGPU_OK; }
    SFGPU_CUDA_TRY(cudaMemcpyAsync(phi, p, sizeof(double) * s->M, cudaMemcpyDeviceToHost, s->stream));
    SFGPU_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return SFGPU_OK;
}

extern "C" int sfgpu_get_mol_scalars(sfgpu_system *s, int mol, double *lngn, double *phibulk, double *lnc) {
    CHECK_SYS(s);
    if (mol < 0 || mol >= s->nmol) return fail(SFGPU_ERR_INVALID, "molecule index");
    MolScal v;
    SFGPU_CUDA_TRY(cudaMemcpyAsync(&v, (MolScal *)s->d_scal + mol, sizeof(v), cudaMemcpyDeviceToHost, s->stream));
    SFGPU_CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (lngn) *lngn = v.lngn;
    if (phibulk) *phibulk = v.phibulk;
    if (lnc) *lnc = v.lnc;
    return SFGPU_OK;
}

extern "C" int sfgpu_system_set_bond_orientation(sfgpu_system *s, int enable) {
    CHECK_SYS(s);
    return s->set_orientation(enable);
}

extern "C" int sfgpu_get_bond_orientation(sfgpu_system *s, int mol, int axis, double *out) {
    CHECK_SYS(s);
    if (!out) return fail(SFGPU_ERR_INVALID, "null output");
    if (!s->orient) return fail(SFGPU_ERR_INVALID, "bond orientation is not enabled");
    if (mol < 0 || mol >= s->nmol) return fail(SFGPU_ERR_INVALID, "molecule index");
    if (axis < 0 || axis >= s->mphi()) return fail(SFGPU_ERR_INVALID, "axis out of range for this lattice");
    const HMol &o = s->mols[mol];
    PtrList pl; pl.n = 0;
    for (int i : o.used) pl.p[pl.n++] = o.d_ori[i] + (size_t)axis * s->M;
    sum_profiles<<<grid_for(s->M), kBlock, 0, s->stream>>>(s->M, pl, s->d_ori_sum);
    SFGPU_CUDA_TRY(cudaGetLastError());
    SFGPU_CUDA_TRY(cudaMemcpyAsync(out, s->d_ori_sum, sizeof(double) * s->M, cudaMemcpyDeviceToHost, s->stream));
    SFGPU_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return SFGPU_OK;
}

extern "C" int sfgpu_get_swf(sfgpu_system *s, int seg, double *g) {
    CHECK_SYS(s);
    if (seg < 0 || seg >= s->nseg || !s->d_gseg[seg]) return fail(SFGPU_ERR_INVALID, "segment index");
    SFGPU_CUDA_TRY(cudaMemcpyAsync(g, s->d_gseg[seg], sizeof(double) * s->M, cudaMemcpyDeviceToHost, s->stream));
    SFGPU_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return SFGPU_OK;
}

// F and the grand potential with their densities (SF_MolList1stO::
// GetFreeEnergy / GetGrandPotential with GetFreeEnergyProfile and
// GetGrandPotentialProfile, SF_MolList1stO.cpp:606-646, 815-826, 1001-1101)
int sfgpu_system::thermo(double *F, double *Omega, double *fe, double *gp) {
    ThermoParam tp;
    memset(&tp, 0, sizeof(tp));
    tp.nseg = nseg; tp.nmol = nmol;
    for (int i = 0; i < nseg; i++) {
        tp.phi[i] = d_phi[i];
        tp.gseg[i] = d_gseg[i] ? d_gseg[i] : d_phi[i];
        tp.gfull[i] = d_gfull[i] ? d_gfull[i] : d_phi[i];
        tp.frozen[i] = freedom[i] == SFGPU_SEG_FROZEN;
    }
    for (int m = 0; m < nmol; m++) {
        tp.invN[m] = 1.0 / mols[m].N;
        tp.N[m] = (double)mols[m].N;
        tp.lnN[m] = log((double)mols[m].N);
        tp.chemintref[m] = mols[m].chemintref;
        for (int i : mols[m].used) tp.mphi[m * SFGPU_MAX_SEG + i] = mols[m].d_phi[i];
    }
    if (charged) {
        q_elec<<<grid_for(M), kBlock, 0, stream>>>(M, qp, d_el);
        tp.el = d_el;
        tp.psi = qp.psi;
        tp.surf = d_surf;
        for (int i = 0; i < nseg; i++) tp.val[i] = valence[i];
        tp.ech = sfk::kElemCharge;
        tp.kT = qp.kT;
    }
    double *dfe = (fe || gp) ? d_ginv[0] : nullptr, *dgp = (fe || gp) ? d_ginv[1] : nullptr;
    thermo_partial<<<nblocks_red, kBlock, 0, stream>>>(H.L, tp, ct, d_wf, d_sb, (const MolScal *)d_scal, d_phib,
                                                      dfe, dgp, d_partial);
    finish_sums<<<1, 32, 0, stream>>>(2, nblocks_red, d_partial, d_misc);
    SFGPU_CUDA_TRY(cudaGetLastError());
    double v[2];
    SFGPU_CUDA_TRY(cudaMemcpyAsync(v, d_misc, sizeof(v), cudaMemcpyDeviceToHost, stream));
    if (fe) SFGPU_CUDA_TRY(cudaMemcpyAsync(fe, dfe, sizeof(double) * M, cudaMemcpyDeviceToHost, stream));
    if (gp) SFGPU_CUDA_TRY(cudaMemcpyAsync(gp, dgp, sizeof(double) * M, cudaMemcpyDeviceToHost, stream));
    SFGPU_CUDA_TRY(cudaStreamSynchronize(stream));
    if (F) *F = v[0];
    if (Omega) *Omega = v[1];
    return SFGPU_OK;
}

extern "C" int sfgpu_lattice_weights(sfgpu_system *s, double *w_lngn, double *w_sum) {
    CHECK_SYS(s);
    if (w_lngn) memcpy(w_lngn, s->H.w_gn.data(), sizeof(double) * s->M);
    if (w_sum) memcpy(w_sum, s->H.w_f.data(), sizeof(double) * s->M);
    return SFGPU_OK;
}

extern "C" int sfgpu_thermo(sfgpu_system *s, double *F, double *Omega, double *fe_profile, double *omega_profile) {
    CHECK_SYS(s);
    return s->thermo(F, Omega, fe_profile, omega_profile);
}

extern "C" int sfgpu_free_energy(sfgpu_system *s, double *F) {
    CHECK_SYS(s);
    return s->free_energy(F);
}

// Lattice-level entry points (Lat1stO::PropagateG, Lat2ndO::PropagateF/B,
// Lattice::SideFraction/Sides, Lat1stO::ComputeLnGN) on device vectors
extern "C" int sfgpu_lat_propagate(sfgpu_system *s, const double *gin, const double *g, double *gout,
                                   double S, int backward) {
    CHECK_SYS(s);
    if (gin == gout) return fail(SFGPU_ERR_INVALID, "gin and gout must differ");
    int gr = grid_for(s->M);
    if (s->logmode) {
        // Lat1DFlat1stOS::PropagateG and the other *1stOS steps on logarithms:
        // interior by the step, surfaces LOGZERO, other boundaries copies
        fill_value<<<gr, kBlock, 0, s->stream>>>(s->M, SFGPU_LOGZERO, gout);
        step1_log_rows<<<grid_rows(s->H.L), kBlock, 0, s->stream>>>(s->H.L, s->logq, s->logc, gin, g, gout, nullptr,
                                                                    nullptr, COMP_NONE);
        set_boundaries<<<gr, kBlock, 0, s->stream>>>(s->H.L, 1, gout);
    } else if (s->K == 1)
        step1<<<gr, kBlock, 0, s->stream>>>(s->H.L, gin, g, gout, nullptr, nullptr, COMP_NONE);
    else if (s->K == 6)
        step2<<<gr, kBlock, 0, s->stream>>>(s->H.L, gin, g, S, gout, nullptr, nullptr, COMP_NONE, backward);
    else
        step2l_rows<<<grid_rows(s->H.L), kBlock, 0, s->stream>>>(s->H.L, gin, g, S, gout, nullptr, nullptr, COMP_NONE,
                                                                backward);
    SFGPU_CUDA_TRY(cudaGetLastError());
    return SFGPU_OK;
}

extern "C" int sfgpu_lat_set_boundaries(sfgpu_system *s, double *p, int components) {
    CHECK_SYS(s);
    if (components != 1 && components != s->K) return fail(SFGPU_ERR_INVALID, "components must be 1 or the lattice's K");
    set_boundaries<<<grid_for(s->M), kBlock, 0, s->stream>>>(s->H.L, components, p);
    SFGPU_CUDA_TRY(cudaGetLastError());
    return SFGPU_OK;
}

extern "C" int sfgpu_lat_side_fraction(sfgpu_system *s, const double *phi, double *rho) {
    CHECK_SYS(s);
    side_kernel<<<grid_for(s->M), kBlock, 0, s->stream>>>(s->H.L, phi, rho);
    SFGPU_CUDA_TRY(cudaGetLastError());
    return SFGPU_OK;
}

extern "C" int sfgpu_lat_lngn(sfgpu_system *s, const double *g, int components, double *lngn) {
    CHECK_SYS(s);
    if (components != 1 && components != s->K) return fail(SFGPU_ERR_INVALID, "components must be 1 or the lattice's K");
    if (s->logmode) {   // ComputeLnGN of the *1stOS lattices: g holds logarithms
        lse_weighted<<<1, 1024, 0, s->stream>>>(s->M, g, s->d_wos, s->d_misc);
        SFGPU_CUDA_TRY(cudaMemcpyAsync(lngn, s->d_misc, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
        SFGPU_CUDA_TRY(cudaStreamSynchronize(s->stream));
        return SFGPU_OK;
    }
    wsum_partial<<<s->nblocks_red, kBlock, 0, s->stream>>>(s->M, components, g, s->d_wgn, s->d_partial);
    finish_sums<<<1, 32, 0, s->stream>>>(1, s->nblocks_red, s->d_partial, s->d_misc);
    double v = 0;
    SFGPU_CUDA_TRY(cudaMemcpyAsync(&v, s->d_misc, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    SFGPU_CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (components > 1) v /= 6.0;
    *lngn = log(v);
    return SFGPU_OK;
}

// ---- composition and normalisation on device vectors --------------------
namespace {
// CorrectDoubleCountG: phi /= G where G > 0, else 0 (tools.cpp:86-90)
__global__ void lat_correct_kernel(int M, const double *__restrict__ G, double *__restrict__ phi) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < M; r += gridDim.x * blockDim.x) {
        const double g = G[r];
        phi[r] = (g > 0) ? phi[r] / g : 0.0;
    }
}
// NormPhiFree: phi *= C
__global__ void lat_scale_kernel(int M, double C, double *__restrict__ phi) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < M; r += gridDim.x * blockDim.x) phi[r] *= C;
}
// NormPhiRestr: C /= exp(ComputeLnGN(Gi)) (first order) or
// 6 exp(ComputeLnGN(Gi)) (second order, whose lnGN already holds the 1/6),
// with the weighted end-point sum in *wsum
__global__ void lat_scale_restr_kernel(int M, double C, int K, const double *__restrict__ wsum,
                                       double *__restrict__ phi) {
    double v = *wsum;
    if (K > 1) v /= 6.0;
    const double lngn = log(v);
    const double c = (K > 1) ? C / (6.0 * exp(lngn)) : C / exp(lngn);
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < M; r += gridDim.x * blockDim.x) phi[r] *= c;
}
}  // namespace

extern "C" int sfgpu_lat_connect(sfgpu_system *s, const double *gb, const double *gf, double *phi, int components) {
    CHECK_SYS(s);
    if (s->logmode) return fail(SFGPU_ERR_UNSUPPORTED, "lattice-level composition on the log-space lattices");
    if (components != s->K) return fail(SFGPU_ERR_INVALID, "components must be the lattice's K");
    if (!gb || !gf || !phi) return fail(SFGPU_ERR_INVALID, "null device vector");
    connect<<<grid_for(s->M), kBlock, 0, s->stream>>>(s->M, components, gb, gf, phi);
    SFGPU_CUDA_TRY(cudaGetLastError());
    return SFGPU_OK;
}

extern "C" int sfgpu_lat_correct_double_count(sfgpu_system *s, double *phi, const double *g) {
    CHECK_SYS(s);
    if (s->logmode) return fail(SFGPU_ERR_UNSUPPORTED, "lattice-level composition on the log-space lattices");
    if (!g || !phi) return fail(SFGPU_ERR_INVALID, "null device vector");
    lat_correct_kernel<<<grid_for(s->M), kBlock, 0, s->stream>>>(s->M, g, phi);
    SFGPU_CUDA_TRY(cudaGetLastError());
    return SFGPU_OK;
}

extern "C" int sfgpu_lat_norm_phi_free(sfgpu_system *s, double *phi, double C) {
    CHECK_SYS(s);
    if (s->logmode) return fail(SFGPU_ERR_UNSUPPORTED, "lattice-level normalisation on the log-space lattices");
    if (!phi) return fail(SFGPU_ERR_INVALID, "null device vector");
    lat_scale_kernel<<<grid_for(s->M), kBlock, 0, s->stream>>>(s->M, C, phi);
    SFGPU_CUDA_TRY(cudaGetLastError());
    return SFGPU_OK;
}

extern "C" int sfgpu_lat_norm_phi_restr(sfgpu_system *s, double *phi, const double *gb, int components, double C) {
    CHECK_SYS(s);
    if (s->logmode) return fail(SFGPU_ERR_UNSUPPORTED, "lattice-level normalisation on the log-space lattices");
    if (components != s->K) return fail(SFGPU_ERR_INVALID, "components must be the lattice's K");
    if (!gb || !phi) return fail(SFGPU_ERR_INVALID, "null device vector");
    wsum_partial<<<s->nblocks_red, kBlock, 0, s->stream>>>(s->M, components, gb, s->d_wgn, s->d_partial);
    finish_sums<<<1, 32, 0, s->stream>>>(1, s->nblocks_red, s->d_partial, s->d_misc);
    lat_scale_restr_kernel<<<grid_for(s->M), kBlock, 0, s->stream>>>(s->M, C, components, s->d_misc, phi);
    SFGPU_CUDA_TRY(cudaGetLastError());
    return SFGPU_OK;
}

// Timing of the dominant kernels on this system's buffers: reps launches of
// a forward step and of a backward step with fused composition, bracketed by
// CUDA events on the system stream.  Algorithmic bytes per launch follow the
// per-site counts of the step: forward 8*(K+1+K) (read G(s-1), G, write
// G(s)), backward 8*(K+1+K+K+2) (also read Gf(s), read and write phi).
extern "C" int sfgpu_profile_propagator(sfgpu_system *s, int reps, double *ms_fwd, double *ms_bwd,
                                        double *bytes_fwd, double *bytes_bwd) {
    CHECK_SYS(s);
    if (reps < 1) return fail(SFGPU_ERR_INVALID, "reps must be positive");
    int mol = -1;
    for (int m = 0; m < s->nmol; m++) if (s->mols[m].type != 0) { mol = m; break; }
    if (mol < 0) return fail(SFGPU_ERR_INVALID, "no chain molecule to time");
    const HMol &o = s->mols[mol];
    const int K = s->K, M = s->M;
    const size_t KM = (size_t)K * M;
    size_t nslices = (size_t)(o.sym ? std::max(1, o.N / 2) : o.N);
    if (nslices < 2) return fail(SFGPU_ERR_INVALID, "chain too short to time");
    const double *G = s->d_gseg[o.seg[0]];
    double *phi = o.d_phi[o.seg[0]];
    const int g = grid_for(M);
    cudaEvent_t e0, e1, e2;
    SFGPU_CUDA_TRY(cudaEventCreate(&e0));
    SFGPU_CUDA_TRY(cudaEventCreate(&e1));
    SFGPU_CUDA_TRY(cudaEventCreate(&e2));
    SFGPU_CUDA_TRY(cudaEventRecord(e0, s->stream));
    for (int r = 0; r < reps; r++) {
        size_t t = 1 + (size_t)r % (nslices - 1);
        if (K == 1)
            s->launch_step1(s->d_gi + (t - 1) * KM, G, s->d_gi + t * KM, nullptr, nullptr, COMP_NONE);
        else
            launch_pdl(step2_rows, dim3(grid_rows(s->H.L)), dim3(kBlock), s->stream, s->H.L,
                       (const double *)(s->d_gi + (t - 1) * KM), G, 0.2, s->d_gi + t * KM, (const double *)nullptr,
                       (double *)nullptr, (int)COMP_NONE, 0, (int)STEP2_PLAIN);
    }
    SFGPU_CUDA_TRY(cudaEventRecord(e1, s->stream));
    for (int r = 0; r < reps; r++) {
        size_t t = (size_t)r % nslices;
        const double *src = s->d_ginv[r & 1];
        double *dst = s->d_ginv[(r + 1) & 1];
        if (K == 1)
            s->launch_step1(src, G, dst, s->d_gi + t * KM, phi, COMP_ACC);
        else
            launch_pdl(step2_rows, dim3(grid_rows(s->H.L)), dim3(kBlock), s->stream, s->H.L, src, G, 0.2, dst,
                       (const double *)(s->d_gi + t * KM), phi, (int)COMP_ACC, 1, (int)STEP2_PLAIN);
    }
    SFGPU_CUDA_TRY(cudaEventRecord(e2, s->stream));
    SFGPU_CUDA_TRY(cudaEventSynchronize(e2));
    float a = 0, b = 0;
    SFGPU_CUDA_TRY(cudaEventElapsedTime(&a, e0, e1));
    SFGPU_CUDA_TRY(cudaEventElapsedTime(&b, e1, e2));
    cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(e2);
    if (ms_fwd) *ms_fwd = a / reps;
    if (ms_bwd) *ms_bwd = b / reps;
    if (bytes_fwd) *bytes_fwd = 8.0 * (2 * K + 1) * M;
    if (bytes_bwd) *bytes_bwd = 8.0 * (3 * K + 3) * M;
    return SFGPU_OK;
}

// Pick the x-chunk depth of the 3D first-order step, and whether the
// software-pipelined form runs it, by timing each candidate on this system's
// buffers (CUDA events, `reps` forward + backward steps each); the fastest is
// kept for all later evaluations.  Other lattices have nothing to tune.
extern "C" int sfgpu_system_autotune(sfgpu_system *s, int reps, int *chosen_xc, double *best_ms) {
    CHECK_SYS(s);
    if (reps < 1) return fail(SFGPU_ERR_INVALID, "reps must be positive");
    if (s->H.L.grad != 3 || s->K != 1) {
        if (chosen_xc) *chosen_xc = s->tile_xc;
        if (best_ms) *best_ms = 0;
        return SFGPU_OK;
    }
    // forward and backward steps are timed by the same profile call; each
    // keeps its own fastest (depth, form)
    // forms: 0 plain, 1 pipelined, 2 (forward only) pipelined with two y rows
    // per thread
    const int cand[] = {2, 4, 8, 16, 32};
    double bf = 1e30, bb = 1e30;
    int fx = s->tile_xc, fp = s->tile_pipelined, bx = s->tile_xc_bwd, bp = s->tile_pipelined_bwd;
    for (int pl = 0; pl < 3; pl++)
        for (int c : cand) {
            s->tile_xc = s->tile_xc_bwd = c;
            s->tile_pipelined = pl;
            s->tile_pipelined_bwd = pl != 0;
            double f = 0, b = 0;
            int rc = sfgpu_profile_propagator(s, reps, &f, &b, nullptr, nullptr);
            if (rc) return rc;
            if (f < bf) { bf = f; fx = c; fp = pl; }
            if (pl < 2 && b < bb) { bb = b; bx = c; bp = pl; }
        }
    s->tile_xc = fx; s->tile_pipelined = fp;
    s->tile_xc_bwd = bx; s->tile_pipelined_bwd = bp;
    if (chosen_xc) *chosen_xc = fx;
    if (best_ms) *best_ms = bf + bb;
    return SFGPU_OK;
}

extern "C" int sfgpu_system_set_tile_pipelined(sfgpu_system *s, int enable) {
    CHECK_SYS(s);
    if (enable < 0 || enable > 2) return fail(SFGPU_ERR_INVALID, "the step form is 0, 1 or 2");
    s->tile_pipelined = enable;
    s->tile_pipelined_bwd = enable != 0;
    return SFGPU_OK;
}

extern "C" int sfgpu_system_set_tile(sfgpu_system *s, int xc) {
    CHECK_SYS(s);
    if (xc < 1 || xc > 1024) return fail(SFGPU_ERR_INVALID, "tile depth must be in 1..1024");
    s->tile_xc = s->tile_xc_bwd = xc;
    return SFGPU_OK;
}
