/*
 * sfgpu.h -- C ABI of the B200-native Scheutjens-Fleer SCF hot path.
 *
 * The library (field_b200/libsfgpu.so) replaces the propagation, composition,
 * segment-potential update and residual steps of SFbox 2.1 (the Wageningen
 * SF-SCF lattice program).  Every entry point is plain C: scalars, raw
 * pointers and sizes, no C++ or torch types.  Device pointers are CUDA
 * global-memory pointers on the current device; host pointers are ordinary
 * process memory.  Every call returns an int status (SFGPU_OK == 0).
 *
 * Index conventions follow SFbox: a lattice with n interior layers per
 * gradient carries one boundary layer on each side, so M = prod(n_i + 2).
 * Site z (0-based here, 1-based in SFbox) is ordered with the LAST gradient
 * fastest: 2D z = x*MY + y, 3D z = x*MY*MZ + y*MZ + z (Lat2DFlat.cpp:43-46,
 * Lat3D.cpp:59-68).  Iteration variables use SFbox's packing: for every site
 * that carries iteration variables, in site order, one value per class of
 * liquid segments with identical interaction parameters
 * (SF_Solve.cpp:53-86, 129-163, 794-812).
 *
 * Reference interfaces replaced (file:line in SFbox):
 *   Lat1stO  PropagateG/ConnectG/CorrectDoubleCountG/ComputeLnGN/NormPhi*  Lat1stO.h:7-50
 *   Lat2ndO  PropagateF/PropagateB/ConnectG(PHI)                            Lat2ndO.h:7-66
 *   SF_Molecule::ComputePhi (Matrix1 / CudaMatrix1)                         SF_Molecule.h:16
 *   SF_Solve::residuals / UpdateSWF / GetResiduals                          SF_Solve.cpp:647,794,527
 *   SFNewton::iterate (Pure_DIIS, LBFGS, TN)                                sfnewton.cpp:566,844
 *   Cuda_tools.h free functions (Forward/Backward/Composition/...)          Cuda_tools.h:4-27
 */
#ifndef SFGPU_H
#define SFGPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define SFGPU_OK               0
#define SFGPU_ERR_INVALID      1   /* bad argument or unsupported combination */
#define SFGPU_ERR_NOMEM        2   /* device or host allocation failed */
#define SFGPU_ERR_CUDA         3   /* a CUDA runtime call failed */
#define SFGPU_ERR_NONFINITE    4   /* NaN/Inf met in a residual or norm */
#define SFGPU_ERR_NOTCONVERGED 5   /* iteration limit reached */
#define SFGPU_ERR_TIMEOUT      6   /* a bounded device wait gave up */
#define SFGPU_ERR_UNSUPPORTED  7   /* feature outside the implemented path */
#define SFGPU_ERR_NODEVICE     8   /* no CUDA device present */

/* ---- enumerations (values equal SFbox's input-choice indices) ---------- */
/* lowerbound/upperbound choices, Lat1DFlat.cpp:26-31, Lat2DFlat.cpp:47-52.
 * The 3D lattice has no 'surface' choice (Lat3D.cpp:68-72); pass MIRROR1,
 * MIRROR2 or PERIODIC there. */
#define SFGPU_BOUND_SURFACE   1
#define SFGPU_BOUND_MIRROR1   2
#define SFGPU_BOUND_MIRROR2   3
#define SFGPU_BOUND_PERIODIC  4

/* geometry: SFbox's choices flat / cylindrical / spherical
 * (SF_System.cpp:378-441) minus one.  Cylindrical takes 1 gradient
 * (Lat1DCyl1stO / Lat1DCyl2ndO) or 2 (Lat2DCyl1stO / Lat2DCyl2ndO), spherical
 * 1 (Lat1DSphere1stO / Lat1DSphere2ndO); the radial coordinate is the first
 * gradient. */
#define SFGPU_GEOM_FLAT        0
#define SFGPU_GEOM_CYLINDRICAL 1
#define SFGPU_GEOM_SPHERICAL   2

/* 3D lattice types, lat : latticetype (Lat3D.cpp:212-259; SF_System.cpp:478-486).
 * STANDARD: six neighbours, propagation and contact weights 1/6 (Lat3D1stO).
 * STENCILS: standard propagation; contacts over the 27-site cube with
 *   lambda_3d[0..3] for the centre, the 6 faces, 12 edges and 8 corners
 *   (Lat3D::Sides, Lat3D.cpp:1725-1785).
 * FCC: first order, 12 neighbours (+-x+-y, +-y+-z, +-x+-z) with weight 1/12
 *   (Lat3DFCC1stO.cpp:56-100); contacts over the 27-site cube, 1/27 each.
 * HEX: first order, 12 neighbours (+-x, +-y, +-z, +-(x-y), +-(x-z), +-(y-z))
 *   with weight 1/12 (Lat3DHEX1stO.cpp:56-100); contacts over the same 12
 *   neighbours, 1/12 each (Lat3D.cpp:1733-1752).
 * Second-order 3D lattices propagate as STANDARD whatever the type
 * (SF_System::NewLat2ndO, SF_System.cpp:378-431) and take the type's
 * contacts. */
#define SFGPU_LATTICE_STANDARD 0
#define SFGPU_LATTICE_STENCILS 1
#define SFGPU_LATTICE_FCC      2
#define SFGPU_LATTICE_HEX      3

/* segment freedom, SF_Segment.cpp:61-65 ('grafted' is not on this path) */
#define SFGPU_SEG_FREE    0
#define SFGPU_SEG_FROZEN  1
#define SFGPU_SEG_PINNED  2

/* molecule freedom, SF_Molecule.cpp:47-54 (free, restricted, solvent) */
#define SFGPU_MOL_FREE       0
#define SFGPU_MOL_RESTRICTED 1
#define SFGPU_MOL_SOLVENT    2
#define SFGPU_MOL_NEUTRALIZER 3   /* mol : freedom : neutralizer (SF_Molecule.cpp:51,
                                     :110-126): its bulk fraction makes the bulk
                                     electroneutral (SF_MolList1stO.cpp:250-266) */

/* solver methods */
#define SFGPU_METHOD_DIIS      1   /* SFNewton::PlainLBFGSDIIS, sfnewton.cpp:566-664 */
#define SFGPU_METHOD_ANDERSON  2   /* DIIS on residual history (project addition) */
#define SFGPU_METHOD_NK        3   /* Newton-Krylov with exact tangent J*v */

/* ---- system description ------------------------------------------------ */
typedef struct {
    int    gradients;          /* 1, 2 or 3 */
    int    geometry;           /* SFGPU_GEOM_* */
    int    order;              /* 1 = first-order chains, 2 = semiflexible (every
                                  geometry; 1D/2D lump the homogeneous directions) */
    int    n_layers[3];        /* interior layers per gradient (unused entries 0) */
    int    bound_lo[3];        /* SFGPU_BOUND_* per gradient */
    int    bound_hi[3];
    double lambda;             /* a-priori step probability l1 (1D/2D); 3D uses 1/6 */
    double lambda_chi;         /* l1 used in contact averages; < 0 means lambda */
    double layer_adjustment;   /* 1D only (Lat1DFlat.cpp:139, Lat1DCylinder.cpp:43); 1 = none */
    double dimensions;         /* curved: spatial dimensions D (default 3) */
    double offset_first_layer; /* curved: offset_first_layer(_x) (default 0) */
    const double *stiff_range; /* 3D second order: M values, nonzero inside 'lat : stiff_range'
                                  (Lat3D.cpp:265-268), or NULL.  Copolymers then
                                  take SF_Copol2ndO_stiff_range's steps: persistence
                                  S inside the range and 0.2 outside (Lat3D2ndO.cpp:
                                  155-247, 680-764), isotropic 1/6 steps at the
                                  chain's last forward and first backward step
                                  (:250-344, :765-850); homopolymers are refused */
    int    lattice_type;       /* SFGPU_LATTICE_* (3 gradients; 0 otherwise) */
    double lambda_3d[4];       /* SFGPU_LATTICE_STENCILS: lambda0..lambda3, each in
                                  [0, 0.5], l0 + 6 l1 + 12 l2 + 8 l3 = 1 within
                                  DBL_EPSILON; lambda3 is then recomputed from
                                  the other three (Lat3D.cpp:246-259) */
    double bondlength;         /* lat : bondlength in m (Lat1DFlat.cpp:123-137); the
                                  Poisson equation of charged systems uses the site
                                  distance bondlength / sqrt(2 dimensions lambda) on
                                  the 1D and 2D lattices (Lat1DFlat.cpp:129,
                                  Lat2DFlat.cpp:209), the bondlength in 3D
                                  (Lat3D.cpp:263); 0 = SFbox's default 3e-10 */
} sfgpu_lattice_desc;

typedef struct {
    int           freedom;     /* SFGPU_SEG_* */
    const double *range;       /* host array of M range values for frozen and
                                  pinned segments (1 inside the range), else NULL */
    /* charges (mon : X : valence / epsilon, SF_Segment.cpp:170-217): the
     * valence in elementary charges and the relative dielectric constant
     * (0 = SFbox's default 80).  Any nonzero valence makes the system
     * charged: the electrostatic potential psi joins the iteration
     * variables (SF_Solve.cpp:164-177) -- on every lattice (1D flat,
     * cylinder, sphere; 2D flat, cylinder; 3D, where no frozen segment may
     * lie on a boundary layer), first or second order, with or without
     * overflow protection. */
    double        valence;
    double        epsilon;
} sfgpu_segment_desc;

typedef struct {
    int        n_blocks;       /* composition (A)n1(B)n2... as blocks */
    const int *block_segment;  /* segment index of each block */
    const int *block_length;   /* length of each block */
    int        freedom;        /* SFGPU_MOL_* */
    double     phibulk;        /* free molecules */
    double     theta;          /* restricted molecules */
    /* symmetric dendrimer, @dend(G, T1, f1, ..., TG, fG) (SF_MolStructure.cpp:116-140,
     * :348-359; SF_Dend1stO): n_generations = G > 0 splits the blocks above into
     * generations of generation_blocks[i] consecutive blocks (Ti, first order
     * lattices), each repeated generation_repeat[i] = fi times around its first
     * segment; 0 for a linear chain */
    int        n_generations;
    const int *generation_blocks;
    const int *generation_repeat;
    /* mol : force (SF_Molecule.cpp:41-43): the constant-force ensemble of
     * first-order copolymers, forward steps biased by +force along x (1D),
     * y (2D cylinder) or z (3D), backward steps by -force (Lat1DFlat1stO.cpp:
     * 116-130, Lat1DCyl1stO.cpp:112-133, Lat2DCyl1stO.cpp:100-126,
     * Lat3D1stO.cpp:94-130); 0 for none.  Homopolymers, dendrimers, the 2D
     * flat lattice and overflow protection refuse it as SFbox does. */
    double     force;
    /* branched first-order molecules: compositions with square brackets
     * (SF_Branched1stO, parsed by SF_ParserBranched.cpp:3-255) and combs
     * @dend(n. main1, spacer, side, main2) (SF_Comb1stO).  The bond tree of
     * the chain's N segments, numbered in the order of the blocks above:
     * bond_parent[s] (s = 1 .. N-1) is the segment that segment s is bonded
     * to on its way to segment 0, bond_parent[s] < s, bond_parent[0] = -1.
     * NULL for linear chains.  Not with dendrimer generations, the force
     * ensemble, second-order lattices or overflow protection. */
    const int *bond_parent;
    /* homopolymer ring (mol : ring : true, SF_MolList1stO.cpp:28-38): the
     * return-probability profile of SF_HomoRing1stO::Matrix1
     * (SF_HomoRing1stO.cpp:110-160) -- free rings of even length on a 1D
     * flat lattice; 0 for none */
    int        ring;
} sfgpu_molecule_desc;

typedef struct {
    sfgpu_lattice_desc         lattice;
    int                        n_segments;
    const sfgpu_segment_desc  *segments;
    const double              *chi;   /* n_segments*n_segments, row-major, symmetric */
    const double              *pf;    /* n_segments*n_segments persistence factors
                                         S for 2nd order (NULL: 0.2 everywhere,
                                         SF_Copol2ndO.cpp:234-247) */
    int                        n_molecules;
    const sfgpu_molecule_desc *molecules;
    int                        overflow_protection;
                               /* sys : overflow_protection (SF_System.cpp:67):
                                  chain statistics in natural logarithms on the
                                  first-order 1D and 2D lattices (Lat1DFlat1stOS,
                                  Lat1DCyl1stOS, Lat1DSphere1stOS, Lat2DFlat1stOS,
                                  Lat2DCyl1stOS); SFGPU_ERR_UNSUPPORTED on 3D and
                                  second-order lattices, where SFbox stops with an
                                  error (SF_System.cpp:395, :478-481).  The lattice-
                                  level propagate and lnGN calls then take and
                                  return logarithms; batches and derivatives
                                  return SFGPU_ERR_UNSUPPORTED. */
    double                     temperature;
                               /* sys : temperature in K (SF_System.cpp:68-69) for
                                  the electrostatic terms; 0 = 298.15 */
} sfgpu_system_desc;

typedef struct sfgpu_system sfgpu_system;   /* opaque handle, owns device buffers */

/* ---- library ------------------------------------------------------------ */
/* Message of the last failed call on this host thread.  SFbox prints GPU
 * errors and continues (Cuda_tools.cu:174-175); here every call returns a
 * status and the text is kept for the caller. */
const char *sfgpu_last_error(void);
/* Number of CUDA devices (SFGPU_ERR_NODEVICE when none).
 * Replaces GPU_present(), Cuda_tools.h:4. */
int sfgpu_device_count(int *count);

/* ---- system lifetime ---------------------------------------------------- */
/* Build the lattice, segment/state tables, molecule chains and device
 * buffers of one system on the current device.  Takes the place of the
 * construction in SF_System::SF_System (SF_System.cpp:13-100) for the hot
 * path and of the per-call cudaMalloc of SF_Homopol1stO::CudaMatrix1
 * (SF_Homopol1stO.cpp:639-643): buffers are allocated once here. */
int sfgpu_system_create(const sfgpu_system_desc *desc, sfgpu_system **out);
/* The same with checkpointed chain storage for residual evaluations: the
 * forward sweep of a copolymer or second-order chain keeps every stride-th
 * propagator slice (Gf at positions 0, k, 2k, ...) and one segment of k
 * slices; the backward sweep recomputes each earlier segment from its
 * checkpoint with the same kernels before composing it.  Memory per chain
 * (ceil(N/k) + k) K M doubles instead of N K M (a 96^3 second-order brush of
 * N = 200 with k = 14: 1.3 GB instead of 9 GB), at the cost of about one
 * extra forward sweep; residuals and profiles are bit-identical to full
 * storage.  This is the memory-saving scheme SFbox selects with
 * mol : X : save_memory (SF_Homopol1stO::Matrix1Long,
 * SF_Homopol1stO.cpp:732-843), with the stride given here.  stride = 0 (or
 * >= N) keeps every slice; overflow-protected systems keep every slice. */
int sfgpu_system_create_checkpointed(const sfgpu_system_desc *desc, int stride, sfgpu_system **out);
int sfgpu_system_destroy(sfgpu_system *sys);
/* M (sites incl. boundaries), number of iteration variables, classes and
 * sites carrying iteration variables (SF_Solve.cpp:129-163). */
int sfgpu_system_info(sfgpu_system *sys, int *M, int *nvar, int *nclass, int *nsites);
/* CUDA stream (cudaStream_t) all work of this system is queued on. */
int sfgpu_system_stream(sfgpu_system *sys, void **stream);
/* Queue all further work of this system on the caller's stream (for example
 * torch.cuda.current_stream().cuda_stream); the caller keeps it alive. */
int sfgpu_system_set_stream(sfgpu_system *sys, void *stream);
int sfgpu_synchronize(sfgpu_system *sys);

/* ---- SF_Solve-level ----------------------------------------------------- */
/* f = residuals(x) on device pointers, asynchronous on the system stream:
 * UpdateSWF + MolQ->ComputePhi + GetResiduals, SF_Solve::residuals
 * (SF_Solve.cpp:647-651). */
int sfgpu_residual(sfgpu_system *sys, const double *x_dev, double *f_dev);
/* same on host arrays, copies included, synchronous */
int sfgpu_residual_host(sfgpu_system *sys, const double *x, double *f);
/* Results of the last residual evaluation (host copies, synchronous):
 * state profile phi (SF_State::GetPhi, SF_State.cpp:302), the profile of one
 * segment type inside one molecule (SF_MolSegment::GetPhi), the segment
 * weighting factor G (SF_MolSegment::GetSWF) and the molecule scalars lnGN,
 * phibulk and ln C (SF_Molecule::GetLnGN/GetPhiBulk/GetLnNormFree). */
int sfgpu_get_phi(sfgpu_system *sys, int segment, double *phi);
int sfgpu_get_mol_phi(sfgpu_system *sys, int molecule, int segment, double *phi);
int sfgpu_get_swf(sfgpu_system *sys, int segment, double *g);
int sfgpu_get_mol_scalars(sfgpu_system *sys, int molecule, double *lngn, double *phibulk, double *lnc);
/* Bond-orientation profiles of second-order lattices: the orientation-
 * resolved composition of Lat2ndO::ConnectG(..., PHI) (Lat2ndO.h:7-66;
 * Lat3D2ndO.cpp:905-918, Lat2D2ndO.cpp:285-304, Lat1D2ndO.cpp:215-227),
 * divided by G and normalised like phi (CorrectDoubleCountG / NormPhi* with
 * PHI, Lat3D2ndO.cpp:986-993, :1031-1046).  Enabling makes every following
 * evaluation also fill, per molecule and segment type, mphi = 3 profiles
 * (2 on Lat1D2ndO) at 2K*8 extra bytes read per site and chain position.
 * sfgpu_get_bond_orientation copies to host (M doubles) the molecule's
 * profile of axis 0 = x_dir, 1 = y_dir (yz_dir in 1D), 2 = z_dir, summed
 * over its segment types as SF_Copol2ndO::GetBondOrientation does
 * (SF_Copol2ndO.cpp:108-116).  Boundary entries are 0.  First-order
 * lattices: SFGPU_ERR_UNSUPPORTED. */
int sfgpu_system_set_bond_orientation(sfgpu_system *sys, int enable);
int sfgpu_get_bond_orientation(sfgpu_system *sys, int molecule, int axis, double *host_out);
/* Helmholtz free energy of the last evaluation,
 * SF_MolList1stO::GetFreeEnergy (SF_MolList1stO.cpp:606-635). */
int sfgpu_free_energy(sfgpu_system *sys, double *F);
/* Thermodynamics of the last evaluation: F (as above) and the grand
 * potential Omega = sum_z L(z) omega(z) (SF_MolList1stO::GetGrandPotential,
 * SF_MolList1stO.cpp:636-646, with GetGrandPotentialProfile :1001-1101; the
 * same formula in SF_MolList2ndO), and, for non-NULL host arrays of M
 * doubles, the free-energy density (GetFreeEnergyProfile, :815-826) and
 * omega(z), both after SubtractBoundaries (boundary layers 0 except
 * surfaces, mirror2 layers halved).  At a converged solution Omega equals
 * F - sum_i n_i mu_i (SFbox's "grand potential2", :648-661). */
int sfgpu_thermo(sfgpu_system *sys, double *F, double *Omega, double *fe_profile, double *omega_profile);
/* Host copies (M doubles each, either may be NULL) of the site weights of
 * lnGN sums (interior sites, mirror2 halves, lattice sites L(z) on curved
 * lattices) and of sums over the lattice such as F or theta
 * (SubtractBoundaries then MultiplyWithLatticeSites, Lat1DFlat.cpp:266-269,
 * 410-415; Lat1DCylinder.cpp:126-141). */
int sfgpu_lattice_weights(sfgpu_system *sys, double *w_lngn, double *w_sum);

/* ---- Lattice-level (device vectors of M or 6*M doubles) ----------------- */
/* gout = one propagator step of gin with segment weights g.  First order:
 * Lat1stO::PropagateG(Gi, G, Gout) (Lat1stO.h:22; Lat1DFlat1stO.cpp:101-113,
 * Lat2DCyl1stO.cpp:72-97, Lat3D1stO.cpp:51-90).  Second order:
 * Lat2ndO::PropagateF (backward = 0) / PropagateB (backward = 1) with
 * persistence factor S (Lat3D2ndO.cpp:65-152, :597-678; lumped 1D/2D:
 * Lat1D2ndO.cpp:33-147, Lat2D2ndO.cpp:32-230).  Boundary entries of gout hold
 * SetBoundaries copies, except on the lumped 1D/2D lattices, whose step
 * writes the interior entries only. */
int sfgpu_lat_propagate(sfgpu_system *sys, const double *gin, const double *g, double *gout,
                        double S, int backward);
/* Lattice::SetBoundaries on 1 or 6 components (Lat3D.cpp:1510-1562; the six
 * components swap direction at mirrors, Lat3D2ndO.cpp:84-89) */
int sfgpu_lat_set_boundaries(sfgpu_system *sys, double *p, int components);
/* rho(z) = contact average of phi: Lattice::SideFraction for 1 and 2
 * gradients (Lat1DFlat.cpp:511-524, Lat2DCylinder.cpp:205-320), Sides for 3
 * (Lat3D.cpp:1729-1785) */
int sfgpu_lat_side_fraction(sfgpu_system *sys, const double *phi, double *rho);
/* Lat1stO::ComputeLnGN (Lat1DFlat1stO.cpp:301-316, Lat3D1stO.cpp:344-370,
 * Lat3D2ndO.cpp:995-1025) of an end-point distribution */
int sfgpu_lat_lngn(sfgpu_system *sys, const double *g, int components, double *lngn);

/* Composition and normalisation on device vectors, for callers that keep
 * their own chain loop over sfgpu_lat_propagate (the Matrix1 drivers,
 * SF_Homopol1stO.cpp:553-622) or port Cuda_tools.h's Composition /
 * CorrectDoubleCounting / NormPhi (Cuda_tools.cu:208-236).  All are
 * asynchronous on the system's stream; K = components is 1 for first order
 * or the lattice's direction count (6 in 3D, 3 or 5 on the lumped 1D/2D
 * lattices, whose lateral groups count with their multiplicity 4 or 2).
 * The log-space lattices (overflow_protection) return SFGPU_ERR_UNSUPPORTED.
 *
 * phi(z) += sum_k gb_k(z) gf_k(z): Lat1stO::ConnectG(GiA, GiB, out)
 * (Lat1stO.h:36; Lat1DFlat1stO.cpp:268-274, Lat3D2ndO.cpp:895-903) */
int sfgpu_lat_connect(sfgpu_system *sys, const double *gb, const double *gf, double *phi, int components);
/* phi(z) /= g(z) where g(z) > 0, else 0: CorrectDoubleCountG (Lat1stO.h:40;
 * Lat1DFlat1stO.cpp:294-300, tools.cpp:86-90) */
int sfgpu_lat_correct_double_count(sfgpu_system *sys, double *phi, const double *g);
/* phi *= C: NormPhiFree (Lat1stO.h:46; Lat1DFlat1stO.cpp:317-322) */
int sfgpu_lat_norm_phi_free(sfgpu_system *sys, double *phi, double C);
/* phi *= C / exp(lnGN(gb)) on first-order lattices, C / (6 exp(lnGN(gb))) on
 * second-order ones, lnGN as sfgpu_lat_lngn: NormPhiRestr (Lat1stO.h:48;
 * Lat1DFlat1stO.cpp:323-331, Lat3D2ndO.cpp:1036-1039).  C is theta/N. */
int sfgpu_lat_norm_phi_restr(sfgpu_system *sys, double *phi, const double *gb, int components, double C);

/* ---- derivatives ------------------------------------------------------- */
/* f = residuals(x) and jv = J(x) v with J the exact Jacobian df/dx, by a
 * forward-mode (tangent) sweep through UpdateSWF, both propagator sweeps, the
 * composition, the lnGN/phibulk normalisations and GetResiduals.  SFbox forms
 * J*v only by finite differences of residuals (SFNewton::Hp,
 * sfnewton.cpp:1662-1688).  f equals sfgpu_residual's bit for bit.  Device
 * pointers, asynchronous; the _host variant copies and synchronises.  The
 * first call allocates the tangent buffers (about the size of the
 * propagator storage). */
int sfgpu_jvp(sfgpu_system *sys, const double *x_dev, const double *v_dev, double *f_dev, double *jv_dev);
int sfgpu_jvp_host(sfgpu_system *sys, const double *x, const double *v, double *f, double *jv);
/* Newton-Krylov iteration on residuals(x) = 0: GMRES(krylov) with exact J*v
 * (Eisenstat-Walker forcing, backtracking line search on |f|), the
 * replacement of SFNewton's numerical-Hessian and truncated-Newton methods
 * (sfnewton.cpp:1627-1688, 1809-1944).  x is a host array (in: guess, out:
 * last iterate; the system's profiles are those of the returned x). */
int sfgpu_solve_nk(sfgpu_system *sys, double *x, double tol, int maxit, int krylov,
                   int *iterations, int *jvps, double *final_error);

/* f = residuals(x) and xbar = J(x)^T w by a reverse (adjoint) sweep:
 * cotangents flow from GetResiduals through the contact averages, the
 * normalisations (lnGN, restricted and solvent phibulk), CorrectDoubleCountG
 * and the two propagator recursions (adjoint propagators run against their
 * primal direction over stored Gf and Gb) to UpdateSWF.  First- and
 * second-order lattices (second order: the transposed six-direction step,
 * with the component swaps at mirrors, scattered by FP64 atomics).  The
 * first call allocates 2*N*K*M doubles for the stored propagators (K = 1 or
 * 6; see sfgpu_system_set_checkpoint for less).  SFbox has no counterpart:
 * its L-BFGS and truncated Newton use finite differences. */
int sfgpu_vjp(sfgpu_system *sys, const double *x_dev, const double *w_dev, double *f_dev, double *xbar_dev);
int sfgpu_vjp_host(sfgpu_system *sys, const double *x, const double *w, double *f, double *xbar);
/* Memory of the reverse sweep: stride 0 (default) stores every forward and
 * backward slice of the longest chain (2 N M doubles); stride k > 0 stores
 * the slices at every k-th position (checkpoints) and recomputes the k
 * slices of one segment at a time when the sweep reaches it, in
 * (2 ceil(N/k) + 2k + 1) M doubles -- k near sqrt(N) is smallest -- for
 * about 1.75x the propagation work; stride -1 picks ceil(sqrt(N)) of the
 * longest chain, the stride of least memory.  Results are identical for
 * every stride (the recomputed slices are computed by the same kernels).
 * The storage is reallocated at the next sfgpu_vjp. */
int sfgpu_system_set_checkpoint(sfgpu_system *sys, int stride);
/* The checkpoint stride by measurement: full storage and strides around
 * sqrt(N) of the longest chain (k/2, k, 2k, N/4), each whose storage fits
 * max_bytes (<= 0: no limit), timed on `reps` reverse sweeps at the host
 * vector x; the fastest is set and returned with its time per sweep. */
int sfgpu_system_autotune_checkpoint(sfgpu_system *sys, const double *x, int reps, double max_bytes, int *stride,
                                     double *best_ms);
/* Sensitivity of the residual to the Flory-Huggins parameters at fixed x
 * (first and second order): dchi[a * nseg + i] = d (w . f(x)) / d chi(a, i)
 * over the entries the residual reads (a = the representative state of a
 * class, SF_Solve.cpp:563-564), 0 elsewhere.  x, w: nvar host values; dchi:
 * nseg * nseg host values.  For a symmetric change of chi(a,b) = chi(b,a)
 * add dchi[a][b] + dchi[b][a].  With the adjoint solution w of J^T w = dL/dx
 * at a converged x, dL/dchi = -(that sum).  No counterpart in SFbox. */
int sfgpu_vjp_chi(sfgpu_system *sys, const double *x, const double *w, double *dchi);
/* Free energy F(x) (as sfgpu_free_energy after a residual at x,
 * SF_MolList1stO::GetFreeEnergy, SF_MolList1stO.cpp:606-635) and its exact
 * gradient dF/dx by the reverse sweep (first and second order).  x, xbar:
 * nvar host values; F: one host value.  No counterpart in SFbox. */
int sfgpu_free_energy_grad(sfgpu_system *sys, const double *x, double *F, double *xbar);
/* Sensitivity of the converged profiles to chi.  x: a solution of
 * residuals(x) = 0 (host, nvar); omega: nseg * M host weights defining
 * L = sum_i sum_z omega[i * M + z] phi_i(z).  Returns dchi[a * nseg + i] =
 * dL / d chi(a, i) through the solution's dependence on chi (implicit
 * function theorem: J^T lam = dL/dx solved by restarted GMRES(krylov) to
 * rtol with the reverse sweep as operator, then dL/dchi = -lam^T df/dchi);
 * for a symmetric change of chi(a,b) = chi(b,a) add both entries.  relres:
 * the relative residual reached (may be NULL).  No counterpart in SFbox. */
int sfgpu_phi_sensitivity_chi(sfgpu_system *sys, const double *x, const double *omega, double *dchi, double rtol,
                              int krylov, int maxcycles, double *relres);
/* L-BFGS (Nocedal 1980 two-loop recursion, m pairs, Armijo backtracking) on
 * |f(x)|^2 / 2 with the exact gradient J^T f from the adjoint sweep; SFbox's
 * LBFGS method (SFNewton::L_BFGS, sfnewton.cpp:1770-1807) iterates on the
 * residual itself.  x is a host array (in: guess, out: last iterate). */
int sfgpu_solve_lbfgs(sfgpu_system *sys, double *x, double tol, int maxit, int m,
                      int *iterations, int *evaluations, double *final_error);

/* ---- measurement ------------------------------------------------------- */
/* Average device time of one forward propagator step and of one backward
 * step with fused composition on this system's buffers (reps launches each,
 * CUDA events on the system stream), with their algorithmic bytes per launch
 * (8 bytes per value read or written once).  Propagator contents are
 * overwritten; call before the next residual. */
int sfgpu_profile_propagator(sfgpu_system *sys, int reps, double *ms_fwd, double *ms_bwd,
                             double *bytes_fwd, double *bytes_bwd);

/* Tile shape of the 3D first-order step (x planes walked per thread block):
 * set it, or let the library time the candidates 2..32 on this system's own
 * buffers and keep the fastest (reps forward + backward steps each; the
 * propagator contents are overwritten).  Other lattices ignore it. */
int sfgpu_system_set_tile(sfgpu_system *sys, int xc);
/* 1: the 3D first-order step runs software-pipelined (plane x+1's loads in
 * flight while plane x is computed, double-buffered tile); 0: the plain
 * x-marching form; 2: pipelined, the forward (composition-free) steps with
 * two y rows of columns per thread.  Results are bit-identical.  By default
 * the composing backward steps run pipelined (x depth 8) and the forward
 * steps plain (depth 4); the autotuner times the forms and depths for each
 * kind of step.  sfgpu_system_set_tile and this call set both kinds. */
int sfgpu_system_set_tile_pipelined(sfgpu_system *sys, int enable);
int sfgpu_system_autotune(sfgpu_system *sys, int reps, int *chosen_xc, double *best_ms);

/* ---- iterations ------------------------------------------------------- */
/* Many systems solved at once, each by sfgpu_solve_diis on its own stream
 * from its own host thread (threads <= 0: one per system): the device
 * interleaves the systems' kernels and every system's per-iteration host
 * round trip hides behind the others' work.  The batched form for instances
 * that fill the GPU one propagator step at a time (3D, second order), where
 * the persistent one-block-per-instance solver (sfgpu_batch_*) would leave
 * most SMs idle; a parameter sweep of such systems (Vary.cpp:127).  x[i]
 * (host) is system i's start and receives its result; status[i] as
 * sfgpu_solve_diis returns it.  Returns the first status other than OK,
 * NOTCONVERGED or NONFINITE, else SFGPU_OK. */
int sfgpu_solve_diis_many(int n, sfgpu_system *const *systems, double *const *x, double tol, int maxit, int m,
                          double eta, int threads, int *status, int *iterations, double *errors);

/* SFbox's Newton iteration (SFNewton::iterate, sfnewton.cpp:844-1143, with
 * Scheutjens' trust-region step search, :1946-2022) over this library's
 * residual: the "plain Newton form".  The Hessian is dense, single
 * precision and held as an LDU factorisation (sfnewton.h:147,
 * newttool.cpp); pseudohessian = 1 (SFbox's default method 'pseudohessian')
 * starts from diag(1 + |g|) and updates it BFGS-style each iteration
 * (:1433-1521), pseudohessian = 0 (method 'hessian') rebuilds it from nvar
 * finite-difference residuals (numhessian, :1627-1652).  SF_Solve's reset
 * heuristics are kept (walking backwards, too many small steps,
 * SF_Solve.cpp:659-727).  Residuals run on the device, the iteration on the
 * host; nvar^2 floats of host memory, refused beyond nvar = 8192.  Stops as
 * SFbox does: accuracy = sqrt(|p| |g| / (1 + |x|)) <= tolerance and
 * |g| <= 10 tolerance (sfnewton.cpp:925, :2040-2042).  x (host) is the start
 * and receives the result; returns SFGPU_ERR_NOTCONVERGED at the iteration
 * limit. */
typedef struct {
    double tolerance;                       /* newton : tolerance (1e-7) */
    int    iterationlimit;                  /* newton : iterationlimit (5000) */
    int    pseudohessian;                   /* 1 pseudohessian (default), 0 hessian */
    double deltamax;                        /* newton : deltamax (0.5) */
    double deltamin;                        /* newton : deltamin (0) */
    int    linesearchlimit;                 /* newton : linesearchlimit (20) */
    double small_alpha;                     /* newton : small_alpha (1e-5) */
    int    max_n_small_alpha;               /* newton : max_n_small_alpha (50) */
    double reset_hessian_criterion;         /* newton : reset_hessian_criterion (1e3) */
    double max_accuracy_for_hessian_scaling;/* (0.1) */
    int    ignore_newton_direction;         /* (0) */
} sfgpu_newton_settings;
/* SFbox's defaults for an input file with a 'newton' block (SF_Solve.cpp:1779-2182) */
int sfgpu_newton_default_settings(sfgpu_newton_settings *settings);
int sfgpu_solve_newton(sfgpu_system *sys, double *x, const sfgpu_newton_settings *settings,
                       int *iterations, int *function_calls, double *accuracy);

/* Pure_DIIS: SFNewton::PlainLBFGSDIIS (sfnewton.cpp:566-664) on the device,
 * coefficients as SFNewton::Ax (sfnewton.cpp:531-557).  x is a host array,
 * in: initial guess, out: last iterate.  Returns SFGPU_ERR_NOTCONVERGED when
 * maxit is reached, SFGPU_ERR_NONFINITE on a NaN/Inf residual. */
int sfgpu_solve_diis(sfgpu_system *sys, double *x, double tol, int maxit, int m, double eta,
                     int *iterations, double *final_error);

/* ---- batched instances (parameter sweeps) --------------------------------- */
/* Many independent first-order systems -- the calculations of a 'var :'
 * sweep, which SFbox runs one after another (Vary::NextCalculation,
 * Vary.cpp:127; SF_Box.cpp:145-177) -- solved together.  m is the DIIS
 * memory (1..16).  3D instances must have the standard lattice type
 * (SFGPU_ERR_UNSUPPORTED otherwise: solve those one by one). */
typedef struct sfgpu_batch sfgpu_batch;
int sfgpu_batch_create(int n, const sfgpu_system_desc *descs, int m, sfgpu_batch **out);
int sfgpu_batch_destroy(sfgpu_batch *batch);
/* number of instances, total iteration variables and the start of every
 * instance in the concatenated x vector */
int sfgpu_batch_info(sfgpu_batch *batch, int *n, long long *total_nvar, long long *offsets);
int sfgpu_batch_set_stream(sfgpu_batch *batch, void *stream);
/* launch shape of the persistent kernel: threads per block (32..1024, a
 * multiple of 32; default 1024, 512, 384 or 256 by lattice size) and whether G of
 * the running segment (and on 1D symmetric homopolymers the running slices,
 * phi and a ring of stored slices) is staged in shared memory (default 1).
 * Results do not depend on it; the autotuner of field_b200.batch times the
 * candidates. */
int sfgpu_batch_set_launch(sfgpu_batch *batch, int threads, int stage);
/* Pure_DIIS (SFNewton::PlainLBFGSDIIS, sfnewton.cpp:566-664) on every
 * instance in one persistent kernel launch: thread blocks take instances
 * from a work queue and iterate them to |f| <= tol on the device.  x_in is
 * the concatenated host vector of initial guesses, x_out (may be NULL, may
 * equal x_in) receives the last iterates; status[i] is SFGPU_OK,
 * SFGPU_ERR_NOTCONVERGED or SFGPU_ERR_NONFINITE. */
int sfgpu_batch_solve(sfgpu_batch *batch, const double *x_in, double *x_out, double tol, int maxit,
                      double eta, int *status, int *iterations, double *errors);
/* the same in three parts: load guesses (host -> device), launch the solve
 * on the device-resident iterate (asynchronous), read results back (x may
 * be NULL to leave the iterates on the device) */
int sfgpu_batch_load(sfgpu_batch *batch, const double *x);
int sfgpu_batch_solve_resident(sfgpu_batch *batch, double tol, int maxit, double eta);
int sfgpu_batch_results(sfgpu_batch *batch, double *x, int *status, int *iterations, double *errors);
/* device time of the last solve launch (CUDA events around the kernel) */
int sfgpu_batch_kernel_ms(sfgpu_batch *batch, double *ms);
/* state profile of one instance after the solve (its last evaluation) */
int sfgpu_batch_get_phi(sfgpu_batch *batch, int instance, int segment, double *phi);

/* ---- allocation-free chain propagation -------------------------------- */
/* No counterpart in SFbox: an addition of this library.
 *
 * For callers that cannot allocate device memory -- code running inside
 * another application's memory pool, a process whose device memory is
 * reserved up front, or anything that must not change the device's
 * allocation state while it runs -- and so cannot create an sfgpu_system
 * (which allocates its buffers once at creation).  This call propagates one
 * first-order chain (N segments, segment index seg_of_s[s] per position, a
 * host array) on the lattice *lat with the caller's device arrays G[i] (M
 * segment weighting factors per segment type i, boundary layers set) and
 * writes, into the caller's device arrays phi[i], the unnormalised volume
 * fraction sum_s Gf(z,s) Gb(z,s) / G(z) of every segment type used, plus
 * lnGN into the caller's device double *lngn.  Multiply phi by phibulk/N
 * (free) or theta/(N exp(lnGN)) (restricted) to normalise.  G and phi are
 * host arrays of nseg device pointers.
 *
 * It calls no cudaMalloc, cudaFree or other allocating routine: all
 * intermediates live in one array inside the library of 2*1024*1024 doubles
 * (16 MiB), which every GPU that loads the library keeps until the process
 * exits.  The chain must satisfy 2*MX + 3*M + 1024 + N*M <= 2097152 (MX =
 * layers of the first gradient incl. boundaries); larger chains are
 * rejected with SFGPU_ERR_INVALID before any work is queued.  The first call
 * on a device looks up the array's device address (once per device, with
 * that device current); make that first call before any stream capture.
 * That address is kept for the life of the process: after a cudaDeviceReset
 * of the device, further calls on it are not supported.  The lattice tables
 * (8*(2*MX + M) bytes) are copied from host memory that the library keeps
 * until the process exits, one copy per distinct lattice.
 * All work is queued on `stream` (0 = legacy default stream).  Every call
 * uses the same array and overwrites it, and nothing in it has to start at
 * zero (phi is cleared by the call); two calls that overlap on the GPU, on
 * different streams or devices sharing a context, race on it. */
int sfgpu_chain_phi_noalloc(const sfgpu_lattice_desc *lat, int N, const int *seg_of_s, int nseg,
                            const double *const *G, double *const *phi, double *lngn, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* SFGPU_H */
