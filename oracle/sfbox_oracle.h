/*
 * sfbox_oracle.h -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * CPU restatement of the SFbox 2.1 SF-SCF hot path, used by tests/, the
 * smoke check and bench.py's CPU-baseline leg to check the CUDA library.
 * Pinned against SFbox itself: oracle/refbuild builds the reference's own
 * C++ sources (with stand-ins for its absent 'fenk' container library and
 * CLAPACK), and tests/golden/reference_cases.npz holds that build's residuals,
 * profiles, lnGN and free energies on one system per lattice family, which
 * this restatement meets to 1e-13 (tests/test_reference_parity.py); it is
 * further checked by known-answer tests derived from the equations.
 */
#ifndef SFBOX_ORACLE_H
#define SFBOX_ORACLE_H
#include "../include/sfgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_system orc_system;

int    orc_create(const sfgpu_system_desc *desc, orc_system **out);
void   orc_destroy(orc_system *s);
int    orc_num_sites(const orc_system *s);          /* M */
int    orc_num_itvar(const orc_system *s);          /* length of x */
int    orc_num_classes(const orc_system *s);
int    orc_itvar_sites(const orc_system *s, int *sites);  /* 0-based site list */
int    orc_class_of_segment(const orc_system *s, int seg); /* -1 for frozen */

/* full residual evaluation x -> f (SF_Solve::residuals, SF_Solve.cpp:647) */
int    orc_residual(orc_system *s, const double *x, double *f);
/* results of the last evaluation */
int    orc_get_phi(const orc_system *s, int seg, double *phi);         /* state phi, M */
int    orc_get_mol_phi(const orc_system *s, int mol, int seg, double *phi);
double orc_get_lngn(const orc_system *s, int mol);
int    orc_bond_orientation(const orc_system *s, int mol, int axis, double *out);  /* 2nd order, M */
int    orc_thermo(orc_system *s, double *F, double *Omega, double *fe, double *gp);  /* profiles M or NULL */
double orc_get_phibulk(const orc_system *s, int mol);
int    orc_get_swf(const orc_system *s, int seg, double *g);           /* segment G (masked) */
double orc_free_energy(orc_system *s);                                 /* SF_MolList1stO.cpp:606 */

/* one propagator step, Gout = G * stencil(Gin) with SFbox boundaries
   (1st order: M values; 2nd order: 6*M values, forward or backward) */
/* stiff_range (iso 0) or isotropic (iso 1) 3D second-order step, 6*M values */
int    orc_propagate_stiff(const orc_system *s, const double *gin, const double *g, double *gout, double S,
                           int backward, int iso);
/* ComputeLnGN of a propagator (on logarithms with overflow protection) */
int    orc_lat_lngn(const orc_system *s, const double *g, double *lngn);
int    orc_propagate(const orc_system *s, const double *gin, const double *g,
                     double *gout, double S, int backward);
/* contact average <phi>(z) of one profile (SideFraction / Sides) */
int    orc_side(const orc_system *s, const double *phi, double *rho);
/* lattice-site weights used by lnGN and the free energy (interior sites) */
int    orc_site_weights(const orc_system *s, double *w);
/* apply SetBoundaries to a profile in place */
int    orc_set_boundaries(const orc_system *s, double *p);

/* Pure_DIIS iteration (SFNewton::PlainLBFGSDIIS, sfnewton.cpp:566-664) */
int    orc_solve_diis(orc_system *s, double *x, double tol, int maxit, int m,
                      double eta, int *iterations, double *final_error);

#ifdef __cplusplus
}
#endif
#endif
