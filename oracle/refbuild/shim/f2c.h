/* f2c.h -- stand-in for the f2c/CLAPACK types SFbox includes
 * (sfnewton.cpp:3, MPS.cpp:3).  Test infrastructure for the oracle's build
 * of the reference sources; the LAPACK routines are served by the LAPACK
 * that ships with scipy (32-bit integers), see lapack_bridge.c. */
#ifndef F2C_SHIM_H
#define F2C_SHIM_H
typedef int integer;
typedef double doublereal;
typedef float real;
typedef int logical;
typedef int ftnlen;
#endif
