// sfgpu_newton.cu -- sfgpu_solve_newton: SFbox's Newton iteration
// (sfgpu_newton.h) over this library's device residual.  Every residual is
// sfgpu_residual_host (x to the device, one asynchronous residual evaluation,
// f back); the dense single-precision Hessian work stays on the host as in
// SFbox (sfnewton.h:147).
#include <cmath>
#include <cstring>

#include "sfgpu_newton.h"
#include "sfgpu_system.h"

extern "C" int sfgpu_newton_default_settings(sfgpu_newton_settings *st) {
    if (!st) return SFGPU_ERR_INVALID;
    std::memset(st, 0, sizeof *st);
    st->tolerance = 1e-7;                      // SF_Solve.cpp:1788
    st->iterationlimit = 5000;                 // :1787
    st->pseudohessian = 1;                     // method pseudohessian (default, :1867)
    st->deltamax = 0.5;                        // :1885
    st->deltamin = 0;                          // :1886
    st->linesearchlimit = 20;                  // sfnewton.cpp:31
    st->small_alpha = 1e-5;                    // SF_Solve.cpp:2168
    st->max_n_small_alpha = 50;                // :2169
    st->reset_hessian_criterion = 1e3;         // :2176
    st->max_accuracy_for_hessian_scaling = 0.1;  // :2181
    st->ignore_newton_direction = 0;           // :2182
    return SFGPU_OK;
}

extern "C" int sfgpu_solve_newton(sfgpu_system *sys, double *x, const sfgpu_newton_settings *settings,
                                  int *iterations, int *function_calls, double *accuracy) {
    if (!sys || !x || !settings) return SFGPU_ERR_INVALID;
    const sfgpu_newton_settings &s = *settings;
    if (!(s.tolerance > 0) || s.iterationlimit < 0 || !(s.deltamax > s.deltamin) || s.deltamin < 0 ||
        s.linesearchlimit < 1)
        return SFGPU_ERR_INVALID;
    int M = 0, nvar = 0, nclass = 0, nsites = 0;
    int rc = sfgpu_system_info(sys, &M, &nvar, &nclass, &nsites);
    if (rc) return rc;
    if (nvar < 1) return SFGPU_ERR_INVALID;
    if ((long long)nvar * nvar > 64LL * 1024 * 1024) {
        sfgpu_set_error(cudaSuccess, "sfgpu_solve_newton: a dense Hessian beyond 64 Mi entries (nvar > 8192)",
                        __FILE__, __LINE__);
        return SFGPU_ERR_UNSUPPORTED;
    }
    auto res = [sys](const double *xv, double *gv) { return sfgpu_residual_host(sys, xv, gv); };
    sfnewton::Newton<decltype(res)> nt{res};
    nt.n = nvar;
    nt.st = s;
    nt.pseudohessian = s.pseudohessian != 0;
    nt.x.assign(x, x + nvar);
    rc = nt.run();
    std::memcpy(x, nt.x.data(), sizeof(double) * nvar);
    if (iterations) *iterations = nt.iterations;
    if (function_calls) *function_calls = nt.functioncalls;
    if (accuracy) *accuracy = nt.accuracy;
    if (rc) return rc;
    if (!(nt.accuracy == fabs(nt.accuracy))) return SFGPU_ERR_NONFINITE;
    const double normg = sqrt(nt.minimum);
    if (s.tolerance < nt.accuracy || s.tolerance * 10 < normg) return SFGPU_ERR_NOTCONVERGED;
    return SFGPU_OK;
}
