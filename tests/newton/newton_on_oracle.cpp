// newton_on_oracle.cpp -- test harness: the library's Newton iteration
// (field_b200/csrc/sfgpu_newton.h, the code sfgpu_solve_newton runs) over the
// CPU oracle's residual, so that its trajectory can be checked against
// SFbox's own Newton (tests/golden/reference_cases.npz) without a GPU.
#include "../../field_b200/csrc/sfgpu_newton.h"
#include "../../oracle/sfbox_oracle.h"

extern "C" int newton_on_oracle(void *orc, int nvar, double *x, const sfgpu_newton_settings *st, int *iterations,
                                int *function_calls, double *accuracy) {
    orc_system *s = static_cast<orc_system *>(orc);
    auto res = [s](const double *xv, double *gv) { return orc_residual(s, xv, gv); };
    sfnewton::Newton<decltype(res)> nt{res};
    nt.n = nvar;
    nt.st = *st;
    nt.pseudohessian = st->pseudohessian != 0;
    nt.x.assign(x, x + nvar);
    int rc = nt.run();
    for (int i = 0; i < nvar; i++) x[i] = nt.x[i];
    *iterations = nt.iterations;
    *function_calls = nt.functioncalls;
    *accuracy = nt.accuracy;
    return rc;
}
