// sfgpu_newton.h -- SFbox's own Newton iteration (the default 'newton'
// method, SFNewton::iterate with Scheutjens' line search) over a residual
// callback.  Header only and free of CUDA: sfgpu_newton.cu runs it over the
// device residual.
//
// This is the plain Newton form SFbox runs when an input file names no
// method ("pseudohessian", SF_Solve.cpp:1867-1869, :1940-1964) or asks for
// "hessian" (:1920-1939): a dense Hessian held in single precision as an LDU
// factorisation, BFGS-style updates of that factorisation, the trust-region
// and step-length rules and SF_Solve's reset heuristics, all O(nvar^2) host
// work per iteration on systems small enough for a dense Hessian (C1:
// nvar = 200).
//
// Followed, by section:
//   iterate loop, Scheutjens branch     sfnewton.cpp:844-1143 (no DIIS)
//   direction (Newton branch)           sfnewton.cpp:1909-1932
//   newhessian / findhessian / numhessian sfnewton.cpp:1417-1521, :1627-1652
//   startderivatives                    sfnewton.cpp:1523-1530
//   zero / linesearch / linecriterion / stepchange / newtrustregion / residue
//                                       sfnewton.cpp:1946-2042
//   inneriteration (reset heuristics)   SF_Solve.cpp:659-760
//   LDU kernels multiply, updateneg, decompos, updatpos, gausa, gausb,
//   signdeterminant, norm2, innerproduct newttool.cpp:3-243
#ifndef SFGPU_NEWTON_H
#define SFGPU_NEWTON_H
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/sfgpu.h"

namespace sfnewton {

// ---- dense LDU tools on a float matrix h[i + n*j] ---------------------------
inline double inner(const double *x, const double *y, int n) {
    double s = 0;
    for (int i = 0; i < n; i++) s += x[i] * y[i];
    return s;
}

inline double norm2(const double *x, int n) {
    double s = 0;
    for (int i = 0; i < n; i++) s += pow(x[i], 2);
    return sqrt(s);
}

inline int sign_det(const float *h, int n) {
    int sign = 1;
    for (int i = 0; i < n; i++)
        if (h[i + i * n] < 0) sign = -sign;
    return sign;
}

// v = alpha * (L D U) w with the factors stored in h
inline void ldu_multiply(double *v, double alpha, const float *h, const double *w, int n) {
    std::vector<double> x(n);
    for (int i = 0; i < n; i++) {
        double sum = 0;
        for (int j = i + 1; j < n; j++) sum += w[j] * h[i + n * j];
        x[i] = (sum + w[i]) * h[i + n * i];
        sum = 0;
        for (int j = 0; j <= i - 1; j++) sum += x[j] * h[i + n * j];
        v[i] = alpha * (sum + x[i]);
    }
}

// rank-one downdate of the factorisation by alpha w w^T (alpha < 0)
inline void ldu_update_neg(float *l, double *w, int n, double alpha) {
    const double dmin = 1.0 / pow(2.0, 54);
    alpha = sqrt(-alpha);
    double t = 0;
    for (int i = 0; i < n; i++) {
        double sum = 0;
        for (int j = 0; j <= i - 1; j++) sum += l[i + n * j] * w[j];
        w[i] = alpha * w[i] - sum;
        t += (w[i] / l[i + n * i]) * w[i];
    }
    t = 1 - t;
    if (t < dmin) t = dmin;
    for (int i = n - 1; i >= 0; i--) {
        const double p = w[i], d = l[i + n * i];
        double b = d * t;
        t += (p / d) * p;
        l[i + n * i] = b / t;
        b = -p / b;
        for (int j = i + 1; j < n; j++) {
            const double lji = l[j + n * i];
            l[j + n * i] = lji + b * w[j];
            w[j] += p * lji;
        }
    }
}

// in-place LDU decomposition of h (Crout order, single precision)
inline void ldu_decompose(float *h, int nvar) {
    float *ha = h - 1;
    for (int i = 1; i <= nvar; i++) {
        float *hai = &ha[(i - 1) * nvar];
        float sum = 0;
        for (int j = 1; j <= i - 1; j++) {
            float *haj = &ha[(j - 1) * nvar];
            float c = haj[i];
            const float l = c / haj[j];
            haj[i] = l;
            c = hai[j];
            hai[j] = c / haj[j];
            sum += l * c;
        }
        hai[i] = hai[i] - sum;
        for (int j = i + 1; j <= nvar; j++) {
            float *haj = &ha[(j - 1) * nvar];
            float lsum = 0, usum = 0;
            for (int k = 1; k <= i - 1; k++) {
                lsum += ha[(k - 1) * nvar + j] * hai[k];
                usum += ha[(k - 1) * nvar + i] * haj[k];
            }
            hai[j] -= lsum;
            haj[i] -= usum;
        }
    }
}

// rank-one update of the factorisation by alpha w v^T
inline void ldu_update_pos(float *l, double *w, double *v, int nvar, double alpha) {
    double *wa = w - 1, *va = v - 1;
    for (int i = 1; i <= nvar; i++) {
        const double vai = va[i];
        float *lai = &l[-1 + (i - 1) * nvar];
        double d = lai[i];
        double b = d + (alpha * wa[i]) * vai;
        lai[i] = b;
        d /= b;
        const double c = vai * alpha / b;
        b = wa[i] * alpha / b;
        alpha *= d;
        for (int j = i + 1; j <= nvar; j++) {
            const double waj = wa[j];
            wa[j] -= wa[i] * lai[j];
            lai[j] *= d;
            lai[j] += c * waj;
            float *laj = &l[-1 + (j - 1) * nvar];
            const double vaj = va[j];
            va[j] -= vai * laj[i];
            laj[i] *= d;
            laj[i] += b * vaj;
        }
    }
}

// forward substitution: dup = -L^{-1} g
inline void ldu_solve_lower(const float *l, double *dup, const double *g, int nvar) {
    double *dupa = dup - 1;
    const double *ga = g - 1;
    for (int i = 1; i <= nvar; i++) {
        double sum = 0;
        const float *lai = &l[i - 1];
        for (int j = 1; j <= i - 1; j++) sum += lai[(j - 1) * nvar] * dupa[j];
        dupa[i] = -ga[i] - sum;
    }
}

// back substitution with the diagonal: p = U^{-1} D^{-1} p
inline void ldu_solve_upper(const float *du, double *p, int nvar) {
    double *pa = p - 1;
    for (int i = nvar; i >= 1; i--) {
        double sum = 0;
        const float *duai = &du[i - 1];
        for (int j = i + 1; j <= nvar; j++) sum += duai[(j - 1) * nvar] * pa[j];
        pa[i] = pa[i] / duai[(i - 1) * nvar] - sum;
    }
}

// ---- the iteration -----------------------------------------------------------
template <class Residual>
struct Newton {
    Residual residual_fn;   // int(const double *x, double *g): SFGPU_OK or an error status
    int n;
    sfgpu_newton_settings st;
    bool pseudohessian;
    // SFNewton state
    std::vector<double> x, x0, xb, p, p0, g, g0;
    std::vector<float> h;
    int it = 0, iterations = 0, lineiterations = 0, functioncalls = 0, trouble = 0, resetiteration = 0;
    double alpha = 1, minimum = 0, accuracy = 0, trustregion = 0, trustfactor = 1, deltamax = 0;
    bool samehessian = false, newtondirection = false, have_h = false;
    int nbits = 53;
    // SF_Solve::inneriteration state
    double minAccuracySoFar = 1e30;
    int smallAlphaCount = 0;
    int rc = SFGPU_OK;

    int residual(double *gout) {
        int r = residual_fn(x.data(), gout);
        functioncalls++;
        if (r != SFGPU_OK) rc = r;
        return r;
    }

    void startderivatives() {
        const float diagonal = 1 + norm2(g.data(), n);
        std::fill(h.begin(), h.end(), 0.0f);
        for (int i = 0; i < n; i++) h[i + n * i] = diagonal;
    }

    void resethessian() {
        trouble = 0;
        startderivatives();
        resetiteration = iterations;
    }

    void numhessian() {
        std::vector<double> g1(n);
        const double dmax2 = pow(2.0, nbits / 2), dmax3 = pow(2.0, nbits / 3);
        for (int i = 0; i < n && rc == SFGPU_OK; i++) {
            const double xt = x[i];
            double di = (1 / (dmax3 * dmax3 * fabs(h[i + n * i]) + dmax3 + fabs(g[i])) + 1 / dmax2) * (1 + fabs(x[i]));
            if (di < st.deltamin) di = st.deltamin;
            x[i] += di;
            residual(g1.data());
            x[i] = xt;
            for (int j = 0; j < n; j++) h[j + n * i] = (g1[j] - g[j]) / di;
        }
        residual(g.data());
    }

    void findhessian() {
        if (samehessian) return;
        if (iterations == 0) resethessian();
        numhessian();
        if (!pseudohessian) {
            ldu_decompose(h.data(), n);
            int ntr = 0;   // SFNewton passes ntr by value: trouble becomes 0
            trouble = ntr;
        }
    }

    void newhessian() {
        const double dmin = 1 / pow(2.0, nbits);
        if (!pseudohessian) {
            findhessian();
        } else if (!samehessian && alpha != 0 && iterations != 0) {
            std::vector<double> y(n), hp(n);
            double py = 0, php = 0, y2 = 0, gg = 0, g2 = 0;
            for (int i = 0; i < n; i++) {
                const double dg = g[i] - g0[i];
                y[i] = dg;
                py += p[i] * dg;
                y2 += pow(y[i], 2);
                gg += g[i] * g0[i];
                g2 += pow(g[i], 2);
            }
            if (!newtondirection) ldu_multiply(hp.data(), 1, h.data(), p.data(), n);
            else for (int i = 0; i < n; i++) hp[i] = -g0[i];
            php = inner(p.data(), hp.data(), n);
            double theta = py / (10 * dmin + alpha * php);
            if (n >= 1 && theta > 0 && iterations == resetiteration + 1 &&
                accuracy > st.max_accuracy_for_hessian_scaling) {
                alpha *= theta;
                py /= theta;
                php /= theta;
                for (int i = 0; i < n; i++) {
                    p[i] /= theta;
                    h[i + n * i] *= theta;
                }
            }
            if (n >= 1) trustfactor *= (4 / (pow(theta - 1, 2) + 1) + 0.5);
            if (n > 1) {
                double sum = alpha * pow(norm2(p.data(), n), 2);
                theta = fabs(py / (alpha * php));
                if (theta < .01) sum /= 0.8;
                else if (theta > 100) sum *= theta / 50;
                for (int i = 0; i < n; i++) y[i] -= alpha * hp[i];
                ldu_update_pos(h.data(), y.data(), p.data(), n, 1.0 / sum);
                trouble -= sign_det(h.data(), n);
                if (trouble < 0) trouble = 0;
                else if (trouble >= 3) resethessian();
            } else if (n >= 1 && py > 0) {
                trouble = 0;
                theta = py > 0.2 * alpha * php ? 1 : 0.8 * alpha * php / (alpha * php - py);
                if (theta < 1) {
                    py = 0;
                    for (int i = 0; i < n; i++) {
                        y[i] = theta * y[i] + (1 - theta) * alpha * hp[i];
                        py += p[i] * y[i];
                    }
                }
                ldu_update_pos(h.data(), y.data(), y.data(), n, 1.0 / (alpha * py));
                ldu_update_neg(h.data(), hp.data(), n, -1.0 / php);
            }
        } else if (!samehessian) {
            resethessian();
        }
    }

    void direction() {
        if (iterations == 0 && !samehessian) {
            h.assign((size_t)n * n, 0.0f);
            have_h = true;
            newhessian();
        }
        newtondirection = true;
        ldu_solve_lower(h.data(), p.data(), g.data(), n);
        ldu_solve_upper(h.data(), p.data(), n);
        newtondirection = st.ignore_newton_direction ? true : sign_det(h.data(), n) > 0;
        if (!newtondirection)
            for (int i = 0; i < n; i++) p[i] *= -1;
    }

    double residue() const {
        return sqrt(norm2(p.data(), n) * norm2(g.data(), n) / (1 + norm2(x.data(), n)));
    }

    // SF_Solve::inneriteration: Hessian resets when the accuracy walks backwards
    // or the step stays small.  Its switches to a full Hessian need an
    // accuracy below min_accuracy_for_hessian, which is 0 unless the input
    // sets n_iterations_for_hessian (SF_Solve.cpp:1948-1952), and are not kept
    void inneriteration() {
        if (iterations > 0) samehessian = false;
        if (accuracy < minAccuracySoFar && iterations > 0 && accuracy == fabs(accuracy)) minAccuracySoFar = accuracy;
        if (accuracy > minAccuracySoFar * st.reset_hessian_criterion && accuracy == fabs(accuracy)) {
            resethessian();
            minAccuracySoFar *= 1.5;
            if (deltamax > 0.005) set_deltamax(0.9 * deltamax);
        }
        if (alpha < st.small_alpha) smallAlphaCount++;
        else smallAlphaCount = 0;
        if (smallAlphaCount == st.max_n_small_alpha) {
            smallAlphaCount = 0;
            resethessian();
            if (deltamax > 0.005) set_deltamax(0.9 * deltamax);
        }
    }

    void set_deltamax(double d) {
        if (d > st.deltamin) deltamax = d;
    }

    void newdirection(int &k) {
        inneriteration();
        p0 = p;
        direction();
        accuracy = residue();
        if (it != k) iterations = it;
    }

    bool zero(double a, bool compute_g) {
        lineiterations++;
        if (lineiterations == 5) {
            // SFNewton re-evaluates at x0 here to detect time-dependent
            // residuals (it only warns); the evaluation is kept for parity of
            // the function-call count
            std::vector<double> keep = x;
            x = x0;
            residual(g.data());
            x = keep;
            for (int i = 0; i < n; i++)
                if (!std::isfinite(g[i])) { a *= -1; break; }
        }
        for (int i = 0; i < n; i++) x[i] = x0[i] + a * p[i];
        bool valid = true;
        if (compute_g) {
            residual(g.data());
            for (int i = 0; i < n && valid; i++)
                if (!std::isfinite(g[i])) { valid = false; g[i] = 1; }
            minimum = pow(norm2(g.data(), n), 2);
        }
        return valid;
    }

    double linecriterion() {
        double normg = norm2(g0.data(), n);
        const double gg0 = inner(g.data(), g0.data(), n) / normg / normg;
        normg = pow(norm2(g.data(), n) / normg, 2);
        if ((gg0 > 1 || normg > 1) && normg - gg0 * fabs(gg0) < 0.2) normg = 1.5 * normg;
        if (gg0 < 0 && normg < 2) return 1;
        if (normg > 10) return .01;
        return 0.4 * (1 + 0.75 * normg) / (normg - gg0 * fabs(gg0) + 0.1);
    }

    double stepchange() {
        double change, crit;
        change = crit = linecriterion();
        while (crit < 0.35 && lineiterations < st.linesearchlimit) {
            alpha /= 4;
            zero(alpha, true);
            crit = linecriterion();
            change = 1;
        }
        return change;
    }

    void newtrustregion() {
        const double normp0 = norm2(p0.data(), n);
        if (normp0 > 0 && trustregion > 2 * alpha * normp0) trustregion = 2 * alpha * normp0;
        trustregion *= trustfactor;
        trustfactor = 1.0;
        if (trustregion > deltamax) trustregion = deltamax;
        if (trustregion < st.deltamin) trustregion = st.deltamin;
    }

    int run() {
        deltamax = st.deltamax;
        trustregion = deltamax;
        trustfactor = 1;
        alpha = 1;
        x0.assign(n, 0); xb.assign(n, 0); p.assign(n, 0); g.assign(n, 0); g0.assign(n, 0); p0.assign(n, 0);
        if (residual(g.data())) return rc;
        minimum = pow(norm2(g.data(), n), 2);
        int k = 0;
        newdirection(k);
        double normg = sqrt(minimum);
        double lowest_error = normg;
        while ((st.tolerance < accuracy || st.tolerance * 10 < normg) && iterations < st.iterationlimit &&
               accuracy == fabs(accuracy) && rc == SFGPU_OK) {
            k = it = iterations = iterations + 1;
            lineiterations = 0;
            newtrustregion();
            const double alphabound = trustregion / (norm2(p.data(), n) + 1 / pow(2.0, nbits));
            x0 = x;
            g0 = g;
            alpha = alphabound < 1 ? alphabound : 1;   // linesearch: one trial step
            zero(alpha, true);
            trustfactor *= stepchange();
            trustfactor *= alpha / alphabound;
            if (accuracy < lowest_error) {
                lowest_error = accuracy;
                xb = x;
            }
            if (!samehessian) newhessian();
            newdirection(k);
            normg = sqrt(minimum);
        }
        return rc;
    }
};

}  // namespace sfnewton


#endif
