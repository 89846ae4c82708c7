/*
 * Host-side piecewise-polynomial potential tables.
 *
 * A potential V(r) on [a, b] is stored as n+1 intervals of 8 floats
 * {m, 1/h, c5, c4, c3, c2, c1, c0}: interval k covers [m-h, m+h] and
 * V(r) = c0 + x*(c1 + x*(c2 + ... )) with x = (r - m)/h. The interval index of r
 * is trunc(alpha0 + r*(alpha1 + r*alpha2)), a quadratic node map chosen from
 * V's sixth derivative. Interval 0 is a linear continuation of interval 1 below
 * a. This is the table format of the reference's potential_init
 * (src/mdcore/src/MxPotential.cpp:1690-1930) and its helpers
 * potential_getfp (:1949-2030), potential_getfp_fixend (:2032-2113),
 * potential_getcoeffs (:2139-2260) and
 * potential_getalpha (:2277-2338); the GPU kernels consume exactly this format.
 *
 * The fit reproduces the reference's FP32 coefficient arrays bit for bit, so
 * every intermediate keeps the reference's precision: node positions, domain
 * bounds, the interval map and the tolerance are single precision (the
 * reference's FPTYPE), the projections and the tridiagonal solve are double.
 * Where the reference mixes the two, this code spells the conversions out.
 */
#include "potential_table.h"

#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

namespace mxg {

namespace {

constexpr int kDegree = 5;               // polynomial degree per interval
constexpr int kChunk = kDegree + 3;      // floats per interval
constexpr int kIvalsFirstLeft = 1;       // first bracket of the interval-count search
constexpr int kIvalsFirstRight = 10;
constexpr int kIvalsMax = 3048;          // upper limit on intervals
constexpr int kSamples = 100;            // Chebyshev samples per interval

/* Chebyshev abscissae cos(j*k*pi/N) for k = 0..6, rounded to float once. */
const std::vector<float> &cheb_cos_table() {
    static std::vector<float> t = [] {
        std::vector<float> v(7 * kSamples);
        for (int k = 0; k < 7; ++k)
            for (int j = 0; j < kSamples; ++j) v[k * kSamples + j] = (float)std::cos(j * k * M_PI / kSamples);
        return v;
    }();
    return t;
}

/* Gauss-Chebyshev nodes/weights used to project V onto the cubic Hermite
 * cardinal functions when solving for interior slopes. */
struct SlopeQuadrature {
    double node[kSamples];
    double weight[kSamples];
    SlopeQuadrature() {
        for (int k = 1; k < kSamples - 1; ++k) {
            node[k] = std::cos(k * M_PI / (kSamples - 1));
            weight[k] = 1.0 / std::sqrt(1.0 - node[k] * node[k]);
        }
        node[0] = 1.0;
        node[kSamples - 1] = -1.0;
        weight[0] = 0.0;
        weight[kSamples - 1] = 0.0;
    }
};

const SlopeQuadrature &slope_quadrature() {
    static SlopeQuadrature q;
    return q;
}

/* Node slopes that minimise the L2 misfit of the piecewise cubic Hermite
 * interpolant: a tridiagonal system over the n+1 nodes. With fixed_ends the
 * end slopes are pinned to fpa, fpb (potential_getfp_fixend); otherwise the
 * end rows are the misfit's own normal equations (potential_getfp, used when
 * a potential has no analytic derivative). */
void solve_node_slopes(const ScalarFn &f, bool fixed_ends, double fpa, double fpb, int n, const float *x,
                       double *fp) {
    // inner products of the Hermite cardinal functions on [-1,1]
    const double cl1[4] = {0.25, -0.25, -0.25, 0.25};
    const double cr1[4] = {-0.25, -0.25, 0.25, 0.25};
    const double l0l1 = 0.1125317885884428;
    const double l1l1 = 0.03215579530433858;
    const double l0r1 = -0.04823369227661384;
    const double l1r1 = -0.02143719641629633;
    const double r0r1 = -0.1125317885884429;
    const double r1r1 = 0.03215579530433859;
    const double l1r0 = 0.04823369227661384;
    const SlopeQuadrature &q = slope_quadrature();

    std::vector<double> fx(n + 1), hx(n), lo(n + 1), diag(n + 1), up(n + 1), rhs(n + 1), pl(n), pr(n);
    for (int i = 0; i <= n; ++i) fx[i] = f(x[i]);
    for (int i = 0; i < n; ++i) hx[i] = x[i + 1] - x[i];  // float difference, widened
    for (int i = 0; i < n; ++i) {
        double sl = 0.0, sr = 0.0;
        const double mid = 0.5 * (x[i] + x[i + 1]);
        const double half = 0.5 * (x[i + 1] - x[i]);
        for (int k = 1; k < kSamples - 1; ++k) {
            const double t = q.node[k];
            const double v = f(mid + half * t);
            sl += q.weight[k] * (v * (cl1[0] + t * (cl1[1] + t * (cl1[2] + t * cl1[3]))));
            sr += q.weight[k] * (v * (cr1[0] + t * (cr1[1] + t * (cr1[2] + t * cr1[3]))));
        }
        pl[i] = sl / (kSamples - 2);
        pr[i] = sr / (kSamples - 2);
    }
    if (fixed_ends) {
        diag[0] = 1.0;
        up[0] = 0.0;
        rhs[0] = fpa;
    } else {
        diag[0] = l1l1 * hx[0];
        up[0] = l1r1 * hx[0];
        rhs[0] = 2 * (pl[0] - fx[0] * l0l1 - fx[1] * l1r0);
    }
    for (int i = 1; i < n; ++i) {
        lo[i] = l1r1 * hx[i - 1];
        diag[i] = r1r1 * hx[i - 1] + l1l1 * hx[i];
        up[i] = l1r1 * hx[i];
        rhs[i] = 2 * (pr[i - 1] - fx[i - 1] * l0r1 - fx[i] * r0r1) + 2 * (pl[i] - fx[i] * l0l1 - fx[i + 1] * l1r0);
    }
    if (fixed_ends) {
        lo[n] = 0.0;
        diag[n] = 1.0;
        rhs[n] = fpb;
    } else {
        lo[n] = l1r1 * hx[n - 1];
        diag[n] = r1r1 * hx[n - 1];
        rhs[n] = 2 * (pr[n - 1] - fx[n - 1] * l0r1 - fx[n] * r0r1);
    }
    for (int i = 1; i <= n; ++i) {  // forward elimination
        const double m = lo[i] / diag[i - 1];
        diag[i] = diag[i] - m * up[i - 1];
        rhs[i] = rhs[i] - m * rhs[i - 1];
    }
    fp[n] = rhs[n] / diag[n];
    for (int i = n - 1; i >= 0; --i) fp[i] = (rhs[i] - up[i] * fp[i + 1]) / diag[i];
}

/* Fills the n interval chunks at c (each kChunk floats) for the nodes xi and
 * returns the largest interval error relative to max(|V|, 1) through err. If
 * c64 is not null it receives the same coefficients before rounding to float.
 * An empty fprime selects the free-end slope solve. */
void fit_intervals(const ScalarFn &f, const ScalarFn &fprime, const float *xi, int n, float *c, double *c64,
                   float *err) {
    const std::vector<float> &ck = cheb_cos_table();
    std::vector<double> fnode(n + 1), slope(n + 1);
    double samples[kSamples];
    for (int k = 0; k <= n; ++k) fnode[k] = f(xi[k]);
    if (fprime)
        solve_node_slopes(f, true, fprime(xi[0]), fprime(xi[n]), n, xi, slope.data());
    else
        solve_node_slopes(f, false, 0.0, 0.0, n, xi, slope.data());

    *err = 0.0f;
    for (int i = 0; i < n; ++i) {
        float *out = c + i * kChunk;
        const double m = (xi[i] + xi[i + 1]) / 2;  // float arithmetic, widened
        const double h = (xi[i + 1] - xi[i]) / 2;
        const double fa = fnode[i], fb = fnode[i + 1];
        const double dfa = slope[i] * h, dfb = slope[i + 1] * h;

        // Chebyshev coefficients phi_j of V on the interval
        double phi[7];
        for (int k = 0; k < kSamples; ++k) samples[k] = f(m + h * std::cos(k * M_PI / kSamples));
        for (int j = 0; j < 7; ++j) {
            phi[j] = (fa + (1 - 2 * (j % 2)) * fb) / 2;
            for (int k = 1; k < kSamples; ++k) phi[j] += samples[k] * ck[j * kSamples + k];
            phi[j] *= 2.0 / kSamples;
        }
        // cubic Hermite part in the Chebyshev basis, then the two degree-4/5
        // corrections that keep end values and slopes fixed
        double t[6];
        t[0] = (4 * (fa + fb) + dfa - dfb) / 4;
        t[1] = -(9 * (fa - fb) + dfa + dfb) / 16;
        t[2] = (dfb - dfa) / 8;
        t[3] = (fa - fb + dfa + dfb) / 16;
        t[4] = 0.0;
        t[5] = 0.0;
        double w = (6 * (t[0] - phi[0]) - 4 * (t[2] - phi[2]) - phi[4]) / (36 + 16 + 1);
        t[0] += -6 * w;
        t[2] += 4 * w;
        t[4] = -w;
        w = (2 * (t[1] - phi[1]) - 3 * (t[3] - phi[3]) - phi[5]) / (4 + 9 + 1);
        t[1] += -2 * w;
        t[3] += 3 * w;
        t[5] = -w;
        // monomials in x on [-1, 1]
        out[7] = t[0] / 2 - t[2] + t[4];
        out[6] = t[1] - 3 * t[3] + 5 * t[5];
        out[5] = 2 * t[2] - 8 * t[4];
        out[4] = 4 * t[3] - 20 * t[5];
        out[3] = 8 * t[4];
        out[2] = 16 * t[5];
        out[1] = 1.0 / h;
        out[0] = m;
        if (c64) {
            double *o = c64 + i * kChunk;
            o[7] = t[0] / 2 - t[2] + t[4];
            o[6] = t[1] - 3 * t[3] + 5 * t[5];
            o[5] = 2 * t[2] - 8 * t[4];
            o[4] = 4 * t[3] - 20 * t[5];
            o[3] = 8 * t[4];
            o[2] = 16 * t[5];
            o[1] = 1.0 / h;
            o[0] = m;
        }

        double vmax = 0.0, emax = 0.0;
        for (int k = 1; k < kSamples; ++k) {
            vmax = std::fmax(std::fabs(samples[k]), vmax);
            const double x = ck[kSamples + k];
            const double e = std::fabs(samples[k] - out[7] -
                                       x * (out[6] + x * (out[5] + x * (out[4] + x * (out[3] + x * out[2])))));
            emax = std::fmax(e, emax);
        }
        emax /= std::fmax(vmax, 1.0);
        *err = std::fmax(emax, (double)*err);
    }
}

/* Node-distribution exponent from a golden-section search on the sixth
 * derivative, 4 decimal digits. */
double node_exponent(const ScalarFn &f6, double a, double b) {
    double xs[kSamples], v6[kSamples];
    double vmax = 0.0;
    const double golden = 2.0 / (1 + std::sqrt(5));
    for (int i = 0; i < kSamples; ++i) {
        xs[i] = ((double)i + 1) / (kSamples + 1);
        v6[i] = f6(a + (b - a) * xs[i]);
        vmax = std::fmax(vmax, std::fabs(v6[i]));
    }
    if (vmax == 0.0) return 1.0;
    auto objective = [&](double al) {
        double best = 0.0;
        for (int j = 0; j < kSamples; ++j) {
            const double t = std::fabs(std::pow(al + 2 * (1 - al) * xs[j], -6) * v6[j]);
            if (t > best) best = t;
        }
        return best;
    };
    double al[4], fa[4];
    al[0] = 0;
    al[3] = 2;
    al[1] = al[3] - 2 * golden;
    al[2] = al[0] + 2 * golden;
    for (int i = 0; i < 4; ++i) fa[i] = objective(al[i]);
    while (al[3] - al[0] > 1.0e-4) {
        int i;
        if (fa[1] < fa[2]) {
            al[3] = al[2]; fa[3] = fa[2];
            al[2] = al[1]; fa[2] = fa[1];
            al[1] = al[3] - (al[3] - al[0]) * golden;
            i = 1;
        } else {
            al[0] = al[1]; fa[0] = fa[1];
            al[1] = al[2]; fa[1] = fa[2];
            al[2] = al[0] + (al[3] - al[0]) * golden;
            i = 2;
        }
        fa[i] = objective(al[i]);
    }
    return (al[0] + al[3]) / 2;
}

/* n+1 nodes on [a, b] where the (unscaled) interval map takes the values
 * i/n, found by Newton iteration in single precision. */
void place_nodes(const float *map, float a, float b, int n, std::vector<float> &xi) {
    const float mtol = 10 * FLT_EPSILON;
    xi.assign(n + 1, 0.0f);
    xi[0] = a;
    xi[n] = b;
    for (int i = 1; i < n; ++i) {
        xi[i] = a + (b - a) * i / n;
        for (int it = 0; it < 1000; ++it) {
            const double e = i - n * (map[0] + xi[i] * (map[1] + xi[i] * map[2]));
            xi[i] += e / (n * (map[1] + 2 * xi[i] * map[2]));
            if (std::fabs(e) < n * mtol) break;
        }
    }
}

/* Interval 0: the linear continuation of interval 1's left end, x = (r - a)/a. */
template <typename T>
void fill_interval0(T *c, float a) {
    c[0] = a;
    c[1] = 1.0 / a;
    double coef[kDegree], deriv[kDegree];
    for (int k = 0; k < kDegree; ++k) {
        coef[k] = c[2 * kChunk - 1 - k];
        deriv[k] = 0.0;
    }
    for (int i = 0; i < kDegree; ++i)
        for (int k = kDegree - 1; k >= i; --k) {
            deriv[i] = coef[k] + (-1.0) * deriv[i];
            coef[k] *= (k - i) * c[kChunk + 1] * a;
        }
    c[kChunk - 1] = deriv[0];
    c[kChunk - 2] = deriv[1];
    c[kChunk - 3] = 0.5 * deriv[2];
    for (int k = 3; k <= kDegree; ++k) c[kChunk - 1 - k] = 0.0;
}

/* The analytic form of a table kind: value and first derivative at the
 * construction parameters (the layout of PotentialTable::params). */
bool form_functions(int form, const std::vector<double> &q, ScalarFn &f, ScalarFn &fp) {
    switch (form) {
    case kFormLJ126: {
        const double A = q[2], B = q[3];
        f = [A, B](double r) {
            const double ir = 1.0 / r, ir2 = ir * ir, ir6 = ir2 * ir2 * ir2, ir12 = ir6 * ir6;
            return A * ir12 - B * ir6;
        };
        fp = [A, B](double r) {
            const double ir = 1.0 / r, ir2 = ir * ir, ir4 = ir2 * ir2, ir12 = ir4 * ir4 * ir4;
            return 6.0 * ir * (-2.0 * A * ir12 + B * ir4 * ir2);
        };
        return true;
    }
    case kFormMorse: {
        const double d = q[0], al = q[1];
        f = [d, al](double r) { return d * (std::pow(M_E, -2 * al * (-1 + r)) - 2 / std::pow(M_E, al * (-1 + r))); };
        fp = [d, al](double r) {
            return d * ((-2 * al) / std::pow(M_E, 2 * al * (-1 + r)) + (2 * al) / std::pow(M_E, al * (-1 + r)));
        };
        return true;
    }
    case kFormHarmonic: {
        const double k = q[0], r0 = q[1];
        f = [k, r0](double r) { return k * (r - r0) * (r - r0); };
        fp = [k, r0](double r) { return 2.0 * k * (r - r0); };
        return true;
    }
    default:
        return false;
    }
}

/* d/dtheta_k of the analytic form (value and first derivative). */
bool form_param_derivative(int form, const std::vector<double> &q, int k, ScalarFn &f, ScalarFn &fp) {
    if (form == kFormLJ126 && (k == 2 || k == 3)) {
        if (k == 2) {  // dV/dA = r^-12
            f = [](double r) { return std::pow(r, -12.0); };
            fp = [](double r) { return -12.0 * std::pow(r, -13.0); };
        } else {  // dV/dB = -r^-6
            f = [](double r) { return -std::pow(r, -6.0); };
            fp = [](double r) { return 6.0 * std::pow(r, -7.0); };
        }
        return true;
    }
    if (form == kFormMorse && (k == 0 || k == 1)) {
        const double d = q[0], al = q[1];
        if (k == 0) {  // V is linear in d
            f = [al](double r) { return std::exp(-2 * al * (r - 1)) - 2 * std::exp(-al * (r - 1)); };
            fp = [al](double r) { return -2 * al * std::exp(-2 * al * (r - 1)) + 2 * al * std::exp(-al * (r - 1)); };
        } else {
            f = [d, al](double r) {
                const double u = r - 1;
                return d * (-2 * u * std::exp(-2 * al * u) + 2 * u * std::exp(-al * u));
            };
            fp = [d, al](double r) {
                const double u = r - 1, e2 = std::exp(-2 * al * u), e1 = std::exp(-al * u);
                return d * (-2 * e2 + 4 * al * u * e2 + 2 * e1 - 2 * al * u * e1);
            };
        }
        return true;
    }
    if (form == kFormHarmonic && (k == 0 || k == 1)) {
        const double kk = q[0], r0 = q[1];
        if (k == 0) {
            f = [r0](double r) { return (r - r0) * (r - r0); };
            fp = [r0](double r) { return 2.0 * (r - r0); };
        } else {
            f = [kk, r0](double r) { return -2.0 * kk * (r - r0); };
            fp = [kk](double) { return -2.0 * kk; };
        }
        return true;
    }
    return false;
}

/* Refit of p's coefficient array for the function f (end slopes from fp) on
 * p's frozen nodes. */
void refit_on_nodes(PotentialTable &p, const ScalarFn &f, const ScalarFn &fp) {
    const int n = p.n;
    std::vector<float> c((size_t)(n + 1) * kChunk, 0.0f);
    std::vector<double> c64((size_t)(n + 1) * kChunk, 0.0);
    float err = 0.0f;
    fit_intervals(f, fp, p.nodes.data(), n, c.data() + kChunk, c64.data() + kChunk, &err);
    fill_interval0(c.data(), p.nodes[0]);
    fill_interval0(c64.data(), p.nodes[0]);
    p.c.swap(c);
    p.c64.swap(c64);
}

}  // namespace

int refit_frozen(PotentialTable &p, const std::vector<double> &params) {
    if (p.kind != kKindTable || p.nodes.empty() || params.size() != p.params.size()) return -1;
    ScalarFn f, fp;
    if (!form_functions(p.form, params, f, fp)) return -1;
    refit_on_nodes(p, f, fp);
    p.params = params;
    if (p.form == kFormMorse) p.r0_plusone = (float)(params[2] + 1);
    return 0;
}

int param_derivative_table(const PotentialTable &p, int k, PotentialTable &out) {
    if (p.kind != kKindTable || p.nodes.empty()) return -1;
    ScalarFn f, fp;
    if (!form_param_derivative(p.form, p.params, k, f, fp)) return -1;
    out = p;
    refit_on_nodes(out, f, fp);
    return 0;
}

int build_table(PotentialTable &p, const ScalarFn &f, const ScalarFn &fp, const ScalarFn &f6, float a, float b,
                float tol) {
    p.a = a;
    p.b = b;
    // stretch the domain slightly so rounding in the index map stays inside
    b += std::fabs(b) * std::sqrt(FLT_EPSILON);
    a -= std::fabs(a) * std::sqrt(FLT_EPSILON);

    const double expo = node_exponent(f6, a, b);
    double w = 1.0 / (a - b);
    w *= w;
    float map[4];
    map[0] = a * a * w - expo * b * a * w;
    map[1] = -2 * a * w + expo * (a + b) * w;
    map[2] = w - expo * w;
    map[3] = 0.0f;
    w = 2 * FLT_EPSILON * (std::fabs(map[0]) + std::fabs(map[1]) + std::fabs(map[2]));
    map[0] -= w * a / (a - b);
    map[1] += w / (a - b);

    // Fits with n intervals into c[kChunk ...]; returns false on failure.
    auto attempt = [&](int n, std::vector<float> &c, float &err) {
        std::vector<float> xi;
        place_nodes(map, a, b, n, xi);
        c.assign((size_t)(n + 1) * kChunk, 0.0f);
        fit_intervals(f, fp, xi.data(), n, c.data() + kChunk, nullptr, &err);
    };

    int l = kIvalsFirstLeft, r = kIvalsFirstRight;
    std::vector<float> cl, cr, cm;
    float el = 0, er = 0, em = 0;
    attempt(l, cl, el);
    int n;
    std::vector<float> *chosen;
    if (el < tol) {
        n = l;
        chosen = &cl;
    } else {
        for (;;) {  // double the count until the tolerance holds
            attempt(r, cr, er);
            if (er < tol) break;
            if (2 * r > kIvalsMax) return -5;  // potential_err_ivalsmax
            l = r;
            el = er;
            cl.swap(cr);
            r *= 2;
        }
        while (r - l > 1) {  // bisection on the interval count
            const int m = 0.5 * (r + l);
            attempt(m, cm, em);
            if (em > tol) {
                l = m;
                el = em;
                cl.swap(cm);
            } else {
                r = m;
                er = em;
                cr.swap(cm);
            }
        }
        n = r;
        chosen = &cr;
    }

    p.n = n;
    p.c = *chosen;
    p.alpha[0] = map[0] * n;
    p.alpha[1] = map[1] * n;
    p.alpha[2] = map[2] * n;
    p.alpha[3] = map[3];
    p.alpha[0] += 1.0;
    place_nodes(map, a, b, n, p.nodes);
    fill_interval0(p.c.data(), a);
    // the unrounded coefficients of the same fit
    std::vector<float> c32(p.c.size(), 0.0f);
    p.c64.assign(p.c.size(), 0.0);
    float err = 0.0f;
    fit_intervals(f, fp, p.nodes.data(), n, c32.data() + kChunk, p.c64.data() + kChunk, &err);
    fill_interval0(p.c64.data(), a);
    return 0;
}

/* ---- the analytic forms (value, first and sixth derivative) ---- */

int make_lj126(PotentialTable &p, double a, double b, double A, double B, double tol) {
    p = PotentialTable();
    p.flags = kFlagR2 | kFlagLJ126;
    ScalarFn f = [A, B](double r) {
        const double ir = 1.0 / r, ir2 = ir * ir, ir6 = ir2 * ir2 * ir2, ir12 = ir6 * ir6;
        return A * ir12 - B * ir6;
    };
    ScalarFn fp = [A, B](double r) {
        const double ir = 1.0 / r, ir2 = ir * ir, ir4 = ir2 * ir2, ir12 = ir4 * ir4 * ir4;
        return 6.0 * ir * (-2.0 * A * ir12 + B * ir4 * ir2);
    };
    ScalarFn f6 = [A, B](double r) {
        const double r2 = r * r, ir2 = 1.0 / r2, ir6 = ir2 * ir2 * ir2, ir12 = ir6 * ir6;
        return 10080.0 * ir12 * (884.0 * A * ir6 - 33.0 * B);
    };
    p.params = {a, b, A, B, tol};
    p.form = kFormLJ126;
    return build_table(p, f, fp, f6, (float)a, (float)b, (float)tol);
}

int make_morse(PotentialTable &p, double d, double al, double r0, double min, double max, double tol) {
    p = PotentialTable();
    p.flags = kFlagR2 | kFlagShifted;
    p.r0_plusone = (float)(r0 + 1);
    // V(s) = d (e^{-2 al (s-1)} - 2 e^{-al (s-1)}) with s the shifted distance
    ScalarFn f = [d, al](double r) { return d * (std::pow(M_E, -2 * al * (-1 + r)) - 2 / std::pow(M_E, al * (-1 + r))); };
    ScalarFn fp = [d, al](double r) {
        return d * ((-2 * al) / std::pow(M_E, 2 * al * (-1 + r)) + (2 * al) / std::pow(M_E, al * (-1 + r)));
    };
    ScalarFn f6 = [d, al](double r) {
        return d * ((64 * std::pow(al, 6)) / std::pow(M_E, 2 * al * (-1 + r)) -
                    (2 * std::pow(al, 6)) / std::pow(M_E, al * (-1 + r)));
    };
    p.params = {d, al, r0, min, max, tol};
    p.form = kFormMorse;
    return build_table(p, f, fp, f6, (float)min, (float)max, (float)tol);
}

int make_harmonic(PotentialTable &p, double k, double r0, double min, double max, double tol) {
    p = PotentialTable();
    p.flags = kFlagHarmonic & kFlagR2;  // the reference combines these with '&' (no flag set)
    ScalarFn f = [k, r0](double r) { return k * (r - r0) * (r - r0); };
    ScalarFn fp = [k, r0](double r) { return 2.0 * k * (r - r0); };
    ScalarFn f6 = [](double) { return 0.0; };
    p.params = {k, r0, min, max, tol};
    p.form = kFormHarmonic;
    return build_table(p, f, fp, f6, (float)min, (float)max, (float)tol);
}

int make_harmonic_angle(PotentialTable &p, double k, double theta0, double min, double max, double tol) {
    p = PotentialTable();
    p.flags = kFlagAngle | kFlagHarmonic;
    // V(c) = k (acos(c) - theta0)^2 in the cosine c, fitted without an analytic
    // derivative (MxPotential.cpp:519-540, 557-594)
    ScalarFn f = [k, theta0](double r) {
        r = std::fmin(1.0, std::fmax(-1.0, r));
        const double theta = std::acos(r);
        return k * (theta - theta0) * (theta - theta0);
    };
    ScalarFn f6 = [](double) { return 0.0; };
    if (min < 0.0) min = 0.0;
    if (max > M_PI) max = M_PI;
    p.params = {k, theta0, min, max, tol};
    p.form = kFormHarmonicAngle;
    return build_table(p, f, ScalarFn(), f6, (float)std::cos(max), (float)std::cos(min), (float)tol);
}

int make_harmonic_dihedral(PotentialTable &p, double K, int n, double delta, double tol) {
    p = PotentialTable();
    if (n < 1) return -1;
    p.flags = kFlagR | kFlagHarmonic | kFlagDihedral;
    // V(c) = K (1 + cos(n phi - delta)) in c = cos(phi), phi in [0, pi]:
    // cos(n phi) = T_n(c), sin(n phi) = U_{n-1}(c) sin(phi) (Chebyshev recurrences),
    // fitted without an analytic derivative (MxPotential.cpp:423-447, 484-516)
    ScalarFn f = [K, n, delta](double r) {
        const double cd = std::cos(delta), sd = std::sin(delta);
        double t0 = 1.0, t1 = r, u0 = 1.0, u1 = 2 * r;
        for (int k = 2; k <= n; ++k) {
            const double t2 = 2 * r * t1 - t0, u2 = 2 * r * u1 - u0;
            t0 = t1;
            t1 = t2;
            u0 = u1;
            u1 = u2;
        }
        const double tn = t1, un1 = u0;  // T_n and U_{n-1}
        if (delta == 0.0) return K * (1.0 + tn);
        if (delta == M_PI) return K * (1.0 - tn);
        if (std::fabs(r) < 1.0) return K * (1.0 + tn * cd + un1 * std::sqrt(1.0 - r * r) * sd);
        return K * (1.0 + tn * cd);
    };
    ScalarFn f6 = [](double) { return 0.0; };
    // end points pulled inside [-1, 1] when delta is not a multiple of pi
    double a = -1.0, b = 1.0;
    if (std::fmod(delta, M_PI) != 0) {
        a = -1.0 / (1.0 + std::sqrt(FLT_EPSILON));
        b = 1.0 / (1.0 + std::sqrt(FLT_EPSILON));
    }
    p.params = {K, (double)n, delta, tol};
    p.form = kFormHarmonicDihedral;
    return build_table(p, f, ScalarFn(), f6, (float)a, (float)b, (float)tol);
}

int make_power(PotentialTable &p, double k, double r0, double alpha, double a, double b, double tol) {
    p = PotentialTable();
    p.flags = kFlagR2 | kFlagScaled;
    ScalarFn f = [k, r0, alpha](double x) { return k * std::pow(std::abs(-r0 + x), alpha); };
    // The reference's derivative adds alpha*k instead of multiplying
    // (MxPotential.cpp:1581-1593); the end slopes of the fit depend on it.
    ScalarFn fp = [k, r0, alpha](double x) { return alpha * k + std::pow(std::abs(-r0 + x), -1 + alpha); };
    ScalarFn f6 = [k, r0, alpha](double x) {
        return (-5 + alpha) * (-4 + alpha) * (-3 + alpha) * (-2 + alpha) * (-1 + alpha) * alpha * k *
               std::pow(std::abs(-r0 + x), -6 + alpha);
    };
    const double range = b - a;
    const double fudge = range / 5;
    double fa = a;
    if (a - fudge >= 0.001) fa = a - fudge;
    p.params = {k, r0, alpha, a, b, tol};
    int rc = build_table(p, f, fp, f6, (float)fa, (float)(1.2 * b), (float)tol);
    p.a = (float)a;
    p.b = (float)b;
    return rc;
}

int make_dpd(PotentialTable &p, double alpha, double gamma, double sigma, double cutoff, bool shifted) {
    p = PotentialTable();
    p.kind = kKindDPD;
    p.dpd_alpha = (float)alpha;
    p.dpd_gamma = (float)gamma;
    p.dpd_sigma = (float)sigma;
    p.a = std::sqrt(FLT_EPSILON);
    p.b = (float)cutoff;
    p.n = 0;
    if (shifted) p.flags |= kFlagShifted;
    p.params = {alpha, gamma, sigma, cutoff, shifted ? 1.0 : 0.0};
    return 0;
}

/* Scalar evaluation with the reference's potential_eval_r semantics
 * (potential_eval.hpp:180-207): the table at r itself, f = dV/dr. */
void eval_r(const PotentialTable &p, float r, float *e, float *f) {
    const int ind = (int)std::max(0.0f, p.alpha[0] + r * (p.alpha[1] + r * p.alpha[2]));
    const float *c = p.c.data() + std::min(ind, p.n) * kChunk;
    const float x = (r - c[0]) * c[1];
    float ee = c[2] * x + c[3];
    float eff = c[2];
    for (int k = 4; k < kChunk; ++k) {
        eff = eff * x + ee;
        ee = ee * x + c[k];
    }
    *e = ee;
    *f = eff * c[1];
}

/* Scalar evaluation with the reference's potential_eval_ex semantics. */
bool eval_ex(const PotentialTable &p, float ri, float rj, float r2, float *e, float *f) {
    const float eps = FLT_EPSILON;
    float r = std::sqrt(r2);
    const float ro = r < eps ? eps : r;
    r = r < p.a ? p.a : r;
    if (p.flags & kFlagScaled)
        r = r / (ri + rj);
    else if (p.flags & kFlagShifted)
        r = r - (ri + rj) + p.r0_plusone;
    const unsigned ind = (unsigned)std::max(0.0f, p.alpha[0] + r * (p.alpha[1] + r * p.alpha[2]));
    if (r > p.b || ind > (unsigned)p.n) return false;
    const float *c = p.c.data() + ind * kChunk;
    const float x = (r - c[0]) * c[1];
    float ee = c[2] * x + c[3];
    float eff = c[2];
    for (int k = 4; k < kChunk; ++k) {
        eff = eff * x + ee;
        ee = ee * x + c[k];
    }
    *e = ee;
    *f = eff * c[1] / ro;
    return true;
}

}  // namespace mxg
