/*
 * Host-side potential tables (see potential_table.cpp for the format).
 */
#pragma once
#include <algorithm>
#include <cstdint>
#include <functional>
#include <vector>

namespace mxg {

using ScalarFn = std::function<double(double)>;

enum : uint32_t {
    kFlagLJ126 = 1u << 0,
    kFlagR2 = 1u << 4,
    kFlagR = 1u << 5,
    kFlagAngle = 1u << 6,
    kFlagHarmonic = 1u << 7,
    kFlagDihedral = 1u << 8,
    kFlagScaled = 1u << 11,
    kFlagShifted = 1u << 12,
};

enum : int { kKindTable = 0, kKindDPD = 1 };

struct PotentialTable {
    int kind = kKindTable;
    uint32_t flags = 0;
    float alpha[4] = {0, 0, 0, 0};
    float r0_plusone = 0.0f;
    float a = 0.0f, b = 0.0f;
    int n = 0;
    std::vector<float> c;  // (n+1)*8
    std::vector<double> c64;  // the same coefficients before rounding to float
    float dpd_alpha = 0, dpd_gamma = 0, dpd_sigma = 0;
    std::vector<double> params;  // construction parameters, for re-fitting
    int form = 0;                // analytic form (kForm*), for frozen-node re-fits
    std::vector<float> nodes;    // the fit's n+1 interval nodes (stretched domain)
};

enum : int { kFormNone = 0, kFormLJ126 = 1, kFormMorse = 2, kFormHarmonic = 3, kFormPower = 4,
             kFormHarmonicAngle = 5, kFormHarmonicDihedral = 6 };

/* Frozen-node re-fit: the table of p's analytic form at new parameters, on p's
 * nodes and interval map (same n), so the coefficients depend linearly on the
 * sampled function. params has the construction parameters' layout. */
int refit_frozen(PotentialTable &p, const std::vector<double> &params);
/* Table (same nodes, map and n as p) of dV/dtheta_k: the derivative of p's
 * coefficients with respect to construction parameter k at p.params. Only
 * parameters that change the tabulated function have one (LJ A, B; Morse d, a;
 * harmonic k, r0); returns -1 otherwise. */
int param_derivative_table(const PotentialTable &p, int k, PotentialTable &out);

int build_table(PotentialTable &p, const ScalarFn &f, const ScalarFn &fp, const ScalarFn &f6, float a, float b,
                float tol);
int make_lj126(PotentialTable &p, double a, double b, double A, double B, double tol);
int make_morse(PotentialTable &p, double d, double alpha, double r0, double min, double max, double tol);
int make_harmonic(PotentialTable &p, double k, double r0, double min, double max, double tol);
int make_power(PotentialTable &p, double k, double r0, double alpha, double a, double b, double tol);
/* k (acos(c) - theta0)^2 on cos(max) <= c <= cos(min), with min clipped to >= 0 and max to <= pi. */
int make_harmonic_angle(PotentialTable &p, double k, double theta0, double min, double max, double tol);
/* K (1 + cos(n phi - delta)) in c = cos(phi) on [-1, 1] (pulled in by sqrt(eps) unless delta is a
 * multiple of pi); n >= 1. */
int make_harmonic_dihedral(PotentialTable &p, double K, int n, double delta, double tol);
int make_dpd(PotentialTable &p, double alpha, double gamma, double sigma, double cutoff, bool shifted);
bool eval_ex(const PotentialTable &p, float ri, float rj, float r2, float *e, float *f);
void eval_r(const PotentialTable &p, float r, float *e, float *f);

}  // namespace mxg
