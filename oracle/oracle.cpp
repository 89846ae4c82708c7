/*
 * Oracle tier B: an independent C++ restatement of the reference's nonbonded
 * force pass, templated on the arithmetic type.
 *
 * TEST INFRASTRUCTURE ONLY: tests/ and bench.py's CPU-baseline leg call it;
 * the product never links it.
 *
 *   T = float   follows the reference's scalar FP32 operation order
 *               (runner_dopair.cpp:91-340, runner_doself.cpp :446-682,
 *               potential_eval.hpp:106-161, dpd_eval.hpp:21-169) with the
 *               pair shift rounded to float as space_getsid does (space.cpp:95-130).
 *   T = double  the same algorithm in FP64 on the same FP32 table coefficients
 *               and the same FP32 positions: the "FP64 CPU oracle" against which
 *               FP32 rounding error is stated.
 * It also offers a second pair term per type pair (a table potential plus a
 * DPD thermostat summed), which the reference cannot express (engine_addpot
 * keeps one potential per pair, engine.cpp:968-977).
 *
 * Pairs are enumerated within each task's cell pair and filtered by the
 * reference's sorted-projection test (runner_dosort.cpp:133-136,
 * runner_dopair.cpp:132-182): a pair is evaluated only when
 * key_j + dnshift - key_i < dmaxdist. With cubic cells the test keeps two
 * quanta of slack and never drops a pair inside the cutoff; with non-cubic
 * cells it does (it uses |shift| where the projection of the shift belongs),
 * and the oracle reproduces that. The whole cell pair is also skipped when the
 * loop's first exit test underflows (unsigned arithmetic, runner_dopair.cpp:167-171),
 * which happens for particles within one key quantum of the shared face.
 * pruning = 0 or 1 applies both tests (the reference), 2 applies neither. The r < a random-direction branch (dpd_eval.hpp:122-131) is not
 * reproduced; such pairs are counted and skipped.
 */
#include "oracle.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

namespace {

const double kCellShift[13][3] = {
    {5.773502691896258e-01, 5.773502691896258e-01, 5.773502691896258e-01},
    {7.071067811865475e-01, 7.071067811865475e-01, 0.0},
    {5.773502691896258e-01, 5.773502691896258e-01, -5.773502691896258e-01},
    {7.071067811865475e-01, 0.0, 7.071067811865475e-01},
    {1.0, 0.0, 0.0},
    {7.071067811865475e-01, 0.0, -7.071067811865475e-01},
    {5.773502691896258e-01, -5.773502691896258e-01, 5.773502691896258e-01},
    {7.071067811865475e-01, -7.071067811865475e-01, 0.0},
    {5.773502691896258e-01, -5.773502691896258e-01, -5.773502691896258e-01},
    {0.0, 7.071067811865475e-01, 7.071067811865475e-01},
    {0.0, 1.0, 0.0},
    {0.0, 7.071067811865475e-01, -7.071067811865475e-01},
    {0.0, 0.0, 1.0},
};

const int kSortlistID[27] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 0, 12, 11, 10, 9, 8, 7, 6, 5, 4, 3, 2, 1, 0};
const bool kFlip[27] = {1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};

template <typename T>
struct Pot {
    int kind;
    unsigned flags;
    int n;
    T alpha[3];
    T a, b, r0p1;
    const float *c;
    T dpd_alpha, dpd_gamma, dpd_sigma, dpd_delta;
};

/* potential_eval_ex in type T; coefficients widened from float. Its integer
 * decisions (the range test and the interval index) are taken as the FP32 code
 * takes them, from the pair's FP32 r2f (equal to r2 when T is float): they are
 * part of the tabulated model, and an FP64 decision flips pairs that lie on a
 * table edge (a lattice's second neighbours sit on the lattice's Morse edge). */
template <typename T>
bool table_eval_ex(const Pot<T> &p, T ri, T rj, T r2, float r2f, T &e, T &f) {
    const T eps = (T)FLT_EPSILON;
    T r = std::sqrt(r2);
    const T ro = r < eps ? eps : r;
    r = r < p.a ? p.a : r;
    if (p.flags & (1u << 11))
        r = r / (ri + rj);
    else if (p.flags & (1u << 12))
        r = r - (ri + rj) + p.r0p1;
    float rf = std::sqrt(r2f);
    const float af = (float)p.a;
    rf = rf < af ? af : rf;
    if (p.flags & (1u << 11))
        rf = rf / ((float)ri + (float)rj);
    else if (p.flags & (1u << 12))
        rf = rf - ((float)ri + (float)rj) + (float)p.r0p1;
    const float t = (float)p.alpha[0] + rf * ((float)p.alpha[1] + rf * (float)p.alpha[2]);
    const unsigned ind = (unsigned)std::max(0.0f, t);
    if (rf > (float)p.b || ind > (unsigned)p.n) return false;
    const float *c = p.c + ind * 8;
    const T x = (r - (T)c[0]) * (T)c[1];
    T ee = (T)c[2] * x + (T)c[3];
    T eff = (T)c[2];
    for (int k = 4; k < 8; ++k) {
        eff = eff * x + ee;
        ee = ee * x + (T)c[k];
    }
    e = ee;
    f = eff * (T)c[1] / ro;
    return true;
}

template <typename T>
struct Setup {
    int N;
    std::vector<T> x, v;  // N*3
    const int *cell;
    const int *type;
    int ncells;
    const double *origin;
    double dim[3];
    T cut2_pair, cut2_self;
    float cut2f_pair, cut2f_self;  // the FP32 cutoff tests (float(cutoff)^2; float(cutoff^2))
    int ntypes;
    std::vector<T> radius;
    const int *pot_of_pair;
    const int *dpd_of_pair;
    std::vector<Pot<T>> pots;
    std::vector<T> body;
    std::vector<float> xf;  // FP32 positions for the pruning keys
    bool prune;
    float bias, dscale;
    int dmaxdist;
    float axes[13][3];
};

/* r2f: the pair's r2 in the reference's FP32 arithmetic, for its integer decisions */
template <typename T>
void pair_force(const Setup<T> &S, int pi, int pj, const T *dx_in, T r2, float r2f, std::vector<T> &f,
                double &epot, long long &nint, long long &nrand, double *vir) {
    const int ti = S.type[pi], tj = S.type[pj];
    const int pidx = S.pot_of_pair[ti * S.ntypes + tj];
    const int didx = S.dpd_of_pair ? S.dpd_of_pair[ti * S.ntypes + tj] : -1;
    for (int which = 0; which < 2; ++which) {
        const int idx = which == 0 ? pidx : didx;
        if (idx < 0) continue;
        const Pot<T> &p = S.pots[idx];
        if (r2f < (float)p.a * (float)p.a) {
            ++nrand;
            continue;
        }
        T dx[3] = {dx_in[0], dx_in[1], dx_in[2]};
        if (p.kind == 1) {
            const T ri = S.radius[ti], rj = S.radius[tj];
            const bool shifted = p.flags & (1u << 12);
            const T cutoff = shifted ? (p.b + ri + rj) : p.b;
            const float cutf = shifted ? ((float)p.b + (float)ri) + (float)rj : (float)p.b;
            if (r2f > cutf * cutf) continue;
            const T r = std::sqrt(r2);
            const T e[3] = {dx[0] / r, dx[1] / r, dx[2] / r};
            const T w[3] = {S.v[3 * pi] - S.v[3 * pj], S.v[3 * pi + 1] - S.v[3 * pj + 1], S.v[3 * pi + 2] - S.v[3 * pj + 2]};
            const T sr = shifted ? r - ri - rj : r;
            const T oc = sr < 0 ? (T)1 : ((T)1 - sr / cutoff);
            const T fc = p.dpd_alpha * oc;
            const T od = oc * oc;
            const T fd = -p.dpd_gamma * od * (e[0] * w[0] + e[1] * w[1] + e[2] * w[2]);
            const T fr = p.dpd_sigma * oc * p.dpd_delta;
            const T ff = fc + fd + fr;
            for (int k = 0; k < 3; ++k) {
                f[3 * pj + k] = f[3 * pj + k] - ff * e[k];
                f[3 * pi + k] = f[3 * pi + k] + ff * e[k];
            }
            if (vir)  // (x_i - x_j) (x) F_i
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) vir[3 * a + b] += (double)dx[a] * (double)(ff * e[b]);
            ++nint;
        } else {
            T ee, ff;
            if (!table_eval_ex(p, S.radius[ti], S.radius[tj], r2, r2f, ee, ff)) continue;
            for (int k = 0; k < 3; ++k) {
                const T wk = ff * dx[k];
                f[3 * pi + k] -= wk;
                f[3 * pj + k] += wk;
            }
            if (vir)
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) vir[3 * a + b] -= (double)dx[a] * (double)(ff * dx[b]);
            epot += (double)ee;
            ++nint;
        }
    }
}

template <typename T>
int run(const Setup<T> &S, const int *tasks, int ntasks, double *f_out, double *epot_out, long long *counts,
        double *vir) {
    if (vir)
        for (int k = 0; k < 9; ++k) vir[k] = 0.0;
    // particles per cell, in index order
    std::vector<std::vector<int>> members(S.ncells);
    for (int p = 0; p < S.N; ++p) members[S.cell[p]].push_back(p);
    std::vector<T> f(3 * (size_t)S.N, (T)0);
    for (int p = 0; p < S.N; ++p)
        for (int k = 0; k < 3; ++k) f[3 * p + k] = S.body[3 * S.type[p] + k];
    double epot = 0.0;
    long long ncand = 0, nint = 0, nrand = 0;
    for (int q = 0; q < ntasks; ++q) {
        const int type = tasks[4 * q], ci0 = tasks[4 * q + 2], cj0 = tasks[4 * q + 3];
        if (type == 1) {  // self
            const std::vector<int> &mem = members[ci0];
            for (size_t a = 0; a < mem.size(); ++a)
                for (size_t b = a + 1; b < mem.size(); ++b) {
                    const int pi = mem[a], pj = mem[b];
                    T dx[3];
                    float dxf[3];
                    for (int k = 0; k < 3; ++k) {
                        dx[k] = S.x[3 * pi + k] - S.x[3 * pj + k];
                        dxf[k] = S.xf[3 * pi + k] - S.xf[3 * pj + k];
                    }
                    const T r2 = dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2];
                    const float r2f = dxf[0] * dxf[0] + dxf[1] * dxf[1] + dxf[2] * dxf[2];
                    ++ncand;
                    if (r2f > S.cut2f_self) continue;
                    pair_force(S, pi, pj, dx, r2, r2f, f, epot, nint, nrand, vir);
                }
        } else if (type == 2) {  // pair, shift and flip as space_getsid
            int ci = ci0, cj = cj0;
            T shift[3];
            for (int k = 0; k < 3; ++k) {
                double s = S.origin[3 * cj + k] - S.origin[3 * ci + k];
                T sk = (T)s;
                if (sk * 2 > S.dim[k])
                    sk = (T)(sk - S.dim[k]);
                else if (sk * 2 < -S.dim[k])
                    sk = (T)(sk + S.dim[k]);
                shift[k] = sk;
            }
            int sid = 0;
            for (int k = 0; k < 3; ++k) sid = 3 * sid + ((shift[k] < 0) ? 0 : ((shift[k] > 0) ? 2 : 1));
            if (kFlip[sid]) {
                std::swap(ci, cj);
                for (int k = 0; k < 3; ++k) shift[k] = -shift[k];
            }
            // the reference's sorted-projection pruning, always in FP32
            // (runner_dosort.cpp:133-136, runner_dopair.cpp:132-182)
            float fshift[3];
            for (int k = 0; k < 3; ++k) {
                const double sd = S.origin[3 * cj + k] - S.origin[3 * ci + k];
                float sk = (float)sd;
                if (sk * 2 > S.dim[k])
                    sk = (float)(sk - S.dim[k]);
                else if (sk * 2 < -S.dim[k])
                    sk = (float)(sk + S.dim[k]);
                fshift[k] = sk;
            }
            const float *nax = S.axes[kSortlistID[sid]];
            const float nsh = std::sqrt(fshift[0] * fshift[0] + fshift[1] * fshift[1] + fshift[2] * fshift[2]);
            const int dnshift = (int)(S.dscale * nsh);
            auto key = [&](int p) {
                const float proj = S.bias + S.xf[3 * p] * nax[0] + S.xf[3 * p + 1] * nax[1] + S.xf[3 * p + 2] * nax[2];
                return (int)(unsigned)(S.dscale * proj);
            };
            if (S.prune && !members[ci].empty() && !members[cj].empty()) {
                // first-iteration exit of the sorted loop (runner_dopair.cpp:167-171): the
                // largest key of cell i against the smallest of cell j, unsigned arithmetic
                int kmax = -1, kmin = 0x7fffffff;
                for (int pi : members[ci]) kmax = std::max(kmax, key(pi));
                for (int pj : members[cj]) kmin = std::min(kmin, key(pj));
                const unsigned gap = (unsigned)kmin + (unsigned)dnshift - (unsigned)kmax;
                if (gap > (unsigned)S.dmaxdist) {
                    ncand += (long long)members[ci].size() * members[cj].size();
                    continue;
                }
            }
            for (int pi : members[ci])
                for (int pj : members[cj]) {
                    if (S.prune && !((unsigned)key(pj) + (unsigned)dnshift - (unsigned)key(pi) < (unsigned)S.dmaxdist)) {
                        ++ncand;
                        continue;
                    }
                    T pix[3], dx[3];
                    float dxf[3];
                    for (int k = 0; k < 3; ++k) {
                        pix[k] = S.x[3 * pi + k] - shift[k];
                        dx[k] = pix[k] - S.x[3 * pj + k];
                        dxf[k] = (S.xf[3 * pi + k] - fshift[k]) - S.xf[3 * pj + k];
                    }
                    const T r2 = dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2];
                    const float r2f = dxf[0] * dxf[0] + dxf[1] * dxf[1] + dxf[2] * dxf[2];
                    ++ncand;
                    if (r2f > S.cut2f_pair) continue;
                    pair_force(S, pi, pj, dx, r2, r2f, f, epot, nint, nrand, vir);
                }
        }
    }
    for (size_t k = 0; k < f.size(); ++k) f_out[k] = (double)f[k];
    *epot_out = epot;
    if (counts) {
        counts[0] = ncand;
        counts[1] = nint;
        counts[2] = nrand;
    }
    return 0;
}

template <typename T>
int build_and_run(const OrcInput *in, double *f_out, double *epot_out, long long *counts, double *vir) {
    Setup<T> S;
    S.N = in->N;
    S.x.resize(3 * (size_t)in->N);
    S.v.resize(3 * (size_t)in->N);
    for (size_t k = 0; k < S.x.size(); ++k) {
        S.x[k] = (T)in->xrel[k];
        S.v[k] = in->vel ? (T)in->vel[k] : (T)0;
    }
    S.cell = in->cell;
    S.type = in->type;
    S.ncells = in->ncells;
    S.origin = in->cell_origin;
    for (int k = 0; k < 3; ++k) S.dim[k] = in->dim[k];
    const float cf = (float)in->cutoff;
    S.cut2f_pair = cf * cf;
    S.cut2f_self = (float)(in->cutoff * in->cutoff);
    if (sizeof(T) == sizeof(float)) {
        S.cut2_pair = (T)(cf * cf);
        S.cut2_self = (T)(float)(in->cutoff * in->cutoff);
    } else {
        S.cut2_pair = (T)(in->cutoff * in->cutoff);
        S.cut2_self = S.cut2_pair;
    }
    S.ntypes = in->ntypes;
    for (int t = 0; t < in->ntypes; ++t) S.radius.push_back((T)in->radius[t]);
    S.pot_of_pair = in->pot_of_pair;
    S.dpd_of_pair = in->dpd_of_pair;
    for (int q = 0; q < in->npots; ++q) {
        Pot<T> p;
        p.kind = in->pot_kind[q];
        p.flags = in->pot_flags[q];
        p.n = in->pot_n[q];
        for (int k = 0; k < 3; ++k) p.alpha[k] = (T)in->pot_alpha[3 * q + k];
        p.a = (T)in->pot_abr[3 * q];
        p.b = (T)in->pot_abr[3 * q + 1];
        p.r0p1 = (T)in->pot_abr[3 * q + 2];
        p.c = in->coef + in->pot_coef_off[q];
        p.dpd_alpha = (T)in->dpd[4 * q];
        p.dpd_gamma = (T)in->dpd[4 * q + 1];
        p.dpd_sigma = (T)in->dpd[4 * q + 2];
        p.dpd_delta = (T)in->dpd[4 * q + 3];
        S.pots.push_back(p);
    }
    for (int t = 0; t < 3 * in->ntypes; ++t) S.body.push_back(in->body ? (T)in->body[t] : (T)0);
    S.xf.assign(in->xrel, in->xrel + 3 * (size_t)in->N);
    double h[3];
    int cdim[3] = {in->cdim[0], in->cdim[1], in->cdim[2]};
    for (int k = 0; k < 3; ++k) h[k] = in->dim[k] / cdim[k];
    S.bias = (float)std::sqrt(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]);
    S.dscale = (float)32767 / (2 * S.bias);
    S.dmaxdist = (int)(2 + S.dscale * ((float)in->cutoff + 2 * 0.0f));
    S.prune = in->pruning != 2;
    for (int q = 0; q < 13; ++q)
        for (int k = 0; k < 3; ++k) S.axes[q][k] = (float)kCellShift[q][k];
    return run(S, in->tasks, in->ntasks, f_out, epot_out, counts, vir);
}

}  // namespace

extern "C" int orc_nonbond_virial(int precision, const OrcInput *in, double *f_out, double *epot_out,
                                  long long *counts, double *virial_out) {
    if (!in || !f_out || !epot_out) return -1;
    if (precision == 32) return build_and_run<float>(in, f_out, epot_out, counts, virial_out);
    if (precision == 64) return build_and_run<double>(in, f_out, epot_out, counts, virial_out);
    return -1;
}

extern "C" int orc_nonbond(int precision, const OrcInput *in, double *f_out, double *epot_out, long long *counts) {
    if (!in || !f_out || !epot_out) return -1;
    if (precision == 32) return build_and_run<float>(in, f_out, epot_out, counts, nullptr);
    if (precision == 64) return build_and_run<double>(in, f_out, epot_out, counts, nullptr);
    return -1;
}
