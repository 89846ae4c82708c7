/* Adjoint (vector-Jacobian product) of one engine step (mxg_adjoint.cu). */
#pragma once
#include "mxg_device.cuh"

namespace mxg {

constexpr int kMaxGradSlots = 16;  // parameter-gradient slots per engine
constexpr int kMaxPotGrads = 4;    // differentiated parameters per potential

enum : int { kGradTable = 0, kGradShift = 1, kGradDpdAlpha = 2, kGradDpdGamma = 3, kGradDpdSigma = 4 };

struct DevPotGrad {      // the differentiated parameters of one potential
    int n;
    int mode[kMaxPotGrads];      // kGrad*
    int slot[kMaxPotGrads];      // gradient slot the parameter adds to
    int coef_off[kMaxPotGrads];  // kGradTable: offset of dV/dtheta's table in the derivative pool
};

struct AdjointView {
    float4 *lam_x, *lam_v;       // [id] adjoints of positions and velocities (in: after the step; out: before)
    float4 *w, *gx, *gv;         // [slot] scratch: force adjoint and the partial sums
    const DevPotGrad *pot_grad;  // per potential
    const float *dcoef;          // derivative tables' coefficient pool
    double *partials;            // [kMaxGradSlots][item] FP64 parameter sums of the pair terms
    double *bond_partials;       // [block][kMaxGradSlots] FP64 parameter sums of the bond terms
    int nslots;
    // the pair terms' work items: (cell, first entry, end entry, part), kVjpParts per cell; part 0
    // adds its own-side sums to gx / gv, part p > 0 writes them to plane p - 1 of pgx / pgv
    const int4 *items;
    int nitems;
    int *item_ctr;               // [0] next item, [1] warps done (zero between launches)
    float4 *pgx, *pgv;           // [part - 1][slot]
};

void launch_positions(const EngineView &v, float4 *x_out, float4 *v_out, cudaStream_t st);
/* Smoothed pair histogram of types (ta, tb) and/or its gradient (see mxg_rdf). */
int launch_rdf(const float4 *x, int n, const double *box, int ta, int tb, int nbins, double dr, double sigma,
               unsigned long long *hist, const double *coef, float4 *grad, cudaStream_t st);
/* Up to kCopyMax device-to-device copies of whole 4-byte words in one launch (the sections of a
 * state snapshot): section k copies words[k] words from src[k] to dst[k]. */
constexpr int kCopyMax = 12;
struct CopySections {
    const unsigned *src[kCopyMax];
    unsigned *dst[kCopyMax];
    unsigned long long words[kCopyMax];
    int n;
};
void launch_copy_sections(const CopySections &c, cudaStream_t st);
/* parts per cell of the pair terms' work items (contiguous groups of the cell's entries) */
int vjp_parts();
/* blocks of the bond-term kernel (each writes kMaxGradSlots partial sums) */
int adjoint_bond_blocks(int num_sms);
void configure_adjoint_kernels();
/* Enqueues the VJP of one step at the engine's current state, whose forces v.force must hold
 * (with the bond pass of that state applied when bv is not null: its flags then mark the bonds
 * that acted in the step). */
void launch_vjp_step(const EngineView &v, const AdjointView &a, const BondedView *bv, int num_sms, double *grad,
                     cudaStream_t st);

}  // namespace mxg
