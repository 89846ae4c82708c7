/*
 * Device-side data layout and helpers shared by the engine kernels.
 *
 * HBM layout (all arrays in slot order = sorted by cell, ascending particle id
 * inside a cell):
 *   pos[slot]   float4  (x, y, z relative to the cell origin, w = type id bits)
 *   vel[slot]   float4  (vx, vy, vz, w = particle id bits)
 *   force[slot] float4  (fx, fy, fz, w unused)
 *   cell_of[slot] int
 * Cells: cell_start[c], cell_count[c]; per cell a CSR list of neighbour
 * entries (neighbour cell, role, float shift) derived from the reference's
 * cell-pair task list. The kernels in this translation unit are compiled
 * without FMA contraction so that every per-pair and per-particle operation
 * rounds exactly as the reference's scalar FP32/FP64 code does.
 */
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace mxg {

constexpr int kChunk = 8;           // floats per table interval
constexpr int kBucket = 32;         // movers per cell per step kept in the cell's bucket (more go to the overflow list)
constexpr int kChunkShift = 8;      // the re-binning's net mover counts per chunk of 256 consecutive cells
constexpr int kScatterWarps = 8;    // re-binning: cells (one warp each) per block
constexpr int kMaxTypes = 64;       // types per engine
constexpr int kWarpsPerBlock = 4;   // force kernel: warps (work items) per block
constexpr int kMaxCellParts = 8;    // force work items per cell at most
constexpr int kOrderMaxItems = 32768;  // work items the occupancy ordering handles at most

/* neighbour-entry roles, relative to the reference's (flipped) cell pair */
enum : int { kRoleSelf = 0, kRoleFirst = 1, kRoleSecond = 2 };

/* cell flags (space_cell.h:48-82) */
enum : unsigned {
    kCellActiveTop = 1u << 5,
    kCellActiveBottom = 1u << 6,
    kCellActiveLeft = 1u << 7,
    kCellActiveRight = 1u << 8,
    kCellActiveFront = 1u << 9,
    kCellActiveBack = 1u << 10,
    kCellActiveAny = (1u << 5) | (1u << 6) | (1u << 7) | (1u << 8) | (1u << 9) | (1u << 10),
};

/* boundary kinds */
enum : unsigned { kBcVelocity = 1u << 0, kBcPeriodic = 1u << 1, kBcFreeslip = 1u << 2 };

/* status word bits */
enum : unsigned {
    kStatusTooFast = 1u << 0,
    kStatusNonFinite = 1u << 2,
};

/* device-side load (engine_load): staging arrays by particle id */
struct LoadView {
    const double *x;         // [3n] global positions
    const float *v;          // [3n] velocities, or null: keep the current ones
    const int *type_of_id;
    const int *rep_of_id;
    float4 *xr;              // cell-relative position, w = type bits
    float4 *vel;             // velocity, w = id bits
    int *cell;               // destination cell, -1 outside the replica's box
    int *fill;               // per cell: particles placed so far
    int *ids;                // slot -> id, before the per-cell ordering
    int *err;                // set when a particle lies outside its box
    const int *slot_now;     // current slot of each id (velocities kept when v is null)
    int n;
};

struct DevPot {          // one per potential, 64 B
    int kind;            // 0 table, 1 DPD
    unsigned flags;
    int n;
    int coef_off;        // float offset into the coefficient pool
    float alpha0, alpha1, alpha2;
    float a, b, r0_plusone;
    float dpd_alpha, dpd_gamma, dpd_sigma, dpd_delta;  // delta = 1/sqrt(dt) as the reference keeps it
    float a2;            // a*a (float)
    float pad;
};

struct DevType {
    double imass;
    double mass;
    float radius;
    int dynamics;        // 0 Newtonian, 1 overdamped
    unsigned flags;      // frozen bits
    float fx, fy, fz;    // constant body force
    int has_force;
    int pad;
    // other single-body force (MxForce.cpp:308-419): 0 none, 2 Berendsen, 3 random, 4 friction
    int sb_kind;
    int sb_steps;        // random/friction: redraw interval in steps, ceil(duration / dt)
    float sb_a, sb_b, sb_c, sb_pad;  // Berendsen: 1/tau; random: mean, std; friction: coef, mean, std
    double target;       // Berendsen: the type's target temperature
    int bpot[6];         // wall potential per face (left, right, front, back, bottom, top), -1 if none
    unsigned wall_mask;  // active-cell bits of the faces with a wall potential
    int large;           // radius > cutoff: the reference's PARTICLE_LARGE (static, interacts with all)
    int cpot;            // potential between this type and the cuboids (engine_add_cuboid_potential), -1 if none
    int pad3;
};

/* A static cuboid (MxCuboid, MxCuboid.hpp; a body with a box shape): centre, half extents,
 * orientation and its inverse as quaternions (x, y, z, w), its axis-aligned bounding box as
 * MxCuboid_UpdateAABB (MxCuboid.cpp:190-221) forms it, and its replica. */
struct DevCuboid {
    float pos[3];
    float size[3];
    float q[4];
    float qi[4];
    float lo[3], hi[3];
    int rep;
    int pad;
};

struct DevSpace {        // one per replica
    double origin[3];    // the box's lower corner
    double hd[3];        // cell size (double, as space.h keeps it)
    double ih[3];        // 1 / cell size (double)
    float h[3], h2[3];   // float(h), float(2h)
    float maxv[3], maxv2[3], maxx[3], maxx2[3];
    float dt;
    float cut2_pair, cut2_self;
    float cut2w_pair, cut2w_self;  // the candidate pass's widened cutoffs (covers the one rounding it skips)
    int cdim[3];
    int cell_offset;
    int ncells;
    int pot_offset;      // offset of this replica's type-pair matrix
    unsigned bc_kind[6];
    float bc_vel[6][3];
    float bc_restore[6];
    unsigned rng_mode;   // 0: reference DPD random term (xi = 1), 1: Philox
    int prune;           // bit 0: per-pair projection test, bit 1: cell-pair exit test (runner_dopair)
    float sort_bias;     // |h| (runner_dopair.cpp:132)
    float sort_dscale;   // SHRT_MAX / (2 |h|)
    int dmaxdist;        // 2 + dscale * cutoff
    int pad2;
    double dt_d;         // the engine's dt in double (species integration)
    double cutoff_d;     // the space's cutoff in double (flux weight)
};

/* normalised sort directions of the 13 sort lists (space_cell.cpp:82-96) */
struct SortAxes {
    float n[13][3];
};

struct DevBond {
    int i, j;            // particle ids
    int pot;             // potential index
    int pad;
    double dissociation;
};

struct DevAngle {
    int i, j, k;         // particle ids; j is the vertex
    int pot;             // potential index (a table in cos(theta))
};

struct DevDihedral {
    int i, j, k, l;      // particle ids; the k end carries the balancing force
    int pot;             // potential index (a table in cos(phi))
    int pad[3];
};

/* Bonded interactions, CSR by particle id. bond_list holds bond indices;
 * angle_list holds angle * 4 + role (0: i, 1: j, 2: k); dihedral_list holds
 * dihedral * 4 + role (0: i, 1: j, 2: k, 3: l). */
struct BondedView {
    const int2 *excl;        // exclusions (i <= j): the pair potential taken back
    const int *excl_off;
    const int *excl_list;    // exclusion * 2 + role (0: i, 1: j)
    const DevBond *bonds;
    unsigned *bond_flags;
    const int *bond_off;
    const int *bond_list;
    const DevAngle *angles;
    const int *angle_off;
    const int *angle_list;
    const DevDihedral *dihedrals;
    const int *dihedral_off;
    const int *dihedral_list;
    const int *slot_of_id;
    double *e_slot;      // per slot: bonded energy of the last pass
};

struct DevFlux {         // one flux entry of a type pair's flux list (MxFlux, Flux.hpp)
    int kind;            // 0 Fick, 1 secrete, 2 uptake
    int ta, tb;          // the entry's type pair (a: loses, b: gains for a positive q)
    int ia, ib;          // species index in a's and b's state vectors
    float k, decay, target;
};

/* Species state vectors and fluxes, by particle id (values and rates are
 * smax floats per particle; a type uses the first nspec of them). */
struct SpeciesView {
    float *value;            // [id * smax + k]
    float *rate;             // [id * smax + k]: flux sum not yet integrated
    const int *nspec;        // per type
    const unsigned *flags;   // per type and species: bit 2 = constant (not integrated)
    const int *flux_off;     // per type pair [ntypes*ntypes + 1]: the pair's entries
    const DevFlux *flux;
    const int *fx_off;       // per cell: full neighbour list (SELF, FIRST and SECOND entries)
    const int *fx_cell;
    const float4 *fx_shift;  // xyz shift of the task, w = role | sort id << 2 | key shift << 8
    int smax;
};

struct EngineView {      // everything a kernel needs, passed by value
    const float4 *pos;
    const float4 *vel;
    float4 *force;
    const int *cell_of;
    const int *cell_start;
    const int *cell_count;
    const int *cell_rep;
    const unsigned *cell_flags;
    const int *nb_off;
    const int *nb_cell;
    const float4 *nb_shift;  // xyz shift, w = bits of role | sid << 2 | dnshift << 8
    const DevPot *pots;
    const float *coef;
    const int *pot_idx;      // per replica: [ntypes*ntypes] potential index or -1
    const int *pot_idx2;     // per replica: second (summed) potential index or -1; null if none
    const DevType *types;
    const DevSpace *spaces;
    int ntypes;
    int ncells;
    int nparts;
    const unsigned long long *step;  // device step counter
    const SortAxes *axes;
    int2 *sort_bounds;               // per cell and sort axis: (min key, max key)
    double *epot_cell;       // per force work item: nonbonded energy of the last force pass
    unsigned *status;
    unsigned long long *pair_stats;  // non-null only for the statistics launch
    double *virial_partials;         // non-null only for the virial launch: [warp][6]
    int has_sb;                      // some type has a Berendsen, random or friction force
    const double *type_ke;           // per type: summed kinetic energy of the state (Berendsen)
    const float4 *persist;           // per particle id: persistent random force (random, friction)
    const int *nb_rev;       // FIRST entries: the pair's plane in the neighbour's received sums
    const int *sec_count;    // per cell: SECOND entries, i.e. planes of received sums
    const int *cell_planes;  // per cell: received planes plus own-side planes of its later work items
    float4 *planes;          // [plane][slot] neighbour-side force sums of once-evaluated pairs
    double *body_e;          // per slot: wall and large-particle energy of the last pass; null when neither exists
    const float4 *body_f;    // per slot: wall and large-particle force of the pass; null when neither exists
    const float4 *large_x;   // large particles: position relative to the replica origin, w = type
    const float4 *large_v;   // large particles: velocity, w = id
    const int *large_rep;    // large particles: replica
    const int *large_pot;    // per replica [ntypes*ntypes]: potential of a (normal, large) type pair, or -1
    int nlarge;
    const int4 *items;       // force work items: (cell, first entry, end entry, part)
    int *item_ctr;           // [0] next work item, [1] warps done (dynamic fetch; zero between launches)
    int *item_order;         // items by decreasing cell occupancy (split cells only), else null
    int dpd_pure;            // every pair potential is DPD with the reference's random term: DPD-only kernel
    int force_variant;       // the force kernel's tile shape (see Tile), chosen by the autotuner
    int nitems;
    const DevCuboid *cuboids;  // static cuboids (all replicas)
    int ncuboids;
    const float4 *dpd_pair;  // DPD-only kernel, per replica and type pair: (rc, alpha, gamma, sigma delta),
                             // (a^2, a, 1/rc, alpha + sigma delta); null otherwise
    int *ovf_list;           // movers beyond their destination's bucket this step: old slot (capacity nparts)
    int *ovf_count;          // entries of ovf_list (re-armed by the re-binning launch)
    int *chunk_delta;        // per chunk of 1 << kChunkShift cells: movers in minus movers out this step
};

#ifdef __CUDACC__
/* ---- exact-rounding helpers (the file is compiled with -fmad=false too) ---- */
__device__ __forceinline__ float dot3_rn(float x, float y, float z) {
    return __fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z));
}

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), counter-based. */
__device__ __forceinline__ uint4 philox4x32(uint4 c, uint2 k) {
    const unsigned M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const unsigned hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
        const unsigned hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += W0;
        k.y += W1;
    }
    return c;
}

/* The reference's projection key of a particle along sort direction n
 * (runner_dosort.cpp:133-136): (unsigned)(dscale * (bias + x.n)) in FP32. */
__device__ __forceinline__ int sort_key(float x, float y, float z, const float *n, float bias, float dscale) {
    const float proj = __fadd_rn(__fadd_rn(__fadd_rn(bias, __fmul_rn(x, n[0])), __fmul_rn(y, n[1])), __fmul_rn(z, n[2]));
    return (int)(unsigned)__fmul_rn(dscale, proj);
}

/* sort_key along the reference's sort direction sid (runner_dosort.cpp's 13 normalised cell
 * shifts, the same FP32 values as SortAxes holds); with sid known at compile time the direction
 * is three immediates. */
__device__ __forceinline__ int sort_key_sid(int sid, float x, float y, float z, float bias, float dscale) {
    constexpr float a = (float)5.773502691896258e-01, b = (float)7.071067811865475e-01;
    float n[3];
    switch (sid) {
        case 0: n[0] = a; n[1] = a; n[2] = a; break;
        case 1: n[0] = b; n[1] = b; n[2] = 0.f; break;
        case 2: n[0] = a; n[1] = a; n[2] = -a; break;
        case 3: n[0] = b; n[1] = 0.f; n[2] = b; break;
        case 4: n[0] = 1.f; n[1] = 0.f; n[2] = 0.f; break;
        case 5: n[0] = b; n[1] = 0.f; n[2] = -b; break;
        case 6: n[0] = a; n[1] = -a; n[2] = a; break;
        case 7: n[0] = b; n[1] = -b; n[2] = 0.f; break;
        case 8: n[0] = a; n[1] = -a; n[2] = -a; break;
        case 9: n[0] = 0.f; n[1] = b; n[2] = b; break;
        case 10: n[0] = 0.f; n[1] = 1.f; n[2] = 0.f; break;
        case 11: n[0] = 0.f; n[1] = b; n[2] = -b; break;
        default: n[0] = 0.f; n[1] = 0.f; n[2] = 1.f; break;
    }
    return sort_key(x, y, z, n, bias, dscale);
}

/* Cell coordinates of global cell c in its replica's grid. */
__device__ __forceinline__ void cell_loc(const DevSpace &S, int c, int loc[3]) {
    const int l = c - S.cell_offset;
    loc[0] = l / (S.cdim[1] * S.cdim[2]);
    loc[1] = (l / S.cdim[2]) % S.cdim[1];
    loc[2] = l % S.cdim[2];
}

/* The bonded code's neighbour-cell shift (bond.cpp:163-170, angle.cpp:155-168):
 * a cell difference of more than one is a periodic wrap. */
__device__ __forceinline__ int wrap_shift(int d) { return d > 1 ? -1 : (d < -1 ? 1 : d); }

/* x + shift*h formed in double and rounded to float, as the reference writes
 * the double product into a float position. */
__device__ __forceinline__ float shifted(float x, int sh, double h) {
    return (float)__dadd_rn((double)x, __dmul_rn(h, (double)sh));
}

/* The bond vector d = x_i - x_j of bond_eval (bond.cpp:163-178): x_i moved into
 * x_j's cell frame by the wrapped cell shift, in the reference's rounding. */
__device__ __forceinline__ void bond_vector(const DevSpace &S, int ci, int cj, const float4 &xi, const float4 &xj,
                                            float d[3]) {
    int loci[3], locj[3];
    cell_loc(S, ci, loci);
    cell_loc(S, cj, locj);
    const float xiv[3] = {xi.x, xi.y, xi.z}, xjv[3] = {xj.x, xj.y, xj.z};
    for (int q = 0; q < 3; ++q) d[q] = __fsub_rn(shifted(xiv[q], wrap_shift(loci[q] - locj[q]), S.hd[q]), xjv[q]);
}

/* uniform in (0,1) from 32 random bits */
__device__ __forceinline__ float u01(unsigned x) { return ((float)(x >> 8) + 0.5f) * (1.0f / 16777216.0f); }

/* Three normal deviates from one Philox draw (Box-Muller on two pairs). */
__device__ __forceinline__ void philox_normal3(unsigned long long step, unsigned a, unsigned b, float &g0,
                                               float &g1, float &g2) {
    const uint4 r = philox4x32(make_uint4(a, b, (unsigned)step, (unsigned)(step >> 32)), make_uint2(0x4d584731u, 0x5f524e44u));
    const float u0 = u01(r.x), u1 = u01(r.y), u2 = u01(r.z), u3 = u01(r.w);
    const float m0 = sqrtf(-2.0f * logf(u0)), m1 = sqrtf(-2.0f * logf(u2));
    float s0, c0, s1, c1;
    sincospif(2.0f * u1, &s0, &c0);
    sincospif(2.0f * u3, &s1, &c1);
    g0 = m0 * c0;
    g1 = m0 * s0;
    g2 = m1 * c1;
}

/* Zero-mean, unit-variance DPD random number for the unordered pair (a, b). */
__device__ __forceinline__ float philox_pair_xi(unsigned long long step, unsigned lo, unsigned hi) {
    const uint4 r = philox4x32(make_uint4(lo, hi, (unsigned)step, (unsigned)(step >> 32)), make_uint2(0x44504431u, 0x58495f31u));
    return 1.7320508075688772f * (2.0f * u01(r.x) - 1.0f);
}


/* Table evaluation with potential_eval_ex semantics (potential_eval.hpp:106-161):
 * returns false when out of range. ri, rj are the particle radii. */
__device__ __forceinline__ bool table_eval_ex(const DevPot &p, const float *__restrict__ coef, float ri, float rj,
                                              float r2, float &e, float &f) {
    float r = sqrtf(r2);
    const float ro = r < 1.19209290e-7f ? 1.19209290e-7f : r;
    r = r < p.a ? p.a : r;
    if (p.flags & (1u << 11))
        r = __fdiv_rn(r, __fadd_rn(ri, rj));
    else if (p.flags & (1u << 12))
        r = __fadd_rn(__fsub_rn(r, __fadd_rn(ri, rj)), p.r0_plusone);
    const float t = __fadd_rn(p.alpha0, __fmul_rn(r, __fadd_rn(p.alpha1, __fmul_rn(r, p.alpha2))));
    const unsigned ind = (unsigned)fmaxf(0.0f, t);
    if (r > p.b || ind > (unsigned)p.n) return false;
    const float4 *c4 = reinterpret_cast<const float4 *>(coef + p.coef_off + ind * kChunk);
    const float4 c0 = __ldg(c4), c1 = __ldg(c4 + 1);
    const float x = __fmul_rn(__fsub_rn(r, c0.x), c0.y);
    float ee = __fadd_rn(__fmul_rn(c0.z, x), c0.w);
    float eff = c0.z;
    eff = __fadd_rn(__fmul_rn(eff, x), ee); ee = __fadd_rn(__fmul_rn(ee, x), c1.x);
    eff = __fadd_rn(__fmul_rn(eff, x), ee); ee = __fadd_rn(__fmul_rn(ee, x), c1.y);
    eff = __fadd_rn(__fmul_rn(eff, x), ee); ee = __fadd_rn(__fmul_rn(ee, x), c1.z);
    eff = __fadd_rn(__fmul_rn(eff, x), ee); ee = __fadd_rn(__fmul_rn(ee, x), c1.w);
    e = ee;
    f = __fdiv_rn(__fmul_rn(eff, c0.y), ro);
    return true;
}

/* Table evaluation with potential_eval semantics (no range check, no
 * radius shift; potential_eval.hpp:67-104), used by bonds. */
__device__ __forceinline__ void table_eval(const DevPot &p, const float *__restrict__ coef, float r2, float &e,
                                           float &f) {
    const float r = sqrtf(r2);
    const float t = __fadd_rn(p.alpha0, __fmul_rn(r, __fadd_rn(p.alpha1, __fmul_rn(r, p.alpha2))));
    // the reference indexes unchecked; r is clamped to [a, b] by the caller, so
    // ind <= n except for rounding at r = b, which is clamped here
    const int ind = min((int)fmaxf(0.0f, t), p.n);
    const float4 *c4 = reinterpret_cast<const float4 *>(coef + p.coef_off + ind * kChunk);
    const float4 c0 = __ldg(c4), c1 = __ldg(c4 + 1);
    const float x = __fmul_rn(__fsub_rn(r, c0.x), c0.y);
    float ee = __fadd_rn(__fmul_rn(c0.z, x), c0.w);
    float eff = c0.z;
    eff = __fadd_rn(__fmul_rn(eff, x), ee); ee = __fadd_rn(__fmul_rn(ee, x), c1.x);
    eff = __fadd_rn(__fmul_rn(eff, x), ee); ee = __fadd_rn(__fmul_rn(ee, x), c1.y);
    eff = __fadd_rn(__fmul_rn(eff, x), ee); ee = __fadd_rn(__fmul_rn(ee, x), c1.z);
    eff = __fadd_rn(__fmul_rn(eff, x), ee); ee = __fadd_rn(__fmul_rn(ee, x), c1.w);
    e = ee;
    f = __fdiv_rn(__fmul_rn(eff, c0.y), r);
}

/* Table evaluation with potential_eval_r semantics (potential_eval.hpp:180-207):
 * the table at r itself, f = dV/dr (not divided by r). Used by angles with
 * r = cos(theta) clamped to [a, b] by the caller; the index is clamped to n. */
__device__ __forceinline__ void table_eval_r(const DevPot &p, const float *__restrict__ coef, float r, float &e,
                                             float &f) {
    const float t = __fadd_rn(p.alpha0, __fmul_rn(r, __fadd_rn(p.alpha1, __fmul_rn(r, p.alpha2))));
    const int ind = min((int)fmaxf(0.0f, t), p.n);
    const float4 *c4 = reinterpret_cast<const float4 *>(coef + p.coef_off + ind * kChunk);
    const float4 c0 = __ldg(c4), c1 = __ldg(c4 + 1);
    const float x = __fmul_rn(__fsub_rn(r, c0.x), c0.y);
    float ee = __fadd_rn(__fmul_rn(c0.z, x), c0.w);
    float eff = c0.z;
    eff = __fadd_rn(__fmul_rn(eff, x), ee); ee = __fadd_rn(__fmul_rn(ee, x), c1.x);
    eff = __fadd_rn(__fmul_rn(eff, x), ee); ee = __fadd_rn(__fmul_rn(ee, x), c1.y);
    eff = __fadd_rn(__fmul_rn(eff, x), ee); ee = __fadd_rn(__fmul_rn(ee, x), c1.z);
    eff = __fadd_rn(__fmul_rn(eff, x), ee); ee = __fadd_rn(__fmul_rn(ee, x), c1.w);
    e = ee;
    f = __fmul_rn(eff, c0.y);
}

#endif  // __CUDACC__

}  // namespace mxg
