/*
 * Force-and-step kernels for sm_100a.
 *
 *   force_kernel      nonbonded cell-pair forces (tables, DPD), single-body
 *                     forces, per-cell FP64 energy. One warp per cell.
 *   bonded_kernel     harmonic/table bonds with dissociation flags, angles.
 *   integrate_kernel  forward Euler (Newtonian / overdamped), speed clamp,
 *                     wall reflection, relocation; counts the next binning.
 *   scatter_kernel    stable re-binning (ascending id inside each cell); each
 *                     cell's new start from chunked net mover counts.
 *   energy kernels    FP64 reductions of potential and kinetic energy.
 *
 * Compiled with -fmad=false: every FP32/FP64 operation on the pair, bond and
 * integrator paths rounds separately, in the reference's order, so per-pair
 * results and all integer outcomes (cell ids, break flags) match the
 * reference's scalar CPU code bit for bit; only the order of the per-particle
 * force sums differs.
 */
#include "mxg_device.cuh"
#include "mxg_kernels.h"

namespace mxg {

namespace {

constexpr unsigned kFull = 0xffffffffu;

}  // namespace

/* ------------------------------------------------------------------------ */
/* sort-key bounds                                                           */
/* ------------------------------------------------------------------------ */

/*
 * Per cell and per sort direction, the smallest and largest projection key of
 * its particles (runner_dosort.cpp:133-141 computes the keys; runner_dopair
 * reads the largest key of its first cell and the smallest of its second,
 * runner_dopair.cpp:167-171). Called by one warp for one cell.
 */
__device__ __forceinline__ void cell_sort_bounds(const float4 *__restrict__ pos, int start, int n, float bias,
                                                 float dscale, const SortAxes *axes, int2 *out) {
    const int lane = threadIdx.x & 31;
    if (n <= 32) {  // one particle per lane
        const bool live = lane < n;
        const float4 q = live ? pos[start + lane] : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int sid = 0; sid < 13; ++sid) {
            const int key = sort_key_sid(sid, q.x, q.y, q.z, bias, dscale);
            const int kmin = __reduce_min_sync(kFull, live ? key : 0x7fffffff);
            const int kmax = __reduce_max_sync(kFull, live ? key : -1);
            if (lane == 0) out[sid] = make_int2(kmin, kmax);
        }
        return;
    }
#pragma unroll
    for (int sid = 0; sid < 13; ++sid) {
        int kmin = 0x7fffffff, kmax = -1;
        for (int k = lane; k < n; k += 32) {
            const float4 q = pos[start + k];
            const int key = sort_key_sid(sid, q.x, q.y, q.z, bias, dscale);
            kmin = min(kmin, key);
            kmax = max(kmax, key);
        }
        kmin = __reduce_min_sync(kFull, kmin);
        kmax = __reduce_max_sync(kFull, kmax);
        if (lane == 0) out[sid] = make_int2(kmin, kmax);
    }
}

/* Key bounds of every cell of the current state, for states that did not come
 * from the re-binning pass (which computes them itself). One warp per cell. */
__global__ void sort_bounds_kernel(EngineView v) {
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < v.ncells; c += warps) {
        const int n = v.cell_count[c];
        if (n == 0) continue;
        const DevSpace &S = v.spaces[v.cell_rep[c]];
        if (!(S.prune & 2)) continue;
        cell_sort_bounds(v.pos, v.cell_start[c], n, S.sort_bias, S.sort_dscale, v.axes, v.sort_bounds + c * 13);
    }
}

/* ------------------------------------------------------------------------ */
/* nonbonded forces                                                          */
/* ------------------------------------------------------------------------ */

/*
 * One warp per work item (a cell with a group of its entries; warps take items
 * from a device counter). Every cell pair is evaluated once, by the
 * cell that is FIRST in the reference's flipped pair (runner_dopair.cpp:91-340);
 * the cell's own pairs (runner_doself, :446-682) are evaluated from both sides.
 * The warp stages up to kOwn of the cell's particles and then, region by
 * region, up to kCap particles (the tile shape, Tile) of its SELF and FIRST neighbour entries (whole
 * entries where they fit) in shared memory. Each own particle is tested
 * against the staged neighbours one per lane, 32 candidates per step, for the
 * cutoff, the reference's pruning and the existence of a potential (pass 1).
 * Interacting candidates are appended, in candidate order, to a per-warp queue
 * with a ballot; every 32 queued pairs are evaluated with one pair per lane
 * (pass 2), so the expensive pair arithmetic runs with the warp's lanes full.
 *
 * The queue is ordered by own particle: the own-side sums of a batch are formed
 * by a segmented shuffle scan and added to the particle's force in shared
 * memory by the segment's last lane; the neighbour-side contributions (the
 * exact negations) are added to per-neighbour sums one segment after another
 * (inside a segment the neighbours are distinct). At the end of a region the
 * neighbour sums are stored in the plane that the neighbour cell reserves for
 * this pair; after the pass, combine_kernel adds each particle's planes in
 * plane order. Every sum has a fixed order: no atomics, deterministic results.
 *
 * FIRST entries stage their shift beside each neighbour particle, so every
 * candidate computes d = (x_i - s) - x_j, the reference's dx for the pair (or
 * its exact negation for a self pair whose first particle is j): r2 and the
 * per-pair force are bit-identical to the reference's.
 */
// kPure: every pair potential is DPD and the random term is the reference's (no Philox):
// the table and Philox code is left out of the kernel (a smaller instruction footprint)
template <bool kDPD, bool kPure = false>
__device__ __forceinline__ void pair_contribution(const EngineView &v, const DevPot &p, int role, bool i_first,
                                                  float dx, float dy, float dz, float r2, float radi, float radj,
                                                  const float4 &vi, const float4 &vj, unsigned rng_mode,
                                                  float &cx, float &cy, float &cz, float &pe, bool &counted) {
    cx = cy = cz = 0.f;
    pe = 0.f;
    counted = false;
    if (kDPD && (kPure || p.kind == 1)) {
        // dpd_eval (dpd_eval.hpp:21-69), in the reference's orientation
        const float r_first = i_first ? radi : radj;
        const float r_second = i_first ? radj : radi;
        const bool shifted = p.flags & (1u << 12);
        const float cutoff = shifted ? __fadd_rn(__fadd_rn(p.b, r_first), r_second) : p.b;
        if (r2 > __fmul_rn(cutoff, cutoff)) return;
        const float r = sqrtf(r2);
        const float ex = __fdiv_rn(dx, r), ey = __fdiv_rn(dy, r), ez = __fdiv_rn(dz, r);
        float wx, wy, wz;  // v_first - v_second
        if (i_first) {
            wx = __fsub_rn(vi.x, vj.x);
            wy = __fsub_rn(vi.y, vj.y);
            wz = __fsub_rn(vi.z, vj.z);
        } else {
            wx = __fsub_rn(vj.x, vi.x);
            wy = __fsub_rn(vj.y, vi.y);
            wz = __fsub_rn(vj.z, vi.z);
        }
        const float sr = shifted ? __fsub_rn(__fsub_rn(r, r_first), r_second) : r;
        const float oc = sr < 0.f ? 1.f : __fsub_rn(1.0f, __fdiv_rn(sr, cutoff));
        const float fc = __fmul_rn(p.dpd_alpha, oc);
        const float od = __fmul_rn(oc, oc);
        const float ev = __fadd_rn(__fadd_rn(__fmul_rn(ex, wx), __fmul_rn(ey, wy)), __fmul_rn(ez, wz));
        const float fd = __fmul_rn(__fmul_rn(-p.dpd_gamma, od), ev);
        float fr = __fmul_rn(__fmul_rn(p.dpd_sigma, oc), p.dpd_delta);
        if (!kPure && rng_mode) {
            const unsigned idi = __float_as_uint(vi.w), idj = __float_as_uint(vj.w);
            fr = fr * philox_pair_xi(*v.step, idi < idj ? idi : idj, idi < idj ? idj : idi);
        }
        const float f = __fadd_rn(__fadd_rn(fc, fd), fr);
        // first particle gets +f e, second -f e; the reference tabulates zero energy for DPD
        const float sg = i_first ? 1.0f : -1.0f;
        cx = sg * __fmul_rn(f, ex);
        cy = sg * __fmul_rn(f, ey);
        cz = sg * __fmul_rn(f, ez);
        counted = i_first;
    } else if (!kPure) {
        float e, f;
        if (!table_eval_ex(p, v.coef, i_first ? radi : radj, i_first ? radj : radi, r2, e, f)) return;
        // first particle gets -f dx, second +f dx
        const float sg = i_first ? -1.0f : 1.0f;
        cx = sg * __fmul_rn(f, dx);
        cy = sg * __fmul_rn(f, dy);
        cz = sg * __fmul_rn(f, dz);
        if (i_first) pe = e;
        counted = i_first;
    }
}

/*
 * Wall potentials of one particle (boundary_eval, boundary_eval.hpp:124-223),
 * faces in the reference's order left, right, front, back, bottom, top: the
 * distance r to the face from the cell-relative position (r = x for a low
 * face, float(h - x) for a high one), kept when r <= b; r^2 < a (the
 * reference compares with a, not a^2) becomes a^2 along the face normal.
 * Tables: potential_eval_ex with the wall's radius 0, f -= f dx. DPD:
 * dpd_boundary_eval against the wall velocity, f += f e (energy 0).
 */
__device__ __noinline__ void boundary_forces(const EngineView &v, const DevSpace &S, unsigned cflags, const DevType &T, float radius,
                                const float4 &x, const float4 &u, float4 &f, double &epot) {
    const unsigned bits[6] = {kCellActiveLeft, kCellActiveRight, kCellActiveFront,
                              kCellActiveBack, kCellActiveBottom, kCellActiveTop};
    const float xr[3] = {x.x, x.y, x.z};
    for (int face = 0; face < 6; ++face) {
        if (!(cflags & bits[face]) || T.bpot[face] < 0) continue;
        const DevPot &p = v.pots[T.bpot[face]];
        const int ax = face >> 1;
        const bool high = face & 1;
        const float r = high ? (float)__dsub_rn(S.hd[ax], (double)xr[ax]) : xr[ax];
        if (!(r <= p.b)) continue;
        float dx[3] = {0.f, 0.f, 0.f};
        dx[ax] = high ? -r : r;
        float r2 = __fmul_rn(r, r);
        if (r2 < p.a) {
            r2 = __fmul_rn(p.a, p.a);
            dx[ax] = high ? -p.a : p.a;  // the face normal times a
        }
        if (p.kind == 1) {
            if (r2 > __fmul_rn(p.b, p.b)) continue;
            const float rr = sqrtf(r2);
            const float e[3] = {__fdiv_rn(dx[0], rr), __fdiv_rn(dx[1], rr), __fdiv_rn(dx[2], rr)};
            const float w[3] = {__fsub_rn(u.x, S.bc_vel[face][0]), __fsub_rn(u.y, S.bc_vel[face][1]),
                                __fsub_rn(u.z, S.bc_vel[face][2])};
            const float oc = __fsub_rn(1.0f, __fdiv_rn(rr, p.b));
            const float fc = __fmul_rn(p.dpd_alpha, oc);
            const float od = __fmul_rn(oc, oc);
            const float ev = __fadd_rn(__fadd_rn(__fmul_rn(e[0], w[0]), __fmul_rn(e[1], w[1])), __fmul_rn(e[2], w[2]));
            const float fd = __fmul_rn(__fmul_rn(-p.dpd_gamma, od), ev);
            const float fr = __fmul_rn(__fmul_rn(p.dpd_sigma, oc), p.dpd_delta);
            const float ff = __fadd_rn(__fadd_rn(fc, fd), fr);
            f.x = __fadd_rn(f.x, __fmul_rn(ff, e[0]));
            f.y = __fadd_rn(f.y, __fmul_rn(ff, e[1]));
            f.z = __fadd_rn(f.z, __fmul_rn(ff, e[2]));
        } else {
            float ee, ff;
            if (!table_eval_ex(p, v.coef, radius, 0.0f, r2, ee, ff)) continue;
            f.x = __fsub_rn(f.x, __fmul_rn(ff, dx[0]));
            f.y = __fsub_rn(f.y, __fmul_rn(ff, dx[1]));
            f.z = __fsub_rn(f.z, __fmul_rn(ff, dx[2]));
            epot += (double)ee;
        }
    }
}

/*
 * Interactions of one particle with the large particles of its replica
 * (particle_largecell_force, runner_dopair.cpp:342-434, run from
 * runner_doself for every particle): the particle's global FP32 position
 * x_rel + cell origin against each large particle's position, no cutoff other
 * than the potential's range, the pair evaluated as potential_eval_super_ex
 * with the particle first (a pair closer than the table minimum gets a Philox
 * direction of length a instead of the per-cell mt19937 draw). Only the
 * particle's side is applied: large particles are static.
 */
__device__ __noinline__ void large_forces(const EngineView &v, int s, const float4 &x, const float4 &u, float radius,
                                          float4 &f, double &epot) {
    const int c = v.cell_of[s];
    const int rep = v.cell_rep[c];
    const DevSpace &S = v.spaces[rep];
    const int l = c - S.cell_offset;
    const int loc[3] = {l / (S.cdim[1] * S.cdim[2]), (l / S.cdim[2]) % S.cdim[1], l % S.cdim[2]};
    const float xr[3] = {x.x, x.y, x.z};
    float pix[3];
    for (int k = 0; k < 3; ++k)
        pix[k] = (float)__dadd_rn((double)xr[k], __dadd_rn(S.origin[k], __dmul_rn((double)loc[k], S.hd[k])));
    const int ti = __float_as_int(x.w);
    for (int j = 0; j < v.nlarge; ++j) {
        if (v.large_rep[j] != rep) continue;
        const float4 xl = v.large_x[j];
        const int tj = __float_as_int(xl.w);
        const int q = v.large_pot[S.pot_offset + ti * v.ntypes + tj];
        if (q < 0) continue;
        const DevPot &p = v.pots[q];
        float dx = __fsub_rn(pix[0], xl.x), dy = __fsub_rn(pix[1], xl.y), dz = __fsub_rn(pix[2], xl.z);
        float r2 = dot3_rn(dx, dy, dz);
        const float4 ul = v.large_v[j];
        if (r2 < p.a2) {
            const unsigned idi = __float_as_uint(u.w), idj = __float_as_uint(ul.w);
            const unsigned lo = idi < idj ? idi : idj, hi = idi < idj ? idj : idi;
            float g0, g1, g2;
            philox_normal3(*v.step, lo, hi, g0, g1, g2);
            const float len = sqrtf(g0 * g0 + g1 * g1 + g2 * g2);
            const float sgn = idi == lo ? 1.0f : -1.0f;
            dx = sgn * g0 * p.a / len;
            dy = sgn * g1 * p.a / len;
            dz = sgn * g2 * p.a / len;
            r2 = p.a2;
        }
        float cx, cy, cz, pe;
        bool counted;
        pair_contribution<true>(v, p, kRoleFirst, true, dx, dy, dz, r2, radius, v.types[tj].radius, u, ul, S.rng_mode,
                                cx, cy, cz, pe, counted);
        f.x += cx;
        f.y += cy;
        f.z += cz;
        epot += (double)pe;
    }
}

/* A force-kernel tile shape: own particles staged at a time, neighbour particles staged
 * per region (a multiple of 32: the candidate pass keeps kCap / 32 of them per lane in
 * registers) and the resident blocks per SM its register budget allows. The autotuner
 * picks one per engine (force_variant); variant 0 is the default. */
template <int kOwnT, int kCapT, int kBlocksT>
struct Tile {
    static constexpr int kOwn = kOwnT, kCap = kCapT, kChunks = kCapT / 32, kBlocks = kBlocksT;
    // the ring queue of pairs (a power of two holding kCap + 31: one own particle queues at
    // most kCap pairs on top of fewer than 32 waiting ones)
    static constexpr int kQ = kCapT + 31 <= 128 ? 128 : 256;
    // a queued pair is (own index << 8 | staged index) in 16 bits; one own particle queues at most
    // kCap pairs on top of fewer than 32 waiting ones
    static_assert(kOwnT >= 1 && kOwnT <= 255 && kCapT % 32 == 0 && kCapT >= 32 && kCapT <= 256, "tile shape");
};
using Tile0 = Tile<32, 96, 5>;
using Tile1 = Tile<32, 64, 6>;
using Tile2 = Tile<64, 96, 5>;
using Tile3 = Tile<32, 128, 4>;
constexpr int kForceVariants = 4;

constexpr int kEnt = 32;            // neighbour entries cached at a time

/* 16-byte asynchronous copy from global to shared memory (cp.async, cached in L1) and the
 * wait for every copy this thread has issued. */
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

template <bool kDPD, class TS>
struct ForceSmem {
    static constexpr int kOwn = TS::kOwn, kCap = TS::kCap;
    float4 nb_x[kCap];              // neighbour position; w = type
    float4 nb_s[kCap];              // shift of FIRST entries, else 0; w = role | entry << 2 | index << 8
    float4 nb_f[kCap];              // neighbour-side force sums of the region: runs of even index
    float4 nb_f1[kCap];             // and of odd index (summed at the region's end)
    float4 nb_v[kDPD ? kCap : 1];   // velocity; w = id
    float4 own_x[kOwn];
    float4 own_v[kDPD ? kOwn : 1];
    float4 own_f[kOwn];
    float4 ent_sh[kEnt];            // staged entries: shift, w = packed role/sort direction/key shift
    int ent_slot[kEnt];             // slot of the entry cell's first particle
    int ent_cnt[kEnt];              // particles of the entry cell
    int ent_rev[kEnt];              // plane of the entry cell's received sums (FIRST entries)
    int reg_beg[kEnt + 1];          // region: first staged index of each region entry
    int reg_jb[kEnt];               // region: index within its cell of the entry's first staged particle
    unsigned long long own_mask[kOwn];  // bit t: a potential exists for (own type, t)
    int nb_key[kCap];               // sort key of the neighbour (per-pair pruning)
    unsigned short queue[TS::kQ];   // own index << 8 | staged index, in candidate order
};

/*
 * dpd_eval (dpd_eval.hpp:21-69) for the DPD-only kernel, the reference's random term (no
 * random number), non-shifted potentials: q0 = (cutoff, alpha, gamma, sigma delta),
 * q1 = (a^2, a, 1 / cutoff, alpha + sigma delta) of the type pair. The cutoff test is the
 * reference's exact one on r2; the force magnitude is formed from one reciprocal square root
 * and fused multiply-adds, f = oc (alpha + sigma delta - gamma oc (e.v)) with oc = 1 - r/rc,
 * e = dx/r (a few units in the last place from the reference's divisions; the force
 * tolerance is 1e-5). The first particle gets +f e, the second -f e.
 */
__device__ __forceinline__ void dpd_fast(const float4 &q0, const float4 &q1, bool i_first, float dx, float dy,
                                         float dz, float r2, const float4 &vi, const float4 &vj, float &cx, float &cy,
                                         float &cz, bool &counted) {
    cx = cy = cz = 0.f;
    counted = false;
    if (r2 > __fmul_rn(q0.x, q0.x)) return;
    const float ir = rsqrtf(r2);
    const float r = __fmul_rn(r2, ir);
    const float ex = __fmul_rn(dx, ir), ey = __fmul_rn(dy, ir), ez = __fmul_rn(dz, ir);
    const float wx = __fsub_rn(vi.x, vj.x), wy = __fsub_rn(vi.y, vj.y), wz = __fsub_rn(vi.z, vj.z);
    // e.(v_first - v_second): dx is first minus second, w is i minus j
    const float ev0 = __fmaf_rn(ex, wx, __fmaf_rn(ey, wy, __fmul_rn(ez, wz)));
    const float ev = i_first ? ev0 : -ev0;
    const float oc = __fmaf_rn(-r, q1.z, 1.0f);
    const float f = __fmul_rn(oc, __fmaf_rn(__fmul_rn(-q0.z, oc), ev, q1.w));
    const float fs = i_first ? f : -f;
    cx = __fmul_rn(fs, ex);
    cy = __fmul_rn(fs, ey);
    cz = __fmul_rn(fs, ez);
    counted = i_first;
}

/* Pass 2 over the nb <= 32 queued pairs from qhead: one interacting pair per
 * lane; own-side segmented sums into own_f, neighbour-side sums into nb_f.
 * kMode 1 counts the pairs (once each), kMode 2 sums the pair virial
 * (x_first - x_second) (x) F_first in FP64 (xx, yy, zz, xy, xz, yz). */
template <bool kDPD, int kMode, bool kPure, class TS>
__device__ __forceinline__ void eval_batch(const EngineView &v, ForceSmem<kDPD, TS> &sm, const float4 *tinfo, int qhead,
                                           int nb, int i0, int own_start, int pot_base, unsigned rng_mode,
                                           float cut2_pair, float cut2_self, bool self_once, double &ecell,
                                           unsigned long long &npair,
                                           double *vir) {
    const int lane = threadIdx.x & 31;
    float cx = 0.f, cy = 0.f, cz = 0.f;
    int il = -1, jj = 0;
    bool nbside = false;
    if (lane < nb) {
        const int cd = sm.queue[(qhead + lane) & (TS::kQ - 1)];
        il = cd >> 8;
        jj = cd & 0xff;
        const int i = i0 + il;
        const float4 xi = sm.own_x[il];
        const float4 b = sm.nb_x[jj];
        const float4 s = sm.nb_s[jj];
        const int meta = __float_as_int(s.w);
        const int role = meta & 3, jl = meta >> 8;
        float dx = __fsub_rn(__fsub_rn(xi.x, s.x), b.x);
        float dy = __fsub_rn(__fsub_rn(xi.y, s.y), b.y);
        float dz = __fsub_rn(__fsub_rn(xi.z, s.z), b.z);
        // a self pair whose first particle is j: the reference's dx is x_j - x_i
        if (role == kRoleSelf && jl < i) {
            dx = -dx;
            dy = -dy;
            dz = -dz;
        }
        float r2 = dot3_rn(dx, dy, dz);
        const float dxo = dx, dyo = dy, dzo = dz;  // before the r < a substitution
        const int ti = __float_as_int(xi.w), tj = __float_as_int(b.w);
        const bool i_first = role == kRoleFirst || (role == kRoleSelf && i < jl);
        // FIRST pairs, and a cell's own pairs when each is evaluated once (by its lower index),
        // put the second particle's share into the staged neighbour's sums
        nbside = role == kRoleFirst || (role == kRoleSelf && self_once);
        // the exact cutoff test of the pair loops (pass 1 queued a superset)
        const bool inside = r2 <= (role == kRoleSelf ? cut2_self : cut2_pair);
        if (kPure && inside) {
            // every pair potential is a DPD potential with the reference's random term: its
            // constants from one compact record per type pair
            const int pk = 2 * (pot_base + ti * v.ntypes + tj);
            const float4 q0 = __ldg(v.dpd_pair + pk), q1 = __ldg(v.dpd_pair + pk + 1);
            if (r2 < q1.x) {
                // potential_eval_super_ex's random direction of length a (Philox here)
                const unsigned idi = __float_as_uint(sm.own_v[il].w), idj = __float_as_uint(sm.nb_v[jj].w);
                const unsigned lo = idi < idj ? idi : idj, hi = idi < idj ? idj : idi;
                float g0, g1, g2;
                philox_normal3(*v.step, lo, hi, g0, g1, g2);
                const float len = sqrtf(g0 * g0 + g1 * g1 + g2 * g2);
                const float sgn = ((idi == lo) == i_first) ? 1.0f : -1.0f;
                dx = sgn * g0 * q1.y / len;
                dy = sgn * g1 * q1.y / len;
                dz = sgn * g2 * q1.y / len;
                r2 = q1.x;
            }
            bool counted;
            dpd_fast(q0, q1, i_first, dx, dy, dz, r2, sm.own_v[il], sm.nb_v[jj], cx, cy, cz, counted);
            if (kMode == 1 && counted) ++npair;
        }
        if (!kPure && inside) {
            const DevPot &p = v.pots[v.pot_idx[pot_base + ti * v.ntypes + tj]];
            if (r2 < p.a2) {
                // potential_eval_super_ex (dpd_eval.hpp:122-131): random direction of
                // length a; here a Philox draw keyed on the step and the id pair
                const unsigned idi = __float_as_uint(kDPD ? sm.own_v[il].w : v.vel[own_start + i].w);
                const unsigned idj =
                    __float_as_uint(kDPD ? sm.nb_v[jj].w : v.vel[sm.ent_slot[(meta >> 2) & 31] + jl].w);
                const unsigned lo = idi < idj ? idi : idj, hi = idi < idj ? idj : idi;
                float g0, g1, g2;
                philox_normal3(*v.step, lo, hi, g0, g1, g2);
                const float len = sqrtf(g0 * g0 + g1 * g1 + g2 * g2);
                // the draw is the displacement first-minus-second for (lo, hi)
                const float sgn = ((idi == lo) == i_first) ? 1.0f : -1.0f;
                dx = sgn * g0 * p.a / len;
                dy = sgn * g1 * p.a / len;
                dz = sgn * g2 * p.a / len;
                r2 = p.a2;
            }
            const float4 vi = kDPD ? sm.own_v[il] : make_float4(0.f, 0.f, 0.f, 0.f);
            const float4 vj = kDPD ? sm.nb_v[jj] : make_float4(0.f, 0.f, 0.f, 0.f);
            float pe;
            bool counted;
            pair_contribution<kDPD, kPure>(v, p, role, i_first, dx, dy, dz, r2, tinfo[ti].w, tinfo[tj].w, vi, vj, rng_mode,
                                    cx, cy, cz, pe, counted);
            ecell += (double)pe;
            if (kMode == 1 && counted) ++npair;
            if (!kPure && v.pot_idx2) {
                // a second potential summed on the same pair (a table potential plus a DPD
                // thermostat), evaluated on the pair's own displacement
                const int q2 = v.pot_idx2[pot_base + ti * v.ntypes + tj];
                if (q2 >= 0) {
                    const DevPot &p2 = v.pots[q2];
                    float r2b = dot3_rn(dxo, dyo, dzo);
                    if (!(r2b < p2.a2)) {
                        float c2x, c2y, c2z, pe2;
                        bool counted2;
                        pair_contribution<kDPD>(v, p2, role, i_first, dxo, dyo, dzo, r2b, tinfo[ti].w, tinfo[tj].w, vi,
                                                vj, rng_mode, c2x, c2y, c2z, pe2, counted2);
                        cx = cx + c2x;
                        cy = cy + c2y;
                        cz = cz + c2z;
                        ecell += (double)pe2;
                    }
                }
            }
        }
        if (kMode == 2 && i_first) {
            vir[0] += (double)dxo * cx;
            vir[1] += (double)dyo * cy;
            vir[2] += (double)dzo * cz;
            vir[3] += (double)dxo * cy;
            vir[4] += (double)dxo * cz;
            vir[5] += (double)dyo * cz;
        }
    }
    // segments: runs of equal own index (inactive lanes form the last one)
    const int il_prev = __shfl_up_sync(kFull, il, 1);
    const unsigned heads = __ballot_sync(kFull, lane == 0 || il != il_prev);
    // neighbour side: the runs in pairs, runs of even index into nb_f and of odd index into
    // nb_f1 (the two runs of a pair cannot add to the same sum, and inside a run the
    // neighbours are distinct), pair after pair: every sum has a fixed order
    const int nseg = __popc(heads & (nb == 32 ? kFull : ((1u << nb) - 1u)));
    const int sidx = __popc(heads & (0xffffffffu >> (31 - lane))) - 1;  // this lane's run
    for (int pr = 0; 2 * pr < nseg; ++pr) {
        if (nbside && lane < nb && (sidx >> 1) == pr) {
            float4 *acc = (sidx & 1) ? sm.nb_f1 : sm.nb_f;
            float4 f = acc[jj];
            f.x = __fsub_rn(f.x, cx);
            f.y = __fsub_rn(f.y, cy);
            f.z = __fsub_rn(f.z, cz);
            acc[jj] = f;
        }
        __syncwarp();
    }
    // own side: segmented inclusive scan, the segment's last lane adds
    const int seg0 = 31 - __clz(heads & (0xffffffffu >> (31 - lane)));
    for (int off = 1; off < 32; off <<= 1) {
        const float ox = __shfl_up_sync(kFull, cx, off);
        const float oy = __shfl_up_sync(kFull, cy, off);
        const float oz = __shfl_up_sync(kFull, cz, off);
        if (lane - off >= seg0) {
            cx = ox + cx;
            cy = oy + cy;
            cz = oz + cz;
        }
    }
    const bool seg_end = lane == 31 || ((heads >> (lane + 1)) & 1u);
    if (il >= 0 && seg_end) {
        float4 f = sm.own_f[il];
        f.x += cx;
        f.y += cy;
        f.z += cz;
        sm.own_f[il] = f;
    }
}

/* Zeroes the plane a cell owes a FIRST neighbour when it evaluates none of the
 * pair's candidates (the cell is empty, or the reference's exit test skips the
 * pair). */
__device__ __forceinline__ void zero_plane(const EngineView &v, int rev, int nstart, int ncount) {
    const int lane = threadIdx.x & 31;
    float4 *dst = v.planes + (size_t)rev * v.nparts + nstart;
    for (int k = lane; k < ncount; k += 32) dst[k] = make_float4(0.f, 0.f, 0.f, 0.f);
}

template <bool kDPD, class TS>
constexpr size_t force_smem_bytes() {
    return sizeof(ForceSmem<kDPD, TS>) * kWarpsPerBlock;
}

template <bool kDPD, int kMode, bool kPure, class TS>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, TS::kBlocks) force_kernel(EngineView v) {
    constexpr int kOwn = TS::kOwn, kCap = TS::kCap, kChunks = TS::kChunks;
    unsigned long long npair = 0;  // interacting pairs counted once (statistics launch only)
    double vir[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // pair virial (virial launch only)
    extern __shared__ float4 force_smem[];
    // per type: constant force (zero if none), radius; after the warps' areas (v.ntypes entries)
    float4 *tinfo = force_smem + sizeof(ForceSmem<kDPD, TS>) * kWarpsPerBlock / sizeof(float4);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    ForceSmem<kDPD, TS> &sm = reinterpret_cast<ForceSmem<kDPD, TS> *>(force_smem)[w];
    const unsigned lt_mask = (1u << lane) - 1u;
    const int ntypes = v.ntypes;
    for (int t = threadIdx.x; t < ntypes; t += blockDim.x) {
        const DevType &T = v.types[t];
        // constant_force (MxForce.cpp:339-344), scale 1
        tinfo[t] = T.has_force ? make_float4(T.fx, T.fy, T.fz, T.radius) : make_float4(0.f, 0.f, 0.f, T.radius);
    }
    __syncthreads();
    // work items: fetched from a counter (the crowded cells' items would otherwise hold
    // their block's slot while the other warps idle); the virial launch keeps a fixed
    // grid-stride assignment, so that its per-warp FP64 partials sum in a fixed order.
    // Every item writes only its own outputs, so the fetch order changes no result.
    const int nwarps = gridDim.x * kWarpsPerBlock;
    auto fetch = [&](int prev) -> int {
        if (kMode == 2) return prev < 0 ? blockIdx.x * kWarpsPerBlock + w : prev + nwarps;
        int t = 0;
        if (lane == 0) {
            t = atomicAdd(v.item_ctr, 1);
            if (v.item_order && t < v.nitems) t = v.item_order[t];
        }
        return __shfl_sync(kFull, t, 0);
    };
    for (int it = fetch(-1); it < v.nitems; it = fetch(it)) {
        const int4 item = v.items[it];
        const int c = item.x, nb0 = item.y, nb1 = item.z, part = item.w;
        const int n = v.cell_count[c];
        double ecell = 0.0;
        if (n == 0) {
            for (int e = nb0; e < nb1 && kMode != 2; ++e) {
                const int pk = __float_as_int(v.nb_shift[e].w);
                if ((pk & 3) != kRoleFirst) continue;
                const int nc = v.nb_cell[e];
                zero_plane(v, v.nb_rev[e], v.cell_start[nc], v.cell_count[nc]);
            }
        } else {
            const int start = v.cell_start[c];
            const DevSpace &S = v.spaces[v.cell_rep[c]];
            const int pot_base = S.pot_offset;
            const float cut2_pair = S.cut2_pair, cut2_self = S.cut2_self;
            const float cut2w_pair = S.cut2w_pair, cut2w_self = S.cut2w_self;
            const unsigned rng_mode = S.rng_mode;
            const bool prune = (S.prune & 1) != 0;      // per-pair projection test
            const bool exit_test = (S.prune & 2) != 0;  // cell-pair exit test
            const float sbias = S.sort_bias, sdscale = S.sort_dscale;
            const int dmaxdist = S.dmaxdist;
            // a cell whose particles fit one own pass evaluates each of its own pairs once
            const bool self_once = n <= kOwn;
            for (int i0 = 0; i0 < n; i0 += kOwn) {
                const int ni = min(kOwn, n - i0);
                __syncwarp();
                for (int k = lane; k < ni; k += 32) {  // kOwn may exceed the warp
                    const float4 x = v.pos[start + i0 + k];
                    sm.own_x[k] = x;
                    const int ti = __float_as_int(x.w);
                    const float4 T = tinfo[ti];  // the body force goes with the cell's first work item
                    sm.own_f[k] = part == 0 ? make_float4(T.x, T.y, T.z, 0.f) : make_float4(0.f, 0.f, 0.f, 0.f);
                    if (kDPD) sm.own_v[k] = v.vel[start + i0 + k];
                    unsigned long long mk = 0ull;
                    for (int t = 0; t < ntypes; ++t)
                        if (v.pot_idx[pot_base + ti * ntypes + t] >= 0) mk |= 1ull << t;  // a lone second term is moved here
                    sm.own_mask[k] = mk;
                }
                for (int g0 = nb0; g0 < nb1; g0 += kEnt) {
                    // ---- entries g0 .. g0+31: lane k loads entry g0 + k; SELF and FIRST entries
                    // with particles are staged (compacted in entry order)
                    const int ek = g0 + lane;
                    int cnt = 0, cstart = 0, rev = -1, skipped = 0;
                    float4 sh = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (ek < nb1) {
                        sh = v.nb_shift[ek];
                        const int pk = __float_as_int(sh.w);
                        const int role = pk & 3;
                        if (role != kRoleSecond) {
                            const int nc = v.nb_cell[ek];
                            cnt = v.cell_count[nc];
                            cstart = v.cell_start[nc];
                            rev = v.nb_rev[ek];
                            if (cnt > 0 && exit_test && role == kRoleFirst) {
                                // runner_dopair.cpp:167-171: kmin(second) + dnshift - kmax(first) in
                                // unsigned arithmetic; above dmaxdist or wrapped, the pair is skipped
                                const int sid = (pk >> 2) & 15;
                                const int2 bc = v.sort_bounds[c * 13 + sid], bn = v.sort_bounds[nc * 13 + sid];
                                const int gap = bn.x + (pk >> 8) - bc.y;
                                if (gap < 0 || gap > dmaxdist) {
                                    skipped = cnt;
                                    cnt = 0;
                                }
                            }
                        }
                    }
                    // skipped pairs owe their neighbour a zero plane (written by the first own chunk)
                    unsigned zmask = __ballot_sync(kFull, skipped > 0 && i0 == 0 && kMode != 2);
                    while (zmask) {
                        const int k = __ffs(zmask) - 1;
                        zmask &= zmask - 1;
                        zero_plane(v, __shfl_sync(kFull, rev, k), __shfl_sync(kFull, cstart, k),
                                   __shfl_sync(kFull, skipped, k));
                    }
                    const unsigned staged = __ballot_sync(kFull, cnt > 0);
                    const int nst = __popc(staged);
                    __syncwarp();
                    if (cnt > 0) {
                        const int k = __popc(staged & lt_mask);
                        sm.ent_sh[k] = sh;
                        sm.ent_slot[k] = cstart;
                        sm.ent_cnt[k] = cnt;
                        sm.ent_rev[k] = rev;
                    }
                    __syncwarp();
                    // ---- regions: consecutive staged entries holding at most kCap particles
                    int ce = 0, jpos = 0;
                    while (ce < nst) {
                        const int rce = ce;
                        const int k = ce + lane;
                        const int jb = lane == 0 ? jpos : 0;
                        const int rem = k < nst ? sm.ent_cnt[k] - jb : 0;
                        int incl = rem;
                        for (int off = 1; off < 32; off <<= 1) {
                            const int o = __shfl_up_sync(kFull, incl, off);
                            if (lane >= off) incl += o;
                        }
                        const int nfit = __popc(__ballot_sync(kFull, k < nst && incl <= kCap));
                        int nent, M;
                        if (nfit == 0) {  // the first entry alone holds more than kCap particles
                            nent = 1;
                            M = kCap;
                            jpos += kCap;
                        } else {
                            nent = nfit;
                            M = __shfl_sync(kFull, incl, nfit - 1);
                            ce += nfit;
                            jpos = 0;
                        }
                        __syncwarp();
                        if (lane < nent) {
                            sm.reg_beg[lane] = incl - rem;
                            sm.reg_jb[lane] = jb;
                        }
                        if (lane == 0) sm.reg_beg[nent] = M;
                        __syncwarp();
                        // ---- stage the region's neighbour particles: positions and velocities go
                        // straight from global to shared memory (cp.async, every load of the region in
                        // flight at once, none through registers); then lane's chunk-u neighbour
                        // (staged index u * 32 + lane) is also kept in registers for pass 1:
                        // neighbour position plus the entry's shift (one rounding away from the
                        // reference's (x_i - s) - x_j): pass 1 is a superset filter with a widened
                        // cutoff; pass 2 applies the exact test on the exact displacement
                        float rbx[kChunks], rby[kChunks], rbz[kChunks];
                        float rc2[kChunks];   // widened cutoff squared; -1 for an empty position
                        int rself[kChunks];   // index of a SELF neighbour within the cell, else -1
                        int rtj[kChunks];     // neighbour type (the entry's sort direction until staged)
#pragma unroll
                        for (int u = 0; u < kChunks; ++u) {
                            const int idx = u * 32 + lane;
                            rbx[u] = rby[u] = rbz[u] = 0.f;
                            rc2[u] = -1.f;
                            rself[u] = -1;
                            rtj[u] = 0;
                            if (idx < M) {
                                int r = 0;
                                for (int step = 16; step > 0; step >>= 1)
                                    if (r + step < nent && sm.reg_beg[r + step] <= idx) r += step;
                                const int ke = rce + r;
                                const int jl = sm.reg_jb[r] + idx - sm.reg_beg[r];
                                const int slot = sm.ent_slot[ke] + jl;
                                const float4 es = sm.ent_sh[ke];
                                const int epk = __float_as_int(es.w);
                                const int role = epk & 3;
                                cp_async16(&sm.nb_x[idx], v.pos + slot);
                                if (kDPD) cp_async16(&sm.nb_v[idx], v.vel + slot);
                                float4 s4 = make_float4(0.f, 0.f, 0.f, __int_as_float(role | (ke << 2) | (jl << 8)));
                                if (role == kRoleFirst) {
                                    s4.x = es.x;
                                    s4.y = es.y;
                                    s4.z = es.z;
                                }
                                sm.nb_s[idx] = s4;
                                sm.nb_f[idx] = make_float4(0.f, 0.f, 0.f, 0.f);
                                sm.nb_f1[idx] = make_float4(0.f, 0.f, 0.f, 0.f);
                                rbx[u] = s4.x;
                                rby[u] = s4.y;
                                rbz[u] = s4.z;
                                rc2[u] = role == kRoleSelf ? cut2w_self : cut2w_pair;
                                rself[u] = role == kRoleSelf ? jl : -1;
                                rtj[u] = (epk >> 2) & 15;
                            }
                        }
                        cp_async_wait_all();
                        __syncwarp();
#pragma unroll
                        for (int u = 0; u < kChunks; ++u) {
                            const int idx = u * 32 + lane;
                            if (idx < M) {
                                const float4 q = sm.nb_x[idx];
                                if (prune) sm.nb_key[idx] = sort_key(q.x, q.y, q.z, v.axes->n[rtj[u]], sbias, sdscale);
                                rbx[u] = __fadd_rn(q.x, rbx[u]);
                                rby[u] = __fadd_rn(q.y, rby[u]);
                                rbz[u] = __fadd_rn(q.z, rbz[u]);
                                rtj[u] = __float_as_int(q.w);
                            }
                        }
                        // the candidate test's form for the whole region: the type test is moot
                        // when every own particle has a potential with every type staged, the
                        // own-index test when no SELF neighbour is staged (2: the full test)
                        int pmode = 2;
                        if (!prune) {
                            unsigned long long rtypes = 0ull;
                            bool rs_any = false;
#pragma unroll
                            for (int u = 0; u < kChunks; ++u)
                                if (u * 32 + lane < M) {
                                    rtypes |= 1ull << rtj[u];
                                    rs_any |= rself[u] >= 0;
                                }
                            rtypes = (unsigned long long)__reduce_or_sync(kFull, (unsigned)rtypes) |
                                     ((unsigned long long)__reduce_or_sync(kFull, (unsigned)(rtypes >> 32)) << 32);
                            bool full = true;
                            for (int k = lane; k < ni; k += 32) full &= (sm.own_mask[k] & rtypes) == rtypes;
                            if (__all_sync(kFull, full)) pmode = __any_sync(kFull, rs_any) ? 1 : 0;
                        }
                        __syncwarp();
                        // ---- pass 1: each own particle against the region, kChunks steps of
                        // 32 candidates, then pass 2 on every full batch of 32 queued pairs.
                        // The squared distance is formed with fused multiply-adds: pass 1 is a
                        // superset filter (widened cutoff), the exact test is pass 2's
                        int qhead = 0, qtail = 0;
                        // il == ni adds no candidates and flushes the queue: one call site of
                        // eval_batch keeps the kernel's instruction footprint small
                        for (int il = 0; il <= ni; ++il) {
                            if (il < ni) {
                                const float4 xi = sm.own_x[il];
                                const int i = i0 + il;
                                unsigned hb[kChunks];
                                bool hv[kChunks];
                                if (pmode == 0) {
#pragma unroll
                                    for (int u = 0; u < kChunks; ++u) {
                                        hb[u] = 0u;
                                        hv[u] = false;
                                        if (u * 32 < M) {
                                            const float dx = __fsub_rn(xi.x, rbx[u]);
                                            const float dy = __fsub_rn(xi.y, rby[u]);
                                            const float dz = __fsub_rn(xi.z, rbz[u]);
                                            const bool hit = __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmul_rn(dz, dz))) <= rc2[u];
                                            hb[u] = __ballot_sync(kFull, hit);
                                            hv[u] = hit;
                                        }
                                    }
                                } else if (pmode == 1) {
#pragma unroll
                                    for (int u = 0; u < kChunks; ++u) {
                                        hb[u] = 0u;
                                        hv[u] = false;
                                        if (u * 32 < M) {
                                            const float dx = __fsub_rn(xi.x, rbx[u]);
                                            const float dy = __fsub_rn(xi.y, rby[u]);
                                            const float dz = __fsub_rn(xi.z, rbz[u]);
                                            const float r2 = __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmul_rn(dz, dz)));
                                            const bool pair_ok = self_once ? (unsigned)rself[u] > (unsigned)i : rself[u] != i;
                                            const bool hit = (r2 <= rc2[u]) & pair_ok;
                                            hb[u] = __ballot_sync(kFull, hit);
                                            hv[u] = hit;
                                        }
                                    }
                                } else {
                                    const unsigned long long mk = sm.own_mask[il];
#pragma unroll
                                    for (int u = 0; u < kChunks; ++u) {
                                        hb[u] = 0u;
                                        hv[u] = false;
                                        if (u * 32 < M) {
                                            const float dx = __fsub_rn(xi.x, rbx[u]);
                                            const float dy = __fsub_rn(xi.y, rby[u]);
                                            const float dz = __fsub_rn(xi.z, rbz[u]);
                                            const float r2 = __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmul_rn(dz, dz)));
                                            // a cell's own pair once (neighbour index above the own one; -1, not
                                            // a SELF neighbour, compares as the largest unsigned value), or from
                                            // both sides when the cell takes several own-particle passes
                                            const bool pair_ok = self_once ? (unsigned)rself[u] > (unsigned)i : rself[u] != i;
                                            bool hit = (r2 <= rc2[u]) & (((mk >> rtj[u]) & 1ull) != 0ull) & pair_ok;
                                            if (prune && hit && rself[u] < 0) {
                                                // runner_dopair's pruning: a pair (first, second) is evaluated
                                                // only when key_second + dnshift - key_first < dmaxdist
                                                // (runner_dopair.cpp:167-182)
                                                const int jj = u * 32 + lane;
                                                const int meta = __float_as_int(sm.nb_s[jj].w);
                                                const int epk = __float_as_int(sm.ent_sh[(meta >> 2) & 31].w);
                                                const int okey = sort_key(xi.x, xi.y, xi.z, v.axes->n[(epk >> 2) & 15],
                                                                          sbias, sdscale);
                                                hit = sm.nb_key[jj] + (epk >> 8) - okey < dmaxdist;
                                            }
                                            hb[u] = __ballot_sync(kFull, hit);
                                            hv[u] = hit;
                                        }
                                    }
                                }
#pragma unroll
                                for (int u = 0; u < kChunks; ++u) {
                                    if (hv[u])
                                        sm.queue[(qtail + __popc(hb[u] & lt_mask)) & (TS::kQ - 1)] =
                                            (unsigned short)((il << 8) | (u * 32 + lane));
                                    qtail += __popc(hb[u]);
                                }
                            }
                            while (qtail - qhead >= 32 || (il == ni && qtail > qhead)) {
                                const int nb = min(32, qtail - qhead);
                                __syncwarp();
                                eval_batch<kDPD, kMode, kPure, TS>(v, sm, tinfo, qhead, nb, i0, start, pot_base, rng_mode, cut2_pair,
                                               cut2_self, self_once, ecell, npair, vir);
                                qhead += nb;
                            }
                        }
                        __syncwarp();
                        // ---- neighbour-side sums of FIRST entries into their planes; those of a
                        // cell's own particles (pairs evaluated once) into their own sums
                        for (int idx = lane; idx < M && kMode != 2; idx += 32) {
                            const int meta = __float_as_int(sm.nb_s[idx].w);
                            const float4 g0 = sm.nb_f[idx], g1 = sm.nb_f1[idx];
                            const float4 g = make_float4(g0.x + g1.x, g0.y + g1.y, g0.z + g1.z, 0.f);
                            if (self_once && (meta & 3) == kRoleSelf) {
                                float4 &o = sm.own_f[meta >> 8];  // one own pass: own index = index in the cell
                                o.x += g.x;
                                o.y += g.y;
                                o.z += g.z;
                                continue;
                            }
                            if ((meta & 3) != kRoleFirst) continue;
                            const int ke = (meta >> 2) & 31;
                            float4 *dst = v.planes + (size_t)sm.ent_rev[ke] * v.nparts + sm.ent_slot[ke] + (meta >> 8);
                            float4 f = g;
                            if (i0 > 0) {  // later own chunks add to the first chunk's sums
                                const float4 o = *dst;
                                f = make_float4(o.x + f.x, o.y + f.y, o.z + f.z, 0.f);
                            }
                            *dst = f;
                        }
                        __syncwarp();
                    }
                }
                __syncwarp();
                for (int k = lane; k < ni; k += 32) {
                    const float4 f = sm.own_f[k];
                    // the cell's first work item writes the force, later ones their own plane
                    float4 *dst = part == 0 ? v.force : v.planes + (size_t)(v.sec_count[c] + part - 1) * v.nparts;
                    if (kMode != 2) dst[start + i0 + k] = make_float4(f.x, f.y, f.z, 0.f);
                }
            }
        }
        for (int off = 16; off > 0; off >>= 1) ecell += __shfl_xor_sync(kFull, ecell, off);
        if (lane == 0 && kMode != 2) v.epot_cell[it] = ecell;
    }
    if (kMode != 2 && lane == 0) {
        // every warp has drawn its last ticket once the done count reaches the grid's warps:
        // the last one re-arms both counters for the next launch on the stream
        if (atomicAdd(v.item_ctr + 1, 1) == nwarps - 1) {
            atomicExch(v.item_ctr, 0);
            atomicExch(v.item_ctr + 1, 0);
        }
    }
    if (kMode == 1) {
        for (int off = 16; off > 0; off >>= 1) npair += __shfl_xor_sync(kFull, npair, off);
        if (lane == 0) atomicAdd(v.pair_stats, npair);
    }
    if (kMode == 2) {  // this warp's virial, lanes summed in a fixed tree (the launch writes nothing else)
        for (int k = 0; k < 6; ++k) {
            double t = vir[k];
            for (int off = 16; off > 0; off >>= 1) t += __shfl_xor_sync(kFull, t, off);
            if (lane == 0) v.virial_partials[(size_t)(blockIdx.x * kWarpsPerBlock + w) * 6 + k] = t;
        }
    }
}

/* The 3x3 pair virial from the warps' partials, in warp order. */
__global__ void virial_reduce_kernel(const double *partials, int nwarps, double *out9) {
    const int k = threadIdx.x;
    if (k >= 6) return;
    double t = 0.0;
    for (int q = 0; q < nwarps; ++q) t += partials[(size_t)q * 6 + k];
    const int rc[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
    out9[rc[k][0] * 3 + rc[k][1]] = t;
    out9[rc[k][1] * 3 + rc[k][0]] = t;
}

/* A particle's own-side force plus, in plane order, the sums its cell received
 * from the cells that evaluated their shared pairs and the own-side sums of its
 * cell's later work items. */
__device__ __forceinline__ float4 total_force(const EngineView &v, int s) {
    float4 f = v.force[s];
    const int np = v.cell_planes[v.cell_of[s]];
    // the planes are read once: eight independent streaming loads in flight, then the
    // additions in plane order (the same sums, bit for bit)
    for (int k0 = 0; k0 < np; k0 += 8) {
        float4 g[8];
#pragma unroll
        for (int q = 0; q < 8; ++q)
            if (k0 + q < np) g[q] = __ldcs(v.planes + (size_t)(k0 + q) * v.nparts + s);
#pragma unroll
        for (int q = 0; q < 8; ++q)
            if (k0 + q < np) {
                f.x += g[q].x;
                f.y += g[q].y;
                f.z += g[q].z;
            }
    }
    if (v.body_f) {  // walls and large particles of this pass (body_kernel)
        const float4 b = v.body_f[s];
        f.x += b.x;
        f.y += b.y;
        f.z += b.z;
    }
    if (v.has_sb) {
        // the velocity-dependent and random single-body forces (MxForce.cpp:330-386)
        const int ti = __float_as_int(v.pos[s].w);
        const DevType &T = v.types[ti];
        if (T.sb_kind >= 2) {
            const float4 u = v.vel[s];
            const int id = __float_as_int(u.w);
            float sx = 0.f, sy = 0.f, sz = 0.f, px = 0.f, py = 0.f, pz = 0.f;
            if (T.sb_kind == 2) {  // berendsen_force: itau ((T0 / KE_type) - 1) v
                const float scale = (float)((double)T.sb_a * ((T.target / v.type_ke[ti]) - 1.0));
                sx = __fmul_rn(scale, u.x);
                sy = __fmul_rn(scale, u.y);
                sz = __fmul_rn(scale, u.z);
            } else {
                const float4 pf = v.persist[id];
                px = pf.x;
                py = pf.y;
                pz = pf.z;
                if (T.sb_kind == 4) {  // friction_force: -coef |v|^2 v
                    const float v2 = __fadd_rn(__fadd_rn(__fmul_rn(u.x, u.x), __fmul_rn(u.y, u.y)), __fmul_rn(u.z, u.z));
                    const float scale = (float)(-1. * (double)T.sb_a * (double)v2);
                    sx = __fmul_rn(scale, u.x);
                    sy = __fmul_rn(scale, u.y);
                    sz = __fmul_rn(scale, u.z);
                }
            }
            f.x += __fadd_rn(sx, px);
            f.y += __fadd_rn(sy, py);
            f.z += __fadd_rn(sz, pz);
        }
    }
    return f;
}

/* ------------------------------------------------------------------------ */
/* species fluxes                                                            */
/* ------------------------------------------------------------------------ */

/*
 * Flux rates of one particle (flux_eval_ex, flux_eval.hpp:33-84, evaluated in
 * the reference's pair loops for every pair within the cutoff whose types have
 * fluxes, runner_dopair.cpp:197-252, 555-611). One thread per particle visits
 * all its neighbour cells (full shell). Each pair is evaluated in the
 * reference's orientation (the FIRST cell's particle first; in a cell, the
 * lower slot first), so both of its particles compute the same weight
 * (1 - r/cutoff)^2 and the same q for every entry of the pair's flux list and
 * each applies its own share: the entry's a particle q_a = q_a - q - decay/2 s_a,
 * its b particle q_b = q_b + q - decay/2 s_b. A cell pair that the reference's
 * sorted loop skips as a whole (its unsigned exit test, runner_dopair.cpp:
 * 167-171) carries no fluxes either. The rates accumulate on top of what the
 * particle carries (cleared when its values are integrated).
 */
__global__ void flux_kernel(EngineView v, SpeciesView sp) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= v.nparts) return;
    const float4 xo = v.pos[s];
    const int to = __float_as_int(xo.w);
    const int id = __float_as_int(v.vel[s].w);
    const int nso = sp.nspec[to];
    if (nso <= 0) return;
    float *rate = sp.rate + (size_t)id * sp.smax;
    float acc[8];
    for (int k = 0; k < 8; ++k) acc[k] = k < sp.smax ? rate[k] : 0.f;
    const int c = v.cell_of[s];
    const DevSpace &S = v.spaces[v.cell_rep[c]];
    const bool exit_test = (S.prune & 2) != 0;
    for (int e = sp.fx_off[c]; e < sp.fx_off[c + 1]; ++e) {
        const int nc = sp.fx_cell[e];
        const float4 sh = sp.fx_shift[e];
        const int pk = __float_as_int(sh.w);
        const int role = pk & 3;
        if (exit_test && role != kRoleSelf) {
            // kmin(second) + dnshift - kmax(first) in unsigned arithmetic, as the force pass
            const int sid = (pk >> 2) & 15;
            const int cf = role == kRoleFirst ? c : nc, cs = role == kRoleFirst ? nc : c;
            const int2 bf = v.sort_bounds[cf * 13 + sid], bs = v.sort_bounds[cs * 13 + sid];
            const int gap = bs.x + (pk >> 8) - bf.y;
            if (v.cell_count[cf] > 0 && v.cell_count[cs] > 0 && (gap < 0 || gap > S.dmaxdist)) continue;
        }
        const int j0 = v.cell_start[nc], j1 = j0 + v.cell_count[nc];
        for (int j = j0; j < j1; ++j) {
            if (j == s) continue;
            const float4 xj = v.pos[j];
            const int tj = __float_as_int(xj.w);
            bool own_first;
            float dx, dy, dz;
            if (role == kRoleSelf) {
                own_first = s < j;
                const float4 &a = own_first ? xo : xj, &b = own_first ? xj : xo;
                dx = __fsub_rn(a.x, b.x);
                dy = __fsub_rn(a.y, b.y);
                dz = __fsub_rn(a.z, b.z);
            } else {
                own_first = role == kRoleFirst;
                const float4 &a = own_first ? xo : xj, &b = own_first ? xj : xo;
                dx = __fsub_rn(__fsub_rn(a.x, sh.x), b.x);
                dy = __fsub_rn(__fsub_rn(a.y, sh.y), b.y);
                dz = __fsub_rn(__fsub_rn(a.z, sh.z), b.z);
            }
            const float r2 = dot3_rn(dx, dy, dz);
            // the pair loop's float cutoff squared; the cell loop's double one as float
            if (r2 > (role == kRoleSelf ? S.cut2_self : S.cut2_pair)) continue;
            const int t1 = own_first ? to : tj, t2 = own_first ? tj : to;
            const int f0 = sp.flux_off[t1 * v.ntypes + t2], f1 = sp.flux_off[t1 * v.ntypes + t2 + 1];
            if (f0 == f1) continue;
            const int id_j = __float_as_int(v.vel[j].w);
            const int id1 = own_first ? id : id_j, id2 = own_first ? id_j : id;
            const float r = __fsqrt_rn(r2);
            float w = (float)__dsub_rn(1.0, __ddiv_rn((double)r, S.cutoff_d));
            w = __fmul_rn(w, w);
            for (int q = f0; q < f1; ++q) {
                const DevFlux F = sp.flux[q];
                // flux_eval_ex: pi is the pair's particle of type a (the first when both are),
                // pj the one of type b (the second when both are)
                const int ida = t1 == F.ta ? id1 : id2, idb = t2 == F.tb ? id2 : id1;
                const float sa = sp.value[(size_t)ida * sp.smax + F.ia], sb = sp.value[(size_t)idb * sp.smax + F.ib];
                float g;
                if (F.kind == 0) {
                    g = __fmul_rn(F.k, __fsub_rn(sa, sb));
                } else if (F.kind == 1) {
                    const float u = __fmul_rn(F.k, __fsub_rn(sa, F.target));
                    g = __fmul_rn(u > 0.f ? 1.f : 0.f, u);
                } else {
                    const float u = __fmul_rn(__fmul_rn(F.k, __fsub_rn(F.target, sb)), sa);
                    g = __fmul_rn(u > 0.f ? 1.f : 0.f, u);
                }
                const float qq = __fmul_rn(w, g);
                const float hd = __fdiv_rn(F.decay, 2.f);
                if (ida == id && F.ia < 8) acc[F.ia] = __fsub_rn(__fsub_rn(acc[F.ia], qq), __fmul_rn(hd, sa));
                if (idb == id && F.ib < 8) acc[F.ib] = __fsub_rn(__fadd_rn(acc[F.ib], qq), __fmul_rn(hd, sb));
            }
        }
    }
    for (int k = 0; k < sp.smax && k < 8; ++k) rate[k] = acc[k];
}

/* Species update after a forward-Euler step (integrate_statevector,
 * Flux.cpp:261-267): value += dt * rate (in double, rounded to float) unless
 * the species is constant, then the rate is cleared. The reference runs it per
 * cell after that cell's particles have moved (engine_advance.cpp:339-343), so
 * a particle that changed cells in this step is in no cell's list at that
 * moment: its values stay and its rates carry over to the next step. */
__global__ void species_integrate_kernel(EngineView v, SpeciesView sp, const int *__restrict__ new_cell) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= v.nparts) return;
    if (new_cell[s] != v.cell_of[s]) return;
    const int t = __float_as_int(v.pos[s].w);
    const int id = __float_as_int(v.vel[s].w);
    const DevSpace &S = v.spaces[v.cell_rep[v.cell_of[s]]];
    for (int k = 0; k < sp.nspec[t]; ++k) {
        const float konst = (sp.flags[t * sp.smax + k] & 4u) ? 0.f : 1.f;
        float &x = sp.value[(size_t)id * sp.smax + k];
        x = (float)__dadd_rn((double)x, __dmul_rn(__dmul_rn(S.dt_d, (double)sp.rate[(size_t)id * sp.smax + k]),
                                                  (double)konst));
    }
    for (int k = 0; k < sp.smax; ++k) sp.rate[(size_t)id * sp.smax + k] = 0.f;
}

/*
 * The number density f[3] of the particles (the reference's MxParticle::number_density),
 * for the current positions, as a force pass leaves it: W(0, rc) from space_prepare
 * (space.cpp:216-236) plus W(r2, rc) for every pair the pair loops reach within the cutoff
 * (runner_dopair.cpp:194-203, 552-559) whose type pair has no potential and no flux, or
 * whose potential evaluates in range (potential_eval_super_ex adds it on success,
 * dpd_eval.hpp:133-166; a pair closer than the table minimum counts at distance a). W is
 * the cubic spline of smoothing_kernel.hpp:37-56 with h = rc; the reference forms r with
 * a 12-bit reciprocal square-root approximation (qsqrt, :19-24), here sqrtf. One thread per
 * particle visits the full shell of its cell (SELF, FIRST and SECOND entries, each pair in
 * the reference's orientation for its r2, the same pruning tests as the force pass), so the
 * sums have a fixed order. Large particles, walls and second summed potentials add nothing.
 */
__device__ __forceinline__ float w_cubic(float r2, float h) {
    const float r = sqrtf(r2);
    const float x = r / h;
    float y;
    if (x < 1.f) {
        const float x2 = x * x;
        y = 1.f - (3.f / 2.f) * x2 + (3.f / 4.f) * x2 * x;
    } else if (x < 2.f) {
        const float a = 2.f - x;
        y = (1.f / 4.f) * a * a * a;
    } else {
        y = 0.f;
    }
    return (float)((double)y / (M_PI * (double)h * (double)h * (double)h));
}

__global__ void number_density_kernel(EngineView v, const int *flux_off, float *nd_out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= v.nparts) return;
    const float4 xo = v.pos[s];
    const int to = __float_as_int(xo.w);
    const int c = v.cell_of[s];
    const DevSpace &S = v.spaces[v.cell_rep[c]];
    const float h = (float)S.cutoff_d;
    float nd = w_cubic(0.f, h);
    if (v.types[to].large) {
        nd_out[__float_as_int(v.vel[s].w)] = nd;
        return;
    }
    const bool prune = (S.prune & 1) != 0, exit_test = (S.prune & 2) != 0;
    for (int e = v.nb_off[c]; e < v.nb_off[c + 1]; ++e) {
        const int nc = v.nb_cell[e];
        const float4 sh = v.nb_shift[e];
        const int pk = __float_as_int(sh.w);
        const int role = pk & 3;
        const int sid = (pk >> 2) & 15;
        if (exit_test && role != kRoleSelf) {
            const int cf = role == kRoleFirst ? c : nc, cs = role == kRoleFirst ? nc : c;
            const int2 bf = v.sort_bounds[cf * 13 + sid], bs = v.sort_bounds[cs * 13 + sid];
            const int gap = bs.x + (pk >> 8) - bf.y;
            if (v.cell_count[cf] > 0 && v.cell_count[cs] > 0 && (gap < 0 || gap > S.dmaxdist)) continue;
        }
        const int j0 = v.cell_start[nc], j1 = j0 + v.cell_count[nc];
        for (int j = j0; j < j1; ++j) {
            if (j == s) continue;
            const float4 xj = v.pos[j];
            const float4 &a = role == kRoleSecond ? xj : xo, &b = role == kRoleSecond ? xo : xj;
            float dx, dy, dz;
            if (role == kRoleSelf) {
                dx = __fsub_rn(a.x, b.x);
                dy = __fsub_rn(a.y, b.y);
                dz = __fsub_rn(a.z, b.z);
            } else {
                dx = __fsub_rn(__fsub_rn(a.x, sh.x), b.x);
                dy = __fsub_rn(__fsub_rn(a.y, sh.y), b.y);
                dz = __fsub_rn(__fsub_rn(a.z, sh.z), b.z);
            }
            const float r2 = dot3_rn(dx, dy, dz);
            if (r2 > (role == kRoleSelf ? S.cut2_self : S.cut2_pair)) continue;
            if (prune && role != kRoleSelf) {
                const float *n = v.axes->n[sid];
                const int kf = sort_key(a.x, a.y, a.z, n, S.sort_bias, S.sort_dscale);
                const int ks = sort_key(b.x, b.y, b.z, n, S.sort_bias, S.sort_dscale);
                if (!(ks + (pk >> 8) - kf < S.dmaxdist)) continue;
            }
            const int tj = __float_as_int(xj.w);
            if (v.types[tj].large) continue;
            const int q = v.pot_idx[S.pot_offset + to * v.ntypes + tj];
            bool counts;
            if (q < 0) {
                counts = !flux_off || flux_off[to * v.ntypes + tj] == flux_off[to * v.ntypes + tj + 1];
            } else {
                const DevPot &p = v.pots[q];
                const float rr2 = r2 < p.a2 ? p.a2 : r2;
                const float ra = role == kRoleSecond ? v.types[tj].radius : v.types[to].radius;
                const float rb = role == kRoleSecond ? v.types[to].radius : v.types[tj].radius;
                if (p.kind == 1) {
                    const float cut = (p.flags & (1u << 12)) ? __fadd_rn(__fadd_rn(p.b, ra), rb) : p.b;
                    counts = !(rr2 > __fmul_rn(cut, cut));
                } else {
                    float ee, ff;
                    counts = table_eval_ex(p, v.coef, ra, rb, rr2, ee, ff);
                }
            }
            if (counts) nd = __fadd_rn(nd, w_cubic(r2, h));
        }
    }
    nd_out[__float_as_int(v.vel[s].w)] = nd;
}

/* Quaternion product a b, components (x, y, z, w), in the arithmetic order of the
 * vector form (b.v a.w + a.v b.w + a.v x b.v, a.w b.w - a.v . b.v). */
__device__ __forceinline__ void quat_mul(const float *a, const float *b, float *o) {
    const float cx = a[1] * b[2] - a[2] * b[1], cy = a[2] * b[0] - a[0] * b[2], cz = a[0] * b[1] - a[1] * b[0];
    o[0] = (b[0] * a[3] + a[0] * b[3]) + cx;
    o[1] = (b[1] * a[3] + a[1] * b[3]) + cy;
    o[2] = (b[2] * a[3] + a[2] * b[3]) + cz;
    o[3] = a[3] * b[3] - ((a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]);
}

/* q v q* : v rotated by the unit quaternion q. */
__device__ __forceinline__ void quat_rotate(const float *q, const float *v, float *out) {
    const float p[4] = {v[0], v[1], v[2], 0.f}, qc[4] = {-q[0], -q[1], -q[2], q[3]};
    float t[4], r[4];
    quat_mul(q, p, t);
    quat_mul(t, qc, r);
    out[0] = r[0];
    out[1] = r[1];
    out[2] = r[2];
}

/*
 * Cuboid forces on one particle (potential_eval_cuboid_particle, cuboid_eval.hpp:73-188,
 * called from runner_doself for the cuboids whose bounding box, widened by the cutoff,
 * meets the particle's cell, :190-201 and :37-55): the particle's global point
 * x_rel + float(cell origin) inside the widened box is taken into the cuboid's frame, and
 * the face it is nearest to (inside) or above (outside) gives the axis: the potential
 * potential_eval_ex(pot, r0 = half size on that axis, radius, distance^2) along that axis,
 * rotated back. No energy is tabulated, as in the reference.
 */
__device__ __noinline__ void cuboid_forces(const EngineView &v, int c, const float4 &x, const DevType &T, float4 &f) {
    const DevSpace &S = v.spaces[v.cell_rep[c]];
    int loc[3];
    cell_loc(S, c, loc);
    const float cut = (float)S.cutoff_d;
    float org[3], bmin[3], bmax[3], pt[3];
    const float xr[3] = {x.x, x.y, x.z};
    for (int k = 0; k < 3; ++k) {
        org[k] = (float)__dadd_rn(S.origin[k], __dmul_rn((double)loc[k], S.hd[k]));
        bmin[k] = org[k] - cut;
        bmax[k] = (org[k] + (float)S.hd[k]) + cut;
        pt[k] = xr[k] + org[k];
    }
    const DevPot &p = v.pots[T.cpot];
    for (int q = 0; q < v.ncuboids; ++q) {
        const DevCuboid &C = v.cuboids[q];
        if (C.rep != v.cell_rep[c]) continue;
        bool meets = true, inside = true;
        for (int k = 0; k < 3; ++k) {
            meets = meets && C.lo[k] <= bmax[k] && C.hi[k] >= bmin[k];
            inside = inside && pt[k] >= C.lo[k] - cut && pt[k] <= C.hi[k] + cut;
        }
        if (!meets || !inside) continue;
        float rel[3] = {pt[0] - C.pos[0], pt[1] - C.pos[1], pt[2] - C.pos[2]}, pl[3];
        quat_rotate(C.qi, rel, pl);
        float dv[3], half[3];
        for (int k = 0; k < 3; ++k) {
            half[k] = C.size[k] / 2.f;
            dv[k] = fabsf(pl[k]) - half[k];
        }
        int ax;
        if (dv[0] < 0 && dv[1] < 0 && dv[2] < 0) {  // inside: the nearest face
            ax = (dv[0] > dv[1] && dv[0] > dv[2]) ? 0 : ((dv[1] > dv[0] && dv[1] > dv[2]) ? 1 : 2);
        } else if (dv[0] < 0 && dv[1] < 0) {
            ax = 2;
        } else if (dv[0] < 0 && dv[2] < 0) {
            ax = 1;
        } else if (dv[1] < 0 && dv[2] < 0) {
            ax = 0;
        } else {
            continue;
        }
        const float dist = fabsf(pl[ax]);
        float ee, ff;
        if (!table_eval_ex(p, v.coef, half[ax], T.radius, __fmul_rn(dist, dist), ee, ff)) continue;
        // -forceVec * force with forceVec zero off the axis (signed zeros kept as the reference forms them)
        float fv[3], fg[3];
        for (int k = 0; k < 3; ++k) fv[k] = (k == ax ? -pl[ax] : -0.f) * ff;
        quat_rotate(C.q, fv, fg);
        f.x += fg[0];
        f.y += fg[1];
        f.z += fg[2];
    }
}

/* Wall potentials of particles in cells next to a bound face, the large particles'
 * interactions and the cuboids' forces (runner_doself's boundary_eval,
 * particle_largecell_force and potential_eval_cuboid_particle, runner_dopair.cpp:
 * 526-535), one thread per slot, before the pass's force kernel; total_force adds the
 * force, the energy goes to the slot's entry. */
__global__ void body_kernel(EngineView v, float4 *body_f) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= v.nparts) return;
    const float4 x = v.pos[s];
    const DevType &T = v.types[__float_as_int(x.w)];
    const int c = v.cell_of[s];
    const unsigned cflags = v.cell_flags[c];
    float4 f = make_float4(0.f, 0.f, 0.f, 0.f);
    double ew = 0.0;
    if (cflags & T.wall_mask) boundary_forces(v, v.spaces[v.cell_rep[c]], cflags, T, T.radius, x, v.vel[s], f, ew);
    if (v.nlarge && !T.large) large_forces(v, s, x, v.vel[s], T.radius, f, ew);
    if (v.ncuboids && T.cpot >= 0) cuboid_forces(v, c, x, T, f);
    body_f[s] = f;
    v.body_e[s] = ew;
}

/* Per type: the summed kinetic energy 0.5 m v^2 (each particle's term in FP32,
 * summed in FP64, engine_kinetic_energy, engine.cpp:1698-1719), the quantity
 * berendsen_force reads. One block per type, fixed summation order. */
__global__ void type_ke_kernel(EngineView v, double *out) {
    __shared__ double part[256];
    const int t = blockIdx.x;
    const double mass = v.types[t].mass;
    double acc = 0.0;
    for (int s = threadIdx.x; s < v.nparts; s += blockDim.x) {
        if (__float_as_int(v.pos[s].w) != t) continue;
        const float4 u = v.vel[s];
        const float e = (float)(0.5 * mass * (double)(u.x * u.x + u.y * u.y + u.z * u.z));
        acc += (double)e;
    }
    part[threadIdx.x] = acc;
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if ((int)threadIdx.x < off) part[threadIdx.x] += part[threadIdx.x + off];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[t] = part[0];
}

/* Redraws the persistent random force of particles whose (time + id) is a
 * multiple of their type's interval (gaussian_force / friction_force,
 * MxForce.cpp:356-381): a normal magnitude N(mean, std) in a uniformly random
 * direction, as MxRandomVector builds it (MxParticle.cpp:1782-1793), drawn from
 * a Philox stream keyed on (time, id) instead of the global mt19937. */
__global__ void persist_kernel(EngineView v, float4 *persist) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= v.nparts) return;
    const DevType &T = v.types[__float_as_int(v.pos[s].w)];
    if (T.sb_kind != 3 && T.sb_kind != 4) return;
    const unsigned id = __float_as_uint(v.vel[s].w);
    const unsigned long long time = *v.step + 1;  // engine_step advances the time before the step
    if ((time + id) % (unsigned long long)T.sb_steps != 0) return;
    const uint4 r = philox4x32(make_uint4(id, 0x52414e44u, (unsigned)time, (unsigned)(time >> 32)),
                               make_uint2(0x46524345u, 0x50455253u));
    const float mean = T.sb_kind == 3 ? T.sb_a : T.sb_b, sd = T.sb_kind == 3 ? T.sb_b : T.sb_c;
    const float g = sqrtf(-2.0f * logf(u01(r.x))) * cospif(2.0f * u01(r.y));
    const float mag = mean + sd * g;
    const float theta = 2.0f * (float)M_PI * u01(r.z);
    const float phi = acosf(1.0f - 2.0f * u01(r.w));
    persist[id] = make_float4(mag * sinf(phi) * cosf(theta), mag * sinf(phi) * sinf(theta), mag * cosf(phi), 0.f);
}

/* Completes the force pass when neither the bond kernel nor the integrator
 * follows it: force = total_force. */
__global__ void combine_kernel(EngineView v) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= v.nparts) return;
    v.force[s] = total_force(v, s);
}

/* ------------------------------------------------------------------------ */
/* bonds                                                                     */
/* ------------------------------------------------------------------------ */

/*
 * The force terms of angle aid exactly as angle_eval computes them
 * (angle.cpp:92-352): positions relative to the vertex j's cell, cos(theta)
 * at j clamped to [-1, 1], the derivatives of cos(theta) with respect to x_i
 * and x_k, the table's [a, b] clamp, and potential_eval_r on the cosine.
 * Returns wi = eff * dcos/dx_i and wk = eff * dcos/dx_k, or false when one of
 * the ids is absent. At cos(theta) = 0 or -1 the reference replaces both
 * derivatives with one random unit vector (a uniform draw in [-1, 1]^3 minus
 * its projection on x_i - x_k, normalised); that draw comes from a Philox
 * stream keyed on (angle, step) here instead of the global mt19937.
 */
__device__ bool angle_terms(const EngineView &v, const BondedView &bv, int aid, float wi[3], float wk[3],
                            float &ee) {
    const DevAngle A = bv.angles[aid];
    if (A.pot < 0) return false;
    const int si = bv.slot_of_id[A.i], sj = bv.slot_of_id[A.j], sk = bv.slot_of_id[A.k];
    if (si < 0 || sj < 0 || sk < 0) return false;
    const int cj = v.cell_of[sj];
    const DevSpace &S = v.spaces[v.cell_rep[cj]];
    int loci[3], locj[3], lock[3];
    cell_loc(S, v.cell_of[si], loci);
    cell_loc(S, cj, locj);
    cell_loc(S, v.cell_of[sk], lock);
    const float4 pi = v.pos[si], pj = v.pos[sj], pk = v.pos[sk];
    const float xiv[3] = {pi.x, pi.y, pi.z}, xj[3] = {pj.x, pj.y, pj.z}, xkv[3] = {pk.x, pk.y, pk.z};
    float xi[3], xk[3], rji[3], rjk[3];
    for (int q = 0; q < 3; ++q) {
        xi[q] = shifted(xiv[q], wrap_shift(loci[q] - locj[q]), S.hd[q]);
        xk[q] = shifted(xkv[q], wrap_shift(lock[q] - locj[q]), S.hd[q]);
        rji[q] = __fsub_rn(xi[q], xj[q]);
        rjk[q] = __fsub_rn(xk[q], xj[q]);
    }
    const float dprod =
        __fadd_rn(__fadd_rn(__fmul_rn(rji[0], rjk[0]), __fmul_rn(rji[1], rjk[1])), __fmul_rn(rji[2], rjk[2]));
    const float inji = __fdiv_rn(1.0f, __fsqrt_rn(dot3_rn(rji[0], rji[1], rji[2])));
    const float injk = __fdiv_rn(1.0f, __fsqrt_rn(dot3_rn(rjk[0], rjk[1], rjk[2])));
    float ct = fmaxf(-1.0f, fminf(1.0f, __fmul_rn(__fmul_rn(dprod, inji), injk)));
    float dxi[3], dxk[3];
    if (ct == 0.0f || ct == -1.0f) {
        const unsigned long long step = *v.step;
        const uint4 r = philox4x32(make_uint4((unsigned)aid, 0x414e474cu, (unsigned)step, (unsigned)(step >> 32)),
                                   make_uint2(0x504c414eu, 0x45524e44u));
        float x[3] = {__fsub_rn(__fmul_rn(2.0f, u01(r.x)), 1.0f), __fsub_rn(__fmul_rn(2.0f, u01(r.y)), 1.0f),
                      __fsub_rn(__fmul_rn(2.0f, u01(r.z)), 1.0f)};
        const float vik[3] = {__fsub_rn(xi[0], xk[0]), __fsub_rn(xi[1], xk[1]), __fsub_rn(xi[2], xk[2])};
        const float d = __fadd_rn(__fadd_rn(__fmul_rn(x[0], vik[0]), __fmul_rn(x[1], vik[1])), __fmul_rn(x[2], vik[2]));
        for (int q = 0; q < 3; ++q) x[q] = __fsub_rn(x[q], __fmul_rn(d, vik[q]));
        const float len = __fsqrt_rn(dot3_rn(x[0], x[1], x[2]));
        for (int q = 0; q < 3; ++q) dxi[q] = dxk[q] = __fdiv_rn(x[q], len);
    } else {
        for (int q = 0; q < 3; ++q) {
            dxi[q] = __fmul_rn(__fsub_rn(__fmul_rn(rjk[q], injk), __fmul_rn(__fmul_rn(ct, rji[q]), inji)), inji);
            dxk[q] = __fmul_rn(__fsub_rn(__fmul_rn(rji[q], inji), __fmul_rn(__fmul_rn(ct, rjk[q]), injk)), injk);
        }
    }
    const DevPot &p = v.pots[A.pot];
    if (ct < p.a || ct > p.b) ct = fmaxf(p.a, fminf(p.b, ct));
    float eff;
    table_eval_r(p, v.coef, ct, ee, eff);
    for (int q = 0; q < 3; ++q) {
        wi[q] = __fmul_rn(eff, dxi[q]);
        wk[q] = __fmul_rn(eff, dxk[q]);
    }
    return true;
}

/*
 * The force terms of dihedral did exactly as dihedral_eval computes them
 * (dihedral.cpp:81-392): positions relative to j's cell, the rays
 * b1 = x_i - x_j, b2 = x_k - x_j, b3 = x_l - x_k, cos(phi) between the planes
 * (i, j, k) and (j, k, l) and its derivatives with respect to x_i, x_j and x_l
 * in the reference's expression order, the clamp to [-1, 1] and to the table's
 * [a, b], and potential_eval_r on the cosine. Returns w = eff * dcos/dx for
 * i, j and l (the k end receives the negated sum), or false when an id is
 * absent.
 */
__device__ bool dihedral_terms(const EngineView &v, const BondedView &bv, int did, float wi[3], float wj[3],
                               float wl[3], float &ee) {
    const DevDihedral D = bv.dihedrals[did];
    if (D.pot < 0) return false;
    const int si = bv.slot_of_id[D.i], sj = bv.slot_of_id[D.j], sk = bv.slot_of_id[D.k], sl = bv.slot_of_id[D.l];
    if (si < 0 || sj < 0 || sk < 0 || sl < 0) return false;
    const int cj = v.cell_of[sj];
    const DevSpace &S = v.spaces[v.cell_rep[cj]];
    int loci[3], locj[3], lock[3], locl[3];
    cell_loc(S, v.cell_of[si], loci);
    cell_loc(S, cj, locj);
    cell_loc(S, v.cell_of[sk], lock);
    cell_loc(S, v.cell_of[sl], locl);
    const float4 pi = v.pos[si], pj = v.pos[sj], pk = v.pos[sk], pl = v.pos[sl];
    const float xiv[3] = {pi.x, pi.y, pi.z}, xj[3] = {pj.x, pj.y, pj.z};
    const float xkv[3] = {pk.x, pk.y, pk.z}, xlv[3] = {pl.x, pl.y, pl.z};
    float xi[3], xk[3], xl[3], b1[3], b2[3], b3[3];
    for (int q = 0; q < 3; ++q) {
        xi[q] = shifted(xiv[q], wrap_shift(loci[q] - locj[q]), S.hd[q]);
        xk[q] = shifted(xkv[q], wrap_shift(lock[q] - locj[q]), S.hd[q]);
        xl[q] = shifted(xlv[q], wrap_shift(locl[q] - locj[q]), S.hd[q]);
        b1[q] = __fsub_rn(xi[q], xj[q]);
        b2[q] = __fsub_rn(xk[q], xj[q]);
        b3[q] = __fsub_rn(xl[q], xk[q]);
    }
#define M(a, b) __fmul_rn(a, b)
#define A(a, b) __fadd_rn(a, b)
#define S_(a, b) __fsub_rn(a, b)
    const float n33 = dot3_rn(b3[0], b3[1], b3[2]);
    const float n22 = dot3_rn(b2[0], b2[1], b2[2]);
    const float n11 = dot3_rn(b1[0], b1[1], b1[2]);
    const float d32 = A(A(M(b3[0], b2[0]), M(b3[1], b2[1])), M(b3[2], b2[2]));      // b3.b2
    const float m12 = S_(S_(M(-b1[0], b2[0]), M(b1[1], b2[1])), M(b1[2], b2[2]));   // -b1.b2
    const float m13 = S_(S_(M(-b1[0], b3[0]), M(b1[1], b3[1])), M(b1[2], b3[2]));   // -b1.b3
    const float g23 = S_(M(n22, n33), M(d32, d32));  // |b2 x b3|^2
    const float g12 = S_(M(n11, n22), M(m12, m12));  // |b1 x b2|^2
    const float g = M(g12, g23);
    const float rg = __fdiv_rn(1.0f, __fsqrt_rn(g));
    const float cphi0 = M(S_(M(m12, d32), M(m13, n22)), rg);
    const float m13x2 = M(2.0f, m13);
    const float pa = M(g12, d32), pb = M(m12, g23), pc = M(g12, n33);
    const float qv = S_(-m12, n22);
    const float rgc = M(__fdiv_rn(1.0f, g), cphi0);
    const float s23 = M(g23, rgc), s12 = M(g12, rgc);
    float u[3], w[3], b1n[3], ddi[3], ddj[3], ddl[3];
    for (int q = 0; q < 3; ++q) {
        b1n[q] = M(b1[q], n22);
        u[q] = A(M(-d32, b2[q]), M(b3[q], n22));   // (b3 n22 - d32 b2)
        w[q] = A(M(m12, b2[q]), b1n[q]);          // (b1 n22 + m12 b2)
    }
    for (int q = 0; q < 3; ++q) {
        const float t = A(S_(xk[q], M(2.0f, xj[q])), xi[q]);  // x_k - 2 x_j + x_i
        ddi[q] = S_(M(u[q], rg), M(w[q], s23));
        ddj[q] = S_(M(A(A(M(t, d32), M(b2[q], m13x2)), M(qv, b3[q])), rg),
                    M(S_(A(A(M(-t, pb), M(b3[q], pa)), M(S_(-b1n[q], M(n11, b2[q])), g23)), M(b2[q], pc)), rgc));
        ddl[q] = S_(M(w[q], rg), M(u[q], s12));
    }
#undef M
#undef A
#undef S_
    float c = fmaxf(-1.0f, fminf(1.0f, cphi0));
    const DevPot &p = v.pots[D.pot];
    if (c < p.a || c > p.b) c = fmaxf(p.a, fminf(p.b, c));
    float eff;
    table_eval_r(p, v.coef, c, ee, eff);
    for (int q = 0; q < 3; ++q) {
        wi[q] = __fmul_rn(eff, ddi[q]);
        wj[q] = __fmul_rn(eff, ddj[q]);
        wl[q] = __fmul_rn(eff, ddl[q]);
    }
    return true;
}

/*
 * The bonded pass (engine_bonded_eval, engine_bonded.cpp:1373-1543:
 * exclusions, bonds, angles, dihedrals). One thread per particle slot; each thread evaluates every
 * bond and angle its particle takes part in and applies its own share, in the
 * bonded lists' index order, so its force receives the same sequence of
 * updates as in the reference's serial loops.
 *
 * Bonds (bond.cpp:99-312) are evaluated from the bond's first particle's point
 * of view; both ends compute the same force/r and the same break decision
 * eff >= dissociation_energy, and the first end clears the active flag.
 * Angles: f_i -= wi, f_k -= wk, f_j += wi + wk; the vertex carries the energy.
 * Dihedrals: f_i -= wi, f_j -= wj, f_l -= wl, f_k += wi + wj + wl; the k end
 * carries the energy.
 */
__global__ void bonded_kernel(EngineView v, BondedView bv) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= v.nparts) return;
    const int id = __float_as_int(v.vel[s].w);
    double eb = 0.0;
    float4 f = total_force(v, s);  // the bonded pass completes the nonbonded force
    // exclusions (exclusion_eval, exclusion.cpp:83-282): the pair's table potential evaluated
    // with potential_eval (no radii shift) on dx = (x_i - x_j) + h shift and taken back,
    // f_i += eff dx, f_j -= eff dx and its energy subtracted, for pairs within the cutoff
    const int x0 = bv.excl_off[id], x1 = bv.excl_off[id + 1];
    for (int k = x0; k < x1; ++k) {
        const int code = bv.excl_list[k];
        const int2 X = bv.excl[code >> 1];
        const int si = bv.slot_of_id[X.x], sj = bv.slot_of_id[X.y];
        if (si < 0 || sj < 0) continue;
        const float4 xi = v.pos[si], xj = v.pos[sj];
        const int ti = __float_as_int(xi.w), tj = __float_as_int(xj.w);
        const int ci = v.cell_of[si], cj = v.cell_of[sj];
        const DevSpace &S = v.spaces[v.cell_rep[ci]];
        const int q = v.pot_idx[S.pot_offset + tj * v.ntypes + ti];
        if (q < 0 || v.pots[q].kind != 0) continue;
        int loci[3], locj[3];
        cell_loc(S, ci, loci);
        cell_loc(S, cj, locj);
        const float xiv[3] = {xi.x, xi.y, xi.z}, xjv[3] = {xj.x, xj.y, xj.z};
        float d[3];
        for (int c3 = 0; c3 < 3; ++c3)
            d[c3] = (float)__dadd_rn((double)__fsub_rn(xiv[c3], xjv[c3]),
                                     __dmul_rn(S.hd[c3], (double)wrap_shift(loci[c3] - locj[c3])));
        const float r2 = dot3_rn(d[0], d[1], d[2]);
        if (r2 > S.cut2_self) continue;
        float ee, eff;
        table_eval(v.pots[q], v.coef, r2, ee, eff);
        const float wx = __fmul_rn(eff, d[0]), wy = __fmul_rn(eff, d[1]), wz = __fmul_rn(eff, d[2]);
        if ((code & 1) == 0) {
            f.x = __fadd_rn(f.x, wx);
            f.y = __fadd_rn(f.y, wy);
            f.z = __fadd_rn(f.z, wz);
            eb -= (double)ee;  // the pair's energy is taken back (exclusion.cpp:279-280)
        } else {
            f.x = __fsub_rn(f.x, wx);
            f.y = __fsub_rn(f.y, wy);
            f.z = __fsub_rn(f.z, wz);
        }
    }
    const int k0 = bv.bond_off[id], k1 = bv.bond_off[id + 1];
    for (int k = k0; k < k1; ++k) {
        const int b = bv.bond_list[k];
        if (!(bv.bond_flags[b] & 1u)) continue;
        const DevBond B = bv.bonds[b];
        const int si = bv.slot_of_id[B.i], sj = bv.slot_of_id[B.j];
        if (si < 0 || sj < 0) continue;
        const int ci = v.cell_of[si];
        const DevSpace &S = v.spaces[v.cell_rep[ci]];
        float d[3];
        bond_vector(S, ci, v.cell_of[sj], v.pos[si], v.pos[sj], d);
        float r2 = dot3_rn(d[0], d[1], d[2]);
        const DevPot &p = v.pots[B.pot];
        const float a2 = __fmul_rn(p.a, p.a), b2 = __fmul_rn(p.b, p.b);
        if (r2 < a2 || r2 > b2) r2 = fmaxf(a2, fminf(b2, r2));
        float ee, eff;
        table_eval(p, v.coef, r2, ee, eff);
        const bool first = (s == si);
        if ((double)eff >= B.dissociation) {
            if (first) bv.bond_flags[b] = 0u;  // MxBond_Destroy (bond.cpp:1001-1013)
            continue;
        }
        const float wx = __fmul_rn(eff, d[0]), wy = __fmul_rn(eff, d[1]), wz = __fmul_rn(eff, d[2]);
        if (first) {
            f.x = __fsub_rn(f.x, wx);
            f.y = __fsub_rn(f.y, wy);
            f.z = __fsub_rn(f.z, wz);
            eb += (double)ee;
        } else {
            f.x = __fadd_rn(f.x, wx);
            f.y = __fadd_rn(f.y, wy);
            f.z = __fadd_rn(f.z, wz);
        }
    }
    const int a0 = bv.angle_off[id], a1 = bv.angle_off[id + 1];
    for (int k = a0; k < a1; ++k) {
        const int code = bv.angle_list[k];
        const int role = code & 3;
        float wi[3], wk[3], ee;
        if (!angle_terms(v, bv, code >> 2, wi, wk, ee)) continue;
        if (role == 0) {
            f.x = __fsub_rn(f.x, wi[0]);
            f.y = __fsub_rn(f.y, wi[1]);
            f.z = __fsub_rn(f.z, wi[2]);
        } else if (role == 2) {
            f.x = __fsub_rn(f.x, wk[0]);
            f.y = __fsub_rn(f.y, wk[1]);
            f.z = __fsub_rn(f.z, wk[2]);
        } else {
            f.x = __fadd_rn(f.x, __fadd_rn(wi[0], wk[0]));
            f.y = __fadd_rn(f.y, __fadd_rn(wi[1], wk[1]));
            f.z = __fadd_rn(f.z, __fadd_rn(wi[2], wk[2]));
            eb += (double)ee;
        }
    }
    const int d0 = bv.dihedral_off[id], d1 = bv.dihedral_off[id + 1];
    for (int k = d0; k < d1; ++k) {
        const int code = bv.dihedral_list[k];
        const int role = code & 3;
        float wi[3], wj[3], wl[3], ee;
        if (!dihedral_terms(v, bv, code >> 2, wi, wj, wl, ee)) continue;
        if (role == 2) {
            f.x = __fadd_rn(f.x, __fadd_rn(__fadd_rn(wi[0], wj[0]), wl[0]));
            f.y = __fadd_rn(f.y, __fadd_rn(__fadd_rn(wi[1], wj[1]), wl[1]));
            f.z = __fadd_rn(f.z, __fadd_rn(__fadd_rn(wi[2], wj[2]), wl[2]));
            eb += (double)ee;
        } else {
            const float *w = role == 0 ? wi : (role == 1 ? wj : wl);
            f.x = __fsub_rn(f.x, w[0]);
            f.y = __fsub_rn(f.y, w[1]);
            f.z = __fsub_rn(f.z, w[2]);
        }
    }
    v.force[s] = f;
    bv.e_slot[s] = eb;
}

constexpr int kVirThreads = 128;

/* A table's value and derivative at s in FP64 on its FP32 coefficients, the interval
 * picked from float(s) as the FP32 code picks it (an integer decision of the model). */
__device__ __forceinline__ void table_value64(const DevPot &p, const float *coef, double sd, double &e, double &dv) {
    const float sf = (float)sd;
    const float t = __fadd_rn(p.alpha0, __fmul_rn(sf, __fadd_rn(p.alpha1, __fmul_rn(sf, p.alpha2))));
    const int ind = min((int)fmaxf(0.0f, t), p.n);
    const float *c = coef + p.coef_off + ind * kChunk;
    const double x = (sd - (double)c[0]) * (double)c[1];
    double ee = (double)c[2] * x + (double)c[3], eff = (double)c[2];
    for (int k = 4; k < 8; ++k) {
        eff = eff * x + ee;
        ee = ee * x + (double)c[k];
    }
    e = ee;
    dv = eff * (double)c[1];
}

/* x_i - x_j in FP64 for particles in cells ci, cj (x_i taken into x_j's frame by the
 * bonded code's wrapped cell shift). */
__device__ __forceinline__ void rel64(const EngineView &v, int si, int sj, double d[3]) {
    const int ci = v.cell_of[si], cj = v.cell_of[sj];
    const DevSpace &S = v.spaces[v.cell_rep[ci]];
    int li[3], lj[3];
    cell_loc(S, ci, li);
    cell_loc(S, cj, lj);
    const float4 a = v.pos[si], b = v.pos[sj];
    const float av[3] = {a.x, a.y, a.z}, bv[3] = {b.x, b.y, b.z};
    for (int q = 0; q < 3; ++q) d[q] = ((double)av[q] + (double)wrap_shift(li[q] - lj[q]) * S.hd[q]) - (double)bv[q];
}

__device__ __forceinline__ void cross64(const double *a, const double *b, double *o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

/* c = u.w / (|u| |w|) and its gradients with respect to u and w. */
__device__ __forceinline__ double cos_grad64(const double *u, const double *w, double *gu, double *gw) {
    const double nu = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    const double nw = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
    const double c = (u[0] * w[0] + u[1] * w[1] + u[2] * w[2]) / (nu * nw);
    for (int q = 0; q < 3; ++q) {
        gu[q] = (w[q] / nw - c * u[q] / nu) / nu;
        gw[q] = (u[q] / nu - c * w[q] / nw) / nw;
    }
    return c;
}

/*
 * The bonded terms' virial, sum over the terms' members of (x_m - x_ref) (x) F_m for the
 * current positions: active bonds (flags after the last pass; a bond whose FP32 f reaches its
 * dissociation energy at these positions would break and adds nothing), d (x) F_i with
 * F_i = -V'(r)/r d; exclusions within the cutoff, d (x) (+V'(r)/r d) (the pair potential taken
 * back, so the pair's term in the nonbonded virial cancels); angles about their vertex,
 * r_ji (x) F_i + r_jk (x) F_k; dihedrals about their j particle,
 * b1 (x) F_i + b2 (x) F_k + (b2 + b3) (x) F_l. Each term is evaluated in FP64 from the FP32
 * positions (the table's interval and clamps decided as in FP32): the FP32 force of a bond
 * near its rest length carries a relative error far above 1e-6 (r - r0 cancels), as the
 * reference's does, and the virial is reported to 1e-6. Degenerate angles (cos = 0 or -1,
 * a random plane in the force pass) add nothing. One thread per term, FP64 sums per thread,
 * per block in thread order; launched only by the energy call.
 */
__global__ void __launch_bounds__(kVirThreads) bonded_virial_kernel(EngineView v, BondedView bv, int nb, int nx,
                                                                    int na, int nd, double *partials) {
    __shared__ double part[kVirThreads * 9];
    double w[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    auto add = [&](const double *r, const double *F) {
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) w[3 * a + b] += r[a] * F[b];
    };
    const int total = nb + nx + na + nd;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        if (t < nb) {
            if (!(bv.bond_flags[t] & 1u)) continue;
            const DevBond B = bv.bonds[t];
            const int si = bv.slot_of_id[B.i], sj = bv.slot_of_id[B.j];
            if (si < 0 || sj < 0) continue;
            const DevPot &p = v.pots[B.pot];
            // the FP32 pass's break decision
            const int ci = v.cell_of[si];
            float df[3];
            bond_vector(v.spaces[v.cell_rep[ci]], ci, v.cell_of[sj], v.pos[si], v.pos[sj], df);
            float r2f = dot3_rn(df[0], df[1], df[2]);
            const float a2 = __fmul_rn(p.a, p.a), b2 = __fmul_rn(p.b, p.b);
            if (r2f < a2 || r2f > b2) r2f = fmaxf(a2, fminf(b2, r2f));
            float ee, eff;
            table_eval(p, v.coef, r2f, ee, eff);
            if ((double)eff >= B.dissociation) continue;
            double d[3];
            rel64(v, si, sj, d);
            const double r = fmin(fmax(sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]), (double)p.a), (double)p.b);
            double e64, dv;
            table_value64(p, v.coef, r, e64, dv);
            const double F[3] = {-dv / r * d[0], -dv / r * d[1], -dv / r * d[2]};
            add(d, F);
        } else if (t < nb + nx) {
            const int2 X = bv.excl[t - nb];
            const int si = bv.slot_of_id[X.x], sj = bv.slot_of_id[X.y];
            if (si < 0 || sj < 0) continue;
            const float4 xi = v.pos[si], xj = v.pos[sj];
            const DevSpace &S = v.spaces[v.cell_rep[v.cell_of[si]]];
            const int q = v.pot_idx[S.pot_offset + __float_as_int(xj.w) * v.ntypes + __float_as_int(xi.w)];
            if (q < 0 || v.pots[q].kind != 0) continue;
            double d[3];
            rel64(v, si, sj, d);
            const float df[3] = {(float)d[0], (float)d[1], (float)d[2]};
            if (dot3_rn(df[0], df[1], df[2]) > S.cut2_self) continue;
            const double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            double e64, dv;
            table_value64(v.pots[q], v.coef, r, e64, dv);
            const double F[3] = {dv / r * d[0], dv / r * d[1], dv / r * d[2]};
            add(d, F);
        } else if (t < nb + nx + na) {
            const DevAngle A = bv.angles[t - nb - nx];
            if (A.pot < 0) continue;
            const int si = bv.slot_of_id[A.i], sj = bv.slot_of_id[A.j], sk = bv.slot_of_id[A.k];
            if (si < 0 || sj < 0 || sk < 0) continue;
            double rji[3], rjk[3], gi[3], gk[3];
            rel64(v, si, sj, rji);
            rel64(v, sk, sj, rjk);
            double c = cos_grad64(rji, rjk, gi, gk);
            if (c == 0.0 || c == -1.0) continue;
            const DevPot &p = v.pots[A.pot];
            c = fmin(fmax(fmin(fmax(c, -1.0), 1.0), (double)p.a), (double)p.b);
            double e64, dv;
            table_value64(p, v.coef, c, e64, dv);
            const double Fi[3] = {-dv * gi[0], -dv * gi[1], -dv * gi[2]}, Fk[3] = {-dv * gk[0], -dv * gk[1], -dv * gk[2]};
            add(rji, Fi);
            add(rjk, Fk);
        } else {
            const DevDihedral D = bv.dihedrals[t - nb - nx - na];
            if (D.pot < 0) continue;
            const int si = bv.slot_of_id[D.i], sj = bv.slot_of_id[D.j], sk = bv.slot_of_id[D.k],
                      sl = bv.slot_of_id[D.l];
            if (si < 0 || sj < 0 || sk < 0 || sl < 0) continue;
            double b1[3], b2[3], b3[3], A3[3], B3[3], gA[3], gB[3];
            rel64(v, si, sj, b1);
            rel64(v, sk, sj, b2);
            rel64(v, sl, sk, b3);
            cross64(b1, b2, A3);
            cross64(b2, b3, B3);
            double c = -cos_grad64(A3, B3, gA, gB);
            for (int q = 0; q < 3; ++q) {
                gA[q] = -gA[q];
                gB[q] = -gB[q];
            }
            double g1[3], g2a[3], g2b[3], g3[3];
            cross64(b2, gA, g1);   // dc/db1 through A = b1 x b2
            cross64(gA, b1, g2a);  // dc/db2 through A
            cross64(b3, gB, g2b);  // dc/db2 through B = b2 x b3
            cross64(gB, b2, g3);   // dc/db3 through B
            const DevPot &p = v.pots[D.pot];
            c = fmin(fmax(fmin(fmax(c, -1.0), 1.0), (double)p.a), (double)p.b);
            double e64, dv;
            table_value64(p, v.coef, c, e64, dv);
            double Fi[3], Fk[3], Fl[3], rl[3];
            for (int q = 0; q < 3; ++q) {
                const double wi = dv * g1[q], wj = dv * (-g1[q] - g2a[q] - g2b[q]), wl = dv * g3[q];
                Fi[q] = -wi;
                Fl[q] = -wl;
                Fk[q] = wi + wj + wl;
                rl[q] = b2[q] + b3[q];
            }
            add(b1, Fi);
            add(b2, Fk);
            add(rl, Fl);
        }
    }
    for (int k = 0; k < 9; ++k) part[threadIdx.x * 9 + k] = w[k];
    __syncthreads();
    if (threadIdx.x < 9) {
        double s9 = 0.0;
        for (int r = 0; r < (int)blockDim.x; ++r) s9 += part[r * 9 + threadIdx.x];
        partials[(size_t)blockIdx.x * 9 + threadIdx.x] = s9;
    }
}

/* out9 += the bonded virial from the blocks' partials, in block order. */
__global__ void bonded_virial_reduce_kernel(const double *partials, int nblocks, double *out9) {
    const int k = threadIdx.x;
    if (k >= 9) return;
    double t = 0.0;
    for (int q = 0; q < nblocks; ++q) t += partials[(size_t)q * 9 + k];
    out9[k] += t;
}

/* ------------------------------------------------------------------------ */
/* integrator                                                                */
/* ------------------------------------------------------------------------ */

/* space_shuffle_local's rule (space.cpp:352-371): delta = (x >= h) - (x < 0). */
__device__ __forceinline__ int cell_delta(float x, float h) { return (x >= h ? 1 : 0) - (x < 0.0f ? 1 : 0); }

/* The move of a particle that left cell c by delta (engine_advance.cpp:204-211):
 * x -= delta*h and the destination by the periodic wrap; then the next force
 * pass's shuffle rule (space.cpp:333-393) once more. Returns the destination. */
__device__ __forceinline__ int relocate(const DevSpace &S, int c, float *xv, int *delta) {
    const int l = c - S.cell_offset;
    int loc[3] = {l / (S.cdim[1] * S.cdim[2]), (l / S.cdim[2]) % S.cdim[1], l % S.cdim[2]};
    for (int pass = 0; pass < 2; ++pass) {
        for (int k = 0; k < 3; ++k) {
            xv[k] = __fsub_rn(xv[k], __fmul_rn((float)delta[k], S.h[k]));
            loc[k] = (loc[k] + delta[k] + S.cdim[k]) % S.cdim[k];
        }
        for (int k = 0; k < 3; ++k) delta[k] = cell_delta(xv[k], S.h[k]);
        if (!(delta[0] | delta[1] | delta[2])) break;
    }
    return S.cell_offset + (loc[0] * S.cdim[1] + loc[1]) * S.cdim[2] + loc[2];
}

/* Appends a particle that moved from cell c to dest to dest's bucket, or, when
 * the bucket is full, to the step's overflow list (at most one entry per
 * particle, so nparts entries always suffice). The reference has no limit on
 * the particles entering a cell (space_cell_add_incomming, space_cell.cpp:
 * 260-290), and neither has this engine. A move between chunks of cells also
 * updates the two chunks' net counts, from which the re-binning forms each
 * cell's new start without a scan over all cells. */
__device__ __forceinline__ void bucket_move(const EngineView &v, int s, int c, int dest, int *in_count, int *in_list,
                                            int *out_count) {
    const int k = atomicAdd(&in_count[dest], 1);
    if (k < kBucket)
        in_list[dest * kBucket + k] = s;
    else
        v.ovf_list[atomicAdd(v.ovf_count, 1)] = s;
    atomicAdd(&out_count[c], 1);
    if ((c >> kChunkShift) != (dest >> kChunkShift)) {
        atomicAdd(&v.chunk_delta[dest >> kChunkShift], 1);
        atomicSub(&v.chunk_delta[c >> kChunkShift], 1);
    }
}

/*
 * Forward Euler for one particle (engine_advance.cpp:126-239): velocity update
 * in FP64 rounded to FP32, per-component speed (or step) clamp, position update,
 * wall reflection (boundary_eval.hpp:30-122), and the move to a neighbour cell
 * with x -= delta*h. The next step's space_shuffle_local rule is applied once
 * more to the moved particle, as engine_force does before the next force pass.
 * Moved particles are appended to the destination cell's bucket (or the overflow list);
 * stayers are counted implicitly (count_old - out + in).
 */
__device__ __forceinline__ void integrate_one(int s, const EngineView &v, float4 *pos, float4 *vel, int *new_cell,
                                              int *in_count, int *in_list, int *out_count, bool add_planes) {
    if (s >= v.nparts) return;
    const int c = v.cell_of[s];
    const DevSpace &S = v.spaces[v.cell_rep[c]];
    float4 x = pos[s];
    float4 u = vel[s];
    const float4 f = add_planes ? total_force(v, s) : v.force[s];
    if (add_planes) v.force[s] = f;  // the integrator completes the nonbonded force
    const DevType &T = v.types[__float_as_int(x.w)];
    const unsigned fz_all = (1u << 2) | (1u << 3) | (1u << 4);
    int dest = c;
    if ((T.flags & fz_all) != fz_all) {
        const float dt = S.dt;
        const double imass = T.imass;
        float xv[3] = {x.x, x.y, x.z}, vv[3] = {u.x, u.y, u.z};
        const float fv[3] = {f.x, f.y, f.z};
        int delta[3];
        bool toofast = false;
        for (int k = 0; k < 3; ++k) {
            const float mask = (T.flags & (1u << (2 + k))) ? 0.0f : 1.0f;
            if (T.dynamics == 0) {
                const double inner = __dadd_rn((double)vv[k], __dmul_rn((double)__fmul_rn(dt, fv[k]), imass));
                const float vk = (float)__dmul_rn((double)mask, inner);
                const float neg = __fdiv_rn(vk, fabsf(vk));
                vv[k] = __fmul_rn(vk, vk) <= S.maxv2[k] ? vk : __fmul_rn(neg, S.maxv[k]);
                xv[k] = __fadd_rn(xv[k], __fmul_rn(dt, vv[k]));
            } else {
                const float dxk = (float)__dmul_rn((double)mask, __dmul_rn((double)__fmul_rn(dt, fv[k]), imass));
                const float neg = __fdiv_rn(dxk, fabsf(dxk));
                xv[k] = __fadd_rn(xv[k], __fmul_rn(dxk, dxk) <= S.maxx2[k] ? dxk : __fmul_rn(neg, S.maxx[k]));
            }
            delta[k] = cell_delta(xv[k], S.h[k]);
            toofast = toofast || (xv[k] >= S.h2[k] || xv[k] <= -S.h[k]);
        }
        if (toofast) atomicOr(v.status, kStatusTooFast);
        if (!(isfinite(xv[0]) && isfinite(xv[1]) && isfinite(xv[2]))) atomicOr(v.status, kStatusNonFinite);
        if (delta[0] | delta[1] | delta[2]) {
            // apply_update_pos_vel: reflect at active walls, in face order
            const unsigned cf = v.cell_flags[c];
            bool enforced = false;
            const unsigned lowbit[3] = {kCellActiveLeft, kCellActiveFront, kCellActiveBottom};
            const unsigned highbit[3] = {kCellActiveRight, kCellActiveBack, kCellActiveTop};
            for (int k = 0; k < 3; ++k) {
                const int lo = 2 * k, hi = 2 * k + 1;
                if ((cf & lowbit[k]) && xv[k] <= 0.0f) {
                    if (S.bc_kind[lo] & kBcFreeslip) {
                        xv[k] = __fmul_rn(-xv[k], 1.0f);
                        vv[k] = __fmul_rn(vv[k], -1.0f);
                        enforced = true;
                    } else if (S.bc_kind[lo] & kBcVelocity) {
                        const float rs = S.bc_restore[lo];
                        xv[k] = __fmul_rn(-xv[k], rs);
                        for (int q = 0; q < 3; ++q)
                            vv[q] = __fsub_rn(__fmul_rn(2.0f, S.bc_vel[lo][q]), __fmul_rn(vv[q], rs));
                        enforced = true;
                    }
                }
                if ((cf & highbit[k]) && (double)xv[k] >= S.hd[k]) {
                    if (S.bc_kind[hi] & kBcFreeslip) {
                        xv[k] = (float)__dsub_rn(S.hd[k], __dmul_rn(__dsub_rn((double)xv[k], S.hd[k]), 1.0));
                        vv[k] = __fmul_rn(vv[k], -1.0f);
                        enforced = true;
                    } else if (S.bc_kind[hi] & kBcVelocity) {
                        const float rs = S.bc_restore[hi];
                        xv[k] = (float)__dsub_rn(__dmul_rn(2.0, S.hd[k]), (double)__fmul_rn(xv[k], rs));
                        for (int q = 0; q < 3; ++q)
                            vv[q] = __fsub_rn(__fmul_rn(2.0f, S.bc_vel[hi][q]), __fmul_rn(vv[q], rs));
                        enforced = true;
                    }
                }
            }
            if (enforced)
                for (int k = 0; k < 3; ++k) delta[k] = cell_delta(xv[k], S.h[k]);
            if (delta[0] | delta[1] | delta[2]) dest = relocate(S, c, xv, delta);
        }
        x.x = xv[0]; x.y = xv[1]; x.z = xv[2];
        u.x = vv[0]; u.y = vv[1]; u.z = vv[2];
        pos[s] = x;
        vel[s] = u;
    }
    new_cell[s] = dest;
    if (dest != c) bucket_move(v, s, c, dest, in_count, in_list, out_count);
}

/*
 * Runge-Kutta 4 (engine_advance_runge_kutta_4, engine_advance.cpp:443-698), in
 * the reference's FP32 expression order: the force of stage k gives
 * vk = f imass and xk (v0, v0 + dt/2 vk_{k-1}, ..., or f imass when
 * overdamped); the weighted sums xk0 + 2 xk1 + 2 xk2 + xk3 (and vk) accumulate
 * in that order. Stage positions p0 + dt/2 xk (p0 + dt xk2 for the last) stay
 * in the step's starting cell, whose frame p0 belongs to. (The reference's
 * engine_force re-bins between stages and leaves p0 in the old cell's frame,
 * so there a particle that crosses a face mid-step lands a cell edge away;
 * here the stages keep one frame.) Velocities change only at the end; like
 * the reference, no speed clamp, no frozen mask and no wall reflection.
 */
struct RkState {
    float4 *p0, *v0;       // step start
    float4 *accx, *accv;   // weighted sums of the stages so far
    float4 *vkp;           // previous stage's vk
};

__global__ void rk_stage_kernel(EngineView v, float4 *pos, RkState rk, int stage, bool add_planes) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= v.nparts) return;
    const DevSpace &S = v.spaces[v.cell_rep[v.cell_of[s]]];
    const float4 x = pos[s];
    const float4 f = add_planes ? total_force(v, s) : v.force[s];
    if (add_planes) v.force[s] = f;
    const DevType &T = v.types[__float_as_int(x.w)];
    const float imf = (float)T.imass;
    const float dtf = S.dt;
    const float hdt = (float)(0.5 * (double)dtf);
    const bool newton = T.dynamics == 0;
    float4 p0, v0, vkp = make_float4(0.f, 0.f, 0.f, 0.f);
    if (stage == 0) {
        p0 = x;
        v0 = v.vel[s];
        rk.p0[s] = p0;
        rk.v0[s] = v0;
    } else {
        p0 = rk.p0[s];
        v0 = rk.v0[s];
        vkp = rk.vkp[s];
    }
    const float fv[3] = {f.x, f.y, f.z}, pv[3] = {p0.x, p0.y, p0.z}, vv[3] = {v0.x, v0.y, v0.z};
    const float kv[3] = {vkp.x, vkp.y, vkp.z};
    float vk[3], xk[3], nx[3];
    bool toofast = false;
    const float4 ax = stage ? rk.accx[s] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 av = stage ? rk.accv[s] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float axv[3] = {ax.x, ax.y, ax.z}, avv[3] = {av.x, av.y, av.z};
    float nax[3], nav[3];
    const float step = stage == 2 ? dtf : hdt;
    for (int k = 0; k < 3; ++k) {
        vk[k] = __fmul_rn(fv[k], imf);
        xk[k] = newton ? (stage == 0 ? vv[k] : __fadd_rn(vv[k], __fmul_rn(hdt, kv[k]))) : vk[k];
        nax[k] = stage == 0 ? xk[k] : __fadd_rn(axv[k], __fmul_rn(2.0f, xk[k]));
        nav[k] = stage == 0 ? vk[k] : __fadd_rn(avv[k], __fmul_rn(2.0f, vk[k]));
        nx[k] = __fadd_rn(pv[k], __fmul_rn(step, xk[k]));
        toofast = toofast || nx[k] >= S.h2[k] || nx[k] <= -S.h[k];  // CHECK_TOOFAST (:424-431)
    }
    if (toofast) atomicOr(v.status, kStatusTooFast);
    rk.accx[s] = make_float4(nax[0], nax[1], nax[2], 0.f);
    rk.accv[s] = make_float4(nav[0], nav[1], nav[2], 0.f);
    rk.vkp[s] = make_float4(vk[0], vk[1], vk[2], 0.f);
    pos[s] = make_float4(nx[0], nx[1], nx[2], x.w);
}

__device__ __forceinline__ void rk_final_one(int s, const EngineView &v, float4 *pos, float4 *vel, const RkState &rk,
                                             int *new_cell, int *in_count, int *in_list, int *out_count,
                                             bool add_planes) {
    if (s >= v.nparts) return;
    const int c = v.cell_of[s];
    const DevSpace &S = v.spaces[v.cell_rep[c]];
    const float4 f = add_planes ? total_force(v, s) : v.force[s];
    if (add_planes) v.force[s] = f;
    const float4 x = pos[s];
    const DevType &T = v.types[__float_as_int(x.w)];
    const float imf = (float)T.imass;
    const float dtf = S.dt;
    const float sixth = (float)((double)dtf / 6.);
    const bool newton = T.dynamics == 0;
    const float4 p0 = rk.p0[s], v0 = rk.v0[s], vkp = rk.vkp[s], ax = rk.accx[s], av = rk.accv[s];
    const float fv[3] = {f.x, f.y, f.z}, pv[3] = {p0.x, p0.y, p0.z}, vv[3] = {v0.x, v0.y, v0.z};
    const float kv[3] = {vkp.x, vkp.y, vkp.z}, axv[3] = {ax.x, ax.y, ax.z}, avv[3] = {av.x, av.y, av.z};
    float xv[3], nv[3] = {vv[0], vv[1], vv[2]};
    bool toofast = false;
    int delta[3];
    for (int k = 0; k < 3; ++k) {
        const float vk = __fmul_rn(imf, fv[k]);
        const float xk = newton ? __fadd_rn(vv[k], __fmul_rn(dtf, kv[k])) : vk;
        if (newton) nv[k] = __fadd_rn(vv[k], __fmul_rn(sixth, __fadd_rn(avv[k], vk)));
        xv[k] = __fadd_rn(pv[k], __fmul_rn(sixth, __fadd_rn(axv[k], xk)));
        delta[k] = cell_delta(xv[k], S.h[k]);
        toofast = toofast || xv[k] >= S.h2[k] || xv[k] <= -S.h[k];
    }
    if (toofast) atomicOr(v.status, kStatusTooFast);
    if (!(isfinite(xv[0]) && isfinite(xv[1]) && isfinite(xv[2]))) atomicOr(v.status, kStatusNonFinite);
    int dest = c;
    if (delta[0] | delta[1] | delta[2]) dest = relocate(S, c, xv, delta);
    pos[s] = make_float4(xv[0], xv[1], xv[2], x.w);
    vel[s] = make_float4(nv[0], nv[1], nv[2], v0.w);
    new_cell[s] = dest;
    if (dest != c) bucket_move(v, s, c, dest, in_count, in_list, out_count);
}

/* ------------------------------------------------------------------------ */
/* re-binning                                                                */
/* ------------------------------------------------------------------------ */

constexpr int kAdvThreads = 256;   // integrator blocks

__global__ void __launch_bounds__(kAdvThreads, 4) integrate_kernel(EngineView v, float4 *pos, float4 *vel,
                                                                int *new_cell, int *in_count, int *in_list,
                                                                int *out_count, bool add_planes) {
    integrate_one(blockIdx.x * blockDim.x + threadIdx.x, v, pos, vel, new_cell, in_count, in_list, out_count,
                  add_planes);
}

__global__ void __launch_bounds__(kAdvThreads, 4) rk_final_kernel(EngineView v, float4 *pos, float4 *vel, RkState rk,
                                                               int *new_cell, int *in_count, int *in_list,
                                                               int *out_count, bool add_planes) {
    rk_final_one(blockIdx.x * blockDim.x + threadIdx.x, v, pos, vel, rk, new_cell, in_count, in_list, out_count,
                 add_planes);
}

/*
 * The stable re-binning into the other buffer: one warp per destination cell, kScatterWarps
 * consecutive cells per block. The cell's new start needs no scan over all cells: it is its
 * old start plus the net number of movers into the cells before it, which the block sums from
 * the integrator's per-chunk net counts (chunks before the block's own) and the per-cell
 * counts of its chunk before its first cell; the block's cells then add up their new counts
 * in order. Stayers keep their relative order (ascending id); movers from the cell's bucket
 * and from the overflow list are merged in by id, so every cell stays sorted by id and the
 * layout does not depend on thread scheduling. The warp then computes the new cell's
 * projection-key bounds for the next force pass.
 *
 * The counts of this step are read by other blocks and stay as they are; the block clears its
 * cells' counts of the other buffer parity (and the grid that parity's chunk counts), which the
 * next step uses. The block that finishes last re-arms its done counter and the overflow list
 * and advances the step counter that keys the Philox streams.
 */
__global__ void __launch_bounds__(kScatterWarps * 32, 5) scatter_kernel(
    EngineView v, int ncells, const float4 *__restrict__ pos, const float4 *__restrict__ vel,
    const int *__restrict__ new_cell, const int *__restrict__ old_start, const int *__restrict__ old_count,
    const int *__restrict__ in_count, const int *__restrict__ in_list, const int *__restrict__ out_count,
    int *new_start, int *new_count, float4 *pos_out, float4 *vel_out, int *cell_out, int *slot_of_id,
    int *clear_in, int *clear_out, int *clear_chunk, int nchunks, unsigned *done, unsigned long long *step) {
    __shared__ int s_net[kScatterWarps], s_n[kScatterWarps];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int c0 = blockIdx.x * kScatterWarps, c = c0 + wid;
    {
        // net movers into the cells [0, c0): whole chunks, then the cells of c0's chunk before c0
        const int k0 = c0 >> kChunkShift, cb = k0 << kChunkShift;
        int net = 0;
        for (int j = tid; j < k0; j += blockDim.x) net += v.chunk_delta[j];
        for (int q = cb + 4 * tid; q < c0; q += 4 * blockDim.x) {  // [cb, c0) holds whole int4 groups
            const int4 a = *reinterpret_cast<const int4 *>(in_count + q);
            const int4 b = *reinterpret_cast<const int4 *>(out_count + q);
            net += ((a.x + a.y) + (a.z + a.w)) - ((b.x + b.y) + (b.z + b.w));
        }
        net = __reduce_add_sync(kFull, net);
        if (lane == 0) {
            s_net[wid] = net;
            s_n[wid] = c < ncells ? old_count[c] - out_count[c] + in_count[c] : 0;
        }
        for (int j = blockIdx.x * blockDim.x + tid; j < nchunks; j += gridDim.x * blockDim.x) clear_chunk[j] = 0;
        __syncthreads();
    }
    if (c < ncells) {
        int base = old_start[c0];
        for (int w = 0; w < kScatterWarps; ++w) base += s_net[w] + (w < wid ? s_n[w] : 0);
        const int os = old_start[c], on = old_count[c];
        const int mtot = in_count[c];
        const int m = min(mtot, kBucket);
        const int nov = mtot > kBucket ? *v.ovf_count : 0;  // the overflow list is scanned only when needed
        // movers into c with an id below myid: from the bucket, then from the overflow list
        auto movers_below = [&](int myid) {
            int r = 0;
            for (int q = 0; q < m; ++q) r += __float_as_int(vel[in_list[c * kBucket + q]].w) < myid;
            for (int q = 0; q < nov; ++q) {
                const int src = v.ovf_list[q];
                r += new_cell[src] == c && __float_as_int(vel[src].w) < myid;
            }
            return r;
        };
        auto stayers_below = [&](int myid) {
            int r = 0;
            for (int k = 0; k < on; ++k) r += (new_cell[os + k] == c) && (__float_as_int(vel[os + k].w) < myid);
            return r;
        };
        auto place = [&](int src, int myid, int dst) {
            pos_out[dst] = pos[src];
            vel_out[dst] = vel[src];
            cell_out[dst] = c;
            slot_of_id[myid] = dst;
        };
        // stayers
        int stay_before = 0;
        for (int k0 = 0; k0 < on; k0 += 32) {
            const int k = k0 + lane;
            bool stay = false;
            int myid = 0;
            if (k < on) {
                stay = new_cell[os + k] == c;
                myid = __float_as_int(vel[os + k].w);
            }
            const unsigned bal = __ballot_sync(kFull, stay);
            if (stay) place(os + k, myid, base + stay_before + __popc(bal & ((1u << lane) - 1u)) + movers_below(myid));
            stay_before += __popc(bal);
        }
        // movers of the bucket
        for (int q0 = 0; q0 < m; q0 += 32) {
            const int q = q0 + lane;
            if (q < m) {
                const int src = in_list[c * kBucket + q];
                const int myid = __float_as_int(vel[src].w);
                place(src, myid, base + stayers_below(myid) + movers_below(myid));
            }
        }
        // movers of the overflow list
        for (int q0 = 0; q0 < nov; q0 += 32) {
            const int q = q0 + lane;
            if (q < nov) {
                const int src = v.ovf_list[q];
                if (new_cell[src] == c) {
                    const int myid = __float_as_int(vel[src].w);
                    place(src, myid, base + stayers_below(myid) + movers_below(myid));
                }
            }
        }
        const int nn = stay_before + mtot;
        if (lane == 0) {
            new_start[c] = base;
            new_count[c] = nn;
            if (c == ncells - 1) new_start[ncells] = base + nn;
            clear_in[c] = 0;
            clear_out[c] = 0;
        }
        // the next force pass's cell-pair exit test reads the new cell's key bounds from the slots
        // just written (the barrier makes the lanes' stores visible to the whole warp)
        const DevSpace &S = v.spaces[v.cell_rep[c]];
        __syncwarp();
        if (nn > 0 && (S.prune & 2))
            cell_sort_bounds(pos_out, base, nn, S.sort_bias, S.sort_dscale, v.axes, v.sort_bounds + c * 13);
    }
    __syncthreads();
    if (tid == 0) {
        __threadfence();
        if (atomicAdd(done, 1u) == gridDim.x - 1) {  // every block is done with the overflow list
            *v.ovf_count = 0;
            *done = 0u;
            *step += 1;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* device-side load and unload                                               */
/* ------------------------------------------------------------------------ */

/*
 * engine_load's placement (space_addpart, space.cpp:431-451, and the first
 * shuffle's rule, space.cpp:352-371) per particle id, on the device: the cell
 * index (int)((x - origin) ih), the cell-relative position float(x - (origin +
 * l h)) in double, one move by delta = (x >= h) - (x < 0) in float; counts
 * the new occupancy. Same arithmetic as the host placement, so the cells and
 * the FP32 positions are bit-identical to it.
 */
__global__ void place_kernel(EngineView v, LoadView ld, int *count) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ld.n) return;
    const DevSpace &S = v.spaces[ld.rep_of_id[p]];
    int ind[3];
    double x[3];
    for (int k = 0; k < 3; ++k) {
        x[k] = ld.x[3 * (size_t)p + k];
        ind[k] = (int)__dmul_rn(__dsub_rn(x[k], S.origin[k]), S.ih[k]);
    }
    if (ind[0] < 0 || ind[0] >= S.cdim[0] || ind[1] < 0 || ind[1] >= S.cdim[1] || ind[2] < 0 || ind[2] >= S.cdim[2]) {
        ld.cell[p] = -1;
        atomicExch(ld.err, 1);
        return;
    }
    float xr[3];
    int delta[3];
    for (int k = 0; k < 3; ++k) {
        xr[k] = (float)__dsub_rn(x[k], __dadd_rn(S.origin[k], __dmul_rn((double)ind[k], S.hd[k])));
        delta[k] = cell_delta(xr[k], S.h[k]);
    }
    if (delta[0] | delta[1] | delta[2])
        for (int k = 0; k < 3; ++k) {
            xr[k] = __fsub_rn(xr[k], __fmul_rn((float)delta[k], S.h[k]));
            ind[k] = (ind[k] + delta[k] + S.cdim[k]) % S.cdim[k];
        }
    const int c = S.cell_offset + (ind[0] * S.cdim[1] + ind[1]) * S.cdim[2] + ind[2];
    ld.cell[p] = c;
    ld.xr[p] = make_float4(xr[0], xr[1], xr[2], __int_as_float(ld.type_of_id[p]));
    // a kept velocity is copied out before the ordering overwrites the slot arrays (given
    // velocities are read by the ordering itself)
    if (!ld.v) {
        float4 u = v.vel[ld.slot_now[p]];
        u.w = __int_as_float(p);
        ld.vel[p] = u;
    }
    atomicAdd(&count[c], 1);
}

/* Exclusive scan of the new occupancy into start[0..ncells] and a copy of the counts (one
 * block, tiles of 8192 cells): a tile's counts are loaded coalesced into shared memory
 * (every load in flight at once; a padding word after each run of eight keeps a thread's
 * run in distinct banks), each thread sums its run of eight, the block scans the run totals
 * (warp shuffles, then the warp totals) and the starts go back out coalesced. Nothing is
 * written when the placement found a particle outside its box. */
constexpr int kScanPer = 8;
constexpr int kScanTile = 1024 * kScanPer;
__device__ __forceinline__ int scan_slot(int i) { return i + i / kScanPer; }
__global__ void __launch_bounds__(1024) load_scan_kernel(const int *__restrict__ count, int ncells, int *start,
                                                         int *count_out, const int *err) {
    __shared__ int tile[kScanTile + kScanTile / kScanPer];
    __shared__ int warp_sums[32];
    if (*err) return;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    int carry = 0;
    for (int t0 = 0; t0 < ncells; t0 += kScanTile) {
        const int m = min(kScanTile, ncells - t0);
#pragma unroll
        for (int k = 0; k < kScanPer; ++k) {
            const int i = k * 1024 + tid;
            const int ci = i < m ? count[t0 + i] : 0;
            tile[scan_slot(i)] = ci;
            if (i < m) count_out[t0 + i] = ci;
        }
        __syncthreads();
        int c[kScanPer], run = 0;
#pragma unroll
        for (int k = 0; k < kScanPer; ++k) {
            c[k] = tile[scan_slot(tid * kScanPer + k)];
            run += c[k];
        }
        int incl = run;
        for (int d = 1; d < 32; d <<= 1) {
            const int t = __shfl_up_sync(kFull, incl, d);
            if (lane >= d) incl += t;
        }
        if (lane == 31) warp_sums[wid] = incl;
        __syncthreads();
        if (wid == 0) {
            int w = warp_sums[lane];
            for (int d = 1; d < 32; d <<= 1) {
                const int t = __shfl_up_sync(kFull, w, d);
                if (lane >= d) w += t;
            }
            warp_sums[lane] = w;
        }
        __syncthreads();
        int excl = carry + (wid ? warp_sums[wid - 1] : 0) + incl - run;
#pragma unroll
        for (int k = 0; k < kScanPer; ++k) {
            tile[scan_slot(tid * kScanPer + k)] = excl;
            excl += c[k];
        }
        carry += warp_sums[31];
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kScanPer; ++k) {
            const int i = k * 1024 + tid;
            if (i < m) start[t0 + i] = tile[scan_slot(i)];
        }
        __syncthreads();
    }
    if (tid == 0) start[ncells] = carry;
}

/* Each particle takes a place in its cell's range (in any order; ordered next). */
__global__ void load_fill_kernel(LoadView ld, const int *__restrict__ start) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ld.n || *ld.err) return;
    const int c = ld.cell[p];
    ld.ids[start[c] + atomicAdd(&ld.fill[c], 1)] = p;
}

/* One warp per cell: its particles in ascending id (rank = number of smaller ids in the
 * cell, compared through warp shuffles), written to the slot arrays, then the cell's
 * projection-key bounds. Nothing is written when the placement failed. */
__global__ void load_order_kernel(EngineView v, LoadView ld, const int *__restrict__ start, float4 *pos_out,
                                  float4 *vel_out, int *cell_out, int *slot_of_id, int2 *sort_bounds) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    if (*ld.err) return;
    for (int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < v.ncells; c += warps) {
        const int s0 = start[c], n = start[c + 1] - s0;
        for (int k0 = 0; k0 < n; k0 += 32) {
            const int k = k0 + lane;
            const int id = k < n ? ld.ids[s0 + k] : 0x7fffffff;
            int rank = 0;
            for (int b0 = 0; b0 < n; b0 += 32) {
                const int other = b0 == k0 ? id : (b0 + lane < n ? ld.ids[s0 + b0 + lane] : 0x7fffffff);
                const int m = min(32, n - b0);
                for (int q = 0; q < m; ++q) rank += __shfl_sync(kFull, other, q) < id;
            }
            if (k < n) {
                const int dst = s0 + rank;
                pos_out[dst] = ld.xr[id];
                if (!ld.v) vel_out[dst] = ld.vel[id];  // given velocities: load_vel_kernel
                cell_out[dst] = c;
                slot_of_id[id] = dst;
            }
        }
        __syncwarp();
        const DevSpace &S = v.spaces[v.cell_rep[c]];
        if (n > 0 && (S.prune & 2)) cell_sort_bounds(pos_out, s0, n, S.sort_bias, S.sort_dscale, v.axes, sort_bounds + c * 13);
    }
}

/* Given velocities into their particles' new slots (after the ordering, once the copy of
 * the velocities has arrived); w = id. */
__global__ void load_vel_kernel(LoadView ld, const int *__restrict__ slot_of_id, float4 *vel_out) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ld.n || *ld.err) return;
    vel_out[slot_of_id[p]] = make_float4(ld.v[3 * (size_t)p], ld.v[3 * (size_t)p + 1], ld.v[3 * (size_t)p + 2],
                                         __int_as_float(p));
}

/* engine_unload's arrays by particle id (engine.cpp:620-784): the global position
 * cell origin + x_rel in double, the velocity, the force of the last pass (from the slot
 * order it was computed in: force_ids = that layout's velocities, w = id), the cell and
 * the cell-relative position. Any output may be null. */
__global__ void unload_kernel(EngineView v, const float4 *__restrict__ force_ids, double *x_out, float *v_out,
                              float *f_out, int *cell_out, float *xrel_out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= v.nparts) return;
    const float4 q = v.pos[s], u = v.vel[s];
    const int id = __float_as_int(u.w);
    const int c = v.cell_of[s];
    if (x_out || xrel_out) {
        const DevSpace &S = v.spaces[v.cell_rep[c]];
        int loc[3];
        cell_loc(S, c, loc);
        const float xr[3] = {q.x, q.y, q.z};
        for (int k = 0; k < 3; ++k) {
            if (x_out)
                x_out[3 * (size_t)id + k] =
                    __dadd_rn(__dadd_rn(S.origin[k], __dmul_rn((double)loc[k], S.hd[k])), (double)xr[k]);
            if (xrel_out) xrel_out[3 * (size_t)id + k] = xr[k];
        }
    }
    if (v_out) {
        v_out[3 * (size_t)id] = u.x;
        v_out[3 * (size_t)id + 1] = u.y;
        v_out[3 * (size_t)id + 2] = u.z;
    }
    if (cell_out) cell_out[id] = c;
    if (f_out) {
        const float4 f = v.force[s];
        const int fid = __float_as_int(force_ids[s].w);
        f_out[3 * (size_t)fid] = f.x;
        f_out[3 * (size_t)fid + 1] = f.y;
        f_out[3 * (size_t)fid + 2] = f.z;
    }
}

/* ------------------------------------------------------------------------ */
/* energies (FP64)                                                           */
/* ------------------------------------------------------------------------ */

/* Deterministic two-stage sums: block partials, then one block. */
__global__ void reduce_energy_kernel(int ncells, const double *__restrict__ epot_cell, int nparts,
                                     const double *__restrict__ ebond_slot, const double *__restrict__ body_e,
                                     const float4 *__restrict__ vel,
                                     const float4 *__restrict__ pos, const DevType *__restrict__ types,
                                     double *partials) {
    __shared__ double s_pot[256], s_kin[256];
    double ep = 0.0, ek = 0.0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncells; c += gridDim.x * blockDim.x) ep += epot_cell[c];
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nparts; s += gridDim.x * blockDim.x) {
        if (ebond_slot) ep += ebond_slot[s];
        if (body_e) ep += body_e[s];
        const float4 u = vel[s];
        const DevType &T = types[__float_as_int(pos[s].w)];
        // engine_kinetic_energy (engine.cpp:1698-1719): float e = 0.5*mass*|v|^2
        const float e = (float)__dmul_rn(__dmul_rn(0.5, T.mass), (double)dot3_rn(u.x, u.y, u.z));
        ek += (double)e;
    }
    s_pot[threadIdx.x] = ep;
    s_kin[threadIdx.x] = ek;
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) {
            s_pot[threadIdx.x] += s_pot[threadIdx.x + off];
            s_kin[threadIdx.x] += s_kin[threadIdx.x + off];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = s_pot[0];
        partials[2 * blockIdx.x + 1] = s_kin[0];
    }
}

__global__ void reduce_final_kernel(int nblocks, const double *partials, double *out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int k = 0; k < nblocks; ++k) {
            a += partials[2 * k];
            b += partials[2 * k + 1];
        }
        out[0] = a;
        out[1] = b;
    }
}

/* ------------------------------------------------------------------------ */
/* launchers                                                                 */
/* ------------------------------------------------------------------------ */

/* dynamic shared memory of a force launch: the warps' areas, then the per-type table */
template <bool kDPD, class TS>
size_t force_launch_bytes(const EngineView &v) {
    return force_smem_bytes<kDPD, TS>() + sizeof(float4) * (size_t)v.ntypes;
}

template <bool kDPD, int kMode, bool kPure, class TS>
void configure_one() {
    const int bytes = (int)(force_smem_bytes<kDPD, TS>() + sizeof(float4) * kMaxTypes);
    cudaFuncSetAttribute(force_kernel<kDPD, kMode, kPure, TS>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    cudaFuncSetAttribute(force_kernel<kDPD, kMode, kPure, TS>, cudaFuncAttributePreferredSharedMemoryCarveout,
                         cudaSharedmemCarveoutMaxShared);
}

template <class TS>
void configure_tile() {
    configure_one<true, 0, false, TS>();
    configure_one<true, 0, true, TS>();
    configure_one<false, 0, false, TS>();
}

void configure_force_kernels() {
    // the force kernel's occupancy is bounded by shared memory: allow its dynamic
    // shared memory and ask for the largest carveout of the unified L1/shared storage
    configure_tile<Tile0>();
    configure_tile<Tile1>();
    configure_tile<Tile2>();
    configure_tile<Tile3>();
    configure_one<true, 1, false, Tile0>();
    configure_one<true, 2, false, Tile0>();
    configure_one<false, 1, false, Tile0>();
    configure_one<false, 2, false, Tile0>();
}

void launch_sort_bounds(const EngineView &v, cudaStream_t st) {
    sort_bounds_kernel<<<(v.ncells * 32 + 255) / 256, 256, 0, st>>>(v);
}

template <bool kDPD, class TS>
void launch_force_tile(const EngineView &v, int grid, cudaStream_t st) {
    if (kDPD && v.dpd_pure)
        force_kernel<true, 0, true, TS><<<grid, kWarpsPerBlock * 32, force_launch_bytes<true, TS>(v), st>>>(v);
    else
        force_kernel<kDPD, 0, false, TS><<<grid, kWarpsPerBlock * 32, force_launch_bytes<kDPD, TS>(v), st>>>(v);
}

/* The statistics and virial launches use the default tile; the force pass the engine's
 * variant (0 to kForceVariants - 1). */
template <bool kDPD>
void launch_force_mode(const EngineView &v, int grid, int variant, cudaStream_t st) {
    const size_t bytes = force_launch_bytes<kDPD, Tile0>(v);
    if (v.pair_stats)
        force_kernel<kDPD, 1, false, Tile0><<<grid, kWarpsPerBlock * 32, bytes, st>>>(v);
    else if (v.virial_partials)
        force_kernel<kDPD, 2, false, Tile0><<<grid, kWarpsPerBlock * 32, bytes, st>>>(v);
    else if (variant == 1)
        launch_force_tile<kDPD, Tile1>(v, grid, st);
    else if (variant == 2)
        launch_force_tile<kDPD, Tile2>(v, grid, st);
    else if (variant == 3)
        launch_force_tile<kDPD, Tile3>(v, grid, st);
    else
        launch_force_tile<kDPD, Tile0>(v, grid, st);
}

/* Work items by decreasing occupancy of their cell (counting sort on the count, capped
 * at 255; ties in any order, which changes no result: each item writes only its own
 * outputs). One block; launched before a force pass when cells are split into several
 * items, so that the most crowded cells' items start first. */
__global__ void item_order_kernel(EngineView v) {
    __shared__ int bin[256];
    __shared__ unsigned char key_s[kOrderMaxItems];  // 255 - min(count, 255) per item
    const int lane = threadIdx.x & 31;
    for (int k = threadIdx.x; k < 256; k += blockDim.x) bin[k] = 0;
    // the keys first, with independent loads in flight (the host orders at most
    // kOrderMaxItems items)
#pragma unroll 8
    for (int it = threadIdx.x; it < v.nitems; it += blockDim.x)
        key_s[it] = (unsigned char)(255 - min(v.cell_count[v.items[it].x], 255));
    __syncthreads();
    // consecutive items mostly share a cell: the lanes of a warp with equal keys take
    // one shared-memory atomic between them (the leader's), the others their rank
    const int nround = (v.nitems + blockDim.x - 1) / blockDim.x;
    for (int pass = 0; pass < 2; ++pass) {
        for (int r = 0; r < nround; ++r) {
            const int it = r * blockDim.x + threadIdx.x;
            const bool live = it < v.nitems;
            const int key = live ? (int)key_s[it] : 256;
            const unsigned peers = __match_any_sync(kFull, key);
            const int leader = __ffs(peers) - 1;
            int base = 0;
            if (lane == leader && live) base = atomicAdd(&bin[key], __popc(peers));
            base = __shfl_sync(kFull, base, leader);
            if (pass == 1 && live) v.item_order[base + __popc(peers & ((1u << lane) - 1u))] = it;
        }
        __syncthreads();
        if (pass == 0 && threadIdx.x < 32) {  // exclusive scan of the 256 bins, 8 bins a lane
            int c[8], sum = 0;
            for (int k = 0; k < 8; ++k) {
                c[k] = bin[lane * 8 + k];
                sum += c[k];
            }
            int incl = sum;
            for (int off = 1; off < 32; off <<= 1) {
                const int o = __shfl_up_sync(kFull, incl, off);
                if (lane >= off) incl += o;
            }
            int run = incl - sum;
            for (int k = 0; k < 8; ++k) {
                bin[lane * 8 + k] = run;
                run += c[k];
            }
        }
        __syncthreads();
    }
}

int force_variants() { return kForceVariants; }

void launch_force(const EngineView &v, bool has_dpd, int grid, bool combine, cudaStream_t st) {
    if (v.item_order && v.nitems > 0 && !v.virial_partials) item_order_kernel<<<1, 1024, 0, st>>>(v);
    if (has_dpd)
        launch_force_mode<true>(v, grid, v.force_variant, st);
    else
        launch_force_mode<false>(v, grid, v.force_variant, st);
    if (combine) combine_kernel<<<(v.nparts + 255) / 256, 256, 0, st>>>(v);
}

void launch_singlebody_prep(const EngineView &v, int ntypes, double *type_ke, float4 *persist, bool redraw,
                            cudaStream_t st) {
    type_ke_kernel<<<ntypes, 256, 0, st>>>(v, type_ke);
    if (redraw) persist_kernel<<<(v.nparts + 255) / 256, 256, 0, st>>>(v, persist);
}

void launch_virial_reduce(const double *partials, int nwarps, double *out9, cudaStream_t st) {
    virial_reduce_kernel<<<1, 32, 0, st>>>(partials, nwarps, out9);
}

int bonded_virial_blocks(int num_sms) { return num_sms * 2; }

void launch_bonded_virial(const EngineView &v, const BondedView &bv, int nb, int nx, int na, int nd, int nblocks,
                          double *partials, double *out9, cudaStream_t st) {
    bonded_virial_kernel<<<nblocks, kVirThreads, 0, st>>>(v, bv, nb, nx, na, nd, partials);
    bonded_virial_reduce_kernel<<<1, 32, 0, st>>>(partials, nblocks, out9);
}

void launch_body(const EngineView &v, float4 *body_f, cudaStream_t st) {
    const int tb = 128;
    body_kernel<<<(v.nparts + tb - 1) / tb, tb, 0, st>>>(v, body_f);
}

void launch_fluxes(const EngineView &v, const SpeciesView &sp, cudaStream_t st) {
    const int tb = 128;
    flux_kernel<<<(v.nparts + tb - 1) / tb, tb, 0, st>>>(v, sp);
}

void launch_species_integrate(const EngineView &v, const SpeciesView &sp, const int *new_cell, cudaStream_t st) {
    const int tb = 256;
    species_integrate_kernel<<<(v.nparts + tb - 1) / tb, tb, 0, st>>>(v, sp, new_cell);
}

void launch_bonded(const EngineView &v, const BondedView &bv, cudaStream_t st) {
    const int tb = 256;
    bonded_kernel<<<(v.nparts + tb - 1) / tb, tb, 0, st>>>(v, bv);
}

void launch_integrate(const EngineView &v, float4 *pos, float4 *vel, int *new_cell, int *in_count, int *in_list,
                      int *out_count, bool add_planes, cudaStream_t st) {
    integrate_kernel<<<(v.nparts + kAdvThreads - 1) / kAdvThreads, kAdvThreads, 0, st>>>(
        v, pos, vel, new_cell, in_count, in_list, out_count, add_planes);
}

void launch_rk_stage(const EngineView &v, float4 *pos, float4 *const *rk, int stage, bool add_planes,
                     cudaStream_t st) {
    const RkState r{rk[0], rk[1], rk[2], rk[3], rk[4]};
    rk_stage_kernel<<<(v.nparts + 255) / 256, 256, 0, st>>>(v, pos, r, stage, add_planes);
}

void launch_rk_final(const EngineView &v, float4 *pos, float4 *vel, float4 *const *rk, int *new_cell, int *in_count,
                     int *in_list, int *out_count, bool add_planes, cudaStream_t st) {
    const RkState r{rk[0], rk[1], rk[2], rk[3], rk[4]};
    rk_final_kernel<<<(v.nparts + kAdvThreads - 1) / kAdvThreads, kAdvThreads, 0, st>>>(
        v, pos, vel, r, new_cell, in_count, in_list, out_count, add_planes);
}

void launch_scatter(const EngineView &v, const float4 *pos, const float4 *vel, const int *new_cell,
                    const int *old_start, const int *old_count, const int *in_count, const int *in_list,
                    const int *out_count, int *new_start, int *new_count, float4 *pos_out, float4 *vel_out,
                    int *cell_out, int *slot_of_id, int *clear_in, int *clear_out, int *clear_chunk, int nchunks,
                    unsigned *ctl, unsigned long long *step, cudaStream_t st) {
    const int grid = (v.ncells + kScatterWarps - 1) / kScatterWarps;
    scatter_kernel<<<grid, kScatterWarps * 32, 0, st>>>(v, v.ncells, pos, vel, new_cell, old_start, old_count,
                                                        in_count, in_list, out_count, new_start, new_count, pos_out,
                                                        vel_out, cell_out, slot_of_id, clear_in, clear_out,
                                                        clear_chunk, nchunks, ctl, step);
}

void launch_number_density(const EngineView &v, const int *flux_off, float *nd_by_id, cudaStream_t st) {
    number_density_kernel<<<(v.nparts + 127) / 128, 128, 0, st>>>(v, flux_off, nd_by_id);
}

void launch_load_place(const EngineView &v, const LoadView &ld, int *count, cudaStream_t st) {
    place_kernel<<<(ld.n + 255) / 256, 256, 0, st>>>(v, ld, count);
}

void launch_load_order(const EngineView &v, const LoadView &ld, const int *count, int *start, int *count_out,
                       float4 *pos_out, float4 *vel_out, int *cell_out, int *slot_of_id, cudaEvent_t vel_ready,
                       cudaStream_t st) {
    load_scan_kernel<<<1, 1024, 0, st>>>(count, v.ncells, start, count_out, ld.err);
    load_fill_kernel<<<(ld.n + 255) / 256, 256, 0, st>>>(ld, start);
    const int tb = 256;
    load_order_kernel<<<(v.ncells * 32 + tb - 1) / tb, tb, 0, st>>>(v, ld, start, pos_out, vel_out, cell_out,
                                                                     slot_of_id, v.sort_bounds);
    if (ld.v) {  // the given velocities, once their copy has arrived
        if (vel_ready) cudaStreamWaitEvent(st, vel_ready, 0);
        load_vel_kernel<<<(ld.n + 255) / 256, 256, 0, st>>>(ld, slot_of_id, vel_out);
    }
}

void launch_unload(const EngineView &v, const float4 *force_ids, double *x, float *vel, float *f, int *cell,
                   float *xrel, cudaStream_t st) {
    unload_kernel<<<(v.nparts + 255) / 256, 256, 0, st>>>(v, force_ids, x, vel, f, cell, xrel);
}

void launch_energy(int ncells, const double *epot_cell, int nparts, const double *ebond_slot, const double *body_e,
                   const float4 *vel, const float4 *pos, const DevType *types, double *partials, int nblocks,
                   double *out, cudaStream_t st) {
    reduce_energy_kernel<<<nblocks, 256, 0, st>>>(ncells, epot_cell, nparts, ebond_slot, body_e, vel, pos, types,
                                                  partials);
    reduce_final_kernel<<<1, 32, 0, st>>>(nblocks, partials, out);
}

}  // namespace mxg
