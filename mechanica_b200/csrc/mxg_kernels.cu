/*
 * Force-and-step kernels for sm_100a.
 *
 *   force_kernel      nonbonded cell-pair forces (tables, DPD), single-body
 *                     forces, per-cell FP64 energy. One warp per cell.
 *   bond_kernel       harmonic/table bonds with dissociation flags.
 *   integrate_kernel  forward Euler (Newtonian / overdamped), speed clamp,
 *                     wall reflection, relocation; counts the next binning.
 *   scan_kernel       exclusive scan of the new cell occupancy.
 *   scatter_kernel    stable re-binning (ascending id inside each cell).
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

__device__ __forceinline__ int next_pow2(int n) {
    int p = 1;
    while (p < n) p <<= 1;
    return p;
}

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

}  // namespace

/* ------------------------------------------------------------------------ */
/* sort-key bounds                                                           */
/* ------------------------------------------------------------------------ */

/*
 * Per cell and per sort direction, the smallest and largest projection key of
 * its particles (runner_dosort.cpp:133-141 computes the keys; runner_dopair
 * reads the largest key of its first cell and the smallest of its second,
 * runner_dopair.cpp:167-171). One warp per cell.
 */
__global__ void sort_bounds_kernel(EngineView v) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < v.ncells; c += warps) {
        const int n = v.cell_count[c];
        if (n == 0) continue;
        const int start = v.cell_start[c];
        const DevSpace &S = v.spaces[v.cell_rep[c]];
        const float bias = S.sort_bias, dscale = S.sort_dscale;
        for (int sid = 0; sid < 13; ++sid) {
            const float *ax = v.axes->n[sid];
            int kmin = 0x7fffffff, kmax = -1;
            for (int k = lane; k < n; k += 32) {
                const float4 q = v.pos[start + k];
                const int key = sort_key(q.x, q.y, q.z, ax, bias, dscale);
                kmin = min(kmin, key);
                kmax = max(kmax, key);
            }
            for (int off = 16; off > 0; off >>= 1) {
                kmin = min(kmin, __shfl_xor_sync(kFull, kmin, off));
                kmax = max(kmax, __shfl_xor_sync(kFull, kmax, off));
            }
            if (lane == 0) v.sort_bounds[c * 13 + sid] = make_int2(kmin, kmax);
        }
    }
}

/* ------------------------------------------------------------------------ */
/* nonbonded forces                                                          */
/* ------------------------------------------------------------------------ */

/*
 * One warp per cell i (grid-stride). The warp's lanes are split into G groups
 * of P = next_pow2(count) lanes: lane (il, g) owns particle il of the cell and
 * the g-th share of every neighbour cell's particles. Neighbour particles are
 * staged 32 at a time in shared memory (coalesced float4 loads) and read back
 * as broadcasts; each lane accumulates the force on its own particle in
 * registers and the G partial sums are combined with warp shuffles, so no
 * global atomics are needed and the result is deterministic.
 *
 * Each neighbour entry carries the role of cell i in the reference's flipped
 * cell pair (runner_dopair.cpp:91-340, runner_doself :446-682): FIRST means the
 * reference computes dx = (x_i - shift) - x_j; SECOND means it computes
 * dx = (x_j - shift) - x_i with i as its second particle. Computing dx in the
 * reference's orientation makes r2 and the per-pair force bit-identical.
 */
template <bool kDPD, bool kStats>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) force_kernel(EngineView v) {
    unsigned long long npair = 0;  // interacting pairs counted once (statistics launch only)
    __shared__ float4 sp[kWarpsPerBlock][32];
    __shared__ float4 sv[kWarpsPerBlock][kDPD ? 32 : 1];
    __shared__ int skey[kWarpsPerBlock][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int c = blockIdx.x * kWarpsPerBlock + w; c < v.ncells; c += gridDim.x * kWarpsPerBlock) {
        const int n = v.cell_count[c];
        double ecell = 0.0;
        if (n > 0) {
            const int start = v.cell_start[c];
            const DevSpace &S = v.spaces[v.cell_rep[c]];
            const int pot_base = S.pot_offset;
            const float cut2_pair = S.cut2_pair, cut2_self = S.cut2_self;
            const unsigned rng_mode = S.rng_mode;
            const bool prune = (S.prune & 1) != 0;       // per-pair projection test
            const bool exit_test = (S.prune & 2) != 0;   // cell-pair exit test
            const float sbias = S.sort_bias, sdscale = S.sort_dscale;
            const int dmaxdist = S.dmaxdist;
            const int P = n >= 32 ? 32 : next_pow2(n);
            const int G = 32 / P;
            const int il = lane & (P - 1), g = lane / P;
            const int nb0 = v.nb_off[c], nb1 = v.nb_off[c + 1];
            for (int i0 = 0; i0 < n; i0 += 32) {
                const int i = i0 + il;
                const bool live = i < n;
                float4 xi = make_float4(0.f, 0.f, 0.f, 0.f);
                float4 vi = make_float4(0.f, 0.f, 0.f, 0.f);
                if (live) {
                    xi = v.pos[start + i];
                    if (kDPD) vi = v.vel[start + i];
                }
                const int ti = __float_as_int(xi.w);
                const DevType &T = v.types[live ? ti : 0];
                const float radi = T.radius;
                float fx = 0.f, fy = 0.f, fz = 0.f;
                if (live && g == 0 && T.has_force) {  // constant_force (MxForce.cpp:339-344), scale 1
                    fx = T.fx;
                    fy = T.fy;
                    fz = T.fz;
                }
                double eacc = 0.0;
                for (int e = nb0; e < nb1; ++e) {
                    const int nc = v.nb_cell[e];
                    const int jn = v.cell_count[nc];
                    if (jn == 0) continue;
                    const int js = v.cell_start[nc];
                    const float4 sh = v.nb_shift[e];
                    const int packed = __float_as_int(sh.w);
                    const int role = packed & 3;
                    // runner_dopair's pruning: a pair (first i, second j) is evaluated only
                    // when key_j + dnshift - key_i < dmaxdist (runner_dopair.cpp:167-182)
                    const bool prune_e = prune && role != kRoleSelf;
                    const int sid = (packed >> 2) & 15;
                    const float *axis = v.axes->n[sid];
                    const int dnshift = packed >> 8;
                    if (exit_test && role != kRoleSelf) {
                        // runner_dopair's first-iteration exit (runner_dopair.cpp:167-171): with the
                        // largest key of the first cell and the smallest of the second, the unsigned
                        // difference kmin + dnshift - kmax exceeds dmaxdist (or wraps below zero)
                        // and the whole cell pair is skipped
                        const int2 bi = v.sort_bounds[c * 13 + sid], bj = v.sort_bounds[nc * 13 + sid];
                        const int kmax_first = role == kRoleFirst ? bi.y : bj.y;
                        const int kmin_second = role == kRoleFirst ? bj.x : bi.x;
                        const int gap = kmin_second + dnshift - kmax_first;
                        if (gap < 0 || gap > dmaxdist) continue;
                    }
                    int mykey = 0;
                    if (prune_e) mykey = sort_key(xi.x, xi.y, xi.z, axis, sbias, sdscale);
                    float ax = xi.x, ay = xi.y, az = xi.z;
                    if (role == kRoleFirst) {
                        ax = __fsub_rn(xi.x, sh.x);
                        ay = __fsub_rn(xi.y, sh.y);
                        az = __fsub_rn(xi.z, sh.z);
                    }
                    const float cut2 = role == kRoleSelf ? cut2_self : cut2_pair;
                    for (int j0 = 0; j0 < jn; j0 += 32) {
                        const int cnt = min(32, jn - j0);
                        __syncwarp();
                        if (lane < cnt) {
                            float4 q = v.pos[js + j0 + lane];
                            if (prune_e) skey[w][lane] = sort_key(q.x, q.y, q.z, axis, sbias, sdscale);
                            if (role == kRoleSecond) {
                                q.x = __fsub_rn(q.x, sh.x);
                                q.y = __fsub_rn(q.y, sh.y);
                                q.z = __fsub_rn(q.z, sh.z);
                            }
                            sp[w][lane] = q;
                            if (kDPD) sv[w][lane] = v.vel[js + j0 + lane];
                        }
                        __syncwarp();
                        if (!live) continue;
                        for (int t = g; t < cnt; t += G) {
                            const int j = j0 + t;
                            if (role == kRoleSelf && j == i) continue;
                            if (prune_e) {
                                const int kf = role == kRoleFirst ? mykey : skey[w][t];
                                const int ks = role == kRoleFirst ? skey[w][t] : mykey;
                                if (!(ks + dnshift - kf < dmaxdist)) continue;
                            }
                            const float4 q = sp[w][t];
                            // dx in the reference's orientation
                            float dx, dy, dz;
                            if (role == kRoleSecond) {
                                dx = __fsub_rn(q.x, xi.x);
                                dy = __fsub_rn(q.y, xi.y);
                                dz = __fsub_rn(q.z, xi.z);
                            } else {
                                dx = __fsub_rn(ax, q.x);
                                dy = __fsub_rn(ay, q.y);
                                dz = __fsub_rn(az, q.z);
                                if (role == kRoleSelf && j < i) {
                                    // the reference's first particle of a self pair is the earlier
                                    // one; x_j - x_i is the exact negation of x_i - x_j
                                    dx = -dx;
                                    dy = -dy;
                                    dz = -dz;
                                }
                            }
                            float r2 = dot3_rn(dx, dy, dz);
                            if (r2 > cut2) continue;
                            const int tj = __float_as_int(q.w);
                            const int pidx = v.pot_idx[pot_base + ti * v.ntypes + tj];
                            if (pidx < 0) continue;
                            const DevPot &p = v.pots[pidx];
                            // which of the two is the reference's first particle
                            const bool i_first = role == kRoleFirst || (role == kRoleSelf && i < j);
                            if (r2 < p.a2) {
                                // potential_eval_super_ex (dpd_eval.hpp:122-131): random direction of
                                // length a; here a Philox draw keyed on the step and the id pair
                                const unsigned idi = __float_as_uint(v.vel[start + i].w);
                                const unsigned idj = __float_as_uint(v.vel[js + j].w);
                                const unsigned lo = idi < idj ? idi : idj, hi = idi < idj ? idj : idi;
                                float g0, g1, g2;
                                philox_normal3(*v.step, lo, hi, g0, g1, g2);
                                const float len = sqrtf(g0 * g0 + g1 * g1 + g2 * g2);
                                // the draw is the displacement first-minus-second for (lo, hi)
                                const bool sign = ((idi == lo) == i_first);
                                const float s = sign ? 1.0f : -1.0f;
                                dx = s * g0 * p.a / len;
                                dy = s * g1 * p.a / len;
                                dz = s * g2 * p.a / len;
                                r2 = p.a2;
                            }
                            if (kDPD && p.kind == 1) {
                                // dpd_eval (dpd_eval.hpp:21-69), in the reference's orientation
                                const DevType &Tj = v.types[tj];
                                const float r_first = i_first ? radi : Tj.radius;
                                const float r_second = i_first ? Tj.radius : radi;
                                const bool shifted = p.flags & (1u << 12);
                                const float cutoff = shifted ? __fadd_rn(__fadd_rn(p.b, r_first), r_second) : p.b;
                                if (r2 > __fmul_rn(cutoff, cutoff)) continue;
                                const float r = sqrtf(r2);
                                const float ex = __fdiv_rn(dx, r), ey = __fdiv_rn(dy, r), ez = __fdiv_rn(dz, r);
                                const float4 vj = sv[w][t];
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
                                if (rng_mode) {
                                    const unsigned idi = __float_as_uint(vi.w), idj = __float_as_uint(vj.w);
                                    fr = fr * philox_pair_xi(*v.step, idi < idj ? idi : idj, idi < idj ? idj : idi);
                                }
                                const float f = __fadd_rn(__fadd_rn(fc, fd), fr);
                                if (i_first) {
                                    fx = __fadd_rn(fx, __fmul_rn(f, ex));
                                    fy = __fadd_rn(fy, __fmul_rn(f, ey));
                                    fz = __fadd_rn(fz, __fmul_rn(f, ez));
                                } else {
                                    fx = __fsub_rn(fx, __fmul_rn(f, ex));
                                    fy = __fsub_rn(fy, __fmul_rn(f, ey));
                                    fz = __fsub_rn(fz, __fmul_rn(f, ez));
                                }
                                // the reference tabulates zero energy for DPD
                                if (kStats && i_first) ++npair;
                            } else {
                                const float radj = v.types[tj].radius;
                                float pe, pf;
                                if (!table_eval_ex(p, v.coef, i_first ? radi : radj, i_first ? radj : radi, r2, pe, pf))
                                    continue;
                                const float wx = __fmul_rn(pf, dx), wy = __fmul_rn(pf, dy), wz = __fmul_rn(pf, dz);
                                if (i_first) {
                                    fx = __fsub_rn(fx, wx);
                                    fy = __fsub_rn(fy, wy);
                                    fz = __fsub_rn(fz, wz);
                                } else {
                                    fx = __fadd_rn(fx, wx);
                                    fy = __fadd_rn(fy, wy);
                                    fz = __fadd_rn(fz, wz);
                                }
                                if (role == kRoleFirst || (role == kRoleSelf && i < j)) {
                                    eacc += (double)pe;
                                    if (kStats) ++npair;
                                }
                            }
                        }
                    }
                }
                // combine the G partial sums of each particle
                for (int off = P; off < 32; off <<= 1) {
                    fx += __shfl_xor_sync(kFull, fx, off);
                    fy += __shfl_xor_sync(kFull, fy, off);
                    fz += __shfl_xor_sync(kFull, fz, off);
                    eacc += __shfl_xor_sync(kFull, eacc, off);
                }
                if (live && g == 0) v.force[start + i] = make_float4(fx, fy, fz, 0.f);
                if (g == 0) ecell += eacc;
            }
        }
        for (int off = 16; off > 0; off >>= 1) ecell += __shfl_xor_sync(kFull, ecell, off);
        if (lane == 0) v.epot_cell[c] = ecell;
    }
    if (kStats) {
        for (int off = 16; off > 0; off >>= 1) npair += __shfl_xor_sync(kFull, npair, off);
        if (lane == 0) atomicAdd(v.pair_stats, npair);
    }
}

/* ------------------------------------------------------------------------ */
/* bonds                                                                     */
/* ------------------------------------------------------------------------ */

/*
 * One thread per particle slot; each thread evaluates every bond its particle
 * takes part in, from the bond's first particle's point of view exactly as
 * bond_eval does (bond.cpp:99-312), and applies its own half of the force.
 * Both ends therefore compute the same force/r and the same break decision
 * eff >= dissociation_energy; the first end clears the bond's active flag.
 */
__global__ void bond_kernel(EngineView v, const DevBond *__restrict__ bonds, unsigned *bond_flags,
                            const int *__restrict__ bond_off, const int *__restrict__ bond_list,
                            const int *__restrict__ slot_of_id, double *__restrict__ ebond_slot) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= v.nparts) return;
    const int id = __float_as_int(v.vel[s].w);
    const int k0 = bond_off[id], k1 = bond_off[id + 1];
    double eb = 0.0;
    if (k0 < k1) {
        float4 f = v.force[s];
        for (int k = k0; k < k1; ++k) {
            const int b = bond_list[k];
            if (!(bond_flags[b] & 1u)) continue;
            const DevBond B = bonds[b];
            const int si = slot_of_id[B.i], sj = slot_of_id[B.j];
            if (si < 0 || sj < 0) continue;
            const int ci = v.cell_of[si], cj = v.cell_of[sj];
            const DevSpace &S = v.spaces[v.cell_rep[ci]];
            const int li = ci - S.cell_offset, lj = cj - S.cell_offset;
            const int loci[3] = {li / (S.cdim[1] * S.cdim[2]), (li / S.cdim[2]) % S.cdim[1], li % S.cdim[2]};
            const int locj[3] = {lj / (S.cdim[1] * S.cdim[2]), (lj / S.cdim[2]) % S.cdim[1], lj % S.cdim[2]};
            const float4 xi = v.pos[si], xj = v.pos[sj];
            const float xiv[3] = {xi.x, xi.y, xi.z}, xjv[3] = {xj.x, xj.y, xj.z};
            float d[3];
            for (int q = 0; q < 3; ++q) {
                int sh = loci[q] - locj[q];
                if (sh > 1)
                    sh = -1;
                else if (sh < -1)
                    sh = 1;
                const float pix = (float)__dadd_rn((double)xiv[q], __dmul_rn(S.hd[q], (double)sh));
                d[q] = __fsub_rn(pix, xjv[q]);
            }
            float r2 = dot3_rn(d[0], d[1], d[2]);
            const DevPot &p = v.pots[B.pot];
            const float a2 = __fmul_rn(p.a, p.a), b2 = __fmul_rn(p.b, p.b);
            if (r2 < a2 || r2 > b2) r2 = fmaxf(a2, fminf(b2, r2));
            float ee, eff;
            table_eval(p, v.coef, r2, ee, eff);
            const bool first = (s == si);
            if ((double)eff >= B.dissociation) {
                if (first) bond_flags[b] = 0u;  // MxBond_Destroy (bond.cpp:1001-1013)
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
        v.force[s] = f;
    }
    ebond_slot[s] = eb;
}

/* ------------------------------------------------------------------------ */
/* integrator                                                                */
/* ------------------------------------------------------------------------ */

/* space_shuffle_local's rule (space.cpp:352-371): delta = (x >= h) - (x < 0). */
__device__ __forceinline__ int cell_delta(float x, float h) { return (x >= h ? 1 : 0) - (x < 0.0f ? 1 : 0); }

/*
 * Forward Euler for one particle (engine_advance.cpp:126-239): velocity update
 * in FP64 rounded to FP32, per-component speed (or step) clamp, position update,
 * wall reflection (boundary_eval.hpp:30-122), and the move to a neighbour cell
 * with x -= delta*h. The next step's space_shuffle_local rule is applied once
 * more to the moved particle, as engine_force does before the next force pass.
 * Moved particles are appended to the destination cell's bucket; stayers are
 * counted implicitly (count_old - out + in).
 */
__global__ void integrate_kernel(EngineView v, float4 *pos, float4 *vel, int *new_cell, int *in_count,
                                 int *in_list, int *out_count) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= v.nparts) return;
    const int c = v.cell_of[s];
    const DevSpace &S = v.spaces[v.cell_rep[c]];
    float4 x = pos[s];
    float4 u = vel[s];
    const float4 f = v.force[s];
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
            if (delta[0] | delta[1] | delta[2]) {
                const int l = c - S.cell_offset;
                int loc[3] = {l / (S.cdim[1] * S.cdim[2]), (l / S.cdim[2]) % S.cdim[1], l % S.cdim[2]};
                for (int pass = 0; pass < 2; ++pass) {
                    for (int k = 0; k < 3; ++k) {
                        xv[k] = __fsub_rn(xv[k], __fmul_rn((float)delta[k], S.h[k]));
                        loc[k] = (loc[k] + delta[k] + S.cdim[k]) % S.cdim[k];
                    }
                    // the next force pass's shuffle (space.cpp:333-393) on the moved particle
                    for (int k = 0; k < 3; ++k) delta[k] = cell_delta(xv[k], S.h[k]);
                    if (!(delta[0] | delta[1] | delta[2])) break;
                }
                dest = S.cell_offset + (loc[0] * S.cdim[1] + loc[1]) * S.cdim[2] + loc[2];
            }
        }
        x.x = xv[0]; x.y = xv[1]; x.z = xv[2];
        u.x = vv[0]; u.y = vv[1]; u.z = vv[2];
        pos[s] = x;
        vel[s] = u;
    }
    new_cell[s] = dest;
    if (dest != c) {
        const int k = atomicAdd(&in_count[dest], 1);
        if (k < kBucket)
            in_list[dest * kBucket + k] = s;
        else
            atomicOr(v.status, kStatusBucketOverflow);
        atomicAdd(&out_count[c], 1);
    }
}

/* ------------------------------------------------------------------------ */
/* re-binning                                                                */
/* ------------------------------------------------------------------------ */

/* New occupancy count_old - out + in, exclusive scan into new_start; single
 * block, each thread scans a contiguous run of cells. */
__global__ void __launch_bounds__(1024) scan_kernel(int ncells, const int *__restrict__ old_count,
                                                   const int *__restrict__ out_count, const int *__restrict__ in_count,
                                                   int *new_start, int *new_count, unsigned long long *step) {
    __shared__ int part[1024];
    const int t = threadIdx.x;
    const int per = (ncells + blockDim.x - 1) / blockDim.x;
    const int b = t * per, e = min(ncells, b + per);
    int sum = 0;
    for (int c = b; c < e; ++c) {
        const int n = old_count[c] - out_count[c] + min(in_count[c], kBucket);
        new_count[c] = n;
        sum += n;
    }
    part[t] = sum;
    __syncthreads();
    for (int off = 1; off < blockDim.x; off <<= 1) {  // Hillis-Steele inclusive scan
        const int add = t >= off ? part[t - off] : 0;
        __syncthreads();
        part[t] += add;
        __syncthreads();
    }
    int run = part[t] - sum;
    for (int c = b; c < e; ++c) {
        new_start[c] = run;
        run += new_count[c];
    }
    if (t == blockDim.x - 1) {
        new_start[ncells] = part[t];
        *step += 1;  // the step counter keying the Philox streams
    }
}

/*
 * One warp per destination cell. Stayers keep their relative order (ascending
 * id); movers are merged in by id, so every cell stays sorted by id and the
 * layout is independent of thread scheduling.
 */
__global__ void scatter_kernel(int ncells, const float4 *__restrict__ pos, const float4 *__restrict__ vel,
                               const int *__restrict__ new_cell, const int *__restrict__ old_start,
                               const int *__restrict__ old_count, int *in_count, const int *__restrict__ in_list,
                               int *out_count, const int *__restrict__ new_start, float4 *pos_out, float4 *vel_out,
                               int *cell_out, int *slot_of_id) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < ncells; c += warps) {
        const int os = old_start[c], on = old_count[c];
        const int m = min(in_count[c], kBucket);
        const int base = new_start[c];
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
            if (stay) {
                int rank = stay_before + __popc(bal & ((1u << lane) - 1u));
                for (int q = 0; q < m; ++q) {
                    const int src = in_list[c * kBucket + q];
                    rank += __float_as_int(vel[src].w) < myid;
                }
                const int dst = base + rank;
                pos_out[dst] = pos[os + k];
                vel_out[dst] = vel[os + k];
                cell_out[dst] = c;
                slot_of_id[myid] = dst;
            }
            stay_before += __popc(bal);
        }
        // movers
        for (int q0 = 0; q0 < m; q0 += 32) {
            const int q = q0 + lane;
            if (q < m) {
                const int src = in_list[c * kBucket + q];
                const int myid = __float_as_int(vel[src].w);
                int rank = 0;
                for (int k = 0; k < on; ++k)
                    rank += (new_cell[os + k] == c) && (__float_as_int(vel[os + k].w) < myid);
                for (int r = 0; r < m; ++r) rank += __float_as_int(vel[in_list[c * kBucket + r]].w) < myid;
                const int dst = base + rank;
                pos_out[dst] = pos[src];
                vel_out[dst] = vel[src];
                cell_out[dst] = c;
                slot_of_id[myid] = dst;
            }
        }
        __syncwarp();
        if (lane == 0) {
            in_count[c] = 0;
            out_count[c] = 0;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* energies (FP64)                                                           */
/* ------------------------------------------------------------------------ */

/* Deterministic two-stage sums: block partials, then one block. */
__global__ void reduce_energy_kernel(int ncells, const double *__restrict__ epot_cell, int nparts,
                                     const double *__restrict__ ebond_slot, const float4 *__restrict__ vel,
                                     const float4 *__restrict__ pos, const DevType *__restrict__ types,
                                     double *partials) {
    __shared__ double s_pot[256], s_kin[256];
    double ep = 0.0, ek = 0.0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncells; c += gridDim.x * blockDim.x) ep += epot_cell[c];
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nparts; s += gridDim.x * blockDim.x) {
        if (ebond_slot) ep += ebond_slot[s];
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

void launch_force(const EngineView &v, bool has_dpd, int grid, cudaStream_t st) {
    const bool stats = v.pair_stats != nullptr;
    sort_bounds_kernel<<<(v.ncells * 32 + 255) / 256, 256, 0, st>>>(v);
    if (has_dpd) {
        if (stats)
            force_kernel<true, true><<<grid, kWarpsPerBlock * 32, 0, st>>>(v);
        else
            force_kernel<true, false><<<grid, kWarpsPerBlock * 32, 0, st>>>(v);
    } else {
        if (stats)
            force_kernel<false, true><<<grid, kWarpsPerBlock * 32, 0, st>>>(v);
        else
            force_kernel<false, false><<<grid, kWarpsPerBlock * 32, 0, st>>>(v);
    }
}

void launch_bonds(const EngineView &v, const DevBond *bonds, unsigned *bond_flags, const int *bond_off,
                  const int *bond_list, const int *slot_of_id, double *ebond_slot, cudaStream_t st) {
    const int tb = 256;
    bond_kernel<<<(v.nparts + tb - 1) / tb, tb, 0, st>>>(v, bonds, bond_flags, bond_off, bond_list, slot_of_id,
                                                        ebond_slot);
}

void launch_integrate(const EngineView &v, float4 *pos, float4 *vel, int *new_cell, int *in_count, int *in_list,
                      int *out_count, cudaStream_t st) {
    const int tb = 256;
    integrate_kernel<<<(v.nparts + tb - 1) / tb, tb, 0, st>>>(v, pos, vel, new_cell, in_count, in_list, out_count);
}

void launch_scan(int ncells, const int *old_count, const int *out_count, const int *in_count, int *new_start,
                 int *new_count, unsigned long long *step, cudaStream_t st) {
    scan_kernel<<<1, 1024, 0, st>>>(ncells, old_count, out_count, in_count, new_start, new_count, step);
}

void launch_scatter(int ncells, const float4 *pos, const float4 *vel, const int *new_cell, const int *old_start,
                    const int *old_count, int *in_count, const int *in_list, int *out_count, const int *new_start,
                    float4 *pos_out, float4 *vel_out, int *cell_out, int *slot_of_id, cudaStream_t st) {
    const int tb = 256;
    const int grid = (ncells * 32 + tb - 1) / tb;
    scatter_kernel<<<grid, tb, 0, st>>>(ncells, pos, vel, new_cell, old_start, old_count, in_count, in_list,
                                         out_count, new_start, pos_out, vel_out, cell_out, slot_of_id);
}

void launch_energy(int ncells, const double *epot_cell, int nparts, const double *ebond_slot, const float4 *vel,
                   const float4 *pos, const DevType *types, double *partials, int nblocks, double *out,
                   cudaStream_t st) {
    reduce_energy_kernel<<<nblocks, 256, 0, st>>>(ncells, epot_cell, nparts, ebond_slot, vel, pos, types, partials);
    reduce_final_kernel<<<1, 32, 0, st>>>(nblocks, partials, out);
}

}  // namespace mxg
