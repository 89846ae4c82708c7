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
 * One warp per cell (grid-stride). The warp stages up to kOwn of the cell's
 * particles and then, region by region, up to kCap particles of its neighbour
 * entries (whole entries where they fit) in shared memory. Each own particle
 * is tested against the staged neighbours one per lane, 32 candidates per
 * step, for the cutoff, the reference's pruning and the existence of a
 * potential (pass 1). Interacting candidates are appended, in candidate order,
 * to a per-warp queue with a ballot; every 32 queued pairs are evaluated with
 * one pair per lane (pass 2), so the expensive pair arithmetic runs with the
 * warp's lanes full. The queue is ordered by own particle, so the per-particle
 * sums of a batch are formed by a segmented shuffle scan in a fixed order and
 * added to the particle's force in shared memory by the segment's last lane:
 * no atomics, deterministic results.
 *
 * Each neighbour entry carries the role of the cell in the reference's flipped
 * cell pair (runner_dopair.cpp:91-340, runner_doself :446-682): FIRST means the
 * reference computes dx = (x_i - shift) - x_j; SECOND means it computes
 * dx = (x_j - shift) - x_i with i as its second particle. Neighbour positions
 * of SECOND entries are staged pre-shifted and FIRST entries stage their shift
 * beside each particle, so every candidate computes d = (x_i - s) - b with one
 * formula; the reference's dx is d or its exact negation, which makes r2 and
 * the per-pair force bit-identical to the reference's.
 */
template <bool kDPD>
__device__ __forceinline__ void pair_contribution(const EngineView &v, const DevPot &p, int role, bool i_first,
                                                  float dx, float dy, float dz, float r2, float radi, float radj,
                                                  const float4 &vi, const float4 &vj, unsigned rng_mode,
                                                  float &cx, float &cy, float &cz, float &pe, bool &counted) {
    cx = cy = cz = 0.f;
    pe = 0.f;
    counted = false;
    if (kDPD && p.kind == 1) {
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
        if (rng_mode) {
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
    } else {
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

constexpr int kOwn = 32;    // own particles staged at a time
constexpr int kCap = 128;   // neighbour particles staged at a time

template <bool kDPD>
struct ForceSmem {
    float4 nb_x[kCap];              // position (pre-shifted for SECOND entries); w = type
    float4 nb_s[kCap];              // shift of FIRST entries, else 0; w = role | entry << 2 | index << 8
    float4 nb_v[kDPD ? kCap : 1];   // velocity; w = id
    float4 own_x[kOwn];
    float4 own_v[kDPD ? kOwn : 1];
    float4 own_f[kOwn];
    float4 ent_sh[32];              // region entries: shift, w = packed role/sort direction/key shift
    int ent_beg[33];                // first staged index of each region entry
    int ent_slot[32];               // slot of the entry cell's first particle
    int ent_jb[32];                 // index (within its cell) of the entry's first staged particle
    int own_mask[kOwn];             // bit t: a potential exists for (own type, t), types < 32
    int nb_key[kCap];               // sort key of the unshifted neighbour (per-pair pruning)
    int queue[64];                  // own index << 16 | staged index, in candidate order
};

/* Pass 2 over queue[0, nb): one interacting pair per lane, segmented sums into
 * own_f. Returns the pairs counted once (statistics launch). */
template <bool kDPD, bool kStats>
__device__ __forceinline__ void eval_batch(const EngineView &v, ForceSmem<kDPD> &sm, int nb, int i0, int own_start,
                                           int pot_base, unsigned rng_mode, double &ecell,
                                           unsigned long long &npair) {
    const int lane = threadIdx.x & 31;
    float cx = 0.f, cy = 0.f, cz = 0.f;
    int il = -1;
    if (lane < nb) {
        const int cd = sm.queue[lane];
        il = cd >> 16;
        const int jj = cd & 0xffff;
        const int i = i0 + il;
        const float4 xi = sm.own_x[il];
        const float4 b = sm.nb_x[jj];
        const float4 s = sm.nb_s[jj];
        const int meta = __float_as_int(s.w);
        const int role = meta & 3, jl = meta >> 8;
        float dx = __fsub_rn(__fsub_rn(xi.x, s.x), b.x);
        float dy = __fsub_rn(__fsub_rn(xi.y, s.y), b.y);
        float dz = __fsub_rn(__fsub_rn(xi.z, s.z), b.z);
        // SECOND: the reference's dx is b - x_i; SELF with the neighbour first: x_j - x_i
        if (role == kRoleSecond || (role == kRoleSelf && jl < i)) {
            dx = -dx;
            dy = -dy;
            dz = -dz;
        }
        float r2 = dot3_rn(dx, dy, dz);
        const int ti = __float_as_int(xi.w), tj = __float_as_int(b.w);
        const DevPot &p = v.pots[v.pot_idx[pot_base + ti * v.ntypes + tj]];
        const bool i_first = role == kRoleFirst || (role == kRoleSelf && i < jl);
        if (r2 < p.a2) {
            // potential_eval_super_ex (dpd_eval.hpp:122-131): random direction of
            // length a; here a Philox draw keyed on the step and the id pair
            const unsigned idi = __float_as_uint(kDPD ? sm.own_v[il].w : v.vel[own_start + i].w);
            const unsigned idj =
                __float_as_uint(kDPD ? sm.nb_v[jj].w : v.vel[sm.ent_slot[(meta >> 2) & 63] + jl].w);
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
        pair_contribution<kDPD>(v, p, role, i_first, dx, dy, dz, r2, v.types[ti].radius, v.types[tj].radius, vi,
                                vj, rng_mode, cx, cy, cz, pe, counted);
        ecell += (double)pe;
        if (kStats && counted) ++npair;
    }
    // segmented inclusive scan: segments are runs of equal own index
    const int il_prev = __shfl_up_sync(kFull, il, 1);
    const unsigned heads = __ballot_sync(kFull, lane == 0 || il != il_prev);
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

template <bool kDPD, bool kStats>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) force_kernel(EngineView v) {
    unsigned long long npair = 0;  // interacting pairs counted once (statistics launch only)
    __shared__ ForceSmem<kDPD> smem_all[kWarpsPerBlock];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    ForceSmem<kDPD> &sm = smem_all[w];
    const unsigned lt_mask = (1u << lane) - 1u;
    const int ntypes = v.ntypes;
    const bool use_mask = ntypes <= 32;
    for (int c = blockIdx.x * kWarpsPerBlock + w; c < v.ncells; c += gridDim.x * kWarpsPerBlock) {
        const int n = v.cell_count[c];
        double ecell = 0.0;
        if (n > 0) {
            const int start = v.cell_start[c];
            const DevSpace &S = v.spaces[v.cell_rep[c]];
            const int pot_base = S.pot_offset;
            const float cut2_pair = S.cut2_pair, cut2_self = S.cut2_self;
            const unsigned rng_mode = S.rng_mode;
            const bool prune = (S.prune & 1) != 0;      // per-pair projection test
            const bool exit_test = (S.prune & 2) != 0;  // cell-pair exit test
            const float sbias = S.sort_bias, sdscale = S.sort_dscale;
            const int dmaxdist = S.dmaxdist;
            const int nb0 = v.nb_off[c], nb1 = v.nb_off[c + 1];
            for (int i0 = 0; i0 < n; i0 += kOwn) {
                const int ni = min(kOwn, n - i0);
                __syncwarp();
                if (lane < ni) {
                    const float4 x = v.pos[start + i0 + lane];
                    sm.own_x[lane] = x;
                    const int ti = __float_as_int(x.w);
                    const DevType &T = v.types[ti];
                    // constant_force (MxForce.cpp:339-344), scale 1
                    sm.own_f[lane] = T.has_force ? make_float4(T.fx, T.fy, T.fz, 0.f) : make_float4(0.f, 0.f, 0.f, 0.f);
                    if (kDPD) sm.own_v[lane] = v.vel[start + i0 + lane];
                    if (use_mask) {
                        int mk = 0;
                        for (int t = 0; t < ntypes; ++t)
                            if (v.pot_idx[pot_base + ti * ntypes + t] >= 0) mk |= 1 << t;
                        sm.own_mask[lane] = mk;
                    }
                }
                int e = nb0, jpos = 0;
                while (e < nb1) {
                    // ---- region: lane k describes entry e + k
                    const int ek = e + lane;
                    int cnt = 0, cstart = 0, pk = 0;
                    float4 sh = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (ek < nb1) {
                        const int nc = v.nb_cell[ek];
                        sh = v.nb_shift[ek];
                        pk = __float_as_int(sh.w);
                        cnt = v.cell_count[nc];
                        cstart = v.cell_start[nc];
                        const int role = pk & 3;
                        if (cnt > 0 && exit_test && role != kRoleSelf) {
                            // runner_dopair.cpp:167-171: kmin(second) + dnshift - kmax(first) in
                            // unsigned arithmetic; above dmaxdist or wrapped, the pair is skipped
                            const int sid = (pk >> 2) & 15;
                            const int2 bc = v.sort_bounds[c * 13 + sid], bn = v.sort_bounds[nc * 13 + sid];
                            const int kmax_first = role == kRoleFirst ? bc.y : bn.y;
                            const int kmin_second = role == kRoleFirst ? bn.x : bc.x;
                            const int gap = kmin_second + (pk >> 8) - kmax_first;
                            if (gap < 0 || gap > dmaxdist) cnt = 0;
                        }
                    }
                    const int jb = lane == 0 ? jpos : 0;
                    const int rem = max(cnt - jb, 0);
                    int incl = rem;
                    for (int off = 1; off < 32; off <<= 1) {
                        const int o = __shfl_up_sync(kFull, incl, off);
                        if (lane >= off) incl += o;
                    }
                    const int nfit = __popc(__ballot_sync(kFull, ek < nb1 && incl <= kCap));
                    int nent, M;
                    if (nfit == 0) {  // the first entry alone holds more than kCap particles
                        nent = 1;
                        M = kCap;
                        jpos += kCap;
                    } else {
                        nent = nfit;
                        M = __shfl_sync(kFull, incl, nfit - 1);
                        e += nfit;
                        jpos = 0;
                    }
                    __syncwarp();
                    if (lane < nent) {
                        sm.ent_beg[lane] = incl - rem;
                        sm.ent_slot[lane] = cstart;
                        sm.ent_jb[lane] = jb;
                        sm.ent_sh[lane] = sh;
                    }
                    if (lane == 0) sm.ent_beg[nent] = M;
                    __syncwarp();
                    if (M == 0) continue;
                    // ---- stage the region's neighbour particles
                    for (int idx = lane; idx < M; idx += 32) {
                        int k = 0;
                        for (int step = 16; step > 0; step >>= 1)
                            if (k + step < nent && sm.ent_beg[k + step] <= idx) k += step;
                        const int jl = sm.ent_jb[k] + idx - sm.ent_beg[k];
                        const int slot = sm.ent_slot[k] + jl;
                        const float4 es = sm.ent_sh[k];
                        const int epk = __float_as_int(es.w);
                        const int role = epk & 3;
                        float4 q = v.pos[slot];
                        if (prune) sm.nb_key[idx] = sort_key(q.x, q.y, q.z, v.axes->n[(epk >> 2) & 15], sbias, sdscale);
                        float4 s4 = make_float4(0.f, 0.f, 0.f, __int_as_float(role | (k << 2) | (jl << 8)));
                        if (role == kRoleSecond) {
                            q.x = __fsub_rn(q.x, es.x);
                            q.y = __fsub_rn(q.y, es.y);
                            q.z = __fsub_rn(q.z, es.z);
                        } else if (role == kRoleFirst) {
                            s4.x = es.x;
                            s4.y = es.y;
                            s4.z = es.z;
                        }
                        sm.nb_x[idx] = q;
                        sm.nb_s[idx] = s4;
                        if (kDPD) sm.nb_v[idx] = v.vel[slot];
                    }
                    __syncwarp();
                    // ---- pass 1 (candidates) and pass 2 (full batches)
                    int qlen = 0;
                    for (int il = 0; il < ni; ++il) {
                        const float4 xi = sm.own_x[il];
                        const int i = i0 + il;
                        const int ti = __float_as_int(xi.w);
                        const int mk = use_mask ? sm.own_mask[il] : 0;
                        for (int jb0 = 0; jb0 < M; jb0 += 32) {
                            const int jj = jb0 + lane;
                            bool hit = false;
                            if (jj < M) {
                                const float4 b = sm.nb_x[jj];
                                const float4 s = sm.nb_s[jj];
                                const int meta = __float_as_int(s.w);
                                const int role = meta & 3;
                                const float dx = __fsub_rn(__fsub_rn(xi.x, s.x), b.x);
                                const float dy = __fsub_rn(__fsub_rn(xi.y, s.y), b.y);
                                const float dz = __fsub_rn(__fsub_rn(xi.z, s.z), b.z);
                                const float r2 = dot3_rn(dx, dy, dz);
                                const int tj = __float_as_int(b.w);
                                hit = r2 <= (role == kRoleSelf ? cut2_self : cut2_pair);
                                hit = hit && (use_mask ? ((mk >> tj) & 1) != 0
                                                       : v.pot_idx[pot_base + ti * ntypes + tj] >= 0);
                                if (role == kRoleSelf) hit = hit && (meta >> 8) != i;
                                if (prune && hit && role != kRoleSelf) {
                                    // runner_dopair's pruning: a pair (first, second) is evaluated
                                    // only when key_second + dnshift - key_first < dmaxdist
                                    // (runner_dopair.cpp:167-182)
                                    const int epk = __float_as_int(sm.ent_sh[(meta >> 2) & 63].w);
                                    const int okey =
                                        sort_key(xi.x, xi.y, xi.z, v.axes->n[(epk >> 2) & 15], sbias, sdscale);
                                    const int kf = role == kRoleFirst ? okey : sm.nb_key[jj];
                                    const int ks = role == kRoleFirst ? sm.nb_key[jj] : okey;
                                    hit = ks + (epk >> 8) - kf < dmaxdist;
                                }
                            }
                            const unsigned hb = __ballot_sync(kFull, hit);
                            if (hit) sm.queue[qlen + __popc(hb & lt_mask)] = (il << 16) | jj;
                            qlen += __popc(hb);
                            if (qlen >= 32) {
                                __syncwarp();
                                eval_batch<kDPD, kStats>(v, sm, 32, i0, start, pot_base, rng_mode, ecell, npair);
                                qlen -= 32;
                                const int moved = lane < qlen ? sm.queue[32 + lane] : 0;
                                __syncwarp();
                                if (lane < qlen) sm.queue[lane] = moved;
                                __syncwarp();
                            }
                        }
                    }
                    if (qlen > 0) {
                        __syncwarp();
                        eval_batch<kDPD, kStats>(v, sm, qlen, i0, start, pot_base, rng_mode, ecell, npair);
                    }
                    __syncwarp();
                }
                __syncwarp();
                if (lane < ni) {
                    const float4 f = sm.own_f[lane];
                    v.force[start + i0 + lane] = make_float4(f.x, f.y, f.z, 0.f);
                }
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

void configure_force_kernels() {
    // the force kernel's occupancy is bounded by shared memory: ask for the
    // largest shared-memory carveout of the unified L1/shared storage
    const int carve = cudaSharedmemCarveoutMaxShared;
    cudaFuncSetAttribute(force_kernel<true, true>, cudaFuncAttributePreferredSharedMemoryCarveout, carve);
    cudaFuncSetAttribute(force_kernel<true, false>, cudaFuncAttributePreferredSharedMemoryCarveout, carve);
    cudaFuncSetAttribute(force_kernel<false, true>, cudaFuncAttributePreferredSharedMemoryCarveout, carve);
    cudaFuncSetAttribute(force_kernel<false, false>, cudaFuncAttributePreferredSharedMemoryCarveout, carve);
}

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
