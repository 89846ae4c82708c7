/*
 * Adjoint (reverse-mode) kernels of the force-and-step path.
 *
 * One forward-Euler step maps (x, v) to (x', v'):
 *     v'_k = clamp(mask_k (v_k + dt f_k(x, v; theta) imass))       (Newtonian)
 *     x'   = x + dt v'
 * or, overdamped, x'_k = x_k + clamp(mask_k dt f_k imass) with v unchanged
 * (engine_advance.cpp:126-239). Given the adjoints (lx, lv) of (x', v'), the
 * step's vector-Jacobian product is
 *     g      = lv + dt lx            (adjoint of v', Newtonian)
 *     gpre_k = clamped_k ? 0 : g_k   (through the speed clamp and the frozen mask)
 *     w      = dt imass gpre         (adjoint of the force on the particle)
 *     lx_in  = lx + sum_pairs J_x^T (w_i - w_j)
 *     lv_in  = gpre + sum_pairs J_v^T (w_i - w_j)
 *     dL/dtheta += sum_pairs (dF_ij/dtheta) . (w_i - w_j)
 * where F_ij is the force of j on i. The pair sums are taken by vjp_pair_kernel
 * over the same cell-pair lists as the force pass, but from both sides (each
 * cell sums its own particles' terms from all 27 neighbour entries), so no
 * cross-warp sums are needed. Parameter gradients are counted once per pair
 * (on the side with the smaller particle id) in FP64.
 *
 * The derivative of a tabulated potential is that of the piecewise polynomial
 * itself, and parameter derivatives use tables of dV/dtheta fitted on the same
 * frozen nodes (the fit is linear in the sampled function), so the gradients
 * are those of the tabulated model the forward pass integrates. Bonds add
 * their terms in vjp_bond_kernel (the break flags held fixed). Wall
 * reflections, angles, dihedrals and exclusions are not differentiated (the
 * adjoint covers periodic boxes, nonbonded potentials, bonds and constant
 * forces).
 */
#include "mxg_adjoint.h"

#include <algorithm>
#include "mxg_device.cuh"

namespace mxg {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kOwnA = 32;              // own particles staged at a time
constexpr int kCapA = 64;              // neighbour particles staged at a time
constexpr int kChunksA = kCapA / 32;
constexpr int kQueueA = 128;           // ring buffer of queued pairs (holds kCapA + 31)
constexpr int kEntA = 32;              // neighbour entries cached at a time
constexpr int kWarpsA = 4;             // warps (work items) per block
constexpr int kVjpParts = 4;           // work items per cell (contiguous groups of its entries)

struct AdjSmem {
    float4 nb_x[kCapA];   // neighbour position (SECOND entries pre-shifted); w = type
    float4 nb_s[kCapA];   // shift of FIRST entries, else 0; w = role | entry << 2 | index << 8
    float4 nb_v[kCapA];   // velocity; w = id
    float4 nb_w[kCapA];   // force adjoint
    float4 own_x[kOwnA];
    float4 own_v[kOwnA];
    float4 own_w[kOwnA];
    float4 own_gx[kOwnA];
    float4 own_gv[kOwnA];
    float4 ent_sh[kEntA];
    int ent_slot[kEntA];
    int ent_cnt[kEntA];
    int reg_beg[kEntA + 1];
    int reg_jb[kEntA];
    unsigned long long own_mask[kOwnA];
    unsigned short queue[kQueueA];
};

constexpr size_t adj_smem_bytes() {
    return (sizeof(AdjSmem) + 32 * kMaxGradSlots * sizeof(double)) * kWarpsA;
}

/* P(x), P'(x), P''(x) of an interval polynomial c[2] x^5 + ... + c[7]. */
__device__ __forceinline__ void poly3(const float *c, float x, float &p, float &dp, float &ddp) {
    p = c[2];
    dp = 0.f;
    float d2 = 0.f;
#pragma unroll
    for (int k = 3; k < 8; ++k) {
        d2 = d2 * x + dp;
        dp = dp * x + p;
        p = p * x + c[k];
    }
    ddp = 2.f * d2;
}

/* Table term: adds J_x^T u to gx and the parameter terms (if count) into g. */
__device__ __forceinline__ void table_vjp(const EngineView &v, const AdjointView &a, int pidx, const DevPot &p,
                                          float radi, float radj, const float3 &d, float r2, const float3 &u,
                                          bool count, float3 &gx, double *g) {
    const float r = sqrtf(r2);
    const float ro = r < 1.19209290e-7f ? 1.19209290e-7f : r;
    const bool clamped = r < p.a;
    const float rr = clamped ? p.a : r;
    float s = rr, dsdr = 1.f;
    if (p.flags & (1u << 11)) {
        s = rr / (radi + radj);
        dsdr = 1.f / (radi + radj);
    } else if (p.flags & (1u << 12)) {
        s = rr - (radi + radj) + p.r0_plusone;
    }
    if (clamped) dsdr = 0.f;
    const float t = p.alpha0 + s * (p.alpha1 + s * p.alpha2);
    const unsigned ind = (unsigned)fmaxf(0.0f, t);
    if (s > p.b || ind > (unsigned)p.n) return;
    const float *c = v.coef + p.coef_off + ind * kChunk;
    const float x = (s - c[0]) * c[1];
    float P, dP, ddP;
    poly3(c, x, P, dP, ddP);
    const float vp = dP * c[1], vpp = ddP * c[1] * c[1];
    const float f = vp / ro;
    const float dfdr = vpp * dsdr / ro - (r >= 1.19209290e-7f ? vp / (ro * ro) : 0.f);
    const float du = d.x * u.x + d.y * u.y + d.z * u.z;
    const float k = r > 0.f ? dfdr / r * du : 0.f;
    // F_i = -f d:  J^T u = -(f u + (df/dr / r)(d.u) d)
    gx.x -= f * u.x + k * d.x;
    gx.y -= f * u.y + k * d.y;
    gx.z -= f * u.z + k * d.z;
    if (!count) return;
    const DevPotGrad &pg = a.pot_grad[pidx];
    for (int q = 0; q < pg.n; ++q) {
        float fth = 0.f;
        if (pg.mode[q] == kGradTable) {
            const float *cd = a.dcoef + pg.coef_off[q] + ind * kChunk;
            float Pq, dPq, ddPq;
            poly3(cd, x, Pq, dPq, ddPq);
            fth = dPq * c[1] / ro;
        } else if (pg.mode[q] == kGradShift) {
            fth = vpp / ro;  // d s / d r0 = 1
        } else {
            continue;
        }
        g[pg.slot[q]] += (double)(-fth * du);
    }
}

/* DPD term (dpd_eval.hpp:21-69 with xi): adds J_x^T u, J_v^T u and the
 * parameter terms. */
__device__ __forceinline__ void dpd_vjp(const EngineView &v, const AdjointView &a, int pidx, const DevPot &p,
                                        float radi, float radj, const float3 &d, float r2, const float3 &vij,
                                        float xi_rand, const float3 &u, bool count, float3 &gx, float3 &gv,
                                        double *g) {
    const bool shifted = p.flags & (1u << 12);
    const float cutoff = shifted ? p.b + radi + radj : p.b;
    if (r2 > cutoff * cutoff || r2 <= 0.f) return;
    const float r = sqrtf(r2);
    const float ir = 1.f / r;
    const float3 e = make_float3(d.x * ir, d.y * ir, d.z * ir);
    const float sr = shifted ? r - radi - radj : r;
    const bool inner = sr < 0.f;
    const float om = inner ? 1.f : 1.f - sr / cutoff;
    const float domdr = inner ? 0.f : -1.f / cutoff;
    const float sv = e.x * vij.x + e.y * vij.y + e.z * vij.z;
    const float eu = e.x * u.x + e.y * u.y + e.z * u.z;
    const float rnd = p.dpd_sigma * xi_rand * p.dpd_delta;
    const float h = p.dpd_alpha * om - p.dpd_gamma * om * om * sv + rnd * om;
    const float dhdr = (p.dpd_alpha - 2.f * p.dpd_gamma * om * sv + rnd) * domdr;
    const float dhds = -p.dpd_gamma * om * om;
    // d(u.F)/dd = dh/dr (e.u) e + dh/ds (e.u) (v - s e)/r + h (u - (e.u) e)/r
    const float a1 = dhdr * eu, a2 = dhds * eu * ir, a3 = h * ir;
    gx.x += a1 * e.x + a2 * (vij.x - sv * e.x) + a3 * (u.x - eu * e.x);
    gx.y += a1 * e.y + a2 * (vij.y - sv * e.y) + a3 * (u.y - eu * e.y);
    gx.z += a1 * e.z + a2 * (vij.z - sv * e.z) + a3 * (u.z - eu * e.z);
    gv.x += dhds * eu * e.x;
    gv.y += dhds * eu * e.y;
    gv.z += dhds * eu * e.z;
    if (!count) return;
    const DevPotGrad &pg = a.pot_grad[pidx];
    for (int q = 0; q < pg.n; ++q) {
        float dth;
        if (pg.mode[q] == kGradDpdAlpha)
            dth = om * eu;
        else if (pg.mode[q] == kGradDpdGamma)
            dth = -om * om * sv * eu;
        else if (pg.mode[q] == kGradDpdSigma)
            dth = om * xi_rand * p.dpd_delta * eu;
        else
            continue;
        g[pg.slot[q]] += (double)dth;
    }
}

__device__ __forceinline__ void term_vjp(const EngineView &v, const AdjointView &a, int pidx, float radi,
                                         float radj, const float3 &d, float r2, const float3 &vij, unsigned ida,
                                         unsigned idb, unsigned rng_mode, const float3 &u, bool count, float3 &gx,
                                         float3 &gv, double *g) {
    const DevPot &p = v.pots[pidx];
    if (r2 < p.a2) return;  // the random-direction branch is not differentiated
    if (p.kind == 1) {
        float xr = 1.0f;
        if (rng_mode) {
            const unsigned lo = ida < idb ? ida : idb, hi = ida < idb ? idb : ida;
            xr = philox_pair_xi(*v.step, lo, hi);
        }
        dpd_vjp(v, a, pidx, p, radi, radj, d, r2, vij, xr, u, count, gx, gv, g);
    } else {
        table_vjp(v, a, pidx, p, radi, radj, d, r2, u, count, gx, g);
    }
}

/* Per slot: the adjoint through the integrator; w = dt imass gpre is the
 * adjoint of the particle's force. f must hold the forces of the state. */
__global__ void adj_prep_kernel(EngineView v, AdjointView a) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= v.nparts) return;
    const float4 x = v.pos[s], u = v.vel[s], f = v.force[s];
    const int id = __float_as_int(u.w);
    const DevType &T = v.types[__float_as_int(x.w)];
    const DevSpace &S = v.spaces[v.cell_rep[v.cell_of[s]]];
    const float4 lx = a.lam_x[id], lv = a.lam_v[id];
    const float lxv[3] = {lx.x, lx.y, lx.z}, lvv[3] = {lv.x, lv.y, lv.z};
    const float uv[3] = {u.x, u.y, u.z}, fv[3] = {f.x, f.y, f.z};
    float w[3] = {0.f, 0.f, 0.f}, gv[3] = {lvv[0], lvv[1], lvv[2]};
    const unsigned fz_all = (1u << 2) | (1u << 3) | (1u << 4);
    if ((T.flags & fz_all) != fz_all) {
        const float dt = S.dt;
        for (int k = 0; k < 3; ++k) {
            const bool frozen = T.flags & (1u << (2 + k));
            if (T.dynamics == 0) {
                // a frozen component gets v' = 0 (the mask), so nothing flows back through it
                const float vk = (float)((double)uv[k] + (double)(dt * fv[k]) * T.imass);
                const bool clamped = frozen || vk * vk > S.maxv2[k];
                const float gk = lvv[k] + dt * lxv[k];
                const float gpre = clamped ? 0.f : gk;
                gv[k] = gpre;
                w[k] = (float)((double)(gpre * dt) * T.imass);
            } else {
                const float dxk = (float)((double)(dt * fv[k]) * T.imass);
                const bool clamped = frozen || dxk * dxk > S.maxx2[k];
                w[k] = clamped ? 0.f : (float)((double)(lxv[k] * dt) * T.imass);
            }
        }
    }
    a.w[s] = make_float4(w[0], w[1], w[2], 0.f);
    a.gx[s] = make_float4(lxv[0], lxv[1], lxv[2], 0.f);
    a.gv[s] = make_float4(gv[0], gv[1], gv[2], 0.f);
}

/* Pair terms of the step's VJP. One warp per cell, full shell (SELF, FIRST and
 * SECOND entries); the structure follows force_kernel: staged regions, a
 * candidate pass one neighbour per lane, then the interacting pairs 32 at a
 * time with per-particle segmented sums. */
__global__ void __launch_bounds__(kWarpsA * 32, 4) vjp_pair_kernel(EngineView v, AdjointView a) {
    extern __shared__ float4 adj_smem[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    AdjSmem &sm = reinterpret_cast<AdjSmem *>(adj_smem)[w];
    double *gl = reinterpret_cast<double *>(reinterpret_cast<AdjSmem *>(adj_smem) + kWarpsA) +
                 (size_t)(w * 32 + lane) * kMaxGradSlots;  // this lane's parameter sums
    for (int q = 0; q < kMaxGradSlots; ++q) gl[q] = 0.0;
    const unsigned lt_mask = (1u << lane) - 1u;
    const int ntypes = v.ntypes;
    const int nwarps = gridDim.x * kWarpsA;
    // work items from a counter (a cell's parts are items of their own, so no warp holds a
    // crowded cell alone); every item writes only its own outputs and parameter partials
    auto fetch = [&]() -> int {
        int t = 0;
        if (lane == 0) t = atomicAdd(a.item_ctr, 1);
        return __shfl_sync(kFull, t, 0);
    };
    for (int it = fetch(); it < a.nitems; it = fetch()) {
        const int4 item = a.items[it];
        const int c = item.x, nb0 = item.y, nb1 = item.z, part = item.w;
        const int n = v.cell_count[c];
        const int start = v.cell_start[c];
        const DevSpace &S = v.spaces[v.cell_rep[c]];
        const int pot_base = S.pot_offset;
        const float cut2_pair = S.cut2_pair, cut2_self = S.cut2_self;
        const float cut2w_pair = S.cut2w_pair, cut2w_self = S.cut2w_self;
        const unsigned rng_mode = S.rng_mode;
        for (int i0 = 0; i0 < n; i0 += kOwnA) {
            const int ni = min(kOwnA, n - i0);
            __syncwarp();
            if (lane < ni) {
                const int sl = start + i0 + lane;
                const float4 x = v.pos[sl];
                sm.own_x[lane] = x;
                sm.own_v[lane] = v.vel[sl];
                sm.own_w[lane] = a.w[sl];
                sm.own_gx[lane] = make_float4(0.f, 0.f, 0.f, 0.f);
                sm.own_gv[lane] = make_float4(0.f, 0.f, 0.f, 0.f);
                const int ti = __float_as_int(x.w);
                unsigned long long mk = 0ull;
                for (int t = 0; t < ntypes; ++t)
                    if (v.pot_idx[pot_base + ti * ntypes + t] >= 0) mk |= 1ull << t;
                sm.own_mask[lane] = mk;
            }
            for (int g0 = nb0; g0 < nb1; g0 += kEntA) {
                const int ek = g0 + lane;
                int cnt = 0, cstart = 0;
                float4 sh = make_float4(0.f, 0.f, 0.f, 0.f);
                if (ek < nb1) {
                    sh = v.nb_shift[ek];
                    const int nc = v.nb_cell[ek];
                    cnt = v.cell_count[nc];
                    cstart = v.cell_start[nc];
                }
                const unsigned staged = __ballot_sync(kFull, cnt > 0);
                const int nst = __popc(staged);
                __syncwarp();
                if (cnt > 0) {
                    const int k = __popc(staged & lt_mask);
                    sm.ent_sh[k] = sh;
                    sm.ent_slot[k] = cstart;
                    sm.ent_cnt[k] = cnt;
                }
                __syncwarp();
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
                    const int nfit = __popc(__ballot_sync(kFull, k < nst && incl <= kCapA));
                    int nent, M;
                    if (nfit == 0) {
                        nent = 1;
                        M = kCapA;
                        jpos += kCapA;
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
                    // lane's chunk-u neighbour (staged index u * 32 + lane) is also kept in registers
                    // for the candidate pass: its position plus the entry's shift, a widened cutoff
                    // (-1: empty), its index in the cell when it is a SELF neighbour (else -1) and its
                    // type; the candidate pass is a superset filter, the drain applies the exact test
                    float rbx[kChunksA], rby[kChunksA], rbz[kChunksA], rc2[kChunksA];
                    int rself[kChunksA], rtj[kChunksA];
                    unsigned long long rtypes = 0ull;
                    bool rs_any = false;
#pragma unroll
                    for (int u = 0; u < kChunksA; ++u) {
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
                            const int role = __float_as_int(es.w) & 3;
                            float4 q = v.pos[slot];
                            float4 s4 = make_float4(0.f, 0.f, 0.f, __int_as_float(role | (ke << 2) | (jl << 8)));
                            if (role == kRoleSecond) {
                                q.x -= es.x;
                                q.y -= es.y;
                                q.z -= es.z;
                            } else if (role == kRoleFirst) {
                                s4.x = es.x;
                                s4.y = es.y;
                                s4.z = es.z;
                            }
                            sm.nb_x[idx] = q;
                            sm.nb_s[idx] = s4;
                            sm.nb_v[idx] = v.vel[slot];
                            sm.nb_w[idx] = a.w[slot];
                            rbx[u] = __fadd_rn(q.x, s4.x);
                            rby[u] = __fadd_rn(q.y, s4.y);
                            rbz[u] = __fadd_rn(q.z, s4.z);
                            rc2[u] = role == kRoleSelf ? cut2w_self : cut2w_pair;
                            rself[u] = role == kRoleSelf ? jl : -1;
                            rtj[u] = __float_as_int(q.w);
                            rtypes |= 1ull << rtj[u];
                            rs_any |= role == kRoleSelf;
                        }
                    }
                    // the candidate test's form for the whole region: the type test is moot when every
                    // own particle has a potential with every type staged, the own-index test when no
                    // SELF neighbour is staged (2: the full test)
                    int pmode = 2;
                    {
                        rtypes = (unsigned long long)__reduce_or_sync(kFull, (unsigned)rtypes) |
                                 ((unsigned long long)__reduce_or_sync(kFull, (unsigned)(rtypes >> 32)) << 32);
                        bool full = true;
                        for (int k = lane; k < ni; k += 32) full &= (sm.own_mask[k] & rtypes) == rtypes;
                        if (__all_sync(kFull, full)) pmode = __any_sync(kFull, rs_any) ? 1 : 0;
                    }
                    __syncwarp();
                    int qhead = 0, qtail = 0;
                    auto drain = [&](int nb) {
                        float3 gx = make_float3(0.f, 0.f, 0.f), gv = make_float3(0.f, 0.f, 0.f);
                        int il = -1;
                        if (lane < nb) {
                            const int cd = sm.queue[(qhead + lane) & (kQueueA - 1)];
                            il = cd >> 8;
                            const int jj = cd & 0xff;
                            const float4 xi = sm.own_x[il], b = sm.nb_x[jj], s = sm.nb_s[jj];
                            const float3 d = make_float3((xi.x - s.x) - b.x, (xi.y - s.y) - b.y, (xi.z - s.z) - b.z);
                            const float r2 = d.x * d.x + d.y * d.y + d.z * d.z;
                            // the exact cutoff test of the pair loops (the candidate pass queued a superset)
                            const bool inside = r2 <= ((__float_as_int(s.w) & 3) == kRoleSelf ? cut2_self : cut2_pair);
                            const float4 vi = sm.own_v[il], vj = sm.nb_v[jj];
                            const float4 wi = sm.own_w[il], wj = sm.nb_w[jj];
                            const float3 u = make_float3(wi.x - wj.x, wi.y - wj.y, wi.z - wj.z);
                            const float3 vij = make_float3(vi.x - vj.x, vi.y - vj.y, vi.z - vj.z);
                            const int ti = __float_as_int(xi.w), tj = __float_as_int(b.w);
                            const unsigned ida = __float_as_uint(vi.w), idb = __float_as_uint(vj.w);
                            const bool count = ida < idb;
                            const float radi = v.types[ti].radius, radj = v.types[tj].radius;
                            // the pair's potential, then a second one summed on it: one call site, so
                            // that the kernel's instruction footprint holds one copy of the terms
                            const int p1 = v.pot_idx[pot_base + ti * ntypes + tj];
                            const int p2 = v.pot_idx2 ? v.pot_idx2[pot_base + ti * ntypes + tj] : -1;
#pragma unroll 1
                            for (int k = 0; k < 2 && inside; ++k) {
                                const int pk = k == 0 ? p1 : p2;
                                if (pk >= 0)
                                    term_vjp(v, a, pk, radi, radj, d, r2, vij, ida, idb, rng_mode, u, count, gx, gv, gl);
                            }
                        }
                        const int il_prev = __shfl_up_sync(kFull, il, 1);
                        const unsigned heads = __ballot_sync(kFull, lane == 0 || il != il_prev);
                        const int seg0 = 31 - __clz(heads & (0xffffffffu >> (31 - lane)));
                        for (int off = 1; off < 32; off <<= 1) {
                            const float o0 = __shfl_up_sync(kFull, gx.x, off), o1 = __shfl_up_sync(kFull, gx.y, off);
                            const float o2 = __shfl_up_sync(kFull, gx.z, off), o3 = __shfl_up_sync(kFull, gv.x, off);
                            const float o4 = __shfl_up_sync(kFull, gv.y, off), o5 = __shfl_up_sync(kFull, gv.z, off);
                            if (lane - off >= seg0) {
                                gx.x = o0 + gx.x;
                                gx.y = o1 + gx.y;
                                gx.z = o2 + gx.z;
                                gv.x = o3 + gv.x;
                                gv.y = o4 + gv.y;
                                gv.z = o5 + gv.z;
                            }
                        }
                        const bool seg_end = lane == 31 || ((heads >> (lane + 1)) & 1u);
                        if (il >= 0 && seg_end) {
                            float4 t = sm.own_gx[il];
                            sm.own_gx[il] = make_float4(t.x + gx.x, t.y + gx.y, t.z + gx.z, 0.f);
                            t = sm.own_gv[il];
                            sm.own_gv[il] = make_float4(t.x + gv.x, t.y + gv.y, t.z + gv.z, 0.f);
                        }
                    };
                    for (int il = 0; il < ni; ++il) {
                        const float4 xi = sm.own_x[il];
                        const int i = i0 + il;
                        unsigned hb[kChunksA];
                        bool hv[kChunksA];
                        // squared distance by fused multiply-adds: a superset filter with a widened cutoff
                        if (pmode == 0) {
#pragma unroll
                            for (int u = 0; u < kChunksA; ++u) {
                                const float dx = __fsub_rn(xi.x, rbx[u]), dy = __fsub_rn(xi.y, rby[u]),
                                            dz = __fsub_rn(xi.z, rbz[u]);
                                hv[u] = __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmul_rn(dz, dz))) <= rc2[u];
                                hb[u] = __ballot_sync(kFull, hv[u]);
                            }
                        } else if (pmode == 1) {
#pragma unroll
                            for (int u = 0; u < kChunksA; ++u) {
                                const float dx = __fsub_rn(xi.x, rbx[u]), dy = __fsub_rn(xi.y, rby[u]),
                                            dz = __fsub_rn(xi.z, rbz[u]);
                                hv[u] = (__fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmul_rn(dz, dz))) <= rc2[u]) & (rself[u] != i);
                                hb[u] = __ballot_sync(kFull, hv[u]);
                            }
                        } else {
                            const unsigned long long mk = sm.own_mask[il];
#pragma unroll
                            for (int u = 0; u < kChunksA; ++u) {
                                const float dx = __fsub_rn(xi.x, rbx[u]), dy = __fsub_rn(xi.y, rby[u]),
                                            dz = __fsub_rn(xi.z, rbz[u]);
                                hv[u] = (__fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmul_rn(dz, dz))) <= rc2[u]) &
                                        (rself[u] != i) & (((mk >> rtj[u]) & 1ull) != 0ull);
                                hb[u] = __ballot_sync(kFull, hv[u]);
                            }
                        }
#pragma unroll
                        for (int u = 0; u < kChunksA; ++u) {
                            if (hv[u])
                                sm.queue[(qtail + __popc(hb[u] & lt_mask)) & (kQueueA - 1)] =
                                    (unsigned short)((il << 8) | (u * 32 + lane));
                            qtail += __popc(hb[u]);
                        }
                        while (qtail - qhead >= 32) {
                            __syncwarp();
                            drain(32);
                            qhead += 32;
                            __syncwarp();
                        }
                    }
                    if (qtail > qhead) {
                        __syncwarp();
                        drain(qtail - qhead);
                    }
                    __syncwarp();
                }
            }
            __syncwarp();
            if (lane < ni) {
                const int sl = start + i0 + lane;
                const float4 gx = sm.own_gx[lane], gv = sm.own_gv[lane];
                if (part == 0) {
                    const float4 bx = a.gx[sl], bv = a.gv[sl];
                    a.gx[sl] = make_float4(bx.x + gx.x, bx.y + gx.y, bx.z + gx.z, 0.f);
                    a.gv[sl] = make_float4(bv.x + gv.x, bv.y + gv.y, bv.z + gv.z, 0.f);
                } else {
                    a.pgx[(size_t)(part - 1) * v.nparts + sl] = gx;
                    a.pgv[(size_t)(part - 1) * v.nparts + sl] = gv;
                }
            }
        }
        // this item's parameter sums, lanes in order; then the lanes' sums start again
        __syncwarp();
        if (lane < kMaxGradSlots && lane < a.nslots) {
            double *base = reinterpret_cast<double *>(reinterpret_cast<AdjSmem *>(adj_smem) + kWarpsA) +
                           (size_t)(w * 32) * kMaxGradSlots;
            double t = 0.0;
            for (int l = 0; l < 32; ++l) t += base[(size_t)l * kMaxGradSlots + lane];
            a.partials[(size_t)lane * a.nitems + it] = t;
        }
        __syncwarp();
        for (int q = 0; q < kMaxGradSlots; ++q) gl[q] = 0.0;
    }
    if (lane == 0) {
        // every warp has drawn its last ticket once the done count reaches the grid's warps:
        // the last one re-arms both counters for the next launch on the stream
        if (atomicAdd(a.item_ctr + 1, 1) == nwarps - 1) {
            atomicExch(a.item_ctr, 0);
            atomicExch(a.item_ctr + 1, 0);
        }
    }
}

constexpr int kBondVjpThreads = 128;
constexpr int kGradPad = kMaxGradSlots + 1;  // shared row stride (doubles): fewer bank conflicts

/*
 * Bond terms of the step's VJP (bond_eval, bond.cpp:99-312, with potential_eval's
 * table semantics). One thread per particle slot visits the bonds of its
 * particle that acted in the step's bond pass: the flags are read after that
 * pass, so a bond broken before the step or by it contributes nothing (the
 * break decision is a step function of the state and is held fixed). With
 * d = x_i - x_j (x_i in x_j's cell frame, as the forward pass forms it) and
 * f = V'(r_c)/r_c at the clamped length r_c = sqrt(clamp(|d|^2, a^2, b^2)),
 * the bond's forces are F_i = -f d = -F_j. For u = w_i - w_j (the force
 * adjoints) its share of the position adjoint is -A u at i and +A u at j, with
 * A = f I + (f'(r)/r) d d^T (f' = 0 where the length is clamped). The
 * parameter terms -(df/dtheta)(d.u) are counted once, at the bond's i end;
 * df/dtheta comes from the tables of dV/dtheta fitted on the bond table's
 * frozen nodes (harmonic k and r0). Parameter sums: per thread in shared
 * memory, then per block in thread order (deterministic).
 */
__global__ void __launch_bounds__(kBondVjpThreads) vjp_bond_kernel(EngineView v, BondedView bv, AdjointView a) {
    __shared__ double gsum[kBondVjpThreads * kGradPad];
    double *g = gsum + threadIdx.x * kGradPad;
    for (int q = 0; q < kMaxGradSlots; ++q) g[q] = 0.0;
    const int stride = gridDim.x * blockDim.x;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < v.nparts; s += stride) {
        const int id = __float_as_int(v.vel[s].w);
        const int k0 = bv.bond_off[id], k1 = bv.bond_off[id + 1];
        if (k0 == k1) continue;
        float gx[3] = {0.f, 0.f, 0.f};
        for (int k = k0; k < k1; ++k) {
            const int b = bv.bond_list[k];
            if (!(bv.bond_flags[b] & 1u)) continue;
            const DevBond B = bv.bonds[b];
            const int si = bv.slot_of_id[B.i], sj = bv.slot_of_id[B.j];
            if (si < 0 || sj < 0 || si == sj) continue;
            const int ci = v.cell_of[si];
            const DevSpace &S = v.spaces[v.cell_rep[ci]];
            float d[3];
            bond_vector(S, ci, v.cell_of[sj], v.pos[si], v.pos[sj], d);
            const DevPot &p = v.pots[B.pot];
            const float r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            const float a2 = p.a * p.a, b2 = p.b * p.b;
            const bool clamped = r2 < a2 || r2 > b2;
            const float rc = sqrtf(fmaxf(a2, fminf(b2, r2)));
            const float t = p.alpha0 + rc * (p.alpha1 + rc * p.alpha2);
            const int ind = min((int)fmaxf(0.0f, t), p.n);
            const float *c = v.coef + p.coef_off + ind * kChunk;
            const float x = (rc - c[0]) * c[1];
            float P, dP, ddP;
            poly3(c, x, P, dP, ddP);
            const float vp = dP * c[1], vpp = ddP * c[1] * c[1];
            const float f = vp / rc;
            const float dfdr = clamped ? 0.f : vpp / rc - vp / (rc * rc);
            const float4 wi = a.w[si], wj = a.w[sj];
            const float u[3] = {wi.x - wj.x, wi.y - wj.y, wi.z - wj.z};
            const float du = d[0] * u[0] + d[1] * u[1] + d[2] * u[2];
            const float kk = dfdr / rc * du;  // r = r_c wherever dfdr is not zero
            const float sg = s == si ? -1.f : 1.f;
            for (int q = 0; q < 3; ++q) gx[q] += sg * (f * u[q] + kk * d[q]);
            if (s != si) continue;
            const DevPotGrad &pg = a.pot_grad[B.pot];
            for (int q = 0; q < pg.n; ++q) {
                if (pg.mode[q] != kGradTable) continue;
                const float *cd = a.dcoef + pg.coef_off[q] + ind * kChunk;
                float Pq, dPq, ddPq;
                poly3(cd, x, Pq, dPq, ddPq);
                g[pg.slot[q]] += (double)(-(dPq * c[1] / rc) * du);
            }
        }
        const float4 o = a.gx[s];
        a.gx[s] = make_float4(o.x + gx[0], o.y + gx[1], o.z + gx[2], 0.f);
    }
    __syncthreads();
    if ((int)threadIdx.x < a.nslots) {
        double t = 0.0;
        for (int r = 0; r < (int)blockDim.x; ++r) t += gsum[r * kGradPad + threadIdx.x];
        a.bond_partials[(size_t)blockIdx.x * kMaxGradSlots + threadIdx.x] = t;
    }
}

/* Per slot: the adjoints back into id order. */
__global__ void adj_finish_kernel(EngineView v, AdjointView a) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= v.nparts) return;
    const int id = __float_as_int(v.vel[s].w);
    float4 gx = a.gx[s], gv = a.gv[s];
    for (int p = 0; p + 1 < kVjpParts; ++p) {  // the later parts' sums, in part order
        const float4 px = a.pgx[(size_t)p * v.nparts + s], pv = a.pgv[(size_t)p * v.nparts + s];
        gx = make_float4(gx.x + px.x, gx.y + px.y, gx.z + px.z, 0.f);
        gv = make_float4(gv.x + pv.x, gv.y + pv.y, gv.z + pv.z, 0.f);
    }
    a.lam_x[id] = gx;
    a.lam_v[id] = gv;
}

/* grad[k] += the step's parameter-gradient partials of slot k: one block per slot, each thread
 * summing a fixed stride of the pair items' partials (contiguous per slot, so a warp's loads
 * are coalesced) and of the bond blocks' partials, then a fixed tree over the threads (the same
 * order on every run). */
constexpr int kGradThreads = 1024;
__global__ void __launch_bounds__(kGradThreads) adj_grad_kernel(AdjointView a, int nitems, int nbond_blocks,
                                                              double *grad) {
    __shared__ double part[kGradThreads];
    const int k = blockIdx.x;
    const double *pk = a.partials + (size_t)k * nitems;
    double t0 = 0.0, t1 = 0.0;  // two independent chains, added at the end
    int q = threadIdx.x;
    for (; q + (int)blockDim.x < nitems; q += 2 * blockDim.x) {
        t0 += pk[q];
        t1 += pk[q + blockDim.x];
    }
    if (q < nitems) t0 += pk[q];
    double t = t0 + t1;
    for (int r = threadIdx.x; r < nbond_blocks; r += blockDim.x) t += a.bond_partials[(size_t)r * kMaxGradSlots + k];
    part[threadIdx.x] = t;
    __syncthreads();
    for (int h = blockDim.x >> 1; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) part[threadIdx.x] += part[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) grad[k] += part[0];
}

/* Absolute positions (x, y, z, type bits) and velocities (v, id bits) by id;
 * the position is the cell origin (double, space.cpp:431-451) plus the
 * cell-relative coordinate. */
__global__ void positions_kernel(EngineView v, float4 *x_out, float4 *v_out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= v.nparts) return;
    const float4 q = v.pos[s], u = v.vel[s];
    const int id = __float_as_int(u.w);
    const int c = v.cell_of[s];
    const DevSpace &S = v.spaces[v.cell_rep[c]];
    const int l = c - S.cell_offset;
    const int loc[3] = {l / (S.cdim[1] * S.cdim[2]), (l / S.cdim[2]) % S.cdim[1], l % S.cdim[2]};
    const float xr[3] = {q.x, q.y, q.z};
    float xa[3];
    for (int k = 0; k < 3; ++k) xa[k] = (float)(S.origin[k] + loc[k] * S.hd[k] + (double)xr[k]);
    if (x_out) x_out[id] = make_float4(xa[0], xa[1], xa[2], q.w);
    if (v_out) v_out[id] = u;
}

/* Gaussian kernel of width sigma at distance t from a bin centre, lowered by
 * its value at 4 sigma so that the cut there is continuous (the loss then has
 * no jumps as pair distances cross a cut). */
__device__ __forceinline__ double rdf_kernel_value(double t, double sigma) {
    return (exp(-0.5 * (t / sigma) * (t / sigma)) - 3.3546262790251185e-04) * (0.3989422804014327 / sigma);
}

constexpr int kRdfTile = 256;
constexpr int kRdfMaxBins = 256;
constexpr double kRdfFixed = 4294967296.0;  // histogram fixed point: 2^32 per unit

/* An FP32 minimum-image distance test that rejects the pairs far beyond the histogram's reach
 * before the exact FP64 distance: its error (a few units in the last place of the box length)
 * is far below kRdfMargin, so every pair the FP64 test keeps passes it, and the same pairs
 * contribute, in the same order, as without it. */
constexpr float kRdfMargin = 1e-2f;
__device__ __forceinline__ bool rdf_may_reach(const float4 &a, const float4 &b, const float *L, const float *iL,
                                              float r2max) {
    float dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
    dx -= L[0] * rintf(dx * iL[0]);
    dy -= L[1] * rintf(dy * iL[1]);
    dz -= L[2] * rintf(dz * iL[2]);
    return dx * dx + dy * dy + dz * dz < r2max;
}

/* The pairs that pass the FP32 test are queued per warp (lane << 8 | tile index, in tile
 * order, then lane order) and evaluated in FP64 32 at a time, one pair per lane, so that the
 * expensive terms run on full warps instead of on the one lane of a warp that found a partner.
 * A warp's queue is drained before the block loads its next tile of partners. */
constexpr int kRdfWarps = kRdfTile / 32;
constexpr int kRdfQueue = 64;  // ring: fewer than 32 waiting plus at most 32 from one partner

/* hist[b] += sum over (i of type ta, j of type tb, i != j) of K(r_ij - c_b),
 * c_b = (b + 1/2) dr, minimum image in the periodic box, terms with
 * |r - c_b| > 4 sigma left out. Fixed-point sums make the result independent
 * of the order of the additions. One lane per particle i. */
__global__ void __launch_bounds__(kRdfTile) rdf_hist_kernel(const float4 *__restrict__ x, int n, double3 box, int ta,
                                                          int tb, int nbins, double dr, double sigma, int chunk,
                                                          unsigned long long *hist) {
    __shared__ float4 tile[kRdfTile];
    __shared__ unsigned long long h[kRdfMaxBins];
    __shared__ unsigned short queue[kRdfWarps][kRdfQueue];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt_mask = (1u << lane) - 1u;
    for (int b = threadIdx.x; b < nbins; b += blockDim.x) h[b] = 0ull;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float4 xi = make_float4(0.f, 0.f, 0.f, 0.f);
    bool active = false;
    if (i < n) {
        xi = x[i];
        active = __float_as_int(xi.w) == ta;
    }
    const double rmax = nbins * dr + 4 * sigma;
    const float Lf[3] = {(float)box.x, (float)box.y, (float)box.z};
    const float iLf[3] = {1.0f / Lf[0], 1.0f / Lf[1], 1.0f / Lf[2]};
    const float r2f = (float)((rmax + kRdfMargin) * (rmax + kRdfMargin));
    const double L[3] = {box.x, box.y, box.z};
    // the FP64 terms of nb <= 32 queued pairs from qh, one per lane
    auto batch = [&](int qh, int nb) {
        const int cd = lane < nb ? queue[w][(qh + lane) & (kRdfQueue - 1)] : 0;
        const int src = cd >> 8;
        const float ax = __shfl_sync(kFull, xi.x, src), ay = __shfl_sync(kFull, xi.y, src),
                    az = __shfl_sync(kFull, xi.z, src);
        if (lane < nb) {
            const float4 xj = tile[cd & 0xff];
            double d[3] = {(double)ax - xj.x, (double)ay - xj.y, (double)az - xj.z};
            for (int q = 0; q < 3; ++q) d[q] -= L[q] * rint(d[q] / L[q]);
            const double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            if (r < rmax) {
                const int b0 = max(0, (int)floor((r - 4 * sigma) / dr)),
                          b1 = min(nbins - 1, (int)floor((r + 4 * sigma) / dr));
                for (int b = b0; b <= b1; ++b) {
                    const double t = r - (b + 0.5) * dr;
                    if (fabs(t) > 4 * sigma) continue;
                    atomicAdd(&h[b], (unsigned long long)llrint(rdf_kernel_value(t, sigma) * kRdfFixed));
                }
            }
        }
        __syncwarp();
    };
    __syncthreads();
    int qh = 0, qt = 0;
    // this block's partners: the tiles of its chunk of the particle range (blockIdx.y)
    const int jend = min(n, (blockIdx.y + 1) * chunk);
    for (int t0 = blockIdx.y * chunk; t0 < jend; t0 += kRdfTile) {
        const int j = t0 + threadIdx.x;
        tile[threadIdx.x] = j < jend ? x[j] : make_float4(0.f, 0.f, 0.f, __int_as_float(-1));
        __syncthreads();
        const int m = min(kRdfTile, jend - t0);
        for (int k = 0; k < m; ++k) {
            const float4 xj = tile[k];
            if (__float_as_int(xj.w) != tb) continue;
            const bool hit = active && t0 + k != i && rdf_may_reach(xi, xj, Lf, iLf, r2f);
            const unsigned bal = __ballot_sync(kFull, hit);
            if (hit) queue[w][(qt + __popc(bal & lt_mask)) & (kRdfQueue - 1)] = (unsigned short)((lane << 8) | k);
            qt += __popc(bal);
            if (qt - qh >= 32) {
                __syncwarp();
                batch(qh, 32);
                qh += 32;
            }
        }
        if (qt > qh) {  // the queue refers to this tile: drain it before the next one
            __syncwarp();
            batch(qh, qt - qh);
            qh = qt;
        }
        __syncthreads();
    }
    for (int b = threadIdx.x; b < nbins; b += blockDim.x)
        if (h[b]) atomicAdd(&hist[b], h[b]);
}

/* grad[i] = sum over partners j of sum_b coef[b] dK(r_ij - c_b)/dr (x_i - x_j)/r
 * for i of type ta (partners tb) and of type tb (partners ta): d loss / d x_i
 * for loss = sum_b G_b(hist) with coef[b] = dG/dhist_b. One lane per particle i; a pair's
 * term is computed by whichever lane holds it in the batch and added by the lane of its i, in
 * queue order, so each i sums its partners in ascending j. */
__global__ void __launch_bounds__(kRdfTile) rdf_grad_kernel(const float4 *__restrict__ x, int n, double3 box, int ta,
                                                          int tb, int nbins, double dr, double sigma, int chunk,
                                                          const double *__restrict__ coef, double *gpart) {
    __shared__ float4 tile[kRdfTile];
    __shared__ unsigned short queue[kRdfWarps][kRdfQueue];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt_mask = (1u << lane) - 1u;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float4 xi = make_float4(0.f, 0.f, 0.f, 0.f);
    int partner = -2;
    if (i < n) {
        xi = x[i];
        const int ti = __float_as_int(xi.w);
        partner = ti == ta ? tb : (ti == tb ? ta : -2);
    }
    const double rmax = nbins * dr + 4 * sigma;
    const float Lf[3] = {(float)box.x, (float)box.y, (float)box.z};
    const float iLf[3] = {1.0f / Lf[0], 1.0f / Lf[1], 1.0f / Lf[2]};
    const float r2f = (float)((rmax + kRdfMargin) * (rmax + kRdfMargin));
    const double L[3] = {box.x, box.y, box.z};
    double g[3] = {0.0, 0.0, 0.0};
    auto batch = [&](int qh, int nb) {
        const int cd = lane < nb ? queue[w][(qh + lane) & (kRdfQueue - 1)] : 0;
        const int src = cd >> 8;
        const float ax = __shfl_sync(kFull, xi.x, src), ay = __shfl_sync(kFull, xi.y, src),
                    az = __shfl_sync(kFull, xi.z, src);
        double c[3] = {0.0, 0.0, 0.0};
        if (lane < nb) {
            const float4 xj = tile[cd & 0xff];
            double d[3] = {(double)ax - xj.x, (double)ay - xj.y, (double)az - xj.z};
            for (int q = 0; q < 3; ++q) d[q] -= L[q] * rint(d[q] / L[q]);
            const double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            if (r < rmax && r > 0.0) {
                const int b0 = max(0, (int)floor((r - 4 * sigma) / dr)),
                          b1 = min(nbins - 1, (int)floor((r + 4 * sigma) / dr));
                double s = 0.0;
                for (int b = b0; b <= b1; ++b) {
                    const double t = r - (b + 0.5) * dr;
                    if (fabs(t) > 4 * sigma) continue;
                    s += coef[b] * exp(-0.5 * (t / sigma) * (t / sigma)) * (0.3989422804014327 / sigma) *
                         (-t / (sigma * sigma));
                }
                // ta == tb counts each unordered pair twice in hist, as i and as j
                const double f = s / r * (ta == tb ? 2.0 : 1.0);
                for (int q = 0; q < 3; ++q) c[q] = f * d[q];
            }
        }
        // each pair's term to the lane of its i, in queue order
        for (int q = 0; q < nb; ++q) {
            const int owner = __shfl_sync(kFull, src, q);
            const double c0 = __shfl_sync(kFull, c[0], q), c1 = __shfl_sync(kFull, c[1], q),
                         c2 = __shfl_sync(kFull, c[2], q);
            if (lane == owner) {
                g[0] += c0;
                g[1] += c1;
                g[2] += c2;
            }
        }
        __syncwarp();
    };
    int qh = 0, qt = 0;
    // this block's partners: the tiles of its chunk of the particle range (blockIdx.y)
    const int jend = min(n, (blockIdx.y + 1) * chunk);
    for (int t0 = blockIdx.y * chunk; t0 < jend; t0 += kRdfTile) {
        const int j = t0 + threadIdx.x;
        tile[threadIdx.x] = j < jend ? x[j] : make_float4(0.f, 0.f, 0.f, __int_as_float(-1));
        __syncthreads();
        const int m = min(kRdfTile, jend - t0);
        for (int k = 0; k < m; ++k) {
            const float4 xj = tile[k];
            const int tj = __float_as_int(xj.w);
            if (tj != ta && tj != tb) continue;
            const bool hit = tj == partner && t0 + k != i && rdf_may_reach(xi, xj, Lf, iLf, r2f);
            const unsigned bal = __ballot_sync(kFull, hit);
            if (hit) queue[w][(qt + __popc(bal & lt_mask)) & (kRdfQueue - 1)] = (unsigned short)((lane << 8) | k);
            qt += __popc(bal);
            if (qt - qh >= 32) {
                __syncwarp();
                batch(qh, 32);
                qh += 32;
            }
        }
        if (qt > qh) {
            __syncwarp();
            batch(qh, qt - qh);
            qh = qt;
        }
        __syncthreads();
    }
    if (i < n)
        for (int q = 0; q < 3; ++q) gpart[((size_t)blockIdx.y * n + i) * 3 + q] = g[q];
}

/* grad[i]: particle i's sums over the partner chunks, added in chunk order (so in ascending
 * partner index, chunk by chunk). */
__global__ void rdf_grad_sum_kernel(const double *__restrict__ gpart, int n, int nchunks, float4 *grad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double g[3] = {0.0, 0.0, 0.0};
    for (int c = 0; c < nchunks; ++c)
        for (int q = 0; q < 3; ++q) g[q] += gpart[((size_t)c * n + i) * 3 + q];
    grad[i] = make_float4((float)g[0], (float)g[1], (float)g[2], 0.f);
}

}  // namespace

void launch_positions(const EngineView &v, float4 *x_out, float4 *v_out, cudaStream_t st) {
    positions_kernel<<<(v.nparts + 255) / 256, 256, 0, st>>>(v, x_out, v_out);
}

int launch_rdf(const float4 *x, int n, const double *box, int ta, int tb, int nbins, double dr, double sigma,
               unsigned long long *hist, const double *coef, float4 *grad, cudaStream_t st) {
    if (nbins < 1 || nbins > kRdfMaxBins) return -1;
    const double3 b = make_double3(box[0], box[1], box[2]);
    const int grid = (n + kRdfTile - 1) / kRdfTile;
    // the partner range split into chunks of whole tiles, one block per (particle tile, chunk),
    // so that a few hundred blocks (not one per SM) hide the candidate test's latency
    int sms = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int ntiles = grid;
    const int nchunks = std::max(1, std::min(ntiles, (6 * sms + grid - 1) / grid));
    const int chunk = ((ntiles + nchunks - 1) / nchunks) * kRdfTile;
    const int nch = (n + chunk - 1) / chunk;
    const dim3 g2(grid, nch);
    if (hist) rdf_hist_kernel<<<g2, kRdfTile, 0, st>>>(x, n, b, ta, tb, nbins, dr, sigma, chunk, hist);
    if (grad) {
        double *gpart = nullptr;
        if (cudaMallocAsync(reinterpret_cast<void **>(&gpart), sizeof(double) * 3 * (size_t)n * nch, st) != cudaSuccess)
            return -2;
        rdf_grad_kernel<<<g2, kRdfTile, 0, st>>>(x, n, b, ta, tb, nbins, dr, sigma, chunk, coef, gpart);
        rdf_grad_sum_kernel<<<(n + 255) / 256, 256, 0, st>>>(gpart, n, nch, grad);
        cudaFreeAsync(gpart, st);
    }
    return 0;
}

/* One thread per word over all sections in order (a section's words are consecutive). */
__global__ void copy_sections_kernel(CopySections c, unsigned long long total) {
    for (unsigned long long t = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; t < total;
         t += (unsigned long long)gridDim.x * blockDim.x) {
        unsigned long long r = t;
        int k = 0;
        while (k < c.n - 1 && r >= c.words[k]) r -= c.words[k++];
        c.dst[k][r] = c.src[k][r];
    }
}

void launch_copy_sections(const CopySections &c, cudaStream_t st) {
    unsigned long long total = 0;
    for (int k = 0; k < c.n; ++k) total += c.words[k];
    if (total == 0) return;
    const int tb = 256;
    const unsigned long long blocks = std::min<unsigned long long>((total + tb - 1) / tb, 148ull * 16);
    copy_sections_kernel<<<(unsigned)blocks, tb, 0, st>>>(c, total);
}

int adjoint_grid(int num_sms) { return num_sms * 4; }
int vjp_parts() { return kVjpParts; }
int adjoint_bond_blocks(int num_sms) { return num_sms * 2; }

void configure_adjoint_kernels() {
    cudaFuncSetAttribute(vjp_pair_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)adj_smem_bytes());
    cudaFuncSetAttribute(vjp_pair_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                         cudaSharedmemCarveoutMaxShared);
}

void launch_vjp_step(const EngineView &v, const AdjointView &a, const BondedView *bv, int num_sms, double *grad,
                     cudaStream_t st) {
    const int tb = 256;
    adj_prep_kernel<<<(v.nparts + tb - 1) / tb, tb, 0, st>>>(v, a);
    const int grid = adjoint_grid(num_sms);
    vjp_pair_kernel<<<grid, kWarpsA * 32, adj_smem_bytes(), st>>>(v, a);
    const int bblocks = bv ? adjoint_bond_blocks(num_sms) : 0;
    if (bv) vjp_bond_kernel<<<bblocks, kBondVjpThreads, 0, st>>>(v, *bv, a);
    adj_finish_kernel<<<(v.nparts + tb - 1) / tb, tb, 0, st>>>(v, a);
    if (a.nslots > 0) adj_grad_kernel<<<a.nslots, kGradThreads, 0, st>>>(a, a.nitems, bblocks, grad);
}

}  // namespace mxg
