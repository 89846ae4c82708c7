/*
 * Pair search for the pairwise bond constructor (bind_pairwise).
 *
 * The reference's make_pairlist (src/mdcore/src/bond.cpp:892-942) visits every
 * pair (a, b), b < a, of a particle list in a double loop on the host and keeps
 * those with |x_a - x_b|^2 <= cutoff^2 (global positions rounded to float, no
 * periodic image, the squared distance summed x, y, z in FP32) whose type pair
 * passes pair_check (bond.cpp:1134-1152). The order of the result is a
 * ascending, then b ascending.
 *
 * Here the same test runs on the device over a uniform grid of cell size
 * slightly above the cutoff: each list entry visits the 27 grid cells around
 * its own, counts its partners b < a, and after an exclusive scan writes them
 * into its own segment, which it then sorts by b. Every pair the double loop
 * accepts has its two grid cells adjacent, so the result, and its order, is
 * the reference's.
 */
#include "mxg_kernels.h"

namespace mxg {

namespace {

struct PairGrid {
    double lo[3];
    double inv;      // 1 / grid cell size
    int g[3];        // grid cells per axis
    float c2;        // cutoff * cutoff in FP32
    int ntypes;      // type-pair mask dimension (0: no mask)
};

__device__ __forceinline__ int grid_axis(double x, double lo, double inv, int g) {
    int q = (int)floor((x - lo) * inv);
    return q < 0 ? 0 : (q >= g ? g - 1 : q);
}

/* Global FP32 position (x_rel + cell origin, formed in double and rounded)
 * and grid cell of each list entry; -1 for ids without a particle or outside
 * the first entry's replica. */
__global__ void pair_gather_kernel(EngineView v, const int *__restrict__ ids, int n, const int *__restrict__ slot_of_id,
                                   int nids, PairGrid G, float4 *gpos, int *gcell, int *gcount) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n) return;
    const int id = ids[a];
    const int s = (id >= 0 && id < nids) ? slot_of_id[id] : -1;
    const int s0 = (ids[0] >= 0 && ids[0] < nids) ? slot_of_id[ids[0]] : -1;
    if (s < 0 || s0 < 0 || v.cell_rep[v.cell_of[s]] != v.cell_rep[v.cell_of[s0]]) {
        gcell[a] = -1;
        return;
    }
    const int c = v.cell_of[s];
    const DevSpace &S = v.spaces[v.cell_rep[c]];
    const int l = c - S.cell_offset;
    const int loc[3] = {l / (S.cdim[1] * S.cdim[2]), (l / S.cdim[2]) % S.cdim[1], l % S.cdim[2]};
    const float4 p = v.pos[s];
    const float xr[3] = {p.x, p.y, p.z};
    float g[3];
    for (int k = 0; k < 3; ++k) {
        const double o = __dadd_rn(S.origin[k], __dmul_rn((double)loc[k], S.hd[k]));
        g[k] = (float)__dadd_rn((double)xr[k], o);
    }
    gpos[a] = make_float4(g[0], g[1], g[2], p.w);
    const int cell = (grid_axis(g[0], G.lo[0], G.inv, G.g[0]) * G.g[1] + grid_axis(g[1], G.lo[1], G.inv, G.g[1])) *
                         G.g[2] +
                     grid_axis(g[2], G.lo[2], G.inv, G.g[2]);
    gcell[a] = cell;
    atomicAdd(&gcount[cell], 1);
}

__global__ void pair_bin_kernel(const int *__restrict__ gcell, int n, const int *__restrict__ gstart, int *gfill,
                                int *members) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n || gcell[a] < 0) return;
    members[gstart[gcell[a]] + atomicAdd(&gfill[gcell[a]], 1)] = a;
}

/* Counts (out == nullptr) or writes and sorts the partners b < a of entry a. */
__global__ void pair_search_kernel(const float4 *__restrict__ gpos, const int *__restrict__ gcell, int n, PairGrid G,
                                   const int *__restrict__ gstart, const int *__restrict__ members,
                                   const unsigned char *__restrict__ mask, int *count, const int *__restrict__ off,
                                   int *out) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n || gcell[a] < 0) {
        if (a < n && !out) count[a] = 0;
        return;
    }
    const float4 pa = gpos[a];
    const int ta = __float_as_int(pa.w);
    const int ca = gcell[a];
    const int cz = ca % G.g[2], cy = (ca / G.g[2]) % G.g[1], cx = ca / (G.g[1] * G.g[2]);
    int k = 0;
    const int base = out ? off[a] : 0;
    for (int dx = -1; dx <= 1; ++dx) {
        const int x = cx + dx;
        if (x < 0 || x >= G.g[0]) continue;
        for (int dy = -1; dy <= 1; ++dy) {
            const int y = cy + dy;
            if (y < 0 || y >= G.g[1]) continue;
            for (int dz = -1; dz <= 1; ++dz) {
                const int z = cz + dz;
                if (z < 0 || z >= G.g[2]) continue;
                const int c = (x * G.g[1] + y) * G.g[2] + z;
                for (int q = gstart[c]; q < gstart[c + 1]; ++q) {
                    const int b = members[q];
                    if (b >= a) continue;
                    const float4 pb = gpos[b];
                    const float d0 = __fsub_rn(pa.x, pb.x), d1 = __fsub_rn(pa.y, pb.y), d2 = __fsub_rn(pa.z, pb.z);
                    const float r2 = dot3_rn(d0, d1, d2);
                    if (!(r2 <= G.c2)) continue;
                    if (G.ntypes && !mask[ta * G.ntypes + __float_as_int(pb.w)]) continue;
                    if (out) out[base + k] = b;
                    ++k;
                }
            }
        }
    }
    if (!out) {
        count[a] = k;
        return;
    }
    for (int i = 1; i < k; ++i) {  // partners in ascending list order
        const int key = out[base + i];
        int j = i - 1;
        while (j >= 0 && out[base + j] > key) {
            out[base + j + 1] = out[base + j];
            --j;
        }
        out[base + j + 1] = key;
    }
}

/* Exclusive scan of n ints into out[0..n] (out[n] = total), one block. */
__global__ void exclusive_scan_kernel(const int *__restrict__ in, int n, int *out) {
    __shared__ int warp_sums[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int base = 0; base < n; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const int x = i < n ? in[i] : 0;
        int s = x;
        for (int d = 1; d < 32; d <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, s, d);
            if (lane >= d) s += t;
        }
        if (lane == 31) warp_sums[warp] = s;
        __syncthreads();
        if (warp == 0) {
            const int nw = blockDim.x >> 5;
            int w = lane < nw ? warp_sums[lane] : 0;
            for (int d = 1; d < 32; d <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, w, d);
                if (lane >= d) w += t;
            }
            if (lane < nw) warp_sums[lane] = w;
        }
        __syncthreads();
        const int excl = carry + (warp ? warp_sums[warp - 1] : 0) + s - x;
        if (i < n) out[i] = excl;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = excl + x;
        __syncthreads();
    }
    if (threadIdx.x == 0) out[n] = carry;
}

template <typename T>
int dev_buf(T **p, size_t n) {
    return cudaMalloc((void **)p, sizeof(T) * (n ? n : 1)) == cudaSuccess ? 0 : -1;
}

}  // namespace

int find_pairs_within(const EngineView &v, const int *slot_of_id, int nids, const double lo[3], const double hi[3],
                      int n, const int *ids_host, float cutoff, const unsigned char *mask_host, int ntypes,
                      std::vector<int> &first, std::vector<int> &second, cudaStream_t st) {
    first.clear();
    second.clear();
    if (n < 2) return 0;
    PairGrid G;
    G.c2 = cutoff * cutoff;
    G.ntypes = mask_host ? ntypes : 0;
    // grid cells a little wider than the cutoff, at most 2^22 of them
    double size = (double)cutoff * 1.001 + 1e-12;
    for (;;) {
        long long total = 1;
        for (int k = 0; k < 3; ++k) {
            G.lo[k] = lo[k];
            G.g[k] = std::max(1, (int)std::ceil((hi[k] - lo[k]) / size));
            total *= G.g[k];
        }
        if (total <= (1LL << 22)) break;
        size *= 1.5;
    }
    G.inv = 1.0 / size;
    const int ncell = G.g[0] * G.g[1] * G.g[2];
    int *d_ids = nullptr, *d_gcell = nullptr, *d_gcount = nullptr, *d_gstart = nullptr, *d_gfill = nullptr;
    int *d_members = nullptr, *d_count = nullptr, *d_off = nullptr, *d_out = nullptr;
    float4 *d_gpos = nullptr;
    unsigned char *d_mask = nullptr;
    int rc = 0;
    auto fail = [&](int code) {
        cudaFree(d_ids); cudaFree(d_gcell); cudaFree(d_gcount); cudaFree(d_gstart); cudaFree(d_gfill);
        cudaFree(d_members); cudaFree(d_count); cudaFree(d_off); cudaFree(d_out); cudaFree(d_gpos); cudaFree(d_mask);
        return code;
    };
    rc |= dev_buf(&d_ids, n);
    rc |= dev_buf(&d_gcell, n);
    rc |= dev_buf(&d_gpos, n);
    rc |= dev_buf(&d_gcount, ncell);
    rc |= dev_buf(&d_gstart, ncell + 1);
    rc |= dev_buf(&d_gfill, ncell);
    rc |= dev_buf(&d_members, n);
    rc |= dev_buf(&d_count, n);
    rc |= dev_buf(&d_off, n + 1);
    if (G.ntypes) rc |= dev_buf(&d_mask, (size_t)ntypes * ntypes);
    if (rc) return fail(-2);
    if (cudaMemcpyAsync(d_ids, ids_host, sizeof(int) * n, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        (G.ntypes && cudaMemcpyAsync(d_mask, mask_host, (size_t)ntypes * ntypes, cudaMemcpyHostToDevice, st) !=
                         cudaSuccess) ||
        cudaMemsetAsync(d_gcount, 0, sizeof(int) * ncell, st) != cudaSuccess ||
        cudaMemsetAsync(d_gfill, 0, sizeof(int) * ncell, st) != cudaSuccess)
        return fail(-21);
    const int tb = 256, nb = (n + tb - 1) / tb;
    pair_gather_kernel<<<nb, tb, 0, st>>>(v, d_ids, n, slot_of_id, nids, G, d_gpos, d_gcell, d_gcount);
    exclusive_scan_kernel<<<1, 1024, 0, st>>>(d_gcount, ncell, d_gstart);
    pair_bin_kernel<<<nb, tb, 0, st>>>(d_gcell, n, d_gstart, d_gfill, d_members);
    pair_search_kernel<<<nb, tb, 0, st>>>(d_gpos, d_gcell, n, G, d_gstart, d_members, d_mask, d_count, nullptr,
                                          nullptr);
    exclusive_scan_kernel<<<1, 1024, 0, st>>>(d_count, n, d_off);
    int total = 0;
    if (cudaMemcpyAsync(&total, d_off + n, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return fail(-21);
    std::vector<int> off(n + 1), out(total);
    if (total > 0) {
        if (dev_buf(&d_out, total)) return fail(-2);
        pair_search_kernel<<<nb, tb, 0, st>>>(d_gpos, d_gcell, n, G, d_gstart, d_members, d_mask, d_count, d_off,
                                              d_out);
        if (cudaMemcpyAsync(out.data(), d_out, sizeof(int) * total, cudaMemcpyDeviceToHost, st) != cudaSuccess)
            return fail(-21);
    }
    if (cudaMemcpyAsync(off.data(), d_off, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return fail(-21);
    first.resize(total);
    second.resize(total);
    for (int a = 0; a < n; ++a)
        for (int q = off[a]; q < off[a + 1]; ++q) {
            first[q] = ids_host[a];
            second[q] = ids_host[out[q]];
        }
    return fail(0);
}

}  // namespace mxg
