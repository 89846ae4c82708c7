/*
 * Particle-group metrics (MxParticleList / MxCluster methods, src/mdcore/src/
 * MxParticleList.cpp:406-458): centre of mass, centre of geometry (centroid),
 * radius of gyration and moment of inertia of a list of particle ids, from the
 * particles' global positions x_rel + cell origin (formed in double, as the
 * reference's `p->x[k] + o[k]`).
 *
 * The formulas are the reference's (src/mdcore/src/metrics.cpp):
 *   centre of mass      sum m x / sum m                                (:366-389)
 *   centroid            sum x / n                                      (:391-412)
 *   radius of gyration  sqrt(sum_i |centroid - x_i|), the sum of the
 *                       distances (not of their squares)               (:330-364)
 *   moment of inertia   about the centre of mass: diagonal
 *                       sum m (dy^2 + dz^2) ..., off-diagonal
 *                       + sum m dx dy ... (no minus sign), symmetric   (:414-466)
 * The reference accumulates in FP32 in list order; here each sum is formed in
 * FP64 by one block (per-thread partials, then a fixed shuffle and shared-memory
 * tree), so results are deterministic and at least as accurate.
 */
#include "mxg_kernels.h"

namespace mxg {

namespace {

constexpr int kGroupThreads = 1024;

__device__ __forceinline__ void global_position(const EngineView &v, int s, double g[3]) {
    const int c = v.cell_of[s];
    const DevSpace &S = v.spaces[v.cell_rep[c]];
    const int l = c - S.cell_offset;
    const int loc[3] = {l / (S.cdim[1] * S.cdim[2]), (l / S.cdim[2]) % S.cdim[1], l % S.cdim[2]};
    const float4 p = v.pos[s];
    const float xr[3] = {p.x, p.y, p.z};
    for (int k = 0; k < 3; ++k) g[k] = (double)xr[k] + (S.origin[k] + (double)loc[k] * S.hd[k]);
}

/* Sums q[0..nq) over the block in a fixed order; the result is valid in thread 0. */
template <int nq>
__device__ __forceinline__ void block_sum(double (&q)[nq], double *red) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int k = 0; k < nq; ++k) {
        double t = q[k];
        for (int off = 16; off > 0; off >>= 1) t += __shfl_xor_sync(0xffffffffu, t, off);
        if (lane == 0) red[w * nq + k] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < nq; ++k) {
            double t = 0.0;
            for (int ww = 0; ww < kGroupThreads / 32; ++ww) t += red[ww * nq + k];
            q[k] = t;
        }
    }
    __syncthreads();
}

/* out[0] sum m, out[1..3] centre of mass, out[4..6] centroid, out[7] radius of
 * gyration, out[8..16] moment of inertia (row-major). One block. */
__global__ void __launch_bounds__(kGroupThreads) group_metrics_kernel(EngineView v, const int *__restrict__ ids,
                                                                      int n, const int *__restrict__ slot_of_id,
                                                                      double *out) {
    __shared__ double red[(kGroupThreads / 32) * 7];
    __shared__ double ctr[6];
    double a[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int i = threadIdx.x; i < n; i += kGroupThreads) {
        const int s = slot_of_id[ids[i]];
        double g[3];
        global_position(v, s, g);
        const double m = v.types[__float_as_int(v.pos[s].w)].mass;
        a[0] += m;
        for (int k = 0; k < 3; ++k) {
            a[1 + k] += m * g[k];
            a[4 + k] += g[k];
        }
    }
    block_sum<7>(a, red);
    if (threadIdx.x == 0) {
        out[0] = a[0];
        for (int k = 0; k < 3; ++k) {
            ctr[k] = a[1 + k] / a[0];
            ctr[3 + k] = a[4 + k] / (double)n;
            out[1 + k] = ctr[k];
            out[4 + k] = ctr[3 + k];
        }
    }
    __syncthreads();
    double b[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // sum |d|, I00, I11, I22, I01, I12, I02
    for (int i = threadIdx.x; i < n; i += kGroupThreads) {
        const int s = slot_of_id[ids[i]];
        double g[3];
        global_position(v, s, g);
        const double m = v.types[__float_as_int(v.pos[s].w)].mass;
        const double e0 = ctr[3] - g[0], e1 = ctr[4] - g[1], e2 = ctr[5] - g[2];
        b[0] += sqrt(e0 * e0 + e1 * e1 + e2 * e2);
        const double d0 = g[0] - ctr[0], d1 = g[1] - ctr[1], d2 = g[2] - ctr[2];
        b[1] += (d1 * d1 + d2 * d2) * m;
        b[2] += (d0 * d0 + d2 * d2) * m;
        b[3] += (d1 * d1 + d0 * d0) * m;
        b[4] += d0 * d1 * m;
        b[5] += d1 * d2 * m;
        b[6] += d0 * d2 * m;
    }
    block_sum<7>(b, red);
    if (threadIdx.x == 0) {
        out[7] = sqrt(b[0]);
        double *I = out + 8;
        I[0] = b[1];
        I[4] = b[2];
        I[8] = b[3];
        I[1] = I[3] = b[4];
        I[5] = I[7] = b[5];
        I[2] = I[6] = b[6];
    }
}

}  // namespace

void launch_group_metrics(const EngineView &v, const int *ids, int n, const int *slot_of_id, double *out,
                          cudaStream_t st) {
    group_metrics_kernel<<<1, kGroupThreads, 0, st>>>(v, ids, n, slot_of_id, out);
}

}  // namespace mxg
