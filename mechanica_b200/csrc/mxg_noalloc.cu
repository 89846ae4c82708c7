/*
 * Kinetic-energy reduction that allocates no device memory.
 *
 * Some callers cannot call cudaMalloc: an application whose device memory is
 * owned and reserved by another allocator (a framework's caching allocator or
 * a fixed memory budget), or a latency-critical loop that must not take the
 * implicit device synchronisation an allocation can cause. For them this file
 * offers mxg_kinetic_energy_noalloc: the caller passes the inputs and the
 * output buffer, and the only scratch memory -- the per-block, per-type partial
 * sums of the two-stage reduction -- is a file-scope __device__ array that
 * every GPU loading the library holds until the process exits.
 *
 * Semantics match engine_kinetic_energy (src/mdcore/src/engine.cpp:1698-1719):
 * per particle e = (float)(0.5 * mass * (vx*vx + vy*vy + vz*vz)), summed in
 * FP64, in total and per type. The summation order is fixed (block partials,
 * then the blocks in order), so repeated calls give identical results.
 */
#include "../../include/mxg.h"

#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

namespace {

constexpr int kNoallocTypes = 64;     // maximum particle types per call
constexpr int kNoallocBlocks = 256;   // stage-1 blocks (grid-stride over particles)
constexpr int kNoallocThreads = 256;
constexpr int kMaxDevices = 64;

/* Stage-1 partials: [block][type]. 256 x 64 doubles = 128 KiB per device. Every
 * slot a call reads is written by the same call's stage 1 first, so nothing has
 * to be cleared between calls. Calls that overlap on the GPU (two streams, or
 * two host threads) race on this array: serialise them. */
static __device__ __align__(256) double g_ke_partials[kNoallocBlocks * kNoallocTypes];

/* Device address of g_ke_partials per device, looked up once per device. */
double *g_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mutex;

/* Stage 1: each block walks its share of the particles in chunks of blockDim;
 * for every chunk the per-particle energies go to shared memory and thread t
 * (t < ntypes) adds the chunk's type-t energies in index order. With one type,
 * every thread keeps a running sum over its chunks and the block adds them in a
 * fixed tree at the end (warp shuffles, then the warps in order): no serial scan. */
__global__ void __launch_bounds__(kNoallocThreads)
    ke_partials_kernel(const float4 *__restrict__ vel, const float4 *__restrict__ pos, int n,
                       const double *__restrict__ type_mass, int ntypes, double *partials) {
    __shared__ float se[kNoallocThreads];
    __shared__ int stype[kNoallocThreads];
    __shared__ double swarp[kNoallocThreads / 32];
    double acc = 0.0;  // thread t < ntypes: running sum of type t (one type: this thread's particles)
    const bool one_type = ntypes == 1;
    for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const int s = base + threadIdx.x;
        float e = 0.0f;
        int t = -1;
        if (s < n) {
            t = __float_as_int(pos[s].w);
            if (t < 0 || t >= ntypes) t = -1;  // type ids outside [0, ntypes) contribute nothing
        }
        if (t >= 0) {
            const float4 u = vel[s];
            const float v2 = __fadd_rn(__fadd_rn(__fmul_rn(u.x, u.x), __fmul_rn(u.y, u.y)), __fmul_rn(u.z, u.z));
            e = (float)__dmul_rn(__dmul_rn(0.5, type_mass[t]), (double)v2);
        }
        if (one_type) {
            acc += (double)e;
            continue;
        }
        se[threadIdx.x] = e;
        stype[threadIdx.x] = t;
        __syncthreads();
        if ((int)threadIdx.x < ntypes)
            for (int k = 0; k < (int)blockDim.x; ++k)
                if (stype[k] == (int)threadIdx.x) acc += (double)se[k];
        __syncthreads();
    }
    if (one_type) {
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
        if ((threadIdx.x & 31) == 0) swarp[threadIdx.x >> 5] = acc;
        __syncthreads();
        if (threadIdx.x == 0) {
            double b = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) b += swarp[w];
            partials[blockIdx.x] = b;
        }
        return;
    }
    if ((int)threadIdx.x < ntypes) partials[blockIdx.x * ntypes + threadIdx.x] = acc;
}

__global__ void ke_final_kernel(const double *partials, int nblocks, int ntypes, double *out) {
    // one thread per type sums the blocks in order; thread 0 then sums the types
    __shared__ double per_type[kNoallocTypes];
    for (int t = threadIdx.x; t < ntypes; t += blockDim.x) {
        double s = 0.0;
        for (int b = 0; b < nblocks; ++b) s += partials[b * ntypes + t];
        per_type[t] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double total = 0.0;
        for (int t = 0; t < ntypes; ++t) total += per_type[t];
        out[0] = total;
        for (int t = 0; t < ntypes; ++t) out[1 + t] = per_type[t];
    }
}

/* Looks up the device address of the scratch array for the current device,
 * once per device. Under lazy module loading this first lookup may also load the
 * module (allocating its code and the array), so callers make the first call at
 * set-up. */
int scratch_for_current_device(double **ptr) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return MXG_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        const cudaError_t err = cudaGetSymbolAddress(&p, g_ke_partials);
        if (err != cudaSuccess) {
            fprintf(stderr, "mxg: cudaGetSymbolAddress failed on device %d: %s\n", dev, cudaGetErrorString(err));
            return MXG_ERR_CUDA;
        }
        g_scratch_ptr[dev] = static_cast<double *>(p);
    }
    *ptr = g_scratch_ptr[dev];
    return MXG_OK;
}

}  // namespace

extern "C" int mxg_kinetic_energy_noalloc(const void *vel, const void *pos, int nparts, const double *type_mass,
                                          int ntypes, double *out, void *stream) {
    if (!vel || !pos || !type_mass || !out) return MXG_ERR_NULL;
    if (nparts < 0 || ntypes < 1) return MXG_ERR_ARG;
    if (ntypes > kNoallocTypes) {
        fprintf(stderr, "mxg_kinetic_energy_noalloc: %d particle types exceed the maximum of %d\n", ntypes,
                kNoallocTypes);
        return MXG_ERR_RANGE;
    }
    double *scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc != MXG_OK) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    ke_partials_kernel<<<kNoallocBlocks, kNoallocThreads, 0, st>>>(static_cast<const float4 *>(vel),
                                                                   static_cast<const float4 *>(pos), nparts,
                                                                   type_mass, ntypes, scratch);
    ke_final_kernel<<<1, kNoallocTypes, 0, st>>>(scratch, kNoallocBlocks, ntypes, out);
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) {
        fprintf(stderr, "mxg_kinetic_energy_noalloc: launch failed: %s\n", cudaGetErrorString(err));
        return MXG_ERR_CUDA;
    }
    return MXG_OK;
}
