/*
 * Host side of the engine behind the C ABI in include/mxg.h.
 *
 * Set-up mirrors the reference engine:
 *   - geometry and cells: engine_init (src/mdcore/src/engine.cpp:1502-1560) and
 *     space_init (src/mdcore/src/space.cpp:626-978), including the cell-pair
 *     task list, its pruning and the sort-ID / flip of every pair
 *     (space_getsid, space.cpp:95-130);
 *   - particle placement: space_addpart (space.cpp:397-477) followed by the
 *     relocation rule of space_shuffle_local (space.cpp:333-393) that the first
 *     engine_force applies;
 *   - integrator constants: engine_advance_forward_euler (engine_advance.cpp:270-280).
 * The task list is turned into per-cell neighbour entries carrying the pair's
 * float shift and the role of the cell in the (flipped) pair, so the device
 * force kernel reproduces each pair's arithmetic exactly.
 *
 * Device state is allocated once at mxg_engine_start and stays resident; a step
 * is five kernels (force, bonds, integrate, scan, scatter) replayed from CUDA
 * graphs, one per buffer parity.
 */
#include "../../include/mxg.h"
#include "mxg_adjoint.h"
#include "mxg_kernels.h"
#include "potential_table.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <numeric>
#include <vector>

struct mxg_potential {
    mxg::PotentialTable t;
};

namespace {

using namespace mxg;

/* sort-ID tables of space_cell.cpp:54-99 (27 shift directions -> 13 sort lists) */
const int kSortlistID[27] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 0, 12, 11, 10, 9, 8, 7, 6, 5, 4, 3, 2, 1, 0};
const bool kCellFlip[27] = {1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};

enum : int { kTaskSelf = 1, kTaskPair = 2, kTaskSort = 3 };  // task.h:31-37

/* normalised shift vector of each of the 13 sort lists (space_cell.cpp:82-96) */
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

struct Task {
    int type, flags, i, j;
};

enum : unsigned {
    kPeriodicX = 1u << 0,
    kPeriodicY = 1u << 1,
    kPeriodicZ = 1u << 2,
};

struct TypeInfo {
    double mass, imass, radius;
    int dynamics;
    unsigned flags;
    float force[3];
    bool has_force;
    int sb_kind = 0;            // 2 Berendsen, 3 random, 4 friction (the type's one single-body force)
    float sb[4] = {0, 0, 0, 0};  // Berendsen: tau; random: mean, std, duration; friction: coef, mean, std, duration
    double target = 0.0;        // target temperature (Berendsen)
    int bpot[6] = {-1, -1, -1, -1, -1, -1};  // wall potential per face (index into pots), -1 if none
    int cpot = -1;                           // potential with the cuboids (index into pots), -1 if none
};

/* A static cuboid: centre, size, orientation qx qy qz from the three angles, its
 * inverse and its axis-aligned bounding box, in the reference's float arithmetic
 * (cuboid_init and MxCuboid_UpdateAABB, MxCuboid.cpp:40-76 and 190-221). */
struct CuboidInfo {
    int rep;
    float pos[3], size[3], q[4], qi[4], lo[3], hi[3];
};

/* quaternion product (x, y, z, w) as the vector form forms it: b.v a.w + a.v b.w + a.v x b.v,
 * a.w b.w - a.v . b.v */
void quat_mul_host(const float *a, const float *b, float *o) {
    const float cx = a[1] * b[2] - a[2] * b[1], cy = a[2] * b[0] - a[0] * b[2], cz = a[0] * b[1] - a[1] * b[0];
    float r[4];
    r[0] = (b[0] * a[3] + a[0] * b[3]) + cx;
    r[1] = (b[1] * a[3] + a[1] * b[3]) + cy;
    r[2] = (b[2] * a[3] + a[2] * b[3]) + cz;
    r[3] = a[3] * b[3] - ((a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]);
    for (int k = 0; k < 4; ++k) o[k] = r[k];
}

void quat_rotate_host(const float *q, const float *v, float *out) {
    const float p[4] = {v[0], v[1], v[2], 0.f}, qc[4] = {-q[0], -q[1], -q[2], q[3]};
    float t[4], r[4];
    quat_mul_host(q, p, t);
    quat_mul_host(t, qc, r);
    for (int k = 0; k < 3; ++k) out[k] = r[k];
}

CuboidInfo make_cuboid(int rep, const float *pos, const float *size, const float *angles) {
    CuboidInfo c;
    c.rep = rep;
    for (int k = 0; k < 3; ++k) {
        c.pos[k] = pos[k];
        c.size[k] = size[k];
    }
    // Quaternion::rotation(angle, axis) = (axis sin(angle / 2), cos(angle / 2)); orientation = qx qy qz
    float qa[3][4];
    for (int k = 0; k < 3; ++k) {
        const float half = angles[k] / 2;
        for (int q = 0; q < 3; ++q) qa[k][q] = q == k ? std::sin(half) : 0.f * std::sin(half);
        qa[k][3] = std::cos(half);
    }
    float qxy[4];
    quat_mul_host(qa[0], qa[1], qxy);
    quat_mul_host(qxy, qa[2], c.q);
    // inverted() = conjugated() / dot()
    const float dot = ((c.q[0] * c.q[0] + c.q[1] * c.q[1]) + c.q[2] * c.q[2]) + c.q[3] * c.q[3];
    for (int q = 0; q < 3; ++q) c.qi[q] = -c.q[q] / dot;
    c.qi[3] = c.q[3] / dot;
    // bounding box of the eight rotated corners; the upper bound starts at the smallest positive
    // float, as the reference initialises it
    float half[3];
    for (int k = 0; k < 3; ++k) {
        half[k] = 0.5f * size[k];
        c.lo[k] = std::numeric_limits<float>::max();
        c.hi[k] = std::numeric_limits<float>::min();
    }
    const float sgn[8][3] = {{1, 1, 1}, {1, -1, 1}, {-1, -1, 1}, {-1, 1, 1},
                             {1, 1, -1}, {1, -1, -1}, {-1, -1, -1}, {-1, 1, -1}};
    for (int i = 0; i < 8; ++i) {
        const float corner[3] = {sgn[i][0] * half[0], sgn[i][1] * half[1], sgn[i][2] * half[2]};
        float r[3];
        quat_rotate_host(c.q, corner, r);
        for (int k = 0; k < 3; ++k) {
            const float pt = r[k] + pos[k];
            c.lo[k] = std::min(c.lo[k], pt);
            c.hi[k] = std::max(c.hi[k], pt);
        }
    }
    return c;
}

struct BondInfo {
    int i, j, pot;
    double dissociation;
};

struct AngleInfo {
    int i, j, k, pot;
};

struct ExclusionInfo {
    int i, j;  // i <= j
    bool operator<(const ExclusionInfo &o) const { return i < o.i || (i == o.i && j < o.j); }
    bool operator==(const ExclusionInfo &o) const { return i == o.i && j == o.j; }
};

struct DihedralInfo {
    int i, j, k, l, pot;
};

#define CUDA_TRY(x)                                                                              \
    do {                                                                                         \
        cudaError_t err_ = (x);                                                                  \
        if (err_ != cudaSuccess) {                                                               \
            fprintf(stderr, "mxg: CUDA error %s at %s:%d\n", cudaGetErrorString(err_), __FILE__, __LINE__); \
            return MXG_ERR_CUDA;                                                                 \
        }                                                                                        \
    } while (0)

template <typename T>
int dev_alloc(T **p, size_t n) {
    *p = nullptr;
    if (n == 0) n = 1;
    if (cudaMalloc((void **)p, n * sizeof(T)) != cudaSuccess) return MXG_ERR_MALLOC;
    return MXG_OK;
}

template <typename T>
int upload(T *dst, const std::vector<T> &src, cudaStream_t st) {
    if (src.empty()) return MXG_OK;
    CUDA_TRY(cudaMemcpyAsync(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, st));
    return MXG_OK;
}

}  // namespace

/* One simulation box (a replica): the reference's space (space.h:136-263) with its
 * cell grid, boundary kinds, cell-pair task list and the global index of its
 * first cell in the engine's concatenated cell array. */
struct Space {
    double origin[3], dim[3];
    int cells[3];
    int bc_kind[6];
    float bc_vel[6][3];
    float bc_restore[6];
    unsigned period = 0;
    int cdim[3];
    double h[3], ih[3];
    int ncells = 0;
    int cell_offset = 0;
    std::vector<unsigned> cell_flags;
    std::vector<double> cell_origin;  // 3 per cell
    std::vector<Task> tasks;          // local cell indices
    std::vector<int> pot_idx;         // max_type^2 potential index per type pair (-1 none)
    std::vector<int> pot2_idx;        // max_type^2 second (summed) potential per type pair (-1 none)

    int cellid(int i, int j, int k) const { return (i * cdim[1] + j) * cdim[2] + k; }

    /* space_getsid (space.cpp:95-130): min-image shift between cell origins,
     * sort ID, and the flip of (ci, cj). shift is single precision. */
    int getsid(int &ci, int &cj, float *shift) const {
        for (int k = 0; k < 3; ++k) {
            shift[k] = (float)(cell_origin[3 * cj + k] - cell_origin[3 * ci + k]);
            if (shift[k] * 2 > dim[k])
                shift[k] = (float)(shift[k] - dim[k]);
            else if (shift[k] * 2 < -dim[k])
                shift[k] = (float)(shift[k] + dim[k]);
        }
        int sid = 0;
        for (int k = 0; k < 3; ++k) sid = 3 * sid + ((shift[k] < 0) ? 0 : ((shift[k] > 0) ? 2 : 1));
        if (kCellFlip[sid]) {
            std::swap(ci, cj);
            for (int k = 0; k < 3; ++k) shift[k] = -shift[k];
        }
        return kSortlistID[sid];
    }

    /* engine_init / MxBoundaryConditions_Init: boundary kinds, periodicity and the
     * raise of periodic axes to 3 cells. */
    int configure(const double *o, const double *d, const int *c, const int *kinds, const float *vel,
                  const float *restore) {
        for (int k = 0; k < 3; ++k) {
            origin[k] = o[k];
            dim[k] = d[k];
            cells[k] = c[k];
            if (c[k] < 1 || !(d[k] > o[k])) return MXG_ERR_ARG;
        }
        for (int f = 0; f < 6; ++f) {
            int kind = kinds ? kinds[f] : MXG_BOUNDARY_PERIODIC;
            const bool noslip = kind == MXG_BOUNDARY_NO_SLIP;
            if (noslip) kind = MXG_BOUNDARY_VELOCITY;  // no-slip = zero-velocity wall
            bc_kind[f] = kind;
            for (int q = 0; q < 3; ++q) bc_vel[f][q] = (vel && !noslip) ? vel[3 * f + q] : 0.f;
            bc_restore[f] = restore ? restore[f] : 1.f;
        }
        // a face pair is periodic when either face is (check_periodicy sets both)
        const int faces[3][2] = {{MXG_FACE_LEFT, MXG_FACE_RIGHT}, {MXG_FACE_FRONT, MXG_FACE_BACK},
                                 {MXG_FACE_BOTTOM, MXG_FACE_TOP}};
        period = 0;
        for (int k = 0; k < 3; ++k) {
            const bool lo = bc_kind[faces[k][0]] & MXG_BOUNDARY_PERIODIC, hi = bc_kind[faces[k][1]] & MXG_BOUNDARY_PERIODIC;
            if (lo || hi) {
                bc_kind[faces[k][0]] = bc_kind[faces[k][1]] = MXG_BOUNDARY_PERIODIC;
                period |= 1u << k;
                if (cells[k] < 3) cells[k] = 3;  // MxBoundaryConditions_Init: >= 3 periodic cells
            }
        }
        return MXG_OK;
    }

    int build(double cutoff) {
        // engine_init: L = (dim - origin)/cells; space_init: cdim = floor(dim/L), h = dim/cdim
        for (int k = 0; k < 3; ++k) {
            const double L = (dim[k] - origin[k]) / cells[k];
            cdim[k] = (int)std::floor(dim[k] / L);
            if (cdim[k] < 1) return MXG_ERR_SPACE;
        }
        ncells = cdim[0] * cdim[1] * cdim[2];
        for (int k = 0; k < 3; ++k) {
            h[k] = dim[k] / cdim[k];
            ih[k] = 1.0 / h[k];
        }
        cell_flags.assign(ncells, 0u);
        cell_origin.assign(3 * ncells, 0.0);
        const unsigned active = MXG_BOUNDARY_FREESLIP | MXG_BOUNDARY_VELOCITY;
        int l[3];
        double o[3];
        for (l[0] = 0; l[0] < cdim[0]; l[0]++) {
            o[0] = origin[0] + l[0] * h[0];
            for (l[1] = 0; l[1] < cdim[1]; l[1]++) {
                o[1] = origin[1] + l[1] * h[1];
                for (l[2] = 0; l[2] < cdim[2]; l[2]++) {
                    o[2] = origin[2] + l[2] * h[2];
                    const int c = cellid(l[0], l[1], l[2]);
                    for (int k = 0; k < 3; ++k) cell_origin[3 * c + k] = o[k];
                    unsigned f = 0;
                    if (l[0] == 0 && (bc_kind[MXG_FACE_LEFT] & active))
                        f |= kCellActiveLeft;
                    else if (l[0] + 1 == cdim[0] && (bc_kind[MXG_FACE_RIGHT] & active))
                        f |= kCellActiveRight;
                    if (l[1] == 0 && (bc_kind[MXG_FACE_FRONT] & active))
                        f |= kCellActiveFront;
                    else if (l[1] + 1 == cdim[1] && (bc_kind[MXG_FACE_BACK] & active))
                        f |= kCellActiveBack;
                    if (l[2] == 0 && (bc_kind[MXG_FACE_BOTTOM] & active))
                        f |= kCellActiveBottom;
                    else if (l[2] + 1 == cdim[2] && (bc_kind[MXG_FACE_TOP] & active))
                        f |= kCellActiveTop;
                    cell_flags[c] = f;
                }
            }
        }
        // cell-pair tasks (space.cpp:797-913); no ghost cells on this path
        int span[3];
        for (int k = 0; k < 3; ++k) span[k] = (int)std::ceil(cutoff * ih[k]);
        const double cutoff2 = cutoff * cutoff;
        tasks.clear();
        for (int i = 0; i < cdim[0]; i++)
            for (int j = 0; j < cdim[1]; j++)
                for (int k = 0; k < cdim[2]; k++) {
                    const int id1 = cellid(i, j, k);
                    for (l[0] = -span[0]; l[0] <= span[0]; l[0]++) {
                        int ii = i + l[0];
                        if (ii < 0) {
                            if (period & kPeriodicX) ii += cdim[0]; else continue;
                        } else if (ii >= cdim[0]) {
                            if (period & kPeriodicX) ii -= cdim[0]; else continue;
                        }
                        for (l[1] = -span[1]; l[1] <= span[1]; l[1]++) {
                            int jj = j + l[1];
                            if (jj < 0) {
                                if (period & kPeriodicY) jj += cdim[1]; else continue;
                            } else if (jj >= cdim[1]) {
                                if (period & kPeriodicY) jj -= cdim[1]; else continue;
                            }
                            for (l[2] = -span[2]; l[2] <= span[2]; l[2]++) {
                                double lh[3];
                                for (int q = 0; q < 3; ++q) lh[q] = h[q] * std::fmax(std::abs(l[q]) - 1, 0);
                                if (lh[0] * lh[0] + lh[1] * lh[1] + lh[2] * lh[2] > cutoff2) continue;
                                int kk = k + l[2];
                                if (kk < 0) {
                                    if (period & kPeriodicZ) kk += cdim[2]; else continue;
                                } else if (kk >= cdim[2]) {
                                    if (period & kPeriodicZ) kk -= cdim[2]; else continue;
                                }
                                const int id2 = cellid(ii, jj, kk);
                                int ci = id1, cj = id2;
                                float shift[3];
                                const int sid = getsid(ci, cj, shift);
                                if (id1 < id2 || (id1 == id2 && l[0] == 0 && l[1] == 0 && l[2] == 0))
                                    tasks.push_back({id1 == id2 ? kTaskSelf : kTaskPair, sid, ci, cj});
                            }
                        }
                    }
                }
        return MXG_OK;
    }

    /* space_addpart's placement plus the first shuffle: local cell index and
     * cell-relative float position. */
    int place(const double *x, int &cell, float *xr) const {
        int ind[3];
        for (int k = 0; k < 3; ++k) ind[k] = (int)((x[k] - origin[k]) * ih[k]);
        for (int k = 0; k < 3; ++k)
            if (ind[k] < 0 || ind[k] >= cdim[k]) return MXG_ERR_SPACE;
        cell = cellid(ind[0], ind[1], ind[2]);
        for (int k = 0; k < 3; ++k) xr[k] = (float)(x[k] - cell_origin[3 * cell + k]);
        int delta[3];
        for (int k = 0; k < 3; ++k) {
            const float hf = (float)h[k];
            delta[k] = (xr[k] >= hf ? 1 : 0) - (xr[k] < 0.0f ? 1 : 0);
        }
        if (delta[0] | delta[1] | delta[2]) {
            int loc[3] = {ind[0], ind[1], ind[2]};
            for (int k = 0; k < 3; ++k) {
                xr[k] -= delta[k] * (float)h[k];
                loc[k] = (loc[k] + delta[k] + cdim[k]) % cdim[k];
            }
            cell = cellid(loc[0], loc[1], loc[2]);
        }
        return MXG_OK;
    }

    /* runner_dopair.cpp:132-136: bias = |h|, dscale = SHRT_MAX/(2 bias),
     * dmaxdist = 2 + dscale*(cutoff + 2*maxdx) with maxdx = 0; FP32. */
    float sort_bias() const { return (float)std::sqrt(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]); }
    float sort_dscale() const { return (float)32767 / (2 * sort_bias()); }
    int dmaxdist(double cutoff) const { return (int)(2 + sort_dscale() * ((float)cutoff + 2 * 0.0f)); }
    int dnshift(const float *shift) const {
        const float ns = std::sqrt(shift[0] * shift[0] + shift[1] * shift[1] + shift[2] * shift[2]);
        return (int)(sort_dscale() * ns);
    }
};

struct mxg_engine {
    // ---- configuration shared by all replicas ----
    double cutoff;
    int max_type = 0;
    double dt = 0.01;
    float max_dist_fraction = 0.05f;
    unsigned rng_mode = 0;
    int pruning = 0;  // 0: the reference's pruning, 1: same with the per-pair test on every grid, 2: none

    // ---- replicas ----
    std::vector<Space> spaces;
    int ncells = 0;  // all replicas

    // ---- model ----
    std::vector<TypeInfo> types;
    std::vector<mxg::PotentialTable> pots;  // private copies
    std::vector<double> px;                 // staged positions (3 per particle)
    std::vector<float> pv;
    std::vector<int> ptype;
    std::vector<int> prep;                  // replica of each particle
    std::vector<int> pcell;                 // given cell (replica-local) of each particle, or -1: placed from px
    std::vector<float> pxr;                 // given cell-relative position (3 per particle) where pcell >= 0
    std::vector<BondInfo> bonds;
    std::vector<AngleInfo> angles;
    std::vector<ExclusionInfo> exclusions;
    std::vector<DihedralInfo> dihedrals;
    std::vector<CuboidInfo> cuboids;
    // ---- species and fluxes ----
    std::vector<int> type_nspec;               // per type (0: no state vector)
    std::vector<std::vector<unsigned>> type_sflags;  // per type and species (bit 2: constant)
    std::vector<std::vector<DevFlux>> flux_lists;    // per unordered type pair (a <= b): a * max_type + b
    std::vector<float> spec_host;              // staged values, nparts * smax
    int smax = 0;
    float *d_spec = nullptr, *d_rate = nullptr;
    int *d_nspec = nullptr, *d_flux_off = nullptr, *d_fx_off = nullptr, *d_fx_cell = nullptr;
    unsigned *d_sflags = nullptr;
    DevFlux *d_flux = nullptr;
    float4 *d_fx_shift = nullptr;
    bool has_fluxes = false;

    // ---- device ----
    bool started = false;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    int nparts = 0;
    int ntypes = 0;
    int cur = 0;
    float4 *d_pos[2] = {nullptr, nullptr}, *d_vel[2] = {nullptr, nullptr};
    float4 *d_force = nullptr;
    int *d_cell_of[2] = {nullptr, nullptr};
    int *d_new_cell = nullptr;
    int *d_cell_start[2] = {nullptr, nullptr}, *d_cell_count[2] = {nullptr, nullptr};
    // movers per cell and per chunk of cells, by step parity: a step counts into its own parity and
    // its re-binning clears the other one, so the counts of the parity about to step are zero
    int *d_in_count[2] = {nullptr, nullptr}, *d_out_count[2] = {nullptr, nullptr};
    int *d_chunk_delta[2] = {nullptr, nullptr};
    int nchunks = 0;
    int *d_in_list = nullptr;
    int *d_ovf_list = nullptr, *d_ovf_count = nullptr;  // movers beyond their destination's bucket
    unsigned *d_rebin_ctl = nullptr;                    // re-binning: finished blocks of the scatter
    // device-side load and unload (allocated at the first call)
    double *d_ld_x = nullptr, *d_ul_x = nullptr;
    float *d_ld_v = nullptr, *d_ul_v = nullptr, *d_ul_f = nullptr, *d_ul_xrel = nullptr;
    float4 *d_ld_xr = nullptr, *d_ld_vel = nullptr;
    int *d_ld_cell = nullptr, *d_ld_ids = nullptr, *d_ld_count = nullptr, *d_ld_fill = nullptr, *d_ld_err = nullptr;
    int *h_ld_err = nullptr;  // pinned: the load's out-of-box flag, read back without a staging copy
    cudaStream_t ld_stream = nullptr;               // the load's velocity copy, beside the placement
    cudaEvent_t ld_x_done = nullptr, ld_v_done = nullptr;
    int *d_type_of_id = nullptr, *d_rep_of_id = nullptr, *d_ul_cell = nullptr;
    int *d_slot_of_id = nullptr;
    int *d_cell_rep = nullptr;
    unsigned *d_cell_flags = nullptr;
    int *d_nb_off = nullptr, *d_nb_cell = nullptr, *d_nb_rev = nullptr, *d_sec_count = nullptr;
    float4 *d_nb_shift = nullptr;
    float4 *d_planes = nullptr;
    int nplanes = 0;
    int4 *d_items = nullptr;            // force work items: (cell, first entry, end entry, part)
    int *d_item_ctr = nullptr;          // the force kernel's work-item counter and finished-warp count
    int *d_item_order = nullptr;        // work items, most crowded cells first (when cells are split)
    bool order_items = false;
    long long occupancy_hint = 0;       // particle count the work-item split is decided on (0: nparts)
    bool dpd_pure = false;              // every pair potential DPD, no summed second term, no Philox
    int *d_cell_planes = nullptr;       // planes summed into each cell's forces
    int nitems = 0;
    DevPot *d_pots = nullptr;
    float *d_coef = nullptr;
    int *d_pot_idx = nullptr;
    int *d_pot_idx2 = nullptr;   // second summed potential per type pair, or -1
    float4 *d_dpd_pair = nullptr;  // DPD-only kernel: two records per replica and type pair
    std::vector<int> h_pot_idx;    // the device's potential index per replica and type pair
    bool has_second = false;
    DevType *d_types = nullptr;
    DevSpace *d_spaces = nullptr;
    SortAxes *d_axes = nullptr;
    int2 *d_sort_bounds = nullptr;
    double *d_epot_cell = nullptr, *d_ebond_slot = nullptr;
    DevBond *d_bonds = nullptr;
    unsigned *d_bond_flags = nullptr;
    // ---- adjoint ----
    struct GradReg {
        int pot, param, slot;
    };
    std::vector<GradReg> grad_regs;        // differentiated (potential, parameter) -> gradient slot
    int grad_slots = 0;
    bool adjoint_stale = true;             // derivative tables need a rebuild
    DevPotGrad *d_pot_grad = nullptr;
    float *d_dcoef = nullptr;
    size_t dcoef_cap = 0;
    float4 *d_adj_w = nullptr, *d_adj_gx = nullptr, *d_adj_gv = nullptr;
    double *d_adj_partials = nullptr;
    int4 *d_adj_items = nullptr;            // the pair VJP's work items
    int *d_adj_ctr = nullptr;
    float4 *d_adj_pgx = nullptr, *d_adj_pgv = nullptr;
    int adj_nitems = 0;
    std::vector<int> h_nb_off;              // per cell: first neighbour entry (host copy)
    double *d_adj_bond_partials = nullptr;
    double *d_virial_partials = nullptr, *d_virial_out = nullptr;
    double *d_bvirial_partials = nullptr;  // bonded virial: per block, 9 components
    float *d_nd = nullptr;                  // number density by id (allocated at the first request)
    int virial_cap = 0;
    int *d_bond_off = nullptr, *d_bond_list = nullptr;
    int2 *d_excl = nullptr;
    int *d_excl_off = nullptr, *d_excl_list = nullptr;
    DevAngle *d_angles = nullptr;
    int *d_angle_off = nullptr, *d_angle_list = nullptr;
    DevDihedral *d_dihedrals = nullptr;
    int *d_dihedral_off = nullptr, *d_dihedral_list = nullptr;
    unsigned *d_status = nullptr;
    unsigned long long *d_step = nullptr;
    double *d_partials = nullptr, *d_energy = nullptr;
    int energy_blocks = 64;
    bool has_dpd = false;
    bool has_sb = false;                // a type has a Berendsen, random or friction force
    bool has_walls = false;             // a type has a wall potential
    int nlarge = 0;                     // large particles (radius > cutoff)
    float4 *d_large_x = nullptr, *d_large_v = nullptr;
    int *d_large_rep = nullptr, *d_large_pot = nullptr;
    double *d_body_e = nullptr;         // per slot: wall and large-particle energy of the last pass
    float4 *d_body_f = nullptr;         // per slot: wall and large-particle force of the pass
    bool has_cuboid_forces = false;     // a cuboid exists and a type has a cuboid potential
    DevCuboid *d_cuboids = nullptr;
    bool has_body() const { return has_walls || nlarge > 0 || has_cuboid_forces; }
    double *d_type_ke = nullptr;
    float4 *d_persist = nullptr;
    int integrator = 0;                 // 0 forward Euler, 1 Runge-Kutta 4 (engine.h EngineIntegrator)
    int force_layout = 0;               // the buffer whose slot order the force array follows
    float4 *d_rk[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};  // RK4 per-slot stage state
    int force_grid = 0;
    int force_variant = 0;              // tile shape of the force kernel (autotuned)
    int num_sms = 148;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    bool use_graphs = true;
    std::vector<void *> allocations;

    ~mxg_engine() {
        for (int k = 0; k < 2; ++k)
            if (graph[k]) cudaGraphExecDestroy(graph[k]);
        for (void *p : allocations) cudaFree(p);
        if (h_ld_err) cudaFreeHost(h_ld_err);
        if (ld_x_done) cudaEventDestroy(ld_x_done);
        if (ld_v_done) cudaEventDestroy(ld_v_done);
        if (ld_stream) cudaStreamDestroy(ld_stream);
        if (own_stream) cudaStreamDestroy(own_stream);
    }

    /* The DPD-only kernel's constants, two records per replica and type pair (see
     * EngineView::dpd_pair); one empty record when that kernel is not used. */
    std::vector<float4> dpd_records(const std::vector<DevPot> &hp) const {
        std::vector<float4> out(dpd_pure ? 2 * h_pot_idx.size() : 1, make_float4(0.f, 0.f, 0.f, 0.f));
        if (!dpd_pure) return out;
        for (size_t k = 0; k < h_pot_idx.size(); ++k) {
            if (h_pot_idx[k] < 0) continue;
            const DevPot &d = hp[h_pot_idx[k]];
            const float sd = d.dpd_sigma * d.dpd_delta;
            out[2 * k] = make_float4(d.b, d.dpd_alpha, d.dpd_gamma, sd);
            out[2 * k + 1] = make_float4(d.a2, d.a, 1.0f / d.b, d.dpd_alpha + sd);
        }
        return out;
    }

    /* Device form of the potentials: one DevPot each and the pooled coefficients. */
    void pot_arrays(std::vector<DevPot> &hp, std::vector<float> &coef) {
        hp.clear();
        coef.clear();
        has_dpd = false;
        for (const auto &t : pots) {
            DevPot d;
            memset(&d, 0, sizeof(d));
            d.kind = t.kind;
            d.flags = t.flags;
            d.n = t.n;
            d.coef_off = (int)coef.size();
            d.alpha0 = t.alpha[0];
            d.alpha1 = t.alpha[1];
            d.alpha2 = t.alpha[2];
            d.a = t.a;
            d.b = t.b;
            d.r0_plusone = t.r0_plusone;
            d.a2 = t.a * t.a;
            d.dpd_alpha = t.dpd_alpha;
            d.dpd_gamma = t.dpd_gamma;
            d.dpd_sigma = t.dpd_sigma;
            d.dpd_delta = (float)(1.f / std::sqrt(dt));  // dpd_eval.hpp:23, from the engine dt
            if (t.kind == kKindDPD) has_dpd = true;
            coef.insert(coef.end(), t.c.begin(), t.c.end());
            hp.push_back(d);
        }
    }

    template <typename T>
    int alloc(T **p, size_t n) {
        int rc = dev_alloc(p, n);
        if (rc == MXG_OK) allocations.push_back((void *)*p);
        return rc;
    }

    DevSpace space_desc(int r, int pot_offset) const {
        const Space &sp = spaces[r];
        DevSpace S;
        memset(&S, 0, sizeof(S));
        const float dtf = (float)dt;
        for (int k = 0; k < 3; ++k) {
            S.hd[k] = sp.h[k];
            S.ih[k] = sp.ih[k];
            S.h[k] = (float)sp.h[k];
            S.h2[k] = (float)(2. * sp.h[k]);
            S.maxv[k] = (S.h[k] * max_dist_fraction) / dtf;
            S.maxv2[k] = S.maxv[k] * S.maxv[k];
            S.maxx[k] = S.h[k] * max_dist_fraction;
            S.maxx2[k] = S.maxx[k] * S.maxx[k];
            S.cdim[k] = sp.cdim[k];
            S.origin[k] = sp.origin[k];
        }
        S.dt = dtf;
        S.dt_d = dt;
        S.cutoff_d = cutoff;
        const float cf = (float)cutoff;
        S.cut2_pair = cf * cf;                  // runner_dopair: float cutoff squared
        S.cut2_self = (float)(cutoff * cutoff);  // runner_doself: s->cutoff2 (double) as float
        // the candidate pass forms x_i - (x_j + s) instead of (x_i - s) - x_j: one rounding of
        // coordinates below 2h apart, covered by a margin far above it (the exact test follows)
        const double hmax = std::max(sp.h[0], std::max(sp.h[1], sp.h[2]));
        const double margin = 2e-5 * (3 * hmax * hmax + cutoff * cutoff);
        S.cut2w_pair = (float)((double)S.cut2_pair + margin);
        S.cut2w_self = (float)((double)S.cut2_self + margin);
        S.cell_offset = sp.cell_offset;
        S.ncells = sp.ncells;
        S.pot_offset = pot_offset;
        for (int f = 0; f < 6; ++f) {
            S.bc_kind[f] = (unsigned)sp.bc_kind[f];
            for (int q = 0; q < 3; ++q) S.bc_vel[f][q] = sp.bc_vel[f][q];
            S.bc_restore[f] = sp.bc_restore[f];
        }
        S.rng_mode = rng_mode;
        // the per-pair projection test can only drop a pair inside the cutoff when
        // the cells are not cubic; the cell-pair exit test applies to every grid
        const bool cubic = sp.h[0] == sp.h[1] && sp.h[1] == sp.h[2];
        S.prune = pruning == 2 ? 0 : (2 | ((pruning == 1 || !cubic) ? 1 : 0));
        S.dmaxdist = sp.dmaxdist(cutoff);
        S.sort_bias = sp.sort_bias();
        S.sort_dscale = sp.sort_dscale();
        return S;
    }

    /* Places every staged particle in its replica (global cell index and
     * cell-relative position) and orders them by cell, then id. */
    int stage(std::vector<float4> &hpos, std::vector<float4> &hvel, std::vector<int> &hcell_of,
              std::vector<int> &hslot, std::vector<int> &hcount, std::vector<int> &hstart) const {
        const int n = (int)ptype.size();
        std::vector<int> cell(n);
        std::vector<float> xr(3 * (size_t)n);
        for (int p = 0; p < n; ++p) {
            const Space &sp = spaces[prep[p]];
            if (pcell[p] >= 0) {  // added with its cell and cell-relative position: kept as given
                cell[p] = sp.cell_offset + pcell[p];
                for (int k = 0; k < 3; ++k) xr[3 * (size_t)p + k] = pxr[3 * (size_t)p + k];
                continue;
            }
            int lc;
            int rc = sp.place(&px[3 * (size_t)p], lc, &xr[3 * (size_t)p]);
            if (rc != MXG_OK) return rc;
            cell[p] = sp.cell_offset + lc;
        }
        std::vector<int> order(n);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cell[a] < cell[b]; });
        hpos.assign(n, make_float4(0.f, 0.f, 0.f, 0.f));
        hvel.assign(n, make_float4(0.f, 0.f, 0.f, 0.f));
        hcell_of.assign(n, 0);
        hslot.assign(n, 0);
        hcount.assign(ncells, 0);
        hstart.assign(ncells + 1, 0);
        for (int s = 0; s < n; ++s) {
            const int p = order[s];
            hpos[s] = make_float4(xr[3 * (size_t)p], xr[3 * (size_t)p + 1], xr[3 * (size_t)p + 2], 0.f);
            int t = ptype[p];
            memcpy(&hpos[s].w, &t, 4);
            hvel[s] = make_float4(pv[3 * (size_t)p], pv[3 * (size_t)p + 1], pv[3 * (size_t)p + 2], 0.f);
            memcpy(&hvel[s].w, &p, 4);
            hcell_of[s] = cell[p];
            hslot[p] = s;
            hcount[cell[p]]++;
        }
        for (int c = 0; c < ncells; ++c) hstart[c + 1] = hstart[c] + hcount[c];
        return MXG_OK;
    }

    EngineView view(int b) const {
        EngineView v;
        v.pos = d_pos[b];
        v.vel = d_vel[b];
        v.force = d_force;
        v.cell_of = d_cell_of[b];
        v.cell_start = d_cell_start[b];
        v.cell_count = d_cell_count[b];
        v.cell_rep = d_cell_rep;
        v.cell_flags = d_cell_flags;
        v.nb_off = d_nb_off;
        v.nb_cell = d_nb_cell;
        v.nb_shift = d_nb_shift;
        v.pots = d_pots;
        v.coef = d_coef;
        v.pot_idx = d_pot_idx;
        v.pot_idx2 = has_second ? d_pot_idx2 : nullptr;
        v.types = d_types;
        v.spaces = d_spaces;
        v.ntypes = ntypes;
        v.ncells = ncells;
        v.nparts = nparts;
        v.step = d_step;
        v.axes = d_axes;
        v.sort_bounds = d_sort_bounds;
        v.epot_cell = d_epot_cell;
        v.status = d_status;
        v.pair_stats = nullptr;
        v.virial_partials = nullptr;
        v.has_sb = has_sb ? 1 : 0;
        v.type_ke = d_type_ke;
        v.persist = d_persist;
        v.nb_rev = d_nb_rev;
        v.sec_count = d_sec_count;
        v.cell_planes = d_cell_planes;
        v.items = d_items;
        v.item_ctr = d_item_ctr;
        v.item_order = order_items ? d_item_order : nullptr;
        v.dpd_pure = dpd_pure ? 1 : 0;
        v.force_variant = force_variant;
        v.nitems = nitems;
        v.planes = d_planes;
        v.body_e = has_body() ? d_body_e : nullptr;
        v.body_f = has_body() ? d_body_f : nullptr;
        v.large_x = d_large_x;
        v.large_v = d_large_v;
        v.large_rep = d_large_rep;
        v.large_pot = d_large_pot;
        v.nlarge = nlarge;
        v.cuboids = d_cuboids;
        v.ncuboids = has_cuboid_forces ? (int)cuboids.size() : 0;
        v.dpd_pair = dpd_pure ? d_dpd_pair : nullptr;
        v.chunk_delta = d_chunk_delta[b];
        v.ovf_list = d_ovf_list;
        v.ovf_count = d_ovf_count;
        return v;
    }

    bool has_bonded() const {
        return !bonds.empty() || !angles.empty() || !dihedrals.empty() || !exclusions.empty();
    }

    BondedView bonded_view() const {
        BondedView bv;
        bv.excl = d_excl;
        bv.excl_off = d_excl_off;
        bv.excl_list = d_excl_list;
        bv.bonds = d_bonds;
        bv.bond_flags = d_bond_flags;
        bv.bond_off = d_bond_off;
        bv.bond_list = d_bond_list;
        bv.angles = d_angles;
        bv.angle_off = d_angle_off;
        bv.angle_list = d_angle_list;
        bv.dihedrals = d_dihedrals;
        bv.dihedral_off = d_dihedral_off;
        bv.dihedral_list = d_dihedral_list;
        bv.slot_of_id = d_slot_of_id;
        bv.e_slot = d_ebond_slot;
        return bv;
    }

    /* The force pass alone (engine_force): the bonded kernel, or the combine
     * kernel when there are no bonded interactions, adds the received planes. */
    void enqueue_force(int b) {
        force_layout = b;
        const EngineView v = view(b);
        if (has_sb) launch_singlebody_prep(v, ntypes, d_type_ke, d_persist, false, stream);
        if (has_body()) launch_body(v, d_body_f, stream);
        launch_force(v, has_dpd, force_grid, !has_bonded(), stream);
        if (has_bonded()) launch_bonded(v, bonded_view(), stream);
        if (has_fluxes) launch_fluxes(v, species_view(), stream);
    }

    SpeciesView species_view() const {
        SpeciesView sp;
        sp.value = d_spec;
        sp.rate = d_rate;
        sp.nspec = d_nspec;
        sp.flags = d_sflags;
        sp.flux_off = d_flux_off;
        sp.flux = d_flux;
        sp.fx_off = d_fx_off;
        sp.fx_cell = d_fx_cell;
        sp.fx_shift = d_fx_shift;
        sp.smax = smax;
        return sp;
    }

    /* One step (engine_step): force pass, bonded pass, integrator and re-binning;
     * the received planes are added by the bonded kernel or, without bonded
     * interactions, by the integrator; the re-binning pass computes the new key
     * bounds. */
    /* ev (optional, 6 events): recorded at the phase boundaries prepare | nonbond | bonded |
     * advance | shuffle (the reference's engine timers). */
    void enqueue_step(int b, cudaEvent_t *ev = nullptr) {
        auto mark = [&](int k) {
            if (ev) cudaEventRecord(ev[k], stream);
        };
        if (integrator == 1) {
            mark(0);
            mark(1);
            mark(2);
            mark(3);
            enqueue_step_rk4(b);
            mark(4);
            mark(5);
            return;
        }
        const EngineView v = view(b);
        mark(0);
        if (has_sb) launch_singlebody_prep(v, ntypes, d_type_ke, d_persist, true, stream);
        if (has_body()) launch_body(v, d_body_f, stream);
        mark(1);
        launch_force(v, has_dpd, force_grid, false, stream);
        mark(2);
        if (has_bonded()) launch_bonded(v, bonded_view(), stream);
        if (has_fluxes) launch_fluxes(v, species_view(), stream);
        mark(3);
        launch_integrate(v, d_pos[b], d_vel[b], d_new_cell, d_in_count[b], d_in_list, d_out_count[b], !has_bonded(),
                         stream);
        if (has_fluxes) launch_species_integrate(v, species_view(), d_new_cell, stream);  // MxFluxes_Integrate
        mark(4);
        enqueue_scatter(v, b);
        mark(5);
    }

    void enqueue_scatter(const EngineView &v, int b) {
        const int nb = 1 - b;
        launch_scatter(v, d_pos[b], d_vel[b], d_new_cell, d_cell_start[b], d_cell_count[b], d_in_count[b], d_in_list,
                       d_out_count[b], d_cell_start[nb], d_cell_count[nb], d_pos[nb], d_vel[nb], d_cell_of[nb],
                       d_slot_of_id, d_in_count[nb], d_out_count[nb], d_chunk_delta[nb], nchunks, d_rebin_ctl,
                       d_step, stream);
    }

    /* One Runge-Kutta 4 step (engine_advance_runge_kutta_4): four force passes (with
     * the bonded pass when present), stage updates in the step's cell frame with fresh key
     * bounds before each intermediate pass, then the final update, re-binning as
     * for Euler. */
    void enqueue_step_rk4(int b) {
        const EngineView v = view(b);
        for (int stage = 0; stage < 4; ++stage) {
            // persistent random forces are redrawn in the first stage only (INTEGRATOR_UPDATE_PERSISTENTFORCE)
            if (has_sb) launch_singlebody_prep(v, ntypes, d_type_ke, d_persist, stage == 0, stream);
            if (has_body()) launch_body(v, d_body_f, stream);
            launch_force(v, has_dpd, force_grid, false, stream);
            if (has_bonded()) launch_bonded(v, bonded_view(), stream);
            if (stage < 3) {
                launch_rk_stage(v, d_pos[b], d_rk, stage, !has_bonded(), stream);
                launch_sort_bounds(v, stream);
            } else {
                launch_rk_final(v, d_pos[b], d_vel[b], d_rk, d_new_cell, d_in_count[b], d_in_list, d_out_count[b],
                                !has_bonded(), stream);
            }
        }
        enqueue_scatter(v, b);
    }

    /* Key bounds for a state that did not come from the re-binning pass. */
    void refresh_bounds() { launch_sort_bounds(view(cur), stream); }

    /* Derivative tables and per-potential parameter descriptors for the VJP. */
    int build_adjoint() {
        std::vector<DevPotGrad> hg(std::max<size_t>(1, pots.size()));
        for (auto &g : hg) memset(&g, 0, sizeof(g));
        std::vector<float> dcoef;
        for (const GradReg &r : grad_regs) {
            const mxg::PotentialTable &t = pots[r.pot];
            DevPotGrad &g = hg[r.pot];
            if (g.n >= kMaxPotGrads) return MXG_ERR_RANGE;
            int mode = -1, off = 0;
            if (t.kind == kKindDPD) {
                mode = r.param == 0 ? kGradDpdAlpha : r.param == 1 ? kGradDpdGamma : r.param == 2 ? kGradDpdSigma : -1;
            } else if (t.form == mxg::kFormMorse && r.param == 2) {
                mode = kGradShift;  // r0 shifts the table's argument
            } else {
                mxg::PotentialTable d;
                if (mxg::param_derivative_table(t, r.param, d) != 0) return MXG_ERR_ARG;
                mode = kGradTable;
                off = (int)dcoef.size();
                dcoef.insert(dcoef.end(), d.c.begin(), d.c.end());
            }
            if (mode < 0) return MXG_ERR_ARG;
            g.mode[g.n] = mode;
            g.slot[g.n] = r.slot;
            g.coef_off[g.n] = off;
            ++g.n;
        }
        if (!d_pot_grad) {
            int rc = alloc(&d_pot_grad, hg.size());
            rc |= alloc(&d_adj_w, (size_t)nparts);
            rc |= alloc(&d_adj_gx, (size_t)nparts);
            rc |= alloc(&d_adj_gv, (size_t)nparts);
            // the pair VJP's work items: each cell's entries in vjp_parts() contiguous groups
            const int P = vjp_parts();
            std::vector<int4> items;
            for (int c = 0; c < ncells; ++c) {
                const int e0 = h_nb_off[c], ne = h_nb_off[c + 1] - e0;
                for (int g = 0; g < P; ++g) items.push_back(make_int4(c, e0 + g * ne / P, e0 + (g + 1) * ne / P, g));
            }
            adj_nitems = (int)items.size();
            rc |= alloc(&d_adj_items, items.size());
            rc |= alloc(&d_adj_ctr, 2);
            rc |= alloc(&d_adj_pgx, (size_t)std::max(1, P - 1) * nparts);
            rc |= alloc(&d_adj_pgv, (size_t)std::max(1, P - 1) * nparts);
            rc |= alloc(&d_adj_partials, (size_t)std::max(1, adj_nitems) * kMaxGradSlots);
            if (rc == MXG_OK) {
                CUDA_TRY(cudaMemsetAsync(d_adj_ctr, 0, 2 * sizeof(int), stream));
                rc = upload(d_adj_items, items, stream);
                if (rc == MXG_OK) CUDA_TRY(cudaStreamSynchronize(stream));
            }
            rc |= alloc(&d_adj_bond_partials, (size_t)adjoint_bond_blocks(num_sms) * kMaxGradSlots);
            if (rc != MXG_OK) return MXG_ERR_MALLOC;
            configure_adjoint_kernels();
        }
        if (dcoef.size() + 8 > dcoef_cap) {
            dcoef_cap = dcoef.size() + 8;
            if (alloc(&d_dcoef, dcoef_cap) != MXG_OK) return MXG_ERR_MALLOC;
        }
        int rc;
        if ((rc = upload(d_pot_grad, hg, stream)) || (rc = upload(d_dcoef, dcoef, stream))) return rc;
        adjoint_stale = false;
        return MXG_OK;
    }

    /* Layout of a state snapshot: byte offsets of its sections (16-byte aligned). */
    struct SnapLayout {
        size_t pos, vel, cell_of, slot_of_id, start, count, step, bonds, spec, rate, persist, total;
    };
    SnapLayout snap_layout() const {
        SnapLayout L;
        size_t o = 0;
        auto take = [&](size_t bytes) {
            const size_t at = o;
            o += (bytes + 15) & ~(size_t)15;
            return at;
        };
        L.pos = take(sizeof(float4) * (size_t)nparts);
        L.vel = take(sizeof(float4) * (size_t)nparts);
        L.cell_of = take(sizeof(int) * (size_t)nparts);
        L.slot_of_id = take(sizeof(int) * (size_t)nparts);
        L.start = take(sizeof(int) * (size_t)(ncells + 1));
        L.count = take(sizeof(int) * (size_t)ncells);
        L.step = take(sizeof(unsigned long long));
        L.bonds = take(sizeof(unsigned) * bonds.size());
        L.spec = take(sizeof(float) * (size_t)nparts * smax);
        L.rate = take(sizeof(float) * (size_t)nparts * smax);
        L.persist = take(has_sb ? sizeof(float4) * (size_t)nparts : 0);
        L.total = o;
        return L;
    }

    int start(cudaStream_t st);
    int build_graphs();
    int load_state(const double *x, const float *v, int n);
};

int mxg_engine::start(cudaStream_t st) {
    if (!st) {
        // graphs cannot be captured on the legacy default stream: use an own stream
        CUDA_TRY(cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking));
        st = own_stream;
    }
    stream = st;
    nparts = (int)ptype.size();
    ntypes = std::max(1, (int)types.size());
    // ---- host staging: placement, ordering ----
    std::vector<float4> hpos, hvel;
    std::vector<int> hcell_of, hslot, hcount, hstart;
    int rc = stage(hpos, hvel, hcell_of, hslot, hcount, hstart);
    if (rc != MXG_OK) return rc;

    // ---- neighbour entries from each replica's task list (global cell indices) ----
    // Each pair task is evaluated once, by the cell in the reference's FIRST role; the
    // forces on the SECOND cell's particles go to one plane of received sums per SECOND
    // entry of that cell (rev), added in plane order after the force pass.
    struct NbEntry {
        int cell;
        float4 shift;
        int rev;
    };
    std::vector<std::vector<NbEntry>> nb(ncells);
    std::vector<int> hsec(ncells, 0);
    std::vector<int> hrep(ncells, 0);
    std::vector<unsigned> hcflags(ncells, 0u);
    for (int r = 0; r < (int)spaces.size(); ++r) {
        const Space &sp = spaces[r];
        const int off = sp.cell_offset;
        for (int c = 0; c < sp.ncells; ++c) {
            hrep[off + c] = r;
            hcflags[off + c] = sp.cell_flags[c];
        }
        for (const Task &t : sp.tasks) {
            if (t.type == kTaskSelf) {
                float4 e = make_float4(0.f, 0.f, 0.f, 0.f);
                int role = kRoleSelf;
                memcpy(&e.w, &role, 4);
                nb[off + t.i].push_back({off + t.i, e, -1});
            } else if (t.type == kTaskPair) {
                int ci = t.i, cj = t.j;
                float shift[3];
                const int sid = sp.getsid(ci, cj, shift);  // runner_dopair recomputes the shift (and flip)
                const int dn = sp.dnshift(shift);
                float4 e1 = make_float4(shift[0], shift[1], shift[2], 0.f), e2 = e1;
                int r1 = kRoleFirst | (sid << 2) | (dn << 8), r2 = kRoleSecond | (sid << 2) | (dn << 8);
                memcpy(&e1.w, &r1, 4);
                memcpy(&e2.w, &r2, 4);
                nb[off + ci].push_back({off + cj, e1, hsec[off + cj]});
                nb[off + cj].push_back({off + ci, e2, -1});
                ++hsec[off + cj];
            }
        }
    }
    // ---- species fluxes: every task of each cell (SELF, FIRST and SECOND entries) for the
    // full-shell flux pass, per-type species tables and the type pairs' flux lists ----
    std::vector<int> fx_off(ncells + 1, 0), fx_cell, hnspec(ntypes, 0), hfoff((size_t)ntypes * ntypes + 1, 0);
    std::vector<float4> fx_shift;
    std::vector<unsigned> hsflags;
    std::vector<DevFlux> hflux;
    smax = 0;
    for (int a = 0; a < (int)type_nspec.size() && a < ntypes; ++a) {
        hnspec[a] = type_nspec[a];
        smax = std::max(smax, type_nspec[a]);
    }
    hsflags.assign((size_t)ntypes * std::max(1, smax), 0u);
    for (int a = 0; a < (int)type_sflags.size() && a < ntypes; ++a)
        for (int k = 0; k < (int)type_sflags[a].size() && k < smax; ++k) hsflags[(size_t)a * smax + k] = type_sflags[a][k];
    for (int a = 0; a < ntypes; ++a)
        for (int b = 0; b < ntypes; ++b) {
            const size_t key = (size_t)std::min(a, b) * max_type + std::max(a, b);
            if (smax > 0 && key < flux_lists.size())
                for (const DevFlux &f : flux_lists[key]) hflux.push_back(f);
            hfoff[(size_t)a * ntypes + b + 1] = (int)hflux.size();
        }
    has_fluxes = smax > 0 && !hflux.empty();
    if (has_fluxes) {
        for (int c = 0; c < ncells; ++c) {
            for (const NbEntry &e : nb[c]) {
                fx_cell.push_back(e.cell);
                fx_shift.push_back(e.shift);  // w: role | sort id << 2 | key shift << 8
            }
            fx_off[c + 1] = (int)fx_cell.size();
        }
    }
    if (smax > 0 && spec_host.size() != (size_t)nparts * smax) spec_host.resize((size_t)nparts * smax, 0.0f);

    // ---- work items: each cell's SELF and FIRST entries split into up to `parts`
    // groups (one warp each) when there are too few cells to fill the GPU. Crowded cells
    // (mean occupancy 16 or more) aim at about three waves of items: their items are long
    // and uneven, and warps fetch items from a counter, so finer items shorten the tail
    // that the most crowded cells leave. Sparse cells aim at one wave of resident warps
    // (5 blocks of kWarpsPerBlock per SM): their items are short and each split adds a
    // staging of the cell's own particles. Item k > 0 of a cell sums its own-side forces
    // into plane sec_count + k - 1 of the cell.
    {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        num_sms = sms;
    }
    const bool crowded = (occupancy_hint > 0 ? occupancy_hint : (long long)nparts) >= 16LL * std::max(1, ncells);
    const int want_warps = num_sms * (crowded ? 64 : 5 * kWarpsPerBlock);
    const int parts = std::max(1, std::min(kMaxCellParts, (want_warps + ncells - 1) / std::max(1, ncells)));
    std::vector<int> nb_off(ncells + 1, 0), nb_cell, nb_rev, hplanes(ncells, 0);
    std::vector<float4> nb_shift;
    std::vector<int4> hitems;
    for (int c = 0; c < ncells; ++c) {
        std::vector<const NbEntry *> self_e, first_e, second_e;
        for (auto &e : nb[c]) {
            int pk;
            memcpy(&pk, &e.shift.w, 4);
            ((pk & 3) == kRoleSelf ? self_e : (pk & 3) == kRoleFirst ? first_e : second_e).push_back(&e);
        }
        const int nf = (int)first_e.size();
        auto push = [&](const NbEntry *e) {
            nb_cell.push_back(e->cell);
            nb_shift.push_back(e->shift);
            nb_rev.push_back(e->rev);
        };
        // a split cell's SELF entry is an item of its own (the crowded cells' n^2 own pairs
        // would otherwise make their first item the longest of the launch)
        const bool self_alone = parts > 1 && !self_e.empty() && nf >= 2;
        const int fgroups = std::max(1, std::min(self_alone ? parts - 1 : parts, nf));
        const int groups = fgroups + (self_alone ? 1 : 0);
        if (self_alone) {
            const int e0 = (int)nb_cell.size();
            for (auto *e : self_e) push(e);
            hitems.push_back(make_int4(c, e0, (int)nb_cell.size(), 0));
        }
        for (int g = 0; g < fgroups; ++g) {
            const int e0 = (int)nb_cell.size();
            if (g == 0 && !self_alone)
                for (auto *e : self_e) push(e);
            for (int k = g * nf / fgroups; k < (g + 1) * nf / fgroups; ++k) push(first_e[k]);
            hitems.push_back(make_int4(c, e0, (int)nb_cell.size(), g + (self_alone ? 1 : 0)));
        }
        for (auto *e : second_e) push(e);
        nb_off[c + 1] = (int)nb_cell.size();
        hplanes[c] = hsec[c] + groups - 1;
    }
    nitems = (int)hitems.size();
    h_nb_off = nb_off;
    // few crowded cells, split into several items each: the launch's length is set by the
    // most crowded cells' items, so they are handed out first (reordered before every force
    // pass). With sparse cells (mean occupancy below 16) the items are short and the
    // ordering launch costs more than the tail it removes.
    order_items = parts > 1 && crowded && nitems <= kOrderMaxItems;
    nplanes = 0;
    for (int c = 0; c < ncells; ++c) nplanes = std::max(nplanes, hplanes[c]);

    // ---- potentials, types, replicas ----
    std::vector<DevPot> hp;
    std::vector<float> coef;
    pot_arrays(hp, coef);
    const int tt = ntypes * ntypes;
    std::vector<int> hpidx((size_t)tt * spaces.size(), -1), hpidx2((size_t)tt * spaces.size(), -1);
    std::vector<DevSpace> hs;
    has_second = false;
    for (int r = 0; r < (int)spaces.size(); ++r) {
        for (int a = 0; a < (int)types.size(); ++a)
            for (int b = 0; b < (int)types.size(); ++b) {
                int p1 = spaces[r].pot_idx[a * max_type + b], p2 = spaces[r].pot2_idx[a * max_type + b];
                if (p1 < 0) std::swap(p1, p2);  // a lone second term acts as the pair's potential
                hpidx[(size_t)r * tt + a * ntypes + b] = p1;
                hpidx2[(size_t)r * tt + a * ntypes + b] = p2;
                if (p2 >= 0) has_second = true;
            }
        hs.push_back(space_desc(r, r * tt));
    }
    // ---- large particles (radius > cutoff: PARTICLE_LARGE, MxParticle.cpp:2091-2093): kept in
    // their cells but static and out of the cell-pair loop; every other particle of the replica
    // interacts with them through the potential of the type pair (particle_largecell_force)
    std::vector<char> is_large(ntypes, 0);
    for (int a = 0; a < (int)types.size(); ++a) is_large[a] = (double)(float)types[a].radius > cutoff;
    std::vector<float4> hlx, hlv;
    std::vector<int> hlrep, hlpot((size_t)tt * spaces.size(), -1);
    for (int id = 0; id < nparts; ++id) {
        if (!is_large[ptype[id]]) continue;
        const Space &sp = spaces[prep[id]];
        float4 q;
        q.x = (float)(px[3 * (size_t)id] - sp.origin[0]);  // position local to the large-particle cell
        q.y = (float)(px[3 * (size_t)id + 1] - sp.origin[1]);
        q.z = (float)(px[3 * (size_t)id + 2] - sp.origin[2]);
        int t = ptype[id];
        memcpy(&q.w, &t, 4);
        hlx.push_back(q);
        float4 w = make_float4(pv[3 * (size_t)id], pv[3 * (size_t)id + 1], pv[3 * (size_t)id + 2], 0.f);
        memcpy(&w.w, &id, 4);
        hlv.push_back(w);
        hlrep.push_back(prep[id]);
    }
    nlarge = (int)hlx.size();
    for (size_t r = 0; r < spaces.size(); ++r)
        for (int a = 0; a < ntypes; ++a)
            for (int b = 0; b < ntypes; ++b) {
                const size_t k = r * tt + (size_t)a * ntypes + b;
                if (!is_large[a] && !is_large[b]) continue;
                if (!is_large[a] && is_large[b]) hlpot[k] = hpidx[k];
                hpidx[k] = -1;  // large particles take no part in the cell-pair loop
                hpidx2[k] = -1;
            }
    dpd_pure = has_dpd && rng_mode == 0;
    for (int k : hpidx)
        if (k >= 0 && (pots[k].kind != kKindDPD || (pots[k].flags & kFlagShifted))) dpd_pure = false;
    for (int k : hpidx2)
        if (k >= 0) dpd_pure = false;
    h_pot_idx = hpidx;
    const std::vector<float4> hdpd = dpd_records(hp);
    has_sb = false;
    has_walls = false;
    has_cuboid_forces = false;
    std::vector<DevType> ht(ntypes);
    for (DevType &d : ht) d.cpot = -1;
    for (int a = 0; a < (int)types.size(); ++a) {
        DevType &d = ht[a];
        memset(&d, 0, sizeof(d));
        d.imass = types[a].imass;
        d.mass = types[a].mass;
        d.radius = (float)types[a].radius;
        d.dynamics = types[a].dynamics;
        d.flags = types[a].flags;
        d.fx = types[a].force[0];
        d.fy = types[a].force[1];
        d.fz = types[a].force[2];
        d.has_force = types[a].has_force ? 1 : 0;
        const TypeInfo &ti = types[a];
        d.sb_kind = ti.sb_kind;
        d.target = ti.target;
        if (ti.sb_kind == 2) {
            d.sb_a = 1 / ti.sb[0];  // berenderson_create keeps 1/tau (MxForce.cpp:388-395)
        } else if (ti.sb_kind == 3 || ti.sb_kind == 4) {
            d.sb_a = ti.sb[0];
            d.sb_b = ti.sb[1];
            d.sb_c = ti.sb[2];
            const float dur = ti.sb_kind == 3 ? ti.sb[2] : ti.sb[3];
            d.sb_steps = std::max(1, (int)std::ceil(dur / dt));  // durration_steps (MxForce.cpp:403,417)
        }
        if (ti.sb_kind) has_sb = true;
        if (is_large[a]) {
            d.large = 1;
            d.flags |= (1u << 2) | (1u << 3) | (1u << 4);  // never integrated (not in any cell of the reference)
        }
        d.cpot = is_large[a] ? -1 : ti.cpot;
        if (d.cpot >= 0 && !cuboids.empty()) has_cuboid_forces = true;
        const unsigned face_bits[6] = {kCellActiveLeft, kCellActiveRight, kCellActiveFront,
                                       kCellActiveBack, kCellActiveBottom, kCellActiveTop};
        for (int f = 0; f < 6; ++f) {
            d.bpot[f] = ti.bpot[f];
            if (ti.bpot[f] >= 0) {
                d.wall_mask |= face_bits[f];
                has_walls = true;
            }
        }
    }
    std::vector<SortAxes> haxes(1);
    for (int q = 0; q < 13; ++q)
        for (int k = 0; k < 3; ++k) haxes[0].n[q][k] = (float)kCellShift[q][k];

    // ---- bonds: CSR by particle id ----
    std::vector<DevBond> hb;
    std::vector<unsigned> hbf;
    std::vector<int> boff(nparts + 1, 0), blist;
    for (const BondInfo &b : bonds) {
        if (b.i < 0 || b.i >= nparts || b.j < 0 || b.j >= nparts) return MXG_ERR_BOND;
        if (prep[b.i] != prep[b.j]) return MXG_ERR_BOND;  // a bond cannot span two replicas
        boff[b.i + 1]++;
        if (b.j != b.i) boff[b.j + 1]++;
    }
    for (int p = 0; p < nparts; ++p) boff[p + 1] += boff[p];
    blist.assign(boff[nparts], 0);
    {
        std::vector<int> fill(boff.begin(), boff.end() - 1);
        for (int k = 0; k < (int)bonds.size(); ++k) {
            blist[fill[bonds[k].i]++] = k;
            if (bonds[k].j != bonds[k].i) blist[fill[bonds[k].j]++] = k;
            DevBond d;
            memset(&d, 0, sizeof(d));
            d.i = bonds[k].i;
            d.j = bonds[k].j;
            d.pot = bonds[k].pot;
            d.dissociation = bonds[k].dissociation;
            hb.push_back(d);
            hbf.push_back(1u);
        }
    }

    // ---- exclusions: CSR by particle id, entries exclusion * 2 + role ----
    std::vector<int2> hx;
    std::vector<int> xoff(nparts + 1, 0), xlist;
    for (const ExclusionInfo &x : exclusions) {
        if (x.i < 0 || x.j >= nparts || prep[x.i] != prep[x.j]) return MXG_ERR_BOND;
        xoff[x.i + 1]++;
        if (x.j != x.i) xoff[x.j + 1]++;
    }
    for (int p = 0; p < nparts; ++p) xoff[p + 1] += xoff[p];
    xlist.assign(xoff[nparts], 0);
    {
        std::vector<int> fill(xoff.begin(), xoff.end() - 1);
        for (int k = 0; k < (int)exclusions.size(); ++k) {
            xlist[fill[exclusions[k].i]++] = 2 * k;
            if (exclusions[k].j != exclusions[k].i) xlist[fill[exclusions[k].j]++] = 2 * k + 1;
            hx.push_back(make_int2(exclusions[k].i, exclusions[k].j));
        }
    }

    // ---- angles: CSR by particle id, entries angle * 4 + role ----
    std::vector<DevAngle> ha;
    std::vector<int> aoff(nparts + 1, 0), alist;
    for (const AngleInfo &a : angles) {
        const int ids[3] = {a.i, a.j, a.k};
        for (int r = 0; r < 3; ++r)
            if (ids[r] < 0 || ids[r] >= nparts) return MXG_ERR_BOND;
        if (prep[a.i] != prep[a.j] || prep[a.k] != prep[a.j]) return MXG_ERR_BOND;
        for (int r = 0; r < 3; ++r) aoff[ids[r] + 1]++;
    }
    for (int p = 0; p < nparts; ++p) aoff[p + 1] += aoff[p];
    alist.assign(aoff[nparts], 0);
    {
        std::vector<int> fill(aoff.begin(), aoff.end() - 1);
        for (int k = 0; k < (int)angles.size(); ++k) {
            const int ids[3] = {angles[k].i, angles[k].j, angles[k].k};
            for (int r = 0; r < 3; ++r) alist[fill[ids[r]]++] = k * 4 + r;
            ha.push_back({angles[k].i, angles[k].j, angles[k].k, angles[k].pot});
        }
    }

    // ---- dihedrals: CSR by particle id, entries dihedral * 4 + role ----
    std::vector<DevDihedral> hd;
    std::vector<int> doff(nparts + 1, 0), dlist;
    for (const DihedralInfo &d : dihedrals) {
        const int ids[4] = {d.i, d.j, d.k, d.l};
        for (int r = 0; r < 4; ++r) {
            if (ids[r] < 0 || ids[r] >= nparts) return MXG_ERR_BOND;
            if (prep[ids[r]] != prep[d.j]) return MXG_ERR_BOND;
        }
        for (int r = 0; r < 4; ++r) doff[ids[r] + 1]++;
    }
    for (int p = 0; p < nparts; ++p) doff[p + 1] += doff[p];
    dlist.assign(doff[nparts], 0);
    {
        std::vector<int> fill(doff.begin(), doff.end() - 1);
        for (int k = 0; k < (int)dihedrals.size(); ++k) {
            const DihedralInfo &d = dihedrals[k];
            const int ids[4] = {d.i, d.j, d.k, d.l};
            for (int r = 0; r < 4; ++r) dlist[fill[ids[r]]++] = k * 4 + r;
            DevDihedral dd;
            memset(&dd, 0, sizeof(dd));
            dd.i = d.i;
            dd.j = d.j;
            dd.k = d.k;
            dd.l = d.l;
            dd.pot = d.pot;
            hd.push_back(dd);
        }
    }

    // ---- device allocation ----
    rc = MXG_OK;
    for (int b = 0; b < 2; ++b) {
        rc |= alloc(&d_pos[b], nparts);
        rc |= alloc(&d_vel[b], nparts);
        rc |= alloc(&d_cell_of[b], nparts);
        rc |= alloc(&d_cell_start[b], ncells + 1);
        rc |= alloc(&d_cell_count[b], ncells);
    }
    rc |= alloc(&d_force, nparts);
    if (integrator == 1)
        for (int k = 0; k < 5; ++k) rc |= alloc(&d_rk[k], nparts);
    rc |= alloc(&d_new_cell, nparts);
    nchunks = (ncells + (1 << kChunkShift) - 1) >> kChunkShift;
    for (int p = 0; p < 2; ++p) {
        rc |= alloc(&d_in_count[p], ncells);
        rc |= alloc(&d_out_count[p], ncells);
        rc |= alloc(&d_chunk_delta[p], nchunks);
    }
    rc |= alloc(&d_in_list, (size_t)ncells * kBucket);
    rc |= alloc(&d_ovf_list, (size_t)nparts);
    rc |= alloc(&d_ovf_count, 1);
    rc |= alloc(&d_rebin_ctl, 1);
    rc |= alloc(&d_slot_of_id, nparts);
    rc |= alloc(&d_cell_rep, ncells);
    rc |= alloc(&d_cell_flags, ncells);
    rc |= alloc(&d_nb_off, ncells + 1);
    rc |= alloc(&d_nb_cell, nb_cell.size());
    rc |= alloc(&d_nb_shift, nb_shift.size());
    rc |= alloc(&d_nb_rev, nb_rev.size());
    rc |= alloc(&d_sec_count, ncells);
    rc |= alloc(&d_cell_planes, ncells);
    rc |= alloc(&d_items, hitems.size());
    rc |= alloc(&d_item_ctr, 2);
    rc |= alloc(&d_item_order, hitems.size());
    rc |= alloc(&d_planes, (size_t)nplanes * nparts);
    rc |= alloc(&d_pots, hp.size());
    rc |= alloc(&d_coef, coef.size() + 8);
    rc |= alloc(&d_pot_idx, hpidx.size());
    rc |= alloc(&d_pot_idx2, hpidx2.size());
    rc |= alloc(&d_dpd_pair, hdpd.size());
    std::vector<DevCuboid> hcub;
    for (const CuboidInfo &ci : cuboids) {
        DevCuboid d;
        memset(&d, 0, sizeof(d));
        for (int k = 0; k < 3; ++k) {
            d.pos[k] = ci.pos[k];
            d.size[k] = ci.size[k];
            d.lo[k] = ci.lo[k];
            d.hi[k] = ci.hi[k];
        }
        for (int k = 0; k < 4; ++k) {
            d.q[k] = ci.q[k];
            d.qi[k] = ci.qi[k];
        }
        d.rep = ci.rep;
        hcub.push_back(d);
    }
    rc |= alloc(&d_cuboids, hcub.size());
    rc |= alloc(&d_types, ht.size());
    rc |= alloc(&d_type_ke, ht.size());
    rc |= alloc(&d_persist, (size_t)nparts);
    rc |= alloc(&d_spaces, hs.size());
    rc |= alloc(&d_axes, 1);
    rc |= alloc(&d_sort_bounds, (size_t)ncells * 13);
    rc |= alloc(&d_epot_cell, nitems);
    rc |= alloc(&d_ebond_slot, nparts);
    rc |= alloc(&d_body_e, nparts);
    rc |= alloc(&d_body_f, nparts);
    rc |= alloc(&d_spec, (size_t)nparts * smax);
    rc |= alloc(&d_rate, (size_t)nparts * smax);
    rc |= alloc(&d_nspec, hnspec.size());
    rc |= alloc(&d_sflags, hsflags.size());
    rc |= alloc(&d_flux_off, hfoff.size());
    rc |= alloc(&d_flux, hflux.size());
    rc |= alloc(&d_fx_off, fx_off.size());
    rc |= alloc(&d_fx_cell, fx_cell.size());
    rc |= alloc(&d_fx_shift, fx_shift.size());
    rc |= alloc(&d_large_x, hlx.size());
    rc |= alloc(&d_large_v, hlv.size());
    rc |= alloc(&d_large_rep, hlrep.size());
    rc |= alloc(&d_large_pot, hlpot.size());
    rc |= alloc(&d_bonds, hb.size());
    rc |= alloc(&d_bond_flags, hbf.size());
    rc |= alloc(&d_bond_off, boff.size());
    rc |= alloc(&d_bond_list, blist.size());
    rc |= alloc(&d_excl, hx.size());
    rc |= alloc(&d_excl_off, xoff.size());
    rc |= alloc(&d_excl_list, xlist.size());
    rc |= alloc(&d_angles, ha.size());
    rc |= alloc(&d_angle_off, aoff.size());
    rc |= alloc(&d_angle_list, alist.size());
    rc |= alloc(&d_dihedrals, hd.size());
    rc |= alloc(&d_dihedral_off, doff.size());
    rc |= alloc(&d_dihedral_list, dlist.size());
    rc |= alloc(&d_status, 1);
    rc |= alloc(&d_step, 1);
    rc |= alloc(&d_partials, 2 * (size_t)energy_blocks);
    rc |= alloc(&d_energy, 2);
    if (rc != MXG_OK) return MXG_ERR_MALLOC;

    for (int p = 0; p < 2; ++p) {
        CUDA_TRY(cudaMemsetAsync(d_in_count[p], 0, sizeof(int) * ncells, stream));
        CUDA_TRY(cudaMemsetAsync(d_out_count[p], 0, sizeof(int) * ncells, stream));
        CUDA_TRY(cudaMemsetAsync(d_chunk_delta[p], 0, sizeof(int) * nchunks, stream));
    }
    CUDA_TRY(cudaMemsetAsync(d_ovf_count, 0, sizeof(int), stream));
    CUDA_TRY(cudaMemsetAsync(d_rebin_ctl, 0, sizeof(unsigned), stream));
    CUDA_TRY(cudaMemsetAsync(d_status, 0, sizeof(unsigned), stream));
    CUDA_TRY(cudaMemsetAsync(d_step, 0, sizeof(unsigned long long), stream));
    CUDA_TRY(cudaMemsetAsync(d_item_ctr, 0, 2 * sizeof(int), stream));
    CUDA_TRY(cudaMemsetAsync(d_epot_cell, 0, sizeof(double) * std::max(1, nitems), stream));
    CUDA_TRY(cudaMemsetAsync(d_ebond_slot, 0, sizeof(double) * std::max(1, nparts), stream));
    CUDA_TRY(cudaMemsetAsync(d_body_e, 0, sizeof(double) * std::max(1, nparts), stream));
    if (smax > 0) CUDA_TRY(cudaMemsetAsync(d_rate, 0, sizeof(float) * (size_t)nparts * smax, stream));
    CUDA_TRY(cudaMemsetAsync(d_force, 0, sizeof(float4) * std::max(1, nparts), stream));
    CUDA_TRY(cudaMemsetAsync(d_persist, 0, sizeof(float4) * std::max(1, nparts), stream));
    CUDA_TRY(cudaMemsetAsync(d_type_ke, 0, sizeof(double) * ht.size(), stream));
    if ((rc = upload(d_pos[0], hpos, stream)) || (rc = upload(d_vel[0], hvel, stream)) ||
        (rc = upload(d_cell_of[0], hcell_of, stream)) || (rc = upload(d_cell_start[0], hstart, stream)) ||
        (rc = upload(d_cell_count[0], hcount, stream)) || (rc = upload(d_slot_of_id, hslot, stream)) ||
        (rc = upload(d_cell_rep, hrep, stream)) || (rc = upload(d_cell_flags, hcflags, stream)) ||
        (rc = upload(d_nb_off, nb_off, stream)) || (rc = upload(d_nb_cell, nb_cell, stream)) ||
        (rc = upload(d_nb_shift, nb_shift, stream)) || (rc = upload(d_nb_rev, nb_rev, stream)) ||
        (rc = upload(d_sec_count, hsec, stream)) || (rc = upload(d_cell_planes, hplanes, stream)) ||
        (rc = upload(d_items, hitems, stream)) || (rc = upload(d_pots, hp, stream)) ||
        (rc = upload(d_coef, coef, stream)) || (rc = upload(d_pot_idx, hpidx, stream)) ||
        (rc = upload(d_pot_idx2, hpidx2, stream)) || (rc = upload(d_dpd_pair, hdpd, stream)) ||
        (rc = upload(d_cuboids, hcub, stream)) ||
        (rc = upload(d_types, ht, stream)) || (rc = upload(d_spaces, hs, stream)) || (rc = upload(d_axes, haxes, stream)) ||
        (rc = upload(d_bonds, hb, stream)) || (rc = upload(d_bond_flags, hbf, stream)) ||
        (rc = upload(d_bond_off, boff, stream)) || (rc = upload(d_bond_list, blist, stream)) ||
        (rc = upload(d_excl, hx, stream)) || (rc = upload(d_excl_off, xoff, stream)) ||
        (rc = upload(d_excl_list, xlist, stream)) || (rc = upload(d_angles, ha, stream)) || (rc = upload(d_angle_off, aoff, stream)) ||
        (rc = upload(d_angle_list, alist, stream)) || (rc = upload(d_dihedrals, hd, stream)) ||
        (rc = upload(d_large_x, hlx, stream)) || (rc = upload(d_large_v, hlv, stream)) ||
        (rc = upload(d_spec, spec_host, stream)) || (rc = upload(d_nspec, hnspec, stream)) ||
        (rc = upload(d_sflags, hsflags, stream)) || (rc = upload(d_flux_off, hfoff, stream)) ||
        (rc = upload(d_flux, hflux, stream)) || (rc = upload(d_fx_off, fx_off, stream)) ||
        (rc = upload(d_fx_cell, fx_cell, stream)) || (rc = upload(d_fx_shift, fx_shift, stream)) ||
        (rc = upload(d_large_rep, hlrep, stream)) || (rc = upload(d_large_pot, hlpot, stream)) ||
        (rc = upload(d_dihedral_off, doff, stream)) || (rc = upload(d_dihedral_list, dlist, stream)))
        return rc;
    CUDA_TRY(cudaStreamSynchronize(stream));

    configure_force_kernels();
    force_grid = std::max(1, std::min((nitems + kWarpsPerBlock - 1) / kWarpsPerBlock, num_sms * 16));
    cur = 0;
    started = true;
    refresh_bounds();
    return build_graphs();
}

int mxg_engine::build_graphs() {
    for (int k = 0; k < 2; ++k)
        if (graph[k]) {
            cudaGraphExecDestroy(graph[k]);
            graph[k] = nullptr;
        }
    if (use_graphs && nparts > 0) {
        for (int b = 0; b < 2; ++b) {
            cudaGraph_t g;
            CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            enqueue_step(b);
            CUDA_TRY(cudaStreamEndCapture(stream, &g));
            CUDA_TRY(cudaGraphInstantiate(&graph[b], g, 0));
            cudaGraphDestroy(g);
        }
    }
    return MXG_OK;
}

/* Re-places all particles from global positions (per id) and velocities (per id, or the
 * current ones when v is null), on the device: the host arrays are copied once and the
 * placement, counting, scan and (cell, id) ordering run as kernels with the host
 * placement's arithmetic. A particle outside its box leaves the state unchanged and returns
 * MXG_ERR_SPACE. */
int mxg_engine::load_state(const double *x, const float *v, int n) {
    if (n != nparts) return MXG_ERR_ARG;
    if (nparts == 0) return MXG_OK;
    if (!h_ld_err && cudaMallocHost((void **)&h_ld_err, sizeof(int)) != cudaSuccess) {
        h_ld_err = nullptr;
        return MXG_ERR_MALLOC;
    }
    if (!d_ld_x) {
        int rc = alloc(&d_ld_x, 3 * (size_t)nparts);
        rc |= alloc(&d_ld_v, 3 * (size_t)nparts);
        rc |= alloc(&d_ld_xr, (size_t)nparts);
        rc |= alloc(&d_ld_vel, (size_t)nparts);
        rc |= alloc(&d_ld_cell, (size_t)nparts);
        rc |= alloc(&d_ld_ids, (size_t)nparts);
        rc |= alloc(&d_ld_count, (size_t)ncells);
        rc |= alloc(&d_ld_fill, (size_t)ncells);
        rc |= alloc(&d_ld_err, 1);
        rc |= alloc(&d_type_of_id, (size_t)nparts);
        rc |= alloc(&d_rep_of_id, (size_t)nparts);
        if (rc != MXG_OK) return MXG_ERR_MALLOC;
        if ((rc = upload(d_type_of_id, ptype, stream)) || (rc = upload(d_rep_of_id, prep, stream))) return rc;
    }
    if (v && !ld_stream) {
        CUDA_TRY(cudaStreamCreateWithFlags(&ld_stream, cudaStreamNonBlocking));
        CUDA_TRY(cudaEventCreateWithFlags(&ld_x_done, cudaEventDisableTiming));
        CUDA_TRY(cudaEventCreateWithFlags(&ld_v_done, cudaEventDisableTiming));
    }
    CUDA_TRY(cudaMemsetAsync(d_ld_count, 0, sizeof(int) * (size_t)ncells, stream));
    CUDA_TRY(cudaMemsetAsync(d_ld_fill, 0, sizeof(int) * (size_t)ncells, stream));
    CUDA_TRY(cudaMemsetAsync(d_ld_err, 0, sizeof(int), stream));
    CUDA_TRY(cudaMemcpyAsync(d_ld_x, x, sizeof(double) * 3 * (size_t)n, cudaMemcpyHostToDevice, stream));
    if (v) {
        // the velocities cross after the positions, on a second stream, while the placement,
        // the scan, the fill and the ordering (which need only the positions) run; only the
        // launch that writes the velocities into their slots waits for them
        CUDA_TRY(cudaEventRecord(ld_x_done, stream));
        CUDA_TRY(cudaStreamWaitEvent(ld_stream, ld_x_done, 0));
        CUDA_TRY(cudaMemcpyAsync(d_ld_v, v, sizeof(float) * 3 * (size_t)n, cudaMemcpyHostToDevice, ld_stream));
        CUDA_TRY(cudaEventRecord(ld_v_done, ld_stream));
    }
    LoadView ld;
    ld.x = d_ld_x;
    ld.v = v ? d_ld_v : nullptr;
    ld.type_of_id = d_type_of_id;
    ld.rep_of_id = d_rep_of_id;
    ld.xr = d_ld_xr;
    ld.vel = d_ld_vel;
    ld.cell = d_ld_cell;
    ld.fill = d_ld_fill;
    ld.ids = d_ld_ids;
    ld.err = d_ld_err;
    ld.slot_now = d_slot_of_id;
    ld.n = n;
    const EngineView ev = view(cur);
    launch_load_place(ev, ld, d_ld_count, stream);
    // the ordering launches write nothing when a particle lay outside its box, so one
    // synchronisation at the end reports the error with the engine's state untouched
    launch_load_order(ev, ld, d_ld_count, d_cell_start[cur], d_cell_count[cur], d_pos[cur], d_vel[cur],
                      d_cell_of[cur], d_slot_of_id, v ? ld_v_done : nullptr, stream);
    CUDA_TRY(cudaMemcpyAsync(h_ld_err, d_ld_err, sizeof(int), cudaMemcpyDeviceToHost, stream));
    CUDA_TRY(cudaStreamSynchronize(stream));  // also: the caller's host arrays are free again
    CUDA_TRY(cudaGetLastError());
    return *h_ld_err ? MXG_ERR_SPACE : MXG_OK;
}

/* ======================================================================== */
/* C ABI                                                                     */
/* ======================================================================== */

extern "C" {

static int wrap_potential(int rc, mxg_potential *p, mxg_potential **out) {
    if (rc != 0) {
        delete p;
        *out = nullptr;
        return MXG_ERR_POTENTIAL;
    }
    *out = p;
    return MXG_OK;
}

int mxg_potential_create_lj126(double a, double b, double A, double B, double tol, mxg_potential **out) {
    if (!out) return MXG_ERR_NULL;
    if (!(a > 0) || !(b > a) || !(tol > 0)) return MXG_ERR_ARG;
    mxg_potential *p = new mxg_potential;
    return wrap_potential(make_lj126(p->t, a, b, A, B, tol), p, out);
}

int mxg_potential_create_morse(double d, double alpha, double r0, double min, double max, double tol,
                               mxg_potential **out) {
    if (!out) return MXG_ERR_NULL;
    if (!(max > min) || !(tol > 0)) return MXG_ERR_ARG;
    mxg_potential *p = new mxg_potential;
    return wrap_potential(make_morse(p->t, d, alpha, r0, min, max, tol), p, out);
}

int mxg_potential_create_harmonic(double k, double r0, double min, double max, double tol, mxg_potential **out) {
    if (!out) return MXG_ERR_NULL;
    if (!(max > min) || !(tol > 0)) return MXG_ERR_ARG;
    mxg_potential *p = new mxg_potential;
    return wrap_potential(make_harmonic(p->t, k, r0, min, max, tol), p, out);
}

int mxg_potential_create_harmonic_angle(double k, double theta0, double min, double max, double tol,
                                       mxg_potential **out) {
    if (!out) return MXG_ERR_NULL;
    if (!(max > min) || !(tol > 0)) return MXG_ERR_ARG;
    mxg_potential *p = new mxg_potential;
    return wrap_potential(make_harmonic_angle(p->t, k, theta0, min, max, tol), p, out);
}

int mxg_potential_create_harmonic_dihedral(double k, int n, double delta, double tol, mxg_potential **out) {
    if (!out) return MXG_ERR_NULL;
    if (n < 1 || !(tol > 0)) return MXG_ERR_ARG;
    mxg_potential *p = new mxg_potential;
    return wrap_potential(make_harmonic_dihedral(p->t, k, n, delta, tol), p, out);
}

int mxg_potential_create_power(double k, double r0, double alpha, double min, double max, double tol,
                               mxg_potential **out) {
    if (!out) return MXG_ERR_NULL;
    if (!(max > min) || !(tol > 0)) return MXG_ERR_ARG;
    mxg_potential *p = new mxg_potential;
    return wrap_potential(make_power(p->t, k, r0, alpha, min, max, tol), p, out);
}

int mxg_potential_create_dpd(double alpha, double gamma, double sigma, double cutoff, int shifted,
                             mxg_potential **out) {
    if (!out) return MXG_ERR_NULL;
    if (!(cutoff > 0)) return MXG_ERR_ARG;
    mxg_potential *p = new mxg_potential;
    return wrap_potential(make_dpd(p->t, alpha, gamma, sigma, cutoff, shifted != 0), p, out);
}

int mxg_potential_info(const mxg_potential *p, int *kind, unsigned *flags, int *n, float *alpha4, float *a, float *b,
                       float *r0_plusone) {
    if (!p) return MXG_ERR_NULL;
    if (kind) *kind = p->t.kind;
    if (flags) *flags = p->t.flags;
    if (n) *n = p->t.n;
    if (alpha4)
        for (int k = 0; k < 4; ++k) alpha4[k] = p->t.alpha[k];
    if (a) *a = p->t.a;
    if (b) *b = p->t.b;
    if (r0_plusone) *r0_plusone = p->t.r0_plusone;
    return MXG_OK;
}

int mxg_potential_coeffs(const mxg_potential *p, float *out, int cap) {
    if (!p) return MXG_ERR_NULL;
    const int len = (int)p->t.c.size();
    if (cap < len) return -len;
    if (len) memcpy(out, p->t.c.data(), sizeof(float) * len);
    return len;
}

int mxg_potential_dpd_params(const mxg_potential *p, float *alpha, float *gamma, float *sigma) {
    if (!p) return MXG_ERR_NULL;
    if (p->t.kind != kKindDPD) return MXG_ERR_POTENTIAL;
    *alpha = p->t.dpd_alpha;
    *gamma = p->t.dpd_gamma;
    *sigma = p->t.dpd_sigma;
    return MXG_OK;
}

int mxg_potential_eval(const mxg_potential *p, float ri, float rj, float r2, float *e, float *f) {
    if (!p || !e || !f) return MXG_ERR_NULL;
    if (p->t.kind != kKindTable) return MXG_ERR_POTENTIAL;
    return eval_ex(p->t, ri, rj, r2, e, f) ? 1 : 0;
}

void mxg_potential_free(mxg_potential *p) { delete p; }

int mxg_engine_init(const double *origin, const double *dim, const int *cells, double cutoff, const int *bc_kind,
                    const float *bc_velocity, const float *bc_restore, int max_type, unsigned flags,
                    mxg_engine **out) {
    (void)flags;
    if (!origin || !dim || !cells || !out) return MXG_ERR_NULL;
    if (!(cutoff > 0) || max_type <= 0 || max_type > kMaxTypes) return MXG_ERR_ARG;
    mxg_engine *e = new mxg_engine;
    e->cutoff = cutoff;
    e->max_type = max_type;
    const int rc = mxg_engine_add_replica(e, origin, dim, cells, bc_kind, bc_velocity, bc_restore);
    if (rc < 0) {
        delete e;
        return rc;
    }
    *out = e;
    return MXG_OK;
}

int mxg_engine_add_replica(mxg_engine *e, const double *origin, const double *dim, const int *cells,
                           const int *bc_kind, const float *bc_velocity, const float *bc_restore) {
    if (!e || !origin || !dim || !cells) return MXG_ERR_NULL;
    if (e->started) return MXG_ERR_STATE;
    Space sp;
    int rc = sp.configure(origin, dim, cells, bc_kind, bc_velocity, bc_restore);
    if (rc != MXG_OK) return rc;
    if ((rc = sp.build(e->cutoff)) != MXG_OK) return rc;
    sp.cell_offset = e->ncells;
    sp.pot_idx.assign((size_t)e->max_type * e->max_type, -1);
    sp.pot2_idx.assign((size_t)e->max_type * e->max_type, -1);
    e->ncells += sp.ncells;
    e->spaces.push_back(std::move(sp));
    return (int)e->spaces.size() - 1;
}

int mxg_engine_nr_replicas(const mxg_engine *e) { return e ? (int)e->spaces.size() : MXG_ERR_NULL; }

int mxg_engine_set_dt(mxg_engine *e, double dt, double max_dist_fraction) {
    if (!e) return MXG_ERR_NULL;
    if (e->started) return MXG_ERR_STATE;
    if (!(dt > 0)) return MXG_ERR_ARG;
    e->dt = dt;
    if (max_dist_fraction > 0) e->max_dist_fraction = (float)max_dist_fraction;
    return MXG_OK;
}

int mxg_engine_set_rng_mode(mxg_engine *e, int mode) {
    if (!e) return MXG_ERR_NULL;
    if (e->started) return MXG_ERR_STATE;
    e->rng_mode = mode ? 1u : 0u;
    return MXG_OK;
}

int mxg_engine_set_pair_pruning(mxg_engine *e, int mode) {
    if (!e) return MXG_ERR_NULL;
    if (e->started) return MXG_ERR_STATE;
    if (mode < 0 || mode > 2) return MXG_ERR_ARG;
    e->pruning = mode;
    return MXG_OK;
}

int mxg_engine_addtype(mxg_engine *e, double mass, double radius, int dynamics, unsigned particle_flags) {
    if (!e) return MXG_ERR_NULL;
    if (e->started) return MXG_ERR_STATE;
    if ((int)e->types.size() >= e->max_type) return MXG_ERR_RANGE;
    if (!(mass > 0)) return MXG_ERR_ARG;
    TypeInfo t;
    t.mass = mass;
    t.imass = 1.0 / mass;
    t.radius = radius;
    t.dynamics = dynamics;
    t.flags = particle_flags;
    t.force[0] = t.force[1] = t.force[2] = 0.f;
    t.has_force = false;
    e->types.push_back(t);
    return (int)e->types.size() - 1;
}

int mxg_engine_addpot_replica(mxg_engine *e, int rep, const mxg_potential *p, int i, int j) {
    if (!e || !p) return MXG_ERR_NULL;
    if (e->started) return MXG_ERR_STATE;
    const int nt = (int)e->types.size();
    if (i < 0 || i >= nt || j < 0 || j >= nt || rep < 0 || rep >= (int)e->spaces.size()) return MXG_ERR_RANGE;
    e->pots.push_back(p->t);
    const int idx = (int)e->pots.size() - 1;
    std::vector<int> &m = e->spaces[rep].pot_idx;
    m[i * e->max_type + j] = idx;  // engine_addpot overwrites: one potential per pair
    m[j * e->max_type + i] = idx;
    return MXG_OK;
}

namespace {
/* New construction parameters for a potential: a frozen-node re-fit for tables;
 * for DPD the three coefficients (the cutoff and the shift flag stay). */
int set_params(mxg::PotentialTable &t, const double *params, int nparams) {
    if (nparams != (int)t.params.size()) return MXG_ERR_ARG;
    if (t.kind == kKindDPD) {
        if (params[3] != t.params[3] || params[4] != t.params[4]) return MXG_ERR_ARG;
        t.dpd_alpha = (float)params[0];
        t.dpd_gamma = (float)params[1];
        t.dpd_sigma = (float)params[2];
        t.params.assign(params, params + nparams);
        return MXG_OK;
    }
    std::vector<double> q(params, params + nparams);
    return mxg::refit_frozen(t, q) == 0 ? MXG_OK : MXG_ERR_ARG;
}
}  // namespace

int mxg_potential_coeffs64(const mxg_potential *p, double *out, int cap) {
    if (!p || !out) return MXG_ERR_NULL;
    const int n = (int)p->t.c64.size();
    for (int k = 0; k < n && k < cap; ++k) out[k] = p->t.c64[k];
    return n;
}

int mxg_potential_params(const mxg_potential *p, double *out, int cap) {
    if (!p) return MXG_ERR_NULL;
    const int n = (int)p->t.params.size();
    for (int k = 0; k < n && k < cap && out; ++k) out[k] = p->t.params[k];
    return n;
}

int mxg_potential_refit(mxg_potential *p, const double *params, int nparams) {
    if (!p || !params) return MXG_ERR_NULL;
    return set_params(p->t, params, nparams);
}

int mxg_potential_param_table(const mxg_potential *p, int k, mxg_potential **out) {
    if (!p || !out) return MXG_ERR_NULL;
    mxg_potential *q = new mxg_potential;
    if (mxg::param_derivative_table(p->t, k, q->t) != 0) {
        delete q;
        return MXG_ERR_ARG;
    }
    *out = q;
    return MXG_OK;
}

int mxg_engine_add_singlebody_force_kind(mxg_engine *e, int type, int kind, const float *params) {
    if (!e || !params) return MXG_ERR_NULL;
    if (e->started) return MXG_ERR_STATE;
    if (type < 0 || type >= (int)e->types.size()) return MXG_ERR_RANGE;
    if (kind < 2 || kind > 4) return MXG_ERR_ARG;
    if (kind == 2 && !(params[0] != 0.f)) return MXG_ERR_ARG;
    TypeInfo &t = e->types[type];
    t.has_force = false;  // engine_add_singlebody_force keeps one force per type
    t.sb_kind = kind;
    for (int k = 0; k < 4; ++k) t.sb[k] = params[k];
    return MXG_OK;
}

int mxg_engine_set_target_temperature(mxg_engine *e, int type, double temperature) {
    if (!e) return MXG_ERR_NULL;
    if (e->started) return MXG_ERR_STATE;
    if (type < 0 || type >= (int)e->types.size()) return MXG_ERR_RANGE;
    e->types[type].target = temperature;
    return MXG_OK;
}

int mxg_engine_set_integrator(mxg_engine *e, int kind) {
    if (!e) return MXG_ERR_NULL;
    if (kind != 0 && kind != 1) return MXG_ERR_ARG;
    if (e->started) return MXG_ERR_STATE;
    e->integrator = kind;
    return MXG_OK;
}

int mxg_engine_addpot_second(mxg_engine *e, int rep, const mxg_potential *p, int i, int j) {
    if (!e || !p) return MXG_ERR_NULL;
    if (e->started) return MXG_ERR_STATE;
    const int nt = (int)e->types.size();
    if (i < 0 || i >= nt || j < 0 || j >= nt || rep < 0 || rep >= (int)e->spaces.size()) return MXG_ERR_RANGE;
    e->pots.push_back(p->t);
    const int idx = (int)e->pots.size() - 1;
    std::vector<int> &m = e->spaces[rep].pot2_idx;
    m[i * e->max_type + j] = idx;
    m[j * e->max_type + i] = idx;
    return MXG_OK;
}

int mxg_engine_pot_index(mxg_engine *e, int rep, int i, int j, int which, int *idx) {
    if (!e || !idx) return MXG_ERR_NULL;
    const int nt = (int)e->types.size();
    if (i < 0 || i >= nt || j < 0 || j >= nt || rep < 0 || rep >= (int)e->spaces.size() || which < 0 || which > 1)
        return MXG_ERR_RANGE;
    const std::vector<int> &m = which == 0 ? e->spaces[rep].pot_idx : e->spaces[rep].pot2_idx;
    *idx = m[i * e->max_type + j];
    return MXG_OK;
}

int mxg_engine_set_pot_params(mxg_engine *e, int idx, const double *params, int nparams) {
    if (!e || !params) return MXG_ERR_NULL;
    if (idx < 0 || idx >= (int)e->pots.size()) return MXG_ERR_RANGE;
    int rc = set_params(e->pots[idx], params, nparams);
    e->adjoint_stale = true;  // dV/dtheta tables depend on the parameters
    if (rc != MXG_OK || !e->started) return rc;
    std::vector<DevPot> hp;
    std::vector<float> coef;
    e->pot_arrays(hp, coef);  // same sizes: a frozen-node refit keeps every table's length
    const std::vector<float4> hdpd = e->dpd_records(hp);
    if ((rc = upload(e->d_pots, hp, e->stream)) || (rc = upload(e->d_coef, coef, e->stream)) ||
        (rc = upload(e->d_dpd_pair, hdpd, e->stream)))
        return rc;
    CUDA_TRY(cudaStreamSynchronize(e->stream));  // the host vectors go out of scope
    return MXG_OK;
}

int mxg_engine_addpot(mxg_engine *e, const mxg_potential *p, int i, int j) {
    return mxg_engine_addpot_replica(e, 0, p, i, j);
}

int mxg_engine_add_singlebody_force(mxg_engine *e, int type, float fx, float fy, float fz) {
    if (!e) return MXG_ERR_NULL;
    if (e->started) return MXG_ERR_STATE;
    if (type < 0 || type >= (int)e->types.size()) return MXG_ERR_RANGE;
    TypeInfo &t = e->types[type];
    t.sb_kind = 0;  // one single-body force per type
    t.force[0] = fx;
    t.force[1] = fy;
    t.force[2] = fz;
    t.has_force = true;
    return MXG_OK;
}

int mxg_engine_addparts_replica(mxg_engine *e, int rep, int n, const double *x, const float *v, const int *type,
                                int *ids_out) {
    if (!e || (n > 0 && (!x || !type))) return MXG_ERR_NULL;
    if (e->started) return MXG_ERR_STATE;
    if (rep < 0 || rep >= (int)e->spaces.size()) return MXG_ERR_RANGE;
    const Space &sp = e->spaces[rep];
    for (int k = 0; k < n; ++k) {
        if (type[k] < 0 || type[k] >= (int)e->types.size()) return MXG_ERR_RANGE;
        int cell;
        float xr[3];
        if (sp.place(&x[3 * (size_t)k], cell, xr) != MXG_OK) return MXG_ERR_SPACE;
    }
    const int first = (int)e->ptype.size();
    for (int k = 0; k < n; ++k) {
        for (int q = 0; q < 3; ++q) {
            e->px.push_back(x[3 * (size_t)k + q]);
            e->pv.push_back(v ? v[3 * (size_t)k + q] : 0.f);
        }
        e->ptype.push_back(type[k]);
        e->prep.push_back(rep);
        e->pcell.push_back(-1);
        for (int q = 0; q < 3; ++q) e->pxr.push_back(0.f);
        if (ids_out) ids_out[k] = first + k;
    }
    return MXG_OK;
}

int mxg_engine_addparts_cellrel(mxg_engine *e, int rep, int n, const int *cell, const float *xrel, const float *v,
                                const int *type, int *ids_out) {
    if (!e || (n > 0 && (!cell || !xrel || !type))) return MXG_ERR_NULL;
    if (e->started) return MXG_ERR_STATE;
    if (rep < 0 || rep >= (int)e->spaces.size()) return MXG_ERR_RANGE;
    const Space &sp = e->spaces[rep];
    for (int k = 0; k < n; ++k) {
        if (type[k] < 0 || type[k] >= (int)e->types.size()) return MXG_ERR_RANGE;
        if (cell[k] < 0 || cell[k] >= sp.ncells) return MXG_ERR_CELL;
        for (int q = 0; q < 3; ++q)
            if (!std::isfinite(xrel[3 * (size_t)k + q])) return MXG_ERR_ARG;
    }
    const int first = (int)e->ptype.size();
    for (int k = 0; k < n; ++k) {
        for (int q = 0; q < 3; ++q) {
            // the global position the cell-relative one stands for (reported before the start)
            e->px.push_back(sp.cell_origin[3 * (size_t)cell[k] + q] + (double)xrel[3 * (size_t)k + q]);
            e->pv.push_back(v ? v[3 * (size_t)k + q] : 0.f);
            e->pxr.push_back(xrel[3 * (size_t)k + q]);
        }
        e->ptype.push_back(type[k]);
        e->prep.push_back(rep);
        e->pcell.push_back(cell[k]);
        if (ids_out) ids_out[k] = first + k;
    }
    return MXG_OK;
}

int mxg_engine_set_occupancy_hint(mxg_engine *e, long long nparts) {
    if (!e) return MXG_ERR_NULL;
    if (e->started) return MXG_ERR_STATE;
    if (nparts < 0) return MXG_ERR_ARG;
    e->occupancy_hint = nparts;
    return MXG_OK;
}

int mxg_engine_addparts(mxg_engine *e, int n, const double *x, const float *v, const int *type, int *ids_out) {
    return mxg_engine_addparts_replica(e, 0, n, x, v, type, ids_out);
}

int mxg_engine_addbonds(mxg_engine *e, int n, const int *i, const int *j, const mxg_potential *p,
                        double dissociation_energy, int *ids_out) {
    if (!e || !p || (n > 0 && (!i || !j))) return MXG_ERR_NULL;
    if (e->started) return MXG_ERR_STATE;
    if (p->t.kind != kKindTable) return MXG_ERR_POTENTIAL;
    e->pots.push_back(p->t);
    const int idx = (int)e->pots.size() - 1;
    for (int k = 0; k < n; ++k) {
        if (ids_out) ids_out[k] = (int)e->bonds.size();
        e->bonds.push_back({i[k], j[k], idx, dissociation_energy});
    }
    return MXG_OK;
}

int mxg_engine_addangles(mxg_engine *e, int n, const int *i, const int *j, const int *k, const mxg_potential *p,
                         int *ids_out) {
    if (!e || !p || (n > 0 && (!i || !j || !k))) return MXG_ERR_NULL;
    if (e->started) return MXG_ERR_STATE;
    if (p->t.kind != kKindTable) return MXG_ERR_POTENTIAL;
    e->pots.push_back(p->t);
    const int idx = (int)e->pots.size() - 1;
    for (int q = 0; q < n; ++q) {
        if (ids_out) ids_out[q] = (int)e->angles.size();
        e->angles.push_back({i[q], j[q], k[q], idx});
    }
    return MXG_OK;
}

int mxg_engine_adddihedrals(mxg_engine *e, int n, const int *i, const int *j, const int *k, const int *l,
                            const mxg_potential *p, int *ids_out) {
    if (!e || !p || (n > 0 && (!i || !j || !k || !l))) return MXG_ERR_NULL;
    if (e->started) return MXG_ERR_STATE;
    if (p->t.kind != kKindTable) return MXG_ERR_POTENTIAL;
    e->pots.push_back(p->t);
    const int idx = (int)e->pots.size() - 1;
    for (int q = 0; q < n; ++q) {
        if (ids_out) ids_out[q] = (int)e->dihedrals.size();
        e->dihedrals.push_back({i[q], j[q], k[q], l[q], idx});
    }
    return MXG_OK;
}

int mxg_engine_pairs_within(mxg_engine *e, int n, const int *ids, float cutoff, const unsigned char *type_mask,
                            int ntypes, int *out_i, int *out_j, int cap, int *count) {
    if (!e || !count || (n > 0 && !ids)) return MXG_ERR_NULL;
    if (!e->started) return MXG_ERR_STATE;
    if (!(cutoff >= 0.0f) || (type_mask && ntypes <= 0)) return MXG_ERR_ARG;
    *count = 0;
    if (n < 2) return MXG_OK;
    for (int q = 0; q < n; ++q)
        if (ids[q] < 0 || ids[q] >= e->nparts) return MXG_ERR_RANGE;
    const Space &sp = e->spaces[e->prep[ids[0]]];
    std::vector<int> a, b;
    const int rc = find_pairs_within(e->view(e->cur), e->d_slot_of_id, e->nparts, sp.origin, sp.dim, n, ids, cutoff,
                                     type_mask, ntypes, a, b, e->stream);
    if (rc == -2) return MXG_ERR_MALLOC;
    if (rc != 0) return MXG_ERR_CUDA;
    *count = (int)a.size();
    if (!out_i || !out_j || cap < (int)a.size()) return out_i || out_j ? MXG_ERR_RANGE : MXG_OK;
    std::copy(a.begin(), a.end(), out_i);
    std::copy(b.begin(), b.end(), out_j);
    return MXG_OK;
}

int mxg_engine_group_metrics(mxg_engine *e, int n, const int *ids, double *out) {
    if (!e || !ids || !out) return MXG_ERR_NULL;
    if (!e->started) return MXG_ERR_STATE;
    if (n < 1) return MXG_ERR_ARG;
    for (int q = 0; q < n; ++q)
        if (ids[q] < 0 || ids[q] >= e->nparts) return MXG_ERR_RANGE;
    int *d_ids = nullptr;
    double *d_out = nullptr;
    if (cudaMalloc(&d_ids, sizeof(int) * (size_t)n) != cudaSuccess) return MXG_ERR_MALLOC;
    if (cudaMalloc(&d_out, sizeof(double) * 17) != cudaSuccess) {
        cudaFree(d_ids);
        return MXG_ERR_MALLOC;
    }
    cudaError_t err = cudaMemcpyAsync(d_ids, ids, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, e->stream);
    if (err == cudaSuccess) {
        launch_group_metrics(e->view(e->cur), d_ids, n, e->d_slot_of_id, d_out, e->stream);
        err = cudaMemcpyAsync(out, d_out, sizeof(double) * 17, cudaMemcpyDeviceToHost, e->stream);
    }
    if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
    cudaFree(d_ids);
    cudaFree(d_out);
    return err == cudaSuccess ? MXG_OK : MXG_ERR_CUDA;
}

int mxg_engine_add_cuboid(mxg_engine *e, int rep, const float *pos, const float *size, const float *angles, int *id) {
    if (!e || !size || !angles) return MXG_ERR_NULL;
    if (e->started) return MXG_ERR_STATE;
    if (rep < 0 || rep >= (int)e->spaces.size()) return MXG_ERR_RANGE;
    float centre[3];
    for (int k = 0; k < 3; ++k) centre[k] = pos ? pos[k] : (float)e->spaces[rep].dim[k] / 2.f;  // engine_center
    e->cuboids.push_back(make_cuboid(rep, centre, size, angles));
    if (id) *id = (int)e->cuboids.size() - 1;
    return MXG_OK;
}

int mxg_engine_set_cuboid_potential(mxg_engine *e, int type, const mxg_potential *p) {
    if (!e || !p) return MXG_ERR_NULL;
    if (e->started) return MXG_ERR_STATE;
    if (type < 0 || type >= (int)e->types.size()) return MXG_ERR_RANGE;
    if (p->t.kind != kKindTable) return MXG_ERR_POTENTIAL;
    e->pots.push_back(p->t);
    e->types[type].cpot = (int)e->pots.size() - 1;
    return MXG_OK;
}

int mxg_engine_cuboid_info(const mxg_engine *e, int id, float *out16) {
    if (!e || !out16) return MXG_ERR_NULL;
    if (id < 0 || id >= (int)e->cuboids.size()) return MXG_ERR_RANGE;
    const CuboidInfo &c = e->cuboids[id];
    for (int k = 0; k < 3; ++k) {
        out16[k] = c.pos[k];
        out16[3 + k] = c.size[k];
        out16[10 + k] = c.lo[k];
        out16[13 + k] = c.hi[k];
    }
    for (int k = 0; k < 4; ++k) out16[6 + k] = c.q[k];
    return MXG_OK;
}

int mxg_engine_set_boundary_potential(mxg_engine *e, int face, int type, const mxg_potential *p) {
    if (!e || !p) return MXG_ERR_NULL;
    if (e->started) return MXG_ERR_STATE;
    if (face < -1 || face > 5 || type < 0 || type >= (int)e->types.size()) return MXG_ERR_RANGE;
    e->pots.push_back(p->t);
    const int idx = (int)e->pots.size() - 1;
    for (int f = 0; f < 6; ++f)
        if (face < 0 || f == face) e->types[type].bpot[f] = idx;
    return MXG_OK;
}

int mxg_engine_set_type_species(mxg_engine *e, int type, int nspec, const unsigned *flags) {
    if (!e || (nspec > 0 && !flags)) return MXG_ERR_NULL;
    if (e->started) return MXG_ERR_STATE;
    if (type < 0 || type >= (int)e->types.size()) return MXG_ERR_RANGE;
    if (nspec < 0 || nspec > 8) return MXG_ERR_ARG;  // state vectors of up to 8 species
    if ((int)e->type_nspec.size() <= type) {
        e->type_nspec.resize(type + 1, 0);
        e->type_sflags.resize(type + 1);
    }
    e->type_nspec[type] = nspec;
    e->type_sflags[type].assign(flags, flags + nspec);
    return MXG_OK;
}

int mxg_engine_add_flux(mxg_engine *e, int kind, int ta, int tb, int ia, int ib, float k, float decay, float target) {
    if (!e) return MXG_ERR_NULL;
    if (e->started) return MXG_ERR_STATE;
    const int nt = (int)e->types.size();
    if (kind < 0 || kind > 2 || ta < 0 || tb < 0 || ta >= nt || tb >= nt) return MXG_ERR_ARG;
    auto nsp = [&](int t) { return t < (int)e->type_nspec.size() ? e->type_nspec[t] : 0; };
    if (ia < 0 || ib < 0 || ia >= nsp(ta) || ib >= nsp(tb)) return MXG_ERR_RANGE;
    const size_t key = (size_t)std::min(ta, tb) * e->max_type + std::max(ta, tb);
    if (e->flux_lists.size() <= key) e->flux_lists.resize(key + 1);
    // one flux object of 8 slots per type pair holds at most 7 entries (MxFluxes_AddFlux, Flux.cpp:294-303)
    if (e->flux_lists[key].size() + 1 >= 8) return MXG_ERR_RANGE;
    DevFlux f;
    f.kind = kind;
    f.ta = ta;
    f.tb = tb;
    f.ia = ia;
    f.ib = ib;
    f.k = k;
    f.decay = decay;
    f.target = target;
    e->flux_lists[key].push_back(f);
    return MXG_OK;
}

int mxg_engine_set_species(mxg_engine *e, int n, int smax, const float *values) {
    if (!e || (n > 0 && !values)) return MXG_ERR_NULL;
    if (smax <= 0 || smax > 8) return MXG_ERR_ARG;
    if (!e->started) {
        // staged by particle id, at the width the start will use
        int width = 0;
        for (int t : e->type_nspec) width = std::max(width, t);
        if (width == 0) return MXG_ERR_STATE;
        const int np = (int)e->ptype.size();
        e->spec_host.assign((size_t)np * width, 0.0f);
        for (int id = 0; id < n && id < np; ++id)
            for (int k = 0; k < std::min(smax, width); ++k) e->spec_host[(size_t)id * width + k] = values[(size_t)id * smax + k];
        return MXG_OK;
    }
    if (e->smax == 0) return MXG_ERR_STATE;
    std::vector<float> buf((size_t)e->nparts * e->smax, 0.0f);
    CUDA_TRY(cudaMemcpyAsync(buf.data(), e->d_spec, sizeof(float) * buf.size(), cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    for (int id = 0; id < n && id < e->nparts; ++id)
        for (int k = 0; k < std::min(smax, e->smax); ++k) buf[(size_t)id * e->smax + k] = values[(size_t)id * smax + k];
    CUDA_TRY(cudaMemcpyAsync(e->d_spec, buf.data(), sizeof(float) * buf.size(), cudaMemcpyHostToDevice, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    return MXG_OK;
}

int mxg_engine_get_species(mxg_engine *e, int n, int smax, float *out) {
    if (!e || (n > 0 && !out)) return MXG_ERR_NULL;
    if (!e->started) return MXG_ERR_STATE;
    if (smax <= 0) return MXG_ERR_ARG;
    if (e->smax == 0) return MXG_OK;
    std::vector<float> buf((size_t)e->nparts * e->smax);
    CUDA_TRY(cudaMemcpyAsync(buf.data(), e->d_spec, sizeof(float) * buf.size(), cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    for (int id = 0; id < n && id < e->nparts; ++id)
        for (int k = 0; k < std::min(smax, e->smax); ++k) out[(size_t)id * smax + k] = buf[(size_t)id * e->smax + k];
    return MXG_OK;
}

int mxg_engine_add_exclusions(mxg_engine *e, int n, const int *i, const int *j) {
    if (!e || (n > 0 && (!i || !j))) return MXG_ERR_NULL;
    if (e->started) return MXG_ERR_STATE;
    for (int q = 0; q < n; ++q) e->exclusions.push_back({std::min(i[q], j[q]), std::max(i[q], j[q])});
    return MXG_OK;
}

int mxg_engine_exclusion_shrink(mxg_engine *e) {
    if (!e) return MXG_ERR_NULL;
    if (e->started) return MXG_ERR_STATE;
    std::sort(e->exclusions.begin(), e->exclusions.end());
    e->exclusions.erase(std::unique(e->exclusions.begin(), e->exclusions.end()), e->exclusions.end());
    return MXG_OK;
}

int mxg_engine_start(mxg_engine *e, void *cuda_stream) {
    if (!e) return MXG_ERR_NULL;
    if (e->started) return MXG_ERR_STATE;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return MXG_ERR_NOCUDA;
    return e->start((cudaStream_t)cuda_stream);
}

int mxg_engine_step(mxg_engine *e, int nsteps) {
    if (!e) return MXG_ERR_NULL;
    if (!e->started) return MXG_ERR_STATE;
    if (e->nparts == 0) return MXG_OK;
    for (int s = 0; s < nsteps; ++s) {
        if (e->graph[e->cur]) {
            CUDA_TRY(cudaGraphLaunch(e->graph[e->cur], e->stream));
        } else {
            e->enqueue_step(e->cur);
            CUDA_TRY(cudaGetLastError());
        }
        e->cur = 1 - e->cur;
        e->force_layout = 1 - e->cur;
    }
    return MXG_OK;
}

int mxg_engine_step_timed(mxg_engine *e, int nsteps, double *ms, int n) {
    if (!e || !ms) return MXG_ERR_NULL;
    if (!e->started) return MXG_ERR_STATE;
    if (n < 15 || nsteps < 0) return MXG_ERR_ARG;
    for (int k = 0; k < n; ++k) ms[k] = 0.0;
    if (e->nparts == 0) return MXG_OK;
    cudaEvent_t ev[6];
    for (int k = 0; k < 6; ++k) CUDA_TRY(cudaEventCreate(&ev[k]));
    // timer ids of the reference (engine.h:113-135): step 0, prepare 1, nonbond 4, bonded 5,
    // advance 11, shuffle 14
    const int slot[5] = {1, 4, 5, 11, 14};
    int rc = MXG_OK;
    for (int s = 0; s < nsteps && rc == MXG_OK; ++s) {
        e->enqueue_step(e->cur, ev);
        if (cudaGetLastError() != cudaSuccess || cudaEventSynchronize(ev[5]) != cudaSuccess) {
            rc = MXG_ERR_CUDA;
            break;
        }
        float t;
        for (int k = 0; k < 5; ++k) {
            cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
            ms[slot[k]] += t;
        }
        cudaEventElapsedTime(&t, ev[0], ev[5]);
        ms[0] += t;
        e->cur = 1 - e->cur;
        e->force_layout = 1 - e->cur;
    }
    for (int k = 0; k < 6; ++k) cudaEventDestroy(ev[k]);
    return rc;
}

int mxg_engine_force(mxg_engine *e) {
    if (!e) return MXG_ERR_NULL;
    if (!e->started) return MXG_ERR_STATE;
    if (e->nparts == 0) return MXG_OK;
    e->enqueue_force(e->cur);
    CUDA_TRY(cudaGetLastError());
    return MXG_OK;
}

int mxg_engine_status(mxg_engine *e) {
    if (!e) return MXG_ERR_NULL;
    if (!e->started) return MXG_OK;
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    unsigned st = 0;
    CUDA_TRY(cudaMemcpy(&st, e->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (st & kStatusNonFinite) return MXG_ERR_NONFINITE;
    if (st & kStatusTooFast) return MXG_ERR_TOOFAST;
    return MXG_OK;
}

int mxg_engine_clear_status(mxg_engine *e) {
    if (!e) return MXG_ERR_NULL;
    if (!e->started) return MXG_OK;
    CUDA_TRY(cudaMemsetAsync(e->d_status, 0, sizeof(unsigned), e->stream));
    return MXG_OK;
}

int mxg_engine_nr_parts(const mxg_engine *e) { return e ? (int)e->ptype.size() : MXG_ERR_NULL; }
int mxg_engine_nr_cells(const mxg_engine *e) { return e ? e->ncells : MXG_ERR_NULL; }

int mxg_engine_unload(mxg_engine *e, int n, double *x, float *v, float *f, int *cell, float *xrel) {
    if (!e) return MXG_ERR_NULL;
    if (!e->started) return MXG_ERR_STATE;
    if (n > e->nparts || n < 0) return MXG_ERR_RANGE;
    if (n == 0) return MXG_OK;
    const size_t N = (size_t)e->nparts;
    // by id on the device (positions: cell origin + x_rel in double), then one copy per array
    if (x && !e->d_ul_x && e->alloc(&e->d_ul_x, 3 * N) != MXG_OK) return MXG_ERR_MALLOC;
    if (v && !e->d_ul_v && e->alloc(&e->d_ul_v, 3 * N) != MXG_OK) return MXG_ERR_MALLOC;
    if (f && !e->d_ul_f && e->alloc(&e->d_ul_f, 3 * N) != MXG_OK) return MXG_ERR_MALLOC;
    if (cell && !e->d_ul_cell && e->alloc(&e->d_ul_cell, N) != MXG_OK) return MXG_ERR_MALLOC;
    if (xrel && !e->d_ul_xrel && e->alloc(&e->d_ul_xrel, 3 * N) != MXG_OK) return MXG_ERR_MALLOC;
    // after a step the forces are in the slot order of the step's starting buffer, whose
    // velocity array still carries the ids in that order
    launch_unload(e->view(e->cur), e->d_vel[e->force_layout], x ? e->d_ul_x : nullptr, v ? e->d_ul_v : nullptr,
                  f ? e->d_ul_f : nullptr, cell ? e->d_ul_cell : nullptr, xrel ? e->d_ul_xrel : nullptr, e->stream);
    const size_t m = (size_t)n;
    if (x) CUDA_TRY(cudaMemcpyAsync(x, e->d_ul_x, sizeof(double) * 3 * m, cudaMemcpyDeviceToHost, e->stream));
    if (v) CUDA_TRY(cudaMemcpyAsync(v, e->d_ul_v, sizeof(float) * 3 * m, cudaMemcpyDeviceToHost, e->stream));
    if (f) CUDA_TRY(cudaMemcpyAsync(f, e->d_ul_f, sizeof(float) * 3 * m, cudaMemcpyDeviceToHost, e->stream));
    if (cell) CUDA_TRY(cudaMemcpyAsync(cell, e->d_ul_cell, sizeof(int) * m, cudaMemcpyDeviceToHost, e->stream));
    if (xrel) CUDA_TRY(cudaMemcpyAsync(xrel, e->d_ul_xrel, sizeof(float) * 3 * m, cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    CUDA_TRY(cudaGetLastError());
    return MXG_OK;
}

int mxg_engine_load(mxg_engine *e, int n, const double *x, const float *v) {
    if (!e || !x) return MXG_ERR_NULL;
    if (!e->started) return MXG_ERR_STATE;
    return e->load_state(x, v, n);
}

int mxg_engine_energy(mxg_engine *e, double *epot, double *ekin, double *virial9) {
    if (!e) return MXG_ERR_NULL;
    if (!e->started) return MXG_ERR_STATE;
    launch_energy(e->nitems, e->d_epot_cell, e->nparts, e->has_bonded() ? e->d_ebond_slot : nullptr,
                  e->has_body() ? e->d_body_e : nullptr, e->d_vel[e->cur], e->d_pos[e->cur], e->d_types, e->d_partials, e->energy_blocks, e->d_energy,
                  e->stream);
    double out[2];
    CUDA_TRY(cudaMemcpyAsync(out, e->d_energy, sizeof(out), cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    if (epot) *epot = out[0];
    if (ekin) *ekin = out[1];
    if (virial9) {
        // the pair virial of the current positions: a force pass in the kernel's
        // virial mode, which writes only its per-warp FP64 partials
        const int nwarps = e->force_grid * kWarpsPerBlock;
        if (nwarps > e->virial_cap) {
            if (e->alloc(&e->d_virial_partials, (size_t)nwarps * 6) != MXG_OK) return MXG_ERR_MALLOC;
            if (!e->d_virial_out && e->alloc(&e->d_virial_out, 9) != MXG_OK) return MXG_ERR_MALLOC;
            e->virial_cap = nwarps;
        }
        EngineView v = e->view(e->cur);
        v.virial_partials = e->d_virial_partials;
        launch_force(v, e->has_dpd, e->force_grid, false, e->stream);
        launch_virial_reduce(e->d_virial_partials, nwarps, e->d_virial_out, e->stream);
        if (e->has_bonded()) {
            // the bonded terms' share (bonds active after the last pass, exclusions, angles, dihedrals)
            const int nblk = bonded_virial_blocks(e->num_sms);
            if (!e->d_bvirial_partials && e->alloc(&e->d_bvirial_partials, (size_t)nblk * 9) != MXG_OK)
                return MXG_ERR_MALLOC;
            launch_bonded_virial(e->view(e->cur), e->bonded_view(), (int)e->bonds.size(), (int)e->exclusions.size(),
                                 (int)e->angles.size(), (int)e->dihedrals.size(), nblk, e->d_bvirial_partials,
                                 e->d_virial_out, e->stream);
        }
        CUDA_TRY(cudaMemcpyAsync(virial9, e->d_virial_out, 9 * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
        CUDA_TRY(cudaStreamSynchronize(e->stream));
        CUDA_TRY(cudaGetLastError());
    }
    return MXG_OK;
}

double mxg_engine_kinetic_energy(mxg_engine *e) {
    double ek = 0.0;
    if (mxg_engine_energy(e, nullptr, &ek, nullptr) != MXG_OK) return -1.0;
    return ek;
}

int mxg_engine_tasks(const mxg_engine *e, int *out, int cap) {
    if (!e) return MXG_ERR_NULL;
    const std::vector<Task> &tasks = e->spaces[0].tasks;
    const int n = (int)tasks.size();
    if (!out) return n;
    if (cap < 4 * n) return -n;
    for (int k = 0; k < n; ++k) {
        out[4 * k] = tasks[k].type;
        out[4 * k + 1] = tasks[k].flags;
        out[4 * k + 2] = tasks[k].i;
        out[4 * k + 3] = tasks[k].j;
    }
    return n;
}

int mxg_engine_bond_flags(mxg_engine *e, unsigned *out, int cap) {
    if (!e) return MXG_ERR_NULL;
    const int n = (int)e->bonds.size();
    if (!out || !e->started) return n;
    if (cap < n) return -n;
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    if (n) CUDA_TRY(cudaMemcpy(out, e->d_bond_flags, sizeof(unsigned) * n, cudaMemcpyDeviceToHost));
    return n;
}

int mxg_engine_set_bond_flags(mxg_engine *e, const unsigned *flags, int n) {
    if (!e || (n > 0 && !flags)) return MXG_ERR_NULL;
    if (!e->started) return MXG_ERR_STATE;
    if (n != (int)e->bonds.size()) return MXG_ERR_RANGE;
    if (n == 0) return MXG_OK;
    std::vector<unsigned> f(flags, flags + n);
    for (unsigned &x : f) x &= 1u;
    int rc = upload(e->d_bond_flags, f, e->stream);
    if (rc != MXG_OK) return rc;
    CUDA_TRY(cudaStreamSynchronize(e->stream));  // the host vector goes out of scope
    return MXG_OK;
}

int mxg_engine_bond_pot_index(const mxg_engine *e, int k, int *idx) {
    if (!e || !idx) return MXG_ERR_NULL;
    if (k < 0 || k >= (int)e->bonds.size()) return MXG_ERR_RANGE;
    *idx = e->bonds[k].pot;
    return MXG_OK;
}

int mxg_engine_space_info(const mxg_engine *e, int *cdim, double *h, int *nr_cells, unsigned *period) {
    if (!e) return MXG_ERR_NULL;
    const Space &sp = e->spaces[0];
    for (int k = 0; k < 3; ++k) {
        if (cdim) cdim[k] = sp.cdim[k];
        if (h) h[k] = sp.h[k];
    }
    if (nr_cells) *nr_cells = sp.ncells;
    if (period) *period = sp.period;
    return MXG_OK;
}

int mxg_engine_device_state(mxg_engine *e, void **pos, void **vel, void **force, void **cell) {
    if (!e) return MXG_ERR_NULL;
    if (!e->started) return MXG_ERR_STATE;
    if (pos) *pos = e->d_pos[e->cur];
    if (vel) *vel = e->d_vel[e->cur];
    if (force) *force = e->d_force;
    if (cell) *cell = e->d_cell_of[e->cur];
    return MXG_OK;
}

int mxg_engine_copy_state(mxg_engine *e, void *host_pos, void *host_vel, int to_device) {
    if (!e || !host_pos || !host_vel) return MXG_ERR_NULL;
    if (!e->started) return MXG_ERR_STATE;
    const size_t bytes = sizeof(float4) * (size_t)e->nparts;
    if (to_device) {
        CUDA_TRY(cudaMemcpyAsync(e->d_pos[e->cur], host_pos, bytes, cudaMemcpyHostToDevice, e->stream));
        CUDA_TRY(cudaMemcpyAsync(e->d_vel[e->cur], host_vel, bytes, cudaMemcpyHostToDevice, e->stream));
        e->refresh_bounds();
    } else {
        CUDA_TRY(cudaMemcpyAsync(host_pos, e->d_pos[e->cur], bytes, cudaMemcpyDeviceToHost, e->stream));
        CUDA_TRY(cudaMemcpyAsync(host_vel, e->d_vel[e->cur], bytes, cudaMemcpyDeviceToHost, e->stream));
    }
    return MXG_OK;
}

int mxg_engine_energy_async(mxg_engine *e, double *host_out2) {
    if (!e || !host_out2) return MXG_ERR_NULL;
    if (!e->started) return MXG_ERR_STATE;
    launch_energy(e->nitems, e->d_epot_cell, e->nparts, e->has_bonded() ? e->d_ebond_slot : nullptr,
                  e->has_body() ? e->d_body_e : nullptr, e->d_vel[e->cur], e->d_pos[e->cur], e->d_types, e->d_partials, e->energy_blocks, e->d_energy,
                  e->stream);
    CUDA_TRY(cudaMemcpyAsync(host_out2, e->d_energy, 2 * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    return MXG_OK;
}

int mxg_engine_snapshot_bytes(const mxg_engine *e, size_t *bytes) {
    if (!e || !bytes) return MXG_ERR_NULL;
    if (!e->started) return MXG_ERR_STATE;
    *bytes = e->snap_layout().total;
    return MXG_OK;
}

int mxg_engine_snapshot(mxg_engine *e, void *dev_buf, int save) {
    if (!e || !dev_buf) return MXG_ERR_NULL;
    if (!e->started) return MXG_ERR_STATE;
    if (((uintptr_t)dev_buf) & 15) return MXG_ERR_ARG;
    const auto L = e->snap_layout();
    char *b = static_cast<char *>(dev_buf);
    const int c = e->cur;
    struct Sec {
        void *dev;
        size_t off, bytes;
    } secs[] = {
        {e->d_pos[c], L.pos, sizeof(float4) * (size_t)e->nparts},
        {e->d_vel[c], L.vel, sizeof(float4) * (size_t)e->nparts},
        {e->d_cell_of[c], L.cell_of, sizeof(int) * (size_t)e->nparts},
        {e->d_slot_of_id, L.slot_of_id, sizeof(int) * (size_t)e->nparts},
        {e->d_cell_start[c], L.start, sizeof(int) * (size_t)(e->ncells + 1)},
        {e->d_cell_count[c], L.count, sizeof(int) * (size_t)e->ncells},
        {e->d_step, L.step, sizeof(unsigned long long)},
        {e->d_bond_flags, L.bonds, sizeof(unsigned) * e->bonds.size()},
        {e->d_spec, L.spec, sizeof(float) * (size_t)e->nparts * e->smax},
        {e->d_rate, L.rate, sizeof(float) * (size_t)e->nparts * e->smax},
        {e->d_persist, L.persist, e->has_sb ? sizeof(float4) * (size_t)e->nparts : 0},
    };
    // every section in one copy launch (whole 4-byte words: every section's size is a multiple of 4)
    CopySections cs;
    cs.n = 0;
    for (const Sec &q : secs) {
        if (q.bytes == 0) continue;
        unsigned *in = static_cast<unsigned *>(q.dev), *out = reinterpret_cast<unsigned *>(b + q.off);
        cs.src[cs.n] = save ? in : out;
        cs.dst[cs.n] = save ? out : in;
        cs.words[cs.n] = q.bytes / 4;
        ++cs.n;
    }
    launch_copy_sections(cs, e->stream);
    CUDA_TRY(cudaGetLastError());
    if (!save) e->refresh_bounds();
    return MXG_OK;
}

int mxg_engine_adjoint_params(mxg_engine *e, int n, const int *pot, const int *param, const int *slot) {
    if (!e || (n > 0 && (!pot || !param || !slot))) return MXG_ERR_NULL;
    std::vector<mxg_engine::GradReg> regs;
    int nslots = 0;
    for (int k = 0; k < n; ++k) {
        if (pot[k] < 0 || pot[k] >= (int)e->pots.size() || slot[k] < 0 || slot[k] >= kMaxGradSlots)
            return MXG_ERR_RANGE;
        regs.push_back({pot[k], param[k], slot[k]});
        nslots = std::max(nslots, slot[k] + 1);
    }
    e->grad_regs = regs;
    e->grad_slots = nslots;
    e->adjoint_stale = true;
    if (e->started) return e->build_adjoint();
    return MXG_OK;
}

int mxg_engine_vjp_step(mxg_engine *e, void *lam_x, void *lam_v, double *grad) {
    return mxg_engine_vjp_step_forces(e, lam_x, lam_v, grad, nullptr);
}

int mxg_engine_save_forces(mxg_engine *e, void *dev_buf) {
    if (!e || !dev_buf) return MXG_ERR_NULL;
    if (!e->started) return MXG_ERR_STATE;
    if (e->nparts == 0) return MXG_OK;
    CUDA_TRY(cudaMemcpyAsync(dev_buf, e->d_force, sizeof(float4) * (size_t)e->nparts, cudaMemcpyDeviceToDevice,
                             e->stream));
    return MXG_OK;
}

int mxg_engine_vjp_step_forces(mxg_engine *e, void *lam_x, void *lam_v, double *grad, const void *forces) {
    if (!e || !lam_x || !lam_v || !grad) return MXG_ERR_NULL;
    if (!e->started) return MXG_ERR_STATE;
    // angles, dihedrals, exclusions, single-body, wall and large-particle forces are not
    // differentiated; bonds are
    if (!e->angles.empty() || !e->dihedrals.empty() || !e->exclusions.empty() || e->has_sb || e->has_walls ||
        e->nlarge)
        return MXG_ERR_ARG;
    if (e->nparts == 0) return MXG_OK;
    if (e->adjoint_stale) {
        const int rc = e->build_adjoint();
        if (rc != MXG_OK) return rc;
    }
    const EngineView v = e->view(e->cur);
    // forces of the step's state; with bonds, the bond pass of the state completes them and
    // leaves the flags of the bonds that acted in the step (as the forward step's pass did)
    const bool bonded = !e->bonds.empty();
    if (forces && !bonded)
        CUDA_TRY(cudaMemcpyAsync(e->d_force, forces, sizeof(float4) * (size_t)e->nparts, cudaMemcpyDeviceToDevice,
                                 e->stream));
    else
        launch_force(v, e->has_dpd, e->force_grid, !bonded, e->stream);
    BondedView bv;
    if (bonded) {
        bv = e->bonded_view();
        launch_bonded(v, bv, e->stream);
    }
    e->force_layout = e->cur;
    AdjointView a;
    a.lam_x = static_cast<float4 *>(lam_x);
    a.lam_v = static_cast<float4 *>(lam_v);
    a.w = e->d_adj_w;
    a.gx = e->d_adj_gx;
    a.gv = e->d_adj_gv;
    a.pot_grad = e->d_pot_grad;
    a.dcoef = e->d_dcoef;
    a.partials = e->d_adj_partials;
    a.items = e->d_adj_items;
    a.nitems = e->adj_nitems;
    a.item_ctr = e->d_adj_ctr;
    a.pgx = e->d_adj_pgx;
    a.pgv = e->d_adj_pgv;
    a.bond_partials = e->d_adj_bond_partials;
    a.nslots = e->grad_slots;
    launch_vjp_step(v, a, bonded ? &bv : nullptr, e->num_sms, grad, e->stream);
    CUDA_TRY(cudaGetLastError());
    return MXG_OK;
}

int mxg_engine_positions(mxg_engine *e, void *x4, void *v4) {
    if (!e) return MXG_ERR_NULL;
    if (!e->started) return MXG_ERR_STATE;
    if (e->nparts == 0) return MXG_OK;
    launch_positions(e->view(e->cur), static_cast<float4 *>(x4), static_cast<float4 *>(v4), e->stream);
    CUDA_TRY(cudaGetLastError());
    return MXG_OK;
}

int mxg_engine_set_step_counter(mxg_engine *e, unsigned long long step) {
    if (!e) return MXG_ERR_NULL;
    if (!e->started) return MXG_ERR_STATE;
    CUDA_TRY(cudaMemcpyAsync(e->d_step, &step, sizeof(step), cudaMemcpyHostToDevice, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    return MXG_OK;
}

int mxg_rdf(const void *x4, int n, const double *box, int type_a, int type_b, int nbins, double dr, double sigma,
            void *hist, const double *coef, void *grad4, void *stream) {
    if (!x4 || !box || (!hist && !grad4) || (grad4 && !coef)) return MXG_ERR_NULL;
    if (n < 0 || !(dr > 0) || !(sigma > 0)) return MXG_ERR_ARG;
    if (n == 0) return MXG_OK;
    const int rc = launch_rdf(static_cast<const float4 *>(x4), n, box, type_a, type_b, nbins, dr, sigma,
                              static_cast<unsigned long long *>(hist), coef, static_cast<float4 *>(grad4),
                              static_cast<cudaStream_t>(stream));
    if (rc == -1) return MXG_ERR_RANGE;
    if (rc == -2) return MXG_ERR_MALLOC;
    CUDA_TRY(cudaGetLastError());
    return MXG_OK;
}

int mxg_engine_finalize(mxg_engine *e) {
    if (!e) return MXG_ERR_NULL;
    if (e->started && e->stream) cudaStreamSynchronize(e->stream);
    delete e;
    return MXG_OK;
}

/* Launches the force kernel reps times on the engine stream between two events
 * and returns the mean duration in milliseconds. */
int mxg_engine_time_force(mxg_engine *e, int reps, double *ms) {
    if (!e || !ms) return MXG_ERR_NULL;
    if (!e->started) return MXG_ERR_STATE;
    cudaEvent_t a, b;
    CUDA_TRY(cudaEventCreate(&a));
    CUDA_TRY(cudaEventCreate(&b));
    const EngineView v = e->view(e->cur);
    CUDA_TRY(cudaEventRecord(a, e->stream));
    for (int r = 0; r < reps; ++r) launch_force(v, e->has_dpd, e->force_grid, true, e->stream);
    e->force_layout = e->cur;
    CUDA_TRY(cudaEventRecord(b, e->stream));
    CUDA_TRY(cudaEventSynchronize(b));
    float t = 0.f;
    cudaEventElapsedTime(&t, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *ms = t / std::max(1, reps);
    return MXG_OK;
}

int mxg_engine_time_force_launches(mxg_engine *e, int reps, void *flush, size_t flush_bytes, double *ms) {
    if (!e || !ms) return MXG_ERR_NULL;
    if (!e->started) return MXG_ERR_STATE;
    if (reps < 1 || (flush_bytes > 0 && !flush)) return MXG_ERR_ARG;
    std::vector<cudaEvent_t> ev(2 * (size_t)reps, nullptr);
    cudaError_t err = cudaSuccess;
    for (auto &x : ev)
        if (err == cudaSuccess) err = cudaEventCreate(&x);
    const EngineView v = e->view(e->cur);
    for (int r = 0; r < reps && err == cudaSuccess; ++r) {
        if (flush_bytes > 0) err = cudaMemsetAsync(flush, 0, flush_bytes, e->stream);
        if (err == cudaSuccess) err = cudaEventRecord(ev[2 * r], e->stream);
        if (err == cudaSuccess) launch_force(v, e->has_dpd, e->force_grid, false, e->stream);
        if (err == cudaSuccess) err = cudaEventRecord(ev[2 * r + 1], e->stream);
    }
    if (err == cudaSuccess) {
        e->enqueue_force(e->cur);  // the complete forces of the state, as engine_force leaves them
        err = cudaStreamSynchronize(e->stream);
    }
    for (int r = 0; r < reps && err == cudaSuccess; ++r) {
        float t = 0.f;
        err = cudaEventElapsedTime(&t, ev[2 * r], ev[2 * r + 1]);
        ms[r] = t;
    }
    for (auto &x : ev)
        if (x) cudaEventDestroy(x);
    return err == cudaSuccess ? MXG_OK : MXG_ERR_CUDA;
}

/* The force kernel's autotuner: every tile shape (own particles and neighbour particles staged
 * per region, see the force kernel's Tile) with candidate CTAs per SM is timed on the current
 * state (the median of five launches each, after one warm launch) and the fastest pair is
 * kept; the step graphs are re-captured with it. The state's occupancy (its density) decides. */
int mxg_engine_autotune(mxg_engine *e) {
    if (!e) return MXG_ERR_NULL;
    if (!e->started) return MXG_ERR_STATE;
    if (e->nparts == 0) return MXG_OK;
    const int cands[] = {2, 4, 6, 8, 12, 16, 24, 32};
    const int max_grid = (e->nitems + kWarpsPerBlock - 1) / kWarpsPerBlock;
    int best = e->force_grid, best_per_sm = 0, best_variant = e->force_variant;
    float best_ms = 1e30f;
    cudaEvent_t ev[6];
    for (auto &x : ev) CUDA_TRY(cudaEventCreate(&x));
    for (int variant = 0; variant < force_variants(); ++variant) {
        e->force_variant = variant;
        const EngineView v = e->view(e->cur);
        for (int per_sm : cands) {
            const int grid = std::max(1, std::min(max_grid, e->num_sms * per_sm));
            launch_force(v, e->has_dpd, grid, true, e->stream);  // warm
            float t[5];
            for (int r = 0; r < 5; ++r) {
                CUDA_TRY(cudaEventRecord(ev[r], e->stream));
                launch_force(v, e->has_dpd, grid, true, e->stream);
                CUDA_TRY(cudaEventRecord(ev[5], e->stream));
                CUDA_TRY(cudaEventSynchronize(ev[5]));
                cudaEventElapsedTime(&t[r], ev[r], ev[5]);
            }
            std::sort(t, t + 5);
            if (t[2] < best_ms) {
                best_ms = t[2];
                best = grid;
                best_per_sm = per_sm;
                best_variant = variant;
            }
            if (grid == max_grid) break;
        }
    }
    for (auto &x : ev) cudaEventDestroy(x);
    e->force_layout = e->cur;
    e->force_grid = best;
    e->force_variant = best_variant;
    const int rc = e->build_graphs();
    return rc != MXG_OK ? rc : best_per_sm;
}

int mxg_engine_force_config(mxg_engine *e, int *variant, int *grid, int set) {
    if (!e || !variant || !grid) return MXG_ERR_NULL;
    if (!set) {
        *variant = e->force_variant;
        *grid = e->force_grid;
        return MXG_OK;
    }
    if (!e->started) return MXG_ERR_STATE;
    if (*variant < 0 || *variant >= force_variants() || *grid < 1) return MXG_ERR_ARG;
    // no more blocks than the work items can occupy (the autotuner's bound too)
    *grid = std::min(*grid, std::max(1, (e->nitems + kWarpsPerBlock - 1) / kWarpsPerBlock));
    e->force_variant = *variant;
    e->force_grid = *grid;
    return e->build_graphs();
}

int mxg_engine_number_density(mxg_engine *e, int n, float *out, double *volume) {
    if (!e || (!out && !volume)) return MXG_ERR_NULL;
    if (!e->started) return MXG_ERR_STATE;
    if (n < 0 || n > e->nparts) return MXG_ERR_RANGE;
    if (e->nparts == 0) {
        if (volume) *volume = 0.0;
        return MXG_OK;
    }
    if (!e->d_nd && e->alloc(&e->d_nd, (size_t)e->nparts) != MXG_OK) return MXG_ERR_MALLOC;
    launch_number_density(e->view(e->cur), e->has_fluxes ? e->d_flux_off : nullptr, e->d_nd, e->stream);
    std::vector<float> h((size_t)e->nparts);
    CUDA_TRY(cudaMemcpyAsync(h.data(), e->d_nd, sizeof(float) * h.size(), cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    CUDA_TRY(cudaGetLastError());
    if (out) std::copy(h.begin(), h.begin() + n, out);
    if (volume) {
        // engine_advance's computed volume: the sum over particles of 1 / number density
        double vol = 0.0;
        for (float x : h) vol += x > 0.f ? (double)(1.f / x) : 0.0;
        *volume = vol;
    }
    return MXG_OK;
}

int mxg_engine_pair_counts(mxg_engine *e, long long *candidates, long long *interacting) {
    if (!e) return MXG_ERR_NULL;
    if (!e->started) return MXG_ERR_STATE;
    // candidates as the reference's task list defines them: sum over pair tasks
    // of n_i*n_j and over self tasks of n(n-1)/2, for the current occupancy
    std::vector<int> cnt(e->ncells);
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    CUDA_TRY(cudaMemcpy(cnt.data(), e->d_cell_count[e->cur], sizeof(int) * e->ncells, cudaMemcpyDeviceToHost));
    long long cand = 0;
    for (const Space &sp : e->spaces)
        for (const Task &t : sp.tasks) {
            const int a = sp.cell_offset + t.i, b = sp.cell_offset + t.j;
            if (t.type == kTaskSelf)
                cand += (long long)cnt[a] * (cnt[a] - 1) / 2;
            else if (t.type == kTaskPair)
                cand += (long long)cnt[a] * cnt[b];
        }
    if (candidates) *candidates = cand;
    if (interacting) {
        // one statistics launch of the force kernel counts the interacting pairs
        // (each pair once, in the reference's orientation)
        unsigned long long *d_cnt = nullptr;
        CUDA_TRY(cudaMalloc(&d_cnt, sizeof(unsigned long long)));
        CUDA_TRY(cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long), e->stream));
        EngineView v = e->view(e->cur);
        v.pair_stats = d_cnt;
        if (e->has_body()) launch_body(v, e->d_body_f, e->stream);
        launch_force(v, e->has_dpd, e->force_grid, true, e->stream);
        e->force_layout = e->cur;
        unsigned long long n = 0;
        CUDA_TRY(cudaMemcpyAsync(&n, d_cnt, sizeof(n), cudaMemcpyDeviceToHost, e->stream));
        CUDA_TRY(cudaStreamSynchronize(e->stream));
        cudaFree(d_cnt);
        *interacting = (long long)n;
    }
    return MXG_OK;
}

}  // extern "C"
