/* Host-callable launchers for the engine kernels (mxg_kernels.cu). */
#pragma once
#include <vector>

#include "mxg_device.cuh"

namespace mxg {

void configure_force_kernels();
/* number of force-kernel tile shapes (EngineView::force_variant ranges over them) */
int force_variants();
/* particle-group metrics (mxg_metrics.cu): out[17] as mxg_engine_group_metrics */
void launch_group_metrics(const EngineView &v, const int *ids, int n, const int *slot_of_id, double *out,
                          cudaStream_t st);
void launch_sort_bounds(const EngineView &v, cudaStream_t st);
/* Before a force pass: the per-type kinetic energy (Berendsen) and, when redraw is set (the
 * step's first force pass), the persistent random forces due at this step. */
void launch_singlebody_prep(const EngineView &v, int ntypes, double *type_ke, float4 *persist, bool redraw,
                            cudaStream_t st);
void launch_virial_reduce(const double *partials, int nwarps, double *out9, cudaStream_t st);
/* out9 += the virial of the bonded terms (nb bonds, nx exclusions, na angles, nd dihedrals) of the
 * current positions; partials: nblocks * 9 doubles of scratch */
int bonded_virial_blocks(int num_sms);
void launch_bonded_virial(const EngineView &v, const BondedView &bv, int nb, int nx, int na, int nd, int nblocks,
                          double *partials, double *out9, cudaStream_t st);
/* combine: add the received planes here (no bond or integrator pass follows) */
void launch_force(const EngineView &v, bool has_dpd, int grid, bool combine, cudaStream_t st);
/* wall and large-particle forces (into body_f) and energies (v.body_e) of the current positions; before
 * the pass's force kernel */
void launch_body(const EngineView &v, float4 *body_f, cudaStream_t st);
/* species flux rates of the current positions (full shell, by particle id), added to the carried rates */
void launch_fluxes(const EngineView &v, const SpeciesView &sp, cudaStream_t st);
/* species values += dt * rates after a forward-Euler step for particles that kept their cell (new_cell
 * from the integrator); v is the state the rates belong to */
void launch_species_integrate(const EngineView &v, const SpeciesView &sp, const int *new_cell, cudaStream_t st);
/* bonds then angles; also adds the received planes (the force pass ran without combine) */
void launch_bonded(const EngineView &v, const BondedView &bv, cudaStream_t st);
/* Forward Euler, walls and relocation: movers into the destination's bucket or the overflow list,
 * counted per cell (in_count, out_count) and, between chunks of cells, in v.chunk_delta. */
void launch_integrate(const EngineView &v, float4 *pos, float4 *vel, int *new_cell, int *in_count, int *in_list,
                      int *out_count, bool add_planes, cudaStream_t st);
/* Runge-Kutta 4: rk[5] = p0, v0, accx, accv, vk of the previous stage (per slot). */
void launch_rk_stage(const EngineView &v, float4 *pos, float4 *const *rk, int stage, bool add_planes,
                     cudaStream_t st);
void launch_rk_final(const EngineView &v, float4 *pos, float4 *vel, float4 *const *rk, int *new_cell, int *in_count,
                     int *in_list, int *out_count, bool add_planes, cudaStream_t st);
/* The stable re-binning into the other buffer: new cell starts and counts (old starts plus the net
 * movers before each cell, from the integrator's per-cell and per-chunk counts in v.chunk_delta),
 * the particles' new slots and the new cells' key bounds. Clears the other parity's counts
 * (clear_in/out per cell, clear_chunk[nchunks]) for the next step, re-arms the overflow list and
 * advances the step counter. ctl: the scatter's done counter (zero before the first launch). */
void launch_scatter(const EngineView &v, const float4 *pos, const float4 *vel, const int *new_cell,
                    const int *old_start, const int *old_count, const int *in_count, const int *in_list,
                    const int *out_count, int *new_start, int *new_count, float4 *pos_out, float4 *vel_out,
                    int *cell_out, int *slot_of_id, int *clear_in, int *clear_out, int *clear_chunk, int nchunks,
                    unsigned *ctl, unsigned long long *step, cudaStream_t st);
/* The particles' number density (f[3] of the reference's particles) for the current positions, by id;
 * flux_off: the species flux lists per type pair (null when there are none). */
void launch_number_density(const EngineView &v, const int *flux_off, float *nd_by_id, cudaStream_t st);
/* engine_load on the device: placement by id into ld's staging arrays, counting into count (zeroed by the
 * caller); ld.err is set when a particle lies outside its box. */
void launch_load_place(const EngineView &v, const LoadView &ld, int *count, cudaStream_t st);
/* The rest of the load: scan of count into start, the slot arrays in (cell, id) order, key bounds. */
void launch_load_order(const EngineView &v, const LoadView &ld, const int *count, int *start, int *count_out,
                       float4 *pos_out, float4 *vel_out, int *cell_out, int *slot_of_id, cudaEvent_t vel_ready,
                       cudaStream_t st);
/* engine_unload's arrays by id on the device (any output may be null); force_ids: the velocities of the slot
 * order the forces were computed in */
void launch_unload(const EngineView &v, const float4 *force_ids, double *x, float *vel, float *f, int *cell,
                   float *xrel, cudaStream_t st);
/* ebond_slot, body_e: per-slot bonded and wall energies of the last pass (null when absent) */
void launch_energy(int ncells, const double *epot_cell, int nparts, const double *ebond_slot, const double *body_e,
                   const float4 *vel, const float4 *pos, const DevType *types, double *partials, int nblocks,
                   double *out, cudaStream_t st);

/* The pairwise bond constructor's pair search (mxg_pairs.cu): pairs (a, b), b < a, of the list ids
 * with |x_a - x_b|^2 <= cutoff^2 in global FP32 coordinates (no periodic image) whose type pair has a
 * nonzero mask entry (mask may be null), in the reference's order. lo, hi bound the replica's box.
 * first/second receive the ids of a and b. Returns 0 or a negative status. */
int find_pairs_within(const EngineView &v, const int *slot_of_id, int nids, const double lo[3], const double hi[3],
                      int n, const int *ids_host, float cutoff, const unsigned char *mask_host, int ntypes,
                      std::vector<int> &first, std::vector<int> &second, cudaStream_t st);

}  // namespace mxg
