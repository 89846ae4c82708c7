/*
 * mxg.h -- C ABI of the B200 force-and-step engine.
 *
 * The entry points replace, one for one, the mdcore engine calls that the
 * reference's Python layer and C drivers make for the force-and-step path
 * (paths relative to the reference project root):
 *
 *   mxg_potential_create_lj126     potential_create_LJ126   src/mdcore/src/MxPotential.cpp:960
 *   mxg_potential_create_morse     potential_create_morse   src/mdcore/src/MxPotential.cpp:3389
 *   mxg_potential_create_harmonic  potential_create_harmonic src/mdcore/src/MxPotential.cpp:335
 *   mxg_potential_create_power     potential_create_power   src/mdcore/src/MxPotential.cpp:1614
 *   mxg_potential_create_harmonic_angle potential_create_harmonic_angle src/mdcore/src/MxPotential.cpp:557
 *   mxg_potential_create_harmonic_dihedral potential_create_harmonic_dihedral src/mdcore/src/MxPotential.cpp:484
 *   mxg_potential_create_dpd       DPDPotential_New         src/mdcore/src/DissapativeParticleDynamics.cpp:134
 *   mxg_potential_eval             potential_eval_ex        src/mdcore/src/potential_eval.hpp:106
 *   mxg_engine_init                engine_init              src/mdcore/include/engine.h:600
 *   mxg_engine_addtype             engine_addtype           src/mdcore/include/engine.h:575
 *   mxg_engine_addpot              engine_addpot            src/mdcore/src/engine.cpp:960
 *   mxg_engine_add_singlebody_force engine_add_singlebody_force src/mdcore/src/engine.cpp:983
 *   mxg_engine_addparts            engine_addpart           src/mdcore/src/engine.cpp:1726
 *   mxg_engine_addbonds            engine_bond_alloc + _bond_init src/mdcore/src/bond.cpp:497
 *   mxg_engine_addangles           engine_angle_alloc + angle_init src/mdcore/src/angle.cpp:659-707
 *   mxg_engine_set_boundary_potential MxBoundaryCondition(s)::set_potential
 *                                  src/mdcore/src/MxBoundaryConditions.cpp:771-836, via bind (MxBind.cpp:74-96)
 *   mxg_engine_set_type_species    a particle type's species list (state vector layout)
 *   mxg_engine_add_flux            MxFluxes_FluxEx src/mdcore/src/Flux.cpp:161-211 (flux, secrete, uptake)
 *   mxg_engine_set_species / mxg_engine_get_species  the particles' species values
 *   mxg_engine_pairs_within        make_pairlist (the pair search of MxBond_PairwiseNew)
 *                                  src/mdcore/src/bond.cpp:892-942
 *   mxg_engine_group_metrics       MxParticles_CenterOfMass / _CenterOfGeometry / _RadiusOfGyration /
 *                                  _MomentOfInertia src/mdcore/src/metrics.cpp:330-466 (the
 *                                  MxParticleList methods, MxParticleList.cpp:406-458)
 *   mxg_engine_add_exclusions      engine_exclusion_add src/mdcore/src/engine_bonded.cpp:1277-1310
 *   mxg_engine_exclusion_shrink    engine_exclusion_shrink src/mdcore/src/engine_bonded.cpp:1235-1262
 *   mxg_engine_adddihedrals        engine_dihedral_addpot + engine_dihedral_add
 *                                  src/mdcore/src/engine_bonded.cpp:1049-1080, 1967-1991
 *   mxg_engine_start               engine_start             src/mdcore/include/engine.h:640
 *   mxg_engine_step                engine_step              src/mdcore/src/engine.cpp:1198
 *   mxg_engine_force               engine_force             src/mdcore/src/engine.cpp:1230
 *   mxg_engine_step_timed          engine_step with the engine timers (engine.h:113-135)
 *   mxg_engine_add_cuboid          engine_addcuboid         src/mdcore/src/engine.cpp:1742
 *   mxg_engine_set_cuboid_potential engine_add_cuboid_potential src/mdcore/src/engine.cpp:1816
 *   mxg_engine_number_density      MxParticle::f[3]: space_prepare's self term (space.cpp:216-236) plus
 *                                  the runners' W(r2, cutoff) per pair (runner_dopair.cpp:194-203)
 *   mxg_engine_load                engine_load              src/mdcore/include/engine.h:612
 *   mxg_engine_unload              engine_unload            src/mdcore/include/engine.h:646
 *   mxg_engine_kinetic_energy      engine_kinetic_energy    src/mdcore/src/engine.cpp:1698
 *   mxg_engine_finalize            engine_finalize          src/mdcore/src/engine.cpp:1418
 *
 * Conventions (as engine.h:33-63): every call returns int, 0 on success and a
 * negative engine_err_* value on failure. GPU-specific failures use the codes
 * below -100. Only plain pointers and sizes cross the boundary; device state
 * stays resident between calls. A CUDA stream may be supplied; all device
 * work of an engine is ordered on that stream.
 */
#ifndef MXG_H_
#define MXG_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes (values of the reference's engine_err_*) */
#define MXG_OK 0
#define MXG_ERR_NULL -1
#define MXG_ERR_MALLOC -2
#define MXG_ERR_SPACE -3
#define MXG_ERR_RANGE -6
#define MXG_ERR_CELL -7
#define MXG_ERR_BOND -11
#define MXG_ERR_POTENTIAL -17
#define MXG_ERR_CUDA -21
#define MXG_ERR_NOCUDA -22
#define MXG_ERR_TOOFAST -29
/* GPU-specific status codes */
#define MXG_ERR_CELL_OVERFLOW -101 /* kept for ABI stability: no longer raised (any number of particles may
                                      enter a cell in one step) */
#define MXG_ERR_NONFINITE -102     /* a position or velocity became NaN/Inf */
#define MXG_ERR_STATE -103         /* call made in the wrong engine state */
#define MXG_ERR_ARG -104           /* invalid argument */

/* potential kinds */
#define MXG_POTENTIAL_TABLE 0
#define MXG_POTENTIAL_DPD 1

/* potential flags (src/mdcore/include/MxPotential.h:52-96) */
#define MXG_POTENTIAL_LJ126 (1u << 0)
#define MXG_POTENTIAL_R2 (1u << 4)
#define MXG_POTENTIAL_R (1u << 5)
#define MXG_POTENTIAL_HARMONIC (1u << 7)
#define MXG_POTENTIAL_SCALED (1u << 11)
#define MXG_POTENTIAL_SHIFTED (1u << 12)

/* boundary kinds per face (src/mdcore/src/MxBoundaryConditions.hpp:15-23) */
#define MXG_BOUNDARY_VELOCITY (1 << 0)
#define MXG_BOUNDARY_PERIODIC (1 << 1)
#define MXG_BOUNDARY_FREESLIP (1 << 2)
#define MXG_BOUNDARY_POTENTIAL (1 << 3) /* with FREESLIP: the "potential" kind */
#define MXG_BOUNDARY_NO_SLIP (1 << 4)

/* faces, in the order the bc arrays use */
#define MXG_FACE_LEFT 0   /* -x */
#define MXG_FACE_RIGHT 1  /* +x */
#define MXG_FACE_FRONT 2  /* -y */
#define MXG_FACE_BACK 3   /* +y */
#define MXG_FACE_BOTTOM 4 /* -z */
#define MXG_FACE_TOP 5    /* +z */

/* particle dynamics (src/mdcore/include/MxParticle.h:48-49) */
#define MXG_NEWTONIAN 0
#define MXG_OVERDAMPED 1

/* particle flags (src/mdcore/include/MxParticle.h:54-70) */
#define MXG_PARTICLE_FROZEN_X (1u << 2)
#define MXG_PARTICLE_FROZEN_Y (1u << 3)
#define MXG_PARTICLE_FROZEN_Z (1u << 4)

typedef struct mxg_potential mxg_potential;
typedef struct mxg_engine mxg_engine;

/* ---- potentials: host-side table fit (FP64 fit, FP32 coefficients) ---- */
int mxg_potential_create_lj126(double a, double b, double A, double B, double tol, mxg_potential **out);
int mxg_potential_create_morse(double d, double alpha, double r0, double min, double max, double tol,
                               mxg_potential **out);
int mxg_potential_create_harmonic(double k, double r0, double min, double max, double tol, mxg_potential **out);
int mxg_potential_create_power(double k, double r0, double alpha, double min, double max, double tol,
                               mxg_potential **out);
/* k (acos(c) - theta0)^2 tabulated in c = cos(theta) on [cos(max), cos(min)], min clipped to >= 0 and
 * max to <= pi, fitted without an analytic derivative (Potential.harmonic_angle,
 * src/mdcore/src/MxPotential.cpp:2577-2590, 557-594). */
int mxg_potential_create_harmonic_angle(double k, double theta0, double min, double max, double tol,
                                        mxg_potential **out);
/* k (1 + cos(n phi - delta)) tabulated in c = cos(phi) on [-1, 1] (pulled in by sqrt(FLT_EPSILON) when
 * delta is not a multiple of pi), n >= 1, fitted without an analytic derivative
 * (Potential.harmonic_dihedral, src/mdcore/src/MxPotential.cpp:2595-2607, 423-516). */
int mxg_potential_create_harmonic_dihedral(double k, int n, double delta, double tol, mxg_potential **out);
int mxg_potential_create_dpd(double alpha, double gamma, double sigma, double cutoff, int shifted,
                             mxg_potential **out);
/* Table description: kind, flags, intervals n, interval map alpha[4], domain [a,b], r0+1. */
int mxg_potential_info(const mxg_potential *p, int *kind, unsigned *flags, int *n, float *alpha4, float *a,
                       float *b, float *r0_plusone);
/* Copies the (n+1)*8 FP32 coefficients; returns their count or -(needed) if cap is short. */
int mxg_potential_coeffs(const mxg_potential *p, float *out, int cap);
/* DPD parameters (alpha, gamma, sigma). */
int mxg_potential_dpd_params(const mxg_potential *p, float *alpha, float *gamma, float *sigma);
/* Host scalar evaluation with potential_eval_ex semantics: returns 1 if in range. */
int mxg_potential_eval(const mxg_potential *p, float ri, float rj, float r2, float *e, float *f);
void mxg_potential_free(mxg_potential *p);
/* Frozen-node re-fit of a table potential at new construction parameters (layout as in
 * mxg_engine_set_pot_params); the interval count, map and nodes stay those of the first fit. For a
 * DPD potential the three coefficients change (cutoff and shift flag must stay). */
int mxg_potential_refit(mxg_potential *p, const double *params, int nparams);
/* The table's coefficients before their rounding to float (FP64, same layout as
 * mxg_potential_coeffs); returns their number. No counterpart in the reference. */
int mxg_potential_coeffs64(const mxg_potential *p, double *out, int cap);
/* The construction parameters of a potential (layout as in mxg_engine_set_pot_params); returns
 * their number, copying at most cap into out (out may be NULL). */
int mxg_potential_params(const mxg_potential *p, double *out, int cap);
/* The table (same nodes, map and interval count) of dV/dtheta_k for construction parameter k of a
 * table potential: LJ A (k=2), B (3); Morse d (0), alpha (1); harmonic k (0), r0 (1). Returns
 * MXG_ERR_ARG for parameters that do not change the tabulated function (Morse r0 only shifts the
 * argument). No counterpart in the reference. */
int mxg_potential_param_table(const mxg_potential *p, int k, mxg_potential **out);

/* ---- engine ---- */
/* bc_kind[6]: MXG_BOUNDARY_* per face (faces above); bc_velocity[18]: wall velocity per face for
 * velocity boundaries; bc_restore[6]: restitution per face. Cells are raised to 3 along periodic
 * axes as the reference does. */
int mxg_engine_init(const double *origin, const double *dim, const int *cells, double cutoff, const int *bc_kind,
                    const float *bc_velocity, const float *bc_restore, int max_type, unsigned flags,
                    mxg_engine **out);
/* ---- independent replicas in one engine (batched ensembles) ---- */
/* Adds another simulation box with its own geometry and boundaries to the engine (before
 * mxg_engine_start); returns its replica index. mxg_engine_init creates replica 0. All replicas
 * share the cutoff, dt, particle types and pruning mode; each has its own potentials per type pair,
 * particles and cell grid, and every step advances all of them with the same kernel launches.
 * No counterpart in the reference, which holds one engine per process (engine.h:708). */
int mxg_engine_add_replica(mxg_engine *e, const double *origin, const double *dim, const int *cells,
                           const int *bc_kind, const float *bc_velocity, const float *bc_restore);
int mxg_engine_nr_replicas(const mxg_engine *e);
/* engine_addpot / engine_addpart for one replica (the plain forms act on replica 0). */
int mxg_engine_addpot_replica(mxg_engine *e, int replica, const mxg_potential *p, int type_i, int type_j);
int mxg_engine_addparts_replica(mxg_engine *e, int replica, int n, const double *x, const float *v,
                                const int *type, int *ids_out);
/* A second potential on a type pair, summed with the pair's first one (a table potential plus a
 * DPD thermostat, say); each term keeps its own cutoff and table. No counterpart in the reference,
 * whose engine_addpot keeps one potential per type pair (engine.cpp:968-977). */
int mxg_engine_addpot_second(mxg_engine *e, int replica, const mxg_potential *p, int type_i, int type_j);
/* The engine's index of the potential bound to (type_i, type_j) of a replica: which = 0 for the
 * pair's potential, 1 for the summed second one; -1 in *idx when there is none. */
int mxg_engine_pot_index(mxg_engine *e, int replica, int type_i, int type_j, int which, int *idx);
/* New construction parameters for the engine's potential idx (the layout the create call takes,
 * minus the trailing output: LJ (a, b, A, B, tol), Morse (d, alpha, r0, min, max, tol), harmonic
 * (k, r0, min, max, tol), DPD (alpha, gamma, sigma, cutoff, shifted)). Tables are re-fitted on their
 * frozen nodes (same interval count and map), so a table's coefficients are a linear function of
 * the sampled potential and parameter derivatives are exact for the tabulated model; on a started
 * engine the device copy is updated in place, ordered on the engine stream. No counterpart in the
 * reference. */
int mxg_engine_set_pot_params(mxg_engine *e, int idx, const double *params, int nparams);
/* Chooses the force kernel's tile shape (own and neighbour particles staged per region: 32/96,
 * 32/64, 64/96 or 32/128) and grid (CTAs per SM) by timing candidate launches on the current state,
 * so the choice follows the state's density; returns the chosen blocks per SM. Call after
 * mxg_engine_start. Tile shapes differ in the order of the FP32 force sums, so two engines compare
 * bit for bit only with the same configuration (mxg_engine_force_config). No counterpart in the
 * reference. */
int mxg_engine_autotune(mxg_engine *e);
/* set = 0: reads the force kernel's tile variant (0-3) and grid (CTAs); set = 1: pins them (after
 * mxg_engine_start; the grid is clamped to the blocks the work items can occupy and written back;
 * the step graphs are re-captured). */
int mxg_engine_force_config(mxg_engine *e, int *variant, int *grid, int set);

/* dt, max-distance fraction (reference default 0.05) */
int mxg_engine_set_dt(mxg_engine *e, double dt, double max_dist_fraction);
/* Returns the new type id (>= 0). */
int mxg_engine_addtype(mxg_engine *e, double mass, double radius, int dynamics, unsigned particle_flags);
int mxg_engine_addpot(mxg_engine *e, const mxg_potential *p, int type_i, int type_j);
int mxg_engine_add_singlebody_force(mxg_engine *e, int type, float fx, float fy, float fz);
/* The other single-body forces of the forces module (engine_add_singlebody_force, engine.cpp:983-1003,
 * with the forces of src/mdcore/src/MxForce.cpp:308-419); like the reference, a type keeps one.
 *   kind 2, Berendsen thermostat (berenderson_tstat): params {tau}; f += (1/tau)(T0/KE_type - 1) v with
 *          KE_type the type's summed kinetic energy (see mxg_engine_set_target_temperature for T0);
 *   kind 3, random (random): params {mean, std, duration}; a persistent force N(mean, std) in a uniformly
 *          random direction, redrawn every ceil(duration/dt) steps (when time + id is a multiple);
 *   kind 4, friction (friction): params {coef, mean, std, duration}; f += -coef |v|^2 v + a persistent
 *          random force as for kind 3.
 * The random draws come from a Philox stream keyed on (time, particle id) instead of the reference's
 * global mt19937. */
int mxg_engine_add_singlebody_force_kind(mxg_engine *e, int type, int kind, const float *params);
/* The type's target temperature (MxParticle.cpp:543-560), which the Berendsen force compares with the
 * type's summed kinetic energy. */
int mxg_engine_set_target_temperature(mxg_engine *e, int type, double temperature);
/* Adds n particles (positions double[3n] in global coordinates, velocities float[3n]); ids_out
 * receives consecutive ids (may be NULL). */
int mxg_engine_addparts(mxg_engine *e, int n, const double *x, const float *v, const int *type, int *ids_out);
/* Adds particles of replica rep by cell (replica-local index, as the engine numbers cells: x-major)
 * and FP32 cell-relative position, kept exactly as given (space_cell's own representation, the
 * state the re-binning leaves): a state taken from another engine with the same space continues
 * bit for bit. Used to hand particles between slabs of a decomposed box. No counterpart call in
 * the reference (its particles enter through engine_addpart's global positions). */
int mxg_engine_addparts_cellrel(mxg_engine *e, int rep, int n, const int *cell, const float *xrel, const float *v,
                                const int *type, int *ids_out);
/* Before mxg_engine_start: the particle count on which the force pass's work-item split (cells split
 * into several items when they are too few to fill the GPU, finer when the mean occupancy is 16 or
 * more) is decided, instead of this engine's own; 0 restores the default. A slab of a decomposed box
 * passes the whole box's count, so that its cells are split, and their sums ordered, as in the
 * undivided box. */
int mxg_engine_set_occupancy_hint(mxg_engine *e, long long nparts);
/* Adds n harmonic/table bonds between particle ids i[k], j[k], all with potential p. */
int mxg_engine_addbonds(mxg_engine *e, int n, const int *i, const int *j, const mxg_potential *p,
                        double dissociation_energy, int *ids_out);
/* Adds n angles i[q]-j[q]-k[q] (vertex j), all with table potential p in cos(theta), evaluated each
 * force pass after the bonds as angle_eval does (src/mdcore/src/angle.cpp:92-352); the vertex carries
 * the energy. ids_out receives consecutive angle indices (may be NULL). */
int mxg_engine_addangles(mxg_engine *e, int n, const int *i, const int *j, const int *k, const mxg_potential *p,
                         int *ids_out);
/* Adds n exclusions (i[q], j[q]): each force pass, before the bonds, the pair's table potential is
 * taken back as exclusion_eval does (src/mdcore/src/exclusion.cpp:83-282): dx = (x_i - x_j) + h shift,
 * kept within the cutoff, potential_eval without the radii shift, f_i += eff dx, f_j -= eff dx, its
 * energy subtracted; pairs
 * whose potential is DPD are skipped. Stored with i <= j (engine_exclusion_add). */
int mxg_engine_add_exclusions(mxg_engine *e, int n, const int *i, const int *j);
/* Sorts the exclusions and drops duplicates (engine_exclusion_shrink). */
int mxg_engine_exclusion_shrink(mxg_engine *e);
/* Adds n dihedrals i[q]-j[q]-k[q]-l[q], all with table potential p in cos(phi), evaluated each force pass
 * after the angles as dihedral_eval does (src/mdcore/src/dihedral.cpp:81-392): the forces on i, j and l
 * are balanced on k, which carries the energy. ids_out receives consecutive dihedral indices (may be NULL). */
int mxg_engine_adddihedrals(mxg_engine *e, int n, const int *i, const int *j, const int *k, const int *l,
                            const mxg_potential *p, int *ids_out);
/* Binds potential p between particles of `type` and a wall: face 0..5 (MXG_FACE_*) or -1 for all six
 * (MxBoundaryCondition::set_potential / MxBoundaryConditions::set_potential,
 * src/mdcore/src/MxBoundaryConditions.cpp:771-836). Evaluated for particles in cells next to a non-periodic
 * face as boundary_eval does (src/mdcore/src/boundary_eval.hpp:124-223): distance r to the face, kept when
 * r <= the potential's b; r^2 below the potential's a (sic, not a^2) is replaced by a^2 along the face
 * normal; tables get potential_eval_ex with wall radius 0, DPD potentials dpd_boundary_eval against the
 * wall velocity. */
int mxg_engine_set_boundary_potential(mxg_engine *e, int face, int type, const mxg_potential *p);
/* Adds a static cuboid to replica rep (engine_addcuboid, src/mdcore/src/engine.cpp:1742; Cuboid(pos, size,
 * orientation), src/mdcore/src/MxCuboid.cpp:40-76): centre pos (NULL: the box centre dim / 2, as
 * engine_center), size, orientation angles about x, y, z (the quaternion qx qy qz). Its bounding box is
 * formed as MxCuboid_UpdateAABB does (MxCuboid.cpp:190-221). id (may be NULL) receives its index. */
int mxg_engine_add_cuboid(mxg_engine *e, int rep, const float *pos, const float *size, const float *angles, int *id);
/* The potential between particles of a type and every cuboid (engine_add_cuboid_potential,
 * src/mdcore/src/engine.cpp:1816-1830; bind(pot, Cuboid, type), MxBind.cpp:67-73), evaluated per particle
 * as potential_eval_cuboid_particle (src/mdcore/src/cuboid_eval.hpp:73-188): the particle's distance from
 * the cuboid's centre along the axis of the face it is nearest to (inside) or above (outside), in the
 * cuboid's frame, through potential_eval_ex with r0 = half the size on that axis. No energy. */
int mxg_engine_set_cuboid_potential(mxg_engine *e, int type, const mxg_potential *p);
/* Cuboid id's geometry: out16 = centre[3], size[3], orientation quaternion (x, y, z, w), box min[3], max[3]. */
int mxg_engine_cuboid_info(const mxg_engine *e, int id, float *out16);
/* Species (chemical cargo) of a particle type: nspec values per particle (at most 8), flags per species
 * (bit 2: constant, SPECIES_KONSTANT: not integrated). Before mxg_engine_start. */
int mxg_engine_set_type_species(mxg_engine *e, int type, int nspec, const unsigned *flags);
/* A flux between types ta and tb on species ia (of ta) and ib (of tb) (MxFluxes_FluxEx,
 * src/mdcore/src/Flux.cpp:161-211): kind 0 Fick, k (s_a - s_b); 1 secrete, max(k (s_a - target), 0);
 * 2 uptake, max(k (target - s_b) s_a, 0); each times (1 - r/cutoff)^2 for every pair within the cutoff
 * (flux_eval_ex, src/mdcore/src/flux_eval.hpp:33-84); decay removes decay/2 s per pair from each side.
 * Both orders of a type pair share one list of at most 7 entries (MxFluxes_AddFlux, Flux.cpp:289-317).
 * After each forward-Euler step, values += dt * rates unless constant, for the particles that kept their
 * cell in that step; the others carry their rates to the next step (MxFluxes_Integrate, Flux.cpp:261-285,
 * run per cell after the cell's particles moved). Before mxg_engine_start. */
int mxg_engine_add_flux(mxg_engine *e, int kind, int ta, int tb, int ia, int ib, float k, float decay, float target);
/* Species values by particle id, values[id * smax + k] for the type's first nspec species. Before start
 * they are staged; after, they replace the device values. */
int mxg_engine_set_species(mxg_engine *e, int n, int smax, const float *values);
int mxg_engine_get_species(mxg_engine *e, int n, int smax, float *out);
/* The pair search of the pairwise bond constructor (make_pairlist, src/mdcore/src/bond.cpp:892-942), on
 * the device over the current state of a started engine: the pairs (ids[a], ids[b]), b < a, of the n
 * listed particles (one replica) whose global FP32 positions are within cutoff (|dx|^2 <= cutoff^2 summed
 * x, y, z, no periodic image) and whose types ti, tj have type_mask[ti * ntypes + tj] != 0 (type_mask may
 * be NULL: every pair of types; the reference's pair_check, bond.cpp:1134-1152), ordered by a, then b.
 * *count receives the number of pairs; out_i/out_j (may be NULL to query the count) receive them when
 * cap is large enough, else MXG_ERR_RANGE. */
int mxg_engine_pairs_within(mxg_engine *e, int n, const int *ids, float cutoff, const unsigned char *type_mask,
                            int ntypes, int *out_i, int *out_j, int cap, int *count);
/* Metrics of a particle group over the current state of a started engine (metrics.cpp:330-466): out[0]
 * total mass, out[1..3] centre of mass, out[4..6] centroid, out[7] radius of gyration (the reference's
 * sqrt of the summed distances to the centroid), out[8..16] moment of inertia about the centre of mass
 * (row-major; off-diagonals + sum m dx dy as in the reference). ids: n >= 1 particle ids. Sums in FP64. */
int mxg_engine_group_metrics(mxg_engine *e, int n, const int *ids, double *out);
/* Builds the cell-pair lists and uploads the state. stream may be NULL (default stream). */
int mxg_engine_start(mxg_engine *e, void *cuda_stream);
/* Runs nsteps forward-Euler steps on the device (forces, bonds, integrate, re-bin). */
int mxg_engine_step(mxg_engine *e, int nsteps);
/* nsteps steps launched one kernel at a time with CUDA events at the phase boundaries; ms[n] (n >= 15)
 * receives the summed milliseconds at the reference's timer ids (engine.h:113-135): 0 step, 1 prepare
 * (single-body and wall/large-particle passes), 4 nonbond, 5 bonded (with species fluxes), 11 advance,
 * 14 shuffle (re-binning); under Runge-Kutta 4 the whole step is counted as advance. */
int mxg_engine_step_timed(mxg_engine *e, int nsteps, double *ms, int n);
/* Computes forces (and energies) for the current positions without advancing. */
int mxg_engine_force(mxg_engine *e);
/* Waits for the engine's stream and returns the device status word as a status code. */
int mxg_engine_status(mxg_engine *e);
int mxg_engine_nr_parts(const mxg_engine *e);
int mxg_engine_nr_cells(const mxg_engine *e);
/* Per-id host copies: absolute positions (double[3n]), velocities, forces (float[3n]), cell index,
 * cell-relative positions. Any pointer may be NULL. */
int mxg_engine_unload(mxg_engine *e, int n, double *x, float *v, float *f, int *cell, float *xrel);
/* Per-id upload of positions (double[3n], global coordinates) and velocities (float[3n]; NULL keeps
 * each particle's velocity); particles are placed as engine_addpart would place them and ordered by
 * (cell, id), both on the device. A position outside its replica's box returns MXG_ERR_SPACE and
 * changes no state. Returns once the engine's stream has finished the load, so the host arrays
 * may be reused at once; the velocities cross on a second stream of the engine's while the
 * placement runs. */
int mxg_engine_load(mxg_engine *e, int n, const double *x, const float *v);
/* Potential energy (nonbonded + bonded) of the last force evaluation and the current kinetic energy,
 * both reduced in FP64 on the device. virial9 (may be NULL): the virial of the current positions,
 * reduced in FP64: the nonbonded pair sum of (x_first - x_second) (x) F_first (one extra force pass
 * that changes no engine state) plus the bonded terms' sum of (x_m - x_ref) (x) F_m (bonds active
 * after the last pass, exclusions, angles about their vertex, dihedrals about their j particle); the
 * reference's MxCalculateVirial returns zeros (metrics.cpp:183,246). */
int mxg_engine_energy(mxg_engine *e, double *epot, double *ekin, double *virial9);
double mxg_engine_kinetic_energy(mxg_engine *e);
/* Cell-pair task list rows (type, sid, i, j) as space_init builds them. */
int mxg_engine_tasks(const mxg_engine *e, int *out, int cap);
/* Bond flags (bit 0 = active); returns the number of bonds. */
int mxg_engine_bond_flags(mxg_engine *e, unsigned *out, int cap);
/* The number density of the particles for the current positions (the reference's
 * MxParticle::number_density, f[3], as a force pass leaves it: space_prepare's W(0, cutoff),
 * src/mdcore/src/space.cpp:216-236, plus W(r^2, cutoff) for every pair the pair loops reach
 * within the cutoff whose type pair has no potential and no flux, or whose potential evaluates
 * in range, src/mdcore/src/runner_dopair.cpp:194-203 and dpd_eval.hpp:133-166; W the cubic
 * spline of smoothing_kernel.hpp:37-56). out: float[n] by particle id (may be NULL); volume (may
 * be NULL): engine_advance's computed volume, the sum of 1 / number density
 * (engine_advance.cpp:184-185), in FP64. The reference forms r with a 12-bit reciprocal
 * square-root approximation; here r = sqrtf(r^2). Large particles, wall potentials and second
 * summed potentials add nothing. Synchronous. */
int mxg_engine_number_density(mxg_engine *e, int n, float *out, double *volume);
/* Replaces the bond flags (n = the number of bonds; bit 0 = active). The reference keeps the flag in
 * each bond (MxBond.flags, src/mdcore/include/bond.h:47-70) and re-creates destroyed bonds through
 * _bond_init (src/mdcore/src/bond.cpp:497); here a trajectory restarted from its first state
 * re-activates the bonds it had then. Ordered on the engine stream. */
int mxg_engine_set_bond_flags(mxg_engine *e, const unsigned *flags, int n);
/* The engine's index of bond k's potential (for mxg_engine_set_pot_params and
 * mxg_engine_adjoint_params). */
int mxg_engine_bond_pot_index(const mxg_engine *e, int k, int *idx);
/* Space description: cdim[3], h[3], nr_cells, period bitmask. */
int mxg_engine_space_info(const mxg_engine *e, int *cdim, double *h, int *nr_cells, unsigned *period);
/* Raw device-resident state in slot order (cell-sorted): pos float4 (xrel, type bits),
 * vel float4 (v, id bits), force float4, cell index per slot; device pointers. */
int mxg_engine_device_state(mxg_engine *e, void **pos, void **vel, void **force, void **cell);
/* Asynchronous copy of the raw slot-order state (pos, vel float4 arrays of nr_parts entries) between
 * host memory (pinned for full speed) and the device, ordered on the engine stream. The layout is the
 * device's own, so a download followed by an upload restores the state exactly. */
int mxg_engine_copy_state(mxg_engine *e, void *host_pos, void *host_vel, int to_device);
/* Enqueues the FP64 energy reduction and an asynchronous copy of (epot, ekin) into host_out2. */
int mxg_engine_energy_async(mxg_engine *e, double *host_out2);
int mxg_engine_finalize(mxg_engine *e);

/* ---- adjoint (reverse-mode gradients of trajectories) ---- No counterpart in the reference. ---- */
/* Bytes of a state snapshot (positions, velocities, cell lists, id map, step counter, bond flags, species
 * values and rates, persistent random single-body forces). */
int mxg_engine_snapshot_bytes(const mxg_engine *e, size_t *bytes);
/* save = 1: copies the current state into dev_buf (device memory, 16-byte aligned); save = 0: makes
 * dev_buf's state current. Ordered on the engine stream; restoring then stepping reproduces the
 * trajectory bit for bit (the step counter that keys the Philox streams is part of the state). */
int mxg_engine_snapshot(mxg_engine *e, void *dev_buf, int save);
/* Registers the differentiated parameters: entry k adds d loss / d (parameter param[k] of the
 * engine's potential pot[k]) into gradient slot slot[k] (< 16; several entries may share a slot).
 * Parameters use the construction layout of mxg_engine_set_pot_params: LJ A (2), B (3); Morse d (0),
 * alpha (1), r0 (2); harmonic k (0), r0 (1); DPD alpha (0), gamma (1), sigma (2). */
int mxg_engine_adjoint_params(mxg_engine *e, int n, const int *pot, const int *param, const int *slot);
/* Vector-Jacobian product of one step taken from the current state. lam_x, lam_v: device float4
 * arrays indexed by particle id, holding the adjoints of the positions and velocities after the step;
 * on return (stream-ordered) they hold the adjoints of the state before it. grad: device double array
 * of the gradient slots, to which the step's parameter terms are added. Periodic boxes, nonbonded
 * potentials (tables, DPD, summed pairs), bonds (bond_eval, src/mdcore/src/bond.cpp:99-312: the
 * table through its length clamp, harmonic k and r0 as parameters; break flags held fixed: a bond
 * broken before or during the step adds nothing) and constant forces; angles, dihedrals, exclusions,
 * wall potentials, large particles and Berendsen/random/friction forces are refused (MXG_ERR_ARG).
 * Wall reflections of the integrator are not differentiated. */
int mxg_engine_vjp_step(mxg_engine *e, void *lam_x, void *lam_v, double *grad);
/* mxg_engine_vjp_step with the forces of the current state given: forces is a device float4 array of
 * nr_parts entries in the current slot order, as mxg_engine_save_forces left it after the step taken
 * from this state. Without bonds the step's force pass is then not repeated (the forces are copied
 * in); with bonds (whose pass also decides the break flags) or forces NULL it is. The adjoint
 * workflow's recompute saves them anyway. */
int mxg_engine_vjp_step_forces(mxg_engine *e, void *lam_x, void *lam_v, double *grad, const void *forces);
/* Copies the forces of the last force pass (total forces, slot order of the state that pass ran on:
 * after mxg_engine_step, the state the step started from) into dev_buf (nr_parts float4), ordered on
 * the engine stream. */
int mxg_engine_save_forces(mxg_engine *e, void *dev_buf);
/* Device float4 arrays by particle id: absolute positions (x, y, z, type bits) and velocities
 * (v, id bits); either pointer may be NULL. Stream-ordered. */
int mxg_engine_positions(mxg_engine *e, void *x4, void *v4);
/* Sets the step counter that keys the Philox streams (after a load, to replay a trajectory). */
int mxg_engine_set_step_counter(mxg_engine *e, unsigned long long step);
/* Gaussian-smoothed pair histogram of particle types (type_a, type_b) in a periodic box:
 * hist[b] += 2^32 * sum over pairs (i of type_a, j of type_b, i != j) of K(r_ij - (b + 1/2) dr),
 * K a Gaussian of width sigma (normalised, minus its value at 4 sigma) cut at |r - centre| > 4 sigma, as uint64 fixed point (device array of
 * nbins <= 256; the sums do not depend on the order of the additions). With coef (device double per
 * bin) and grad4 (device float4 per particle): grad4[i] = d(sum_b coef[b] hist[b]) / d x_i, unscaled.
 * x4: device float4 (x, y, z, type bits) per particle; box: host double[3]. The workload's loss
 * (an A-B radial distribution) is built on it. No counterpart in the reference. */
int mxg_rdf(const void *x4, int n, const double *box, int type_a, int type_b, int nbins, double dr, double sigma,
            void *hist, const double *coef, void *grad4, void *stream);

/* The integrator (engine.h EngineIntegrator, set by universe_init from the `integrator` keyword,
 * src/MxSimulator.cpp:218-230): 0 forward Euler (engine_advance_forward_euler), 1 Runge-Kutta 4
 * (engine_advance_runge_kutta_4, engine_advance.cpp:443-698). Set before mxg_engine_start. The RK4
 * stages keep the step's cell frame (the reference re-bins between stages and leaves the stage
 * origin in the old cell's frame, so a particle crossing a face mid-step lands a cell edge away
 * there). */
int mxg_engine_set_integrator(mxg_engine *e, int kind);
/* DPD random term: 0 = reference semantics (xi = 1, dpd_eval.hpp:57), 1 = Philox stream keyed on
 * (step, particle id pair). Set before mxg_engine_start. */
int mxg_engine_set_rng_mode(mxg_engine *e, int mode);
/* Pair pruning of cell pairs as the reference's sorted loops do it (runner_dopair.cpp:132-182):
 * (a) a candidate pair is skipped when the quantised projections of the two particles on the pair's
 * sort axis, plus the shift length, differ by dmaxdist or more; with cubic cells this never drops a
 * pair inside the cutoff, with non-cubic cells it does; (b) the whole cell pair is skipped when the
 * largest key of its first cell and the smallest key of its second give a difference below zero
 * (unsigned wrap) or above dmaxdist, which happens when particles sit within one key quantum of the
 * shared face. mode 0 (default): (a) on non-cubic grids, (b) always -- the reference's result;
 * 1: (a) and (b) on every grid; 2: neither (every pair inside the cutoff). Set before start. */
int mxg_engine_set_pair_pruning(mxg_engine *e, int mode);
/* Clears the device status word. */
int mxg_engine_clear_status(mxg_engine *e);
/* Launches the nonbonded force kernel reps times back to back on the engine stream and returns the
 * mean CUDA-event duration of one launch in milliseconds (state is not advanced). */
int mxg_engine_time_force(mxg_engine *e, int reps, double *ms);

/* ---- timing of the force kernel (for roofline reporting) ---- */
/* reps launches of the nonbonded force kernel alone (with the occupancy ordering when the engine
 * uses it), each between its own pair of CUDA events on the engine stream, flush_bytes of device
 * memory at flush (may be NULL with 0 bytes) zeroed before every launch outside the events so that
 * each launch starts with a cold L2; ms[r] receives launch r's milliseconds. The forces of the
 * state are recomputed in full afterwards; the state is not advanced. */
int mxg_engine_time_force_launches(mxg_engine *e, int reps, void *flush, size_t flush_bytes, double *ms);
/* Pair statistics for the last force evaluation: candidate and interacting pair counts as the
 * reference's task list defines them (counted on the device when enabled). */
int mxg_engine_pair_counts(mxg_engine *e, long long *candidates, long long *interacting);

/* ---- allocation-free entry point ---- */
/* No counterpart in the reference. Kinetic energy of nparts particles, computed like
 * engine_kinetic_energy (float e = 0.5*mass*|v|^2 per particle, summed in FP64), for callers
 * that cannot call cudaMalloc -- an application whose device memory is reserved by another
 * allocator, or a latency-critical loop that must not take an allocation's implicit device
 * synchronisation. vel and pos are device arrays of nparts float4 in the engine's layout (pos.w
 * holds the type id bits, see mxg_engine_device_state); type_mass is a device array of ntypes
 * doubles; out is a device array of 1 + ntypes doubles receiving the total and the per-type sums.
 * Work is enqueued on stream (NULL = default stream). The reduction's scratch is a file-scope
 * device array of 256 x 64 doubles (128 KiB, held by every GPU that loads the library until the
 * process exits): ntypes above 64 is rejected with MXG_ERR_RANGE. Type ids outside [0, ntypes)
 * contribute nothing. The first call on a device looks the array's address up for that device
 * (cudaGetSymbolAddress); with CUDA's lazy module loading (the default since CUDA 12) that first
 * call, or the first launch, may also load this library's device code, which allocates device
 * memory for the code and the array and can synchronise the device: make the first call per device
 * during set-up, outside any allocation-free or latency-critical region and before any stream
 * capture. After it, calls allocate nothing: no cudaMalloc, cudaFree or allocating library routine
 * is called. Calls that overlap on the GPU share the array and race; serialise them. */
int mxg_kinetic_energy_noalloc(const void *vel, const void *pos, int nparts, const double *type_mass, int ntypes,
                               double *out, void *stream);

#ifdef __cplusplus
}
#endif
#endif
