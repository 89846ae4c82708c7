/*
 * C driver for the reference engine compiled in place (oracle tier A).
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/ and by bench.py's CPU baseline
 * leg to run the reference's own CPU code path; the product never loads it.
 *
 * Each entry point performs exactly what the reference's Python layer does
 * for the same user call, but without the Python object model:
 *   mxref_init            universe_init (src/MxSimulator.cpp:349-420)
 *   mxref_add_type        particle type defaults (src/MxParticle.cpp:1395-1420,
 *                         imass = 1/mass at :1266)
 *   mxref_add_particles   particle_init_ex (src/MxParticle.cpp:2062-2119);
 *                         positions pass through a float 3-vector first
 *   mxref_potential_*     the Potential factories (src/mdcore/src/MxPotential.cpp
 *                         :2459-2473 LJ, :2545-2559 harmonic, :2652-2667 Morse,
 *                         :2738-2750 DPD)
 *   mxref_bind            engine_addpot (src/mdcore/src/engine.cpp:960-981)
 *   mxref_bind_force      MxConstantForce + engine_add_singlebody_force
 *                         (src/mdcore/src/MxForce.cpp:508-519, engine.cpp:983-1003)
 *   mxref_add_bonds       _bond_init (src/mdcore/src/bond.cpp:497-529)
 *   mxref_add_angles      angle_init (src/mdcore/src/angle.cpp:659-707)
 *   mxref_pairwise        MxBond_PairwiseNew (src/mdcore/src/bond.cpp:944-989)
 *   mxref_add_flux        MxFluxes_FluxEx (src/mdcore/src/Flux.cpp:161-211)
 *   mxref_add_exclusions  engine_exclusion_add (src/mdcore/src/engine_bonded.cpp:1277-1310)
 *   mxref_set_species     the particles' species state vectors (values and flags)
 *   mxref_bind_boundary_potential  MxBoundaryCondition(s)::set_potential
 *                         (src/mdcore/src/MxBoundaryConditions.cpp:771-836)
 *   mxref_add_dihedrals   engine_dihedral_addpot + engine_dihedral_add
 *                         (src/mdcore/src/engine_bonded.cpp:1049-1080, 1967-1991)
 *   mxref_step            engine_step (src/mdcore/src/engine.cpp:1198)
 *   mxref_force           engine_force (src/mdcore/src/engine.cpp:1230)
 * The engine is a process-wide singleton in the reference, so one process
 * holds one reference engine; tests run each scenario in a fresh process.
 */
#include "mdcore_config.h"
#include "engine.h"
#include "MxParticle.h"
#include "MxPotential.h"
#include "DissapativeParticleDynamics.hpp"
#include "potential_eval.hpp"
#include "bond.h"
#include "angle.h"
#include "MxParticleList.hpp"
#include "Flux.hpp"
#include "CStateVector.hpp"
#include "task.h"
#include "MxForce.h"
#include "../../rendering/NOMStyle.hpp"
#include <vector>
#include <cstring>
#include <limits>
#include <algorithm>
#include <cmath>
#include "MxCuboid.hpp"

extern PyTypeObject MxConstantForce_Type;
extern PyTypeObject MxAngle_Type;
extern PyTypeObject MxBondHandle_Type;
MxPotential *potential_create_morse(double d, double a, double r0, double min, double max, double tol);
MxPotential *potential_create_power(double k, double r0, double alpha, double a, double b, double tol);

static std::vector<NOMStyle *> g_styles;

extern "C" {

int mxref_init(const double *origin, const double *dim, const int *cells_in, double cutoff,
               const char *bc_x, const char *bc_y, const char *bc_z, double dt,
               double max_distance, int nr_types_max) {
    if (engine::types == NULL) {
        engine::types = (MxParticleType *)calloc(engine::max_type, sizeof(MxParticleType));
        engine::nr_types = 0;
    }
    int cells[3] = {cells_in[0], cells_in[1], cells_in[2]};
    PyObject *bc = PyDict_New();
    PyObject *sx = PyUnicode_FromString(bc_x), *sy = PyUnicode_FromString(bc_y), *sz = PyUnicode_FromString(bc_z);
    PyDict_SetItemString(bc, "x", sx);
    PyDict_SetItemString(bc, "y", sy);
    PyDict_SetItemString(bc, "z", sz);
    Py_DECREF(sx); Py_DECREF(sy); Py_DECREF(sz);
    int rc = engine_init(&_Engine, origin, dim, cells, cutoff, bc, nr_types_max, engine_flag_none);
    if (rc != 0) return rc;
    _Engine.dt = dt;
    _Engine.temperature = 1;
    _Engine.integrator = EngineIntegrator::FORWARD_EULER;
    if (max_distance >= 0) _Engine.particle_max_dist_fraction = max_distance / _Engine.s.h[0];
    return 0;
}

int mxref_add_type(double mass, double radius, int dynamics) {
    int id = engine::nr_types;
    if (id >= engine::max_type) return -1;
    MxParticleType *t = &engine::types[id];
    bzero(t, sizeof(MxParticleType));
    t->id = id;
    t->mass = mass;
    t->imass = 1.0 / mass;
    t->radius = radius;
    t->minimum_radius = 0.0;
    t->dynamics = (unsigned char)dynamics;
    NOMStyle *st = (NOMStyle *)calloc(1, sizeof(NOMStyle));
    st->flags = STYLE_VISIBLE;
    g_styles.push_back(st);
    t->style = st;
    engine::nr_types = id + 1;
    return id;
}

/* Adds n particles; x and v are n*3 arrays; returns the id of the first. */
int mxref_add_particles(int n, const double *x, const double *v, const int *type) {
    int first = -1;
    for (int k = 0; k < n; ++k) {
        MxParticleType *t = &engine::types[type[k]];
        MxParticle part;
        bzero(&part, sizeof(MxParticle));
        part.radius = t->radius;
        part.mass = t->mass;
        part.imass = t->imass;
        part.id = engine_next_partid(&_Engine);
        part.typeId = t->id;
        part.flags = t->particle_flags;
        part.creation_time = _Engine.time;
        part.clusterId = -1;
        part.position = Magnum::Vector3((float)x[3 * k], (float)x[3 * k + 1], (float)x[3 * k + 2]);
        part.velocity = Magnum::Vector3((float)v[3 * k], (float)v[3 * k + 1], (float)v[3 * k + 2]);
        if (part.radius > _Engine.s.cutoff) part.flags |= PARTICLE_LARGE;
        MxParticle *p = NULL;
        double pos[] = {part.position[0], part.position[1], part.position[2]};
        int rc = engine_addpart(&_Engine, &part, pos, &p);
        if (rc < 0) return rc;
        if (first < 0) first = p->id;
        p->clusterId = -1;
    }
    return first;
}

void *mxref_potential_lj126(double a, double b, double A, double B, double tol) {
    return potential_create_LJ126(a, b, A, B, tol);
}
void *mxref_potential_morse(double d, double a, double r0, double min, double max, double tol) {
    return potential_create_morse(d, a, r0, min, max, tol);
}
void *mxref_potential_harmonic(double k, double r0, double min, double max, double tol) {
    return potential_create_harmonic(min, max, k, r0, tol);
}
/* Potential.harmonic_angle(k, theta0, min, max, tol) (MxPotential.cpp:2577-2590) */
void *mxref_potential_harmonic_angle(double k, double theta0, double min, double max, double tol) {
    return potential_create_harmonic_angle(min, max, k, theta0, tol);
}
void *mxref_potential_power(double k, double r0, double alpha, double min, double max, double tol) {
    return potential_create_power(k, r0, alpha, min, max, tol);
}
void *mxref_potential_dpd(double alpha, double gamma, double sigma, double cutoff, int shifted) {
    return DPDPotential_New((float)alpha, (float)gamma, (float)sigma, (float)cutoff, shifted != 0);
}

int mxref_potential_info(void *vp, int *n, float *alpha4, float *a, float *b, unsigned *flags,
                         float *r0_plusone, int *kind) {
    MxPotential *p = (MxPotential *)vp;
    if (!p) return -1;
    *n = p->n;
    for (int k = 0; k < 4; ++k) alpha4[k] = p->alpha[k];
    *a = p->a;
    *b = p->b;
    *flags = p->flags;
    *r0_plusone = p->r0_plusone;
    *kind = (int)p->kind;
    return 0;
}

int mxref_potential_coeffs(void *vp, float *out, int cap) {
    MxPotential *p = (MxPotential *)vp;
    int len = (p->n + 1) * potential_chunk;
    if (!p->c) return 0;
    if (cap < len) return -len;
    memcpy(out, p->c, sizeof(float) * len);
    return len;
}

int mxref_dpd_params(void *vp, float *alpha, float *gamma, float *sigma) {
    DPDPotential *p = (DPDPotential *)vp;
    *alpha = p->alpha;
    *gamma = p->gamma;
    *sigma = p->sigma;
    return 0;
}

/* The reference's inline table evaluators, called on scalars. */
int mxref_potential_eval_ex(void *vp, float ri, float rj, float r2, float *e, float *f) {
    return potential_eval_ex((MxPotential *)vp, ri, rj, r2, e, f) ? 1 : 0;
}
void mxref_potential_eval(void *vp, float r2, float *e, float *f) {
    potential_eval((MxPotential *)vp, r2, e, f);
}

int mxref_bind(void *pot, int ti, int tj) { return engine_addpot(&_Engine, (MxPotential *)pot, ti, tj); }

int mxref_bind_force(int type, float fx, float fy, float fz) {
    if (PyType_Ready(&MxForce_Type) < 0 || PyType_Ready(&MxConstantForce_Type) < 0) return -1;
    PyObject *obj = PyType_GenericAlloc(&MxConstantForce_Type, 0);
    if (!obj) return -1;
    PyObject *val = Py_BuildValue("[fff]", fx, fy, fz);
    PyObject *args = PyTuple_Pack(1, val);
    int rc = MxConstantForce_Type.tp_init(obj, args, NULL);
    Py_DECREF(args);
    Py_DECREF(val);
    if (rc != 0) return -1;
    return engine_add_singlebody_force(&_Engine, (MxForce *)obj, type, -1);
}

extern "C" PyObject *mxref_make_berendsen(float tau);
extern "C" PyObject *mxref_make_random(float std, float mean, float durration);
extern "C" PyObject *mxref_make_friction(float coef, float std, float mean, float durration);

/* The other single-body forces of MxForce.cpp:308-419 (berendsen_force,
 * gaussian_force, friction_force), created as the forces module creates them
 * (MxForce.cpp:213-259) and bound with engine_add_singlebody_force
 * (engine.cpp:983-1003), with the module's arguments:
 * kind 1: berenderson_tstat(a = tau); 2: random(a = std, b = mean, c = durration);
 * 3: friction(a = coef, b = std, c = mean, d = durration). */
int mxref_bind_singlebody(int type, int kind, float a, float b, float c, float d) {
    // engine_add_singlebody_force type-checks against MxConstantForce_Type
    if (PyType_Ready(&MxForce_Type) < 0 || PyType_Ready(&MxConstantForce_Type) < 0) return -1;
    PyObject *obj = kind == 1 ? mxref_make_berendsen(a) : kind == 2 ? mxref_make_random(a, b, c)
                                                                    : mxref_make_friction(a, b, c, d);
    if (!obj) return -1;
    return engine_add_singlebody_force(&_Engine, (MxForce *)obj, type, -1);
}

/* The type's target temperature, which berendsen_force compares with the type's
 * summed kinetic energy (MxParticle.cpp:543-560). */
int mxref_set_target_temperature(int type, double t) {
    if (type < 0 || type >= engine::nr_types) return -1;
    engine::types[type].target_energy = t;
    return 0;
}

int mxref_add_bonds(int n, const int *pi, const int *pj, void *pot, double dissociation) {
    for (int k = 0; k < n; ++k) {
        MxBond *bond = NULL;
        int id = engine_bond_alloc(&_Engine, &bond);
        if (id < 0) return id;
        bond->flags = 0;
        bond->i = pi[k];
        bond->j = pj[k];
        bond->half_life = 0;
        bond->dissociation_energy = dissociation;
        bond->style = NULL;
        if (bond->i >= 0 && bond->j >= 0) {
            bond->flags |= BOND_ACTIVE;
            _Engine.nr_active_bonds++;
        }
        bond->potential = (MxPotential *)pot;
    }
    return 0;
}

/* Angle(potential, p1, p2, p3) (src/mdcore/src/angle.cpp:659-707): an engine-owned
 * record from engine_angle_alloc (engine_bonded.cpp:1087-1129) holding the three
 * ids and the potential. */
int mxref_add_angles(int n, const int *pi, const int *pj, const int *pk, void *pot) {
    if (PyType_Ready(&MxAngle_Type) < 0) return -1;
    for (int k = 0; k < n; ++k) {
        MxAngle *a = NULL;
        int rc = engine_angle_alloc(&_Engine, &MxAngle_Type, &a);
        if (rc < 0) return rc;
        a->i = pi[k];
        a->j = pj[k];
        a->k = pk[k];
        a->potential = (MxPotential *)pot;
    }
    return 0;
}

/* The angle part of the last bonded pass (s->epot_angle, engine_bonded.cpp:1525-1528). */
double mxref_epot_angle(void) { return _Engine.s.epot_angle; }

/* Potential.harmonic_dihedral(k, n, delta, tol) (MxPotential.cpp:2595-2607) */
void *mxref_potential_harmonic_dihedral(double k, int n, double delta, double tol) {
    return potential_create_harmonic_dihedral(k, n, delta, tol);
}

/* engine_dihedral_addpot (engine_bonded.cpp:1967-1991) once, then engine_dihedral_add
 * (engine_bonded.cpp:1049-1080) per dihedral i-j-k-l. */
int mxref_add_dihedrals(int n, const int *pi, const int *pj, const int *pk, const int *pl, void *pot) {
    int pid = engine_dihedral_addpot(&_Engine, (MxPotential *)pot);
    if (pid < 0) return pid;
    for (int q = 0; q < n; ++q) {
        int rc = engine_dihedral_add(&_Engine, pi[q], pj[q], pk[q], pl[q], pid);
        if (rc < 0) return rc;
    }
    return 0;
}

double mxref_epot_dihedral(void) { return _Engine.s.epot_dihedral; }

/* The pairwise bond constructor, MxBond_PairwiseNew (src/mdcore/src/bond.cpp:944-989), on a
 * particle list of n ids with potential pot; npairs (a[q], b[q]) type pairs restrict the bonded
 * types as Universe.bind_pairwise's pairs argument does (none: every pair). The new bonds are
 * appended to the engine's bond array; returns their number or a negative status. */
int mxref_pairwise(int n, const int *ids, float cutoff, void *pot, int npairs, const int *ta, const int *tb) {
    if (PyType_Ready(&MxBondHandle_Type) < 0) return -1;
    MxParticleList list;
    memset((void *)&list, 0, sizeof(list));
    std::vector<int32_t> parts(ids, ids + n);
    list.parts = parts.data();
    list.nr_parts = n;
    list.size_parts = n;
    PyObject *pairs = NULL;
    if (npairs > 0) {
        pairs = PyList_New(npairs);
        for (int q = 0; q < npairs; ++q)
            PyList_SET_ITEM(pairs, q, PyTuple_Pack(2, (PyObject *)&engine::types[ta[q]],
                                                   (PyObject *)&engine::types[tb[q]]));
    }
    const int before = _Engine.nr_bonds;
    PyObject *args = PyTuple_New(0);
    PyObject *bonds = MxBond_PairwiseNew((MxPotential *)pot, &list, cutoff, pairs, args, NULL);
    Py_DECREF(args);
    // the pair list is kept: its tuples hold the engine's type records, which
    // are plain structs here and must never reach a zero reference count
    if (!bonds) return -1;
    Py_DECREF(bonds);
    return _Engine.nr_bonds - before;
}

/* bind(pot, boundary condition, type) (src/mdcore/src/MxBind.cpp:74-96): face 0..5 in the order left,
 * right, front, back, bottom, top (MxBoundaryCondition::set_potential), or -1 for all six
 * (MxBoundaryConditions::set_potential). */
int mxref_bind_boundary_potential(int face, int type, void *pot) {
    if (type < 0 || type >= engine::nr_types) return -1;
    MxBoundaryConditions &bc = _Engine.boundary_conditions;
    MxBoundaryCondition *faces[6] = {&bc.left, &bc.right, &bc.front, &bc.back, &bc.bottom, &bc.top};
    MxParticleType *t = &engine::types[type];
    if (face < 0)
        bc.set_potential(t, (MxPotential *)pot);
    else if (face < 6)
        faces[face]->set_potential(t, (MxPotential *)pot);
    else
        return -1;
    return 0;
}

/* One flux between types ta and tb on their species ia and ib, as MxFluxes_FluxEx
 * (src/mdcore/src/Flux.cpp:161-211) registers it without the species-name lookup:
 * kind 0 Fick, 1 secrete, 2 uptake; one MxFluxes object shared by (ta, tb) and (tb, ta). */
int mxref_add_flux(int kind, int ta, int tb, int ia, int ib, float k, float decay, float target) {
    if (ta < 0 || tb < 0 || ta >= engine::nr_types || tb >= engine::nr_types) return -1;
    const int i1 = _Engine.max_type * ta + tb, i2 = _Engine.max_type * tb + ta;
    MxFluxes *f = _Engine.fluxes[i1];
    if (!f) f = MxFluxes_New(8);
    if (!f) return -2;
    f = MxFluxes_AddFlux((FluxKind)kind, f, (int16_t)ta, (int16_t)tb, ia, ib, k, decay, target);
    _Engine.fluxes[i1] = f;
    _Engine.fluxes[i2] = f;
    return 0;
}

/* Species state vectors (values, zero rates, the type's per-species flags) for particles
 * 0..n-1: nspec[type] species each, values[id * smax + k], flags[type * smax + k]. */
int mxref_set_species(int n, int smax, const int *nspec, const unsigned *flags, const float *values) {
    space *s = &_Engine.s;
    for (int id = 0; id < n; ++id) {
        MxParticle *p = id < s->nr_parts ? s->partlist[id] : NULL;
        if (!p) continue;
        const int ns = nspec[p->typeId];
        if (ns <= 0) continue;
        CStateVector *sv = new CStateVector();
        sv->size = ns;
        sv->fvec = new float[ns];
        sv->q = new float[ns]();
        sv->species_flags = new uint32_t[ns];
        for (int k = 0; k < ns; ++k) {
            sv->fvec[k] = values[(size_t)id * smax + k];
            sv->species_flags[k] = flags[(size_t)p->typeId * smax + k];
        }
        p->state_vector = sv;
    }
    return 0;
}

/* Species values by particle id (out[id * smax + k]); missing entries are left alone. */
int mxref_get_species(int n, int smax, float *out) {
    space *s = &_Engine.s;
    for (int id = 0; id < n; ++id) {
        MxParticle *p = id < s->nr_parts ? s->partlist[id] : NULL;
        if (!p || !p->state_vector) continue;
        for (int k = 0; k < p->state_vector->size && k < smax; ++k) out[(size_t)id * smax + k] = p->state_vector->fvec[k];
    }
    return 0;
}

/* engine_exclusion_add (src/mdcore/src/engine_bonded.cpp:1277-1310) for n pairs. */
int mxref_add_exclusions(int n, const int *pi, const int *pj) {
    for (int q = 0; q < n; ++q) {
        int rc = engine_exclusion_add(&_Engine, pi[q], pj[q]);
        if (rc < 0) return rc;
    }
    return 0;
}

/* Particle ids of the engine's bonds in creation order. */
int mxref_bond_ids(int *bi, int *bj, int cap) {
    for (int k = 0; k < _Engine.nr_bonds && k < cap; ++k) {
        bi[k] = _Engine.bonds[k].i;
        bj[k] = _Engine.bonds[k].j;
    }
    return _Engine.nr_bonds;
}

int mxref_start(int nr_runners) { return engine_start(&_Engine, nr_runners, nr_runners); }

int mxref_step(int nsteps) {
    for (int k = 0; k < nsteps; ++k) {
        int rc = engine_step(&_Engine);
        if (rc != 0) return rc;
    }
    return 0;
}

int mxref_force(void) { return engine_force(&_Engine); }

/* EngineIntegrator (engine.h): 0 forward Euler, 1 Runge-Kutta 4, as universe_init sets it
 * from the integrator keyword (src/MxSimulator.cpp:218-230,380). */
int mxref_set_integrator(int kind) {
    _Engine.integrator = kind == 1 ? EngineIntegrator::RUNGE_KUTTA_4 : EngineIntegrator::FORWARD_EULER;
    return 0;
}

int mxref_nr_parts(void) { return _Engine.s.nr_parts; }

/* Per-id state: cell-relative position, absolute position (double), velocity,
 * force, cell index and type. Missing ids get cell = -1. */
int mxref_get_state(int n, float *xrel, double *xabs, float *v, float *f, int *cell, int *type) {
    space *s = &_Engine.s;
    for (int id = 0; id < n; ++id) {
        MxParticle *p = id < s->nr_parts ? s->partlist[id] : NULL;
        if (!p) { cell[id] = -1; continue; }
        space_cell *c = s->celllist[id];
        cell[id] = (int)(c - s->cells);
        type[id] = p->typeId;
        for (int k = 0; k < 3; ++k) {
            xrel[3 * id + k] = p->x[k];
            xabs[3 * id + k] = c->origin[k] + p->x[k];
            v[3 * id + k] = p->v[k];
            f[3 * id + k] = p->f[k];
        }
    }
    return 0;
}

/* Adds a static cuboid the way cuboid_init does (MxCuboid.cpp:40-76; that file is not
 * compiled here): the orientation qx qy qz from Quaternion::rotation's formula
 * (axis sin(a/2), cos(a/2)), its inverse as conjugated() / dot(), the bounding box as
 * MxCuboid_UpdateAABB forms it (its upper bound starting at the smallest positive float);
 * then the reference's own engine_addcuboid. */
int mxref_add_cuboid(const float *pos, const float *size, const float *angles) {
    MxCuboid c;
    memset((void *)&c, 0, sizeof(c));
    c.position = Magnum::Vector3(pos[0], pos[1], pos[2]);
    c.size = Magnum::Vector3(size[0], size[1], size[2]);
    const Magnum::Vector3 axes[3] = {Magnum::Vector3::xAxis(), Magnum::Vector3::yAxis(), Magnum::Vector3::zAxis()};
    Magnum::Quaternion q[3];
    for (int k = 0; k < 3; ++k) {
        const float half = angles[k] / 2;
        q[k] = Magnum::Quaternion(axes[k] * std::sin(half), std::cos(half));
    }
    c.orientation = q[0] * q[1] * q[2];
    const float dot = Magnum::Math::dot(c.orientation.vector(), c.orientation.vector()) +
                      c.orientation.scalar() * c.orientation.scalar();
    c.inv_orientation = Magnum::Quaternion(-c.orientation.vector() / dot, c.orientation.scalar() / dot);
    Magnum::Vector3 mn = Magnum::Vector3(std::numeric_limits<float>::max());
    Magnum::Vector3 mx = Magnum::Vector3(std::numeric_limits<float>::min());
    const Magnum::Vector3 h = 0.5 * c.size;
    const Magnum::Vector3 pts[8] = {
        c.orientation.transformVector({h[0], h[1], h[2]}) + c.position,
        c.orientation.transformVector({h[0], -h[1], h[2]}) + c.position,
        c.orientation.transformVector({-h[0], -h[1], h[2]}) + c.position,
        c.orientation.transformVector({-h[0], h[1], h[2]}) + c.position,
        c.orientation.transformVector({h[0], h[1], -h[2]}) + c.position,
        c.orientation.transformVector({h[0], -h[1], -h[2]}) + c.position,
        c.orientation.transformVector({-h[0], -h[1], -h[2]}) + c.position,
        c.orientation.transformVector({-h[0], h[1], -h[2]}) + c.position,
    };
    for (int i = 0; i < 8; ++i)
        for (int k = 0; k < 3; ++k) {
            mn[k] = std::min(mn[k], pts[i][k]);
            mx[k] = std::max(mx[k], pts[i][k]);
        }
    c.aabb._min = mn;
    c.aabb._max = mx;
    MxCuboid *res = NULL;
    return engine_addcuboid(&_Engine, &c, &res);
}

int mxref_bind_cuboid(void *pot, int type) {
    return engine_add_cuboid_potential(&_Engine, (MxPotential *)pot, type);
}

/* Per-id number density f[3] (MxParticle::number_density) of the last force pass. */
int mxref_number_density(int n, float *out) {
    space *s = &_Engine.s;
    for (int id = 0; id < n; ++id) {
        MxParticle *p = id < s->nr_parts ? s->partlist[id] : NULL;
        out[id] = p ? p->f[3] : 0.f;
    }
    return 0;
}

int mxref_space_info(int *cdim, double *h, int *nr_cells, int *nr_tasks, unsigned *period) {
    space *s = &_Engine.s;
    for (int k = 0; k < 3; ++k) { cdim[k] = s->cdim[k]; h[k] = s->h[k]; }
    *nr_cells = s->nr_cells;
    *nr_tasks = s->nr_tasks;
    *period = s->period;
    return 0;
}

/* Task list as rows of (type, flags, i, j). */
int mxref_get_tasks(int *out, int cap) {
    space *s = &_Engine.s;
    if (cap < 4 * s->nr_tasks) return -s->nr_tasks;
    for (int k = 0; k < s->nr_tasks; ++k) {
        out[4 * k] = s->tasks[k].type;
        out[4 * k + 1] = s->tasks[k].flags;
        out[4 * k + 2] = s->tasks[k].i;
        out[4 * k + 3] = s->tasks[k].j;
    }
    return s->nr_tasks;
}

int mxref_cell_flags(unsigned *out, double *origin) {
    space *s = &_Engine.s;
    for (int c = 0; c < s->nr_cells; ++c) {
        out[c] = s->cells[c].flags;
        for (int k = 0; k < 3; ++k) origin[3 * c + k] = s->cells[c].origin[k];
    }
    return s->nr_cells;
}

int mxref_bond_flags(unsigned *out, int n) {
    for (int k = 0; k < n && k < _Engine.nr_bonds; ++k) out[k] = _Engine.bonds[k].flags;
    return _Engine.nr_bonds;
}

/* epot: s->epot (after engine_force it holds the bonded part only; engine_advance
 * adds the per-cell nonbonded energies); cell_sum: the per-cell nonbonded
 * energies of the last force pass (space_cell.epot). */
void mxref_energies(double *epot, double *cell_sum, double *epot_bond, double *ekin) {
    *epot = _Engine.s.epot;
    double cs = 0.0;
    for (int c = 0; c < _Engine.s.nr_cells; ++c) cs += _Engine.s.cells[c].epot;
    *cell_sum = cs;
    *epot_bond = _Engine.s.epot_bond;
    *ekin = engine_kinetic_energy(&_Engine);
}

double mxref_max_dist_fraction(void) { return _Engine.particle_max_dist_fraction; }

}
