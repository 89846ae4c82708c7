/*
 * Link glue for the in-place build of the reference engine (oracle tier A).
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the product links or loads this.
 *
 * The reference's hot-path translation units (space, runners, pair loops,
 * integrator, exclusions, bonds, angles, dihedrals, fluxes, potentials) are compiled unmodified
 * from the reference checkout. They reference a handful of symbols that live
 * in subsystems that are outside the force-and-step path (rendering styles,
 * clusters, events, timers, rigid constraints, Verlet
 * lists). This file defines those symbols as inert stand-ins so the engine
 * links; none of them is reached by the configurations the oracle runs (no
 * clusters, rigids or events).
 */
#include <random>

#include "mdcore_config.h"
#include "engine.h"
#include "MxParticle.h"
#include "MxPotential.h"
#include "bond.h"
#include "angle.h"
#include "MxCuboid.hpp"
#include "MxBody.hpp"
#include "MxCluster.hpp"
#include "MxParticleList.hpp"
#include "../../MxUtil.h"
#include "../../rendering/NOMStyle.hpp"
#include "MxBind.hpp"
#include <CEvent.hpp>
#include <cstdarg>

engine _Engine;

PerformanceTimer::PerformanceTimer(unsigned id) : _start(0), _id(id) {}
PerformanceTimer::~PerformanceTimer() {}
WallTime::WallTime() : start(0) {}
WallTime::~WallTime() {}
double MxWallTime() { return 0.0; }

int engine_rigid_eval(struct engine *) { return 0; }
extern "C" int runner_verlet_fill(struct runner *, struct space_cell *, struct space_cell *, FPTYPE *) { return 0; }
extern "C" int runner_verlet_eval(struct runner *, struct space_cell *, FPTYPE *) { return 0; }

MxParticle::MxParticle() { bzero(this, sizeof(MxParticle)); }
bool MxParticle::verify() { return true; }
MxParticleHandle *MxParticle::py_particle() { return nullptr; }
MxParticle *MxParticle_Get(PyObject *) { return nullptr; }
HRESULT MxParticle_Verify() { return S_OK; }
HRESULT MxParticleType::addpart(int32_t) { return S_OK; }
HRESULT MxParticleType::del_part(int32_t) { return S_OK; }
MxParticleType *MxParticleType_ForEngine(struct engine *, double, double, const char *, const char *) { return nullptr; }
PyObject *MxParticleList_Pack(Py_ssize_t, ...) { return nullptr; }
MxParticleList *MxParticleList_All() { return nullptr; }

void MxCuboid_UpdateAABB(MxCuboid *) {}
MxCuboid::MxCuboid() {}
int MxCluster_ComputeAggregateQuantities(struct MxCluster *) { return 0; }

NOMStyle *NOMStyle_NewEx(const Magnum::Color3 &, uint32_t) { return nullptr; }
int NOMStyle_Check(const PyObject *) { return 0; }
Magnum::Color3 Color3_Parse(const std::string &) { return Magnum::Color3(); }

CMulticastTimeEvent *CMulticastTimeEvent_New() { return nullptr; }
HRESULT CMulticastTimeEvent_Invoke(CMulticastTimeEvent *, double) { return S_OK; }
PyObject *MxPotential_Bind(MxPotential *, PyObject *, PyObject *) { Py_RETURN_NONE; }
int MxParticle_Check(PyObject *) { return 0; }
MxParticleType *MxParticleType_Get(PyObject *) { return nullptr; }
/* MxRandomVector (src/mdcore/src/MxParticle.cpp:1782-1793, a file the oracle Makefile
 * does not compile): a normal magnitude N(mean, std) in a uniformly random
 * direction, restated with the same construction on a default-seeded mt19937
 * as carbon's global generator (the random-force tests compare
 * statistics, not draws). */
std::mt19937 CRandom;
Magnum::Vector3 MxRandomVector(float mean, float std) {
    std::normal_distribution<> dist{mean, std};
    std::uniform_real_distribution<double> uniform01(0.0, 1.0);
    float theta = 2 * M_PI * uniform01(CRandom);
    float phi = acos(1 - 2 * uniform01(CRandom));
    float r = dist(CRandom);
    return Magnum::Vector3{r * sinf(phi) * cosf(theta), r * sinf(phi) * sinf(theta), r * cosf(phi)};
}
MxBody::MxBody() {}
