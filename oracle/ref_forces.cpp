/*
 * TEST INFRASTRUCTURE ONLY (oracle tier A): the reference's
 * src/mdcore/src/MxForce.cpp, compiled in place by inclusion (the Makefile
 * passes its path), plus exported wrappers of its file-static force
 * constructors so that the driver can bind the forces the reference's Python
 * `forces` module creates. The wrappers keep the argument order of the module's
 * own calls (py_random_create / py_friction_create pass (std, mean) into
 * parameters declared (mean, std), MxForce.cpp:18-19,226-246), so the bound
 * forces are exactly those `forces.random(std, mean)` and
 * `forces.friction(coef, std, mean)` produce in the reference.
 */
#include MXREF_FORCE_SRC

extern "C" PyObject *mxref_make_berendsen(float tau) { return berenderson_create(tau); }
extern "C" PyObject *mxref_make_random(float std, float mean, float durration) {
    return random_create(std, mean, durration);
}
extern "C" PyObject *mxref_make_friction(float coef, float std, float mean, float durration) {
    return friction_create(coef, std, mean, durration);
}
