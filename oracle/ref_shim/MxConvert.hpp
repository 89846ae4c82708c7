/* Stand-in for the reference's Python<->C++ conversion helpers (MxConvert /
 * CConvert), enough for the reference's own argument parsing to run:
 * numbers, bools, strings, 3-vectors and raw objects. */
#pragma once
#include "carbon.h"
#include <Magnum/Magnum.h>
#include <limits>
namespace mx {
template <typename T> struct shim_conv;
template <> struct shim_conv<double> {
    static bool check(PyObject *o) { return PyFloat_Check(o) || PyLong_Check(o); }
    static double from(PyObject *o) { double v = PyFloat_AsDouble(o); if (PyErr_Occurred()) throw std::invalid_argument("not a number"); return v; }
    static PyObject *to(double v) { return PyFloat_FromDouble(v); }
};
template <> struct shim_conv<float> {
    static bool check(PyObject *o) { return shim_conv<double>::check(o); }
    static float from(PyObject *o) { return (float)shim_conv<double>::from(o); }
    static PyObject *to(float v) { return PyFloat_FromDouble(v); }
};
template <> struct shim_conv<int> {
    static bool check(PyObject *o) { return PyLong_Check(o); }
    static int from(PyObject *o) { long v = PyLong_AsLong(o); if (PyErr_Occurred()) throw std::invalid_argument("not an int"); return (int)v; }
    static PyObject *to(int v) { return PyLong_FromLong(v); }
};
template <> struct shim_conv<unsigned> {
    static bool check(PyObject *o) { return PyLong_Check(o); }
    static unsigned from(PyObject *o) { return (unsigned)PyLong_AsUnsignedLong(o); }
    static PyObject *to(unsigned v) { return PyLong_FromUnsignedLong(v); }
};
template <> struct shim_conv<long> {
    static bool check(PyObject *o) { return PyLong_Check(o); }
    static long from(PyObject *o) { return PyLong_AsLong(o); }
    static PyObject *to(long v) { return PyLong_FromLong(v); }
};
template <> struct shim_conv<bool> {
    static bool check(PyObject *o) { return PyBool_Check(o); }
    static bool from(PyObject *o) { return PyObject_IsTrue(o) == 1; }
    static PyObject *to(bool v) { return PyBool_FromLong(v); }
};
template <> struct shim_conv<std::string> {
    static bool check(PyObject *o) { return PyUnicode_Check(o); }
    static std::string from(PyObject *o) { const char *s = PyUnicode_AsUTF8(o); if (!s) throw std::invalid_argument("not a string"); return s; }
    static PyObject *to(const std::string &v) { return PyUnicode_FromString(v.c_str()); }
};
template <> struct shim_conv<PyObject *> {
    static bool check(PyObject *o) { return o != nullptr; }
    static PyObject *from(PyObject *o) { return o; }
    static PyObject *to(PyObject *v) { Py_XINCREF(v); return v; }
};
template <> struct shim_conv<Magnum::Vector3> {
    static bool check(PyObject *o) { return PySequence_Check(o) && PySequence_Size(o) == 3; }
    static Magnum::Vector3 from(PyObject *o) {
        if (!check(o)) throw std::invalid_argument("expected a 3-sequence");
        Magnum::Vector3 r;
        for (int i = 0; i < 3; ++i) {
            PyObject *it = PySequence_GetItem(o, i);
            r[i] = (float)PyFloat_AsDouble(it);
            Py_XDECREF(it);
        }
        return r;
    }
    static PyObject *to(const Magnum::Vector3 &v) { return Py_BuildValue("(fff)", v[0], v[1], v[2]); }
};
template <> struct shim_conv<Magnum::Vector3i> {
    static bool check(PyObject *o) { return PySequence_Check(o) && PySequence_Size(o) == 3; }
    static Magnum::Vector3i from(PyObject *o) {
        Magnum::Vector3i r;
        for (int i = 0; i < 3; ++i) { PyObject *it = PySequence_GetItem(o, i); r[i] = (int)PyLong_AsLong(it); Py_XDECREF(it); }
        return r;
    }
    static PyObject *to(const Magnum::Vector3i &v) { return Py_BuildValue("(iii)", v[0], v[1], v[2]); }
};
template <typename T> PyObject *cast(const T &x) { return shim_conv<T>::to(x); }
inline PyObject *cast(uint32_t x) { return PyLong_FromUnsignedLong(x); }
inline PyObject *cast(int16_t x) { return PyLong_FromLong(x); }
template <typename T> T cast(PyObject *o) { return shim_conv<T>::from(o); }
template <typename T> bool check(PyObject *o) { return o && shim_conv<T>::check(o); }
inline PyObject *shim_arg_lookup(const char *name, int index, PyObject *args, PyObject *kwargs) {
    if (kwargs) { PyObject *v = PyDict_GetItemString(kwargs, name); if (v) return v; }
    if (args && PyTuple_Check(args) && index < PyTuple_Size(args)) return PyTuple_GetItem(args, index);
    return nullptr;
}
template <typename T> T arg(const char *name, int index, PyObject *args, PyObject *kwargs) {
    PyObject *v = shim_arg_lookup(name, index, args, kwargs);
    if (!v) throw std::invalid_argument(std::string("missing argument ") + name);
    return cast<T>(v);
}
template <typename T> T arg(const char *name, int index, PyObject *args, PyObject *kwargs, T deflt) {
    PyObject *v = shim_arg_lookup(name, index, args, kwargs);
    return v ? cast<T>(v) : deflt;
}
}
