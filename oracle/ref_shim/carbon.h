/* Shim for the carbon support library (absent from the reference checkout).
 * Test infrastructure only: lets the reference's own potential-table sources
 * compile in place so the oracle can be pinned against them. */
#pragma once
#include <Python.h>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <sstream>
#include <string>
#include <stdexcept>
#include <iostream>
#include <random>

#define CAPI_FUNC(RTYPE) RTYPE
/* carbon's spellings of the CPython type-object header initialisers */
#define CObject_HEAD_INIT(type) PyVarObject_HEAD_INIT(type, 0)
#define CVarObject_HEAD_INIT(type, size) PyVarObject_HEAD_INIT(type, size)
#define CAPI_DATA(RTYPE) extern RTYPE
#define CAPI_STRUCT(NAME) struct NAME

/* carbon's process-wide generator (defined in ref_glue.cpp) */
extern std::mt19937 CRandom;

typedef int32_t HRESULT;
#define S_OK ((HRESULT)0)
#define E_FAIL ((HRESULT)0x80004005L)
#define E_INVALIDARG ((HRESULT)0x80070057L)
#define SUCCEEDED(hr) (((HRESULT)(hr)) >= 0)
#define FAILED(hr) (((HRESULT)(hr)) < 0)
#define MX_FUNCTION __func__

inline void *CAligned_Malloc(size_t size, size_t align) {
    void *p = nullptr;
    if (posix_memalign(&p, align < sizeof(void *) ? sizeof(void *) : align, size ? size : align) != 0) return nullptr;
    return p;
}
inline void CAligned_Free(void *p) { free(p); }

enum { LOG_FATAL = 1, LOG_CRITICAL, LOG_ERROR, LOG_WARNING, LOG_NOTICE, LOG_INFORMATION, LOG_DEBUG, LOG_TRACE };
struct ShimNullLog {
    template <typename T> ShimNullLog &operator<<(const T &) { return *this; }
};
#define Log(level) ShimNullLog()

inline HRESULT shim_c_exp(const std::exception &e) {
    PyErr_SetString(PyExc_RuntimeError, e.what());
    return E_FAIL;
}
#define c_error(code, msg) (code)
#define C_EXP(e) shim_c_exp(e)
#define C_ERR(code, msg) (PyErr_SetString(PyExc_RuntimeError, msg), (code))
#define CErr_Set(code, msg, line, file, func) (code)

#define C_RETURN_EXP(e) do { shim_c_exp(e); return NULL; } while (0)
#define C_ERR_BOOL(x) (x)

namespace carbon {
inline PyObject *cast(const std::string &s) { return PyUnicode_FromString(s.c_str()); }
template <typename T> T cast(PyObject *o);
struct sequence {
    PyObject *o = nullptr;
    int size() const { return (int)PySequence_Size(o); }
    PyObject *get(int i) const { PyObject *r = PySequence_GetItem(o, i); Py_XDECREF(r); return r; }
};
template <typename T> bool check(PyObject *o);
template <> inline bool check<sequence>(PyObject *o) { return o && (PyList_Check(o) || PyTuple_Check(o)); }
template <> inline bool check<std::string>(PyObject *o) { return o && PyUnicode_Check(o); }
template <> inline sequence cast<sequence>(PyObject *o) { return sequence{o}; }
template <> inline std::string cast<std::string>(PyObject *o) { const char *s = PyUnicode_AsUTF8(o); return s ? s : ""; }
inline std::string str(PyObject *o) { PyObject *s = PyObject_Str(o); std::string r = s ? PyUnicode_AsUTF8(s) : "<object>"; Py_XDECREF(s); return r; }
}

/* Species state vector attached to particles (chemical cargo): the layout the
 * engine's flux code touches (values, rates, per-species flags). */
struct CStateVector {
    float *fvec = nullptr;
    float *q = nullptr;
    uint32_t *species_flags = nullptr;
    struct CSpeciesList *species = nullptr;
    int size = 0;
    void reset() {}
};
struct CType : PyTypeObject {};
inline int CType_IsSubtype(CType *a, CType *b) { return a == b; }
