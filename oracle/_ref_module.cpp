// Module initialisation for the reference's own C core, built unmodified
// from its sources (c/bmgs/bmgs.cpp, c/bc.cpp, c/operators.cpp,
// c/woperators.cpp, c/transformers.cpp, c/fd_preconditioner.cpp,
// c/gpaw_utils.cpp).
//
// TEST INFRASTRUCTURE ONLY: this module is the CPU reference that parity
// tests, smoke() and bench.py's CPU-baseline leg compare against.  Nothing
// in the gpaw_b200 package imports it.
//
// It registers the entry points of the finite-difference hot path under
// the names the reference's extension uses for them (c/_gpaw.h): Operator,
// WOperator, Transformer, fd_precond.
#define __GPAW_SHOULD_IMPORT_NUMPY
#include "python_utils.h"

extern "C++" {
PyObject* NewOperatorObject(PyObject* self, PyObject* args);
PyObject* NewWOperatorObject(PyObject* self, PyObject* args);
PyObject* NewTransformerObject(PyObject* self, PyObject* args);
PyObject* fd_precond(PyObject* self, PyObject* args);
}
extern PyTypeObject OperatorType;
extern PyTypeObject WOperatorType;
extern PyTypeObject TransformerType;

static PyMethodDef ref_methods[] = {
    {"Operator", NewOperatorObject, METH_VARARGS, "reference FD operator"},
    {"WOperator", NewWOperatorObject, METH_VARARGS,
     "reference weighted FD operator"},
    {"Transformer", NewTransformerObject, METH_VARARGS,
     "reference restrict/interpolate transformer"},
    {"fd_precond", fd_precond, METH_VARARGS,
     "reference multigrid preconditioner"},
    {NULL, NULL, 0, NULL}};

static struct PyModuleDef ref_module = {PyModuleDef_HEAD_INIT, "_gpaw_ref",
                                        "reference FD hot path (oracle)", -1,
                                        ref_methods};

PyMODINIT_FUNC PyInit__gpaw_ref(void)
{
    import_array1(NULL);
    if (PyType_Ready(&OperatorType) < 0) return NULL;
    if (PyType_Ready(&WOperatorType) < 0) return NULL;
    if (PyType_Ready(&TransformerType) < 0) return NULL;
    return PyModule_Create(&ref_module);
}
