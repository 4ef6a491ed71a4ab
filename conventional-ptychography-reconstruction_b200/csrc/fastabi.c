/* fastabi.c -- a CPython fast-call binding of the two C-ABI entry points the
 * training step calls every minibatch (ptycho_fwd_adj, ptycho_scale_pair).
 *
 * ctypes converts each of ptycho_fwd_adj's 21 arguments through its generic
 * conversion machinery on every call; this module takes them as a vector of
 * Python ints (device pointers from Tensor.data_ptr(), sizes) or None (NULL)
 * and calls the library function directly.  It calls the functions through
 * addresses handed over by `bind` (taken from the ctypes handle of
 * libptycho_b200.so), so there is one copy of the library and its state in the
 * process.  No computation happens here; errors come back as the library's
 * status codes.
 */
#define PY_SSIZE_T_CLEAN
#include <Python.h>
#include <stddef.h>
#include <stdint.h>

typedef int (*fwd_adj_fn)(const float*, int, int, const float*, int, int, const int32_t*, const float*, int,
                          const int32_t*, int, int, double*, double*, float*, float*, unsigned, void*, size_t,
                          int32_t*, void*);
typedef int (*scale_pair_fn)(const float*, float*, long long, const float*, float*, long long, const double*,
                             void*);

static fwd_adj_fn g_fwd_adj = NULL;
static scale_pair_fn g_scale_pair = NULL;

static int as_ptr(PyObject* o, void** out) {
  if (o == Py_None) {
    *out = NULL;
    return 0;
  }
  *out = PyLong_AsVoidPtr(o);
  return (*out == NULL && PyErr_Occurred()) ? -1 : 0;
}

static int as_int(PyObject* o, long* out) {
  *out = PyLong_AsLong(o);
  return (*out == -1 && PyErr_Occurred()) ? -1 : 0;
}

static PyObject* bind(PyObject* self, PyObject* const* args, Py_ssize_t n) {
  void *a = NULL, *b = NULL;
  (void)self;
  if (n != 2) {
    PyErr_SetString(PyExc_TypeError, "bind(fwd_adj_address, scale_pair_address)");
    return NULL;
  }
  if (as_ptr(args[0], &a) || as_ptr(args[1], &b)) return NULL;
  g_fwd_adj = (fwd_adj_fn)a;
  g_scale_pair = (scale_pair_fn)b;
  Py_RETURN_NONE;
}

/* fwd_adj(O, H, W, P, M, N, tl, Imeas, F, batch, B, loss_type, loss_per_pattern,
 *         loss_total, dO, dP, flags, workspace, workspace_bytes, status, stream) -> status */
static PyObject* fwd_adj(PyObject* self, PyObject* const* args, Py_ssize_t n) {
  void* p[21];
  long v[21];
  static const int is_ptr[21] = {1, 0, 0, 1, 0, 0, 1, 1, 0, 1, 0, 0, 1, 1, 1, 1, 0, 1, 0, 1, 1};
  (void)self;
  if (n != 21) {
    PyErr_SetString(PyExc_TypeError, "fwd_adj takes 21 arguments");
    return NULL;
  }
  if (!g_fwd_adj) {
    PyErr_SetString(PyExc_RuntimeError, "fastabi.bind was not called");
    return NULL;
  }
  for (int i = 0; i < 21; ++i) {
    if (is_ptr[i] ? as_ptr(args[i], &p[i]) : as_int(args[i], &v[i])) return NULL;
  }
  const int rc = g_fwd_adj((const float*)p[0], (int)v[1], (int)v[2], (const float*)p[3], (int)v[4], (int)v[5],
                           (const int32_t*)p[6], (const float*)p[7], (int)v[8], (const int32_t*)p[9], (int)v[10],
                           (int)v[11], (double*)p[12], (double*)p[13], (float*)p[14], (float*)p[15],
                           (unsigned)v[16], p[17], (size_t)v[18], (int32_t*)p[19], p[20]);
  return PyLong_FromLong(rc);
}

/* scale_pair(a, a_out, na, b, b_out, nb, scale, stream) -> status */
static PyObject* scale_pair(PyObject* self, PyObject* const* args, Py_ssize_t n) {
  void* p[8];
  long v[8];
  static const int is_ptr[8] = {1, 1, 0, 1, 1, 0, 1, 1};
  (void)self;
  if (n != 8) {
    PyErr_SetString(PyExc_TypeError, "scale_pair takes 8 arguments");
    return NULL;
  }
  if (!g_scale_pair) {
    PyErr_SetString(PyExc_RuntimeError, "fastabi.bind was not called");
    return NULL;
  }
  for (int i = 0; i < 8; ++i) {
    if (is_ptr[i] ? as_ptr(args[i], &p[i]) : as_int(args[i], &v[i])) return NULL;
  }
  const int rc = g_scale_pair((const float*)p[0], (float*)p[1], (long long)v[2], (const float*)p[3], (float*)p[4],
                              (long long)v[5], (const double*)p[6], p[7]);
  return PyLong_FromLong(rc);
}

static PyMethodDef methods[] = {
    {"bind", (PyCFunction)(void (*)(void))bind, METH_FASTCALL, "bind(fwd_adj_address, scale_pair_address)"},
    {"fwd_adj", (PyCFunction)(void (*)(void))fwd_adj, METH_FASTCALL, "ptycho_fwd_adj (21 arguments)"},
    {"scale_pair", (PyCFunction)(void (*)(void))scale_pair, METH_FASTCALL, "ptycho_scale_pair (8 arguments)"},
    {NULL, NULL, 0, NULL}};

static struct PyModuleDef module = {PyModuleDef_HEAD_INIT, "_fastabi", NULL, -1, methods, NULL, NULL, NULL, NULL};

PyMODINIT_FUNC PyInit__fastabi(void) { return PyModule_Create(&module); }
