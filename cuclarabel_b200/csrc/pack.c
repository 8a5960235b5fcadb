/* pack.c -- CPython extension: the clgpu_problem array of a batch.
 *
 * BatchSolver(problems) hands the library one clgpu_problem per instance
 * (src/solver.jl:5-70 takes the same P, q, A, b, cones per Solver).  The
 * library copies every host array during clgpu_solver_create, so the
 * structs can point straight into the caller's numpy / scipy arrays: this
 * module walks the problem list once, checks each problem's arrays, and
 * fills the structs and the flat cone lists without copying any matrix.
 *
 * pack(problems, structs) -> (ct, cd, cp, dims, p_nnz, a_nnz) or None
 *   problems  sequence of (P, q, A, b, cones) tuples
 *   structs   writable buffer of len(problems) clgpu_problem structs
 *   ct, cd    bytes: int32 cone types / dims, concatenated (one spare entry)
 *   cp        bytes: float64 cone parameters, concatenated
 *   dims      bytes: int32 (n, m) per instance
 * None means "take the general path": a problem whose P or A is not a
 * canonical scipy CSC matrix with int32 indices and float64 values, whose
 * q or b is not a contiguous float64 vector, whose cones are not a list of
 * cone objects, or whose shapes disagree (the general path then raises the
 * reference's message).  The structs' pointers stay valid while the
 * problems' arrays and the returned cone lists are alive. */
#define PY_SSIZE_T_CLEAN
#include <Python.h>

#include <stdint.h>
#include <string.h>

#include "../../include/clgpu.h"

/* contiguous 1-D buffer of n items of the given size and kind ('i' integer,
 * 'f' floating); its address in *ptr.  0 when obj does not qualify. */
static int vec_of(PyObject *obj, Py_ssize_t itemsize, char kind, const void **ptr,
                  Py_ssize_t *n) {
  Py_buffer v;
  if (PyObject_GetBuffer(obj, &v, PyBUF_C_CONTIGUOUS | PyBUF_FORMAT) != 0) {
    PyErr_Clear();
    return 0;
  }
  int ok = v.ndim == 1 && v.itemsize == itemsize && v.format != NULL;
  if (ok) {
    const char *f = v.format;
    if (*f == '<' || *f == '=' || *f == '@') ++f;
    if (kind == 'i')
      ok = (f[0] == 'i' || (f[0] == 'l' && itemsize == (Py_ssize_t)sizeof(long))) && f[1] == 0;
    else
      ok = f[0] == 'd' && f[1] == 0;
  }
  if (ok) {
    *ptr = v.buf;
    *n = v.shape ? v.shape[0] : v.len / itemsize;
  }
  PyBuffer_Release(&v);
  return ok;
}

/* canonical CSC matrix of the given shape: its three arrays */
static int csc_of(PyObject *M, Py_ssize_t rows, Py_ssize_t cols, const int **p,
                  const int **i, const double **x, Py_ssize_t *nnz) {
  int ok = 0;
  PyObject *fmt = PyObject_GetAttrString(M, "format");
  PyObject *canon = NULL, *shape = NULL, *ip = NULL, *ii = NULL, *ix = NULL;
  if (!fmt || !PyUnicode_Check(fmt) || PyUnicode_CompareWithASCIIString(fmt, "csc") != 0)
    goto done;
  canon = PyObject_GetAttrString(M, "has_canonical_format");
  if (!canon || PyObject_IsTrue(canon) != 1) goto done;
  shape = PyObject_GetAttrString(M, "shape");
  if (!shape || !PyTuple_Check(shape) || PyTuple_GET_SIZE(shape) != 2) goto done;
  if (PyLong_AsSsize_t(PyTuple_GET_ITEM(shape, 0)) != rows ||
      PyLong_AsSsize_t(PyTuple_GET_ITEM(shape, 1)) != cols)
    goto done;
  ip = PyObject_GetAttrString(M, "indptr");
  ii = PyObject_GetAttrString(M, "indices");
  ix = PyObject_GetAttrString(M, "data");
  if (!ip || !ii || !ix) goto done;
  Py_ssize_t np_, ni, nx;
  if (!vec_of(ip, 4, 'i', (const void **)p, &np_) || np_ != cols + 1) goto done;
  if (!vec_of(ii, 4, 'i', (const void **)i, &ni)) goto done;
  if (!vec_of(ix, 8, 'f', (const void **)x, &nx) || nx != ni) goto done;
  *nnz = nx;
  ok = 1;
done:
  if (PyErr_Occurred()) PyErr_Clear();
  Py_XDECREF(fmt);
  Py_XDECREF(canon);
  Py_XDECREF(shape);
  Py_XDECREF(ip);
  Py_XDECREF(ii);
  Py_XDECREF(ix);
  return ok;
}

/* integer attribute, or -1 */
static long attr_long(PyObject *o, const char *name) {
  PyObject *a = PyObject_GetAttrString(o, name);
  if (!a) {
    PyErr_Clear();
    return -1;
  }
  long v = -1;
  PyObject *ix = PyNumber_Index(a);  /* Python and numpy integers */
  if (ix) {
    v = PyLong_AsLong(ix);
    Py_DECREF(ix);
  }
  if (PyErr_Occurred()) {
    PyErr_Clear();
    v = -1;
  }
  Py_DECREF(a);
  return v;
}

static PyObject *pack(PyObject *self, PyObject *args) {
  (void)self;
  PyObject *probs, *structs_obj;
  if (!PyArg_ParseTuple(args, "OO", &probs, &structs_obj)) return NULL;
  PyObject *seq = PySequence_Fast(probs, "problems must be a sequence");
  if (!seq) return NULL;
  const Py_ssize_t B = PySequence_Fast_GET_SIZE(seq);
  Py_buffer sb;
  if (PyObject_GetBuffer(structs_obj, &sb, PyBUF_WRITABLE | PyBUF_C_CONTIGUOUS) != 0) {
    Py_DECREF(seq);
    return NULL;
  }
  if (sb.len < B * (Py_ssize_t)sizeof(clgpu_problem)) {
    PyBuffer_Release(&sb);
    Py_DECREF(seq);
    PyErr_SetString(PyExc_ValueError, "structs buffer too small");
    return NULL;
  }
  clgpu_problem *out = (clgpu_problem *)sb.buf;
  PyObject *result = NULL, *ctb = NULL, *cdb = NULL, *cpb = NULL, *dmb = NULL;
  /* pass 1: cone count */
  Py_ssize_t ncone = 0;
  for (Py_ssize_t k = 0; k < B; ++k) {
    PyObject *t = PySequence_Fast_GET_ITEM(seq, k);
    if (!PyTuple_Check(t) || PyTuple_GET_SIZE(t) != 5 || !PyList_Check(PyTuple_GET_ITEM(t, 4)))
      goto fallback;
    ncone += PyList_GET_SIZE(PyTuple_GET_ITEM(t, 4));
  }
  ctb = PyBytes_FromStringAndSize(NULL, (ncone + 1) * 4);
  cdb = PyBytes_FromStringAndSize(NULL, (ncone + 1) * 4);
  cpb = PyBytes_FromStringAndSize(NULL, (ncone + 1) * 8);
  dmb = PyBytes_FromStringAndSize(NULL, (B > 0 ? B : 1) * 8);
  if (!ctb || !cdb || !cpb || !dmb) goto error;
  int *ct = (int *)PyBytes_AS_STRING(ctb), *cd = (int *)PyBytes_AS_STRING(cdb);
  double *cp = (double *)PyBytes_AS_STRING(cpb);
  int32_t *dims = (int32_t *)PyBytes_AS_STRING(dmb);
  ct[ncone] = cd[ncone] = 0;
  cp[ncone] = 0.0;
  long long p_nnz = 0, a_nnz = 0;
  Py_ssize_t c0 = 0;
  for (Py_ssize_t k = 0; k < B; ++k) {
    PyObject *t = PySequence_Fast_GET_ITEM(seq, k);
    PyObject *P = PyTuple_GET_ITEM(t, 0), *q = PyTuple_GET_ITEM(t, 1);
    PyObject *A = PyTuple_GET_ITEM(t, 2), *b = PyTuple_GET_ITEM(t, 3);
    PyObject *cones = PyTuple_GET_ITEM(t, 4);
    const double *qp, *bp;
    Py_ssize_t n, m;
    if (!vec_of(q, 8, 'f', (const void **)&qp, &n) || !vec_of(b, 8, 'f', (const void **)&bp, &m))
      goto fallback;
    if (n > INT32_MAX || m > INT32_MAX) goto fallback;
    clgpu_problem *o = &out[k];
    Py_ssize_t pn, an;
    if (!csc_of(P, n, n, &o->Pp, &o->Pi, &o->Px, &pn)) goto fallback;
    if (!csc_of(A, m, n, &o->Ap, &o->Ai, &o->Ax, &an)) goto fallback;
    /* cones: type code (class attribute), dim, alpha; rows they cover */
    const Py_ssize_t nc = PyList_GET_SIZE(cones);
    long long nv = 0;
    for (Py_ssize_t j = 0; j < nc; ++j) {
      PyObject *c = PyList_GET_ITEM(cones, j);
      const long code = attr_long(c, "code");
      long d = 3;
      double a = 0.0;
      if (code == CLGPU_CONE_ZERO || code == CLGPU_CONE_NONNEG || code == CLGPU_CONE_SOC ||
          code == CLGPU_CONE_PSD) {
        d = attr_long(c, "dim");
        if (d < 0 || d > INT32_MAX) goto fallback;
      } else if (code == CLGPU_CONE_POW) {
        PyObject *al = PyObject_GetAttrString(c, "alpha");
        if (!al) goto fallback;
        a = PyFloat_AsDouble(al);
        Py_DECREF(al);
        if (PyErr_Occurred()) goto fallback;
      } else if (code != CLGPU_CONE_EXP) {
        goto fallback;
      }
      ct[c0 + j] = (int)code;
      cd[c0 + j] = (int)d;
      cp[c0 + j] = a;
      nv += code == CLGPU_CONE_PSD ? (long long)d * (d + 1) / 2 : d;
    }
    if (nv != m) goto fallback;
    o->n = (int)n;
    o->m = (int)m;
    o->q = qp;
    o->b = bp;
    o->ncones = (int)nc;
    o->cone_types = ct + c0;
    o->cone_dims = cd + c0;
    o->cone_params = cp + c0;
    dims[2 * k] = (int32_t)n;
    dims[2 * k + 1] = (int32_t)m;
    p_nnz += pn;
    a_nnz += an;
    c0 += nc;
  }
  result = Py_BuildValue("(OOOOLL)", ctb, cdb, cpb, dmb, p_nnz, a_nnz);
  goto done;
fallback:
  if (PyErr_Occurred()) PyErr_Clear();
  result = Py_None;
  Py_INCREF(result);
  goto done;
error:
  result = NULL;
done:
  Py_XDECREF(ctb);
  Py_XDECREF(cdb);
  Py_XDECREF(cpb);
  Py_XDECREF(dmb);
  PyBuffer_Release(&sb);
  Py_DECREF(seq);
  return result;
}

static PyMethodDef methods[] = {
    {"pack", pack, METH_VARARGS,
     "pack(problems, structs) -> (ct, cd, cp, dims, p_nnz, a_nnz) or None"},
    {NULL, NULL, 0, NULL}};

static struct PyModuleDef module = {PyModuleDef_HEAD_INIT, "_pack",
                                    "clgpu_problem arrays of a batch", -1, methods,
                                    NULL, NULL, NULL, NULL};

PyMODINIT_FUNC PyInit__pack(void) { return PyModule_Create(&module); }
