/* pyjobs.c - CPython helper of fastpoly_b200.Context.batch: fills the fpx_job
 * records of a batch from its Python job tuples.
 *
 * A batch of thousands of jobs spent about 2 us per job in the Python loop that
 * did this (tuple unpacking, one ctypes object per array to read its address,
 * list appends), as long as the GPU takes for the whole config-sized batch.
 * Here each array is read through the buffer protocol and each record written
 * in place, with the Python loop's semantics:
 *   ("conv", p, a, b[, n])   n absent or None: the full product
 *   ("inv" | "log" | "exp" | "sqrt", p, a, n)
 *   ("pow", p, a, k, n)
 *   ("divmod", p, a, b)
 * Arrays that are not C-contiguous 4-byte unsigned buffers go through the
 * caller's converter (numpy.ascontiguousarray(..., uint32)); the converted
 * arrays are returned so that the caller keeps them alive for the call.
 * Output capacities (words) go to caps[0..m) (first output) and caps[m..2m)
 * (divmod remainder); the caller places the outputs.
 */
#define PY_SSIZE_T_CLEAN
#include <Python.h>

#include <stdint.h>
#include <string.h>

#include "fpx_b200.h"

/* Address and length of a uint32 buffer, converting through `conv` if needed
 * (the converted object is appended to `keep`). */
static int get_u32(PyObject* obj, PyObject* conv, PyObject* keep, const uint32_t** ptr, size_t* len) {
  Py_buffer v;
  if (PyObject_GetBuffer(obj, &v, PyBUF_C_CONTIGUOUS | PyBUF_FORMAT) == 0) {
    const char* f = v.format ? v.format : "B";
    if (f[0] == '=' || f[0] == '<' || f[0] == '@') ++f;
    const int ok = v.itemsize == 4 && (strcmp(f, "I") == 0 || (sizeof(unsigned long) == 4 && strcmp(f, "L") == 0));
    if (ok) {
      *ptr = (const uint32_t*)v.buf;
      *len = (size_t)(v.len / 4);
      PyBuffer_Release(&v);
      return 0;
    }
    PyBuffer_Release(&v);
  } else {
    PyErr_Clear();
  }
  PyObject* c = PyObject_CallOneArg(conv, obj);
  if (!c) return -1;
  if (PyList_Append(keep, c) < 0) {
    Py_DECREF(c);
    return -1;
  }
  Py_DECREF(c);  /* `keep` holds it */
  if (PyObject_GetBuffer(c, &v, PyBUF_C_CONTIGUOUS | PyBUF_FORMAT) < 0) return -1;
  if (v.itemsize != 4) {
    PyBuffer_Release(&v);
    PyErr_SetString(PyExc_TypeError, "converter did not return a 4-byte array");
    return -1;
  }
  *ptr = (const uint32_t*)v.buf;
  *len = (size_t)(v.len / 4);
  PyBuffer_Release(&v);
  return 0;
}

/* int(x) as an unsigned 64-bit value (OverflowError outside [0, 2^64)). */
static int get_u64(PyObject* x, uint64_t* out) {
  PyObject* i = PyNumber_Long(x);
  if (!i) return -1;
  const unsigned long long v = PyLong_AsUnsignedLongLong(i);
  Py_DECREF(i);
  if (v == (unsigned long long)-1 && PyErr_Occurred()) return -1;
  *out = (uint64_t)v;
  return 0;
}

static size_t min_sz(size_t a, size_t b) { return a < b ? a : b; }
static size_t max1(size_t a) { return a ? a : 1; }

/* fill(jobs, records_addr, caps_addr, ops, conv) -> keep */
static PyObject* fill(PyObject* self, PyObject* args) {
  (void)self;
  PyObject *jobs, *ops, *conv;
  unsigned long long rec_addr, cap_addr;
  if (!PyArg_ParseTuple(args, "OKKOO", &jobs, &rec_addr, &cap_addr, &ops, &conv)) return NULL;
  PyObject* seq = PySequence_Fast(jobs, "jobs must be a sequence");
  if (!seq) return NULL;
  const Py_ssize_t m = PySequence_Fast_GET_SIZE(seq);
  fpx_job* rec = (fpx_job*)(uintptr_t)rec_addr;
  int64_t* caps = (int64_t*)(uintptr_t)cap_addr;
  PyObject* keep = PyList_New(0);
  if (!keep) goto fail_seq;
  for (Py_ssize_t i = 0; i < m; ++i) {
    PyObject* jb = PySequence_Fast(PySequence_Fast_GET_ITEM(seq, i), "a job must be a tuple");
    if (!jb) goto fail;
    const Py_ssize_t nj = PySequence_Fast_GET_SIZE(jb);
    PyObject** it = PySequence_Fast_ITEMS(jb);
    fpx_job* j = rec + i;
    uint64_t p = 0, k = 0, n = 0;
    size_t na = 0, nb = 0;
    const uint32_t *a = NULL, *b = NULL;
    if (nj < 3) {
      PyErr_Format(PyExc_ValueError, "batch job %zd: too few fields", i);
      goto fail_jb;
    }
    PyObject* code = PyDict_GetItemWithError(ops, it[0]);
    if (!code) {
      if (!PyErr_Occurred()) PyErr_SetObject(PyExc_KeyError, it[0]);
      goto fail_jb;
    }
    const long op = PyLong_AsLong(code);
    if (op == -1 && PyErr_Occurred()) goto fail_jb;
    if (get_u64(it[1], &p) < 0) goto fail_jb;
    if (p > 0xffffffffull) {
      PyErr_Format(PyExc_OverflowError, "batch job %zd: modulus out of range", i);
      goto fail_jb;
    }
    if (get_u32(it[2], conv, keep, &a, &na) < 0) goto fail_jb;
    size_t cap1 = 1, cap2 = 0;
    if (op == FPX_OP_CONV || op == FPX_OP_DIVMOD) {
      if (nj < 4) {
        PyErr_Format(PyExc_ValueError, "batch job %zd: missing second operand", i);
        goto fail_jb;
      }
      if (get_u32(it[3], conv, keep, &b, &nb) < 0) goto fail_jb;
    }
    if (op == FPX_OP_CONV) {
      n = SIZE_MAX;
      if (nj >= 5 && it[4] != Py_None && get_u64(it[4], &n) < 0) goto fail_jb;
      const size_t cap = na && nb && n ? min_sz(na, n) + min_sz(nb, n) - 1 : 0;
      cap1 = max1(min_sz(cap, n));
    } else if (op == FPX_OP_POW) {
      if (nj < 5) {
        PyErr_Format(PyExc_ValueError, "batch job %zd: pow needs (p, a, k, n)", i);
        goto fail_jb;
      }
      if (get_u64(it[3], &k) < 0 || get_u64(it[4], &n) < 0) goto fail_jb;
      cap1 = max1(n);
    } else if (op == FPX_OP_DIVMOD) {
      cap1 = max1(na);
      cap2 = max1(nb);
    } else {
      if (nj < 4) {
        PyErr_Format(PyExc_ValueError, "batch job %zd: missing length", i);
        goto fail_jb;
      }
      if (get_u64(it[3], &n) < 0) goto fail_jb;
      cap1 = max1(n);
    }
    memset(j, 0, sizeof *j);
    j->op = (int)op;
    j->p = (uint32_t)p;
    j->a = na ? a : NULL;
    j->la = na;
    j->b = nb ? b : NULL;
    j->lb = nb;
    j->k = k;
    j->n = n;
    caps[i] = (int64_t)cap1;
    caps[m + i] = (int64_t)cap2;
    Py_DECREF(jb);
    continue;
  fail_jb:
    Py_DECREF(jb);
    goto fail;
  }
  Py_DECREF(seq);
  return keep;
fail:
  Py_DECREF(keep);
fail_seq:
  Py_DECREF(seq);
  return NULL;
}

static PyMethodDef methods[] = {
    {"fill", fill, METH_VARARGS, "fill(jobs, records_addr, caps_addr, ops, conv) -> arrays to keep alive"},
    {NULL, NULL, 0, NULL}};

static struct PyModuleDef module = {PyModuleDef_HEAD_INIT, "_fpx_jobs", "fpx_job records from Python job tuples",
                                    -1, methods, NULL, NULL, NULL, NULL};

PyMODINIT_FUNC PyInit__fpx_jobs(void) { return PyModule_Create(&module); }
