/* _hostptr.c -- CPython helper of the Python binding (host only, no CUDA).
 *
 * collect(seq, ptr, dims) reads, through the buffer protocol, the host address and
 * the side of every matrix of a batch in one C loop and writes them into `ptr`
 * (len(seq) uint64) and `dims` (len(seq) int32).  A matrix is taken as it is when
 * it exports a C-contiguous 2-D buffer of complex128 ("Zd") with equal sides; the
 * indices of all other items are returned in a list (their slots are left 0) for
 * the caller to convert or reject.  The addresses stay valid while the caller holds
 * the matrices.  A Python loop over the same attributes costs about a microsecond
 * per matrix: 80 ms of host time for a batch of 65,536.
 */
#define PY_SSIZE_T_CLEAN
#include <Python.h>
#include <stdint.h>
#include <string.h>

static int is_complex128(const char* f) {
  if (!f) return 0;
  if (f[0] == '<' || f[0] == '=' || f[0] == '@') ++f;
  return strcmp(f, "Zd") == 0;
}

static PyObject* collect(PyObject* self, PyObject* args) {
  (void)self;
  PyObject *seq, *pobj, *dobj;
  if (!PyArg_ParseTuple(args, "OOO", &seq, &pobj, &dobj)) return NULL;
  PyObject* fast = PySequence_Fast(seq, "collect: a sequence of matrices is required");
  if (!fast) return NULL;
  const Py_ssize_t n = PySequence_Fast_GET_SIZE(fast);
  Py_buffer pb, db;
  if (PyObject_GetBuffer(pobj, &pb, PyBUF_WRITABLE | PyBUF_C_CONTIGUOUS) < 0) {
    Py_DECREF(fast);
    return NULL;
  }
  if (PyObject_GetBuffer(dobj, &db, PyBUF_WRITABLE | PyBUF_C_CONTIGUOUS) < 0) {
    PyBuffer_Release(&pb);
    Py_DECREF(fast);
    return NULL;
  }
  PyObject* redo = NULL;
  if (pb.len < n * (Py_ssize_t)sizeof(uint64_t) || db.len < n * (Py_ssize_t)sizeof(int32_t)) {
    PyErr_SetString(PyExc_ValueError, "collect: output buffers shorter than the batch");
    goto done;
  }
  redo = PyList_New(0);
  if (!redo) goto done;
  uint64_t* ptr = (uint64_t*)pb.buf;
  int32_t* dims = (int32_t*)db.buf;
  PyObject** items = PySequence_Fast_ITEMS(fast);
  for (Py_ssize_t i = 0; i < n; ++i) {
    Py_buffer v;
    int ok = 0;
    if (PyObject_GetBuffer(items[i], &v, PyBUF_C_CONTIGUOUS | PyBUF_FORMAT) == 0) {
      if (v.ndim == 2 && v.shape && v.shape[0] == v.shape[1] && v.shape[0] <= INT32_MAX && v.itemsize == 16 &&
          is_complex128(v.format)) {
        ptr[i] = (uint64_t)(uintptr_t)v.buf;
        dims[i] = (int32_t)v.shape[0];
        ok = 1;
      }
      PyBuffer_Release(&v);
    } else {
      PyErr_Clear();
    }
    if (!ok) {
      ptr[i] = 0;
      dims[i] = 0;
      PyObject* idx = PyLong_FromSsize_t(i);
      if (!idx || PyList_Append(redo, idx) < 0) {
        Py_XDECREF(idx);
        Py_CLEAR(redo);
        goto done;
      }
      Py_DECREF(idx);
    }
  }
done:
  PyBuffer_Release(&db);
  PyBuffer_Release(&pb);
  Py_DECREF(fast);
  return redo;
}

static PyMethodDef methods[] = {
    {"collect", collect, METH_VARARGS, "collect(seq, ptr, dims) -> indices of the items to convert first"},
    {NULL, NULL, 0, NULL}};

static struct PyModuleDef module = {PyModuleDef_HEAD_INIT, "_hostptr", NULL, -1, methods, NULL, NULL, NULL, NULL};

PyMODINIT_FUNC PyInit__hostptr(void) { return PyModule_Create(&module); }
