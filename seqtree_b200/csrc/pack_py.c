/* Packing of the Python mirror's sequence lists: one pass over a list of ASCII str objects
 * that copies their characters into one buffer and records int64 offsets, without building a
 * joined string first.  Built as the extension module seqtree_b200._pack (CPython C API); the
 * CUDA library itself does not depend on Python.
 *
 *   _pack.pack(list) -> (bytearray data, bytearray offsets) or None
 *   _pack.gather(data, offsets, rows) -> (bytearray data, bytearray offsets)
 *
 * None means the list holds something else than compact ASCII str objects (other types,
 * non-ASCII text); the caller then takes its general path.  offsets holds count + 1 int64
 * values, data at least one byte. */
#define PY_SSIZE_T_CLEAN
#include <Python.h>

#include <stdint.h>
#include <string.h>

static PyObject* pack(PyObject* self, PyObject* arg) {
    (void)self;
    if (!PyList_Check(arg)) Py_RETURN_NONE;
    const Py_ssize_t n = PyList_GET_SIZE(arg);
    int64_t total = 0;
    for (Py_ssize_t i = 0; i < n; ++i) {
        PyObject* s = PyList_GET_ITEM(arg, i);
        if (!PyUnicode_Check(s) || !PyUnicode_IS_COMPACT_ASCII(s)) Py_RETURN_NONE;
        total += (int64_t)PyUnicode_GET_LENGTH(s);
    }
    PyObject* data = PyByteArray_FromStringAndSize(NULL, total > 0 ? (Py_ssize_t)total : 1);
    if (!data) return NULL;
    PyObject* off = PyByteArray_FromStringAndSize(NULL, (Py_ssize_t)((n + 1) * 8));
    if (!off) {
        Py_DECREF(data);
        return NULL;
    }
    char* d = PyByteArray_AS_STRING(data);
    int64_t* o = (int64_t*)PyByteArray_AS_STRING(off);
    if (total == 0) d[0] = 0;
    int64_t w = 0;
    o[0] = 0;
    for (Py_ssize_t i = 0; i < n; ++i) {
        PyObject* s = PyList_GET_ITEM(arg, i);
        const Py_ssize_t l = PyUnicode_GET_LENGTH(s);
        memcpy(d + w, PyUnicode_DATA(s), (size_t)l);
        w += l;
        o[i + 1] = w;
    }
    return Py_BuildValue("(NN)", data, off);
}

/* gather(data, offsets, rows) -> (bytearray data, bytearray int64 offsets): the listed rows of a
 * packed set (bytes `data`, count + 1 int64 `offsets`), in the listed order; `rows` is int64.
 * IndexError for a row outside [0, count), ValueError for malformed offsets. */
static PyObject* gather(PyObject* self, PyObject* args) {
    (void)self;
    Py_buffer data, off, rows;
    if (!PyArg_ParseTuple(args, "y*y*y*", &data, &off, &rows)) return NULL;
    PyObject* result = NULL;
    const int64_t* o = (const int64_t*)off.buf;
    const int64_t* r = (const int64_t*)rows.buf;
    const Py_ssize_t count = off.len / 8 - 1, n = rows.len / 8;
    if (off.len % 8 || rows.len % 8 || count < 0) {
        PyErr_SetString(PyExc_ValueError, "offsets and rows must be int64 arrays");
        goto done;
    }
    int64_t total = 0;
    for (Py_ssize_t i = 0; i < n; ++i) {
        if (r[i] < 0 || r[i] >= count) {
            PyErr_SetString(PyExc_IndexError, "row index out of range");
            goto done;
        }
        const int64_t a = o[r[i]], b = o[r[i] + 1];
        if (a < 0 || b < a || b > (int64_t)data.len) {
            PyErr_SetString(PyExc_ValueError, "offsets out of order or past the data");
            goto done;
        }
        total += b - a;
    }
    {
        PyObject* od = PyByteArray_FromStringAndSize(NULL, total > 0 ? (Py_ssize_t)total : 1);
        PyObject* oo = od ? PyByteArray_FromStringAndSize(NULL, (Py_ssize_t)((n + 1) * 8)) : NULL;
        if (!od || !oo) {
            Py_XDECREF(od);
            goto done;
        }
        char* d = PyByteArray_AS_STRING(od);
        int64_t* w = (int64_t*)PyByteArray_AS_STRING(oo);
        const char* src = (const char*)data.buf;
        if (total == 0) d[0] = 0;
        int64_t at = 0;
        w[0] = 0;
        for (Py_ssize_t i = 0; i < n; ++i) {
            const int64_t a = o[r[i]], len = o[r[i] + 1] - a;
            memcpy(d + at, src + a, (size_t)len);
            at += len;
            w[i + 1] = at;
        }
        result = Py_BuildValue("(NN)", od, oo);
    }
done:
    PyBuffer_Release(&data);
    PyBuffer_Release(&off);
    PyBuffer_Release(&rows);
    return result;
}

static PyMethodDef methods[] = {
    {"pack", pack, METH_O, "Pack a list of ASCII str into (bytearray data, bytearray int64 offsets)."},
    {"gather", gather, METH_VARARGS,
     "The listed rows of a packed set: (bytearray data, bytearray int64 offsets)."},
    {NULL, NULL, 0, NULL},
};

static struct PyModuleDef module = {PyModuleDef_HEAD_INIT, "_pack", NULL, -1, methods,
                                    NULL, NULL, NULL, NULL};

PyMODINIT_FUNC PyInit__pack(void) { return PyModule_Create(&module); }
