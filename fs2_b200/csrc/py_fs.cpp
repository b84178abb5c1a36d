// py_fs.cpp -- the CPython extension fs._fs on top of libfs2gpu.
//
// Drop-in for the reference's extension (py/py_package.cpp:28-157 and the
// py/py_*.cpp wrappers it lists) for the particle-mesh / COLA / 2LPT path:
// the same method names, PyArg_ParseTuple formats and PyCapsule names
// ("_Particles", "_FFT", "_PowerSpectrum").  Every method parses its
// arguments and calls one or two functions of the C ABI (include/fs2gpu.h);
// error codes become the Python exceptions the reference raises.
//
// The leapfrog integrator and the snapshot writer are provided too; the
// reference's methods outside this path (FoF, kd-tree, Gadget writer, Mem)
// are not.
#define PY_SSIZE_T_CLEAN
#include <Python.h>
#define NPY_NO_DEPRECATED_API NPY_1_7_API_VERSION
#include <numpy/arrayobject.h>

#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "fs2gpu.h"

namespace {

fs2g_ctx* g_ctx = nullptr;
int g_loglevel = 2;

// status code -> Python exception, as the reference's wrappers map C++
// exceptions (e.g. py/py_pm.cpp:76-82); returns NULL for `return`.
PyObject* raise(int code) {
  const char* msg = fs2g_last_error();
  PyObject* type = PyExc_RuntimeError;
  switch(code) {
    case FS2G_ERR_ASSERTION: type = PyExc_AssertionError; break;
    case FS2G_ERR_IO:        type = PyExc_IOError; break;
    case FS2G_ERR_MEMORY:    type = PyExc_MemoryError; break;
    case FS2G_ERR_VALUE:     type = PyExc_ValueError; break;
    case FS2G_ERR_INDEX:     type = PyExc_IndexError; break;
    default:                 type = PyExc_RuntimeError; break;
  }
  PyErr_SetString(type, msg && *msg ? msg : "fs2gpu error");
  return nullptr;
}

fs2g_ctx* ctx() {
  if(!g_ctx) {
    int dev = 0;
    if(const char* e = std::getenv("FS2_DEVICE")) dev = std::atoi(e);
    int r = fs2g_ctx_create(dev, &g_ctx);
    if(r != FS2G_OK) { raise(r); g_ctx = nullptr; }
  }
  return g_ctx;
}

#define CTX_OR_NULL(c) fs2g_ctx* c = ctx(); if(!c) return nullptr
#define CHECK(call) do { int r_ = (call); if(r_ != FS2G_OK) return raise(r_); } while(0)

template<class T> T* capsule(PyObject* o, const char* name) {
  // py_assert_ptr semantics (py/py_assert.h:9-10): TypeError on a bad capsule
  // (PyCapsule_GetPointer's own ValueError is replaced, as there)
  T* p = (T*) PyCapsule_GetPointer(o, name);
  if(!p) PyErr_SetString(PyExc_TypeError, "py_assersion error");
  return p;
}

void particles_destructor(PyObject* o) {
  fs2g_particles* p = (fs2g_particles*) PyCapsule_GetPointer(o, "_Particles");
  if(p) fs2g_particles_free(p);
}

void power_destructor(PyObject* o) {
  fs2g_power* p = (fs2g_power*) PyCapsule_GetPointer(o, "_PowerSpectrum");
  if(p) fs2g_power_free(p);
}

void fft_destructor(PyObject* o) {
  fs2g_fft* f = (fs2g_fft*) PyCapsule_GetPointer(o, "_FFT");
  if(f) fs2g_fft_free(f);
}

// a float32 (n, 3) array of one particle field
PyObject* field_rows(fs2g_particles* p, int field) {
  size_t n = 0;
  fs2g_particles_len(p, &n);
  npy_intp dims[2] = {(npy_intp) n, 3};
  PyObject* arr = PyArray_ZEROS(2, dims, NPY_FLOAT, 0);
  if(!arr) return nullptr;
  int r;
  Py_BEGIN_ALLOW_THREADS
  r = fs2g_particles_copy_out(p, field, PyArray_DATA((PyArrayObject*) arr), 0, n);
  Py_END_ALLOW_THREADS
  if(r != FS2G_OK) { Py_DECREF(arr); return raise(r); }
  return arr;
}

// ------------------------------------------------------------------ msg / comm
PyObject* py_set_loglevel(PyObject*, PyObject* args) {
  int level;
  if(!PyArg_ParseTuple(args, "i", &level)) return nullptr;
  g_loglevel = level;
  Py_RETURN_NONE;
}
PyObject* py_comm_mpi_init(PyObject*, PyObject*) { Py_RETURN_NONE; }
PyObject* py_comm_mpi_finalise(PyObject*, PyObject*) { Py_RETURN_NONE; }
PyObject* py_comm_hello(PyObject*, PyObject*) {
  PySys_WriteStdout("Hello from node 0 / 1\n");
  Py_RETURN_NONE;
}
PyObject* py_comm_this_node(PyObject*, PyObject*) { return Py_BuildValue("i", 0); }
PyObject* py_comm_n_nodes(PyObject*, PyObject*) { return Py_BuildValue("i", 1); }
PyObject* py_config_precision(PyObject*, PyObject*) { return Py_BuildValue("s", "single"); }

// ------------------------------------------------------------------ cosmology
PyObject* py_cosmology_init(PyObject*, PyObject* args) {   // py_cosmology.cpp:4
  double om;
  if(!PyArg_ParseTuple(args, "d", &om)) return nullptr;
  CHECK(fs2g_cosmology_init(om));
  Py_RETURN_NONE;
}
PyObject* py_cosmology_D_growth(PyObject*, PyObject* args) {   // :18
  double a, D;
  if(!PyArg_ParseTuple(args, "d", &a)) return nullptr;
  CHECK(fs2g_cosmology_D_growth(a, &D));
  return Py_BuildValue("d", D);
}
PyObject* py_cosmology_D2_growth(PyObject*, PyObject* args) {   // :28
  double a, D, D2;
  if(!PyArg_ParseTuple(args, "d", &a)) return nullptr;
  CHECK(fs2g_cosmology_D_growth(a, &D));
  CHECK(fs2g_cosmology_D2_growth(a, D, &D2));
  return Py_BuildValue("d", D2);
}

// ------------------------------------------------------------------ power
PyObject* py_power_alloc(PyObject*, PyObject* args) {   // py_power.cpp:12
  PyObject* bytes;
  if(!PyArg_ParseTuple(args, "O&", PyUnicode_FSConverter, &bytes)) return nullptr;
  char* filename; Py_ssize_t len;
  PyBytes_AsStringAndSize(bytes, &filename, &len);
  fs2g_power* ps = nullptr;
  int r = fs2g_power_alloc(filename, &ps);
  Py_DECREF(bytes);
  if(r != FS2G_OK) {
    if(r == FS2G_ERR_IO) {
      PyErr_SetString(PyExc_IOError, "PowerSpectrum File Error");
      return nullptr;
    }
    return raise(r);
  }
  return PyCapsule_New(ps, "_PowerSpectrum", power_destructor);
}
PyObject* py_power_n(PyObject*, PyObject* args) {   // py_power.cpp:66
  PyObject* o;
  if(!PyArg_ParseTuple(args, "O", &o)) return nullptr;
  fs2g_power* ps = capsule<fs2g_power>(o, "_PowerSpectrum");
  if(!ps) return nullptr;
  int n; CHECK(fs2g_power_n(ps, &n));
  return Py_BuildValue("i", n);
}
PyObject* py_power_i(PyObject*, PyObject* args) {   // py_power.cpp:120
  PyObject* o; int i;
  if(!PyArg_ParseTuple(args, "Oi", &o, &i)) return nullptr;
  fs2g_power* ps = capsule<fs2g_power>(o, "_PowerSpectrum");
  if(!ps) return nullptr;
  double k, P; CHECK(fs2g_power_i(ps, i, &k, &P));
  return Py_BuildValue("dd", k, P);
}
PyObject* py_power_sigma(PyObject*, PyObject* args) {   // py_power.cpp:51
  PyObject* o; double R;
  if(!PyArg_ParseTuple(args, "Od", &o, &R)) return nullptr;
  fs2g_power* ps = capsule<fs2g_power>(o, "_PowerSpectrum");
  if(!ps) return nullptr;
  double s; CHECK(fs2g_power_sigma(ps, R, &s));
  return Py_BuildValue("d", s);
}
PyObject* py_power_P(PyObject*, PyObject* args) {
  PyObject* o; double k;
  if(!PyArg_ParseTuple(args, "Od", &o, &k)) return nullptr;
  fs2g_power* ps = capsule<fs2g_power>(o, "_PowerSpectrum");
  if(!ps) return nullptr;
  double P; CHECK(fs2g_power_P(ps, k, &P));
  return Py_BuildValue("d", P);
}

// ------------------------------------------------------------------ particles
fs2g_particles* particles_arg(PyObject* o) {
  return capsule<fs2g_particles>(o, "_Particles");
}

PyObject* py_particles_alloc(PyObject*, PyObject* args) {   // py_particles.cpp:143
  unsigned long long np; double boxsize;
  if(!PyArg_ParseTuple(args, "Kd", &np, &boxsize)) return nullptr;
  CTX_OR_NULL(c);
  fs2g_particles* p = nullptr;
  CHECK(fs2g_particles_alloc(c, (size_t) np, boxsize, &p));
  return PyCapsule_New(p, "_Particles", particles_destructor);
}
PyObject* py_particles_len(PyObject*, PyObject* args) {   // :166
  PyObject* o;
  if(!PyArg_ParseTuple(args, "O", &o)) return nullptr;
  fs2g_particles* p = particles_arg(o); if(!p) return nullptr;
  size_t n; CHECK(fs2g_particles_len(p, &n));
  return Py_BuildValue("k", (unsigned long) n);
}
PyObject* py_particles_np_total(PyObject*, PyObject* args) {   // :358
  PyObject* o;
  if(!PyArg_ParseTuple(args, "O", &o)) return nullptr;
  fs2g_particles* p = particles_arg(o); if(!p) return nullptr;
  uint64_t n; CHECK(fs2g_particles_np_total(p, &n));
  return Py_BuildValue("k", (unsigned long) n);
}
PyObject* py_particles_update_np_total(PyObject*, PyObject* args) {   // :273
  PyObject* o;
  if(!PyArg_ParseTuple(args, "O", &o)) return nullptr;
  fs2g_particles* p = particles_arg(o); if(!p) return nullptr;
  CHECK(fs2g_particles_update_np_total(p));
  Py_RETURN_NONE;
}
PyObject* py_particles_id_asarray(PyObject*, PyObject* args) {   // :291
  PyObject* o;
  if(!PyArg_ParseTuple(args, "O", &o)) return nullptr;
  fs2g_particles* p = particles_arg(o); if(!p) return nullptr;
  size_t n = 0; fs2g_particles_len(p, &n);
  npy_intp dims[1] = {(npy_intp) n};
  PyObject* arr = PyArray_ZEROS(1, dims, NPY_UINT64, 0);
  if(!arr) return nullptr;
  int r;
  Py_BEGIN_ALLOW_THREADS
  r = fs2g_particles_copy_out(p, FS2G_FIELD_ID, PyArray_DATA((PyArrayObject*) arr), 0, n);
  Py_END_ALLOW_THREADS
  if(r != FS2G_OK) { Py_DECREF(arr); return raise(r); }
  return arr;
}
PyObject* py_particles_x_asarray(PyObject*, PyObject* args) {   // :306
  PyObject* o; int x_type;
  if(!PyArg_ParseTuple(args, "Oi", &o, &x_type)) return nullptr;
  fs2g_particles* p = particles_arg(o); if(!p) return nullptr;
  static const int fields[3] = {FS2G_FIELD_X, FS2G_FIELD_DX1, FS2G_FIELD_DX2};
  if(x_type < 0 || x_type > 2) {
    PyErr_SetString(PyExc_TypeError, "py_assersion error");
    return nullptr;
  }
  return field_rows(p, fields[x_type]);
}
PyObject* py_particles_v_asarray(PyObject*, PyObject* args) {
  PyObject* o;
  if(!PyArg_ParseTuple(args, "O", &o)) return nullptr;
  fs2g_particles* p = particles_arg(o); if(!p) return nullptr;
  return field_rows(p, FS2G_FIELD_V);
}
PyObject* py_particles_force_asarray(PyObject*, PyObject* args) {   // :343
  PyObject* o;
  if(!PyArg_ParseTuple(args, "O", &o)) return nullptr;
  fs2g_particles* p = particles_arg(o); if(!p) return nullptr;
  return field_rows(p, FS2G_FIELD_FORCE);
}
PyObject* py_particles_periodic_wrapup(PyObject*, PyObject* args) {   // :371
  PyObject* o;
  if(!PyArg_ParseTuple(args, "O", &o)) return nullptr;
  fs2g_particles* p = particles_arg(o); if(!p) return nullptr;
  CHECK(fs2g_particles_periodic_wrapup(p));
  Py_RETURN_NONE;
}
PyObject* py_particles_clear(PyObject*, PyObject* args) {   // :386
  PyObject* o;
  if(!PyArg_ParseTuple(args, "O", &o)) return nullptr;
  fs2g_particles* p = particles_arg(o); if(!p) return nullptr;
  CHECK(fs2g_particles_clear(p));
  Py_RETURN_NONE;
}
PyObject* py_particles_append(PyObject*, PyObject* args) {   // :403-462
  PyObject *o, *arr;
  if(!PyArg_ParseTuple(args, "OO", &o, &arr)) return nullptr;
  fs2g_particles* p = particles_arg(o); if(!p) return nullptr;
  if(arr != Py_None) {
    Py_buffer view;
    if(PyObject_GetBuffer(arr, &view, PyBUF_ANY_CONTIGUOUS | PyBUF_FORMAT) == -1)
      return nullptr;
    if(view.ndim != 2) {
      PyErr_SetString(PyExc_TypeError, "Expected a 2-dimensional array");
      PyBuffer_Release(&view);
      return nullptr;
    }
    if(std::strcmp(view.format, "d") != 0) {
      PyErr_SetString(PyExc_TypeError, "Expected an array of doubles");
      PyBuffer_Release(&view);
      return nullptr;
    }
    if(view.shape[1] < 3) {
      PyErr_SetString(PyExc_TypeError, "Expected at least 3 columns for x y z");
      PyBuffer_Release(&view);
      return nullptr;
    }
    const ptrdiff_t rs = view.strides[0]/(ptrdiff_t) sizeof(double);
    const ptrdiff_t cs = view.strides[1]/(ptrdiff_t) sizeof(double);
    int r = fs2g_particles_append(p, (const double*) view.buf,
                                  (size_t) view.shape[0], rs, cs);
    PyBuffer_Release(&view);
    if(r != FS2G_OK) return raise(r);
  }
  else CHECK(fs2g_particles_update_np_total(p));
  Py_RETURN_NONE;
}

// the 14-column float view of sizeof(Particle)/sizeof(Float) rows that
// py_particles_getitem and py_particles_slice return (:217-270, :180-215):
// x, v, dx1, dx2 and the 8-byte id in columns 12-13
PyObject* particle_rows(fs2g_particles* p, const std::vector<size_t>& sel,
                        bool wrap_x, double boxsize) {
  size_t n = 0; fs2g_particles_len(p, &n);
  std::vector<float> f[4];
  std::vector<uint64_t> id(n);
  static const int fields[4] = {FS2G_FIELD_X, FS2G_FIELD_V, FS2G_FIELD_DX1,
                                FS2G_FIELD_DX2};
  for(int k = 0; k < 4; k++) {
    f[k].resize(3*n);
    if(n) { int r = fs2g_particles_copy_out(p, fields[k], f[k].data(), 0, n);
            if(r != FS2G_OK) return raise(r); }
  }
  if(n) { int r = fs2g_particles_copy_out(p, FS2G_FIELD_ID, id.data(), 0, n);
          if(r != FS2G_OK) return raise(r); }
  npy_intp dims[2] = {(npy_intp) sel.size(), 14};
  PyObject* arr = PyArray_ZEROS(2, dims, NPY_FLOAT, 0);
  if(!arr) return nullptr;
  float* out = (float*) PyArray_DATA((PyArrayObject*) arr);
  const float L = (float) boxsize;
  for(size_t j = 0; j < sel.size(); j++) {
    const size_t i = sel[j];
    for(int k = 0; k < 4; k++)
      for(int c = 0; c < 3; c++) {
        float v = f[k][3*i + c];
        if(wrap_x && k == 0) { if(v < 0) v += L; if(v >= L) v -= L; }
        out[14*j + 3*k + c] = v;
      }
    std::memcpy(out + 14*j + 12, &id[i], 8);
  }
  return arr;
}

PyObject* py_particles_getitem(PyObject*, PyObject* args) {   // :217-270
  PyObject *o, *index;
  if(!PyArg_ParseTuple(args, "OO", &o, &index)) return nullptr;
  fs2g_particles* p = particles_arg(o); if(!p) return nullptr;
  size_t n = 0; fs2g_particles_len(p, &n);
  if(PyNumber_Check(index)) {
    long i = PyLong_AsLong(index);
    if(i == -1 && PyErr_Occurred()) return nullptr;
    if(i < 0) i = (long) n + i;
    if(i < 0 || i >= (long) n) { PyErr_SetNone(PyExc_IndexError); return nullptr; }
    float x[3];
    CHECK(fs2g_particles_copy_out(p, FS2G_FIELD_X, x, (size_t) i, 1));
    return Py_BuildValue("(ddd)", (double) x[0], (double) x[1], (double) x[2]);
  }
  if(PySlice_Check(index)) {
    Py_ssize_t start, stop, step, length;
    if(PySlice_GetIndicesEx(index, (Py_ssize_t) n, &start, &stop, &step, &length))
      return nullptr;
    std::vector<size_t> sel;
    for(Py_ssize_t k = 0, i = start; k < length; k++, i += step) sel.push_back((size_t) i);
    double L; fs2g_particles_boxsize(p, &L);
    return particle_rows(p, sel, false, L);
  }
  PyErr_SetString(PyExc_TypeError, "index must be an integer or a slice");
  return nullptr;
}

PyObject* py_particles_slice(PyObject*, PyObject* args) {   // :180-215
  PyObject* o; double frac;
  if(!PyArg_ParseTuple(args, "Od", &o, &frac)) return nullptr;
  fs2g_particles* p = particles_arg(o); if(!p) return nullptr;
  size_t n = 0; fs2g_particles_len(p, &n);
  double Ld; fs2g_particles_boxsize(p, &Ld);
  const float L = (float) Ld, x_max = (float)(frac*L);
  std::vector<float> x(3*n);
  if(n) CHECK(fs2g_particles_copy_out(p, FS2G_FIELD_X, x.data(), 0, n));
  std::vector<size_t> sel;
  for(size_t i = 0; i < n; i++) {
    float z = x[3*i + 2];
    if(z < 0) z += L;
    if(z >= L) z -= L;
    if(z < x_max) sel.push_back(i);
  }
  return particle_rows(p, sel, true, Ld);
}

// extra accessors (no reference counterpart)
PyObject* py_particles_set(PyObject*, PyObject* args) {
  // _particles_set(_p, field, array): field 'x','v','dx1','dx2','f' as
  // float32 (n, 3) rows, or 'id' as uint64 (n,); sets np_local = n
  PyObject *o, *arr; const char* name;
  if(!PyArg_ParseTuple(args, "OsO", &o, &name, &arr)) return nullptr;
  fs2g_particles* p = particles_arg(o); if(!p) return nullptr;
  int field = -1;
  std::string s(name);
  if(s == "x") field = FS2G_FIELD_X; else if(s == "v") field = FS2G_FIELD_V;
  else if(s == "dx1") field = FS2G_FIELD_DX1; else if(s == "dx2") field = FS2G_FIELD_DX2;
  else if(s == "f" || s == "force") field = FS2G_FIELD_FORCE;
  else if(s == "id") field = FS2G_FIELD_ID;
  else { PyErr_SetString(PyExc_ValueError, "unknown field"); return nullptr; }
  const int type = field == FS2G_FIELD_ID ? NPY_UINT64 : NPY_FLOAT;
  PyArrayObject* a = (PyArrayObject*) PyArray_FROMANY(arr, type, 1, 2,
                                                      NPY_ARRAY_C_CONTIGUOUS | NPY_ARRAY_ALIGNED);
  if(!a) return nullptr;
  const size_t n = (size_t) PyArray_DIM(a, 0);
  if(field != FS2G_FIELD_ID && (PyArray_NDIM(a) != 2 || PyArray_DIM(a, 1) != 3)) {
    Py_DECREF(a);
    PyErr_SetString(PyExc_ValueError, "expected an (n, 3) array");
    return nullptr;
  }
  int r;
  Py_BEGIN_ALLOW_THREADS
  r = fs2g_particles_copy_in(p, field, PyArray_DATA(a), 0, n);
  Py_END_ALLOW_THREADS
  Py_DECREF(a);
  if(r != FS2G_OK) return raise(r);
  CHECK(fs2g_particles_set_np(p, n));
  CHECK(fs2g_particles_update_np_total(p));
  Py_RETURN_NONE;
}

PyObject* py_particles_a(PyObject*, PyObject* args) {
  // _particles_a(_p) -> (a_x, a_v, a_f); _particles_a(_p, ax, av, af) sets
  PyObject* o; double ax = -1, av = -1, af = -1;
  if(!PyArg_ParseTuple(args, "O|ddd", &o, &ax, &av, &af)) return nullptr;
  fs2g_particles* p = particles_arg(o); if(!p) return nullptr;
  if(PyTuple_Size(args) == 4) CHECK(fs2g_particles_set_a(p, ax, av, af));
  CHECK(fs2g_particles_get_a(p, &ax, &av, &af));
  return Py_BuildValue("ddd", ax, av, af);
}

PyObject* py_particles_boxsize(PyObject*, PyObject* args) {
  PyObject* o;
  if(!PyArg_ParseTuple(args, "O", &o)) return nullptr;
  fs2g_particles* p = particles_arg(o); if(!p) return nullptr;
  double L; CHECK(fs2g_particles_boxsize(p, &L));
  return Py_BuildValue("d", L);
}

// ------------------------------------------------------------------ LPT
PyObject* py_lpt(PyObject*, PyObject* args) {   // py_lpt.cpp:9-42
  PyObject* py_ps; int nc; double a, boxsize; unsigned long seed;
  const char* kind;
  if(!PyArg_ParseTuple(args, "iddkOs", &nc, &boxsize, &a, &seed, &py_ps, &kind))
    return nullptr;
  fs2g_power* ps = capsule<fs2g_power>(py_ps, "_PowerSpectrum");
  if(!ps) return nullptr;
  CTX_OR_NULL(c);
  fs2g_particles* p = nullptr;
  int r;
  Py_BEGIN_ALLOW_THREADS
  r = fs2g_lpt(c, nc, boxsize, a, seed, ps, kind, &p);
  Py_END_ALLOW_THREADS
  if(r != FS2G_OK) return raise(r);
  return PyCapsule_New(p, "_Particles", particles_destructor);
}

PyObject* py_lpt_from_draws(PyObject*, PyObject* args) {
  // _lpt_from_draws(nc, boxsize, a, u_phase, u_ampl, _ps, kind)
  PyObject *py_ps, *up, *ua; int nc; double a, boxsize; const char* kind;
  if(!PyArg_ParseTuple(args, "iddOOOs", &nc, &boxsize, &a, &up, &ua, &py_ps, &kind))
    return nullptr;
  fs2g_power* ps = capsule<fs2g_power>(py_ps, "_PowerSpectrum");
  if(!ps) return nullptr;
  PyArrayObject* A = (PyArrayObject*) PyArray_FROMANY(up, NPY_DOUBLE, 1, 3, NPY_ARRAY_CARRAY_RO);
  if(!A) return nullptr;
  PyArrayObject* B = (PyArrayObject*) PyArray_FROMANY(ua, NPY_DOUBLE, 1, 3, NPY_ARRAY_CARRAY_RO);
  if(!B) { Py_DECREF(A); return nullptr; }
  const npy_intp need = (npy_intp) nc*nc*(nc/2);
  if(PyArray_SIZE(A) != need || PyArray_SIZE(B) != need) {
    Py_DECREF(A); Py_DECREF(B);
    PyErr_SetString(PyExc_ValueError, "draws must hold nc*nc*(nc/2) values");
    return nullptr;
  }
  fs2g_ctx* c = ctx();
  if(!c) { Py_DECREF(A); Py_DECREF(B); return nullptr; }
  fs2g_particles* p = nullptr;
  int r;
  Py_BEGIN_ALLOW_THREADS
  r = fs2g_lpt_from_draws(c, nc, boxsize, a, (const double*) PyArray_DATA(A),
                          (const double*) PyArray_DATA(B), ps, kind, &p);
  Py_END_ALLOW_THREADS
  Py_DECREF(A); Py_DECREF(B);
  if(r != FS2G_OK) return raise(r);
  return PyCapsule_New(p, "_Particles", particles_destructor);
}

PyObject* py_lpt_from_delta_k(PyObject*, PyObject* args) {
  // _lpt_from_delta_k(nc, boxsize, a, delta_k complex64 [nc][nc][nc/2+1], kind)
  PyObject* dk; int nc; double a, boxsize; const char* kind;
  if(!PyArg_ParseTuple(args, "iddOs", &nc, &boxsize, &a, &dk, &kind)) return nullptr;
  PyArrayObject* A = (PyArrayObject*) PyArray_FROMANY(dk, NPY_COMPLEX64, 1, 3, NPY_ARRAY_CARRAY_RO);
  if(!A) return nullptr;
  if(PyArray_SIZE(A) != (npy_intp) nc*nc*(nc/2 + 1)) {
    Py_DECREF(A);
    PyErr_SetString(PyExc_ValueError, "delta_k must hold nc*nc*(nc/2+1) values");
    return nullptr;
  }
  fs2g_ctx* c = ctx();
  if(!c) { Py_DECREF(A); return nullptr; }
  fs2g_particles* p = nullptr;
  int r;
  Py_BEGIN_ALLOW_THREADS
  r = fs2g_lpt_from_delta_k(c, nc, boxsize, a, (const float*) PyArray_DATA(A), kind, &p);
  Py_END_ALLOW_THREADS
  Py_DECREF(A);
  if(r != FS2G_OK) return raise(r);
  return PyCapsule_New(p, "_Particles", particles_destructor);
}

PyObject* py_lpt_draws(PyObject*, PyObject* args) {
  // _lpt_draws(nc, seed) -> (u_phase, u_ampl), each [nc][nc][nc/2] float64
  int nc; unsigned long seed;
  if(!PyArg_ParseTuple(args, "ik", &nc, &seed)) return nullptr;
  if(nc < 2) { PyErr_SetString(PyExc_ValueError, "nc must be at least 2"); return nullptr; }
  npy_intp dims[3] = {nc, nc, nc/2};
  PyObject* A = PyArray_ZEROS(3, dims, NPY_DOUBLE, 0);
  PyObject* B = PyArray_ZEROS(3, dims, NPY_DOUBLE, 0);
  if(!A || !B) { Py_XDECREF(A); Py_XDECREF(B); return nullptr; }
  int r = fs2g_lpt_draws(nullptr, nc, seed, (double*) PyArray_DATA((PyArrayObject*) A),
                         (double*) PyArray_DATA((PyArrayObject*) B));
  if(r != FS2G_OK) { Py_DECREF(A); Py_DECREF(B); return raise(r); }
  return Py_BuildValue("NN", A, B);
}

PyObject* py_lpt_set_offset(PyObject*, PyObject* args) {   // py_lpt.cpp:44
  double offset;
  if(!PyArg_ParseTuple(args, "d", &offset)) return nullptr;
  CHECK(fs2g_lpt_set_offset(offset));
  Py_RETURN_NONE;
}

PyObject* py_lpt_set_zeldovich_force(PyObject*, PyObject* args) {   // py_lpt.cpp:57
  PyObject* o; double a;
  if(!PyArg_ParseTuple(args, "Od", &o, &a)) return nullptr;
  fs2g_particles* p = particles_arg(o); if(!p) return nullptr;
  CTX_OR_NULL(c);
  CHECK(fs2g_lpt_set_zeldovich_force(c, p, a));
  Py_RETURN_NONE;
}

// ------------------------------------------------------------------ PM
#define PM_PARTICLE_CALL(fn) \
  PyObject* o; \
  if(!PyArg_ParseTuple(args, "O", &o)) return nullptr; \
  fs2g_particles* p = particles_arg(o); if(!p) return nullptr; \
  CTX_OR_NULL(c); \
  int r; \
  Py_BEGIN_ALLOW_THREADS \
  r = fn(c, p); \
  Py_END_ALLOW_THREADS \
  if(r != FS2G_OK) return raise(r);

PyObject* py_pm_init(PyObject*, PyObject* args) {   // py_pm.cpp:10
  int nc_pm; double pm_factor, boxsize;
  if(!PyArg_ParseTuple(args, "idd", &nc_pm, &pm_factor, &boxsize)) return nullptr;
  CTX_OR_NULL(c);
  CHECK(fs2g_pm_init(c, nc_pm, pm_factor, boxsize));
  Py_RETURN_NONE;
}
PyObject* py_pm_compute_density(PyObject*, PyObject* args) {   // py_pm.cpp:34
  PM_PARTICLE_CALL(fs2g_pm_compute_density)
  fs2g_fft* f = nullptr;
  CHECK(fs2g_pm_fft(c, &f));
  return PyCapsule_New(f, "_FFT", nullptr);   // owned by the pm module
}
PyObject* py_pm_compute_force(PyObject*, PyObject* args) {   // py_pm.cpp:59
  PM_PARTICLE_CALL(fs2g_pm_compute_force)
  Py_RETURN_NONE;
}
PyObject* py_pm_send_positions(PyObject*, PyObject* args) {   // py_pm.cpp:88
  PM_PARTICLE_CALL(fs2g_pm_send_positions)
  Py_RETURN_NONE;
}
PyObject* py_pm_get_forces(PyObject*, PyObject* args) {   // py_pm.cpp:127
  PM_PARTICLE_CALL(fs2g_pm_get_forces)
  Py_RETURN_NONE;
}
PyObject* py_pm_domain_init(PyObject*, PyObject* args) {   // py_pm.cpp:183
  PyObject* o;
  if(!PyArg_ParseTuple(args, "O", &o)) return nullptr;
  if(!particles_arg(o)) return nullptr;
  Py_RETURN_NONE;   // no domain decomposition on one GPU
}
PyObject* py_pm_set_packet_size(PyObject*, PyObject* args) {   // py_pm.cpp:201
  int packet_size;
  if(!PyArg_ParseTuple(args, "i", &packet_size)) return nullptr;
  Py_RETURN_NONE;   // no halo packets on one GPU
}
PyObject* py_pm_check_total_density(PyObject*, PyObject*) {   // py_pm.cpp:113
  CTX_OR_NULL(c);
  CHECK(fs2g_pm_check_total_density(c));
  Py_RETURN_NONE;
}
PyObject* py_pm_force(PyObject*, PyObject* args) {
  // fs.pm.force in one call (py/fs/pm.py:17-31)
  PM_PARTICLE_CALL(fs2g_pm_force)
  Py_RETURN_NONE;
}
PyObject* py_pm_set_deposit_mode(PyObject*, PyObject* args) {
  const char* mode;
  if(!PyArg_ParseTuple(args, "s", &mode)) return nullptr;
  CTX_OR_NULL(c);
  std::string m(mode);
  int code = m == "atomic" ? FS2G_DEPOSIT_ATOMIC
           : m == "deterministic" ? FS2G_DEPOSIT_DETERMINISTIC : -1;
  if(code < 0) {
    PyErr_SetString(PyExc_ValueError, "deposit mode is 'atomic' or 'deterministic'");
    return nullptr;
  }
  CHECK(fs2g_pm_set_deposit_mode(c, code));
  Py_RETURN_NONE;
}
PyObject* py_pm_set_bin_tile(PyObject*, PyObject* args) {
  int shape;
  if(!PyArg_ParseTuple(args, "i", &shape)) return nullptr;
  CTX_OR_NULL(c);
  CHECK(fs2g_pm_set_bin_tile(c, shape));
  Py_RETURN_NONE;
}
PyObject* py_pm_bin_tile(PyObject*, PyObject*) {
  CTX_OR_NULL(c);
  int shape = -1, tx = 0, ty = 0, tz = 0;
  CHECK(fs2g_pm_get_bin_tile(c, &shape, &tx, &ty, &tz));
  return Py_BuildValue("(iiii)", shape, tx, ty, tz);
}
PyObject* py_pm_set_check(PyObject*, PyObject* args) {
  int on;
  if(!PyArg_ParseTuple(args, "p", &on)) return nullptr;
  CTX_OR_NULL(c);
  CHECK(fs2g_pm_set_check(c, on));
  Py_RETURN_NONE;
}
PyObject* py_pm_free(PyObject*, PyObject*) {
  CTX_OR_NULL(c);
  CHECK(fs2g_pm_free(c));
  Py_RETURN_NONE;
}
PyObject* py_pm_set_fft_engine(PyObject*, PyObject* args) {
  const char* e;
  if(!PyArg_ParseTuple(args, "s", &e)) return nullptr;
  CTX_OR_NULL(c);
  std::string m(e);
  int code = m == "auto" ? FS2G_FFT_AUTO : m == "cufft" ? FS2G_FFT_CUFFT
             : m == "fused" ? FS2G_FFT_FUSED : -1;
  if(code < 0) {
    PyErr_SetString(PyExc_ValueError, "FFT engine is 'auto', 'cufft' or 'fused'");
    return nullptr;
  }
  CHECK(fs2g_pm_set_fft_engine(c, code));
  Py_RETURN_NONE;
}
PyObject* py_pm_set_fft_tile(PyObject*, PyObject* args) {
  int w;
  if(!PyArg_ParseTuple(args, "i", &w)) return nullptr;
  CTX_OR_NULL(c);
  CHECK(fs2g_pm_set_fft_tile(c, w));
  Py_RETURN_NONE;
}
PyObject* py_pm_set_keep_delta_k(PyObject*, PyObject* args) {
  int on;
  if(!PyArg_ParseTuple(args, "p", &on)) return nullptr;
  CTX_OR_NULL(c);
  CHECK(fs2g_pm_set_keep_delta_k(c, on));
  Py_RETURN_NONE;
}
PyObject* py_pm_fused(PyObject*, PyObject*) {
  CTX_OR_NULL(c);
  int f = 0; CHECK(fs2g_pm_fft_engine(c, &f));
  return PyBool_FromLong(f);
}
PyObject* py_pm_delta_k(PyObject*, PyObject*) {
  CTX_OR_NULL(c);
  int n = 0; CHECK(fs2g_pm_nc(c, &n));
  if(n <= 0) { PyErr_SetString(PyExc_RuntimeError, "PM not initialised; call pm_init()."); return nullptr; }
  npy_intp dims[3] = {n, n, n/2 + 1};
  PyObject* arr = PyArray_ZEROS(3, dims, NPY_COMPLEX64, 0);
  if(!arr) return nullptr;
  int r = fs2g_pm_delta_k_copy_out(c, (float*) PyArray_DATA((PyArrayObject*) arr));
  if(r != FS2G_OK) { Py_DECREF(arr); return raise(r); }
  return arr;
}
PyObject* py_pm_force_mesh(PyObject*, PyObject* args) {
  int axis;
  if(!PyArg_ParseTuple(args, "i", &axis)) return nullptr;
  CTX_OR_NULL(c);
  int n = 0; CHECK(fs2g_pm_nc(c, &n));
  if(n <= 0) { PyErr_SetString(PyExc_RuntimeError, "PM not initialised; call pm_init()."); return nullptr; }
  npy_intp dims[3] = {n, n, n};
  PyObject* arr = PyArray_ZEROS(3, dims, NPY_FLOAT, 0);
  if(!arr) return nullptr;
  int r = fs2g_pm_force_mesh_copy_out(c, axis, (float*) PyArray_DATA((PyArrayObject*) arr));
  if(r != FS2G_OK) { Py_DECREF(arr); return raise(r); }
  return arr;
}

// ------------------------------------------------------------------ COLA
PyObject* py_cola_kick(PyObject*, PyObject* args) {   // py_cola.cpp:4
  PyObject* o; double a_vel;
  if(!PyArg_ParseTuple(args, "Od", &o, &a_vel)) return nullptr;
  fs2g_particles* p = particles_arg(o); if(!p) return nullptr;
  CTX_OR_NULL(c);
  CHECK(fs2g_cola_kick(c, p, a_vel));
  Py_RETURN_NONE;
}
PyObject* py_cola_drift(PyObject*, PyObject* args) {   // py_cola.cpp:24
  PyObject* o; double a_pos;
  if(!PyArg_ParseTuple(args, "Od", &o, &a_pos)) return nullptr;
  fs2g_particles* p = particles_arg(o); if(!p) return nullptr;
  CTX_OR_NULL(c);
  CHECK(fs2g_cola_drift(c, p, a_pos));
  Py_RETURN_NONE;
}
// py_leapfrog.cpp:5-61: the same "Od" arguments as the reference
PyObject* py_leapfrog_initial_velocity(PyObject*, PyObject* args) {
  PyObject* o; double a;
  if(!PyArg_ParseTuple(args, "Od", &o, &a)) return nullptr;
  fs2g_particles* p = particles_arg(o); if(!p) return nullptr;
  CTX_OR_NULL(c);
  CHECK(fs2g_leapfrog_initial_velocity(c, p, a));
  Py_RETURN_NONE;
}
PyObject* py_leapfrog_kick(PyObject*, PyObject* args) {
  PyObject* o; double a_vel;
  if(!PyArg_ParseTuple(args, "Od", &o, &a_vel)) return nullptr;
  fs2g_particles* p = particles_arg(o); if(!p) return nullptr;
  CTX_OR_NULL(c);
  CHECK(fs2g_leapfrog_kick(c, p, a_vel));
  Py_RETURN_NONE;
}
PyObject* py_leapfrog_drift(PyObject*, PyObject* args) {
  PyObject* o; double a_pos;
  if(!PyArg_ParseTuple(args, "Od", &o, &a_pos)) return nullptr;
  fs2g_particles* p = particles_arg(o); if(!p) return nullptr;
  CTX_OR_NULL(c);
  CHECK(fs2g_leapfrog_drift(c, p, a_pos));
  Py_RETURN_NONE;
}
PyObject* py_cola_step(PyObject*, PyObject* args) {
  PyObject* o; double a_vel, a_pos;
  if(!PyArg_ParseTuple(args, "Odd", &o, &a_vel, &a_pos)) return nullptr;
  fs2g_particles* p = particles_arg(o); if(!p) return nullptr;
  CTX_OR_NULL(c);
  int r;
  Py_BEGIN_ALLOW_THREADS
  r = fs2g_cola_step(c, p, a_vel, a_pos);
  Py_END_ALLOW_THREADS
  if(r != FS2G_OK) return raise(r);
  Py_RETURN_NONE;
}
PyObject* py_cola_velocity(PyObject*, PyObject* args) {
  PyObject* o;
  if(!PyArg_ParseTuple(args, "O", &o)) return nullptr;
  fs2g_particles* p = particles_arg(o); if(!p) return nullptr;
  CTX_OR_NULL(c);
  size_t n = 0; fs2g_particles_len(p, &n);
  npy_intp dims[2] = {(npy_intp) n, 3};
  PyObject* arr = PyArray_ZEROS(2, dims, NPY_FLOAT, 0);
  if(!arr) return nullptr;
  int r = fs2g_cola_velocity(c, p, (float*) PyArray_DATA((PyArrayObject*) arr));
  if(r != FS2G_OK) { Py_DECREF(arr); return raise(r); }
  return arr;
}

// ------------------------------------------------------------------ FFT
PyObject* py_fft_alloc(PyObject*, PyObject* args) {   // py_fft.cpp:28
  int nc;
  if(!PyArg_ParseTuple(args, "i", &nc)) return nullptr;
  CTX_OR_NULL(c);
  fs2g_fft* f = nullptr;
  CHECK(fs2g_fft_alloc(c, nc, &f));
  return PyCapsule_New(f, "_FFT", fft_destructor);
}
PyObject* py_fft_set_test_data(PyObject*, PyObject* args) {   // py_fft.cpp:57
  PyObject* o;
  if(!PyArg_ParseTuple(args, "O", &o)) return nullptr;
  fs2g_fft* f = capsule<fs2g_fft>(o, "_FFT"); if(!f) return nullptr;
  CHECK(fs2g_fft_set_test_data(f));
  Py_RETURN_NONE;
}
PyObject* py_fft_fx_global_as_array(PyObject*, PyObject* args) {   // py_fft.cpp:87
  PyObject* o;
  if(!PyArg_ParseTuple(args, "O", &o)) return nullptr;
  fs2g_fft* f = capsule<fs2g_fft>(o, "_FFT"); if(!f) return nullptr;
  int nc = 0; CHECK(fs2g_fft_nc(f, &nc));
  npy_intp dims[3] = {nc, nc, nc};
  PyObject* arr = PyArray_ZEROS(3, dims, NPY_FLOAT, 0);
  if(!arr) return nullptr;
  int r;
  Py_BEGIN_ALLOW_THREADS
  r = fs2g_fft_fx_copy_out(f, (float*) PyArray_DATA((PyArrayObject*) arr));
  Py_END_ALLOW_THREADS
  if(r != FS2G_OK) { Py_DECREF(arr); return raise(r); }
  return arr;
}

// ------------------------------------------------------------------ context
PyObject* py_synchronize(PyObject*, PyObject*) {
  CTX_OR_NULL(c);
  int r;
  Py_BEGIN_ALLOW_THREADS
  r = fs2g_ctx_synchronize(c);
  Py_END_ALLOW_THREADS
  if(r != FS2G_OK) return raise(r);
  Py_RETURN_NONE;
}
PyObject* py_set_timing(PyObject*, PyObject* args) {
  int on;
  if(!PyArg_ParseTuple(args, "p", &on)) return nullptr;
  CTX_OR_NULL(c);
  CHECK(fs2g_ctx_set_timing(c, on));
  if(on) CHECK(fs2g_ctx_reset_timing(c));
  Py_RETURN_NONE;
}
PyObject* py_get_timing(PyObject*, PyObject*) {
  CTX_OR_NULL(c);
  const int ns = fs2g_stage_count();
  std::vector<double> ms(ns); std::vector<long> cnt(ns);
  CHECK(fs2g_ctx_get_timing(c, ms.data(), cnt.data(), ns));
  PyObject* d = PyDict_New();
  for(int i = 0; i < ns; i++) {
    if(cnt[i] == 0) continue;
    PyObject* v = Py_BuildValue("(dl)", ms[i], cnt[i]);
    PyDict_SetItemString(d, fs2g_stage_name(i), v);
    Py_DECREF(v);
  }
  return d;
}
PyObject* py_kernel_launches(PyObject*, PyObject*) {
  CTX_OR_NULL(c);
  long n = 0; CHECK(fs2g_ctx_kernel_launches(c, &n));
  return Py_BuildValue("l", n);
}
PyObject* py_set_stream(PyObject*, PyObject* args) {
  // _set_stream(cudaStream_t as int); 0 restores the context's own stream
  unsigned long long s;
  if(!PyArg_ParseTuple(args, "K", &s)) return nullptr;
  CTX_OR_NULL(c);
  CHECK(fs2g_ctx_set_stream(c, (void*)(uintptr_t) s));
  Py_RETURN_NONE;
}
PyObject* py_ctx_address(PyObject*, PyObject*) {
  // the context pointer, for callers that use the C ABI directly (ctypes)
  CTX_OR_NULL(c);
  return PyLong_FromVoidPtr((void*) c);
}
PyObject* py_particles_address(PyObject*, PyObject* args) {
  PyObject* o;
  if(!PyArg_ParseTuple(args, "O", &o)) return nullptr;
  fs2g_particles* p = particles_arg(o); if(!p) return nullptr;
  return PyLong_FromVoidPtr((void*) p);
}

PyMethodDef methods[] = {
  {"set_loglevel", py_set_loglevel, METH_VARARGS, "set loglevel: 0=debug, 1=verbose, ..."},
  {"comm_mpi_init", py_comm_mpi_init, METH_VARARGS, "no MPI on one GPU (rank 0 of 1)"},
  {"comm_mpi_finalise", py_comm_mpi_finalise, METH_VARARGS, "no MPI on one GPU"},
  {"comm_hello", py_comm_hello, METH_VARARGS, "Test print statement"},
  {"comm_this_node", py_comm_this_node, METH_VARARGS, "rank of this node (0)"},
  {"comm_n_nodes", py_comm_n_nodes, METH_VARARGS, "number of nodes (1)"},

  {"_cosmology_init", py_cosmology_init, METH_VARARGS, "_cosmology_init(omega_m0)"},
  {"_cosmology_D_growth", py_cosmology_D_growth, METH_VARARGS, "_cosmology_D_growth(a)"},
  {"_cosmology_D2_growth", py_cosmology_D2_growth, METH_VARARGS, "_cosmology_D2_growth(a)"},

  {"_power_alloc", py_power_alloc, METH_VARARGS, "allocate a new _ps object"},
  {"_power_n", py_power_n, METH_VARARGS, "_power_n(_ps); number of P(k) data"},
  {"_power_i", py_power_i, METH_VARARGS, "_power_i(_ps, i); (k[i], P[i])"},
  {"_power_sigma", py_power_sigma, METH_VARARGS, "_power_sigma(_ps, R)"},
  {"_power_P", py_power_P, METH_VARARGS, "_power_P(_ps, k)"},

  {"_particles_alloc", py_particles_alloc, METH_VARARGS, "allocate a new _particles object"},
  {"_particles_slice", py_particles_slice, METH_VARARGS, "particles with x[2] < frac*boxsize"},
  {"_particles_len", py_particles_len, METH_VARARGS, "local number of particles"},
  {"_particles_np_total", py_particles_np_total, METH_VARARGS, "total number of particles"},
  {"_particles_update_np_total", py_particles_update_np_total, METH_VARARGS, "update np_total"},
  {"_particles_getitem", py_particles_getitem, METH_VARARGS, "_particles_getitem(_particles, index)"},
  {"_particles_id_asarray", py_particles_id_asarray, METH_VARARGS, "_particles_id_asarray(_particles)"},
  {"_particles_x_asarray", py_particles_x_asarray, METH_VARARGS, "_particles_x_asarray(_particles, 0|1|2)"},
  {"_particles_v_asarray", py_particles_v_asarray, METH_VARARGS, "_particles_v_asarray(_particles)"},
  {"_particles_force_asarray", py_particles_force_asarray, METH_VARARGS, "_particles_force_asarray(_particles)"},
  {"_particles_periodic_wrapup", py_particles_periodic_wrapup, METH_VARARGS, "_particles_periodic_wrapup(_particles)"},
  {"_particles_clear", py_particles_clear, METH_VARARGS, "_particles_clear(_particles)"},
  {"_particles_append", py_particles_append, METH_VARARGS, "_particles_append(_particles, x)"},
  {"_particles_set", py_particles_set, METH_VARARGS, "_particles_set(_particles, field, array)"},
  {"_particles_a", py_particles_a, METH_VARARGS, "_particles_a(_particles[, a_x, a_v, a_f])"},
  {"_particles_boxsize", py_particles_boxsize, METH_VARARGS, "_particles_boxsize(_particles)"},

  {"_lpt", py_lpt, METH_VARARGS, "_lpt(nc, boxsize, a, seed, _ps, kind)"},
  {"_lpt_from_draws", py_lpt_from_draws, METH_VARARGS, "_lpt_from_draws(nc, boxsize, a, u_phase, u_ampl, _ps, kind)"},
  {"_lpt_from_delta_k", py_lpt_from_delta_k, METH_VARARGS, "_lpt_from_delta_k(nc, boxsize, a, delta_k, kind)"},
  {"_lpt_draws", py_lpt_draws, METH_VARARGS, "_lpt_draws(nc, seed)"},
  {"_lpt_set_offset", py_lpt_set_offset, METH_VARARGS, "_lpt_set_offset(offset)"},
  {"_lpt_set_zeldovich_force", py_lpt_set_zeldovich_force, METH_VARARGS, "_lpt_set_zeldovich_force(_particles, a)"},

  {"_pm_init", py_pm_init, METH_VARARGS, "_pm_init(nc_pm, pm_factor, boxsize)"},
  {"_pm_compute_force", py_pm_compute_force, METH_VARARGS, "_pm_compute_force(_particles)"},
  {"_pm_compute_density", py_pm_compute_density, METH_VARARGS, "_pm_compute_density(_particles)"},
  {"_pm_domain_init", py_pm_domain_init, METH_VARARGS, "_pm_domain_init(_particles)"},
  {"_pm_send_positions", py_pm_send_positions, METH_VARARGS, "_pm_send_positions(_particles)"},
  {"_pm_check_total_density", py_pm_check_total_density, METH_VARARGS, "_pm_check_total_density()"},
  {"_pm_get_forces", py_pm_get_forces, METH_VARARGS, "_pm_get_forces(_particles)"},
  {"_pm_set_packet_size", py_pm_set_packet_size, METH_VARARGS, "_pm_set_packet_size(packet_size)"},
  {"_pm_force", py_pm_force, METH_VARARGS, "_pm_force(_particles)"},
  {"_pm_set_deposit_mode", py_pm_set_deposit_mode, METH_VARARGS, "_pm_set_deposit_mode('atomic'|'deterministic')"},
  {"_pm_set_bin_tile", py_pm_set_bin_tile, METH_VARARGS, "_pm_set_bin_tile(shape): -1 autotune, 0..4 fixed"},
  {"_pm_bin_tile", py_pm_bin_tile, METH_NOARGS, "(shape, tx, ty, tz) of the last deterministic deposit"},
  {"_pm_set_check", py_pm_set_check, METH_VARARGS, "_pm_set_check(on)"},
  {"_pm_free", py_pm_free, METH_VARARGS, "_pm_free(); release the PM mesh"},
  {"_pm_set_fft_engine", py_pm_set_fft_engine, METH_VARARGS, "_pm_set_fft_engine('auto'|'cufft'|'fused')"},
  {"_pm_set_fft_tile", py_pm_set_fft_tile, METH_VARARGS, "_pm_set_fft_tile(4|8)"},
  {"_pm_set_keep_delta_k", py_pm_set_keep_delta_k, METH_VARARGS, "_pm_set_keep_delta_k(on)"},
  {"_pm_fused", py_pm_fused, METH_VARARGS, "True if the fused FFT pipeline serves the PM mesh"},
  {"_pm_delta_k", py_pm_delta_k, METH_VARARGS, "_pm_delta_k()"},
  {"_pm_force_mesh", py_pm_force_mesh, METH_VARARGS, "_pm_force_mesh(axis)"},

  {"_cola_kick", py_cola_kick, METH_VARARGS, "_cola_kick(_particles, a_vel)"},
  {"_leapfrog_initial_velocity", py_leapfrog_initial_velocity, METH_VARARGS,
   "_leapfrog_initial_velocity(_particles, a)"},
  {"_leapfrog_kick", py_leapfrog_kick, METH_VARARGS,
   "_leapfrog_kick(_particles, a_vel); update particle velocities to a_vel"},
  {"_leapfrog_drift", py_leapfrog_drift, METH_VARARGS,
   "_leapfrog_drift(_particles, a_pos); update particle positions to a_pos"},
  {"_cola_drift", py_cola_drift, METH_VARARGS, "_cola_drift(_particles, a_pos)"},
  {"_cola_step", py_cola_step, METH_VARARGS, "_cola_step(_particles, a_vel, a_pos)"},
  {"_cola_velocity", py_cola_velocity, METH_VARARGS, "_cola_velocity(_particles)"},

  {"_fft_alloc", py_fft_alloc, METH_VARARGS, "_fft_alloc(nc)"},
  {"_fft_set_test_data", py_fft_set_test_data, METH_VARARGS, "_fft_set_test_data(_fft)"},
  {"_fft_fx_global_as_array", py_fft_fx_global_as_array, METH_VARARGS, "_fft_fx_global_as_array(_fft)"},

  {"config_precision", py_config_precision, METH_VARARGS, "get 'single' or 'double'"},

  {"_synchronize", py_synchronize, METH_VARARGS, "wait for the GPU and report device errors"},
  {"_set_timing", py_set_timing, METH_VARARGS, "_set_timing(on)"},
  {"_get_timing", py_get_timing, METH_VARARGS, "{stage: (ms, launches)}"},
  {"_kernel_launches", py_kernel_launches, METH_VARARGS, "kernels launched by libfs2gpu"},
  {"_set_stream", py_set_stream, METH_VARARGS, "_set_stream(cudaStream_t)"},
  {"_ctx_address", py_ctx_address, METH_VARARGS, "fs2g_ctx* of this module"},
  {"_particles_address", py_particles_address, METH_VARARGS, "fs2g_particles* of a capsule"},
  {nullptr, nullptr, 0, nullptr}
};

PyModuleDef module = {
  PyModuleDef_HEAD_INIT, "_fs", "B200 particle-mesh / COLA / 2LPT (fs2 drop-in)",
  -1, methods, nullptr, nullptr, nullptr, nullptr
};

}  // namespace

PyMODINIT_FUNC PyInit__fs(void) {
  import_array();
  return PyModule_Create(&module);
}
