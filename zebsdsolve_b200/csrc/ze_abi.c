// libzebsdsolve.so: the reference's own C ABI (zebsdsolve 0.2.8, src/exports.zig and
// src/native_api.zig; the 77 calls python/zebsdsolve/_native.py binds, and the four more the web
// module uses), over this package's engine.
//
// Every ze_* below has the reference's argument types and struct layouts (include/zebsdsolve.h).
// A call takes the interpreter lock and hands its arguments, as plain integers (addresses, sizes,
// indices) and floats, to zebsdsolve_b200.ze_abi.call(name, ...), which carries it out on the
// engine and its CUDA library; the result comes back as the call's return type. Loaded into a
// Python process (the reference's own package loads it with ctypes) it uses that interpreter; a
// native host links libpython3.12 as well, and the first call starts an interpreter.
//
// Built by zebsdsolve_b200/build.py with gcc; the Python C API is resolved at load time.
#define PY_SSIZE_T_CLEAN
#include <Python.h>
#include <dlfcn.h>
#include <pthread.h>
#include <stdarg.h>
#include <stdint.h>
#include <string.h>

#include "../../include/zebsdsolve.h"

#define ZE_EXPORT __attribute__((visibility("default")))
#define A(p) ((unsigned long long)(uintptr_t)(p))
#define Z(n) ((unsigned long long)(n))

static PyObject* g_call = NULL;
static pthread_once_t g_once = PTHREAD_ONCE_INIT;

// A native host: start an interpreter and let go of its lock (PyGILState_Ensure takes it per call).
static void start_python(void) {
  if (!Py_IsInitialized()) {
    Py_InitializeEx(0);
    PyEval_SaveThread();
  }
}

// <root>/zebsdsolve_b200/libzebsdsolve.so → <root>, put on sys.path when the package is not
// importable as it stands (a host that loads the library by its path).
static void add_package_root(void) {
  Dl_info info;
  if (!dladdr((void*)&add_package_root, &info) || !info.dli_fname) return;
  char path[4096];
  strncpy(path, info.dli_fname, sizeof(path) - 1);
  path[sizeof(path) - 1] = 0;
  for (int k = 0; k < 2; ++k) {
    char* s = strrchr(path, '/');
    if (!s) {
      strcpy(path, ".");
      break;
    }
    *s = 0;
  }
  PyObject* sp = PySys_GetObject("path");  // borrowed
  PyObject* p = PyUnicode_FromString(path[0] ? path : "/");
  if (sp && p) PyList_Append(sp, p);
  Py_XDECREF(p);
}

// zebsdsolve_b200.ze_abi.call, imported once (the lock held).
static PyObject* dispatcher(void) {
  if (g_call) return g_call;
  PyObject* m = PyImport_ImportModule("zebsdsolve_b200.ze_abi");
  if (!m) {
    PyErr_Clear();
    add_package_root();
    m = PyImport_ImportModule("zebsdsolve_b200.ze_abi");
  }
  if (!m) {
    PyErr_Print();
    return NULL;
  }
  g_call = PyObject_GetAttrString(m, "call");
  Py_DECREF(m);
  if (!g_call) PyErr_Print();
  return g_call;
}

enum { R_INT, R_FLOAT, R_NONE };

// call(name, *args) with args built from fmt ("(s...)": the name first); the result as a long
// long (R_INT; -1 when the call could not be made) or a double (R_FLOAT; 0 then).
static void vcall(int kind, long long* oi, double* od, const char* fmt, va_list ap) {
  pthread_once(&g_once, start_python);
  PyGILState_STATE st = PyGILState_Ensure();
  if (oi) *oi = -1;
  if (od) *od = 0.0;
  PyObject* fn = dispatcher();
  PyObject* args = fn ? Py_VaBuildValue(fmt, ap) : NULL;
  PyObject* r = args ? PyObject_CallObject(fn, args) : NULL;
  if (r) {
    if (kind == R_INT && r != Py_None) {
      long long v = PyLong_AsLongLong(r);
      if (v == -1 && PyErr_Occurred()) PyErr_Print(); else *oi = v;
    } else if (kind == R_FLOAT && r != Py_None) {
      double v = PyFloat_AsDouble(r);
      if (v == -1.0 && PyErr_Occurred()) PyErr_Print(); else *od = v;
    }
  } else if (PyErr_Occurred()) {
    PyErr_Print();
  }
  Py_XDECREF(r);
  Py_XDECREF(args);
  PyGILState_Release(st);
}

static long long ci(const char* fmt, ...) {
  long long v;
  va_list ap;
  va_start(ap, fmt);
  vcall(R_INT, &v, NULL, fmt, ap);
  va_end(ap);
  return v;
}

// a size or count: never negative
static size_t cz(const char* fmt, ...) {
  long long v;
  va_list ap;
  va_start(ap, fmt);
  vcall(R_INT, &v, NULL, fmt, ap);
  va_end(ap);
  return v < 0 ? 0 : (size_t)v;
}

static double cd(const char* fmt, ...) {
  double v;
  va_list ap;
  va_start(ap, fmt);
  vcall(R_FLOAT, NULL, &v, fmt, ap);
  va_end(ap);
  return v;
}

static void cv(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vcall(R_NONE, NULL, NULL, fmt, ap);
  va_end(ap);
}

// ── creation (native_api.zig:18-50) ──

ZE_EXPORT const char* ze_version(void) { return "0.2.8"; }

ZE_EXPORT void* ze_create(const char* lib_path) {
  long long h = ci("(sK)", "ze_create", A(lib_path));
  return h > 0 ? (void*)(uintptr_t)h : NULL;
}

ZE_EXPORT size_t ze_create_error(char* buf, size_t cap) { return cz("(sKK)", "ze_create_error", A(buf), Z(cap)); }
ZE_EXPORT void ze_destroy(void* e) {
  if (e) cv("(sK)", "ze_destroy", A(e));
}

// ── plumbing (exports.zig:30-66) ──

ZE_EXPORT size_t ze_adapter(void* e, char* buf, size_t cap) { return cz("(sKKK)", "ze_adapter", A(e), A(buf), Z(cap)); }
ZE_EXPORT size_t ze_error(void* e, char* buf, size_t cap) { return cz("(sKKK)", "ze_error", A(e), A(buf), Z(cap)); }
ZE_EXPORT int32_t ze_configure(void* e, const char* json, size_t len) {
  return (int32_t)ci("(sKKK)", "ze_configure", A(e), A(json), Z(len));
}
ZE_EXPORT size_t ze_settings(void* e, char* buf, size_t cap) { return cz("(sKKK)", "ze_settings", A(e), A(buf), Z(cap)); }
ZE_EXPORT size_t ze_events(void* e, char* buf, size_t cap) { return cz("(sKKK)", "ze_events", A(e), A(buf), Z(cap)); }
ZE_EXPORT void ze_cancel(void* e) { cv("(sK)", "ze_cancel", A(e)); }

// ── scan (exports.zig:70-122, 447-466, 823-836) ──

ZE_EXPORT int32_t ze_open_scan(void* e, const char* paths, size_t len) {
  return (int32_t)ci("(sKKK)", "ze_open_scan", A(e), A(paths), Z(len));
}
ZE_EXPORT int32_t ze_set_patterns(void* e, const void* data, size_t len, uint32_t pixel, uint32_t rows, uint32_t cols,
                                  uint32_t h, uint32_t w) {
  return (int32_t)ci("(sKKKIIIII)", "ze_set_patterns", A(e), A(data), Z(len), pixel, rows, cols, h, w);
}
ZE_EXPORT int32_t ze_synthesize(void* e, float* quats, int32_t* phase, int32_t* grain, size_t n) {
  return (int32_t)ci("(sKKKKK)", "ze_synthesize", A(e), A(quats), A(phase), A(grain), Z(n));
}
ZE_EXPORT void ze_close_scan(void* e) { cv("(sK)", "ze_close_scan", A(e)); }
ZE_EXPORT void ze_scan_info(void* e, ze_ScanInfo* out) { cv("(sKK)", "ze_scan_info", A(e), A(out)); }
ZE_EXPORT uint32_t ze_scan_overview_kind(void* e) { return (uint32_t)cz("(sK)", "ze_scan_overview_kind", A(e)); }
ZE_EXPORT int64_t ze_scan_overview(void* e, float* out, size_t cap) {
  return ci("(sKKK)", "ze_scan_overview", A(e), A(out), Z(cap));
}
ZE_EXPORT size_t ze_scan_format(void* e, char* buf, size_t cap) {
  return cz("(sKKK)", "ze_scan_format", A(e), A(buf), Z(cap));
}
ZE_EXPORT int32_t ze_stored_orientations(void* e, double* euler, int32_t* phase, uint64_t n) {
  return (int32_t)ci("(sKKKK)", "ze_stored_orientations", A(e), A(euler), A(phase), Z(n));
}

// ── geometry (exports.zig:124-158) ──

ZE_EXPORT void ze_get_geometry(void* e, ze_Geometry* out) { cv("(sKK)", "ze_get_geometry", A(e), A(out)); }
ZE_EXPORT void ze_set_geometry(void* e, const ze_Geometry* in) { cv("(sKK)", "ze_set_geometry", A(e), A(in)); }

// ── phases and master simulation (exports.zig:160-398) ──

ZE_EXPORT int32_t ze_add_phase(void* e, const char* path, size_t len) {
  return (int32_t)ci("(sKKK)", "ze_add_phase", A(e), A(path), Z(len));
}
ZE_EXPORT void ze_clear_phases(void* e) { cv("(sK)", "ze_clear_phases", A(e)); }
ZE_EXPORT uint32_t ze_phase_count(void* e) { return (uint32_t)cz("(sK)", "ze_phase_count", A(e)); }
ZE_EXPORT int32_t ze_phase_info(void* e, uint32_t index, ze_PhaseInfo* out) {
  return (int32_t)ci("(sKIK)", "ze_phase_info", A(e), index, A(out));
}
ZE_EXPORT int32_t ze_master_image(void* e, uint32_t phase, float* out, size_t len) {
  return (int32_t)ci("(sKIKK)", "ze_master_image", A(e), phase, A(out), Z(len));
}
ZE_EXPORT int32_t ze_sim_read_cif(void* e, const char* text, size_t len) {
  return (int32_t)ci("(sKKK)", "ze_sim_read_cif", A(e), A(text), Z(len));
}
ZE_EXPORT int32_t ze_sim_set_crystal(void* e, const char* json, size_t len) {
  return (int32_t)ci("(sKKK)", "ze_sim_set_crystal", A(e), A(json), Z(len));
}
ZE_EXPORT int32_t ze_sim_edit_crystal(void* e, const char* json, size_t len) {
  return (int32_t)ci("(sKKK)", "ze_sim_edit_crystal", A(e), A(json), Z(len));
}
ZE_EXPORT int64_t ze_sim_crystal(void* e, void* out, size_t cap) {
  return ci("(sKKK)", "ze_sim_crystal", A(e), A(out), Z(cap));
}
ZE_EXPORT int64_t ze_cell_info(void* e, uint32_t cells, void* out, size_t cap) {
  return ci("(sKIKK)", "ze_cell_info", A(e), cells, A(out), Z(cap));
}
ZE_EXPORT int32_t ze_cell_view(void* e, const float* view_rot, float zoom, uint32_t highlight, uint32_t cells,
                               uint32_t width, uint32_t height, uint32_t* out, size_t len) {
  return (int32_t)ci("(sKKdIIIIKK)", "ze_cell_view", A(e), A(view_rot), (double)zoom, highlight, cells, width, height,
                     A(out), Z(len));
}
ZE_EXPORT int64_t ze_sim_energy(void* e, void* out, size_t cap) {
  return ci("(sKKK)", "ze_sim_energy", A(e), A(out), Z(cap));
}
ZE_EXPORT int32_t ze_sim_run(void* e, ze_SimSummary* out) { return (int32_t)ci("(sKK)", "ze_sim_run", A(e), A(out)); }
ZE_EXPORT int32_t ze_sim_sheets(void* e, float* out, size_t cap) {
  return (int32_t)ci("(sKKK)", "ze_sim_sheets", A(e), A(out), Z(cap));
}
ZE_EXPORT int32_t ze_sim_add_phase(void* e, const char* name, size_t len) {
  return (int32_t)ci("(sKKK)", "ze_sim_add_phase", A(e), A(name), Z(len));
}
ZE_EXPORT int64_t ze_sim_npz(void* e, void* out, size_t cap) { return ci("(sKKK)", "ze_sim_npz", A(e), A(out), Z(cap)); }
ZE_EXPORT int32_t ze_sphere_view(void* e, int32_t source, uint32_t stored, int32_t bin, int32_t site,
                                 uint32_t projection, const float* view_rot, float zoom, uint32_t width,
                                 uint32_t height, uint32_t* out, size_t len) {
  return (int32_t)ci("(sKiIiiIKdIIKK)", "ze_sphere_view", A(e), source, stored, bin, site, projection, A(view_rot),
                     (double)zoom, width, height, A(out), Z(len));
}

// ── patterns (exports.zig:401-476) ──

ZE_EXPORT int32_t ze_pattern_shape(void* e, uint32_t full, uint32_t* out) {
  return (int32_t)ci("(sKIK)", "ze_pattern_shape", A(e), full, A(out));
}
ZE_EXPORT int32_t ze_pattern(void* e, uint64_t cell, uint32_t processed, uint32_t full, float* out, size_t len) {
  return (int32_t)ci("(sKKIIKK)", "ze_pattern", A(e), Z(cell), processed, full, A(out), Z(len));
}
ZE_EXPORT uint32_t ze_nlpar_view(void* e, float* out, float* shares, size_t cap) {
  return (uint32_t)cz("(sKKKK)", "ze_nlpar_view", A(e), A(out), A(shares), Z(cap));
}
ZE_EXPORT int64_t ze_lattice(void* e, uint32_t want, uint64_t* out, size_t cap) {
  return ci("(sKIKK)", "ze_lattice", A(e), want, A(out), Z(cap));
}
ZE_EXPORT double ze_pixel_angle(void* e) { return cd("(sK)", "ze_pixel_angle", A(e)); }
ZE_EXPORT int32_t ze_pattern_stats(void* e, const uint64_t* cells, size_t n, float* out, size_t len) {
  return (int32_t)ci("(sKKKKK)", "ze_pattern_stats", A(e), A(cells), Z(n), A(out), Z(len));
}
ZE_EXPORT int32_t ze_simulate(void* e, uint32_t phase, const uint64_t* cells, const float* quats, size_t n,
                              uint32_t full, float* out, size_t len) {
  return (int32_t)ci("(sKIKKKIKK)", "ze_simulate", A(e), phase, A(cells), A(quats), Z(n), full, A(out), Z(len));
}

// ── the pattern-centre vote and the plane fit (exports.zig:478-591) ──

ZE_EXPORT int32_t ze_fit_pc(void* e, ze_PcResult* out) { return (int32_t)ci("(sKK)", "ze_fit_pc", A(e), A(out)); }
ZE_EXPORT int32_t ze_pc_scores(void* e, uint32_t* shape, double* axes, size_t axes_cap, float* scores, size_t cap) {
  return (int32_t)ci("(sKKKKKK)", "ze_pc_scores", A(e), A(shape), A(axes), Z(axes_cap), A(scores), Z(cap));
}
ZE_EXPORT uint32_t ze_pc_level_count(void* e) { return (uint32_t)cz("(sK)", "ze_pc_level_count", A(e)); }
ZE_EXPORT int32_t ze_pc_level(void* e, uint32_t i, uint32_t* shape, uint32_t* info, double* axes, size_t axes_cap,
                              float* scores, size_t cap, uint32_t* pat_best, float* pat_ncc, size_t pat_cap) {
  return (int32_t)ci("(sKIKKKKKKKKK)", "ze_pc_level", A(e), i, A(shape), A(info), A(axes), Z(axes_cap), A(scores),
                     Z(cap), A(pat_best), A(pat_ncc), Z(pat_cap));
}
ZE_EXPORT int32_t ze_pc_level_scores(void* e, uint32_t i, float* out, size_t cap) {
  return (int32_t)ci("(sKIKK)", "ze_pc_level_scores", A(e), i, A(out), Z(cap));
}
ZE_EXPORT int32_t ze_pc_level_ballots(void* e, uint32_t i, float* out, size_t cap, double* info) {
  return (int32_t)ci("(sKIKKK)", "ze_pc_level_ballots", A(e), i, A(out), Z(cap), A(info));
}
ZE_EXPORT int32_t ze_fit_auto(void* e, ze_PlaneResult* out) { return (int32_t)ci("(sKK)", "ze_fit_auto", A(e), A(out)); }
ZE_EXPORT int32_t ze_fit_plane(void* e, ze_PlaneResult* out) {
  return (int32_t)ci("(sKK)", "ze_fit_plane", A(e), A(out));
}
ZE_EXPORT size_t ze_plane_points(void* e, ze_PlanePoint* out, size_t cap) {
  return cz("(sKKK)", "ze_plane_points", A(e), A(out), Z(cap));
}
ZE_EXPORT int32_t ze_fit_patterns(void* e, uint64_t* cells, int32_t* phases, float* quats, float* ncc, size_t cap) {
  return (int32_t)ci("(sKKKKKK)", "ze_fit_patterns", A(e), A(cells), A(phases), A(quats), A(ncc), Z(cap));
}

// ── indexing (exports.zig:594-723) ──

ZE_EXPORT int32_t ze_index_begin(void* e) { return (int32_t)ci("(sK)", "ze_index_begin", A(e)); }
ZE_EXPORT int64_t ze_index_step(void* e) { return ci("(sK)", "ze_index_step", A(e)); }
ZE_EXPORT int32_t ze_tune_begin(void* e) { return (int32_t)ci("(sK)", "ze_tune_begin", A(e)); }
ZE_EXPORT int32_t ze_tune_trial(void* e) { return (int32_t)ci("(sK)", "ze_tune_trial", A(e)); }
ZE_EXPORT int32_t ze_tune_report(void* e, double seconds) {
  return (int32_t)ci("(sKd)", "ze_tune_report", A(e), seconds);
}
ZE_EXPORT int32_t ze_chance(void* e, uint32_t phase, float* out) {
  return (int32_t)ci("(sKIK)", "ze_chance", A(e), phase, A(out));
}
ZE_EXPORT void ze_index_status(void* e, ze_IndexStatus* out) { cv("(sKK)", "ze_index_status", A(e), A(out)); }
ZE_EXPORT void ze_sweep(void* e, uint32_t i, uint32_t* out) { cv("(sKIK)", "ze_sweep", A(e), i, A(out)); }
ZE_EXPORT int32_t ze_index_cells(void* e, const uint64_t* cells, size_t n, float* out, size_t len) {
  return (int32_t)ci("(sKKKKK)", "ze_index_cells", A(e), A(cells), Z(n), A(out), Z(len));
}
ZE_EXPORT int32_t ze_index_cells_by(void* e, const uint64_t* cells, size_t n, uint32_t method, uint32_t bandwidth,
                                    uint32_t dict_grid, float* out, size_t len) {
  return (int32_t)ci("(sKKKIIIKK)", "ze_index_cells_by", A(e), A(cells), Z(n), method, bandwidth, dict_grid, A(out),
                     Z(len));
}
ZE_EXPORT int32_t ze_cell_under(void* e, uint64_t cell, const ze_Geometry* geo, uint32_t bandwidth, uint32_t full,
                                float* recs, size_t n_recs, float* sim, size_t len) {
  return (int32_t)ci("(sKKKIIKKKK)", "ze_cell_under", A(e), Z(cell), A(geo), bandwidth, full, A(recs), Z(n_recs),
                     A(sim), Z(len));
}
ZE_EXPORT int64_t ze_results(void* e, uint32_t kind, void* out, size_t len) {
  return ci("(sKIKK)", "ze_results", A(e), kind, A(out), Z(len));
}

// ── results out (exports.zig:726-881) ──

ZE_EXPORT int32_t ze_map(void* e, uint32_t kind, uint8_t* out, size_t len) {
  return (int32_t)ci("(sKIKK)", "ze_map", A(e), kind, A(out), Z(len));
}
ZE_EXPORT int32_t ze_ipf_key(void* e, uint32_t phase, uint32_t size, uint32_t lower, uint8_t* out, size_t len,
                             float* box) {
  return (int32_t)ci("(sKIIIKKK)", "ze_ipf_key", A(e), phase, size, lower, A(out), Z(len), A(box));
}
ZE_EXPORT int64_t ze_export(void* e, uint32_t kind, void* buf, size_t cap) {
  return ci("(sKIKK)", "ze_export", A(e), kind, A(buf), Z(cap));
}
ZE_EXPORT int64_t ze_export_h5oina(void* e, void* buf, size_t cap) {
  return ci("(sKKK)", "ze_export_h5oina", A(e), A(buf), Z(cap));
}
ZE_EXPORT int64_t ze_identify_frame(void* e, const double* euler, const int32_t* phase, uint64_t n, char* buf,
                                    size_t cap) {
  return ci("(sKKKKKK)", "ze_identify_frame", A(e), A(euler), A(phase), Z(n), A(buf), Z(cap));
}
ZE_EXPORT size_t ze_frame(void* e, char* buf, size_t cap) { return cz("(sKKK)", "ze_frame", A(e), A(buf), Z(cap)); }
ZE_EXPORT int32_t ze_set_frame(void* e, const char* json, size_t len) {
  return (int32_t)ci("(sKKK)", "ze_set_frame", A(e), A(json), Z(len));
}
ZE_EXPORT void ze_reduce(void* e, uint32_t phase, float* q, double* euler) {
  cv("(sKIKK)", "ze_reduce", A(e), phase, A(q), A(euler));
}
ZE_EXPORT double ze_disorientation(void* e, uint32_t phase, const float* a, const float* b) {
  return cd("(sKIKK)", "ze_disorientation", A(e), phase, A(a), A(b));
}

// ── tests and profiling (exports.zig:883-931) ──

ZE_EXPORT int32_t ze_compile_wgsl(void* e, const char* code, size_t code_len, const char* entry, size_t entry_len,
                                  char* msg, size_t cap) {
  return (int32_t)ci("(sKKKKKKK)", "ze_compile_wgsl", A(e), A(code), Z(code_len), A(entry), Z(entry_len), A(msg),
                     Z(cap));
}
ZE_EXPORT size_t ze_shader(uint32_t index, char* name, size_t name_cap, void* buf, size_t cap) {
  if (name && name_cap) name[0] = 0;
  return cz("(sIKKKK)", "ze_shader", index, A(name), Z(name_cap), A(buf), Z(cap));
}
ZE_EXPORT void ze_gpu_counts(void* e, uint32_t* out) { cv("(sKK)", "ze_gpu_counts", A(e), A(out)); }
ZE_EXPORT int32_t ze_profile(void* e, uint32_t on) { return (int32_t)ci("(sKI)", "ze_profile", A(e), on); }
ZE_EXPORT size_t ze_profile_report(void* e, char* buf, size_t cap) {
  return cz("(sKKK)", "ze_profile_report", A(e), A(buf), Z(cap));
}
