// extern "C" entry points onto the reference's own matcher and feature code,
// compiled unmodified from cpp/matchers/matchers.cpp and
// cpp/featextract/featextract.cpp (test infrastructure only: the oracle's
// check of its own restatement and the timed CPU baseline).
//
// The reference functions take and return numpy arrays as PyObject*; Python
// loads this library with ctypes.PyDLL and passes py_object arguments.  Call
// cbmv_ref_init() once first: it initialises the numpy C-API tables of both
// reference translation units.
#include <Python.h>
#include <sched.h>
#include <stdlib.h>

extern "C" int stub_import_numpy_libmatchers(void);
extern "C" int stub_import_numpy_libfeatextract(void);

// cpp/matchers/matchers.cpp:24,209,353,440,515,557
PyObject* nccNister(PyObject*, PyObject*, int, int);
PyObject* census(PyObject*, PyObject*, int, int);
PyObject* sadsob(PyObject*, PyObject*, int, int);
PyObject* zsad(PyObject*, PyObject*, int, int);
PyObject* sobel(PyObject*);
int initthreads();
// cpp/featextract/featextract.cpp:24-516
PyObject* swap_axes(PyObject*);
PyObject* swap_axes_back(PyObject*);
PyObject* get_cost(PyObject*);
PyObject* get_right_cost(PyObject*);
PyObject* generate_d_indices(PyObject*, int, int);
PyObject* get_samples(PyObject*, PyObject*);
PyObject* extract_pkrn(PyObject*, PyObject*, double);
PyObject* extract_pkrn_test(PyObject*, double);
PyObject* extract_aml(PyObject*, PyObject*, double);
PyObject* extract_aml_testing(PyObject*, double);
PyObject* get_left_cost_from_right(PyObject*);
PyObject* generate_labels(PyObject*);

static int g_threads = 0;

extern "C" int cbmv_ref_threads(void) {
  if (g_threads > 0) return g_threads;
  const char* env = getenv("CBMV_REF_THREADS");
  int n = env ? atoi(env) : 0;
  if (n <= 0) {
    cpu_set_t set;
    CPU_ZERO(&set);
    n = sched_getaffinity(0, sizeof(set), &set) == 0 ? CPU_COUNT(&set) : 1;
  }
  g_threads = n > 0 ? n : 1;
  return g_threads;
}

extern "C" void cbmv_ref_set_threads(int n) { g_threads = n; }

extern "C" int cbmv_ref_init(void) {
  if (stub_import_numpy_libmatchers() < 0) return -1;
  if (stub_import_numpy_libfeatextract() < 0) return -2;
  return 0;
}

extern "C" {
PyObject* ref_nccNister(PyObject* l, PyObject* r, int d, int w) { return nccNister(l, r, d, w); }
PyObject* ref_census(PyObject* l, PyObject* r, int d, int w) { return census(l, r, d, w); }
PyObject* ref_sadsob(PyObject* l, PyObject* r, int d, int w) { return sadsob(l, r, d, w); }
PyObject* ref_zsad(PyObject* l, PyObject* r, int d, int w) { return zsad(l, r, d, w); }
PyObject* ref_sobel(PyObject* im) { return sobel(im); }
int ref_initthreads(void) { return initthreads(); }
PyObject* ref_swap_axes(PyObject* c) { return swap_axes(c); }
PyObject* ref_swap_axes_back(PyObject* c) { return swap_axes_back(c); }
PyObject* ref_get_cost(PyObject* c) { return get_cost(c); }
PyObject* ref_get_right_cost(PyObject* c) { return get_right_cost(c); }
PyObject* ref_generate_d_indices(PyObject* gt, int maxd, int thr) { return generate_d_indices(gt, maxd, thr); }
PyObject* ref_get_samples(PyObject* v, PyObject* s) { return get_samples(v, s); }
PyObject* ref_extract_ratio_samples(PyObject* v, PyObject* s, double e) { return extract_pkrn(v, s, e); }
PyObject* ref_extract_ratio(PyObject* v, double e) { return extract_pkrn_test(v, e); }
PyObject* ref_extract_likelihood_samples(PyObject* v, PyObject* s, double sg) { return extract_aml(v, s, sg); }
PyObject* ref_extract_likelihood(PyObject* v, double sg) { return extract_aml_testing(v, sg); }
PyObject* ref_get_left_cost(PyObject* c) { return get_left_cost_from_right(c); }
PyObject* ref_generate_labels(PyObject* s) { return generate_labels(s); }
}
