// extern "C" entry points onto the reference's own cost-optimisation kernels,
// compiled unmodified from cpp/post/post.cu (test infrastructure only: the
// "reference as shipped" arm of the benchmark and the check of the oracle's
// restatement of those kernels).  The reference file is included at build
// time from where it lies (see oracle/Makefile); nothing of it is copied.
//
// The reference exposes its kernels through boost.python, with device
// buffers held by the classes CUDA_double_array / CUDA_float_array
// (post.cu:63-170).  Here each buffer is an opaque handle; Python loads this
// library with ctypes.PyDLL and restates the driver of test.py:341-449 on
// top of these calls.
#include CBMV_REF_POST_CU

extern "C" {
int refpost_import_numpy(void) { return stub_import_numpy_post(); }
int refpost_InitCUDA(void) { return InitCUDA() ? 1 : 0; }
int refpost_sync(void) { return (int)cudaDeviceSynchronize(); }

void* refpost_double_new(PyObject* a) { return new CUDA_double_array(a); }
void refpost_double_delete(void* h) { delete static_cast<CUDA_double_array*>(h); }
void refpost_double_zero(void* h) { static_cast<CUDA_double_array*>(h)->set_to_zero(); }
PyObject* refpost_double_get(void* h) { return static_cast<CUDA_double_array*>(h)->get_array(); }
void* refpost_float_new(PyObject* a) { return new CUDA_float_array(a); }
void refpost_float_delete(void* h) { delete static_cast<CUDA_float_array*>(h); }
void refpost_float_zero(void* h) { static_cast<CUDA_float_array*>(h)->set_to_zero(); }
PyObject* refpost_float_get(void* h) { return static_cast<CUDA_float_array*>(h)->get_array(); }

void refpost_sgm(void* l, void* r, void* in, void* out, void* tmp, float pi1, float pi2,
                 float tau_so, float alpha1, float q1, float q2, int direction) {
  sgm_w((CUDA_float_array*)l, (CUDA_float_array*)r, (CUDA_double_array*)in,
        (CUDA_double_array*)out, (CUDA_double_array*)tmp, pi1, pi2, tau_so, alpha1, q1, q2,
        direction);
}
void refpost_cross(void* in, void* out, int L1, float tau1) {
  cross_w((CUDA_float_array*)in, (CUDA_float_array*)out, L1, tau1);
}
void refpost_cbca(void* lc, void* rc, void* vol, void* out, int direction) {
  cbca_W((CUDA_float_array*)lc, (CUDA_float_array*)rc, (CUDA_double_array*)vol,
         (CUDA_double_array*)out, direction);
}
void refpost_subpixel(void* d, void* cost, void* out) {
  subpixel_enchancement_w((CUDA_float_array*)d, (CUDA_double_array*)cost, (CUDA_float_array*)out);
}
void refpost_median2d(void* in, void* out, int k) {
  median2d_w((CUDA_float_array*)in, (CUDA_float_array*)out, k);
}
void refpost_mean2d(void* in, void* out, PyObject* kernel, float alpha2) {
  mean2d_w((CUDA_float_array*)in, (CUDA_float_array*)out, kernel, alpha2);
}
void refpost_swap_axis(void* in, void* out) {
  swap_axis_w((CUDA_double_array*)in, (CUDA_double_array*)out);
}
void refpost_swap_axis_back(void* in, void* out) {
  swap_axis_back_w((CUDA_double_array*)in, (CUDA_double_array*)out);
}
void refpost_copy_double(void* in, void* out) {
  CUDA_copy_double((CUDA_double_array*)in, (CUDA_double_array*)out);
}
void refpost_copy_float(void* in, void* out) {
  CUDA_copy_float((CUDA_float_array*)in, (CUDA_float_array*)out);
}
void refpost_divide_double(void* in, double v) { CUDA_divide_double((CUDA_double_array*)in, v); }
void refpost_outlier_detection(void* d0, void* d1, void* out, int disp_max) {
  outlier_detection_w((CUDA_float_array*)d0, (CUDA_float_array*)d1, (CUDA_float_array*)out,
                      disp_max);
}
void refpost_interpolate_mismatch(void* d0, void* outlier, void* out) {
  interpolate_mismatch_w((CUDA_float_array*)d0, (CUDA_float_array*)outlier,
                         (CUDA_float_array*)out);
}
void refpost_interpolate_occlusion(void* d0, void* outlier, void* out) {
  interpolate_occlusion_w((CUDA_float_array*)d0, (CUDA_float_array*)outlier,
                          (CUDA_float_array*)out);
}
}
