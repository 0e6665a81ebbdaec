// Minimal stand-in for <boost/python.hpp>, test infrastructure only.
//
// The reference's native modules (cpp/matchers/matchers.cpp,
// cpp/featextract/featextract.cpp, cpp/post/post.cu) are boost.python
// extensions.  Boost is not installed here, and the oracle does not need the
// boost.python registration machinery: it calls the reference functions
// directly from extern "C" wrappers (oracle/ref_harness.cpp,
// oracle/post_ref_harness.cu).  This header supplies just enough of the
// boost.python surface for those sources to compile unmodified:
//   def(), numeric::array::set_module_and_type(), class_<>/init<>, and
//   BOOST_PYTHON_MODULE, whose body becomes a function that is never called.
// It also exposes the numpy C-API initialiser of the including translation
// unit as stub_import_numpy() so the wrapper can initialise the API table.
#pragma once
#include <Python.h>


namespace boost { namespace python {
template <class F> inline void def(const char*, F) {}
namespace numeric { struct array {
  static void set_module_and_type(const char*, const char*) {}
}; }
template <class... A> struct init {};
template <class T> struct class_ {
  template <class I> class_(const char*, I) {}
  template <class F> class_& def(const char*, F) { return *this; }
};
} }

// The module body is compiled (so it type-checks) but never executed.
#define BOOST_PYTHON_MODULE(name)                                           \
  extern "C" int stub_import_numpy_##name(void) { return _import_array(); } \
  static void* stub_unused_module_body_##name(void) __attribute__((unused)); \
  static void* stub_unused_module_body_##name(void)
