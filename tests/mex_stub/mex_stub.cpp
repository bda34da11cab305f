// Implementation of the stand-in MEX API declared in mex.h (tests only).
#include "mex.h"

#include <cstdlib>
#include <cstring>
#include <string>

struct mxArray_tag {
  void *data;
  mwSize m, n;
  bool owned;
};

namespace {
std::string g_last_error;
int g_errors = 0;
}  // namespace

extern "C" {

double *mxGetPr(const mxArray *a) { return a ? static_cast<double *>(a->data) : nullptr; }

double mxGetScalar(const mxArray *a) { return (a && a->data) ? *static_cast<const double *>(a->data) : 0.0; }

mxArray *mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID cls, mxComplexity flag) {
  if (cls != mxDOUBLE_CLASS || flag != mxREAL) return nullptr;
  mxArray *a = new mxArray_tag;
  a->m = m;
  a->n = n;
  a->owned = true;
  a->data = std::calloc(m * n > 0 ? m * n : 1, sizeof(double));
  return a;
}

void mexErrMsgTxt(const char *msg) {
  g_last_error = msg ? msg : "";
  ++g_errors;
}

mxArray *mex_stub_wrap(void *data, mwSize m, mwSize n) {
  mxArray *a = new mxArray_tag;
  a->data = data;
  a->m = m;
  a->n = n;
  a->owned = false;
  return a;
}

void *mex_stub_data(const mxArray *a) { return a ? a->data : nullptr; }
mwSize mex_stub_rows(const mxArray *a) { return a ? a->m : 0; }
mwSize mex_stub_cols(const mxArray *a) { return a ? a->n : 0; }

void mex_stub_free(mxArray *a) {
  if (!a) return;
  if (a->owned) std::free(a->data);
  delete a;
}

const char *mex_stub_last_error(void) { return g_last_error.c_str(); }
int mex_stub_error_count(void) { return g_errors; }

}  // extern "C"
