// kh_kernel.cu -- placeholder, implemented below in a later step.
#include "runtime.h"
extern "C" int adf_kh_pressure(adf_ctx*, const adf_kh_desc*, const float*, const float*, float*) {
  return adf::fail(ADF_E_STATE, "adf_kh_pressure: not built");
}
