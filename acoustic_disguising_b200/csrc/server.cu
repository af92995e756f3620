// server.cu -- placeholder.
#include "runtime.h"
extern "C" {
int adf_gf_solve_batch(adf_ctx*, int64_t, adf_gf_request*, int) { return adf::fail(ADF_E_STATE, "not built"); }
int adf_server_start(adf_ctx*, size_t, int, adf_server**) { return adf::fail(ADF_E_STATE, "not built"); }
int adf_server_submit(adf_server*, const adf_gf_request*, int64_t*) { return adf::fail(ADF_E_STATE, "not built"); }
int adf_server_poll(adf_server*, int64_t, int*, double*) { return adf::fail(ADF_E_STATE, "not built"); }
int adf_server_cancel(adf_server*, int64_t) { return adf::fail(ADF_E_STATE, "not built"); }
int adf_server_drain(adf_server*) { return adf::fail(ADF_E_STATE, "not built"); }
int adf_server_stop(adf_server*) { return adf::fail(ADF_E_STATE, "not built"); }
}
