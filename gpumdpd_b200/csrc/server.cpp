// server.cpp -- continuous-batching job server (filled in below the plain engine).
#include "../../include/dpd_b200.h"
extern "C" {
int dpd_server_create(double, int, const dpd_tuning*, dpd_server** out) { if (out) *out = nullptr; return DPD_E_STATE; }
int dpd_server_submit(dpd_server*, const char*, const dpd_system*, int64_t*) { return DPD_E_STATE; }
int dpd_server_step(dpd_server*, int*, int*) { return DPD_E_STATE; }
int dpd_server_result(dpd_server*, int64_t, dpd_job_result*) { return DPD_E_STATE; }
int dpd_server_job_state(dpd_server*, int64_t, double*, double*) { return DPD_E_STATE; }
int dpd_server_job_rdf(dpd_server*, int64_t, double*, int64_t*) { return DPD_E_STATE; }
int dpd_server_stats(dpd_server*, int64_t*, double*, int64_t*) { return DPD_E_STATE; }
const char* dpd_server_last_error(dpd_server*) { return "server not built"; }
int dpd_server_destroy(dpd_server*) { return DPD_OK; }
}
