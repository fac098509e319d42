// adapter_oracle_shim.cpp -- TEST INFRASTRUCTURE ONLY.  A libqmcgpu.so
// stand-in that forwards the qmc_* entry points the adapter classes call
// (miniqmc_b200/adapter/) to the CPU oracle's oracle_* ones, so that the
// reference's drivers linked with the adapter run on a machine without a
// GPU.  tests/test_adapter_over_oracle.py builds it into a temporary
// directory and puts that directory first on LD_LIBRARY_PATH.
#include "qmcgpu.h"

extern "C" {

#define FORWARD(name, params, args) \
  int oracle_##name params;         \
  int qmc_##name params { return oracle_##name args; }

FORWARD(system_create, (const qmc_system_desc* d, int p, qmc_system** o), (d, p, o))
FORWARD(system_destroy, (qmc_system* s), (s))
FORWARD(nio_jastrows, (const double* l, qmc_functor* a, qmc_functor* b, qmc_functor* c, qmc_functor* d),
        (l, a, b, c, d))
FORWARD(nio_j3, (const double* l, qmc_j3_functor* s, qmc_j3_functor* d), (l, s, d))
FORWARD(walkers_create, (qmc_system* s, int n, int k, qmc_walkers** o), (s, n, k, o))
FORWARD(walkers_destroy, (qmc_walkers* w), (w))
FORWARD(walkers_set_positions, (qmc_walkers* w, const double* R), (w, R))
FORWARD(pset_make_move, (qmc_walkers* w, int i, const double* d), (w, i, d))
FORWARD(pset_accept_reject, (qmc_walkers* w, int i, const int* a), (w, i, a))
FORWARD(wf_evaluate_log, (qmc_walkers* w, double* l), (w, l))
FORWARD(wf_eval_grad, (qmc_walkers* w, int i, double* g), (w, i, g))
FORWARD(wf_ratio_grad, (qmc_walkers* w, int i, double* r, double* g), (w, i, r, g))
FORWARD(wf_ratio, (qmc_walkers* w, int i, double* r), (w, i, r))
FORWARD(wf_evaluate_ratios, (qmc_walkers* w, int k, int i, int n, const double* p, double* r), (w, k, i, n, p, r))
FORWARD(wf_accept_restore, (qmc_walkers* w, int i, const int* a), (w, i, a))
FORWARD(wf_complete_updates, (qmc_walkers* w), (w))
FORWARD(wf_evaluate_gl, (qmc_walkers* w, double* G, double* L, double* l), (w, G, L, l))
FORWARD(spo_evaluate_v, (qmc_system* s, int n, const double* p, double* v), (s, n, p, v))
FORWARD(spo_evaluate_vgh, (qmc_system* s, int n, const double* p, double* v, double* g, double* h),
        (s, n, p, v, g, h))

int qmc_init(int) { return QMC_OK; }

const char* qmc_status_string(int s)
{
  static const char* names[] = {"QMC_OK",          "QMC_ERR_ARG",      "QMC_ERR_CUDA",  "QMC_ERR_OOM",
                                "QMC_ERR_SINGULAR", "QMC_ERR_NONFINITE", "QMC_ERR_TIMEOUT", "QMC_ERR_STATE",
                                "QMC_ERR_NODEVICE", "QMC_ERR_ADMISSION", "QMC_ERR_CAPACITY"};
  return s >= 0 && s < 11 ? names[s] : "QMC_ERR_?";
}

const char* qmc_last_error(void) { return "the oracle reports no detail"; }

} // extern "C"
