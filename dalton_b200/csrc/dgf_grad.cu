// Gradient and one-electron entry points (filled in below the Fock build).
#include "dgf_internal.h"

extern "C" int dgf_grad2e(dgf_ctx *, const double *, double, double, double *) { return DGF_ERR_UNSUPPORTED; }
extern "C" int dgf_grad2e_device(dgf_ctx *, const double *, double, double, double *, void *) {
  return DGF_ERR_UNSUPPORTED;
}
extern "C" int dgf_oneint(dgf_ctx *, double *, double *, double *) { return DGF_ERR_UNSUPPORTED; }
extern "C" int dgf_grad1e(dgf_ctx *, const double *, const double *, double *) { return DGF_ERR_UNSUPPORTED; }
