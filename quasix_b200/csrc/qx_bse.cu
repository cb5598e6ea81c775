// BSE-TDA and contour-deformation entry points (filled in below the GW chain).
#include "qx_internal.cuh"

extern "C" {
void qx_davidson_config_default(qx_davidson_config* c) {
  c->n_roots = 3;
  c->max_iter = 100;
  c->max_space = 60;
  c->tol_residual = 1e-5;
  c->lindep_threshold = 1e-12;
  c->level_shift = 0.001;
}
qx_status qx_bse_create(qx_ctx*, qx_bse**, int, int, int, const double*, const double*, const double*,
                        const double*, const double*, int, int) { return QX_ERR_NOT_IMPLEMENTED; }
qx_status qx_bse_destroy(qx_bse*) { return QX_OK; }
qx_status qx_bse_apply(qx_bse*, const double*, double*, int) { return QX_ERR_NOT_IMPLEMENTED; }
qx_status qx_bse_davidson(qx_bse*, const qx_davidson_config*, double*, double*, int*, double*, int*) {
  return QX_ERR_NOT_IMPLEMENTED;
}
qx_status qx_bse_w0(qx_ctx*, const double*, const double*, int, int, int, double*) { return QX_ERR_NOT_IMPLEMENTED; }
qx_status qx_g0w0_cd(qx_ctx*, const double*, const double*, const double*, int, int, int, const int*, int, int, double,
                     double, int, int, double*, double*, double*, double*) {
  return QX_ERR_NOT_IMPLEMENTED;
}
}
