// Contour surgery and node redistribution (contours.f90:350-933).
#include "state.cuh"

namespace casl {
int surgery_dev(casl_handle *h) { (void)h; return CASL_EUNSUPPORTED; }
int renode_host(casl_handle *h, const double *, const double *, int, double *, double *, int,
                int *) {
  (void)h;
  return CASL_EUNSUPPORTED;
}
}  // namespace casl
