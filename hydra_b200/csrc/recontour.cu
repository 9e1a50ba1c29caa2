// Recontouring (congen.f90:24-441).
#include "state.cuh"

namespace casl {
int recontour_dev(casl_handle *h, const double *) { (void)h; return CASL_EUNSUPPORTED; }
}  // namespace casl
