// kernels_analysis.cu -- closure flood fill and aggregate labels (device).
#include "soup_internal.h"

namespace soup {

int run_closure(Batch&, uint32_t, const uint32_t*, uint32_t, const uint32_t*, uint32_t, const double*, double, double,
                double, SoupClosureResult*, std::string& err) {
  err = "closure: not built yet";
  return SOUP_E_STATE;
}
int run_amphiphiles(Batch&, uint32_t, uint32_t*, uint32_t*, std::string& err) {
  err = "amphiphiles: not built yet";
  return SOUP_E_STATE;
}
int run_aggregates(Batch&, uint32_t, const uint32_t*, uint32_t, double, uint32_t*, uint32_t*, std::string& err) {
  err = "aggregates: not built yet";
  return SOUP_E_STATE;
}

}  // namespace soup
