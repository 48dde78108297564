// Dynamic-plan kernel instantiations (lengths without a static plan).
#include "dfft_internal.h"

namespace dfft {

const void* dynamic_kernel(int dbl) {
  if (dbl) return reinterpret_cast<const void*>(&axis_pass_dynamic<double, 16>);
  return reinterpret_cast<const void*>(&axis_pass_dynamic<float, 16>);
}

}  // namespace dfft
