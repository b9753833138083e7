// Toeplitz-GEMM row filter (tensor cores). Placeholder until the tcgen05
// kernel lands: reports unsupported so the FFT filter is used.
#include "fbp_internal.h"

namespace fbp {

bool toeplitz_supported(int) { return false; }

int launch_filter_toeplitz(fbp_context* ctx, const RowSet&, int, int) {
  return set_error(ctx, FBP_ERR_UNSUPPORTED, "Toeplitz filter not available in this build");
}

}  // namespace fbp
