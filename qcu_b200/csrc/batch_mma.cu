// Tensor-core contraction path of the batched inner dslash (placeholder until
// the kernel lands): reports itself unavailable so the autotuner skips it.
#include "batch.h"

namespace qcu {

void launch_bdslash_mma(int, const BatchArgs &, const BDslOp &, cudaStream_t) {
  throw Error(1, "tensor-core batched dslash is not available");
}

}  // namespace qcu
