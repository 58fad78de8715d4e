// k_perm_fp64.cu -- item-kernel instantiations for the "perm_fp64" branch sets (split for
// parallel compilation; see gbs_items.cuh).
#include "gbs_items.cuh"

namespace gbsb {
#define GBSB_LIST_PERM_FP64(X) X(br1(kFnPerm, kTierFp64))
GBSB_DEFINE_GROUP(perm_fp64, GBSB_LIST_PERM_FP64)
}  // namespace gbsb
