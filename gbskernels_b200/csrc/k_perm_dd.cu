// k_perm_dd.cu -- item-kernel instantiations for the "perm_dd" branch sets (split for
// parallel compilation; see gbs_items.cuh).
#include "gbs_items.cuh"

namespace gbsb {
#define GBSB_LIST_PERM_DD(X) X(br1(kFnPerm, kTierDD))
GBSB_DEFINE_GROUP(perm_dd, GBSB_LIST_PERM_DD)
}  // namespace gbsb
