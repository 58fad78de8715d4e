// k_haf_dd.cu -- item-kernel instantiations for the "haf_dd" branch sets (split for
// parallel compilation; see gbs_items.cuh).
#include "gbs_items.cuh"

namespace gbsb {
#define GBSB_LIST_HAF_DD(X) X(br1(kFnHaf, kTierDD)) X(br1(kFnLhaf, kTierDD))
GBSB_DEFINE_GROUP(haf_dd, GBSB_LIST_HAF_DD)
}  // namespace gbsb
