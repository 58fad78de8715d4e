// k_haf.cu -- item-kernel instantiations for the "haf" branch sets (split for
// parallel compilation; see gbs_items.cuh).
#include "gbs_items.cuh"

namespace gbsb {
#define GBSB_LIST_HAF(X) X(br1(kFnHaf, kTierFp64)) X(br1(kFnHaf, kTierKappa)) X(br1(kFnLhaf, kTierFp64)) X(br1(kFnLhaf, kTierKappa)) X(kBrHafLhafFp64)
GBSB_DEFINE_GROUP(haf, GBSB_LIST_HAF)
}  // namespace gbsb
