// k_mixed.cu -- item-kernel instantiations for the "mixed" branch sets (split for
// parallel compilation; see gbs_items.cuh).
#include "gbs_items.cuh"

namespace gbsb {
#define GBSB_LIST_MIXED(X) X(kBrServe) X(kBrMixed)
GBSB_DEFINE_GROUP(mixed, GBSB_LIST_MIXED)
}  // namespace gbsb
