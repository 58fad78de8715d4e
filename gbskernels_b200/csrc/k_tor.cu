// k_tor.cu -- item-kernel instantiations for the "tor" branch sets (split for
// parallel compilation; see gbs_items.cuh).
#include "gbs_items.cuh"

namespace gbsb {
#define GBSB_LIST_TOR(X) X(br1(kFnTor, kTierFp64)) X(br1(kFnTor, kTierKappa)) X(br1(kFnTor, kTierDD))
GBSB_DEFINE_GROUP(tor, GBSB_LIST_TOR)
}  // namespace gbsb
