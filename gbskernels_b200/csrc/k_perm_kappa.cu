// k_perm_kappa.cu -- item-kernel instantiations for the "perm_kappa" branch sets (split for
// parallel compilation; see gbs_items.cuh).
#include "gbs_items.cuh"

namespace gbsb {
#define GBSB_LIST_PERM_KAPPA(X) X(br1(kFnPerm, kTierKappa))
GBSB_DEFINE_GROUP(perm_kappa, GBSB_LIST_PERM_KAPPA)
}  // namespace gbsb
