// k_perm_cert.cu -- item-kernel instantiation for the certified permanent (split
// for parallel compilation; see gbs_items.cuh).
#include "gbs_items.cuh"

namespace gbsb {
#define GBSB_LIST_PERM_CERT(X) X(br1(kFnPerm, kTierCert)) X(br1(kFnPerm, kTierCertDD))
GBSB_DEFINE_GROUP(perm_cert, GBSB_LIST_PERM_CERT)
}  // namespace gbsb
