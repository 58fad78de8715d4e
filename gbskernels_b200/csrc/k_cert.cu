// k_cert.cu -- item-kernel instantiations for the certified hafnian, loop hafnian
// and torontonian (split for parallel compilation; see gbs_items.cuh).
#include "gbs_items.cuh"

namespace gbsb {
#define GBSB_LIST_CERT(X) X(br1(kFnHaf, kTierCert)) X(br1(kFnLhaf, kTierCert)) X(br1(kFnTor, kTierCert)) \
  X(br1(kFnTor, kTierCertDD)) X(br1(kFnHaf, kTierCertDD)) X(br1(kFnLhaf, kTierCertDD))
GBSB_DEFINE_GROUP(cert, GBSB_LIST_CERT)
}  // namespace gbsb
