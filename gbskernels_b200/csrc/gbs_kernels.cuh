// gbs_kernels.cuh -- work-item descriptors and the launch interface shared by the
// kernels (gbs_kernels.cu) and the host runtime (host_api.cu).
//
// Every evaluation is cut into WORK ITEMS: (instance, first subset, subset count).
// A warp evaluates one item at a time and writes one partial; the warp that
// completes the LAST item of an instance sums that instance's partials in item
// order and writes the result.  The decomposition of an instance into items is a
// pure function of (function, tier, size), so a value is bit-identical whether the
// instance runs alone, in a per-size launch or inside a mixed persistent batch.
#pragma once

#include <cstdint>

namespace gbsb {

// function codes (the reference's Session numbering, core/host_api.cu:472-480)
enum : int { kFnPerm = 0, kFnHaf = 1, kFnLhaf = 2, kFnTor = 3 };
// tier codes (kTierCertDD: double-double value + rigorous bound)
enum : int { kTierFp64 = 0, kTierDD = 1, kTierKappa = 2, kTierCert = 3, kTierCertDD = 4 };

__host__ __device__ constexpr int ft_code(int fn, int tier) { return fn * 8 + tier; }
__host__ __device__ constexpr int ft_fn(int ft) { return ft >> 3; }
__host__ __device__ constexpr int ft_tier(int ft) { return ft & 7; }
__host__ __device__ constexpr bool tier_certified(int tier) { return tier == kTierCert || tier == kTierCertDD; }

struct InstDesc {       // 32 bytes
  long long off;        // offset (in doubles) of the matrix in the packed input buffer
  int dim;              // matrix side as evaluated (lhaf odd N already augmented; tor 2n)
  int ft;               // ft_code(func, tier)
  int item0;            // first work item
  int nitems;           // number of work items
  int param;            // tor: prefix depth g; perm: log2 of the Gray range per lane
  int real_in;          // tor: 1 if the matrix is real (imaginary parts all zero)
};

struct WorkItem {       // 24 bytes
  int inst;
  int pad;
  unsigned long long lo;     // first subset mask / Gray index / prefix pattern
  unsigned long long count;  // number of subsets / Gray indices / prefix patterns
};

// log2 of the subsets per hafnian / loop-hafnian work item in the binary64 tiers
// (the planner and the allocation-free entry share it, so values agree bit for bit)
constexpr int kHafItemLog2 = 7;

// Branch sets compiled into an item kernel (bit ft_code).  A launch uses the
// smallest compiled set covering the (function, tier) pairs of its batch.
constexpr unsigned br1(int fn, int tier) { return 1u << ft_code(fn, tier); }
constexpr unsigned kBrHafLhafFp64 = br1(kFnHaf, kTierFp64) | br1(kFnLhaf, kTierFp64);
// haf / lhaf / tor in fp64, fp64 + indicator and certified: the serving mix
constexpr unsigned kBrServe = kBrHafLhafFp64 | br1(kFnTor, kTierFp64) | br1(kFnHaf, kTierKappa) |
                              br1(kFnLhaf, kTierKappa) | br1(kFnTor, kTierKappa) | br1(kFnHaf, kTierCert) |
                              br1(kFnLhaf, kTierCert) | br1(kFnTor, kTierCert);
// haf / lhaf / tor in every tier
constexpr unsigned kBrMixed = kBrServe | br1(kFnHaf, kTierDD) | br1(kFnLhaf, kTierDD) | br1(kFnTor, kTierDD) |
                              br1(kFnHaf, kTierCertDD) | br1(kFnLhaf, kTierCertDD) | br1(kFnTor, kTierCertDD);

// Device buffers of one launch.
struct ItemLaunch {
  const double* mats;      // packed matrices (complex interleaved; real-tor as complex too)
  const InstDesc* insts;
  const WorkItem* items;
  const int* order;        // optional queue order (item indices, heaviest first); null = identity
  int n_items;
  const int* n_items_dev = nullptr;  // optional: the item count, read on the device (a queue planned there)
  int* head;               // queue head (atomic), zeroed before launch
  int* done;               // per-instance completed-item counters, zeroed before launch
  double* part;            // 4 doubles per item (re_hi, re_lo, im_hi, im_lo)
  double* paux;            // 1 double per item (sum |term|)
  int* pst;                // 1 int per item (status)
  double* out;             // 2 doubles per instance (complex value)
  double* aux_out;         // 1 double per instance
  int* st_out;             // 1 int per instance
  int ws_doubles;          // per-warp shared workspace (doubles)
  int haf_smax;            // max matrix side among haf/lhaf instances (layout)
};

}  // namespace gbsb
