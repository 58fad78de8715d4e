// Host checks of the hafnian workspace layout (gbskernels_b200/csrc/haf_pt.cuh, the
// same __host__ __device__ functions the kernels and the planner use), for the CPU
// test tests/test_haf_layout.py.  The binary64 power loop writes and reads whole
// live column tiles on the 8-tile path (columns s .. 4 ntn - 1 hold zeros), so its
// accesses stay inside the warp's workspace only if, for every subset size s of a
// launch whose largest matrix side is smax:
//   * the power's row stride holds every live tile's columns (ps(s) >= 4 ntn(s));
//   * one strip of the power fits its region (16 ps(s) <= 16 ps(smax));
//   * the staged C (rows(s) x cs(s), its padding rows zeroed over the whole stride)
//     fits its region and its stride holds the columns the tiles read (cs >= 4 ntn);
//   * d, zero-padded to whole tiles ((s + 3) & ~3 entries), fits its region.
#include <cstdio>

#include "haf_pt.cuh"

using namespace gbsb;

extern "C" int t_haf_layout_check(char* msg, int msglen) {
  int bad = 0;
  auto fail = [&](const char* what, int smax, int s, bool cert) {
    if (bad++ == 0) std::snprintf(msg, (size_t)msglen, "%s: smax=%d s=%d cert=%d", what, smax, s, (int)cert);
  };
  for (int cert = 0; cert < 2; ++cert)
    for (int smax = 2; smax <= kHafMaxN; smax += 2) {
      const HafLayout L = haf_layout(smax, cert != 0);
      const bool wide = smax > 16;
      const int c_region = (L.p_off - L.c_off) / 2;   // complex entries
      const int p_region = (L.y_off - L.p_off) / 2;
      const int d_region = (L.gi_off - L.d_off) / 2;
      if (L.total % 2 != 0) fail("workspace not a 16-byte multiple", smax, 0, cert);
      if (!(L.c_off <= L.p_off && L.p_off <= L.y_off && L.y_off <= L.d_off && L.d_off <= L.gi_off &&
            L.gi_off <= L.acc_off && L.acc_off <= L.ring_off && L.ring_off <= L.total))
        fail("offsets out of order", smax, 0, cert);
      for (int s = 2; s <= smax; s += 2) {
        const int ntn = (2 * s + 7) >> 3;
        const int ccols = 4 * ntn;
        const int cs = haf_c_stride(s);
        const int ps = haf_p_stride(s, wide);
        const int rows = 16 * haf_strips(s);
        if (ntn > (wide ? 8 : 4)) fail("more live tiles than the path has", smax, s, cert);
        if (cs < ccols) fail("C stride below the tiles' columns", smax, s, cert);
        if (rows * cs > c_region) fail("staged C outside its region", smax, s, cert);
        if (16 * ps > p_region) fail("power strip outside its region", smax, s, cert);
        if (wide && ps < ccols) fail("power stride below the live tiles' columns", smax, s, cert);
        if (!wide && ps < s) fail("power stride below s", smax, s, cert);
        if (((s + 3) & ~3) > d_region) fail("padded d outside its region", smax, s, cert);
      }
    }
  return bad;
}
