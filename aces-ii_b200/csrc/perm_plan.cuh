// perm_plan.cuh -- the adjoint of one resort term as an inverse resort.
//
// A resort term reads out[i0,i1,i2,i3] (row-major, extents n) from
// src[i0*s0 + i1*s1 + i2*s2 + i3*s3].  When the strides of the axes longer
// than 1 are those of a dense row-major block of src in some axis order, the
// term is a bijection between out and that block, and its adjoint
//   src_bar[i . s] += alpha * out_bar[i]          (a scattered update)
// is the resort of out_bar into the block itself:
//   blk_bar[j0,j1,j2,j3] += alpha * out_bar[j . t],
// with the block's axes in decreasing source stride (m = their extents, padded
// with leading 1s) and t the row-major strides of out along those axes.  That
// runs as an accumulating gather with coalesced stores.  Plain C++: no device
// code, so the plan is checked on the host.
#pragma once

namespace acesb200 {

// true and (m, t) for a dense bijective term; false (use the scatter) else
inline bool inverse_perm_plan(const int n[4], const long long s[4], int m[4], long long t[4]) {
  long long ostr[4];
  ostr[3] = 1;
  for (int k = 2; k >= 0; --k) ostr[k] = ostr[k + 1] * n[k + 1];
  int ax[4], r = 0;
  for (int k = 0; k < 4; ++k) {
    if (n[k] < 1) return false;
    if (n[k] > 1) ax[r++] = k;
  }
  // axes longer than 1 by decreasing source stride (insertion sort, r <= 4)
  for (int i = 1; i < r; ++i)
    for (int j = i; j > 0 && s[ax[j - 1]] < s[ax[j]]; --j) {
      const int x = ax[j];
      ax[j] = ax[j - 1];
      ax[j - 1] = x;
    }
  // dense row-major block: innermost stride 1, each outer stride the product
  // of the inner extents
  long long expect = 1;
  for (int j = r - 1; j >= 0; --j) {
    if (s[ax[j]] != expect) return false;
    expect *= n[ax[j]];
  }
  for (int j = 0; j < 4; ++j) {
    m[j] = 1;
    t[j] = 0;
  }
  for (int j = 0; j < r; ++j) {
    m[4 - r + j] = n[ax[j]];
    t[4 - r + j] = ostr[ax[j]];
  }
  return true;
}

}  // namespace acesb200
