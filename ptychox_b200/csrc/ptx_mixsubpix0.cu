// Mixed-radix sub-pixel conventional kernels, length group 0 (the coded groups of
// ptx_mix_lengths.h: every {2,3,5}-smooth side 16..1000 that is not a power of two).
#include "ptx_mix_lengths.h"
#include "ptx_mixsubpix.cuh"

namespace ptx {

const MixSubpixOps* mix_subpix_ops_group0(int n) {
#define PTX_MIXSP_CASE(N) \
  case N:                 \
    return mixsp::Ops<N>::table();
  switch (n) {
    PTX_MIXCODED_GROUP0(PTX_MIXSP_CASE)
    default:
      return nullptr;
  }
#undef PTX_MIXSP_CASE
}

const MixSubpixOps* mix_subpix_ops_group1(int n);
const MixSubpixOps* mix_subpix_ops_group2(int n);
const MixSubpixOps* mix_subpix_ops_group3(int n);
const MixSubpixOps* mix_subpix_ops_group4(int n);
const MixSubpixOps* mix_subpix_ops_group5(int n);
const MixSubpixOps* mix_subpix_ops_group6(int n);
const MixSubpixOps* mix_subpix_ops_group7(int n);

const MixSubpixOps* mix_subpix_ops(int n) {
  if (n < 16 || n > 1024 || (n & (n - 1)) == 0) return nullptr;
  const MixSubpixOps* (*const groups[])(int) = {mix_subpix_ops_group0, mix_subpix_ops_group1, mix_subpix_ops_group2,
                                                mix_subpix_ops_group3, mix_subpix_ops_group4, mix_subpix_ops_group5,
                                                mix_subpix_ops_group6, mix_subpix_ops_group7};
  for (auto* g : groups) {
    if (const MixSubpixOps* ops = g(n)) return ops;
  }
  return nullptr;
}

}  // namespace ptx
