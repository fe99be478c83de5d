// Mixed-radix coded / near-field kernels, length group 0 (ptx_mix_lengths.h).
#include "ptx_mix_lengths.h"
#include "ptx_mixcoded.cuh"

namespace ptx {

const MixCodedOps* mix_coded_ops_group0(int n) {
#define PTX_MIXCODED_CASE(N) \
  case N:                    \
    return mixcoded::Ops<N>::table();
  switch (n) {
    PTX_MIXCODED_GROUP0(PTX_MIXCODED_CASE)
    default:
      return nullptr;
  }
#undef PTX_MIXCODED_CASE
}

const MixCodedOps* mix_coded_ops_group1(int n);
const MixCodedOps* mix_coded_ops_group2(int n);
const MixCodedOps* mix_coded_ops_group3(int n);
const MixCodedOps* mix_coded_ops_group4(int n);
const MixCodedOps* mix_coded_ops_group5(int n);
const MixCodedOps* mix_coded_ops_group6(int n);
const MixCodedOps* mix_coded_ops_group7(int n);

const MixCodedOps* mix_coded_ops(int n) {
  if (n < 16 || n > 1024 || (n & (n - 1)) == 0) return nullptr;
  const MixCodedOps* (*const groups[])(int) = {mix_coded_ops_group0, mix_coded_ops_group1, mix_coded_ops_group2,
                                               mix_coded_ops_group3, mix_coded_ops_group4, mix_coded_ops_group5,
                                               mix_coded_ops_group6, mix_coded_ops_group7};
  for (auto* g : groups) {
    if (const MixCodedOps* ops = g(n)) return ops;
  }
  return nullptr;
}

}  // namespace ptx
