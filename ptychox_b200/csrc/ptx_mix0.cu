// Mixed-radix conventional kernels, length group 0 (ptx_mix_lengths.h).
#include "ptx_mix.cuh"
#include "ptx_mix_lengths.h"

namespace ptx {

const MixOps* mix_ops_group0(int n) {
#define PTX_MIX_CASE(N) \
  case N:               \
    return mixk::Ops<N>::table();
  switch (n) {
    PTX_MIX_GROUP0(PTX_MIX_CASE)
    default:
      return nullptr;
  }
#undef PTX_MIX_CASE
}

const MixOps* mix_ops_group1(int n);
const MixOps* mix_ops_group2(int n);
const MixOps* mix_ops_group3(int n);
const MixOps* mix_ops_group4(int n);
const MixOps* mix_ops_group5(int n);
const MixOps* mix_ops_group6(int n);
const MixOps* mix_ops_group7(int n);

const MixOps* mix_ops(int n) {
  if (n < 6 || n > 1024 || (n & (n - 1)) == 0) return nullptr;
  const MixOps* (*const groups[])(int) = {mix_ops_group0, mix_ops_group1, mix_ops_group2, mix_ops_group3,
                                          mix_ops_group4, mix_ops_group5, mix_ops_group6, mix_ops_group7};
  for (auto* g : groups) {
    if (const MixOps* ops = g(n)) return ops;
  }
  return nullptr;
}

}  // namespace ptx
