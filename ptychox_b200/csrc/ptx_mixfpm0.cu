// Mixed-radix Fourier ptychography kernels, length group 0 (ptx_mix_lengths.h).
#include "ptx_mix_lengths.h"
#include "ptx_mixfpm.cuh"

namespace ptx {

const MixFpmOps* mix_fpm_ops_group0(int n) {
#define PTX_MIXFPM_CASE(N) \
  case N:                  \
    return mixfpm::Ops<N>::table();
  switch (n) {
    PTX_MIXFPM_GROUP0(PTX_MIXFPM_CASE)
    default:
      return nullptr;
  }
#undef PTX_MIXFPM_CASE
}

const MixFpmOps* mix_fpm_ops_group1(int n);
const MixFpmOps* mix_fpm_ops_group2(int n);
const MixFpmOps* mix_fpm_ops_group3(int n);
const MixFpmOps* mix_fpm_ops_group4(int n);
const MixFpmOps* mix_fpm_ops_group5(int n);
const MixFpmOps* mix_fpm_ops_group6(int n);
const MixFpmOps* mix_fpm_ops_group7(int n);

const MixFpmOps* mix_fpm_ops(int n) {
  if (n < 4 || n > 1024) return nullptr;
  const MixFpmOps* (*const groups[])(int) = {mix_fpm_ops_group0, mix_fpm_ops_group1, mix_fpm_ops_group2,
                                             mix_fpm_ops_group3, mix_fpm_ops_group4, mix_fpm_ops_group5,
                                             mix_fpm_ops_group6, mix_fpm_ops_group7};
  for (auto* g : groups) {
    if (const MixFpmOps* ops = g(n)) return ops;
  }
  return nullptr;
}

}  // namespace ptx
