// Mixed-radix Fourier ptychography kernels, length group 2 (ptx_mix_lengths.h).
#include "ptx_mix_lengths.h"
#include "ptx_mixfpm.cuh"

namespace ptx {

const MixFpmOps* mix_fpm_ops_group2(int n) {
#define PTX_MIXFPM_CASE(N) \
  case N:                  \
    return mixfpm::Ops<N>::table();
  switch (n) {
    PTX_MIXFPM_GROUP2(PTX_MIXFPM_CASE)
    default:
      return nullptr;
  }
#undef PTX_MIXFPM_CASE
}

}  // namespace ptx
