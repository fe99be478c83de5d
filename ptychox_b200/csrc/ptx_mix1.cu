// Mixed-radix conventional kernels, length group 1 (ptx_mix_lengths.h).
#include "ptx_mix.cuh"
#include "ptx_mix_lengths.h"

namespace ptx {

const MixOps* mix_ops_group1(int n) {
#define PTX_MIX_CASE(N) \
  case N:               \
    return mixk::Ops<N>::table();
  switch (n) {
    PTX_MIX_GROUP1(PTX_MIX_CASE)
    default:
      return nullptr;
  }
#undef PTX_MIX_CASE
}

}  // namespace ptx
