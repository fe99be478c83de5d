// Mixed-radix conventional kernels, length group 5 (ptx_mix_lengths.h).
#include "ptx_mix.cuh"
#include "ptx_mix_lengths.h"

namespace ptx {

const MixOps* mix_ops_group5(int n) {
#define PTX_MIX_CASE(N) \
  case N:               \
    return mixk::Ops<N>::table();
  switch (n) {
    PTX_MIX_GROUP5(PTX_MIX_CASE)
    default:
      return nullptr;
  }
#undef PTX_MIX_CASE
}

}  // namespace ptx
