// Mixed-radix coded / near-field kernels, length group 4 (ptx_mix_lengths.h).
#include "ptx_mix_lengths.h"
#include "ptx_mixcoded.cuh"

namespace ptx {

const MixCodedOps* mix_coded_ops_group4(int n) {
#define PTX_MIXCODED_CASE(N) \
  case N:                    \
    return mixcoded::Ops<N>::table();
  switch (n) {
    PTX_MIXCODED_GROUP4(PTX_MIXCODED_CASE)
    default:
      return nullptr;
  }
#undef PTX_MIXCODED_CASE
}

}  // namespace ptx
