// Mixed-radix sub-pixel conventional kernels, length group 5 (the coded groups of
// ptx_mix_lengths.h: every {2,3,5}-smooth side 16..1000 that is not a power of two).
#include "ptx_mix_lengths.h"
#include "ptx_mixsubpix.cuh"

namespace ptx {

const MixSubpixOps* mix_subpix_ops_group5(int n) {
#define PTX_MIXSP_CASE(N) \
  case N:                 \
    return mixsp::Ops<N>::table();
  switch (n) {
    PTX_MIXCODED_GROUP5(PTX_MIXSP_CASE)
    default:
      return nullptr;
  }
#undef PTX_MIXSP_CASE
}

}  // namespace ptx
