// fp_f16.cu -- the forward projector's kernels for __half volumes (fp_kernels.cuh).
#include "fp_kernels.cuh"

namespace ctr {

void launch_forward_f16(const Geometry& G, const FpArgs& a, size_t smem, cudaStream_t st)
{
    launch_forward_kinds<__half>(G, a, smem, st);
}

}  // namespace ctr
