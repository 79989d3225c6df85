// fp_bf16.cu -- the forward projector's kernels for __nv_bfloat16 volumes (fp_kernels.cuh).
#include "fp_kernels.cuh"

namespace ctr {

void launch_forward_bf16(const Geometry& G, const FpArgs& a, size_t smem, cudaStream_t st)
{
    launch_forward_kinds<__nv_bfloat16>(G, a, smem, st);
}

}  // namespace ctr
