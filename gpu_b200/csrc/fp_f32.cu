// fp_f32.cu -- the forward projector's kernels for float volumes (fp_kernels.cuh).
#include "fp_kernels.cuh"

namespace ctr {

void launch_forward_f32(const Geometry& G, const FpArgs& a, size_t smem, cudaStream_t st)
{
    launch_forward_kinds<float>(G, a, smem, st);
}

}  // namespace ctr
