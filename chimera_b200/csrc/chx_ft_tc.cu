// chx_ft_tc.cu -- split-BF16 FT contraction on the tcgen05 tensor cores.
#include "chx_common.cuh"

namespace chx {

int64_t ft_batch_tc_scratch(int rows, int nk, int nR) { return 0; }

int ft_batch_tc(const double *chi, int rows, int nk, const double *basis, int nR, double *out,
                void *scratch, int64_t scratch_bytes, cudaStream_t st) {
    set_error("ft_batch: tensor-core path not built yet");
    return CHX_ERR_UNSUPPORTED;
}

}  // namespace chx
