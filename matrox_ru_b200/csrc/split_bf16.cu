// Split-BF16 evaluation path (tcgen05 tensor cores).  Placeholder until the kernels land:
// plans created with MXB_PREC_SPLIT_BF16 report MXB_ERR_UNSUPPORTED.
#include "plan.h"

namespace mxb {

int row_tile_for(int precision) { return precision == MXB_PREC_SPLIT_BF16 ? 128 : 64; }

int Plan::setup_split_bf16(const mxb_cds_desc &)
{
    set_error("split-BF16 path not built yet");
    return MXB_ERR_UNSUPPORTED;
}

int Plan::run_split_bf16(const std::vector<Launch> &, const double *, double *, int, int, cudaStream_t)
{
    set_error("split-BF16 path not built yet");
    return MXB_ERR_UNSUPPORTED;
}

void Plan::free_split_bf16() {}

}  // namespace mxb
