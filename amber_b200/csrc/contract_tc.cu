// Mixed-precision (split-BF16×3) tcgen05 contraction — see below.
#include "common.cuh"

namespace amber {
int contract_mixed(amber_cuda_ctx *c, const uint16_t *, const uint16_t *, const uint16_t *, const uint16_t *,
                   const uint16_t *, const uint16_t *, long, long, double *)
{
    return fail(c, AMBER_ERR_ARG, "mixed-precision contraction not built yet");
}
}  // namespace amber
