// k_search.cu -- m-domain search (placeholder until the contraction kernels land)
#include "pftcc_internal.cuh"
namespace pftcc {
int search_mdomain(pftcc_handle *h, int, const float *, int, int, pftcc_best *)
{
    return set_err(h, PFTCC_ERR_UNSUPPORTED, "m-domain search not built yet");
}
}  // namespace pftcc
