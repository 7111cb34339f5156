// svo_dedup.cu -- Morton-keyed unique vertices, edges and faces of the octree.
#include "svo_internal.h"

namespace svo {

int build_dedup(cudaMemPool_t, cudaStream_t, const EmitParams &, const EmitParams *, uint64_t n_out[3], uint64_t *out[3],
                int) {
    for (int k = 0; k < 3; ++k) {
        n_out[k] = 0;
        out[k] = nullptr;
    }
    return SVO_ERR_UNSUPPORTED;
}

}  // namespace svo
