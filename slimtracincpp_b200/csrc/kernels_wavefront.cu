// Wavefront form of the trace path (stage kernels over compacted queues).
#include "kernels.h"
#include "tracer_core.cuh"

namespace slim {

cudaError_t launch_render_wavefront(const DevScene &S, const DevFrame &F, const WavefrontBuffers &B, int block,
                                    cudaStream_t stream) {
    return launch_render_fused(S, F, block, stream);
}

}  // namespace slim
