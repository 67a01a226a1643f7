#include "host_common.h"
namespace slim {
int bake_texture(const uint8_t *, uint32_t, uint32_t, uint32_t, uint32_t, SlimTexture *, SlimTextureMip *,
                 SlimTexelQuad *, uint32_t *, uint32_t *) {
    return set_error(SLIM_ERR_STATE, "texture baker not built yet");
}
}  // namespace slim
