// Restarted reflected-Halpern PDHG engine (placeholder until implemented).
#include "vk_engine.cuh"

namespace vk {

std::unique_ptr<Engine> make_halpern_engine(const DeviceModel &, const vk_options &, cudaStream_t) {
    throw Unsupported("the Halpern scheme is not available in this build");
}

} // namespace vk
