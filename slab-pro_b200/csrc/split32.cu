#include "engine.hpp"
namespace slab {
std::unique_ptr<Path> make_split32(const Terrain&, const slab_params&, cudaStream_t, Ctl*, Ctl*) {
    throw Error{SLAB_E_ARG, "FP32_SPLIT path not built yet"};
}
}  // namespace slab
