// PSV engine (in progress).
#include "engine.cuh"
namespace dsm {
Engine* make_psv_engine(const dsm_psv_setup_t*, const dsm_options_t*) {
    throw Error(DSM_ERR_INVALID, "PSV engine not built yet");
}
}  // namespace dsm
