// Entry points of the pipelines that are not built yet: they fail loudly.
#include "tbg_runtime.h"

namespace tbg {
int run_learned_join(const tbg_config &, const Row *, uint64_t, const Row *, uint64_t,
                     tbg_row_out *, uint64_t, Workspace &, cudaStream_t, JoinRun *) {
    return set_error(TBG_ERR_UNKNOWN_ALGO, "LRN is not built yet");
}
}  // namespace tbg
