#include "index.hpp"
namespace hrnn {


void insert_dynamic(Index&, const float*, const uint64_t*, size_t, unsigned, bool) { fail(HRNN_ERR_STATE, "insertPointDynamic: not built yet"); }
void build_rknng_mutable(Index&) { fail(HRNN_ERR_STATE, "buildRKNNG_mutable: not built yet"); }
}
