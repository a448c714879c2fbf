#include "index.hpp"
namespace hrnn {
void refine_knng(Index&, int, int) { fail(HRNN_ERR_STATE, "refineKNNG: not built yet"); }
void add_points(Index&, const float*, const uint64_t*, size_t) { fail(HRNN_ERR_STATE, "addPoint: not built yet"); }
void insert_dynamic(Index&, const float*, const uint64_t*, size_t, unsigned, bool) { fail(HRNN_ERR_STATE, "insertPointDynamic: not built yet"); }
void build_rknng_mutable(Index&) { fail(HRNN_ERR_STATE, "buildRKNNG_mutable: not built yet"); }
}
