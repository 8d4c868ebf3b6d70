// Interpreter instantiations (prefix wsi) of the hash GROUP BY scan.  The scan kernels are
// split over several translation units so that they compile in parallel.
#include "ws_internal.h"
#include "ws_interp.cuh"

WS_K_HASH(ws::InterpEv, wsi)
WS_K_MULTI_HASH(ws::InterpEv, wsi)

namespace ws {
void interpSyms_hash(const void** s) {
  s[K_HASH] = (const void*)wsi_hash;
  s[K_MULTI_HASH] = (const void*)wsi_multi_hash;
}
}  // namespace ws
