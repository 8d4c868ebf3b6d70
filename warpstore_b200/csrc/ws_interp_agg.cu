// Interpreter instantiations (prefix wsi) of the no-key, dense shared-row and dense global-row
// scans.  The scan kernels are split over several translation units so that they compile in parallel.
#include "ws_internal.h"
#include "ws_interp.cuh"

WS_K_NOKEYS(ws::InterpEv, wsi)
WS_K_DENSE_SHARED(ws::InterpEv, wsi)
WS_K_DENSE_GLOBAL(ws::InterpEv, wsi)
WS_K_MULTI_NOKEYS(ws::InterpEv, wsi)

namespace ws {
void interpSyms_agg(const void** s) {
  s[K_NOKEYS] = (const void*)wsi_nokeys;
  s[K_DENSE_SHARED] = (const void*)wsi_dense_shared;
  s[K_DENSE_GLOBAL] = (const void*)wsi_dense_global;
  s[K_MULTI_NOKEYS] = (const void*)wsi_multi_nokeys;
}
}  // namespace ws
