// Interpreter instantiations (prefix wsi) of the dense private-row scans (direct and staged).  The scan kernels are
// split over several translation units so that they compile in parallel.
#include "ws_internal.h"
#include "ws_interp.cuh"

WS_K_DENSE_PRIV(ws::InterpEv, wsi)
WS_K_MULTI_DENSE_PRIV(ws::InterpEv, wsi)

namespace ws {
void interpSyms_priv(const void** s) {
  s[K_DENSE_PRIV] = (const void*)wsi_dense_priv;
  s[K_DENSE_PRIV_STAGED] = (const void*)wsi_dense_priv_staged;
  s[K_MULTI_DENSE_PRIV] = (const void*)wsi_multi_dense_priv;
}
}  // namespace ws
