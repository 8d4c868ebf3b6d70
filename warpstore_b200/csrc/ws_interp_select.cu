// Interpreter instantiations (prefix wsi) of the selection passes.  The scan kernels are
// split over several translation units so that they compile in parallel.
#include "ws_internal.h"
#include "ws_interp.cuh"

WS_K_SELECT_COUNT(ws::InterpEv, wsi)
WS_K_SELECT_WRITE(ws::InterpEv, wsi)

namespace ws {
void interpSyms_select(const void** s) {
  s[K_SELECT_COUNT] = (const void*)wsi_select_count;
  s[K_SELECT_WRITE] = (const void*)wsi_select_write;
}
}  // namespace ws
