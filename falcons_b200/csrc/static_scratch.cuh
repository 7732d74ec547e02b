// Static device scratch of the allocation-free decompress entry point.
#pragma once

namespace fb2 {

// Address of the FALCONS_NOALLOC_SCRATCH_BYTES static scratch region on the current device.  The
// first call on a device does the set-up (module and kernel loads); later calls only read a cached
// pointer.  Every caller on a device shares the one region.
void *static_scratch_current_device();

}  // namespace fb2
