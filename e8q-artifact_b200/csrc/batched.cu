// Batched search path (persistent work-queue kernel). Under construction:
// the entry point fails loudly until the kernel lands.
#include "workspace.h"

namespace e8qc {

int batched_search(const DevIndex&, Workspace&, const float*, size_t, const uint32_t*,
                   const uint32_t*, size_t, size_t, size_t, uint32_t*, float*, size_t,
                   cudaStream_t) {
    fail(E8QC_EINVAL, "batched search mode is not available in this build");
}

}  // namespace e8qc
