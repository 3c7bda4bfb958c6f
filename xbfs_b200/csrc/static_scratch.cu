// Fixed device scratch for xbfs_bfs_noalloc: one file-scope array per device,
// part of this translation unit's module image, so its storage is reserved
// when the CUDA runtime loads the module into a context, never by a call
// into this library. With the runtime's default lazy module loading that
// happens on the first cudaGetSymbolAddress below (the first
// xbfs_bfs_noalloc on that device); with CUDA_MODULE_LOADING=EAGER it
// happens when the context is created. Nothing here relies on the array's
// zero initial contents: every traversal clears the parts it reads first.
#include <cuda_runtime.h>

#include "xbfs.h"

static __device__ __align__(256) unsigned char g_noalloc_scratch[XBFS_NOALLOC_SCRATCH_BYTES];

namespace xbfs {

// Address of the scratch array on the CURRENT device; the caller makes the
// traversal's device current first and checks the returned code.
cudaError_t noalloc_scratch_address(void** ptr) {
  return cudaGetSymbolAddress(ptr, g_noalloc_scratch);
}

}  // namespace xbfs
