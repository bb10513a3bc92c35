/* Host stand-in for <cuda_runtime.h> when the reference's GPU sampler sources are compiled
 * as host C++ by oracle/ref/build_ref.py (mode-B emulation).  TEST INFRASTRUCTURE ONLY.
 * Everything the compiled device code needs comes from devshim.h, included first. */
#include "devshim.h"
