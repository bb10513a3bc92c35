/* Host stand-in for <device_launch_parameters.h> (mode-B emulation).  TEST INFRASTRUCTURE ONLY. */
#include "devshim.h"
