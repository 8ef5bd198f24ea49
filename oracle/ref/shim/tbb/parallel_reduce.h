/* TBB header stand-in (see tbb_shim_core.h). TEST INFRASTRUCTURE ONLY. */
#include "tbb_shim_core.h"
