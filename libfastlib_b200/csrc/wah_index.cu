// Range evaluation of relic / bin indexes (filled in by the index kernels).
#include "../../include/wahgpu.h"
