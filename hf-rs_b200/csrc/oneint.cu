// One-electron integrals on the device.
#include "hfg_ctx.h"
