// SCF driver (device resident).
#include "hfg_ctx.h"
