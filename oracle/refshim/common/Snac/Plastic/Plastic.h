#include "snac_shim_core.h"
#include "snac_shim_plastic.h"
