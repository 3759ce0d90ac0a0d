#include "snac_shim_core.h"
