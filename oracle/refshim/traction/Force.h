#include "snac_shim_traction.h"
