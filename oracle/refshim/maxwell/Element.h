#include "snac_shim_maxwell.h"
