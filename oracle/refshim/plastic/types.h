#include "snac_shim_plastic.h"
