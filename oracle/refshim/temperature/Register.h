#include "snac_shim_temperature.h"
