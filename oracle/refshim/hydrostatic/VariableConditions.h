#include "snac_shim_hydro.h"
