#include "snac_shim_winkler.h"
