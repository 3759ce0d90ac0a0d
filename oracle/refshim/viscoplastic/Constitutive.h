#include "snac_shim_viscoplastic.h"
