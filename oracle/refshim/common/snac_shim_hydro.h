/* hydrostatic IC plugin */
#ifndef SNAC_SHIM_HYDRO_H
#define SNAC_SHIM_HYDRO_H
#include "snac_shim_core.h"
#include "mpi.h"
void _SnacHydroStaticIC_IC(void* context);
void _SnacHydroStaticIC_IC_Spherical(void* context);
#endif
