/* Shim for Snac/plugins/tractionBC/Force.c (the SnacTractionBC plugin): the
 * declarations its own headers would provide. */
#ifndef SNAC_SHIM_TRACTION_H
#define SNAC_SHIM_TRACTION_H
#include "snac_shim_core.h"
void _SnacTractionBC_Force_Apply(void* _context, Node_LocalIndex node_lI, double speedOfSound, Mass* mass,
                                 Mass* inertialMass, Force* force, Force* balance);
#endif
