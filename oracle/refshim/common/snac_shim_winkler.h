/* Shim for Snac/plugins/winkler/Force.c (the SnacWinklerForce plugin): the
 * declarations its own headers would provide. */
#ifndef SNAC_SHIM_WINKLER_H
#define SNAC_SHIM_WINKLER_H
#include "snac_shim_core.h"
void _SnacWinklerForce_Apply(void* _context, Node_LocalIndex node_lI, double speedOfSound, Mass* mass,
                             Mass* inertialMass, Force* force, Force* balance);
void _SnacWinklerForce_Apply_Spherical(void* _context, Node_LocalIndex node_lI, double speedOfSound, Mass* mass,
                                       Mass* inertialMass, Force* force, Force* balance);
/* Register.c's globals (the spherical variant only) */
extern double Spherical_RMin, Spherical_RMax;
#endif
