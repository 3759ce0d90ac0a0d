/* Maxwell plugin: element extension (maxwell/Element.h) */
#ifndef SNAC_SHIM_MAXWELL_H
#define SNAC_SHIM_MAXWELL_H
#include "snac_shim_core.h"
typedef double Maxwell;
typedef struct _SnacMaxwell_Element {
    double viscosity[Tetrahedra_Count];
} SnacMaxwell_Element;
extern ExtensionInfo_Index SnacMaxwell_ElementHandle;
void _SnacMaxwell_Constitutive(void* context, Element_LocalIndex element_lI);
#endif
