/* plastic plugin: element extension (plastic/Element.h) and handles */
#ifndef SNAC_SHIM_PLASTIC_H
#define SNAC_SHIM_PLASTIC_H
#include "snac_shim_core.h"
#include "snac_shim_nr.h"
typedef struct _SnacPlastic_Element {
    Strain plasticStrain[Tetrahedra_Count];
    Strain aps;
} SnacPlastic_Element;
extern ExtensionInfo_Index SnacPlastic_ElementHandle;
void SnacPlastic_Constitutive(void* context, Element_LocalIndex element_lI);
#endif
