/* visco-plastic plugin: element extension (viscoplastic/Element.h) */
#ifndef SNAC_SHIM_VISCOPLASTIC_H
#define SNAC_SHIM_VISCOPLASTIC_H
#include "snac_shim_core.h"
#include "snac_shim_nr.h"
typedef double ViscoPlastic;
typedef struct _SnacViscoPlastic_Element {
    Strain plasticStrain[Tetrahedra_Count];
    double viscosity[Tetrahedra_Count];
    Strain aps;
    StrainTensor plasticstrainTensor[Tetrahedra_Count];
    StrainTensor creepstrainTensor[Tetrahedra_Count];
} SnacViscoPlastic_Element;
extern ExtensionInfo_Index SnacViscoPlastic_ElementHandle;
void SnacViscoPlastic_Constitutive(void* context, Element_LocalIndex element_lI);
#endif
