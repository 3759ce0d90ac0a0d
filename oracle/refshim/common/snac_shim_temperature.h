/* temperature plugin: node/element/context extensions (temperature/Node.h,
 * Element.h, Context.h) and hooks */
#ifndef SNAC_SHIM_TEMPERATURE_H
#define SNAC_SHIM_TEMPERATURE_H
#include "snac_shim_core.h"
typedef double HeatFlux[3];
typedef struct _SnacTemperature_Node {
    double temperature;
    double temperature0;
} SnacTemperature_Node;
typedef struct _SnacTemperature_Element {
    HeatFlux heatFlux[Tetrahedra_Count];
    Stress thermalStress[Tetrahedra_Count];
} SnacTemperature_Element;
typedef struct _SnacTemperature_Context {
    double topTemp;
    double bottomTemp;
    CompositeVC* temperatureBCs;
    FILE* temperatureOut;
    FILE* temperatureCheckpoint;
} SnacTemperature_Context;
extern ExtensionInfo_Index SnacTemperature_NodeHandle;
extern ExtensionInfo_Index SnacTemperature_ElementHandle;
extern ExtensionInfo_Index SnacTemperature_ContextHandle;
void SnacTemperature_LoopElements(void* context);
void SnacTemperature_LoopNodes(void* context);
void Snac_HeatFlux(void* context, Element_LocalIndex element_lI);
void Snac_Heat(void* context, Node_LocalIndex node_lI, double sourceterm);
void UpdateAverageTemp_LoopElements(void* context);
void SnacTemperature_BoundaryConditions(void* context);
void SnacTemperature_HeatFluxBC(void* context);
void _SnacTemperature_Top2BottomSweep(Node_LocalIndex node_lI, Variable_Index var_I, void* context, void* result);
void _SnacTemperature_InitialConditions(void* context);
#define Snac_Node_At_T(self, index) Snac_Node_At(self, index)
#endif
