/*
 * SnacCuda — a SNAC plugin that runs the explicit Lagrangian step of a
 * Snac_Context on a B200 through libsnac_b200 (include/snac_gpu.h).
 *
 * Loaded like any other SNAC plugin (after the physics plugins in the
 * <import> list; found by StGermain's PluginLoader as SnacCudamodule.so,
 * StGermain/Base/Extensibility/src/PluginLoader.c:359-370), its
 * _SnacCuda_Construct replaces, with EntryPoint_Replace
 * (StGermain/Base/Extensibility/src/EntryPoint.c:735):
 *   AbstractContext_EP_Initialise  "SnacTimeStepZero"  -> SnacCuda_TimeStepZero
 *       (Snac/libSnac/src/Context.c:978-1036: the device model is built from
 *        the context as the plugin ICs left it, then step zero runs there)
 *   Snac_EP_LoopElementsEnergy / Snac_EP_LoopNodesEnergy (temperature runs)
 *   Snac_EP_CalcStresses           "default"  (Context.c:1102-1117)
 *   Snac_EP_LoopNodesMomentum      "default"  (Context.c:1120-1154)
 *   Snac_EP_LoopElementsMomentum   "default"  (Context.c:1156-1184)
 *   AbstractContext_EP_Sync        "SnacSync" (Context.c:1208-1268)
 * and prepends SnacCuda_BeginStep to AbstractContext_EP_Solve (the device's
 * step counter and dt, AbstractContext.c:874-890) and SnacCuda_SyncHost to
 * AbstractContext_EP_Dump, so the reference's own writers, and any host
 * plugin that runs on a dump step, read an up-to-date context.
 *
 * The context stays canonical on the host between syncs: SnacCuda_SyncHost
 * copies the device state into mesh->node / mesh->element and the plugins'
 * extensions (unpack), SnacCuda_SyncDevice copies it back (pack) after a
 * host plugin (the remesher) changed it.  One rank only (the device model
 * is the whole mesh); a decomposed context is refused at step zero.
 */
#ifndef __Snac_Cuda_h__
#define __Snac_Cuda_h__

#include "snac_gpu.h"

extern const Type SnacCuda_Type;
extern ExtensionInfo_Index SnacCuda_ContextHandle;

/* The plugin's context extension. */
typedef struct SnacCuda_Context {
    snac_gpu* gpu;
    int constitutive;               /* SNAC_RHEOLOGY_* of the one constitutive hook */
    int temperature;                /* SnacTemperature loaded */
    int druckerPrager;              /* visco-plastic with a Drucker-Prager phase: the tensor is kept */
    ExtensionInfo_Index plasticElement, viscoPlasticElement, maxwellElement, temperatureNode, temperatureContext;
    long long ne, nn;
    /* the ABI's element-major host arrays (snac_state_view) */
    double* coord;
    double* velocity;
    double* stress;
    double* plasticStrain;
    double* viscosity;
    double* temperature_;
    double* force;
    double* inertialMass;
    double* plasticStrainTensor;    /* visco-plastic: plasticstrainTensor (Drucker-Prager phases) */
} SnacCuda_Context;

/* Arrays a descriptor points into while snac_gpu_create reads it. */
typedef struct SnacCuda_DescStore {
    snac_material* materials;
    int* elementMaterial;
    double* initStress;
    double* initVelocity;
    double* initTemperature;
    unsigned char* velocityBCMask;
    double* velocityBCValue;
    unsigned char* temperatureBCMask;
    double* temperatureBCValue;
    int* dpMaxIterations;
    double* dpTolerance;
    double* cohesionScale;   /* per element, when the phases were grouped into scaled bases */
    double* frictionScale;
    double* viscScale;
} SnacCuda_DescStore;

Index _SnacCuda_Register(PluginsManager* pluginsMgr);
void* _SnacCuda_DefaultNew(Name name);
void _SnacCuda_Construct(void* component, Stg_ComponentFactory* cf, void* data);

/* The constitutive plugin and extensions the context carries (hook names on
 * Snac_EP_Constitutive, extension keys); 0 or a negative SNAC_GPU_E* code. */
int SnacCuda_Inspect(Snac_Context* context, SnacCuda_Context* self);
/* Descriptor of the device model from the context after its ICs: mesh, phase
 * table, per-element phases, the state as initial values, and the velocity /
 * temperature conditions resolved per node by applying the context's own
 * CompositeVCs (so last-VC-wins holds by construction). */
int SnacCuda_FillDesc(Snac_Context* context, SnacCuda_Context* self, snac_gpu_desc* desc, SnacCuda_DescStore* store);
void SnacCuda_FreeDescStore(SnacCuda_DescStore* store);
/* context -> ABI arrays (coordinates, velocities, tet stresses, plastic
 * strain, viscosity, temperature) */
void SnacCuda_Pack(Snac_Context* context, SnacCuda_Context* self);
/* ABI arrays -> context (the same fields, plus the nodal force and inertial mass) */
void SnacCuda_Unpack(Snac_Context* context, SnacCuda_Context* self);

/* hooks */
void SnacCuda_TimeStepZero(void* context, void* data);
void SnacCuda_BeginStep(void* context);
void SnacCuda_LoopElementsEnergy(void* context);
void SnacCuda_LoopNodesEnergy(void* context);
void SnacCuda_CalcStresses(void* context);
void SnacCuda_LoopNodesMomentum(void* context);
void SnacCuda_LoopElementsMomentum(void* context);
void SnacCuda_Sync(void* context);
void SnacCuda_SyncHost(void* context);
void SnacCuda_SyncDevice(void* context);

#endif /* __Snac_Cuda_h__ */
