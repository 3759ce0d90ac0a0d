/*
 * snac_shim_core.h — the subset of StGermain / libSnac declarations that the
 * reference's hot-path sources need in order to compile as they stand.
 *
 * TEST INFRASTRUCTURE ONLY.  Written for this build (no reference header is
 * used: the Makefile compiles with -I- so that the quoted includes of the
 * reference sources resolve here).  Struct layouts follow the reference where
 * the sources depend on them:
 *   - Snac_Element_Tetrahedra keeps the field order of Snac/libSnac/src/Element.h:45-60
 *     (the visco-plastic hook reads one tensor past "strain", i.e. "stress");
 *   - Snac_Material follows Snac/libSnac/src/Material.h:54-112;
 * everything else is a minimal stand-in (one rank, no MPI, no XML).
 */
#ifndef SNAC_SHIM_CORE_H
#define SNAC_SHIM_CORE_H

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <assert.h>

/* ---- StGermain base types ---------------------------------------------- */
typedef unsigned int Index;
typedef unsigned int Element_LocalIndex;
typedef unsigned int Element_DomainIndex;
typedef unsigned int Element_GlobalIndex;
typedef unsigned int Element_NodeIndex;
typedef unsigned int Node_LocalIndex;
typedef unsigned int Node_DomainIndex;
typedef unsigned int Node_GlobalIndex;
typedef unsigned int Node_ElementIndex;
typedef unsigned int IndexSet_Index;
typedef unsigned int ExtensionInfo_Index;
typedef unsigned int EntryPoint_Index;
typedef unsigned int Variable_Index;
typedef Index IJK[3];
typedef double Coord[3];
typedef int Bool;
#define True 1
#define False 0
typedef const char* Type;
typedef const char* Name;
typedef size_t ArithPointer;

#define Tetrahedra_Point_Count 4
#define Tetrahedra_Surface_Count 4
#define Tetrahedra_Surface_Point_Count 3

/* streams and firewalls: the shim records the first failure instead of exiting */
typedef struct Stream { int dummy; } Stream;
extern int shim_firewall_count;
extern char shim_firewall_msg[512];
void shim_firewall(const char* fmt, ...);
#define Journal_Printf(stream, ...) ((void)0)
#define Journal_DPrintf(stream, ...) ((void)0)
#define Journal_Firewall(cond, stream, ...) \
    do { if (!(cond)) shim_firewall("firewall: " #cond); } while (0)
#ifdef NDEBUG
#define Journal_DFirewall(cond, stream, ...) ((void)0)
#else
#define Journal_DFirewall(cond, stream, ...) Journal_Firewall(cond, stream, __VA_ARGS__)
#endif
#define Journal_OFirewall(cond, stream, file, func, line, ...) \
    do { if (!(cond)) shim_firewall("firewall: " #cond); } while (0)

/* dictionaries: nothing is ever found */
typedef struct Dictionary_Entry_Value { struct Dictionary_Entry_Value* next; } Dictionary_Entry_Value;
typedef struct Dictionary { int dummy; } Dictionary;
#define Dictionary_Get(dict, key) ((Dictionary_Entry_Value*)0)
#define Dictionary_Entry_Value_GetFirstElement(v) ((Dictionary_Entry_Value*)0)
#define Dictionary_Entry_Value_AsString(v) ("")
#define Dictionary_Entry_Value_AsDictionary(v) ((Dictionary*)0)
#define Dictionary_Entry_Value_AsDouble(v) (0.0)

/* extension managers: item index from the item pointer, one array per handle;
 * name[h] is the extension's key (the plugin Type that added it, NULL while the
 * slot is unused), count the number of items (1 for the context) */
#define SHIM_MAX_EXTENSIONS 8
typedef struct ExtensionManager {
    char* base;
    size_t stride;
    char* ext[SHIM_MAX_EXTENSIONS];
    size_t extsize[SHIM_MAX_EXTENSIONS];
    const char* name[SHIM_MAX_EXTENSIONS];
    size_t count;
    unsigned owned;  /* slots allocated by ExtensionManager_Add (freed with the context) */
} ExtensionManager;
/* ExtensionManager.c:678-699 (not found: (unsigned)-1) and the
 * ExtensionManager_Add macro of ExtensionManager.h:184 */
ExtensionInfo_Index ExtensionManager_GetHandle(void* mgr, Name name);
ExtensionInfo_Index ExtensionManager_Add(void* mgr, Name name, size_t size);
#define ExtensionManager_Get(mgr, item, handle)                                                  \
    ((void*)((mgr)->ext[(handle)] +                                                              \
             (((size_t)((char*)(item) - (mgr)->base)) / (mgr)->stride) * (mgr)->extsize[(handle)]))

/* decomposition / layout: one rank, the whole mesh */
typedef struct HexaMD HexaMD;
struct HexaMD {
    Index nodeGlobal3DCounts[3];
    Index elementGlobal3DCounts[3];
    Index partition3DCounts[3];
    Bool partitionedAxis[3];
    Index elementLocal3DCounts[1][3];
    Index procsInUse;
    Element_GlobalIndex (*elementMapLocalToGlobal)(void* decomp, Element_LocalIndex lI);
};
typedef struct BlockGeometry { double min[3], max[3]; } BlockGeometry;
typedef struct ElementLayout { BlockGeometry* geometry; } ElementLayout;
typedef struct MeshLayout { HexaMD* decomp; ElementLayout* elementLayout; } MeshLayout;
#define _MeshDecomp_Node_LocalToGlobal1D(decomp, lI) (lI)
#define _MeshDecomp_Element_LocalToGlobal1D(decomp, lI) (lI)
#define RegularMeshUtils_Node_1DTo3D(decomp, gI, pi, pj, pk)                                    \
    do {                                                                                         \
        *(pi) = (gI) % (decomp)->nodeGlobal3DCounts[0];                                          \
        *(pj) = ((gI) / (decomp)->nodeGlobal3DCounts[0]) % (decomp)->nodeGlobal3DCounts[1];      \
        *(pk) = (gI) / ((decomp)->nodeGlobal3DCounts[0] * (decomp)->nodeGlobal3DCounts[1]);      \
    } while (0)
#define RegularMeshUtils_Element_1DTo3D(decomp, gI, pi, pj, pk)                                   \
    do {                                                                                          \
        *(pi) = (gI) % (decomp)->elementGlobal3DCounts[0];                                        \
        *(pj) = ((gI) / (decomp)->elementGlobal3DCounts[0]) % (decomp)->elementGlobal3DCounts[1]; \
        *(pk) = (gI) / ((decomp)->elementGlobal3DCounts[0] * (decomp)->elementGlobal3DCounts[1]); \
    } while (0)

/* variable conditions: applied through a per-node mask (last VC wins) */
typedef struct VariableCondition VariableCondition;
typedef VariableCondition CompositeVC;
struct VariableCondition {
    Index indexCount;
    Index* indexTbl;
    void (*applyToIndex)(VariableCondition* self, Index node, void* context);
    void (*apply)(VariableCondition* self, void* context);
};
#define VariableCondition_ApplyToIndex(vc, idx, ctx) ((vc)->applyToIndex((vc), (idx), (ctx)))
#define VariableCondition_Apply(vc, ctx) ((vc)->apply((vc), (ctx)))

/* entry points: named lists of named hooks (StGermain/Base/Extensibility/src/
 * EntryPoint.c), looked up by name on the context; the constitutive entry
 * point of the hot loop is called through KeyCall with the one hook the
 * driver installs */
typedef void* Func_Ptr;
typedef const char* Hook_AddedBy;
typedef unsigned long SizeT;
typedef struct Hook {
    Name name;
    Func_Ptr funcPtr;
    Hook_AddedBy addedBy;
} Hook;
#define SHIM_MAX_HOOKS 16
typedef struct Stg_ObjectList {
    unsigned count;
    Hook* data[SHIM_MAX_HOOKS];
    Hook store[SHIM_MAX_HOOKS];
} Stg_ObjectList;
typedef struct EntryPoint {
    Name name;
    Stg_ObjectList* hooks;
    Stg_ObjectList list;
} EntryPoint;
void* Stg_ObjectList_Get(void* list, Name name);
void EntryPoint_Append(void* ep, Name name, Func_Ptr funcPtr, Hook_AddedBy addedBy);
void EntryPoint_Prepend(void* ep, Name name, Func_Ptr funcPtr, Hook_AddedBy addedBy);
void EntryPoint_InsertBefore(void* ep, Name hookToInsertBefore, Name name, Func_Ptr funcPtr, Hook_AddedBy addedBy);
void EntryPoint_Replace(void* ep, Name hookToReplace, Name name, Func_Ptr funcPtr, Hook_AddedBy addedBy);
void EntryPoint_ReplaceAll(void* ep, Name name, Func_Ptr funcPtr, Hook_AddedBy addedBy);
void EntryPoint_Remove(void* ep, Name name);
#define KeyCall(ctx, key, cast) ((cast)((ctx)->shim_ep_run[(key)]))
#define KeyHandle(ctx, key) ((void*)&(ctx)->shim_ep[(key)])
#define Context_GetEntryPoint(ctx, name) shim_get_entry_point((void*)(ctx), (name))
EntryPoint* shim_get_entry_point(void* context, Name name);

/* MPI with one rank */
#define MPI_Barrier(comm) (0)
#define MPI_Allreduce(in, out, n, type, op, comm) (*(out) = *(in), 0)
#define MPI_Recv(buf, n, type, src, tag, comm, st) (0)
#define MPI_Send(buf, n, type, dst, tag, comm) (0)

/* ---- libSnac: units.h, types.h ------------------------------------------------ */
typedef double Velocity[3];
typedef double Force[3];
typedef double InertialMass;
typedef double Volume;
typedef double Area;
typedef double StrainRateTensor[3][3];
typedef double StrainRate;
typedef double StrainTensor[3][3];
typedef double Strain;
typedef double StressTensor[3][3];
typedef double Stress;
typedef double Normal[3];
typedef double Density;
typedef double Mass;
typedef double Rotation[3][3];
typedef unsigned int Material_Index;
typedef unsigned int Snac_Material_Rheology;
typedef unsigned int Tetrahedra_Index;
typedef unsigned int Tetrahedra_Surface_Index;
typedef enum { Snac_Force_Quick, Snac_Force_Normal, Snac_Force_Accurate, Snac_Force_Complete } Snac_ForceCalcType;

/* ---- Material.h ------------------------------------------------------------------- */
#define Snac_Material_Elastic 0x00000001
#define Snac_Material_Plastic 0x00000002
#define Snac_Material_Maxwell 0x00000004
#define Snac_Material_ViscoPlastic 0x00000008
typedef enum { mohrcoulomb, druckerprager } plModel;
typedef struct _Snac_Material {
    Snac_Material_Rheology rheology;
    double phsDensity;
    double alpha, beta;
    double lambda, mu;
    plModel yieldcriterion;
    unsigned int maxiterations;
    double constitutivetolerance;
    unsigned int nsegments;
    double* plstrain;
    double* frictionAngle;
    double* dilationAngle;
    double* cohesion;
    double ten_off;
    Bool putSeeds;
    double vis_min, vis_max, refvisc, refsrate, reftemp, activationE, activationV;
    double srexponent, srexponent1, srexponent2;
    double viscosity;
    double thermal_conduct, heatCapacity;
} Snac_Material;

/* ---- Node.h, Element.h ----------------------------------------------------------- */
typedef struct _Snac_Node {
    Velocity velocity;
    Force force;
    double dh, residualFr, residualFt;
    Mass inertialMass;
} Snac_Node;

typedef struct _Snac_Element_Tetrahedra_Surface {
    Area area;
    Normal normal;
} Snac_Element_Tetrahedra_Surface;

typedef struct _Snac_Element_Tetrahedra {
    Volume old_volume;
    Volume volume;
    Snac_Element_Tetrahedra_Surface surface[Tetrahedra_Surface_Count];
    StrainRateTensor strainRate;
    StrainTensor strain;
    StressTensor stress;
    Density density;
    double avgTemp;
    Material_Index material_I;
} Snac_Element_Tetrahedra;

#define Tetrahedra_Count 10
#define Node_Element_Count 8
#define Node_Element_Tetrahedra_Count 5

typedef struct _Snac_Element {
    Material_Index material_I;
    Volume volume;
    StrainRate strainRate;
    Stress stress;
    double hydroPressure;
    double rzbo;
    double bottomPressure;
    int irheology;
    Snac_Element_Tetrahedra tetra[Tetrahedra_Count];
} Snac_Element;

/* ---- Mesh and context -------------------------------------------------------------- */
typedef struct Mesh {
    MeshLayout* layout;
    Index nodeLocalCount, nodeDomainCount, elementLocalCount, elementDomainCount;
    Snac_Node* node;
    Snac_Element* element;
    Coord* nodeCoord;
    Node_DomainIndex** elementNodeTbl;
    Element_DomainIndex** nodeElementTbl;
    Node_ElementIndex* nodeElementCountTbl;
    Node_DomainIndex** nodeNeighbourTbl;
    Node_GlobalIndex* nodeL2G;
    ExtensionManager* elementExtensionMgr;
    ExtensionManager* nodeExtensionMgr;
} Mesh;

typedef void(Snac_Constitutive_CallCast)(void* entryPoint, void* context, Element_LocalIndex element_lI);

typedef struct _Snac_Context Snac_Context;
struct _Snac_Context {
    Mesh* mesh;
    MeshLayout* meshLayout;
    Dictionary* dictionary;
    const char* outputPath;
    ExtensionManager* extensionMgr;
    int rank;
    int communicator;
    unsigned int timeStep;
    unsigned int restartTimestep;
    unsigned int loop;
    Bool spherical;
    Bool computeThermalStress;
    double topo_kappa, topoGradMax, topoGradCriterion;
    Snac_Material* materialProperty;
    double dt;
    Type dtType;
    double strain_inert, speedOfSound, minLengthScale, initMinLengthScale;
    double pisos, gravity, demf;
    CompositeVC* velocityBCs;
    Stream* snacInfo;
    Stream* snacError;
    Stream* debug;
    Stream* info;
    Stream* verbose;
    Snac_ForceCalcType forceCalcType;
    EntryPoint_Index constitutiveK;
    void* shim_ep_run[2];
    EntryPoint shim_ep[2];
    EntryPoint* shim_eps;  /* the named entry points of this context */
    unsigned shim_ep_count;
};

/* AbstractContext.c:55-72 and Context.c:70-82 entry point names */
extern const Name AbstractContext_EP_Initialise;
extern const Name AbstractContext_EP_Dt;
extern const Name AbstractContext_EP_Solve;
extern const Name AbstractContext_EP_Sync;
extern const Name AbstractContext_EP_Dump;
extern const Name Snac_EP_LoopNodesEnergy;
extern const Name Snac_EP_CalcStresses;
extern const Name Snac_EP_Constitutive;
extern const Name Snac_EP_LoopNodesMomentum;
extern const Name Snac_EP_Force;
extern const Name Snac_EP_LoopElementsMomentum;
typedef Snac_Context Context;

extern const Name Snac_DtType_Constant;
extern const Name Snac_DtType_Dynamic;
extern const Name Snac_DtType_Wave;
extern const Name Snac_EP_LoopElementsEnergy;

/* ---- plugins: PluginsManager.h:101, Codelet.h:62, Stg_ComponentFactory.h:236 --------- */
typedef void Stg_Component;
typedef struct Stg_ComponentFactory Stg_ComponentFactory;
typedef Stg_Component*(Stg_ComponentFactory_ConstructByNameFunc)(void* cf, Name name, Type type, Bool essential,
                                                                 void* data);
struct Stg_ComponentFactory {
    void* context;
    Stg_ComponentFactory_ConstructByNameFunc* constructByName;
};
#define Stg_ComponentFactory_ConstructByName(cf, componentName, type, isEssential, data) \
    (type*)((Stg_ComponentFactory*)(cf))->constructByName((cf), (componentName), type##_Type, (isEssential), (data))
typedef void(Stg_Component_ConstructFunction)(void* component, Stg_ComponentFactory* cf, void* data);
typedef struct Codelet {
    Type type;
    Name name;
    Stg_Component_ConstructFunction* _construct;
} Codelet;
typedef struct PluginsManager PluginsManager;
Index PluginsManager_Submit(void* pluginsMgr, Name codeletName, Name version, void* (*defaultNew)(Name));
void* _Codelet_New(SizeT size, Type type, void* del, void* print, void* copy, void* defaultNew, void* construct,
                   void* build, void* init, void* execute, void* destroy, Name name);
#define _Codelet_Delete NULL
#define _Codelet_Print NULL
#define _Codelet_Copy NULL
#define _Codelet_Build NULL
#define _Codelet_Initialise NULL
#define _Codelet_Execute NULL
#define _Codelet_Destroy NULL
extern const Type Snac_Context_Type;

/* ---- shortcuts.h ------------------------------------------------------------------ */
#define Snac_Node_At(self, index) (&(self)->mesh->node[(index)])
#define Snac_Element_At(self, index) (&(self)->mesh->element[(index)])
#define Snac_Element_Node_P(self, element, index) \
    (&(self)->mesh->node[(self)->mesh->elementNodeTbl[(element)][(index)]])
#define Snac_NodeCoord_P(self, node_I) (&(self)->mesh->nodeCoord[node_I])
#define Snac_Element_NodeCoord(self, element, index) \
    (self)->mesh->nodeCoord[(self)->mesh->elementNodeTbl[element][index]]

/* ---- TetrahedraTables.h / Tetrahedra.h -------------------------------------------- */
extern const Element_NodeIndex TetraToNode[Tetrahedra_Count][Tetrahedra_Point_Count];
extern const unsigned int FaceToNode[Tetrahedra_Surface_Count][Tetrahedra_Surface_Point_Count];
extern const Tetrahedra_Index NodeToTetra[Node_Element_Count][Node_Element_Tetrahedra_Count];
extern const Tetrahedra_Index NodeToSurface[Node_Element_Count][Node_Element_Tetrahedra_Count];
extern const Index TriToNode[2][3];
Volume Tetrahedra_Volume(Coord coord1, Coord coord2, Coord coord3, Coord coord4);
Area Tetrahedra_SurfaceArea(Coord coord1, Coord coord2, Coord coord3);
void Tetrahedra_SurfaceNormal(Coord coord1, Coord coord2, Coord coord3, Normal* normal);

/* ---- hook prototypes ----------------------------------------------------------------- */
void Snac_UpdateElementMomentum(void* context, Element_LocalIndex element_lI, double* elementMinLengthScale);
void Snac_UpdateElementMomentum_Restart(void* context, Element_LocalIndex element_lI, double* elementMinLengthScale);
void Snac_StrainRate(void* context, Element_LocalIndex element_lI);
void Snac_Stress(void* context, Element_LocalIndex element_lI);
void Snac_Force(void* context, Node_LocalIndex node_lI, double speedOfSound, Mass* mass, Mass* inertialMass,
                Force* force, Force* balance);
void Snac_UpdateNodeMomentum(void* context, Node_LocalIndex node_lI, Mass inertialMass, Force force);
void Snac_UpdateNodeMomentum_PreProcess(void* context, Node_LocalIndex node_lI, Mass inertialMass, Force force);
void getMaxTopoGrad(void* context, Node_LocalIndex node_lI);
void Snac_UpdateNodeMomentum_DiffTopo(void* context, Node_LocalIndex node_lI, Mass inertialMass, Force force);
void Snac_UpdateNodeMomentum_UpdateInteriorTopo(void* context, Node_LocalIndex node_lI, Mass inertialMass, Force force);
void Snac_UpdateNodeMomentum_AdjustEdgeTopo(void* context, Node_LocalIndex node_lI, Mass inertialMass, Force force);

#endif
