/* mphysics.h -- the reference engine's exported-function API (MPhysicsAPI),
 * served by libhfgrid.so for the grid half of the step.
 *
 * Same names and argument meaning as MPhysics/MPhysics.h:14-104 of
 * junwei-jiang/Hybrid-Fluid-Simulation (FP32 `Real` build), exported with C
 * linkage and default visibility instead of __declspec(dllexport).  A caller
 * of the reference DLL links these symbols unchanged:
 *
 *   initMPhysics / freeMPhysics / update / loadScene  (MPhysics.cpp:6-29)
 *   getEulerParticleSize, copyEulerParticlesPos/VelToCPU,
 *   getEulerGridInfo                                 (MPhysics.cpp:183-205,262-266,349-365)
 *   copyFluidSDFToCPU / copyFluidSDFGradientToCPU    (MPhysics.cpp:207-247)
 *
 * The projective-particle half of the reference (copyPositionToCPU,
 * copyVelToCPU, getParticleSize, neighbour and cell data, rigid-boundary
 * instances) is outside this library: those entry points exist so the symbol
 * set matches, report zero sizes and record "not supported".
 *
 * In C++ the functions are declared in namespace MPhysicsAPI, as in the
 * reference, so `MPhysicsAPI::update(dt)` compiles unchanged; their C
 * linkage makes the symbol names the plain function names.
 *
 * The reference returns nothing and prints on failure; these functions keep
 * the void signatures and record the failure for mphysics_last_error().
 * Calls are serialised by an internal mutex (the reference is single
 * threaded).  Scenes are stepped in name order, like the reference's
 * std::map iteration (MPhysics.cpp:19-25).
 */
#ifndef MPHYSICS_H
#define MPHYSICS_H

#ifdef __cplusplus
namespace MPhysicsAPI {
extern "C" {
#define MPHYSICS_REF(T) T&
/* C++ callers keep the reference's default arguments (MPhysics.h:49-67). */
#define MPHYSICS_DEFAULT(v) = v
#else
#define MPHYSICS_REF(T) T*
#define MPHYSICS_DEFAULT(v)
#endif

#define MPHYSICS_API __attribute__((visibility("default")))

MPHYSICS_API void initMPhysics(void);
MPHYSICS_API void freeMPhysics(void);
MPHYSICS_API void update(float vDeltaTime);
/* vSceneFile: a path to a JSON scene, or the JSON text itself (SceneManager.cpp:9-17). */
MPHYSICS_API void loadScene(const char* vSceneFile);

MPHYSICS_API void copyPositionToCPU(const char* vSimulatorName, float* voPosition);
MPHYSICS_API void copyVelToCPU(const char* vSimulatorName, float* voVel);
MPHYSICS_API void copyEulerParticlesPosToCPU(const char* vSimulatorName, float* voPosition);
MPHYSICS_API void copyEulerParticlesVelToCPU(const char* vSimulatorName, float* voVel);
MPHYSICS_API void copyFluidSDFToCPU(const char* vSimulatorName, float* voSDF);
MPHYSICS_API void copyFluidSDFGradientToCPU(const char* vSimulatorName, float* voSDFGradientX,
                                            float* voSDFGradientY, float* voSDFGradientZ);

MPHYSICS_API unsigned int instanceRigidBoundary(
    const char* vSimulatorName, unsigned int vBoundaryIndex, float vPosX MPHYSICS_DEFAULT(0.0f),
    float vPosY MPHYSICS_DEFAULT(0.0f), float vPosZ MPHYSICS_DEFAULT(0.0f), float R00 MPHYSICS_DEFAULT(1.0f),
    float R01 MPHYSICS_DEFAULT(0.0f), float R02 MPHYSICS_DEFAULT(0.0f), float R10 MPHYSICS_DEFAULT(0.0f),
    float R11 MPHYSICS_DEFAULT(1.0f), float R12 MPHYSICS_DEFAULT(0.0f), float R20 MPHYSICS_DEFAULT(0.0f),
    float R21 MPHYSICS_DEFAULT(0.0f), float R22 MPHYSICS_DEFAULT(1.0f));
MPHYSICS_API void transformRigidBoundary(
    const char* vSimulatorName, unsigned int vBoundaryIndex, unsigned int vBoundaryInstanceIndex,
    float vPosX MPHYSICS_DEFAULT(0.0f), float vPosY MPHYSICS_DEFAULT(0.0f), float vPosZ MPHYSICS_DEFAULT(0.0f),
    float R00 MPHYSICS_DEFAULT(1.0f), float R01 MPHYSICS_DEFAULT(0.0f), float R02 MPHYSICS_DEFAULT(0.0f),
    float R10 MPHYSICS_DEFAULT(0.0f), float R11 MPHYSICS_DEFAULT(1.0f), float R12 MPHYSICS_DEFAULT(0.0f),
    float R20 MPHYSICS_DEFAULT(0.0f), float R21 MPHYSICS_DEFAULT(0.0f), float R22 MPHYSICS_DEFAULT(1.0f));
MPHYSICS_API unsigned int getParticleSize(const char* vSimulatorName);
MPHYSICS_API unsigned int getEulerParticleSize(const char* vSimulatorName);
MPHYSICS_API unsigned int getNeighborDataSize(const char* vSimulatorName);
MPHYSICS_API void copyParticleNeighborDataToCPU(const char* vSimulatorName, unsigned int* voNeighborData,
                                                unsigned int* voNeighborCount, unsigned int* voNeighborOffset);
MPHYSICS_API void getGridInfo(const char* vSimulatorName, MPHYSICS_REF(float) voGridMinX,
                              MPHYSICS_REF(float) voGridMinY, MPHYSICS_REF(float) voGridMinZ,
                              MPHYSICS_REF(float) voGridDeltaX, MPHYSICS_REF(float) voGridDeltaY,
                              MPHYSICS_REF(float) voGridDeltaZ, MPHYSICS_REF(unsigned int) voGridDimX,
                              MPHYSICS_REF(unsigned int) voGridDimY, MPHYSICS_REF(unsigned int) voGridDimZ,
                              MPHYSICS_REF(unsigned int) voMetaGridDimX, MPHYSICS_REF(unsigned int) voMetaGridDimY,
                              MPHYSICS_REF(unsigned int) voMetaGridDimZ,
                              MPHYSICS_REF(unsigned int) voMetaGridDimGroupSize,
                              MPHYSICS_REF(unsigned int) voMetaGridDimBlockSize,
                              MPHYSICS_REF(unsigned int) voCellCount, MPHYSICS_REF(float) voCellSize);
MPHYSICS_API void getEulerGridInfo(const char* vSimulatorName, MPHYSICS_REF(float) voGridOriginX,
                                   MPHYSICS_REF(float) voGridOriginY, MPHYSICS_REF(float) voGridOriginZ,
                                   MPHYSICS_REF(float) voGridSpacingX, MPHYSICS_REF(float) voGridSpacingY,
                                   MPHYSICS_REF(float) voGridSpacingZ);
MPHYSICS_API void copyCellDataToCPU(const char* vSimulatorName, unsigned int* voCellParticleCounts,
                                    unsigned int* voCellParticleOffsets);

/* Added by this library: the message of the last failed MPhysics call ("" if none). */
MPHYSICS_API const char* mphysics_last_error(void);
/* Added by this library: the grid solver behind a loaded simulator, for the
 * hfg_solver_* API (NULL if the name is unknown). */
MPHYSICS_API void* mphysics_grid_solver(const char* vSimulatorName);

#ifdef __cplusplus
}  /* extern "C" */
}  /* namespace MPhysicsAPI */
#endif
#endif /* MPHYSICS_H */
