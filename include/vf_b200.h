/*
 * vf_b200.h -- C ABI of virtualfluids_b200, a B200 (sm_100a) implementation of
 * VirtualFluids' single-GPU lattice-Boltzmann time step.
 *
 * Every entry point takes plain pointers and sizes, launches on the given CUDA
 * stream (NULL = legacy default stream) and returns a status code; nothing
 * calls exit().  The device arrays follow the layout the reference's
 * LBMSimulationParameter uses (src/gpu/core/Parameter/Parameter.h:67-254):
 *
 *   distributions  27 * numberOfLBnodes elements, direction-major
 *                  (f[d * numberOfLBnodes + k], CudaMemoryManager.cpp:169),
 *                  holding the shifted populations f_d - w_d;
 *   neighborX/Y/Z  numberOfLBnodes uint32, the sparse index of the next node in
 *                  the positive axis direction, node 0 a dummy
 *                  (GridImp.cpp:2146-2185);
 *   fluid node list uint32 sparse indices (GridImp.cpp:965-986).
 *
 * The storage argument selects the element type of the distributions:
 * VFB_FP32 (float), VFB_FP64 (double), and the precision form (16-bit storage,
 * FP32 arithmetic): VFB_FP16 (IEEE half of the deviation times 2^12),
 * VFB_BF16 (bfloat16), VFB_FX16 (int16 q with f_d - w_d = q * w_d * 2^-17:
 * deviations below a quarter of the weight at a uniform step, saturating
 * beyond) and VFB_FX16W (int16 q with f_d - w_d = q * w_d * R_d * 2^-15,
 * R_d = 1/4 for the rest population, 1/2 for the faces, 1 for the edges and
 * corners: the range of flows whose deviations leave FX16's); no counterpart
 * in the reference.  Arrays documented as "compute
 * precision" are double for VFB_FP64 and float otherwise.
 */
#ifndef VF_B200_H
#define VF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define VFB_OK 0
#define VFB_ERR_INVALID_ARGUMENT (-1)
#define VFB_ERR_CUDA (-2)
#define VFB_ERR_UNSUPPORTED (-3)
#define VFB_ERR_NOT_FINITE (-4)
#define VFB_ERR_OUT_OF_RANGE (-5)
#define VFB_ERR_CONFIGURATION (-6)

/* storage formats */
#define VFB_FP32 0
#define VFB_FP64 1
#define VFB_FP16 2
#define VFB_BF16 3
#define VFB_FX16 4
#define VFB_FX16W 5

/* CollisionTemplate (src/gpu/core/Calculation/Calculation.h:55-68) */
#define VFB_TEMPLATE_DEFAULT 0
#define VFB_TEMPLATE_WRITE_MACRO_VARS 1
#define VFB_TEMPLATE_APPLY_BODY_FORCE 2
#define VFB_TEMPLATE_ALL_FEATURES 3

/* GEO types of typeOfGridNode (Calculation.h:38-48) */
#define VFB_GEO_SOLID 15
#define VFB_GEO_VOID 16
#define VFB_GEO_FLUID 19

/* library version (major * 10000 + minor * 100 + patch) */
int vfb_version(void);
/* message of the last failing call on this host thread ("" if none) */
const char* vfb_last_error(void);
/* bytes of one stored population for a storage format, 0 if unknown */
int vfb_storage_bytes(int storage);
/* copy bytes from device memory to host memory on the stream and wait for it
 * (a convenience for hosts without their own CUDA runtime binding, e.g. to
 * read arrays that vfb_sim_stress_list points at) */
int vfb_copy_device_to_host(void* dst, const void* src, size_t bytes, void* stream);

/*
 * Collision arguments.  Mirrors vf::gpu::GPUCollisionParameter
 * (src/gpu/core/Utilities/RunCollision.cuh:49-72); the three global forces and
 * the quadric limiters are passed by value instead of as device pointers.
 */
typedef struct vfb_collision_args {
    void* distributions;
    unsigned long long numberOfLBnodes;
    const uint32_t* neighborX;
    const uint32_t* neighborY;
    const uint32_t* neighborZ;
    const uint32_t* fluidNodeIndices;
    uint32_t numberOfFluidNodes;
    double omega;
    double forces[3];          /* global acceleration (Parameter::getForcesDev) */
    double forceFactor;        /* 2^-level (KernelUtilities.h:56-64) */
    double quadricLimiters[3]; /* P, M, D (Parameter.cpp:69) */
    int isEvenTimestep;
    int collisionTemplate;     /* VFB_TEMPLATE_* */
    void* rho;                 /* compute precision, numberOfLBnodes; templates 1 and 3 */
    void* vx;
    void* vy;
    void* vz;
    void* bodyForceX;          /* compute precision, numberOfLBnodes; templates 2 and 3 */
    void* bodyForceY;
    void* bodyForceZ;
} vfb_collision_args;

/*
 * K17 compressible cumulant collision fused with esoteric-twist streaming over
 * a fluid-node list.  Replaces K17CompressibleNavierStokes<None>::runOnIndices
 * (src/gpu/core/Kernel/Compressible/NavierStokes/K17/K17CompressibleNavierStokes.cu:103-145),
 * i.e. vf::gpu::runCollision<K17> (src/gpu/core/Utilities/RunCollision.cuh:74-143).
 */
int vfb_k17_collision(int storage, const vfb_collision_args* args, void* stream);

/*
 * BGK compressible collision fused with esoteric-twist streaming.  Replaces
 * B92CompressibleNavierStokes::run
 * (src/gpu/core/Kernel/Compressible/NavierStokes/B92/B92CompressibleNavierStokes.cu:43-57),
 * which visits every node whose typeOfGridNode is neither GEO_SOLID nor
 * GEO_VOID; pass the fluid-node list of those nodes (the reference's fluid-node
 * list is exactly that set).  Only omega, the arrays, the node list and
 * isEvenTimestep of args are used.
 */
int vfb_bgk_collision(int storage, const vfb_collision_args* args, void* stream);

/*
 * Collision plan: a one-off analysis of a level's fluid-node list and
 * neighbour arrays that lets the planned kernels fetch runs of regular nodes
 * with bulk copies (cp.async.bulk) one warp tile ahead and skip the index
 * chain for them (virtualfluids_b200/csrc/collision_tiled.cu).  Building a
 * plan copies the index arrays to the host once.  The planned kernels compute
 * exactly what vfb_k17_collision / vfb_bgk_collision compute; they require a
 * 16-byte aligned distributions array and the same index arrays (pointers,
 * sizes) the plan was built for.  No counterpart in the reference, whose
 * kernels always follow the index chain (KernelUtilities.h:221-245).
 */
typedef struct vfb_collision_plan vfb_collision_plan;
int vfb_collision_plan_create(int storage, const vfb_collision_args* args, vfb_collision_plan** plan, void* stream);
int vfb_collision_plan_destroy(vfb_collision_plan* plan);
/* out6: tiles, bulk tiles, lane-by-lane tiles, bulk-fed nodes, periodic
 * wrap nodes served inside bulk tiles, nodes collided lane by lane */
int vfb_collision_plan_stats(const vfb_collision_plan* plan, unsigned long long* out6);
/* VFB_OK, or VFB_ERR_CUDA if a bounded wait of a planned kernel ran out
 * (synchronises the stream) */
int vfb_collision_plan_check(const vfb_collision_plan* plan, void* stream);
/*
 * BC epilogue of a plan: the post-collision BC lists of the plan's level, in
 * the order the schedule runs them.  Every list entry whose node the plan's
 * tiles collide, and whose active links all write cells that no collision
 * and no other entry reads in the same step (the cell's reader, the node
 * across the link, is a boundary stopper or a solid node, not a fluid node),
 * is applied by the planned collision kernel right after that node's own
 * collision, from the values the kernel has just stored, instead of by a
 * separate BC launch after the whole collision; the result is the same.
 * Nodes listed in excludedNodes (device array, e.g. a stress list whose kernel
 * runs between the post-collision lists) are never taken.  fused (device,
 * one byte per entry) receives 1 for the entries the epilogue applies; the
 * caller runs the remaining entries with vfb_bc_post after the collision as
 * before.  The lists' arrays must stay valid while the plan is used; nLists 0
 * removes the epilogue.  VFB_ERR_UNSUPPORTED for the direct-load and
 * per-thread pipelined tile configurations.  No reference counterpart.
 */
typedef struct vfb_bc_epilogue_list {
    int kind;                   /* a post-collision VFB_BC_* kind */
    const int32_t* k;
    const void* q;              /* 27 * numberOfBCnodes, direction-major, compute precision */
    const void* Vx;             /* velocity kinds */
    const void* Vy;
    const void* Vz;
    const uint32_t* locations;  /* the list's location table (vfb_bc_locations), required */
    uint32_t numberOfBCnodes;
    uint8_t* fused;             /* output */
} vfb_bc_epilogue_list;
int vfb_collision_plan_set_bc_epilogue(vfb_collision_plan* plan, const vfb_bc_epilogue_list* lists, int nLists,
                                       double omega, const int32_t* excludedNodes, uint32_t nExcluded, void* stream);
/* out2: nodes and entries the plan's BC epilogue applies */
int vfb_collision_plan_epilogue_stats(const vfb_collision_plan* plan, unsigned long long* out2);

/* planned K17CompressibleNavierStokes::runOnIndices / B92 run */
int vfb_k17_collision_planned(const vfb_collision_plan* plan, const vfb_collision_args* args, void* stream);
int vfb_bgk_collision_planned(const vfb_collision_plan* plan, const vfb_collision_args* args, void* stream);

/*
 * Boundary conditions.  The lattice a BC kernel runs on, and one compacted BC
 * list: QforBoundaryConditions (src/gpu/core/Calculation/Calculation.h:105-117)
 * with k the BC node indices, q the subgrid distances direction-major
 * (q[d * numberOfBCnodes + i], src/gpu/core/Utilities/KernelUtilities.h:140-169;
 * a direction is active when 0 <= q <= 1) and Vx/Vy/Vz the per-node wall
 * velocity of a velocity BC.  q and the velocities are compute-precision arrays.
 */
typedef struct vfb_bc_lattice {
    void* distributions;
    unsigned long long numberOfLBnodes;
    const uint32_t* neighborX;
    const uint32_t* neighborY;
    const uint32_t* neighborZ;
    double omega;
    int isEvenTimestep; /* the parity the reference passes at this call */
} vfb_bc_lattice;

typedef struct vfb_bc_list {
    const int32_t* k;
    const void* q;
    const void* Vx;
    const void* Vy;
    const void* Vz;
    uint32_t numberOfBCnodes;
    /* optional (NULL: the kernels walk the neighbour arrays as the reference
     * does): the eight locations of every entry's node, locations[l * n + i]
     * for location l of entry i (vfb_bc_locations); no reference counterpart */
    const uint32_t* locations;
} vfb_bc_list;

/* The location table of a BC list (vfb_bc_list.locations): for each entry i
 * the eight locations k, nX[k], nY[k], nY[nX[k]], nZ[k], nZ[nX[k]], nZ[nY[k]],
 * nZ[nY[nX[k]]] of its node k (KernelUtilities.h:221-245) into the device
 * array out (8 * numberOfBCnodes uint32).  Computed once per list, it spares
 * every BC launch the chain of dependent neighbour loads.  No reference
 * counterpart. */
int vfb_bc_locations(const int32_t* k, uint32_t numberOfBCnodes, const uint32_t* neighborX,
                     const uint32_t* neighborY, const uint32_t* neighborZ, uint32_t* out, void* stream);

/* post-collision BC kinds (BoundaryConditionFactory.h:75-94) */
#define VFB_BC_NOSLIP_INTERPOLATED 0   /* NoSlipInterpolatedCompressible_Device, NoSlip/NoSlipInterpolatedCompressible.cu:44-378 */
#define VFB_BC_NOSLIP_BOUNCE_BACK 1    /* NoSlipBounceBack_Device, NoSlip/NoSlipBounceBack.cu */
#define VFB_BC_VELOCITY_INTERPOLATED 2 /* VelocityInterpolatedCompressible_Device, Velocity/VelocityInterpolatedCompressible.cu:44-418 */
#define VFB_BC_VELOCITY_BOUNCE_BACK 3  /* VelocityBounceBack_Device, Velocity/VelocityBounceBack.cu */
#define VFB_BC_SLIP 4                  /* SlipCompressible_Device, Slip/SlipCompressible.cu:45-550 */
#define VFB_BC_VELOCITY_WITH_PRESSURE 5 /* VelocityWithPressureInterpolatedCompressible_Device,
                                           Velocity/VelocityWithPressureInterpolatedCompressible.cu */

/*
 * One post-collision BC kernel over a list (one thread per BC node).  Replaces
 * the host launchers NoSlipInterpolatedCompressible / NoSlipBounceBack
 * (src/gpu/core/BoundaryConditions/NoSlip/NoSlip.cu:81-98),
 * VelocityInterpolatedCompressible / VelocityBounceBack (Velocity/Velocity.cu)
 * and SlipCompressible (Slip/Slip.cu), called by
 * BoundaryConditionKernelManager::runVelocityBCKernelPost / runNoSlipBCKernelPost
 * / runSlipBCKernelPost (BoundaryConditionKernelManager.cpp:257-344) in the
 * order velocity, no-slip, slip.  The velocity arrays are read by the velocity
 * kinds only.
 */
int vfb_bc_post(int kind, int storage, const vfb_bc_lattice* lattice, const vfb_bc_list* list, void* stream);

/* wall-model (stress) BC kinds (StressBC, BoundaryConditionFactory.h:110-117) */
#define VFB_BC_STRESS_INTERPOLATED 6          /* StressCompressible_Device, Stress/StressCompressible.cu:50-762 */
#define VFB_BC_STRESS_BOUNCE_BACK 7           /* StressBounceBackCompressible_Device, Stress/StressBounceBackCompressible.cu:50-679 */
#define VFB_BC_STRESS_BOUNCE_BACK_PRESSURE 8  /* StressBounceBackPressureCompressible_Device,
                                                 Stress/StressBounceBackPressureCompressible.cu */

/* A stress list: the reference's stressBC (QforBoundaryConditions) with the
 * level's wallModel arrays (CudaMemoryManager.cpp:1139-1200, GridGenerator.cpp:319-341).
 * Arrays of reals are in the compute precision (double for VFB_FP64, float
 * otherwise); all are device arrays of numberOfBCnodes entries except q
 * (27 * numberOfBCnodes, direction-major). */
typedef struct vfb_stress_list {
    const int32_t* k;              /* BC nodes */
    const int32_t* kN;             /* velocity sampling node of each entry */
    const void* q;
    const void* normalX;           /* wall normal (unit, into the fluid) */
    const void* normalY;
    const void* normalZ;
    void* Vx;                      /* filtered velocity at the sampling node (updated every call) */
    void* Vy;
    void* Vz;
    void* Vx1;                     /* filtered velocity at the wall node (updated every call) */
    void* Vy1;
    void* Vz1;
    const int32_t* samplingOffset; /* wallModel.samplingOffset: sampling height in nodes */
    const void* z0;                /* wallModel.z0: roughness length in lattice units */
    void* uStar;                   /* monitors (wallModel.u_star, Fx, Fy, Fz): all four or none (NULL) */
    void* Fx;
    void* Fy;
    void* Fz;
    uint32_t numberOfBCnodes;
    const uint32_t* locations;     /* optional location table, as vfb_bc_list.locations */
} vfb_stress_list;

/*
 * One wall-model BC kernel over a stress list (one thread per entry).
 * Replaces the host launchers StressCompressible, StressBounceBackCompressible
 * and StressBounceBackPressureCompressible (Stress.cu:42-160), run by
 * BoundaryConditionKernelManager::runStressWallModelKernelPost
 * (BoundaryConditionKernelManager.cpp:330-334) after the slip BC.  vx, vy, vz
 * are the level's macroscopic velocity arrays (numberOfLBnodes entries), read
 * at the sampling nodes: the reference's launchers pass velocityX, velocityY
 * and velocityY again as vz, and the simulation here passes the same.
 * turbViscosity (numberOfLBnodes entries) may be NULL: no turbulence model,
 * the interpolated kind relaxes with omega.  Monitors are written when uStar
 * is non-NULL (hasWallModelMonitor).
 */
int vfb_bc_stress(int kind, int storage, const vfb_bc_lattice* lattice, const vfb_stress_list* list,
                  const void* turbViscosity, const void* vx, const void* vy, const void* vz, void* stream);

/*
 * The pre-collision non-equilibrium pressure BC of one directional list
 * (QforDirectionalBoundaryCondition, Calculation.h:119-127).  Replaces
 * PressureNonEquilibriumCompressible (src/gpu/core/BoundaryConditions/Pressure/Pressure.cu),
 * i.e. PressureNonEquilibriumCompressible_Device
 * (Pressure/PressureNonEquilibriumCompressible.cu:45-311): k the BC nodes, kN
 * their inner neighbours, rhoBC the prescribed drho (compute precision),
 * direction the D3Q27 id of the outward normal (1..6: P00, M00, 0P0, 0M0, 00P,
 * 00M).  lattice->omega is not used.
 */
int vfb_bc_pressure_noneq(int storage, const vfb_bc_lattice* lattice, const int32_t* k, const int32_t* kN,
                          const void* rhoBC, uint32_t numberOfBCnodes, int direction, void* stream);

/*
 * The non-reflecting outflow of one directional list, in the pre-collision
 * slot of the pressure BC.  Replaces OutflowNonReflecting and, with
 * pressureCorrection != 0, OutflowNonReflectingPressureCorrection
 * (src/gpu/core/BoundaryConditions/Outflow/Outflow.cu:44-84; kernels
 * OutflowNonReflecting.cu:50-276 and OutflowNonReflectingPressureCorrection.cu:51-241),
 * which BoundaryConditionFactory returns for PressureBC::OutflowNonReflective
 * and ::OutflowNonReflectivePressureCorrection (BoundaryConditionFactory.cpp:162-166).
 * k, kN, direction as for vfb_bc_pressure_noneq; correctionFactor is
 * Parameter::outflowPressureCorrectionFactor (used with the correction only).
 * lattice->omega is not used.
 */
int vfb_bc_outflow_nonreflecting(int storage, const vfb_bc_lattice* lattice, const int32_t* k, const int32_t* kN,
                                 uint32_t numberOfBCnodes, int direction, int pressureCorrection,
                                 double correctionFactor, void* stream);

/*
 * Grid scaling between a level and the next finer one.  Mirrors the
 * gridScaling function type (src/gpu/core/GridScaling/GridScalingFactory.h:46)
 * with the interface cells of InterpolationCells / ICellNeigh
 * (src/gpu/core/Calculation/Calculation.h:72-89): cell i is given by the base
 * (most negative) coarse node coarseCells[i] and the base fine node
 * fineCells[i] of its 2x2x2 source block (coarse-to-fine), or by the coarse
 * node at its centre coarseCells[i] and the base fine node fineCells[i]
 * (fine-to-coarse); offsetX/Y/Z (compute precision) shift the interpolation
 * point for refinement into a wall.  isEvenTimestep is the coarse level's
 * parity; the fine level is always read / written in the even view, as in the
 * reference.  Replace scaleCoarseToFineCompressible<false> and
 * scaleFineToCoarseCompressible<false> (GridScaling/Scaling.cuh:44-58;
 * kernels scaleCoarseToFineCompressible.cu:305-528, scaleFineToCoarseCompressible.cu:76-124),
 * called by GridScalingKernelManager::runCoarseToFineKernelLB /
 * runFineToCoarseKernelLB (GridScalingKernelManager.cpp:64-74).
 */
typedef struct vfb_scaling_args {
    void* distributionsCoarse;
    void* distributionsFine;
    const uint32_t* neighborXcoarse;
    const uint32_t* neighborYcoarse;
    const uint32_t* neighborZcoarse;
    const uint32_t* neighborXfine;
    const uint32_t* neighborYfine;
    const uint32_t* neighborZfine;
    unsigned long long numberOfLBnodesCoarse;
    unsigned long long numberOfLBnodesFine;
    int isEvenTimestep;
    const uint32_t* coarseCells;
    const uint32_t* fineCells;
    uint32_t numberOfCells;
    double omegaCoarse;
    double omegaFine;
    const void* offsetX;
    const void* offsetY;
    const void* offsetZ;
    /* coarse to fine only: bit c of fineWriteMask[27 i + d] set = cell i
     * writes direction d of its fine node at corner c (bit 0 x, 1 y, 2 z);
     * NULL = every cell writes everything.  Cells of a real grid write some
     * memory cells more than once (cells repeated across periodic seams, edge
     * stoppers whose locations alias other nodes'); the reference kernel
     * races there.  vfb_scaling_write_mask gives the mask under which the
     * result is that of the cells applied one by one in list order. */
    const uint8_t* fineWriteMask;
    /* optional (NULL: the kernels walk the neighbour arrays): the 3x3x3 block
     * of node indices above each cell's coarse / fine base node,
     * coarseBlocks[27 i + x + 3 y + 9 z] (vfb_scaling_blocks), so that a
     * launch reads the cell's nodes in one round instead of a chain of
     * dependent neighbour loads.  No counterpart in the reference. */
    const uint32_t* coarseBlocks;
    const uint32_t* fineBlocks;
} vfb_scaling_args;

/* the blocks of vfb_scaling_args.coarseBlocks / fineBlocks for numberOfCells
 * base nodes (device arrays; out holds 27 * numberOfCells uint32), walked
 * along the reference's neighbour paths */
int vfb_scaling_blocks(const uint32_t* cells, uint32_t numberOfCells, const uint32_t* neighborX,
                       const uint32_t* neighborY, const uint32_t* neighborZ, uint32_t* out, void* stream);
int vfb_scale_coarse_to_fine(int storage, const vfb_scaling_args* args, void* stream);
int vfb_scale_fine_to_coarse(int storage, const vfb_scaling_args* args, void* stream);
/* vfb_scale_fine_to_coarse then vfb_scale_coarse_to_fine, in one launch (the
 * two lists' cells in one grid).  Valid only when neither list reads a cell
 * the other writes (vfb_scaling_independent), so that the reference's order
 * (fine to coarse first, UpdateGrid27.cpp:89-93) does not matter.  No
 * counterpart in the reference. */
int vfb_scale_interface(int storage, const vfb_scaling_args* fineToCoarse, const vfb_scaling_args* coarseToFine,
                        void* stream);
/* Host arrays: *independent = 1 when, in both parities, no fine cell the
 * coarse-to-fine cells write (under cfMask, NULL = all) is read by the
 * fine-to-coarse cells and no coarse cell the fine-to-coarse cells write is
 * read by the coarse-to-fine cells; else 0.  No counterpart in the reference. */
int vfb_scaling_independent(const uint32_t* fineToCoarseCoarseCells, const uint32_t* fineToCoarseFineCells,
                            uint32_t numberOfFineToCoarseCells, const uint32_t* coarseToFineCoarseCells,
                            const uint32_t* coarseToFineFineCells, uint32_t numberOfCoarseToFineCells,
                            const uint8_t* coarseToFineWriteMask, const uint32_t* neighborXcoarse,
                            const uint32_t* neighborYcoarse, const uint32_t* neighborZcoarse,
                            unsigned long long numberOfLBnodesCoarse, const uint32_t* neighborXfine,
                            const uint32_t* neighborYfine, const uint32_t* neighborZfine,
                            unsigned long long numberOfLBnodesFine, int* independent);
/* the same interpolation on the host (host arrays, VFB_FP32 or VFB_FP64),
 * with the library's own arithmetic; for checks without a GPU.  No
 * counterpart in the reference. */
int vfb_debug_scale_host(int coarseToFine, int precision, const vfb_scaling_args* args);
/* Host arrays: for numberOfCells coarse-to-fine cells with base fine nodes
 * fineCells, the write mask (27 bytes per cell) under which every memory cell
 * is written only by its last writer in the order cells, then corners as the
 * reference visits them.  No counterpart in the reference. */
int vfb_scaling_write_mask(const uint32_t* fineCells, uint32_t numberOfCells, const uint32_t* neighborXfine,
                           const uint32_t* neighborYfine, const uint32_t* neighborZfine,
                           unsigned long long numberOfLBnodesFine, uint8_t* mask);

/*
 * Grid builder (host only).  Builds the sparse grid of a box and exports the
 * arrays the kernels consume, bit for bit those of the reference's
 * MultipleGridBuilder / LevelGridBuilder (src/gpu/GridGenerator/grid/GridBuilder/
 * MultipleGridBuilder.cpp, LevelGridBuilder.cpp:395-944, GridImp.cpp:914-1121,
 * Side.cpp:64-215, GridInterface.cpp:60-428).  spec (at least 61 values):
 * [0..6] coarse grid start x, y, z, end x, y, z, delta
 * (MultipleGridBuilder::addCoarseGrid); [7..9] periodic x, y, z
 * (setPeriodicBoundaryCondition); [10] refinement box present, [11..16] the box
 * (min x, y, z, max x, y, z; MultipleGridBuilder::addGrid with a Cuboid);
 * [17..18] layers fine / between levels (setNumberOfLayers, used when [17] > 0);
 * [19] solid primitive (addGeometry, meshed on the finest level): 1 a Cuboid
 * with [20..25] its extent, 2 a Sphere with [20..23] centre and radius (its
 * links' q values from the ray intersection, GridImp::calculateQs), 3 a
 * Cylinder with [20..25] centre, radius, height and axis (0 x, 1 y, 2 z;
 * no ray intersection, like the cuboid), 4 a VerticalCylinder with [20..24]
 * centre, radius and height, 5 a Conglomerate (Conglomerate::add / subtract)
 * of [62] added and [63] subtracted primitives, 7 values each (kind 1..4 and
 * its parameters as above) from [64] on, n >= 64 + 7 parts (no ray
 * intersection); [26] geometry BC (1 = no-slip, setNoSlipBoundaryCondition
 * (GEOMETRY)); [30..59] up to six side BCs as (side 0..5 = MX PX MY PY MZ PZ,
 * type 1 no-slip / 2 velocity / 3 pressure / 4 slip, three values) applied in
 * order (setNoSlip / setVelocity / setPressure / setSlipBoundaryCondition);
 * [60] enableThinWalls (with a solid: boundary nodes without a fluid neighbour become solid stoppers); [61] finest level of the box (0 =
 * 1; needs n >= 62).  Returns a handle, NULL on error.  Array names per level:
 * "geo", "neighborX/Y/Z", "neighborNeg", "coordX/Y/Z", "fluid", "dims",
 * "velocity.k/.q/.vx/.vy/.vz", "slip.k/.q/.nx/.ny/.nz", "geometry.k/.q",
 * "pressure.count", "pressure<i>.k/.kN/.rho/.q/.dir" and, on every level but the
 * finest, the interface cells to the next level: "cf.coarse/.fine/.offX/.offY/
 * .offZ" and "fc.coarse/.fine/.offX/.offY/.offZ" (getGridInterfaceIndices,
 * getOffsetCF / getOffsetFC).
 */
void* vfb_grid_build(const double* spec, int n);
int vfb_grid_levels(void* grid);
/* number of elements of an array (-1 if unknown) and their size in bytes */
long long vfb_grid_count(void* grid, int level, const char* name);
int vfb_grid_elem_size(void* grid, int level, const char* name);
/* copies the array into out (count * elem_size bytes) */
int vfb_grid_copy(void* grid, int level, const char* name, void* out);
void vfb_grid_free(void* grid);
/* An empty grid container to be filled array by array by another grid
 * provider (e.g. grids made by the reference's own builder or read from
 * files), with the names and element types vfb_grid_build exports; levels
 * above 0 may add the interface cells of the level and the next finer one:
 * "cf.coarse", "cf.fine", "fc.coarse", "fc.fine" (uint32) and "cf.offX/Y/Z",
 * "fc.offX/Y/Z" (double), the arrays of LevelGridBuilder::getGridInterfaceIndices /
 * getOffsetCF / getOffsetFC (LevelGridBuilder.cpp:395-944).  The role of the
 * reference's GridProvider (GridGenerator.cpp:91-1035). */
void* vfb_grid_create(int levels);
int vfb_grid_put(void* grid, int level, const char* name, int elemSize, long long count, const void* data);

/*
 * Simulation: the host side of the time step.  Mirrors Simulation /
 * UpdateGrid27 of the reference (src/gpu/core/Calculation/Simulation.cpp:117-441,
 * UpdateGrid27.cpp:54-96,228-308): it owns every level's device arrays
 * (uploaded from a vfb_grid handle), selects the collision and BC kernels like
 * KernelFactory / BoundaryConditionFactory, and runs the recursive per-level
 * substep schedule
 *   updateGrid(level): if level is not the finest, updateGrid(level + 1) twice;
 *                      collision; post-collision BCs (velocity, no-slip, slip,
 *                      geometry); parity swap; pre-collision BCs (pressure);
 *                      if not the finest, fine-to-coarse then coarse-to-fine.
 * Level l uses nu_l = nu * 2^l, omega_l = 1 / (3 nu_l + 1/2) and force factor
 * 2^-l (Parameter.cpp:395-420).
 */
typedef struct vfb_sim_params {
    int storage;               /* VFB_FP32 / FP64 / FP16 / BF16 */
    int collisionKernel;       /* 0 "K17CompressibleNavierStokes", 1 "BGKCompSP27" (KernelTypes.h:36-38) */
    int velocityBC;            /* VFB_BC_VELOCITY_INTERPOLATED, VFB_BC_VELOCITY_BOUNCE_BACK or VFB_BC_VELOCITY_WITH_PRESSURE */
    int noSlipBC;              /* VFB_BC_NOSLIP_INTERPOLATED, VFB_BC_NOSLIP_BOUNCE_BACK, -1 NoSlipDelayBounceBack (no kernel) */
    int geometryBC;            /* as noSlipBC, for the geometry list; or a velocity kind when the grid gives
                                  the geometry a velocity (geometry.vx/vy/vz) */
    int slipBC;                /* VFB_BC_SLIP or -1 */
    int pressureBC;            /* 0 PressureNonEquilibriumCompressible, 1 OutflowNonReflective,
                                  2 OutflowNonReflectivePressureCorrection, -1 none */
    double viscosity;          /* coarse-level kinematic viscosity, lattice units */
    double forces[3];          /* global acceleration */
    double quadricLimiters[3]; /* default 0.01 each (Parameter.cpp:69) */
    int usePlan;               /* 1: the planned (bulk-copy) collision kernels */
    int useGraphs;             /* 1: replay two coarse steps at a time from a captured CUDA graph */
    int useInitNeq;            /* 1: vfb_sim_init_level writes equilibrium plus the strain-rate part
                                  (Parameter::setUseInitNeq); the grid must carry neighborNeg */
    double outflowPressureCorrectionFactor; /* pressureBC 2 (Parameter::setOutflowPressureCorrectionFactor) */
    double velocityRatio;      /* Parameter::getVelocityRatio (world to lattice units): the geometry list's
                                  velocities are divided by it at upload, in the compute precision, as
                                  GridGenerator.cpp:507-513 does (side velocity BCs are not scaled);
                                  0 or 1: no scaling */
    int stressBC;              /* VFB_BC_STRESS_INTERPOLATED / _BOUNCE_BACK / _BOUNCE_BACK_PRESSURE, -1 none
                                  (BoundaryConditionFactory::setStressBoundaryCondition); runs after the slip
                                  BC on the grid's stress lists (UpdateGrid27.cpp:243-245) */
    int hasWallModelMonitor;   /* 1: the stress kernels write u* and the wall momentum per entry
                                  (Parameter::setHasWallModelMonitor) */
    int bcEpilogue;            /* 1: with usePlan, the planned collision applies the post-collision BCs of
                                  its wall nodes itself (vfb_collision_plan_set_bc_epilogue; the same
                                  result); 0: separate BC launches for every entry */
} vfb_sim_params;

typedef struct vfb_simulation vfb_simulation;
/* uploads every level of grid (a vfb_grid_build handle; it may be freed afterwards) */
int vfb_sim_create(const vfb_sim_params* params, void* grid, vfb_simulation** sim, void* stream);
int vfb_sim_destroy(vfb_simulation* sim);
int vfb_sim_levels(const vfb_simulation* sim);
/* equilibrium (or, with useInitNeq, non-equilibrium) populations from host
 * arrays (compute precision, numberOfLBnodes of the level) into both parity
 * views, odd then even (PreProcessorImp.cpp:50-58) */
int vfb_sim_init_level(vfb_simulation* sim, int level, const void* rho, const void* vx, const void* vy, const void* vz,
                       void* stream);
/* coarse time steps (each runs 2^l substeps of level l).  With useGraphs,
 * the launches of two coarse steps (after which every level's parity is back
 * where it started) are captured once into a CUDA graph on an internal
 * stream, after two ordinary warm-up steps, and replayed into the given
 * stream; an odd remainder runs ordinarily.  No counterpart in the reference,
 * which launches every kernel from the host every substep. */
int vfb_sim_run(vfb_simulation* sim, unsigned int steps, void* stream);
/* macroscopic fields of a level into host arrays (compute precision); synchronises */
int vfb_sim_macroscopic(vfb_simulation* sim, int level, void* rho, void* vx, void* vy, void* vz, void* stream);
/* FP64 sums over the level's fluid nodes (see vfb_mass_and_energy) */
int vfb_sim_mass_and_energy(vfb_simulation* sim, int level, double* out3, void* stream);
/* KineticEnergyAnalyzer::run (src/gpu/core/PostProcessor/KineticEnergyAnalyzer.cu:66-108,137-154):
 * out2[0] = sum of (drho + 1) |u|^2 / 2 over the level's nodes whose type is
 * fluid and whose six axis neighbours (reached as the reference reaches them,
 * through neighborX/Y/Z and the inverse neighbour) are fluid, divided by their
 * number; out2[1] = that number.  The sum is FP64 (the reference reduces in
 * the working precision).  Synchronises the stream. */
int vfb_sim_kinetic_energy(vfb_simulation* sim, int level, double* out2, void* stream);
/* EnstrophyAnalyzer::run (src/gpu/core/PostProcessor/EnstrophyAnalyzer.cu:63-98)
 * on a level: out2[0] = the mean of 1/2 (drho + 1) |curl u|^2 over the fluid
 * nodes whose six axis neighbours are fluid (FP64 sum), out2[1] = their
 * number.  Computes the macroscopic fields into temporary device arrays
 * first; synchronises the stream. */
int vfb_sim_enstrophy(vfb_simulation* sim, int level, double* out2, void* stream);
/* vfb_saturated_populations on a level's populations */
int vfb_sim_saturated_populations(vfb_simulation* sim, int level, unsigned long long* count, void* stream);
/*
 * Adjoint of the time step (no counterpart in the reference, which has no
 * adjoint).  The differentiated step is the reference's single-level
 * UpdateGrid27 step (UpdateGrid27.cpp:54-96): K17 collision with the global
 * force (K17CompressibleNavierStokes.h:87-591, RunCollision.cuh:88-114), the
 * velocity list (VelocityInterpolatedCompressible.cu:44-418), the no-slip and
 * geometry lists (NoSlipInterpolatedCompressible.cu:44-378), the parity swap
 * and the pressure lists (PressureNonEquilibriumCompressible.cu:45-311).
 * Other configurations (several levels, BGK, 16-bit storage, bounce-back,
 * slip or outflow lists) return VFB_ERR_UNSUPPORTED.
 *
 * vfb_sim_adjoint_forward runs `steps` time steps from the current state (the
 * state advances, as with vfb_sim_run), keeping a copy of the state every
 * checkpointInterval steps, and returns in *J the objective on the final state
 *     J = sum_j wx[j] ux(k_j) + wy[j] uy(k_j) + wz[j] uz(k_j),
 * u = (momentum) / (1 + drho) of node k_j = objectiveNodes[j] (host arrays).
 * vfb_sim_adjoint_backward then computes, for L with dL/dJ = seed,
 *     dVelocity[c * n + i] = dL / dU_c of entry i of the level's velocity list
 *                            (c = 0, 1, 2 for x, y, z; n entries; host array),
 *     dForces[c]           = dL / d(global force c)   (host array of 3),
 * by recomputing each checkpoint segment with taped inputs and running the
 * hand-written adjoint kernels backwards through it.  With checkpointInterval
 * >= steps the run is one segment and the forward pass records the tapes
 * itself, so the backward pass recomputes nothing (the same tape memory).
 * Either output may be NULL.  Both calls synchronise the stream.  Device
 * memory: a state copy per checkpoint, and per segment 27 values per fluid
 * node and per BC node and step.
 */
int vfb_sim_adjoint_forward(vfb_simulation* sim, unsigned int steps, unsigned int checkpointInterval,
                            const uint32_t* objectiveNodes, const double* wx, const double* wy, const double* wz,
                            uint32_t numberOfObjectiveNodes, double* J, void* stream);
int vfb_sim_adjoint_backward(vfb_simulation* sim, double seed, double* dVelocity, double* dForces, void* stream);
/* the schedule of the last vfb_sim_adjoint_forward: out2[0] = 1 when the
 * velocity, no-slip and geometry lists run in one launch per step (no list
 * writes a cell another list reads or writes), out2[1] = 1 when the forward
 * pass taped its only segment (the backward pass recomputes nothing) */
int vfb_sim_adjoint_schedule(const vfb_simulation* sim, int* out2);
/* Parameter::setForcing (Parameter.cpp:463) on a running simulation (the next steps use
 * the new global force); no reference counterpart as an in-run setter */
int vfb_sim_set_forces(vfb_simulation* sim, const double* forces3);
/* the velocity values of every entry of a level's velocity list (host arrays
 * of the list's length), as the grid generator's getVelocityValues hands them
 * over (GridGenerator.cpp:345-363); they take effect from the next step */
int vfb_sim_set_velocity_bc(vfb_simulation* sim, int level, const double* vx, const double* vy, const double* vz,
                            void* stream);

/*
 * The output of a level in one read of its populations (the work of
 * Simulation::readAndWriteFiles, Simulation.cpp:595-739, with the analyzers
 * KineticEnergyAnalyzer.cu:66-154 and EnstrophyAnalyzer.cu:63-98): out8 =
 * {sum of drho over the fluid list, sum of (1 + drho)|u|^2/2 over it,
 * non-finite nodes, the kinetic-energy analyzer's mean, its node count, the
 * enstrophy analyzer's mean, its node count (0 without an inverse neighbour
 * array), the fluid-list length}, sums in FP64; the same values as
 * vfb_sim_mass_and_energy, vfb_sim_kinetic_energy and vfb_sim_enstrophy.  The
 * fields drho, vx, vy, vz (compute precision, numberOfLBnodes) are copied into
 * the host arrays given (NULL: not copied).  Synchronises the stream.
 */
int vfb_sim_output(vfb_simulation* sim, int level, double* out8, void* rho, void* vx, void* vy, void* vz,
                   void* stream);

/*
 * The level's stress list as the stress kernels see it (device pointers owned
 * by the simulation; numberOfBCnodes 0 when the level has none): the wall
 * model's filter states and, with hasWallModelMonitor, u* and the wall
 * momentum per entry (the arrays a WallModelProbe reads,
 * Samplers/WallModelProbe.cu:203-218).
 */
int vfb_sim_stress_list(vfb_simulation* sim, int level, vfb_stress_list* out);

/* out3: nodes and BC entries the level's collision applies in its BC
 * epilogue, and the entries left to separate BC launches (all of them
 * without the epilogue) */
int vfb_sim_bc_epilogue_stats(vfb_simulation* sim, int level, unsigned long long* out3);

/* the level's device population array and its parity, for inspection */
int vfb_sim_level_state(vfb_simulation* sim, int level, void** distributions, unsigned long long* numberOfLBnodes,
                        int* isEvenTimestep, double* omega);

/*
 * Equilibrium initialisation of one parity view from drho and velocity
 * (compute precision arrays of numberOfLBnodes).  Replaces
 * InitNavierStokesCompressible_Device
 * (src/gpu/core/PreProcessor/PreProcessorStrategy/InitNavierStokesCompressible/InitNavierStokesCompressible_Device.cu:44-212);
 * nodes whose geo is GEO_SOLID or GEO_VOID are skipped.  PreProcessorImp::init
 * (PreProcessorImp.cpp:50-58) calls it for the odd then the even view.
 */
int vfb_init_equilibrium(int storage, void* distributions, unsigned long long numberOfLBnodes, const uint32_t* geo,
                         const uint32_t* neighborX, const uint32_t* neighborY, const uint32_t* neighborZ,
                         const void* rho, const void* vx, const void* vy, const void* vz, int isEvenTimestep,
                         void* stream);

/*
 * Non-equilibrium initialisation of one parity view: the equilibrium of
 * (drho, u) plus the first-order strain-rate part built from the central
 * differences of u over the six axis neighbours (the negative ones reached
 * through neighborInverse, the -x-y-z neighbour, and two positive steps).
 * Replaces InitNavierStokesCompressibleNonEquilibrium_Device
 * (src/gpu/core/PreProcessor/PreProcessorStrategy/InitNavierStokesCompressible/InitNavierStokesCompressible_Device.cu:216-500),
 * which InitNavierStokesCompressible::init (InitNavierStokesCompressible.cu:63-83)
 * launches when Parameter::getUseInitNeq() is set.  Nodes whose geo is
 * GEO_SOLID or GEO_VOID get 96 in their rest population, as in the reference
 * (FP16 storage: its largest finite value, 96 being out of its scaled range).
 * omega in (0, 2).
 */
int vfb_init_nonequilibrium(int storage, void* distributions, unsigned long long numberOfLBnodes, const uint32_t* geo,
                            const uint32_t* neighborX, const uint32_t* neighborY, const uint32_t* neighborZ,
                            const uint32_t* neighborInverse, const void* rho, const void* vx, const void* vy,
                            const void* vz, double omega, int isEvenTimestep, void* stream);

/*
 * The enstrophy analyzer over one level's macroscopic fields (device arrays
 * of numberOfLBnodes in the compute precision: precision VFB_FP64 or
 * VFB_FP32).  Per fluid node whose six axis neighbours are fluid:
 * 1/2 (drho + 1) |curl u|^2, each axis with the widest central difference
 * (order 8, 6, 4 or 2) whose stencil stays on fluid nodes
 * (EnstrophyAnalyzer.cu:112-338, enstrophyKernel / enstrophyFunction).
 * out2[0] = the mean over those nodes (FP64 sum; the reference sums in the
 * working precision), out2[1] = their number.  Synchronises the stream.
 */
int vfb_enstrophy(int precision, const void* rho, const void* vx, const void* vy, const void* vz,
                  unsigned long long numberOfLBnodes, const uint32_t* geo, const uint32_t* neighborX,
                  const uint32_t* neighborY, const uint32_t* neighborZ, const uint32_t* neighborInverse,
                  double* out2, void* stream);

/*
 * One pass over all nodes: the fields of vfb_macroscopic (into rho/vx/vy/vz,
 * device arrays of the compute precision) and FP64 sums into the host array
 * out5 = {sum of drho, sum of (1 + drho)|u|^2/2 and the non-finite count over
 * the nodes with bit 0 of nodeMask set (the fluid list), the energy sum and
 * the count over the nodes with bit 1 set (the kinetic-energy analyzer's
 * set)}.  nodeMask: uint8 per node.  Synchronises the stream.  No reference
 * counterpart as one pass (MacroscopicQuantities.cu and
 * KineticEnergyAnalyzer.cu:66-154 in separate ones).
 */
int vfb_output_pass(int storage, const void* distributions, unsigned long long numberOfLBnodes, const uint32_t* geo,
                    const uint32_t* neighborX, const uint32_t* neighborY, const uint32_t* neighborZ,
                    const uint8_t* nodeMask, int isEvenTimestep, void* rho, void* vx, void* vy, void* vz,
                    double* out5, void* stream);

/*
 * drho and velocity of every node from the populations of the given parity
 * (pyramid sums, src/lbm/MacroscopicQuantities.h:117-127); nodes with geo
 * GEO_SOLID or GEO_VOID get zeros.  Outputs are compute-precision arrays of
 * numberOfLBnodes.  The counterpart of calculateMacroscopicQuantitiesCompressible
 * (src/gpu/core/PostProcessor/MacroscopicQuantities.cu).
 */
int vfb_macroscopic(int storage, const void* distributions, unsigned long long numberOfLBnodes, const uint32_t* geo,
                    const uint32_t* neighborX, const uint32_t* neighborY, const uint32_t* neighborZ,
                    int isEvenTimestep, void* rho, void* vx, void* vy, void* vz, void* stream);

/*
 * Global sums in FP64 over a node list: out[0] = sum of drho, out[1] = sum of
 * (drho + 1) * |u|^2 / 2, out[2] = number of non-finite nodes.  out is a HOST
 * array of 3 doubles; the call synchronises the stream.  The kinetic-energy
 * definition is that of KineticEnergyAnalyzer::run
 * (src/gpu/core/PostProcessor/KineticEnergyAnalyzer.cu:66-108) with FP64
 * accumulation instead of the reference's working-precision reduction.
 */
int vfb_mass_and_energy(int storage, const void* distributions, unsigned long long numberOfLBnodes,
                        const uint32_t* neighborX, const uint32_t* neighborY, const uint32_t* neighborZ,
                        const uint32_t* nodeIndices, uint32_t numberOfIndices, int isEvenTimestep, double* out,
                        void* stream);

/*
 * The number of stored populations at either end of the FX16 / FX16W range
 * (int16 codes 32767 and -32768) in slots 1..26 of such a population array,
 * i.e. deviations |f - w| that reached the end of the format's range (a
 * quarter of the weight for FX16) and were clipped on store.  0 for every
 * other storage (their ranges are not reached by lattice flows).  A read-only pass over the array; synchronises the stream.
 * No counterpart in the reference, which has no 16-bit storage.
 */
int vfb_saturated_populations(int storage, const void* distributions, unsigned long long numberOfLBnodes,
                              unsigned long long* count, void* stream);

/*
 * vfb_mass_and_energy without any allocation: same arguments, same sums in
 * the same order.  No counterpart in the reference.  It is for callers that
 * cannot allocate device memory where they want the sums (a host whose pool
 * allocator owns all of HBM, or a monitor inside a solver loop whose memory
 * footprint must stay fixed).  Its scratch is a fixed 24 KiB device array in
 * the library (partial sums of at most 1024 blocks), held by every GPU that
 * loads the library until exit; a launch that would need more blocks is
 * rejected with VFB_ERR_OUT_OF_RANGE.  The first call on each device looks up
 * the array's device address; make that first call before any stream
 * capture.  All calls on a device share the array, so calls that overlap on
 * the GPU (other streams, other host threads) race; the call synchronises its
 * stream before it returns.  The looked-up address belongs to the device's
 * context: after a cudaDeviceReset of that device in the same process it is
 * stale, so do not call this entry point on that device again after a reset.
 */
int vfb_mass_and_energy_static(int storage, const void* distributions, unsigned long long numberOfLBnodes,
                               const uint32_t* neighborX, const uint32_t* neighborY, const uint32_t* neighborZ,
                               const uint32_t* nodeIndices, uint32_t numberOfIndices, int isEvenTimestep,
                               double* out, void* stream);

/* Check hook of the grid builder's side q rule: the q values of a node on
 * side `side` (0..5 = MX PX MY PY MZ PZ) whose neighbours are all boundary
 * stoppers, after the sides alreadySet[0..nSet) (Side::setQs, Side.cpp:149-215). */
int vfb_debug_side_qs(int side, const int* alreadySet, int nSet, double* q27);
/*
 * One node of the K17 (op 0) or BGK (op 1) collision on the host with the
 * library's own arithmetic (the code the kernels run), for checks without a
 * GPU.  precision: VFB_FP64 or VFB_FP32; f27 in/out, out4 = drho, vx, vy, vz.
 * No counterpart in the reference.
 */
int vfb_debug_collide_node(int op, int precision, double* f27, double omega, const double* limiters,
                           const double* force, double* out4);
/*
 * The reverse sweep of one node's K17 collision on the host with the code the
 * collision adjoint kernel runs: f27 = pre-collision populations, lam27 in =
 * adjoint of the post-collision populations, out = adjoint of the
 * pre-collision populations; gforce3 = adjoint of the half force (fx, fy, fz)
 * that vfb_debug_collide_node takes.  precision: VFB_FP64 or VFB_FP32.
 * No counterpart in the reference.
 */
int vfb_debug_k17_adjoint_node(int precision, const double* f27, double* lam27, double omega, const double* limiters,
                               const double* force, double* gforce3);
/*
 * One node of the non-equilibrium initialisation on the host with the code
 * the kernel runs: drhoVelocity4 = drho, vx, vy, vz; gradient9[3a + b] =
 * d u_a / d x_b; f27 out, direction order.  precision: VFB_FP64 or VFB_FP32.
 * No counterpart in the reference.
 */
int vfb_debug_init_nonequilibrium_node(int precision, const double* drhoVelocity4, const double* gradient9,
                                       double omega, double* f27);
/*
 * The enstrophy node values on the host with the code the kernel runs
 * (host arrays of the compute precision): out[k] the value, counted[k] 1
 * where the node enters the mean.  No counterpart in the reference.
 */
int vfb_debug_enstrophy_nodes(int precision, const void* rho, const void* vx, const void* vy, const void* vz,
                              unsigned long long numberOfLBnodes, const uint32_t* geo, const uint32_t* neighborX,
                              const uint32_t* neighborY, const uint32_t* neighborZ, const uint32_t* neighborInverse,
                              double* out, int* counted);

#ifdef __cplusplus
}
#endif

#endif /* VF_B200_H */
