/*
 * rp3dg.h -- C ABI of the B200 collision-and-dynamics hot path.
 *
 * Everything here is plain C: pointers, sizes and POD structs, no C++ or torch
 * types.  The library (reactphysics3d_b200/_lib/librp3dg.so) owns all device
 * memory it allocates; callers own the buffers they pass in.
 *
 * Reference interfaces replaced (paths inside ReactPhysics3D v0.10.2):
 *   - the narrow-phase data contract NarrowPhaseInput / NarrowPhaseInfoBatch
 *       include/reactphysics3d/collision/narrowphase/NarrowPhaseInput.h:52-160
 *       include/reactphysics3d/collision/narrowphase/NarrowPhaseInfoBatch.h:48-190
 *     and the six algorithm entry points
 *       bool XxxAlgorithm::testCollision(NarrowPhaseInfoBatch&, uint32 start,
 *                                        uint32 n, [bool clipWithPrevAxis,]
 *                                        MemoryAllocator&)
 *       (SphereVsSphereAlgorithm.h:68, SphereVsCapsuleAlgorithm.h:68,
 *        CapsuleVsCapsuleAlgorithm.h:68, SphereVsConvexPolyhedronAlgorithm.h:70,
 *        CapsuleVsConvexPolyhedronAlgorithm.h:70,
 *        ConvexPolyhedronVsConvexPolyhedronAlgorithm.h:68)
 *   - the temporal-coherence cache LastFrameCollisionInfo
 *       include/reactphysics3d/engine/OverlappingPairs.h:55-93
 *   - the per-pair contact output ContactPointInfo
 *       include/reactphysics3d/collision/ContactPointInfo.h:46-64
 *
 * Return convention: 0 on success, a negative RP3DG_E* code on failure;
 * rp3dg_last_error() gives a message.  The reference reports errors by
 * assert + log only, so every failure mode here is new and explicit.
 */
#ifndef RP3DG_H
#define RP3DG_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* NB_MAX_CONTACT_POINTS_IN_NARROWPHASE_INFO, configuration.h:109 */
#define RP3DG_MAX_CONTACTS_PER_PAIR 16

/* error codes */
#define RP3DG_OK 0
#define RP3DG_EINVAL -1      /* bad argument (null pointer, unknown algorithm, bad shape) */
#define RP3DG_ECUDA -2       /* a CUDA runtime call failed */
#define RP3DG_ENOMEM -3      /* a device allocation failed */
#define RP3DG_ECAPACITY -4   /* a fixed-capacity table is full */
#define RP3DG_ENODEV -5      /* no CUDA device */

/* Collision shape kinds.  The reference's CollisionShapeType has SPHERE,
 * CAPSULE, CONVEX_POLYHEDRON, CONCAVE_SHAPE (CollisionShape.h:49); boxes and
 * convex meshes are both CONVEX_POLYHEDRON there and are told apart by
 * CollisionShapeName.  Here the concrete kind is stored directly. */
enum rp3dg_shape_kind {
    RP3DG_SHAPE_SPHERE = 0,
    RP3DG_SHAPE_CAPSULE = 1,
    RP3DG_SHAPE_BOX = 2,
    RP3DG_SHAPE_CONVEX_MESH = 3,
    RP3DG_SHAPE_HEIGHTFIELD = 4,  /* CONCAVE_SHAPE / HEIGHTFIELD */
    RP3DG_SHAPE_CONCAVE_MESH = 5  /* CONCAVE_SHAPE / TRIANGLE_MESH */
};

/* Narrow-phase algorithms, same numbering as the reference's
 * NarrowPhaseAlgorithmType (CollisionDispatch.h:42-50). */
enum rp3dg_algorithm {
    RP3DG_ALGO_NONE = 0,
    RP3DG_ALGO_SPHERE_VS_SPHERE = 1,
    RP3DG_ALGO_SPHERE_VS_CAPSULE = 2,
    RP3DG_ALGO_CAPSULE_VS_CAPSULE = 3,
    RP3DG_ALGO_SPHERE_VS_CONVEX_POLYHEDRON = 4,
    RP3DG_ALGO_CAPSULE_VS_CONVEX_POLYHEDRON = 5,
    RP3DG_ALGO_CONVEX_POLYHEDRON_VS_CONVEX_POLYHEDRON = 6
};

typedef struct rp3dg_float4 { float x, y, z, w; } rp3dg_float4;

/* One collision shape (32 bytes).
 *   sphere:       params = (radius, 0, 0, 0)
 *   capsule:      params = (radius, halfHeight, 0, 0)
 *                 (the reference stores mHalfHeight = height * 0.5,
 *                  CapsuleShape.cpp:41, and getHeight() = 2 * halfHeight)
 *   box:          params = (halfExtent.x, .y, .z, 0)
 *   convex mesh:  params unused; mesh = index returned by
 *                 rp3dg_create_convex_mesh_shape (mesh + scale instance)
 *   height field: params unused; mesh = index returned by
 *                 rp3dg_create_heightfield (a concave shape: it collides
 *                 only inside a world, through the middle phase)
 *   concave mesh: params unused; mesh = index returned by
 *                 rp3dg_create_concave_mesh_shape (concave, like a height
 *                 field) */
typedef struct rp3dg_shape {
    float params[4];
    int32_t kind;
    int32_t mesh;
    int32_t reserved[2];
} rp3dg_shape;

/* LastFrameCollisionInfo (OverlappingPairs.h:55-93) packed into 16 bytes. */
#define RP3DG_LF_IS_VALID        0x01u
#define RP3DG_LF_WAS_COLLIDING   0x02u
#define RP3DG_LF_WAS_USING_GJK   0x04u
#define RP3DG_LF_WAS_USING_SAT   0x08u
#define RP3DG_LF_SAT_FACE_POLY1  0x10u
#define RP3DG_LF_SAT_FACE_POLY2  0x20u
#define RP3DG_LF_IS_OBSOLETE     0x40u
typedef struct rp3dg_lastframe {
    float gjk_axis[3];        /* gjkSeparatingAxis, initially (0,1,0) */
    uint8_t flags;            /* RP3DG_LF_* bits */
    uint8_t sat_face;         /* satMinAxisFaceIndex */
    uint8_t sat_edge1;        /* satMinEdge1Index */
    uint8_t sat_edge2;        /* satMinEdge2Index */
} rp3dg_lastframe;

/* A batch of pairs for one algorithm, struct-of-arrays.  All pointers are
 * device pointers for rp3dg_narrowphase_device and host pointers for
 * rp3dg_narrowphase_host.  pos*.w is ignored; rot* are unit quaternions
 * stored (x, y, z, w) like the reference's Quaternion. */
typedef struct rp3dg_pair_batch {
    uint32_t n;
    const int32_t* shape1;          /* index into the context's shape table */
    const int32_t* shape2;
    const rp3dg_float4* pos1;       /* shape1ToWorldTransform position */
    const rp3dg_float4* rot1;       /* shape1ToWorldTransform orientation */
    const rp3dg_float4* pos2;
    const rp3dg_float4* rot2;
    const uint8_t* report_contacts; /* NULL: every pair reports contacts */
    rp3dg_lastframe* cache;         /* in/out; NULL: fresh (isValid=false), not written */
} rp3dg_pair_batch;

/* Per-pair results.  Contact slot k of pair i lives at index k * n + i
 * (slot-major, so that consecutive pairs write consecutive addresses).
 *   normal_depth = (world normal from shape 1 to shape 2, penetration depth)
 *   local1       = (contact point in shape-1 local space, 0)
 *   local2       = (contact point in shape-2 local space, 0)
 * Slots >= nb_contacts[i] are left untouched.  max_contacts (1..16) bounds the
 * slots the caller allocated; points beyond it are counted in nb_contacts
 * only up to max_contacts, exactly like the reference's cap of 16. */
typedef struct rp3dg_contact_batch {
    uint8_t* is_colliding;
    uint8_t* nb_contacts;
    rp3dg_float4* normal_depth;
    rp3dg_float4* local1;
    rp3dg_float4* local2;
    uint32_t max_contacts;
} rp3dg_contact_batch;

typedef struct rp3dg_ctx rp3dg_ctx;

/* ---- context ---------------------------------------------------------- */

/* Create a context on CUDA device `device` with its own stream.
 * Replaces the PhysicsCommon + world memory managers (MemoryManager.h:72). */
int rp3dg_create(int device, rp3dg_ctx** out);
void rp3dg_destroy(rp3dg_ctx* ctx);
const char* rp3dg_last_error(const rp3dg_ctx* ctx);
/* cudaStream_t of the context, as void* (for callers that order work). */
void* rp3dg_stream(rp3dg_ctx* ctx);
int rp3dg_synchronize(rp3dg_ctx* ctx);

/* ---- shapes (immutable after creation) -------------------------------- */

/* Convex mesh from polygon faces: replaces
 * PhysicsCommon::createConvexMesh(const PolygonVertexArray&, ...)
 * (PhysicsCommon.h:214; ConvexMesh::init ConvexMesh.cpp:47-79).  Builds the
 * half-edge structure (HalfEdgeStructure.cpp:34-127), Newell face normals
 * (ConvexMesh.cpp:217-240) and the centroid (ConvexMesh.cpp:83-108) on the
 * host.  vertices: nb_vertices * 3 floats; faces: face_sizes[f] indices each,
 * concatenated in face_indices.  Returns the mesh id in *mesh_id. */
int rp3dg_create_convex_mesh(rp3dg_ctx* ctx, const float* vertices, uint32_t nb_vertices,
                             const uint32_t* face_indices, const uint32_t* face_sizes,
                             uint32_t nb_faces, int32_t* mesh_id);

/* Convex mesh shape = mesh + scale: replaces
 * PhysicsCommon::createConvexMeshShape(ConvexMesh*, const Vector3& scaling)
 * (PhysicsCommon.h:196; scaled normals ConvexMeshShape.cpp:50-70).
 * Returns the instance id to store in rp3dg_shape.mesh. */
int rp3dg_create_convex_mesh_shape(rp3dg_ctx* ctx, int32_t mesh_id, float sx, float sy, float sz,
                                   int32_t* instance_id);

/* Read back the tables built for a mesh instance (for parity checks):
 * half-edges as 4 uint32 (vertexIndex, twinEdgeIndex, faceIndex,
 * nextEdgeIndex), face normals (3 floats), face first edge, centroid. */
int rp3dg_get_convex_mesh_tables(rp3dg_ctx* ctx, int32_t instance_id,
                                 uint32_t* nb_vertices, uint32_t* nb_faces, uint32_t* nb_half_edges,
                                 uint32_t* half_edges, float* face_normals, uint32_t* face_edge,
                                 float* centroid, uint32_t capacity_half_edges, uint32_t capacity_faces);

/* Height field + height-field shape: replaces
 * PhysicsCommon::createHeightField(nbGridColumns, nbGridRows, data,
 * HeightDataType::HEIGHT_FLOAT_TYPE, messages) (HeightField::init,
 * HeightField.cpp:47-90) followed by PhysicsCommon::createHeightFieldShape(
 * heightField, scaling) (HeightFieldShape.cpp:40-43).  heights holds
 * nb_columns * nb_rows floats, heights[y * nb_columns + x]; grid column x lies
 * along local X, row y along local Z, one unit apart before scaling, and the
 * local bounds are centred on the origin.  nb_columns and nb_rows must be at
 * least 2 (the reference's init fails otherwise).  Returns the id to store in
 * rp3dg_shape.mesh with kind RP3DG_SHAPE_HEIGHTFIELD. */
int rp3dg_create_heightfield(rp3dg_ctx* ctx, uint32_t nb_columns, uint32_t nb_rows, const float* heights,
                             float sx, float sy, float sz, int32_t* heightfield_id);

/* Triangle mesh: replaces PhysicsCommon::createTriangleMesh(
 * TriangleVertexArray(nb_vertices, vertices, 12, nb_triangles, indices, 12,
 * VERTEX_FLOAT_TYPE, INDEX_INTEGER_TYPE[, normals, 12, NORMAL_FLOAT_TYPE]),
 * messages) (TriangleMesh::init, TriangleMesh.cpp:42-67): triangles of
 * almost zero area or with an almost zero edge dropped, unused vertices
 * removed (:91-240), angle-weighted vertex normals when `normals` is NULL
 * (:277-333), and the DynamicAABBTree of the triangles built on the host by
 * inserting them in order (:242-266).  vertices: nb_vertices * 3 floats;
 * indices: 3 per triangle.  RP3DG_EINVAL where the reference's mesh is
 * invalid (an index out of range, no triangle left, a normal too short). */
int rp3dg_create_triangle_mesh(rp3dg_ctx* ctx, const float* vertices, uint32_t nb_vertices, const uint32_t* indices,
                               uint32_t nb_triangles, const float* normals, int32_t* mesh_id);
/* Concave mesh shape = triangle mesh + scale: replaces
 * PhysicsCommon::createConcaveMeshShape(TriangleMesh*, const Vector3& scaling)
 * (scaled vertex normals ConcaveMeshShape.cpp:56-76).  Returns the instance
 * id to store in rp3dg_shape.mesh with kind RP3DG_SHAPE_CONCAVE_MESH. */
int rp3dg_create_concave_mesh_shape(rp3dg_ctx* ctx, int32_t mesh_id, float sx, float sy, float sz,
                                    int32_t* instance_id);
/* Read back a triangle mesh as built (for parity checks): its vertices and
 * vertex normals (3 floats each) and triangles (3 indices), up to the
 * capacities; the counts are always written. */
int rp3dg_get_triangle_mesh(rp3dg_ctx* ctx, int32_t mesh_id, uint32_t* nb_vertices, uint32_t* nb_triangles,
                            float* vertices, float* normals, uint32_t* triangles, uint32_t capacity_vertices,
                            uint32_t capacity_triangles);

/* Replace the context's shape table (device copy of `shapes`). */
int rp3dg_set_shapes(rp3dg_ctx* ctx, const rp3dg_shape* shapes, uint32_t nb_shapes);

/* ---- narrow phase ----------------------------------------------------- */

/* Run one algorithm over a batch whose arrays are already in device memory,
 * asynchronously on the context stream.  clip_with_previous_axis mirrors the
 * clipWithPreviousAxisIfStillColliding argument (true in
 * CollisionDetectionSystem::computeNarrowPhase, false for world queries). */
int rp3dg_narrowphase_device(rp3dg_ctx* ctx, int algorithm, const rp3dg_pair_batch* pairs,
                             const rp3dg_contact_batch* out, int clip_with_previous_axis);

/* Same, with every array in host memory: uploads the batch, runs it, copies
 * the results back and synchronizes.  This is the call a CPU-side engine
 * would make in place of XxxAlgorithm::testCollision.  Only the contact slots
 * some pair of the batch uses are copied back; slot k >= nb_contacts[i] of
 * pair i holds unspecified values afterwards.  Pinned host buffers make the
 * copies asynchronous DMA transfers. */
int rp3dg_narrowphase_host(rp3dg_ctx* ctx, int algorithm, const rp3dg_pair_batch* pairs,
                           const rp3dg_contact_batch* out, int clip_with_previous_axis);

/* The whole narrow phase of a step on host arrays: replaces
 * CollisionDetectionSystem::testNarrowPhaseCollision(NarrowPhaseInput&)
 * (CollisionDetectionSystem.cpp:618-660), which runs the batches of a
 * NarrowPhaseInput (NarrowPhaseInput.h:52-160) one algorithm after the
 * other.  Batch b (algorithms[b], pairs[b], outs[b]) gives the results of
 * rp3dg_narrowphase_host on it; the batches overlap on the device: the
 * upload of one batch runs during the kernels of the one before, and each
 * batch's results go back while the next one computes.  The device packs a
 * batch's contacts densely (no gaps for pairs without contacts), the packed
 * records and the flags and counts come back as plain copies, and the host
 * threads write the contact slots k < nb_contacts[i] of the caller's arrays
 * (the other slots are left untouched), so the outputs may be in pageable
 * or page-locked memory.  Synchronizes before returning. */
int rp3dg_narrowphase_input_host(rp3dg_ctx* ctx, uint32_t nb_batches, const int32_t* algorithms,
                                 const rp3dg_pair_batch* pairs, const rp3dg_contact_batch* outs,
                                 int clip_with_previous_axis);

/* Measurement entry point, no counterpart in the reference engine: runs
 * the same batch as rp3dg_narrowphase_device through the event-counting
 * build of the kernels (same results, slower) and returns, in events[0..
 * RP3DG_NP_EVENTS-1], how many times the pairs' code paths executed each
 * step of the reference's algorithms: 0 polyhedron-pair transforms, 1 face
 * test, 2 box support, 3 convex-mesh support vertex, 4 triangle support,
 * 5 capsule support, 6 polyhedron-1 edge, 7 Gauss-map test, 8 edge distance,
 * 9 face-clipping set-up, 10 anti-parallel face candidate, 11 incident
 * vertex, 12 clipping plane, 13 clipped input vertex, 14 plane-segment
 * intersection, 15 clipped-vertex depth, 16 face contact, 17 edge contact,
 * 18 GJK set-up, 19 GJK iteration, 20-22 simplex closest point (2, 3, 4
 * points), 23 GJK contact, 24 SAT sphere face, 25 SAT sphere contact,
 * 26 SAT capsule face, 27 SAT capsule edge, 28 capsule edge axis, 29 capsule
 * clipping plane, 30 closed-form pair test, 31 closed-form contact,
 * 32 in-margin capsule face, 33 triangle smooth normal; 34-39 zero.
 * Learned proposals are not used.  Synchronizes the context stream. */
#define RP3DG_NP_EVENTS 40
int rp3dg_narrowphase_count_events(rp3dg_ctx* ctx, int algorithm, const rp3dg_pair_batch* pairs,
                                   const rp3dg_contact_batch* out, int clip_with_previous_axis,
                                   unsigned long long* events);

/* Measurement entry point, no counterpart in the reference engine: FP32
 * throughput of the device in operations per second, measured with a
 * microkernel of independent chains timed with CUDA events (best of five
 * launches after a warm-up).  fused = 0: separate multiplies and adds
 * (round-to-nearest intrinsics, the arithmetic the narrow-phase kernels are
 * compiled to: no contraction); fused = 1: fused multiply-adds counted as two
 * operations.  Touches no clock or power setting. */
int rp3dg_measure_fp32_peak(int device, int fused, double* ops_per_second);

/* Device-side error bits accumulated by the kernels since the last clear
 * (bit 0: a pair or collider named a shape outside the shape table; such
 * pairs are reported as not colliding; bit 1: a GJK run hit the
 * 1024-iteration safety bound; bit 2: a dynamics-stage index or range was
 * out of bounds and that manifold, island or collider was skipped; bit 3: a
 * broad-phase group id was not below nb_groups).  Synchronizes the context
 * stream. */
int rp3dg_device_errors(rp3dg_ctx* ctx, uint32_t* flags, int clear);

/* ---- learned separating-axis proposal ----------------------------------
 * No counterpart in the reference engine.  A 24 -> 64 -> 64 -> 16 MLP (bf16
 * weights, fp32 accumulation) proposes a separating feature for convex
 * polyhedron pairs: 0..2 a face of polyhedron 1 along local x/y/z, 3..5 a face
 * of polyhedron 2 along x/y/z, 6..14 an edge pair (axis of 1 * 3 + axis of
 * 2, box-box only), 15 none.  When enabled, the convex-polyhedron narrow
 * phase tests the proposal with the reference's exact SAT test before its
 * full SAT and skips the full SAT when the proposal separates the shapes; the
 * contacts are unchanged, the cached separating feature may differ.
 * RP3DG_MLP_NPARAMS fp32 parameters: w1[24][64] b1[64] w2[64][64] b2[64]
 * w3[64][16] b3[16]. */
#define RP3DG_MLP_NPARAMS 6800
#define RP3DG_MLP_FEATURES 24
#define RP3DG_MLP_CLASSES 16

/* He-uniform initialisation from a seed; clears the Adam state. */
int rp3dg_axis_mlp_init(rp3dg_ctx* ctx, uint64_t seed);
int rp3dg_axis_mlp_get_params(rp3dg_ctx* ctx, float* params);
int rp3dg_axis_mlp_set_params(rp3dg_ctx* ctx, const float* params);
/* Features (n x 24 floats, device) of a device pair batch of polyhedron pairs. */
int rp3dg_axis_features(rp3dg_ctx* ctx, const rp3dg_pair_batch* pairs, float* features);
/* Class labels (device) of a device pair batch from the outcome of a fresh
 * full-SAT narrow phase (its is_colliding output and the cache it wrote). */
int rp3dg_axis_labels(rp3dg_ctx* ctx, const rp3dg_pair_batch* pairs, const uint8_t* is_colliding, uint8_t* labels);
/* Gradients (device, RP3DG_MLP_NPARAMS floats) of the mean softmax
 * cross-entropy over n device samples; *loss (host, may be NULL) receives it. */
int rp3dg_axis_mlp_grads(rp3dg_ctx* ctx, const float* features, const uint8_t* labels, uint32_t n, float* grads,
                         float* loss);
/* rp3dg_axis_mlp_grads without allocating device memory.  No counterpart in
 * the reference engine.  For callers that must not allocate once they run: a
 * host application that gives the engine a fixed GPU memory budget at
 * start-up and forbids later cudaMalloc calls (an allocation can stall the
 * whole device and can fail once the budget is spent), whereas
 * rp3dg_axis_mlp_grads grows its scratch with cudaMalloc for larger batches.
 * The scratch here is a fixed array inside the library (4.4 MB, held by every
 * GPU that loads the library until exit): n is limited to 4096 samples
 * (RP3DG_ECAPACITY beyond).  All calls share the array and it keeps the last
 * call's contents; calls that overlap on the GPU race.  The first call on a
 * device looks up the array's device address; make it before any stream
 * capture.  Same outputs as rp3dg_axis_mlp_grads. */
int rp3dg_axis_mlp_grads_noalloc(rp3dg_ctx* ctx, const float* features, const uint8_t* labels, uint32_t n,
                                 float* grads, float* loss);
/* One Adam step (lr, betas 0.9/0.999, eps 1e-8) on n device samples. */
int rp3dg_axis_mlp_train_step(rp3dg_ctx* ctx, const float* features, const uint8_t* labels, uint32_t n, float lr,
                              float* loss);
/* Tensor-core inference: classes (device) of n device feature rows. */
int rp3dg_axis_mlp_predict(rp3dg_ctx* ctx, const float* features, uint32_t n, uint8_t* classes);
/* Use the proposal in the convex-polyhedron narrow phase (0 = off, default). */
int rp3dg_set_learned_axis(rp3dg_ctx* ctx, int enable);
/* Proposals tested and confirmed since the last clear (synchronizes). */
int rp3dg_learned_axis_stats(rp3dg_ctx* ctx, uint64_t* tested, uint64_t* confirmed, int clear);

/* ---- contact manifolds ------------------------------------------------ */

/* Manifold of every colliding convex pair, as the reference builds it after
 * the narrow phase: all points of the pair in one manifold
 * (CollisionDetectionSystem::processPotentialContacts,
 * CollisionDetectionSystem.cpp:1198-1391), reduced to at most 4 points when it
 * has more (reduceContactPoints, :1483-1662, using the shape-1 orientation
 * rot1 of the batch) and de-duplicated (points closer than 0.01,
 * removeDuplicatedContactPointsInManifold, :1673-1705).  Device arrays, in
 * place: the kept points move to slots 0..k-1 in manifold order and
 * nb_contacts becomes k; kept (n x 4, may be NULL) receives the original slot
 * of each kept point (255 = none).  When pairs->cache is not NULL the step
 * also updates the temporal-coherence records as the reference does before
 * the next frame (processPotentialContacts with updateLastFrameInfo,
 * :1209-1217): IS_VALID set, WAS_COLLIDING = is_colliding.  Only rot1 and
 * cache of the pair batch are read.  Asynchronous on the context stream. */
int rp3dg_reduce_contacts_device(rp3dg_ctx* ctx, const rp3dg_pair_batch* pairs, const rp3dg_contact_batch* contacts,
                                 uint8_t* kept);

/* rp3dg_narrowphase_host followed on the device by rp3dg_reduce_contacts_device:
 * the per-algorithm narrow phase and the convex manifold step of
 * CollisionDetectionSystem (:1198-1458) in one call on host arrays; only the
 * (at most 4) kept slots are copied back.  kept (host, n x 4) may be NULL. */
int rp3dg_narrowphase_manifolds_host(rp3dg_ctx* ctx, int algorithm, const rp3dg_pair_batch* pairs,
                                     const rp3dg_contact_batch* out, int clip_with_previous_axis, uint8_t* kept);

/* ---- dynamics stage of a world step ------------------------------------ */

/* The part of PhysicsWorld::update (src/engine/PhysicsWorld.cpp:239-307) that
 * runs after the contacts are created:
 *   updateBodiesInverseWorldInertiaTensors (:310-318,
 *     RigidBody::computeWorldInertiaTensorInverse, RigidBody.h:246-262),
 *   DynamicsSystem::integrateRigidBodiesVelocities (DynamicsSystem.cpp:117-183),
 *   ContactSolverSystem::init / initializeForIsland / warmStart / solve x
 *     iterations / storeImpulses (ContactSolverSystem.cpp:66-818),
 *   DynamicsSystem::integrateRigidBodiesPositions and updateBodiesState
 *     (DynamicsSystem.cpp:44-110),
 * bit-identical to the reference's float build for worlds without joints.
 *
 * Bodies follow the reference's rigid-body component order: the first
 * n_enabled are integrated; the others (static and sleeping bodies) are only
 * read, through their velocities and world inverse inertia.  Islands are
 * ranges of the manifold array (which is in the solver's order: islands in
 * order); manifolds of different islands may share only bodies with zero
 * inverse mass and zero inverse inertia (static or kinematic), which the
 * solver never moves, so islands are solved in parallel.  The solver does not
 * write the velocities of such bodies (the reference adds signed zeros to
 * them, which can only turn a -0 component into +0). */
typedef struct rp3dg_bodies {
    uint32_t n;                          /* bodies */
    uint32_t n_enabled;                  /* bodies [0, n_enabled) are integrated */
    rp3dg_float4* position;              /* in/out: transform position (xyz) */
    rp3dg_float4* orientation;           /* in/out: transform orientation (x, y, z, w) */
    rp3dg_float4* com_world;             /* in/out: centre of mass, world frame */
    const rp3dg_float4* com_local;       /* centre of mass, body frame */
    rp3dg_float4* linear_velocity;       /* in/out */
    rp3dg_float4* angular_velocity;      /* in/out */
    const rp3dg_float4* force;           /* external force, world frame */
    const rp3dg_float4* torque;          /* external torque, world frame */
    const rp3dg_float4* inv_inertia_local; /* diagonal of the local inverse inertia tensor */
    rp3dg_float4* inv_inertia_world;     /* in/out: 3 rows per body (row r of body i at 3*i+r);
                                            written for enabled bodies, read for the others */
    const rp3dg_float4* mass;            /* x mass, y inverse mass, z linear damping, w angular damping */
    const rp3dg_float4* linear_lock;     /* linear lock-axis factors */
    const rp3dg_float4* angular_lock;    /* angular lock-axis factors */
    const uint8_t* gravity;              /* 1 = gravity applies to the body */
} rp3dg_bodies;

typedef struct rp3dg_colliders {
    uint32_t n;                          /* colliders, component order */
    uint32_t n_enabled;                  /* colliders [0, n_enabled) get new world transforms */
    const int32_t* body;                 /* body index of each collider */
    const rp3dg_float4* local_position;  /* local-to-body transform */
    const rp3dg_float4* local_orientation;
    rp3dg_float4* world_position;        /* in/out: local-to-world transform */
    rp3dg_float4* world_orientation;
    const rp3dg_float4* material;        /* x sqrt(friction coefficient) (Material::mFrictionCoefficientSqrt),
                                            y bounciness */
} rp3dg_colliders;

typedef struct rp3dg_manifolds {
    uint32_t n;                          /* contact manifolds, solver order */
    const int32_t* ids;                  /* 4 per manifold: body1, body2, collider1, collider2 */
    const uint32_t* point_start;         /* first contact point of the manifold */
    const uint8_t* nb_points;            /* 1..4 */
    rp3dg_float4* friction_vector1;      /* in/out (warm start / stored) */
    rp3dg_float4* friction_vector2;      /* in/out */
    rp3dg_float4* friction_impulse;      /* in/out: x friction 1, y friction 2, z twist */
} rp3dg_manifolds;

typedef struct rp3dg_points {
    uint32_t n;
    const rp3dg_float4* normal_depth;    /* world normal (body 1 -> body 2), penetration depth */
    const rp3dg_float4* local1;          /* contact point, collider-1 frame */
    const rp3dg_float4* local2;          /* contact point, collider-2 frame */
    float* penetration_impulse;          /* in/out */
    uint8_t* is_resting;                 /* in/out (1 after the step, as the reference sets it) */
} rp3dg_points;

typedef struct rp3dg_islands {
    uint32_t n;
    const uint32_t* manifold_start;      /* each island is manifolds [start, start + count) */
    const uint32_t* manifold_count;
} rp3dg_islands;

typedef struct rp3dg_dynamics_params {
    float dt;
    float gravity[3];                    /* world gravity (WorldSettings::gravity) */
    int32_t gravity_enabled;             /* PhysicsWorld::isGravityEnabled */
    int32_t velocity_iterations;         /* WorldSettings::defaultVelocitySolverNbIterations (6) */
    int32_t split_impulse;               /* ContactSolverSystem::isSplitImpulseActive (1) */
    float restitution_velocity_threshold; /* WorldSettings::restitutionVelocityThreshold (0.5) */
} rp3dg_dynamics_params;

/* One dynamics stage on device arrays (asynchronous on the context stream). */
int rp3dg_dynamics_step_device(rp3dg_ctx* ctx, const rp3dg_dynamics_params* params, const rp3dg_bodies* bodies,
                               const rp3dg_colliders* colliders, const rp3dg_manifolds* manifolds,
                               const rp3dg_points* points, const rp3dg_islands* islands);
/* The same on host arrays (copied in and out, synchronous). */
int rp3dg_dynamics_step_host(rp3dg_ctx* ctx, const rp3dg_dynamics_params* params, const rp3dg_bodies* bodies,
                             const rp3dg_colliders* colliders, const rp3dg_manifolds* manifolds,
                             const rp3dg_points* points, const rp3dg_islands* islands);

/* ---- broad phase ------------------------------------------------------ */

/* Colliders in the broad phase.  rp3dg_broadphase_update_device restates
 * BroadPhaseSystem::updateCollidersComponents (src/systems/BroadPhaseSystem.cpp:
 * 155-185): the world AABB of each collider from its shape
 * (CollisionShape::computeTransformedAABB, CollisionShape.cpp:54-90; spheres
 * SphereShape.cpp:49-58) and the fat-AABB update of
 * DynamicAABBTree::updateObject (DynamicAABBTree.cpp:186-214: kept while it
 * contains the new AABB, else the new AABB grown by 4% of its extent per
 * side), bit-identical.  rp3dg_broadphase_pairs_device returns the set the
 * reference's overlapping pairs hold after its broad phase
 * (CollisionDetectionSystem::computeBroadPhase / updateOverlappingPairs /
 * removeNonOverlappingPairs, CollisionDetectionSystem.cpp:103-343): every
 * pair of colliders of different bodies in the same group whose fat AABBs
 * overlap (AABB::testCollision, inclusive) and whose category / mask bits
 * accept each other, as (lower, higher) collider index.  The reference's
 * no-collision body pairs (joints with collision disabled) are not applied.
 * The order of the pairs is deterministic but is not the reference's (which
 * follows its tree).  The search is a linear BVH (axis RP3DG_BROADPHASE_LBVH:
 * Morton-sorted fat-AABB centres, group in the high key bits, Karras tree,
 * bottom-up refit, warp-cooperative traversal) or a sort and sweep along
 * axis 0, 1 or 2; both return the same set. */
#define RP3DG_BROADPHASE_LBVH (-1)
typedef struct rp3dg_broadphase {
    uint32_t n;                           /* colliders in the broad phase */
    uint32_t n_update;                    /* colliders [0, n_update) get new AABBs (the enabled ones) */
    uint32_t nb_groups;                   /* worlds; 0 or 1 = one world (group may be NULL) */
    const int32_t* shape;                 /* shape-table index of each collider */
    const int32_t* body;                  /* body of each collider */
    const int32_t* group;                 /* world of each collider, 0..nb_groups-1, or NULL */
    const uint16_t* category;             /* collision category bits, or NULL (0xffff) */
    const uint16_t* mask;                 /* collide-with mask bits, or NULL (0xffff) */
    const rp3dg_float4* world_position;   /* local-to-world transform of each collider */
    const rp3dg_float4* world_orientation;
    const uint8_t* force_reinsert;        /* the shape changed size, or NULL */
    rp3dg_float4* fat_min;                /* in/out: fat AABB of each collider */
    rp3dg_float4* fat_max;
    uint8_t* moved;                       /* out, n_update: 1 = reinserted (BroadPhaseSystem::mMovedShapes) */
} rp3dg_broadphase;

int rp3dg_broadphase_update_device(rp3dg_ctx* ctx, const rp3dg_broadphase* bp);
/* Pairs on device arrays: pairs (2 x capacity int32) receives up to capacity
 * pairs; *count (device) the number found (may exceed capacity).  axis:
 * RP3DG_BROADPHASE_LBVH (-1) for the LBVH, 0, 1 or 2 for the sweep axis.
 * Device error bit 4 is set if an LBVH traversal ran out of stack (not
 * reachable: the tree of 96-bit keys is at most 96 levels deep). */
int rp3dg_broadphase_pairs_device(rp3dg_ctx* ctx, const rp3dg_broadphase* bp, int axis, int32_t* pairs,
                                  uint32_t capacity, uint32_t* count);
/* The same on host arrays (fat_min, fat_max, body, group, category, mask);
 * *count is written on the host.  Synchronous. */
int rp3dg_broadphase_pairs_host(rp3dg_ctx* ctx, const rp3dg_broadphase* bp, int axis, int32_t* pairs,
                                uint32_t capacity, uint32_t* count);

/* ---- world step --------------------------------------------------------
 * A physics world stepped like PhysicsWorld::update(decimal timeStep)
 * (include/reactphysics3d/engine/PhysicsWorld.h:352, body
 * src/engine/PhysicsWorld.cpp:239-307).  The floating-point work of a step
 * runs on the GPU (world AABBs and the fat-AABB test of the broad phase, the
 * narrow phase, the manifold step, warm starting, inertia, velocity
 * integration, the contact solver, position integration); the host keeps the
 * order-defining bookkeeping of the reference (its dynamic AABB tree topology,
 * the moved-collider set, the persistent overlapping-pair arrays, contact-pair
 * order, islands, component order and sleeping) so that every step processes
 * pairs, contacts and constraints in the reference's own order and the results
 * are the reference float build's, bit for bit.  Worlds with convex
 * colliders (sphere, capsule, box, convex mesh) and height fields, simulation
 * colliders only (no triggers), with ball-and-socket, hinge, fixed and slider
 * joints, are supported.
 *
 * rp3dg_world_create mirrors this sequence of reference calls, body by body:
 *   b = world->createRigidBody(Transform(position, orientation));
 *   for each collider c of the body, in order:
 *       c = b->addCollider(shape, Transform(local position, local orientation));
 *       c->getMaterial().setFrictionCoefficient / setBounciness / setMassDensity;
 *       c->setCollisionCategoryBits(category); c->setCollideWithMaskBits(mask);
 *   if (type == DYNAMIC) b->updateMassPropertiesFromColliders(); else b->setType(type);
 *   b->setLinearDamping; setAngularDamping; setLinearLockAxisFactor;
 *   setAngularLockAxisFactor; enableGravity; setIsAllowedToSleep;
 *   if (type != STATIC) { b->setLinearVelocity; b->setAngularVelocity; }
 * Colliders are given grouped by body, bodies in ascending order. */
#define RP3DG_BODY_STATIC 0     /* BodyType::STATIC (RigidBody.h) */
#define RP3DG_BODY_KINEMATIC 1
#define RP3DG_BODY_DYNAMIC 2

typedef struct rp3dg_world_settings {      /* PhysicsWorld::WorldSettings (PhysicsWorld.h:80-140) */
    float gravity[3];                       /* (0, -9.81, 0) */
    int32_t velocity_iterations;            /* defaultVelocitySolverNbIterations, 6 */
    int32_t sleeping_enabled;               /* isSleepingEnabled, 1 */
    float sleep_linear_velocity;            /* defaultSleepLinearVelocity, 0.02 */
    float sleep_angular_velocity;           /* defaultSleepAngularVelocity, 3 degrees/s in rad/s */
    float time_before_sleep;                /* defaultTimeBeforeSleep, 1 */
    float restitution_velocity_threshold;   /* 0.5 */
    float persistent_contact_distance_threshold; /* 0.03 */
    float cos_angle_similar_contact_manifold;    /* 0.95 */
    int32_t position_iterations;            /* defaultPositionSolverNbIterations, 3 (joints) */
} rp3dg_world_settings;

typedef struct rp3dg_body_desc {
    int32_t type;                  /* RP3DG_BODY_* */
    float position[3];
    float orientation[4];          /* unit quaternion (x, y, z, w) */
    float linear_velocity[3];
    float angular_velocity[3];
    float linear_damping;
    float angular_damping;
    float linear_lock[3];          /* lock-axis factors, (1, 1, 1) = free */
    float angular_lock[3];
    int32_t gravity_enabled;
    int32_t allowed_to_sleep;
} rp3dg_body_desc;

typedef struct rp3dg_collider_desc {
    int32_t body;                  /* body index */
    int32_t shape;                 /* index into the context's shape table */
    float position[3];             /* local-to-body transform */
    float orientation[4];
    float friction;                /* Material::setFrictionCoefficient */
    float bounciness;              /* Material::setBounciness */
    float mass_density;            /* Material::setMassDensity */
    uint16_t category;             /* collision category bits (0x0001 by default) */
    uint16_t mask;                 /* collide-with mask bits (0xffff by default) */
    uint32_t flags;                /* RP3DG_COLLIDER_TRIGGER: Collider::setIsTrigger(true) after creation */
} rp3dg_collider_desc;
/* A trigger collider (Collider::setIsTrigger, Collider.cpp:250-257) is not a
 * simulation collider: its pairs are tested without contact points, a
 * colliding one becomes a contact pair that no island takes, and the world
 * reports it through rp3dg_world_get_trigger_events instead of the contact
 * events.  It still counts for the body's mass properties. */
#define RP3DG_COLLIDER_TRIGGER 1u

/* A joint, as PhysicsWorld::createJoint(JointInfo) (PhysicsWorld.cpp:467-580)
 * creates it from a BallAndSocketJointInfo / HingeJointInfo / FixedJointInfo /
 * SliderJointInfo with a world-space anchor (and hinge or slider axis),
 * followed for a ball-and-socket joint with a cone limit by
 * joint->enableConeLimit(true) and joint->setConeLimitHalfAngle(angle).  Only
 * the NON_LINEAR_GAUSS_SEIDEL position correction (the default) is built.
 * The hinge and slider joints share the limit and motor fields: angles in
 * radians and a torque for a hinge, translations along the axis and a force
 * for a slider (minTranslationLimit, maxTranslationLimit, maxMotorForce). */
#define RP3DG_JOINT_BALL_AND_SOCKET 0
#define RP3DG_JOINT_HINGE 1
#define RP3DG_JOINT_FIXED 2
#define RP3DG_JOINT_SLIDER 3
typedef struct rp3dg_joint_desc {
    int32_t type;                  /* RP3DG_JOINT_* */
    int32_t body1, body2;          /* body indices of the world */
    float anchor[3];               /* anchor point, world space, at creation */
    float axis[3];                 /* hinge: rotation axis; slider: sliding axis; world space */
    int32_t collision_enabled;     /* JointInfo::isCollisionEnabled (0: the two bodies never collide) */
    int32_t cone_limit_enabled;    /* ball-and-socket */
    float cone_half_angle;         /* ball-and-socket, radians (PI by default) */
    int32_t limit_enabled;         /* hinge, slider */
    float min_angle, max_angle;    /* hinge: angle limits, radians; slider: translation limits (-1, 1 when disabled, the reference's defaults) */
    int32_t motor_enabled;         /* hinge, slider */
    float motor_speed, max_motor_torque;  /* hinge: rad/s, N m; slider: m/s, N (maxMotorForce) */
} rp3dg_joint_desc;

typedef struct rp3dg_world rp3dg_world;

typedef struct rp3dg_world_stats {
    uint32_t overlapping_pairs;    /* enabled overlapping pairs (convex and convex vs concave) after the broad phase */
    uint32_t disabled_pairs;       /* pairs of two sleeping / static bodies */
    uint32_t narrowphase_tests;    /* narrow-phase tests this step (pairs and height-field triangles) */
    uint32_t contact_pairs;        /* colliding pairs */
    uint32_t manifolds;            /* contact manifolds given to the solver */
    uint32_t contact_points;
    uint32_t islands;
    uint32_t enabled_bodies;       /* awake non-static bodies after the step */
    uint32_t moved_colliders;      /* colliders reinserted in the broad-phase tree by the step */
    uint32_t reserved;
} rp3dg_world_stats;

/* Build a world on ctx's device (the shape table must be set).  The world
 * keeps pointers to nothing the caller owns. */
int rp3dg_world_create(rp3dg_ctx* ctx, const rp3dg_world_settings* settings, const rp3dg_body_desc* bodies,
                       uint32_t nb_bodies, const rp3dg_collider_desc* colliders, uint32_t nb_colliders,
                       rp3dg_world** out);
void rp3dg_world_destroy(rp3dg_world* world);
/* createJoint for each of the n joints, in order; before the first update.
 * The joints are solved in islands with their bodies, warm-started, with
 * the reference's velocity solve and non-linear Gauss-Seidel position
 * correction (SolveBallAndSocketJointSystem.cpp, SolveFixedJointSystem.cpp,
 * SolveHingeJointSystem.cpp, SolveSliderJointSystem.cpp). */
int rp3dg_world_add_joints(rp3dg_world* world, const rp3dg_joint_desc* joints, uint32_t n);
/* HingeJoint::setMotorSpeed / SliderJoint::setMotorSpeed (HingeJoint.cpp:168,
 * SliderJoint.cpp:210) between updates, on joint `joint` (index in the order
 * the joints were added) of world `world` (0 for rp3dg_world_create, the
 * group index otherwise): a changed speed wakes the joint's two bodies.
 * RP3DG_EINVAL for a ball-and-socket or fixed joint. */
int rp3dg_world_set_motor_speed(rp3dg_world* world, uint32_t world_index, uint32_t joint, float speed);
/* PhysicsWorld::update(dt): one step (synchronous). */
int rp3dg_world_update(rp3dg_world* world, float dt);
/* Body state in creation order (host arrays of nb_bodies rows, any may be
 * NULL): position (x, y, z), orientation (x, y, z, w), linear and angular
 * velocity (x, y, z), sleeping flag. */
int rp3dg_world_get_bodies(rp3dg_world* world, float* position, float* orientation, float* linear_velocity,
                           float* angular_velocity, uint8_t* sleeping);
/* Overlapping-pair ids (pairNumbers of the two broad-phase ids,
 * mathematics_functions.h:428-433) in the reference's array order: enabled
 * convex pairs (OverlappingPairs::mConvexPairs), disabled ones
 * (mDisabledConvexPairs), then the convex vs concave pairs (mConcavePairs,
 * mDisabledConcavePairs).  *n receives the total; at most capacity are
 * written. */
int rp3dg_world_get_pairs(rp3dg_world* world, uint64_t* pair_ids, uint32_t capacity, uint32_t* n);
/* Contact manifolds of the last step in the solver's order: per manifold the
 * creation indices of body 1 and body 2 and the number of points (host
 * arrays, capacity rows); per point (capacity_points rows, may be NULL)
 * normal + penetration depth and the two local points as float4. */
int rp3dg_world_get_contacts(rp3dg_world* world, int32_t* body1, int32_t* body2, uint8_t* nb_points,
                             uint32_t capacity, float* normal_depth, float* local1, float* local2,
                             uint32_t capacity_points, uint32_t* nb_manifolds, uint32_t* nb_contact_points);
int rp3dg_world_get_stats(rp3dg_world* world, rp3dg_world_stats* stats);

/* Contact solver of the world step.  RP3DG_SOLVER_EXACT (the default) is the
 * drop-in: ContactSolverSystem::solve (ContactSolverSystem.cpp:479-759) in
 * the reference's constraint order, bit-identical.  RP3DG_SOLVER_GRAPH_COLORED
 * has no counterpart in the reference and is not a drop-in: the manifolds'
 * conflict graph (manifolds sharing a movable body) is coloured on the GPU
 * and every pass runs colour after colour, the manifolds of a colour in
 * parallel, with the reference's per-manifold arithmetic; the order differs,
 * so the results do (worlds with joints keep the exact solver).  With stats,
 * each step records the velocity constraint residual over the contact points
 * after the last iteration and the bodies' energies after the step. */
#define RP3DG_SOLVER_EXACT 0
#define RP3DG_SOLVER_GRAPH_COLORED 1
typedef struct rp3dg_solver_stats {
    double residual_rms;      /* over the contact points: |n.dv| where the impulse is positive, else max(0, -n.dv) */
    double residual_max;
    double kinetic_energy;    /* sum of 1/2 m v^2 + 1/2 w.I.w over the enabled dynamic bodies */
    double potential_energy;  /* sum of -m g.x over the same bodies */
    uint32_t contact_points;
    uint32_t colors;          /* graph-coloured solver: colours used, colouring rounds */
    uint32_t coloring_rounds;
    uint32_t reserved;
} rp3dg_solver_stats;
int rp3dg_world_set_solver(rp3dg_world* world, int solver, int stats);
/* Statistics of the last step (zero before a step with stats on). */
int rp3dg_world_get_solver_stats(rp3dg_world* world, rp3dg_solver_stats* out);

/* The contact events of the last update, as EventListener::onContact
 * receives them (CollisionDetectionSystem::reportContacts,
 * CollisionDetectionSystem.cpp:1729-1738, and CollisionCallback::CallbackData,
 * CollisionCallback.cpp:79-134): the update's contact pairs in their creation
 * order, then the lost contact pairs (pairs that touched in the previous
 * frame and were removed by the broad phase or no longer touch).  Each event
 * has ContactPair::getEventType's type and, for a contact pair of an island,
 * its contact points (world normal and penetration depth, local points on
 * the two colliders; a pair outside the islands and a lost pair have none),
 * copied into the points arrays from `first_point`. */
#define RP3DG_CONTACT_START 0
#define RP3DG_CONTACT_STAY 1
#define RP3DG_CONTACT_EXIT 2
typedef struct rp3dg_contact_event {
    int32_t body1, body2;          /* creation indices */
    int32_t collider1, collider2;  /* creation indices */
    int32_t type;                  /* RP3DG_CONTACT_* */
    uint32_t first_point;          /* index of its first point in the points arrays */
    uint32_t nb_points;            /* ContactPair::getNbContactPoints */
} rp3dg_contact_event;
/* Host arrays with room for `capacity` events and `capacity_points` points
 * (float4 rows: normal + depth, local point 1, local point 2; any may be
 * NULL); the counts are written even when the arrays are short. */
int rp3dg_world_get_contact_events(rp3dg_world* world, uint32_t world_index, rp3dg_contact_event* events,
                                   uint32_t capacity, float* normal_depth, float* local1, float* local2,
                                   uint32_t capacity_points, uint32_t* nb_events, uint32_t* nb_points);

/* The trigger events of the last update: EventListener::onTrigger through
 * CollisionDetectionSystem::reportTriggers (CollisionDetectionSystem.cpp:
 * 1745-1757) and OverlapCallback::CallbackData (OverlapCallback.cpp:70-92):
 * the contact pairs of trigger colliders in creation order (type
 * RP3DG_CONTACT_START for OverlapStart, RP3DG_CONTACT_STAY for OverlapStay),
 * then the lost ones (RP3DG_CONTACT_EXIT for OverlapExit); no points.  The
 * contact events leave trigger pairs out (CollisionCallback.cpp:84-103). */
int rp3dg_world_get_trigger_events(rp3dg_world* world, uint32_t world_index, rp3dg_contact_event* events,
                                   uint32_t capacity, uint32_t* nb_events);

/* Debug rendering (DebugRenderer, src/utils/DebugRenderer.cpp) as headless
 * buffers: the items of DebugRenderer::DebugItem (DebugRenderer.h:73-91). */
#define RP3DG_DEBUG_COLLIDER_AABB            0x01u
#define RP3DG_DEBUG_COLLIDER_BROADPHASE_AABB 0x02u
#define RP3DG_DEBUG_COLLISION_SHAPE          0x04u
#define RP3DG_DEBUG_CONTACT_POINT            0x08u
#define RP3DG_DEBUG_CONTACT_NORMAL           0x10u
#define RP3DG_DEBUG_COLLISION_SHAPE_NORMAL   0x20u
/* DebugRenderer::DebugLine and DebugTriangle (DebugRenderer.h:95-146):
 * points and 0xRRGGBB colours, the same 32- and 48-byte layouts. */
typedef struct rp3dg_debug_line {
    float p1[3];
    uint32_t color1;
    float p2[3];
    uint32_t color2;
} rp3dg_debug_line;
typedef struct rp3dg_debug_triangle {
    float p1[3];
    uint32_t color1;
    float p2[3];
    uint32_t color2;
    float p3[3];
    uint32_t color3;
} rp3dg_debug_triangle;
/* PhysicsWorld::setIsDebugRenderingEnabled(items != 0) with
 * DebugRenderer::setIsDebugItemDisplayed(item, true) for each RP3DG_DEBUG_*
 * bit of `items` (every world of a group).  From the next update on, each
 * update ends with the primitives of DebugRenderer::onContact (a sphere of
 * radius 0.1 and a 1 m normal per contact point of the update's contact
 * pairs, DebugRenderer.cpp:530-560) followed by those of
 * computeDebugRenderingPrimitives (DebugRenderer.cpp:482-527: per body with
 * debug enabled, per collider, its AABB, fat broad-phase AABB and shape
 * triangles and face normals), with the default colours, computed on the GPU
 * in the reference's order and arithmetic. */
int rp3dg_world_set_debug_rendering(rp3dg_world* world, uint32_t items);
/* Body::setIsDebugEnabled (Body.cpp:509-512; false for a new body) for body
 * `body` of world `world_index`, or for every body of it when body < 0. */
int rp3dg_world_set_body_debug(rp3dg_world* world, uint32_t world_index, int32_t body, int enabled);
/* DebugRenderer::getLinesArray / getTrianglesArray after the last update of
 * world `world_index`: up to cap_lines lines and cap_triangles triangles
 * into `lines` / `triangles` (host memory, or device memory of the world's
 * device when `device` is non-zero; either may be NULL with capacity 0); the
 * counts are written even when the arrays are short. */
int rp3dg_world_get_debug_primitives(rp3dg_world* world, uint32_t world_index, rp3dg_debug_line* lines,
                                     uint32_t cap_lines, rp3dg_debug_triangle* triangles, uint32_t cap_triangles,
                                     uint32_t* nb_lines, uint32_t* nb_triangles, int device);

/* PhysicsWorld::raycast(ray, callback, raycastWithCategoryMaskBits)
 * (PhysicsWorld.h:486-490) for a batch of rays, each traced as the reference
 * traces one: DynamicAABBTree::raycast (DynamicAABBTree.cpp:684-747) over the
 * world's broad-phase tree in its stack order, the category filter
 * (BroadPhaseSystem.cpp:224-240), Collider::raycast into the collider's local
 * space (Collider.cpp:173-192) and the shape's raycast (SphereShape.cpp:61,
 * CapsuleShape.cpp:97, BoxShape.cpp:62, ConvexMeshShape.cpp:107,
 * HeightFieldShape.cpp:76 with HeightField.cpp:258-361 and
 * TriangleShape.cpp:143), with one of three RaycastCallback behaviours:
 *   CLOSEST  notifyRaycastHit returns hitFraction (the ray is clipped to each
 *            hit; the last hit reported is the result)
 *   ANY      returns 0 (the first hit in traversal order stops the ray)
 *   ALL      returns 1 (every hit is reported, in traversal order)
 * The world's state is the one after its last update. */
#define RP3DG_RAYCAST_CLOSEST 0
#define RP3DG_RAYCAST_ANY 1
#define RP3DG_RAYCAST_ALL 2
typedef struct rp3dg_ray {
    float point1[3];               /* Ray::point1, world space */
    float point2[3];               /* Ray::point2 */
    float max_fraction;            /* Ray::maxFraction (1 by default) */
    uint32_t category_mask;        /* raycastWithCategoryMaskBits (0xFFFF by default) */
} rp3dg_ray;
typedef struct rp3dg_raycast_hit { /* RaycastInfo */
    float world_point[3];
    float world_normal[3];
    float hit_fraction;
    int32_t body;                  /* creation index of the body */
    int32_t collider;              /* creation index of the collider */
    int32_t flags;                 /* bit 0: a height-field walk stopped at its cell limit (where the
                                      reference's walk does not end: a ray with an exactly zero z
                                      direction entering on a cell boundary) */
} rp3dg_raycast_hit;
/* n rays of world `world_index` (0 for rp3dg_world_create): hits holds
 * max_hits records per ray (ray i at hits[i * max_hits]), nb_hits[i] the
 * number of hits the callback received (it may exceed max_hits in ALL mode;
 * CLOSEST and ANY keep one record, the last received).  Host arrays. */
int rp3dg_world_raycast(rp3dg_world* world, uint32_t world_index, const rp3dg_ray* rays, uint32_t n, int32_t mode,
                        uint32_t max_hits, rp3dg_raycast_hit* hits, uint32_t* nb_hits);
/* The same with device arrays; returns when the results are written.
 * kernel_ms (may be NULL) receives the traversal kernel's duration. */
int rp3dg_world_raycast_device(rp3dg_world* world, uint32_t world_index, const rp3dg_ray* rays, uint32_t n,
                               int32_t mode, uint32_t max_hits, rp3dg_raycast_hit* hits, uint32_t* nb_hits,
                               float* kernel_ms);

/* Many independent worlds stepped together (the batch of the many-worlds
 * workload): nb_worlds worlds, world k made of bodies[body_offsets[k] ..
 * body_offsets[k+1]) and colliders[collider_offsets[k] .. collider_offsets[k+1])
 * (collider body indices local to the world), each built like
 * rp3dg_world_create and each stepping exactly as its own PhysicsWorld would
 * (bit-identical to a reference world per world).  One rp3dg_world_update
 * steps every world; the GPU work of all worlds runs in shared launches and
 * the order bookkeeping of the worlds on nb_threads host threads.  The
 * returned handle works with rp3dg_world_update / _destroy / _get_stats /
 * _set_profiling / _get_phase_times (rp3dg_world_get_bodies then returns all
 * worlds' bodies, world after world); the calls below read one world.  No
 * counterpart in the reference, where each world is its own PhysicsWorld. */
int rp3dg_world_group_create(rp3dg_ctx* ctx, const rp3dg_world_settings* settings, uint32_t nb_worlds,
                             const uint32_t* body_offsets, const rp3dg_body_desc* bodies,
                             const uint32_t* collider_offsets, const rp3dg_collider_desc* colliders,
                             int nb_threads, rp3dg_world** out);
int rp3dg_world_group_add_joints(rp3dg_world* group, uint32_t world, const rp3dg_joint_desc* joints, uint32_t n);
int rp3dg_world_group_get_bodies(rp3dg_world* group, uint32_t world, float* position, float* orientation,
                                 float* linear_velocity, float* angular_velocity, uint8_t* sleeping);
int rp3dg_world_group_get_pairs(rp3dg_world* group, uint32_t world, uint64_t* pair_ids, uint32_t capacity,
                                uint32_t* n);
int rp3dg_world_group_get_contacts(rp3dg_world* group, uint32_t world, int32_t* body1, int32_t* body2,
                                   uint8_t* nb_points, uint32_t capacity, float* normal_depth, float* local1,
                                   float* local2, uint32_t capacity_points, uint32_t* nb_manifolds,
                                   uint32_t* nb_contact_points);
/* Phase profiling (instrumentation; no counterpart in the reference, whose
 * profiler is a compile-time option): when enabled, each step drains the
 * stream at phase boundaries and accumulates wall-clock milliseconds per
 * phase: 0 broad phase (host), 1 middle phase (host), 2 narrow phase and
 * manifold step (GPU), 3 contact pairs and islands (host), 4 contact packing
 * and warm start (GPU), 5 dynamics stage (GPU), 6 collider update and tree
 * reinsertion, 7 sleeping and end of step; 8-12 parts of the middle phase,
 * 13-15 parts of the broad phase (tree queries, pair removal, narrow-phase
 * items).  Enabling resets the counters. */
int rp3dg_world_set_profiling(rp3dg_world* world, int enable);
/* Host threads of a world's bookkeeping (no counterpart in the reference,
 * whose update runs on one thread).  A group spreads its worlds over them; a
 * single world runs its broad-phase tree queries on them (the tree does not
 * change while it is queried, and the pairs are still processed in the
 * moved set's order, so results do not depend on the count).  A world from
 * rp3dg_world_create starts with 1. */
int rp3dg_world_set_threads(rp3dg_world* world, int threads);
/* Where the broad-phase trees of a world's bookkeeping live (no counterpart
 * in the reference).  With device trees, every world's DynamicAABBTree
 * (DynamicAABBTree.cpp:219-638) sits in one device pool: the reinsertions of
 * the moved colliders run on the GPU, one thread per world in the
 * reference's order, and the moved colliders' queries one thread per query;
 * the host keeps the moved set, the leaves' boxes and the pairs, and copies
 * a world's tree back before a world raycast reads it.  Results are
 * identical either way.  A group of 2 or more worlds of at most 8192
 * colliders each starts with device trees, any other world with host trees. */
int rp3dg_world_set_device_trees(rp3dg_world* world, int enable);
int rp3dg_world_get_device_trees(rp3dg_world* world, int* enabled);
/* Autotuner of the dynamics stage's island scheduling (no counterpart in the
 * reference): over the next steps, candidate settings of one parameter at a
 * time are tried on successive steps, `rounds` steps each, and timed with
 * CUDA events around the stage (per manifold); the fastest is kept.  The
 * parameters (islands of up to small_max manifolds: one thread each; above
 * giant_min: one CTA each; persistent CTAs per SM of the warp-per-island
 * kernel: large_per_sm) only decide which kernel takes which island, so
 * results are identical for every candidate.  The tuning takes
 * 9 x rounds steps. */
int rp3dg_world_autotune(rp3dg_world* world, int rounds);
/* out[0..3] = small_max, giant_min, large_per_sm, 1 while tuning. */
int rp3dg_world_get_tuning(rp3dg_world* world, uint32_t* out);
int rp3dg_world_get_phase_times(rp3dg_world* world, double* ms, uint32_t n);

/* Number of kernels this context launched so far (instrumentation; a
 * convex-polyhedron batch takes two). */
uint64_t rp3dg_kernel_launches(const rp3dg_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif /* RP3DG_H */
