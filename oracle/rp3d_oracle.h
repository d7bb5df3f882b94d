/* Test infrastructure, not product code.
 *
 * rp3d_oracle: a plain-C restatement of ReactPhysics3D v0.10.2's narrow-phase
 * algorithms (single precision, one pair at a time, the reference's operation
 * order) used as a CPU checker for the CUDA library.  It consumes and produces
 * the struct-of-arrays batches of include/rp3dg.h.  It is pinned against the
 * reference engine itself (oracle/_ref, built from the reference sources) by
 * tests/test_oracle_vs_reference.py and against the committed golden fixtures.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 */
#ifndef RP3D_ORACLE_H
#define RP3D_ORACLE_H
#include "../include/rp3dg.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Convex mesh from polygon faces (ConvexMesh::init, ConvexMesh.cpp:47-79). */
int rp3do_create_convex_mesh(const float* vertices, uint32_t nb_vertices, const uint32_t* face_indices,
                             const uint32_t* face_sizes, uint32_t nb_faces, int32_t* mesh_id);
/* Mesh + scale (ConvexMeshShape, ConvexMeshShape.cpp:38-70). */
int rp3do_create_convex_mesh_shape(int32_t mesh_id, float sx, float sy, float sz, int32_t* instance_id);
int rp3do_get_convex_mesh_tables(int32_t instance_id, uint32_t* nb_vertices, uint32_t* nb_faces,
                                 uint32_t* nb_half_edges, uint32_t* half_edges, float* face_normals,
                                 uint32_t* face_edge, float* centroid, uint32_t cap_he, uint32_t cap_faces);
/* Forget every mesh (tests call it between cases). */
void rp3do_reset(void);

/* One algorithm over a host batch; same semantics as rp3dg_narrowphase_host. */
int rp3do_narrowphase(int algorithm, const rp3dg_shape* shapes, uint32_t nb_shapes, const rp3dg_pair_batch* pairs,
                      const rp3dg_contact_batch* out, int clip_with_previous_axis);

/* Convex-pair manifold reduction (<= 4 points, de-duplicated), in place. */
int rp3do_reduce_contacts(const rp3dg_pair_batch* pairs, const rp3dg_contact_batch* contacts, uint8_t* kept);

/* Dynamics stage of a world step, same semantics as rp3dg_dynamics_step_host
 * except that the velocities of read-only bodies receive the solver's
 * signed-zero updates exactly as the reference's arrays do. */
int rp3do_dynamics_step(const rp3dg_dynamics_params* params, const rp3dg_bodies* bodies,
                        const rp3dg_colliders* colliders, const rp3dg_manifolds* manifolds,
                        const rp3dg_points* points, const rp3dg_islands* islands);

/* Broad phase: world AABB of each collider from its shape and local-to-world
 * transform, then the fat-AABB update (moved = reinserted); mesh_bounds holds
 * 6 floats (min, max) per convex-mesh instance, scaled. */
int rp3do_broadphase_update(const rp3dg_shape* shapes, const float* mesh_bounds, uint32_t n, const int32_t* shape,
                            const rp3dg_float4* world_position, const rp3dg_float4* world_orientation,
                            const uint8_t* force_reinsert, rp3dg_float4* fat_min, rp3dg_float4* fat_max,
                            uint8_t* moved);
/* Overlapping pairs (i < j) of fat AABBs, brute force. */
long rp3do_broadphase_pairs(uint32_t n, const rp3dg_float4* fat_min, const rp3dg_float4* fat_max, const int32_t* body,
                            const int32_t* group, const uint16_t* category, const uint16_t* mask, int32_t* pairs,
                            long cap);

#ifdef __cplusplus
}
#endif
#endif
