// Host runtime behind the C ABI of include/rp3dg.h: context (device, stream),
// immutable shape tables (box topology, convex-mesh arenas), the shape table,
// and the narrow-phase entry points.  Convex-mesh set-up restates
// ConvexMesh::init (reference src/collision/ConvexMesh.cpp:47-264) and
// HalfEdgeStructure::computeHalfEdges (src/collision/HalfEdgeStructure.cpp:34-127)
// in single precision with the reference's operation order, so the tables the
// kernels read are bit-identical to the ones the reference builds.
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdlib>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "../../include/rp3dg.h"
#include "broadphase_launch.h"
#include "contacts_launch.h"
#include "dynamics_launch.h"
#include "mlp_launch.h"
#include "np_launch.h"
#include "rp3dg_internal.h"
#include "world_order.h"

using rp3dg::BoxTables;
using rp3dg::MeshHdr;

namespace {

struct HalfEdge { uint32_t vertex, twin, face, next; };

struct MeshTopo {
    std::vector<float> verts;  // nv*3
    std::vector<uint32_t> face_start, face_count, face_verts, face_edge;
    std::vector<HalfEdge> edges;
    std::vector<float> normals;  // nf*3 (unit, unscaled mesh)
    std::vector<float> area2;    // nf: length of the Newell normal (twice the face area)
    float centroid[3] = {0, 0, 0};
    float bmin[3] = {0, 0, 0}, bmax[3] = {0, 0, 0};  // ConvexMesh::mBounds
    float volume = 0.0f;                             // ConvexMesh::mVolume
    uint32_t nv = 0, nf = 0;
};

// TriangleMesh (TriangleMesh.h): the vertices and vertex normals left after
// the unused ones were removed, the kept triangles, and the DynamicAABBTree
// of the triangles as RayNode records
struct TriMesh {
    std::vector<float> verts, normals;   // 3 per vertex
    std::vector<uint32_t> tris;          // 3 per triangle
    std::vector<rp3dg::RayNode> nodes;
    int32_t root = -1;
    float bmin[3] = {0, 0, 0}, bmax[3] = {0, 0, 0};  // getBounds: the root's AABB
};

struct MeshInstance {
    int32_t mesh;
    float scale[3];
    std::vector<float> sverts;   // vertex * scale
    std::vector<float> snormals; // scaled unit normals
    float scentroid[3];
};

// HalfEdgeStructure::computeHalfEdges: half-edges are appended in pairs when
// the second face using an undirected edge is met (earlier face's half-edge
// first); next pointers follow each face's winding; a face's edgeIndex is its
// closing half-edge (last vertex -> first vertex).
bool compute_half_edges(const std::vector<uint32_t>& face_start, const std::vector<uint32_t>& face_count,
                        const std::vector<uint32_t>& face_verts, uint32_t nv, std::vector<HalfEdge>& out,
                        std::vector<uint32_t>& face_edge) {
    typedef std::pair<uint32_t, uint32_t> Key;
    std::map<Key, HalfEdge> pending;      // the reference's 'edges' map
    std::map<Key, Key> next_key;          // 'nextEdges'
    std::map<Key, uint32_t> index_of;     // 'mapEdgeToIndex'
    std::vector<Key> key_of;              // 'mapEdgeIndexToKey'
    std::vector<Key> face_key(face_count.size());
    out.clear();
    for (uint32_t f = 0; f < face_count.size(); f++) {
        const uint32_t n = face_count[f];
        const uint32_t* fv = face_verts.data() + face_start[f];
        Key first(0, 0), prev(0, 0);
        for (uint32_t v = 0; v < n; v++) {
            const uint32_t v1 = fv[v], v2 = fv[v == n - 1 ? 0 : v + 1];
            if (v1 >= nv || v2 >= nv) return false;
            const Key k12(v1, v2), k21(v2, v1);
            HalfEdge e{v1, 0, f, 0};
            if (v == 0) first = k12;
            else next_key[prev] = k12;
            if (v == n - 1) next_key[k12] = first;
            pending.emplace(k12, e);
            face_key[f] = k12;
            auto it = pending.find(k21);
            if (it != pending.end() && index_of.find(k21) == index_of.end()) {
                const uint32_t idx = uint32_t(out.size());
                it->second.twin = idx + 1;
                e.twin = idx;
                if (key_of.size() < idx + 2) key_of.resize(idx + 2);
                key_of[idx] = k21;
                key_of[idx + 1] = k12;
                index_of[k12] = idx + 1;
                index_of[k21] = idx;
                out.push_back(it->second);
                out.push_back(e);
            }
            prev = k12;
        }
    }
    for (uint32_t i = 0; i < out.size(); i++) {
        auto nk = next_key.find(key_of[i]);
        if (nk == next_key.end()) return false;
        auto ni = index_of.find(nk->second);
        if (ni == index_of.end()) return false;
        out[i].next = ni->second;
    }
    face_edge.resize(face_count.size());
    for (uint32_t f = 0; f < face_count.size(); f++) {
        auto fi = index_of.find(face_key[f]);
        if (fi == index_of.end()) return false;
        face_edge[f] = fi->second;
    }
    // A closed, consistently wound mesh: twins pair up, and walking `next`
    // from each face's edge returns to it after exactly face_count steps.
    // The kernels walk these cycles, so anything else is rejected here.
    for (uint32_t i = 0; i < out.size(); i++) {
        if (out[i].twin >= out.size() || out[out[i].twin].twin != i || out[i].next >= out.size()) return false;
    }
    if (out.size() != face_verts.size()) return false;
    for (uint32_t f = 0; f < face_count.size(); f++) {
        uint32_t e = face_edge[f], steps = 0;
        do {
            if (out[e].face != f) return false;
            e = out[e].next;
        } while (e != face_edge[f] && ++steps <= face_count[f]);
        if (steps + 1 != face_count[f]) return false;
    }
    return true;
}

BoxTables make_box_tables() {
    // PhysicsCommon::initBoxShapeHalfEdgeStructure (reference src/engine/PhysicsCommon.cpp:73-109)
    static const uint32_t faces[24] = {0, 1, 2, 3, 1, 5, 6, 2, 4, 7, 6, 5, 4, 0, 3, 7, 4, 5, 1, 0, 2, 6, 7, 3};
    std::vector<uint32_t> fs(6), fc(6, 4), fv(faces, faces + 24), fe;
    for (int f = 0; f < 6; f++) fs[f] = 4 * f;
    std::vector<HalfEdge> edges;
    compute_half_edges(fs, fc, fv, 8, edges, fe);
    BoxTables t;
    std::memset(&t, 0, sizeof(t));
    for (int e = 0; e < 24; e++) {
        t.edges[e][0] = uint8_t(edges[e].vertex);
        t.edges[e][1] = uint8_t(edges[e].twin);
        t.edges[e][2] = uint8_t(edges[e].face);
        t.edges[e][3] = uint8_t(edges[e].next);
    }
    for (int i = 0; i < 24; i++) t.face_verts[i] = uint8_t(faces[i]);
    for (int f = 0; f < 6; f++) t.face_edge[f] = uint8_t(fe[f]);
    // Axis-aligned Gauss-map data (see BoxTables): vertex v has +x for
    // v in {1,2,5,6}, +y for {2,3,6,7}, +z for {0,1,2,3}; face normals are
    // 0:+z 1:+x 2:-z 3:-x 4:-y 5:+y.
    auto pos = [](int v, int axis) {
        const int masks[3] = {0x66, 0xCC, 0x0F};
        return (masks[axis] >> v) & 1;
    };
    const int face_axis[6] = {2, 0, 2, 0, 1, 1};
    const int face_neg[6] = {0, 0, 1, 1, 1, 0};
    for (int e = 0; e < 24; e++) {
        const int v1 = edges[e].vertex, v2 = edges[edges[e].twin].vertex;
        int k = 0;
        for (int ax = 0; ax < 3; ax++)
            if (pos(v1, ax) != pos(v2, ax)) k = ax;
        const int negD = pos(v1, k) ? 0 : 1;  // v1.k - v2.k = +2h when v1 is on the positive side
        const int f1 = edges[e].face, f2 = edges[edges[e].twin].face;
        // c = -normal: negative when the normal is positive
        t.gauss[e][0] = uint8_t(k | (negD << 2));
        t.gauss[e][1] = uint8_t(face_axis[f1] | ((face_neg[f1] ? 0 : 1) << 2));
        t.gauss[e][2] = uint8_t(face_axis[f2] | ((face_neg[f2] ? 0 : 1) << 2));
        t.gauss[e][3] = 0;
    }
    int fillc[3] = {0, 0, 0};
    for (int e = 0; e < 24; e += 2) {
        const int k = t.gauss[e][0] & 3;
        if (fillc[k] < 4) t.axis_edges[k][fillc[k]++] = uint8_t(e);
    }
    // PhysicsCommon::initTriangleShapeHalfEdgeStructure (reference
    // src/engine/PhysicsCommon.cpp:111-130): the two faces of a triangle
    static const uint32_t tri_faces[6] = {0, 1, 2, 0, 2, 1};
    std::vector<uint32_t> tfs = {0, 3}, tfc = {3, 3}, tfv(tri_faces, tri_faces + 6), tfe;
    std::vector<HalfEdge> tedges;
    compute_half_edges(tfs, tfc, tfv, 3, tedges, tfe);
    for (int e = 0; e < 6; e++) {
        t.tri_edges[e][0] = uint8_t(tedges[e].vertex);
        t.tri_edges[e][1] = uint8_t(tedges[e].twin);
        t.tri_edges[e][2] = uint8_t(tedges[e].face);
        t.tri_edges[e][3] = uint8_t(tedges[e].next);
    }
    t.tri_face_edge[0] = uint8_t(tfe[0]);
    t.tri_face_edge[1] = uint8_t(tfe[1]);
    return t;
}

}  // namespace

struct rp3dg_ctx {
    int device = 0;
    int num_sms = 148;
    int smem_optin = 0;   // cudaDevAttrMaxSharedMemoryPerBlockOptin
    cudaStream_t stream = nullptr;
    std::string err;
    uint64_t launches = 0;
    // shapes
    rp3dg_shape* d_shapes = nullptr;
    uint32_t nb_shapes = 0, cap_shapes = 0;
    std::vector<rp3dg_shape> host_shapes;
    // convex meshes
    std::vector<MeshTopo> meshes;
    std::vector<MeshInstance> instances;
    std::vector<uint32_t> arena;  // host copy of the device mesh arena
    uint32_t* d_arena = nullptr;
    size_t cap_arena = 0;
    // device error word written by the kernels (bit 0: a pair named a shape outside the table)
    uint32_t* d_error = nullptr;
    // path-event counters of rp3dg_narrowphase_count_events (NP_EVENT_COUNT words)
    unsigned long long* d_events = nullptr;
    // polyhedron batches: the lists of mesh pairs by shape combination and their counters
    uint32_t* d_plist = nullptr;
    size_t cap_plist = 0;
    // staging buffers for rp3dg_narrowphase_host
    void* d_stage = nullptr;
    size_t cap_stage = 0;
    // rp3dg_narrowphase_input_host: device staging of all batches; an
    // upload stream, a stream for each batch's flags / counts / record
    // count and one for its packed contacts beside the compute stream; four
    // events per batch; page-locked host staging of the flags, counts and
    // caches (h_imeta), of the packed contacts copied with the flags
    // (h_ispec) and of those copied once their count is known (h_irec)
    void* d_istage = nullptr;
    size_t cap_istage = 0;
    cudaStream_t s_up = nullptr, s_pub = nullptr, s_rec = nullptr;
    std::vector<cudaEvent_t> events;
    void *h_imeta = nullptr, *h_irec = nullptr, *h_ispec = nullptr;
    size_t cap_imeta = 0, cap_irec = 0, cap_ispec = 0;
    std::vector<uint32_t> last_pairs, last_records;   // per batch position: the last call's pairs and records
    // learned separating-axis MLP: one device block holding the fp32
    // parameters, Adam moments, gradients, packed bf16 fragments, loss word
    // and proposal counters; training scratch grows with the batch
    char* d_mlp = nullptr;
    float* d_mlp_scratch = nullptr;
    uint8_t* d_proposals = nullptr;
    uint32_t cap_proposals = 0;
    uint32_t* d_perm = nullptr;     // pair order of a learned batch, then 32 counters
    uint32_t cap_perm = 0;
    size_t cap_mlp_scratch = 0;
    int mlp_step = 0;
    bool mlp_ready = false;
    bool learned_axis = false;
    // dynamics stage: per-body velocity scratch and solver records
    void* d_dyn = nullptr;
    size_t cap_dyn = 0;
    // staging buffers for rp3dg_dynamics_step_host
    void* d_dyn_stage = nullptr;
    size_t cap_dyn_stage = 0;
    // broad phase: local bounds of every shape (min, max float4 pairs),
    // pair-search scratch and host-call staging
    float* d_shape_bounds = nullptr;
    uint32_t cap_shape_bounds = 0;
    void* d_bp = nullptr;
    size_t cap_bp = 0;
    void* d_bp_stage = nullptr;
    size_t cap_bp_stage = 0;
    // height fields (device heights in HfDesc::heights)
    std::vector<rp3dg::HfDesc> hfields;
    // triangle meshes and concave mesh shape instances (device arrays in
    // each CmDesc)
    std::vector<TriMesh> trimeshes;
    std::vector<rp3dg::CmDesc> cmeshes;
};

namespace {
constexpr size_t MLP_PARAM_BYTES = size_t(RP3DG_MLP_NPARAMS) * 4;
constexpr size_t MLP_OFF_PARAMS = 0;
constexpr size_t MLP_OFF_M = MLP_OFF_PARAMS + MLP_PARAM_BYTES;
constexpr size_t MLP_OFF_V = MLP_OFF_M + MLP_PARAM_BYTES;
constexpr size_t MLP_OFF_G = MLP_OFF_V + MLP_PARAM_BYTES;
constexpr size_t MLP_OFF_PACKED = (MLP_OFF_G + MLP_PARAM_BYTES + 255) & ~size_t(255);
constexpr size_t MLP_PACKED_BYTES = 16384;  // >= sizeof(rp3dg::MlpPacked)
constexpr size_t MLP_OFF_LOSS = MLP_OFF_PACKED + MLP_PACKED_BYTES;
constexpr size_t MLP_OFF_STATS = MLP_OFF_LOSS + 256;
constexpr size_t MLP_BLOCK_BYTES = MLP_OFF_STATS + 256;
float* mlp_params(rp3dg_ctx* c) { return reinterpret_cast<float*>(c->d_mlp + MLP_OFF_PARAMS); }
float* mlp_m(rp3dg_ctx* c) { return reinterpret_cast<float*>(c->d_mlp + MLP_OFF_M); }
float* mlp_v(rp3dg_ctx* c) { return reinterpret_cast<float*>(c->d_mlp + MLP_OFF_V); }
float* mlp_g(rp3dg_ctx* c) { return reinterpret_cast<float*>(c->d_mlp + MLP_OFF_G); }
rp3dg::MlpPacked* mlp_packed(rp3dg_ctx* c) { return reinterpret_cast<rp3dg::MlpPacked*>(c->d_mlp + MLP_OFF_PACKED); }
float* mlp_loss(rp3dg_ctx* c) { return reinterpret_cast<float*>(c->d_mlp + MLP_OFF_LOSS); }
unsigned long long* mlp_stats(rp3dg_ctx* c) { return reinterpret_cast<unsigned long long*>(c->d_mlp + MLP_OFF_STATS); }
}  // namespace

namespace {

int fail(rp3dg_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return code;
}

// Device arrays are read with vector loads: float4 arrays and the 16-byte
// cache records need 16-byte alignment, int32 arrays 4-byte.
bool aligned(const void* ptr, uintptr_t a) { return (reinterpret_cast<uintptr_t>(ptr) & (a - 1)) == 0; }

int cuda_fail(rp3dg_ctx* ctx, cudaError_t e, const char* what) {
    return fail(ctx, RP3DG_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// Lay out every instance: headers first, then per-instance tables.
void rebuild_arena(rp3dg_ctx* ctx) {
    std::vector<uint32_t>& w = ctx->arena;
    const uint32_t nin = uint32_t(ctx->instances.size());
    const uint32_t hdr_words = nin * (sizeof(MeshHdr) / 4);
    w.assign(hdr_words, 0u);
    auto push_f = [&](float x) { uint32_t u; std::memcpy(&u, &x, 4); w.push_back(u); };
    for (uint32_t k = 0; k < nin; k++) {
        const MeshInstance& in = ctx->instances[k];
        const MeshTopo& m = ctx->meshes[in.mesh];
        MeshHdr h;
        std::memset(&h, 0, sizeof(h));
        h.nv = m.nv; h.nf = m.nf; h.nhe = uint32_t(m.edges.size());
        h.off_verts = uint32_t(w.size());
        for (float x : m.verts) push_f(x);
        h.off_sverts = uint32_t(w.size());
        for (float x : in.sverts) push_f(x);
        h.off_normals = uint32_t(w.size());
        for (float x : in.snormals) push_f(x);
        h.off_face_start = uint32_t(w.size());
        for (uint32_t x : m.face_start) w.push_back(x);
        h.off_face_count = uint32_t(w.size());
        for (uint32_t x : m.face_count) w.push_back(x);
        h.off_face_verts = uint32_t(w.size());
        for (uint32_t x : m.face_verts) w.push_back(x);
        h.off_face_edge = uint32_t(w.size());
        for (uint32_t x : m.face_edge) w.push_back(x);
        h.off_edges = uint32_t(w.size());
        for (const HalfEdge& e : m.edges) { w.push_back(e.vertex); w.push_back(e.twin); w.push_back(e.face); w.push_back(e.next); }
        h.centroid[0] = in.scentroid[0]; h.centroid[1] = in.scentroid[1]; h.centroid[2] = in.scentroid[2];
        std::memcpy(w.data() + k * (sizeof(MeshHdr) / 4), &h, sizeof(h));
    }
}

int upload_arena(rp3dg_ctx* ctx) {
    const size_t bytes = ctx->arena.size() * 4;
    if (bytes > ctx->cap_arena) {
        if (ctx->d_arena) cudaFree(ctx->d_arena);
        ctx->d_arena = nullptr;
        cudaError_t e = cudaMalloc(&ctx->d_arena, bytes);
        if (e != cudaSuccess) { ctx->cap_arena = 0; return cuda_fail(ctx, e, "cudaMalloc(mesh arena)"); }
        ctx->cap_arena = bytes;
    }
    cudaError_t e = cudaMemcpyAsync(ctx->d_arena, ctx->arena.data(), bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    return e == cudaSuccess ? 0 : cuda_fail(ctx, e, "upload mesh arena");
}

}  // namespace

namespace rp3dg {
int dynamics_step_flags(rp3dg_ctx* ctx, const rp3dg_dynamics_params* pr, const rp3dg_bodies* b,
                        const rp3dg_colliders* c, const rp3dg_manifolds* m, const rp3dg_points* p,
                        const rp3dg_islands* is, const uint8_t* b_enabled, const uint8_t* c_enabled,
                        const DynJoints* joints = nullptr, const DynTuning* tune = nullptr,
                        const DynSolver* solver = nullptr);
int broadphase_update_flags(rp3dg_ctx* ctx, const rp3dg_broadphase* bp, const uint8_t* enabled);
}  // namespace rp3dg

// host copy of the shape table (world set-up reads it; C++ linkage)
namespace rp3dg {
int get_shapes_host(rp3dg_ctx* ctx, std::vector<rp3dg_shape>* out) {
    if (!ctx || !out) return RP3DG_EINVAL;
    *out = ctx->host_shapes;
    return 0;
}
// the device shape table and its local bounds (2 float4 per shape)
int get_shape_device(rp3dg_ctx* ctx, const rp3dg_shape** shapes, const float4** bounds) {
    if (!ctx) return RP3DG_EINVAL;
    *shapes = ctx->d_shapes;
    *bounds = reinterpret_cast<const float4*>(ctx->d_shape_bounds);
    return 0;
}
// all height fields of the context, by id, and the device convex-mesh arena
// (world raycasts)
int get_heightfields(rp3dg_ctx* ctx, std::vector<HfDesc>* out) {
    if (!ctx || !out) return RP3DG_EINVAL;
    *out = ctx->hfields;
    return 0;
}
// ConvexMeshShape::getVolume (ConvexMeshShape.h:230-232) and the extents of
// ConvexMesh::getLocalInertiaTensor (ConvexMesh.h:200-211): volume * sx * sy
// * sz, and 0.5 * scale * (bounds max - bounds min)
int get_mesh_mass(rp3dg_ctx* ctx, int32_t instance, float* volume, float* extent) {
    if (!ctx || instance < 0 || size_t(instance) >= ctx->instances.size()) return RP3DG_EINVAL;
    const MeshInstance& in = ctx->instances[size_t(instance)];
    const MeshTopo& m = ctx->meshes[size_t(in.mesh)];
    *volume = m.volume * in.scale[0] * in.scale[1] * in.scale[2];
    for (int a = 0; a < 3; a++) extent[a] = (0.5f * in.scale[a]) * (m.bmax[a] - m.bmin[a]);
    return 0;
}
// face vertex counts of a convex-mesh instance (debug rendering)
int get_mesh_face_counts(rp3dg_ctx* ctx, int32_t instance, std::vector<uint32_t>* counts) {
    if (!ctx || !counts || instance < 0 || size_t(instance) >= ctx->instances.size()) return RP3DG_EINVAL;
    const MeshTopo& m = ctx->meshes[size_t(ctx->instances[size_t(instance)].mesh)];
    *counts = m.face_count;
    return 0;
}
int get_mesh_arena_device(rp3dg_ctx* ctx, const uint32_t** words) {
    if (!ctx || !words) return RP3DG_EINVAL;
    *words = ctx->d_arena;
    return 0;
}
// all concave mesh shape instances of the context, by id
int get_cmeshes(rp3dg_ctx* ctx, std::vector<CmDesc>* out) {
    if (!ctx || !out) return RP3DG_EINVAL;
    *out = ctx->cmeshes;
    return 0;
}
// a height field of the context (world set-up and middle phase)
int get_heightfield(rp3dg_ctx* ctx, int32_t id, HfDesc* out) {
    if (!ctx || !out || id < 0 || size_t(id) >= ctx->hfields.size()) return RP3DG_EINVAL;
    *out = ctx->hfields[size_t(id)];
    return 0;
}
// error message of a world call, readable through rp3dg_last_error
void set_error(rp3dg_ctx* ctx, const std::string& msg) {
    if (ctx) ctx->err = msg;
}
}  // namespace rp3dg

extern "C" {

int rp3dg_create(int device, rp3dg_ctx** out) {
    if (!out) return RP3DG_EINVAL;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return RP3DG_ENODEV;
    if (device < 0 || device >= count) return RP3DG_EINVAL;
    rp3dg_ctx* ctx = new rp3dg_ctx();
    ctx->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&ctx->d_error, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemsetAsync(ctx->d_error, 0, sizeof(uint32_t), ctx->stream);
    if (e != cudaSuccess) { delete ctx; return RP3DG_ECUDA; }
    const BoxTables t = make_box_tables();
    rp3dg::upload_box_tables(t, ctx->stream);
    rp3dg_events_upload_box_tables(&t, ctx->stream);
    rp3dg::upload_mlp_box_tables(t, ctx->stream);
    e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) { cudaStreamDestroy(ctx->stream); delete ctx; return RP3DG_ECUDA; }
    *out = ctx;
    return 0;
}

void rp3dg_destroy(rp3dg_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    cudaFree(ctx->d_shapes);
    cudaFree(ctx->d_arena);
    cudaFree(ctx->d_stage);
    cudaFree(ctx->d_istage);
    if (ctx->s_up) cudaStreamDestroy(ctx->s_up);
    if (ctx->s_pub) cudaStreamDestroy(ctx->s_pub);
    if (ctx->s_rec) cudaStreamDestroy(ctx->s_rec);
    cudaFreeHost(ctx->h_imeta);
    cudaFreeHost(ctx->h_irec);
    cudaFreeHost(ctx->h_ispec);
    for (cudaEvent_t ev : ctx->events) cudaEventDestroy(ev);
    cudaFree(ctx->d_error);
    cudaFree(ctx->d_events);
    cudaFree(ctx->d_plist);
    cudaFree(ctx->d_mlp);
    cudaFree(ctx->d_mlp_scratch);
    cudaFree(ctx->d_proposals);
    cudaFree(ctx->d_perm);
    cudaFree(ctx->d_dyn);
    cudaFree(ctx->d_dyn_stage);
    cudaFree(ctx->d_shape_bounds);
    cudaFree(ctx->d_bp);
    cudaFree(ctx->d_bp_stage);
    for (auto& h : ctx->hfields) cudaFree(const_cast<float*>(h.heights));
    for (auto& c : ctx->cmeshes) {
        cudaFree(const_cast<uint32_t*>(c.tris));
        cudaFree(const_cast<float*>(c.sverts));
        cudaFree(const_cast<float*>(c.snormals));
        cudaFree(const_cast<rp3dg::RayNode*>(c.nodes));
    }
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char* rp3dg_last_error(const rp3dg_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

void* rp3dg_stream(rp3dg_ctx* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

int rp3dg_synchronize(rp3dg_ctx* ctx) {
    if (!ctx) return RP3DG_EINVAL;
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    return e == cudaSuccess ? 0 : cuda_fail(ctx, e, "cudaStreamSynchronize");
}

uint64_t rp3dg_kernel_launches(const rp3dg_ctx* ctx) { return ctx ? ctx->launches : 0; }

int rp3dg_device_errors(rp3dg_ctx* ctx, uint32_t* flags, int clear) {
    if (!ctx || !flags) return fail(ctx, RP3DG_EINVAL, "null argument");
    cudaSetDevice(ctx->device);
    cudaError_t e = cudaMemcpyAsync(flags, ctx->d_error, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess && clear) e = cudaMemsetAsync(ctx->d_error, 0, sizeof(uint32_t), ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    return e == cudaSuccess ? 0 : cuda_fail(ctx, e, "read device error word");
}

int rp3dg_create_convex_mesh(rp3dg_ctx* ctx, const float* vertices, uint32_t nv, const uint32_t* face_indices,
                             const uint32_t* face_sizes, uint32_t nf, int32_t* mesh_id) {
    if (!ctx || !vertices || !face_indices || !face_sizes || !mesh_id) return fail(ctx, RP3DG_EINVAL, "null argument");
    if (nv == 0 || nf == 0) return fail(ctx, RP3DG_EINVAL, "empty mesh");
    if (nv > rp3dg::MAX_MESH_VERTICES || nf > rp3dg::MAX_MESH_FACES)
        return fail(ctx, RP3DG_ECAPACITY, "mesh exceeds 4096 vertices or 256 faces");
    MeshTopo m;
    m.nv = nv; m.nf = nf;
    m.verts.assign(vertices, vertices + 3 * size_t(nv));
    uint32_t total = 0;
    for (uint32_t f = 0; f < nf; f++) {
        if (face_sizes[f] < 3) return fail(ctx, RP3DG_EINVAL, "face with fewer than three vertices");
        if (face_sizes[f] > rp3dg::MAX_FACE_VERTICES) return fail(ctx, RP3DG_ECAPACITY, "face with more than 16 vertices");
        m.face_start.push_back(total);
        m.face_count.push_back(face_sizes[f]);
        total += face_sizes[f];
    }
    m.face_verts.assign(face_indices, face_indices + total);
    if (!compute_half_edges(m.face_start, m.face_count, m.face_verts, nv, m.edges, m.face_edge))
        return fail(ctx, RP3DG_EINVAL, "faces do not form a closed half-edge mesh");
    if (m.edges.size() > rp3dg::MAX_MESH_HALF_EDGES) return fail(ctx, RP3DG_ECAPACITY, "mesh exceeds 256 half-edges");
    // centroid: ConvexMesh::copyVertices (ConvexMesh.cpp:83-108), sequential sum then division
    float c[3] = {0.0f, 0.0f, 0.0f};
    for (uint32_t i = 0; i < nv; i++) { c[0] = c[0] + m.verts[3 * i]; c[1] = c[1] + m.verts[3 * i + 1]; c[2] = c[2] + m.verts[3 * i + 2]; }
    const float fnv = float(nv);
    m.centroid[0] = c[0] / fnv; m.centroid[1] = c[1] / fnv; m.centroid[2] = c[2] / fnv;
    // Newell normals, normalised: ConvexMesh::computeFacesNormals / computeFaceNormal (ConvexMesh.cpp:185-240)
    m.normals.resize(3 * size_t(nf));
    for (uint32_t f = 0; f < nf; f++) {
        float n[3] = {0.0f, 0.0f, 0.0f};
        const uint32_t cnt = m.face_count[f];
        for (uint32_t i = cnt - 1, j = 0; j < cnt; i = j, j++) {
            const float* a = &m.verts[3 * m.face_verts[m.face_start[f] + i]];
            const float* b = &m.verts[3 * m.face_verts[m.face_start[f] + j]];
            const float x = (a[1] - b[1]) * (a[2] + b[2]);
            const float y = (a[2] - b[2]) * (a[0] + b[0]);
            const float z = (a[0] - b[0]) * (a[1] + b[1]);
            n[0] = n[0] + x; n[1] = n[1] + y; n[2] = n[2] + z;
        }
        const float len = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        if (!(len > FLT_EPSILON)) return fail(ctx, RP3DG_EINVAL, "face with zero area");
        m.normals[3 * f] = n[0] / len; m.normals[3 * f + 1] = n[1] / len; m.normals[3 * f + 2] = n[2] / len;
        m.area2.push_back(len);
    }
    // bounds: ConvexMesh::copyVertices (AABB::inflateWithPoint over the vertices)
    for (int a = 0; a < 3; a++) m.bmin[a] = m.bmax[a] = m.verts[size_t(a)];
    for (uint32_t i = 0; i < nv; i++)
        for (int a = 0; a < 3; a++) {
            const float v = m.verts[3 * i + a];
            m.bmin[a] = std::min(m.bmin[a], v);
            m.bmax[a] = std::max(m.bmax[a], v);
        }
    // ConvexMesh::computeVolume (ConvexMesh.cpp:248-264): sum over the faces of
    // (first vertex . unit normal) * (Newell normal length * 0.5), |sum| / 3
    {
        float sum = 0.0f;
        for (uint32_t f = 0; f < nf; f++) {
            const float area = m.area2[f] * 0.5f;
            const float* v = &m.verts[3 * m.face_verts[m.face_start[f]]];
            const float* n = &m.normals[3 * f];
            sum += (v[0] * n[0] + v[1] * n[1] + v[2] * n[2]) * area;
        }
        m.volume = std::fabs(sum) / 3.0f;
    }
    ctx->meshes.push_back(std::move(m));
    *mesh_id = int32_t(ctx->meshes.size() - 1);
    return 0;
}

int rp3dg_create_convex_mesh_shape(rp3dg_ctx* ctx, int32_t mesh_id, float sx, float sy, float sz,
                                   int32_t* instance_id) {
    if (!ctx || !instance_id) return fail(ctx, RP3DG_EINVAL, "null argument");
    if (mesh_id < 0 || size_t(mesh_id) >= ctx->meshes.size()) return fail(ctx, RP3DG_EINVAL, "unknown mesh id");
    if (!(sx > 0.0f && sy > 0.0f && sz > 0.0f)) return fail(ctx, RP3DG_EINVAL, "scale must be positive");
    const MeshTopo& m = ctx->meshes[mesh_id];
    MeshInstance in;
    in.mesh = mesh_id;
    in.scale[0] = sx; in.scale[1] = sy; in.scale[2] = sz;
    in.sverts.resize(3 * size_t(m.nv));
    for (uint32_t i = 0; i < m.nv; i++) {
        in.sverts[3 * i] = m.verts[3 * i] * sx;
        in.sverts[3 * i + 1] = m.verts[3 * i + 1] * sy;
        in.sverts[3 * i + 2] = m.verts[3 * i + 2] * sz;
    }
    // ConvexMeshShape::computeScaledFacesNormals (ConvexMeshShape.cpp:50-70):
    // the reciprocal scale is computed in double and stored as float
    const float inv[3] = {float(1.0 / double(sx)), float(1.0 / double(sy)), float(1.0 / double(sz))};
    in.snormals.resize(3 * size_t(m.nf));
    for (uint32_t f = 0; f < m.nf; f++) {
        const float x = inv[0] * m.normals[3 * f], y = inv[1] * m.normals[3 * f + 1], z = inv[2] * m.normals[3 * f + 2];
        const float len = std::sqrt(x * x + y * y + z * z);
        in.snormals[3 * f] = x / len; in.snormals[3 * f + 1] = y / len; in.snormals[3 * f + 2] = z / len;
    }
    in.scentroid[0] = m.centroid[0] * sx; in.scentroid[1] = m.centroid[1] * sy; in.scentroid[2] = m.centroid[2] * sz;
    ctx->instances.push_back(std::move(in));
    rebuild_arena(ctx);
    cudaSetDevice(ctx->device);
    const int rc = upload_arena(ctx);
    if (rc) { ctx->instances.pop_back(); rebuild_arena(ctx); return rc; }
    *instance_id = int32_t(ctx->instances.size() - 1);
    return 0;
}

int rp3dg_get_convex_mesh_tables(rp3dg_ctx* ctx, int32_t instance_id, uint32_t* nb_vertices, uint32_t* nb_faces,
                                 uint32_t* nb_half_edges, uint32_t* half_edges, float* face_normals,
                                 uint32_t* face_edge, float* centroid, uint32_t cap_he, uint32_t cap_faces) {
    if (!ctx) return RP3DG_EINVAL;
    if (instance_id < 0 || size_t(instance_id) >= ctx->instances.size()) return fail(ctx, RP3DG_EINVAL, "unknown instance");
    const MeshInstance& in = ctx->instances[instance_id];
    const MeshTopo& m = ctx->meshes[in.mesh];
    *nb_vertices = m.nv; *nb_faces = m.nf; *nb_half_edges = uint32_t(m.edges.size());
    if (m.edges.size() > cap_he || m.nf > cap_faces) return fail(ctx, RP3DG_ECAPACITY, "output capacity too small");
    for (size_t e = 0; e < m.edges.size(); e++) {
        half_edges[4 * e] = m.edges[e].vertex; half_edges[4 * e + 1] = m.edges[e].twin;
        half_edges[4 * e + 2] = m.edges[e].face; half_edges[4 * e + 3] = m.edges[e].next;
    }
    std::memcpy(face_normals, in.snormals.data(), in.snormals.size() * sizeof(float));
    std::memcpy(face_edge, m.face_edge.data(), m.face_edge.size() * sizeof(uint32_t));
    std::memcpy(centroid, in.scentroid, 3 * sizeof(float));
    return 0;
}

int rp3dg_create_heightfield(rp3dg_ctx* ctx, uint32_t nb_columns, uint32_t nb_rows, const float* heights,
                             float sx, float sy, float sz, int32_t* heightfield_id) {
    if (!ctx || !heights || !heightfield_id) return fail(ctx, RP3DG_EINVAL, "null argument");
    if (nb_columns < 2 || nb_rows < 2)
        return fail(ctx, RP3DG_EINVAL, "the number of grid columns and grid rows must be at least two");
    if (size_t(nb_columns) * nb_rows > (size_t(1) << 30)) return fail(ctx, RP3DG_EINVAL, "height field too large");
    if (!(sx > 0.0f) || !(sy > 0.0f) || !(sz > 0.0f)) return fail(ctx, RP3DG_EINVAL, "scale must be positive");
    const size_t n = size_t(nb_columns) * nb_rows;
    // HeightField::copyData (HeightField.cpp:93-133): minimum and maximum
    // over the grid, then the height origin
    float mn = heights[0], mx = heights[0];
    for (uint32_t x = 0; x < nb_columns; x++)
        for (uint32_t y = 0; y < nb_rows; y++) {
            const float h = heights[size_t(y) * nb_columns + x];
            if (!(h == h)) return fail(ctx, RP3DG_EINVAL, "height is NaN");
            if (h < mn) mn = h;
            if (h > mx) mx = h;
        }
    rp3dg::HfDesc d{};
    d.ncol = nb_columns;
    d.nrow = nb_rows;
    d.width = float(nb_columns - 1);
    d.length = float(nb_rows - 1);
    d.origin = -(mx - mn) * 0.5f - mn;
    // HeightField::init (:72-79): local bounds centred on the origin
    const float halfHeight = (mx - mn) * 0.5f;
    d.bmin[0] = -d.width * 0.5f; d.bmin[1] = -halfHeight; d.bmin[2] = -d.length * 0.5f;
    d.bmax[0] = d.width * 0.5f;  d.bmax[1] = halfHeight;  d.bmax[2] = d.length * 0.5f;
    d.scale[0] = sx; d.scale[1] = sy; d.scale[2] = sz;
    cudaSetDevice(ctx->device);
    float* dh = nullptr;
    cudaError_t e = cudaMalloc(&dh, n * sizeof(float));
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc(heights)");
    e = cudaMemcpyAsync(dh, heights, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) { cudaFree(dh); return cuda_fail(ctx, e, "upload heights"); }
    d.heights = dh;
    *heightfield_id = int32_t(ctx->hfields.size());
    ctx->hfields.push_back(d);
    return 0;
}

namespace {
float vlen3(const float* a) { return std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }
float vdot3(const float* a, const float* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
void vsub3(const float* a, const float* b, float* o) { o[0] = a[0] - b[0]; o[1] = a[1] - b[1]; o[2] = a[2] - b[2]; }
void vcross3(const float* a, const float* b, float* o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
// Vector3::normalize (Vector3.h:219-227): three divisions, short vectors kept
void vnormalize3(float* a) {
    const float l = vlen3(a);
    if (l < FLT_EPSILON) return;
    a[0] /= l;
    a[1] /= l;
    a[2] /= l;
}
float as_float(int v) {
    float f;
    std::memcpy(&f, &v, 4);
    return f;
}
}  // namespace

int rp3dg_create_triangle_mesh(rp3dg_ctx* ctx, const float* vertices, uint32_t nv, const uint32_t* indices,
                               uint32_t nt, const float* normals, int32_t* mesh_id) {
    if (!ctx || !vertices || !indices || !mesh_id) return fail(ctx, RP3DG_EINVAL, "null argument");
    if (nv == 0 || nt == 0) return fail(ctx, RP3DG_EINVAL, "a triangle mesh needs vertices and triangles");
    // TriangleMesh::computeEpsilon (TriangleMesh.cpp:70-88)
    float mx[3] = {0.0f, 0.0f, 0.0f};
    for (uint32_t i = 0; i < nv; i++)
        for (int k = 0; k < 3; k++) {
            const float a = std::fabs(vertices[3 * size_t(i) + k]);
            if (a > mx[k]) mx[k] = a;
        }
    const float eps = 3 * (mx[0] + mx[1] + mx[2]) * FLT_EPSILON;
    const float eps2 = eps * eps;
    // copyData (:91-214): the triangles of non-zero area and edges, their
    // vertices (and given normals) stored at the user's vertex indices
    TriMesh m;
    m.verts.assign(3 * size_t(nv), 0.0f);
    m.normals.assign(3 * size_t(nv), 0.0f);
    std::vector<uint8_t> used(nv, 0);
    bool valid = true;
    std::string why;
    for (uint32_t i = 0; i < nt; i++) {
        const uint32_t* id = indices + 3 * size_t(i);
        bool face_ok = true;
        for (int v = 0; v < 3; v++)
            if (id[v] >= nv) {
                face_ok = false;
                valid = false;
                why = "the face with index " + std::to_string(i) + " has a vertex index out of range";
            }
        if (!face_ok) continue;
        const float* v1 = vertices + 3 * size_t(id[0]);
        const float* v2 = vertices + 3 * size_t(id[1]);
        const float* v3 = vertices + 3 * size_t(id[2]);
        float e31[3], e21[3], fn[3], e32[3], e13[3];
        vsub3(v3, v1, e31);
        vsub3(v2, v1, e21);
        vcross3(e31, e21, fn);
        const bool zero_area = vdot3(fn, fn) < eps2;
        vsub3(v3, v2, e32);
        vsub3(v1, v3, e13);
        const bool zero_edge = vdot3(e21, e21) < eps2 || vdot3(e32, e32) < eps2 || vdot3(e13, e13) < eps2;
        if (zero_area || zero_edge) continue;
        float vn[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        if (normals)
            for (int v = 0; v < 3; v++) {
                for (int k = 0; k < 3; k++) vn[v][k] = normals[3 * size_t(id[v]) + k];
                if (vdot3(vn[v], vn[v]) < eps2) {
                    valid = false;
                    why = "the provided normal of a vertex is too small";
                }
            }
        const float* vp[3] = {v1, v2, v3};
        for (int v = 0; v < 3; v++) {
            for (int k = 0; k < 3; k++) {
                m.normals[3 * size_t(id[v]) + k] = vn[v][k];
                m.verts[3 * size_t(id[v]) + k] = vp[v][k];
            }
            m.tris.push_back(id[v]);
            used[id[v]] = 1;
        }
    }
    // removeUnusedVertices (:217-240): every unused vertex but the first is
    // removed and the later indices shift down
    std::vector<uint32_t> shift(nv, 0);
    std::vector<float> kv, kn;
    uint32_t removed = 0;
    for (uint32_t i = 0; i < nv; i++) {
        shift[i] = removed;
        if (i > 0 && !used[i]) {
            removed++;
            continue;
        }
        for (int k = 0; k < 3; k++) {
            kv.push_back(m.verts[3 * size_t(i) + k]);
            kn.push_back(m.normals[3 * size_t(i) + k]);
        }
    }
    for (uint32_t& t : m.tris) t -= shift[t];
    m.verts.swap(kv);
    m.normals.swap(kn);
    if (m.tris.empty()) {
        valid = false;
        why = "the mesh does not have any valid triangle faces";
    }
    if (!valid) return fail(ctx, RP3DG_EINVAL, "triangle mesh: " + why);
    const uint32_t nkept = uint32_t(m.tris.size() / 3), nvk = uint32_t(m.verts.size() / 3);
    // computeVerticesNormals (:277-333): angle-weighted face normals
    if (!normals) {
        for (uint32_t f = 0; f < nkept; f++) {
            const float* tv[3] = {&m.verts[3 * size_t(m.tris[3 * f])], &m.verts[3 * size_t(m.tris[3 * f + 1])],
                                  &m.verts[3 * size_t(m.tris[3 * f + 2])]};
            float d[3];
            float len[3];
            vsub3(tv[1], tv[0], d);
            len[0] = vlen3(d);
            vsub3(tv[2], tv[1], d);
            len[1] = vlen3(d);
            vsub3(tv[0], tv[2], d);
            len[2] = vlen3(d);
            for (uint32_t v = 0; v < 3; v++) {
                const uint32_t prev = v == 0 ? 2 : v - 1, next = v == 2 ? 0 : v + 1;
                float a[3], b[3], n[3];
                vsub3(tv[next], tv[v], a);
                vsub3(tv[prev], tv[v], b);
                const float dp = vdot3(a, b);
                const float lab = len[prev] * len[v];
                float cosA = dp / lab;
                cosA = (cosA < 0.0f) ? 0.0f : cosA;   // std::max(cosA, 0)
                cosA = (1.0f < cosA) ? 1.0f : cosA;   // std::min(cosA, 1)
                const float angle = std::acos(cosA);
                vcross3(a, b, n);
                vnormalize3(n);
                float* acc = &m.normals[3 * size_t(m.tris[3 * f + v])];
                for (int k = 0; k < 3; k++) acc[k] += angle * n[k];
            }
        }
        for (uint32_t v = 0; v < nvk; v++) vnormalize3(&m.normals[3 * size_t(v)]);
    }
    // initBVHTree (:242-266): the triangles' AABBs (AABB::createAABBForTriangle,
    // AABB.h:260-282) inserted in order into a tree without fattening
    rp3dg::order::Tree tree;
    for (uint32_t f = 0; f < nkept; f++) {
        const float* p0 = &m.verts[3 * size_t(m.tris[3 * f])];
        const float* p1 = &m.verts[3 * size_t(m.tris[3 * f + 1])];
        const float* p2 = &m.verts[3 * size_t(m.tris[3 * f + 2])];
        rp3dg::order::Box b;
        for (int k = 0; k < 3; k++) {
            b.mn[k] = p0[k];
            b.mx[k] = p0[k];
            if (p1[k] < b.mn[k]) b.mn[k] = p1[k];
        }
        for (int k = 0; k < 3; k++)
            if (p2[k] < b.mn[k]) b.mn[k] = p2[k];
        for (int k = 0; k < 3; k++)
            if (p1[k] > b.mx[k]) b.mx[k] = p1[k];
        for (int k = 0; k < 3; k++)
            if (p2[k] > b.mx[k]) b.mx[k] = p2[k];
        tree.add_object(b, int(f));
    }
    m.nodes.resize(tree.nodes.size());
    for (size_t k = 0; k < tree.nodes.size(); k++) {
        const rp3dg::order::Tree::Node& N = tree.nodes[k];
        const bool leaf = N.height == 0;
        const int c0 = leaf ? -2 - N.data : N.child[0];
        const int c1 = leaf ? -1 : N.child[1];
        m.nodes[k].lo = make_float4(N.box.mn[0], N.box.mn[1], N.box.mn[2], as_float(c0));
        m.nodes[k].hi = make_float4(N.box.mx[0], N.box.mx[1], N.box.mx[2], as_float(c1));
    }
    m.root = tree.root;
    for (int k = 0; k < 3; k++) {
        m.bmin[k] = tree.nodes[size_t(tree.root)].box.mn[k];
        m.bmax[k] = tree.nodes[size_t(tree.root)].box.mx[k];
    }
    *mesh_id = int32_t(ctx->trimeshes.size());
    ctx->trimeshes.push_back(std::move(m));
    return 0;
}

int rp3dg_create_concave_mesh_shape(rp3dg_ctx* ctx, int32_t mesh_id, float sx, float sy, float sz,
                                    int32_t* instance_id) {
    if (!ctx || !instance_id) return fail(ctx, RP3DG_EINVAL, "null argument");
    if (mesh_id < 0 || size_t(mesh_id) >= ctx->trimeshes.size()) return fail(ctx, RP3DG_EINVAL, "unknown triangle mesh");
    if (!(sx > 0.0f) || !(sy > 0.0f) || !(sz > 0.0f)) return fail(ctx, RP3DG_EINVAL, "scale must be positive");
    const TriMesh& m = ctx->trimeshes[size_t(mesh_id)];
    const uint32_t nv = uint32_t(m.verts.size() / 3), nt = uint32_t(m.tris.size() / 3);
    const float sc[3] = {sx, sy, sz};
    // getTriangleVertices (ConcaveMeshShape.cpp:79-89): vertex * scale;
    // computeScaledVerticesNormals (:56-76): Vector3(1.0 / scale) * normal,
    // divided by its length
    std::vector<float> sv(3 * size_t(nv)), sn(3 * size_t(nv));
    const float inv_d[3] = {float(1.0 / double(sx)), float(1.0 / double(sy)), float(1.0 / double(sz))};
    for (uint32_t v = 0; v < nv; v++) {
        float n[3];
        for (int k = 0; k < 3; k++) {
            sv[3 * size_t(v) + k] = m.verts[3 * size_t(v) + k] * sc[k];
            n[k] = inv_d[k] * m.normals[3 * size_t(v) + k];
        }
        const float l = vlen3(n);
        for (int k = 0; k < 3; k++) sn[3 * size_t(v) + k] = n[k] / l;
    }
    rp3dg::CmDesc d{};
    d.nv = nv;
    d.nt = nt;
    d.root = m.root;
    d.mesh = uint32_t(mesh_id);
    for (int k = 0; k < 3; k++) {
        d.scale[k] = sc[k];
        d.inv_scale[k] = 1.0f / sc[k];
    }
    cudaSetDevice(ctx->device);
    uint32_t* dt = nullptr;
    float *dv = nullptr, *dn = nullptr;
    rp3dg::RayNode* dnodes = nullptr;
    cudaError_t e = cudaMalloc(&dt, m.tris.size() * 4);
    if (e == cudaSuccess) e = cudaMalloc(&dv, sv.size() * 4);
    if (e == cudaSuccess) e = cudaMalloc(&dn, sn.size() * 4);
    if (e == cudaSuccess) e = cudaMalloc(&dnodes, m.nodes.size() * sizeof(rp3dg::RayNode));
    if (e == cudaSuccess) e = cudaMemcpyAsync(dt, m.tris.data(), m.tris.size() * 4, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dv, sv.data(), sv.size() * 4, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dn, sn.data(), sn.size() * 4, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dnodes, m.nodes.data(), m.nodes.size() * sizeof(rp3dg::RayNode), cudaMemcpyHostToDevice,
                            ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        cudaFree(dt);
        cudaFree(dv);
        cudaFree(dn);
        cudaFree(dnodes);
        return cuda_fail(ctx, e, "upload concave mesh");
    }
    d.tris = dt;
    d.sverts = dv;
    d.snormals = dn;
    d.nodes = dnodes;
    *instance_id = int32_t(ctx->cmeshes.size());
    ctx->cmeshes.push_back(d);
    return 0;
}

int rp3dg_get_triangle_mesh(rp3dg_ctx* ctx, int32_t mesh_id, uint32_t* nb_vertices, uint32_t* nb_triangles,
                            float* vertices, float* normals, uint32_t* triangles, uint32_t cap_v, uint32_t cap_t) {
    if (!ctx || !nb_vertices || !nb_triangles) return fail(ctx, RP3DG_EINVAL, "null argument");
    if (mesh_id < 0 || size_t(mesh_id) >= ctx->trimeshes.size()) return fail(ctx, RP3DG_EINVAL, "unknown triangle mesh");
    const TriMesh& m = ctx->trimeshes[size_t(mesh_id)];
    *nb_vertices = uint32_t(m.verts.size() / 3);
    *nb_triangles = uint32_t(m.tris.size() / 3);
    const size_t nv = std::min<size_t>(*nb_vertices, cap_v), nt = std::min<size_t>(*nb_triangles, cap_t);
    if (vertices) std::memcpy(vertices, m.verts.data(), nv * 12);
    if (normals) std::memcpy(normals, m.normals.data(), nv * 12);
    if (triangles) std::memcpy(triangles, m.tris.data(), nt * 12);
    return 0;
}

int rp3dg_set_shapes(rp3dg_ctx* ctx, const rp3dg_shape* shapes, uint32_t nb) {
    if (!ctx || (!shapes && nb)) return fail(ctx, RP3DG_EINVAL, "null argument");
    for (uint32_t i = 0; i < nb; i++) {
        const rp3dg_shape& s = shapes[i];
        if (s.kind < RP3DG_SHAPE_SPHERE || s.kind > RP3DG_SHAPE_CONCAVE_MESH) return fail(ctx, RP3DG_EINVAL, "unknown shape kind");
        if (s.kind == RP3DG_SHAPE_CONCAVE_MESH && (s.mesh < 0 || size_t(s.mesh) >= ctx->cmeshes.size()))
            return fail(ctx, RP3DG_EINVAL, "shape refers to an unknown concave mesh instance");
        if (s.kind == RP3DG_SHAPE_HEIGHTFIELD && (s.mesh < 0 || size_t(s.mesh) >= ctx->hfields.size()))
            return fail(ctx, RP3DG_EINVAL, "shape refers to an unknown height field");
        if (s.kind == RP3DG_SHAPE_CONVEX_MESH && (s.mesh < 0 || size_t(s.mesh) >= ctx->instances.size()))
            return fail(ctx, RP3DG_EINVAL, "shape refers to an unknown convex mesh instance");
    }
    cudaSetDevice(ctx->device);
    if (nb > ctx->cap_shapes) {
        cudaFree(ctx->d_shapes);
        ctx->d_shapes = nullptr;
        cudaError_t e = cudaMalloc(&ctx->d_shapes, size_t(nb) * sizeof(rp3dg_shape));
        if (e != cudaSuccess) { ctx->cap_shapes = 0; return cuda_fail(ctx, e, "cudaMalloc(shapes)"); }
        ctx->cap_shapes = nb;
    }
    // local bounds of every shape (CollisionShape::getLocalBounds): sphere
    // (BoxShape.cpp:149-151, SphereShape.h:160-164, CapsuleShape.cpp:90-94),
    // convex mesh: the mesh's vertex bounds (ConvexMesh.cpp:83-99) times the
    // scale (ConvexMeshShape.cpp:208-212, AABB::applyScale)
    std::vector<float> bounds(size_t(nb) * 8, 0.0f);
    for (uint32_t i = 0; i < nb; i++) {
        const rp3dg_shape& sh = shapes[i];
        const float* p = sh.params;
        float* b = &bounds[8 * size_t(i)];
        switch (sh.kind) {
            case RP3DG_SHAPE_SPHERE: b[0] = -p[0]; b[1] = -p[0]; b[2] = -p[0]; b[4] = p[0]; b[5] = p[0]; b[6] = p[0]; break;
            case RP3DG_SHAPE_CAPSULE:
                b[0] = -p[0]; b[1] = -p[1] - p[0]; b[2] = -p[0]; b[4] = p[0]; b[5] = p[1] + p[0]; b[6] = p[0]; break;
            case RP3DG_SHAPE_BOX: b[0] = -p[0]; b[1] = -p[1]; b[2] = -p[2]; b[4] = p[0]; b[5] = p[1]; b[6] = p[2]; break;
            case RP3DG_SHAPE_HEIGHTFIELD: {
                // HeightFieldShape::getLocalBounds (HeightFieldShape.cpp:46-50): bounds * scale
                const rp3dg::HfDesc& h = ctx->hfields[size_t(sh.mesh)];
                for (int k = 0; k < 3; k++) { b[k] = h.bmin[k] * h.scale[k]; b[4 + k] = h.bmax[k] * h.scale[k]; }
                break;
            }
            case RP3DG_SHAPE_CONCAVE_MESH: {
                // ConcaveMeshShape::getLocalBounds (ConcaveMeshShape.cpp:276-285):
                // the triangle tree's root AABB * scale
                const rp3dg::CmDesc& c = ctx->cmeshes[size_t(sh.mesh)];
                const TriMesh& m = ctx->trimeshes[size_t(c.mesh)];
                for (int k = 0; k < 3; k++) { b[k] = m.bmin[k] * c.scale[k]; b[4 + k] = m.bmax[k] * c.scale[k]; }
                break;
            }
            default: {
                const MeshInstance& in = ctx->instances[size_t(sh.mesh)];
                const MeshTopo& m = ctx->meshes[size_t(in.mesh)];
                float mn[3] = {m.verts[0], m.verts[1], m.verts[2]}, mx[3] = {mn[0], mn[1], mn[2]};
                for (uint32_t v = 0; v < m.nv; v++)
                    for (int k = 0; k < 3; k++) {
                        const float x = m.verts[3 * v + k];
                        if (x > mx[k]) mx[k] = x;
                        if (x < mn[k]) mn[k] = x;
                    }
                for (int k = 0; k < 3; k++) { b[k] = mn[k] * in.scale[k]; b[4 + k] = mx[k] * in.scale[k]; }
            }
        }
    }
    if (nb > ctx->cap_shape_bounds) {
        cudaFree(ctx->d_shape_bounds);
        ctx->d_shape_bounds = nullptr;
        cudaError_t e = cudaMalloc(&ctx->d_shape_bounds, bounds.size() * sizeof(float));
        if (e != cudaSuccess) { ctx->cap_shape_bounds = 0; return cuda_fail(ctx, e, "cudaMalloc(shape bounds)"); }
        ctx->cap_shape_bounds = nb;
    }
    if (nb) {
        cudaError_t e = cudaMemcpyAsync(ctx->d_shapes, shapes, size_t(nb) * sizeof(rp3dg_shape), cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(ctx->d_shape_bounds, bounds.data(), bounds.size() * sizeof(float), cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "upload shapes");
    }
    ctx->nb_shapes = nb;
    ctx->host_shapes.assign(shapes, shapes + nb);
    return 0;
}

namespace {
int grow(rp3dg_ctx* ctx, void** buf, size_t* cap, size_t need, const char* what);
int grow_pinned(rp3dg_ctx* ctx, void** buf, size_t* cap, size_t need, const char* what);
// polyhedron batches of at least this many pairs are grouped by class
constexpr uint32_t NP_GROUP_MIN_PAIRS = 4096;

// Checks of a device-array narrow-phase call and the kernel arguments it gives
// (learned proposals off); returns 0 or an error code, 1 for an empty batch.
int np_args(rp3dg_ctx* ctx, int algorithm, const rp3dg_pair_batch* p, const rp3dg_contact_batch* out,
            int clip_with_previous_axis, rp3dg::NpArgs& a) {
    if (!ctx || !p || !out) return fail(ctx, RP3DG_EINVAL, "null argument");
    if (algorithm < RP3DG_ALGO_SPHERE_VS_SPHERE || algorithm > RP3DG_ALGO_CONVEX_POLYHEDRON_VS_CONVEX_POLYHEDRON)
        return fail(ctx, RP3DG_EINVAL, "unknown algorithm");
    if (p->n == 0) return 1;
    if (!p->shape1 || !p->shape2 || !p->pos1 || !p->rot1 || !p->pos2 || !p->rot2)
        return fail(ctx, RP3DG_EINVAL, "null pair array");
    if (!out->is_colliding || !out->nb_contacts || !out->normal_depth || !out->local1 || !out->local2)
        return fail(ctx, RP3DG_EINVAL, "null output array");
    if (out->max_contacts < 1 || out->max_contacts > RP3DG_MAX_CONTACTS_PER_PAIR)
        return fail(ctx, RP3DG_EINVAL, "max_contacts must be in 1..16");
    if (!ctx->d_shapes) return fail(ctx, RP3DG_EINVAL, "no shape table (rp3dg_set_shapes)");
    if (!aligned(p->pos1, 16) || !aligned(p->rot1, 16) || !aligned(p->pos2, 16) || !aligned(p->rot2, 16) ||
        !aligned(p->cache, 16) || !aligned(out->normal_depth, 16) || !aligned(out->local1, 16) ||
        !aligned(out->local2, 16) || !aligned(p->shape1, 4) || !aligned(p->shape2, 4))
        return fail(ctx, RP3DG_EINVAL, "misaligned device array (float4 and cache arrays need 16 bytes, shape ids 4)");
    a.n = p->n;
    a.nb_shapes = ctx->nb_shapes;
    a.error = ctx->d_error;
    a.max_contacts = out->max_contacts;
    a.clip = clip_with_previous_axis ? 1 : 0;
    a.mesh_nwords = uint32_t(ctx->arena.size());
    a.mesh_words = ctx->d_arena;
    a.stage_mesh = (algorithm >= RP3DG_ALGO_SPHERE_VS_CONVEX_POLYHEDRON && a.mesh_nwords > 0 &&
                    size_t(a.mesh_nwords) * 4 <= rp3dg::MESH_STAGE_MAX_BYTES) ? 1 : 0;
    a.shapes = ctx->d_shapes;
    a.shape1 = p->shape1; a.shape2 = p->shape2;
    a.pos1 = reinterpret_cast<const float4*>(p->pos1); a.rot1 = reinterpret_cast<const float4*>(p->rot1);
    a.pos2 = reinterpret_cast<const float4*>(p->pos2); a.rot2 = reinterpret_cast<const float4*>(p->rot2);
    a.report = p->report_contacts;
    a.cache = p->cache;
    a.is_colliding = out->is_colliding;
    a.nb_contacts = out->nb_contacts;
    a.normal_depth = reinterpret_cast<float4*>(out->normal_depth);
    a.local1 = reinterpret_cast<float4*>(out->local1);
    a.local2 = reinterpret_cast<float4*>(out->local2);
    a.mlp = nullptr;
    a.mlp_stats = nullptr;
    a.proposals = nullptr;
    a.tri = nullptr;
    a.perm = nullptr;
    a.events = nullptr;
    a.plist = nullptr;
    a.work = nullptr;
    if (algorithm == RP3DG_ALGO_CONVEX_POLYHEDRON_VS_CONVEX_POLYHEDRON) {
        // the mesh pairs' lists (three of n words) after their six counters
        const size_t words = 3 * size_t(p->n) + 8;
        cudaSetDevice(ctx->device);
        const int rc = grow(ctx, reinterpret_cast<void**>(&ctx->d_plist), &ctx->cap_plist, words * 4,
                            "cudaMalloc(polyhedron pair lists)");
        if (rc) return rc;
        a.work = ctx->d_plist;
        a.plist = ctx->d_plist + 8;
    }
    return 0;
}
}  // namespace

int rp3dg_narrowphase_device(rp3dg_ctx* ctx, int algorithm, const rp3dg_pair_batch* p, const rp3dg_contact_batch* out,
                             int clip_with_previous_axis) {
    rp3dg::NpArgs a;
    const int rc = np_args(ctx, algorithm, p, out, clip_with_previous_axis, a);
    if (rc != 0) return rc > 0 ? 0 : rc;
    const bool learned = ctx->learned_axis && ctx->mlp_ready && algorithm == RP3DG_ALGO_CONVEX_POLYHEDRON_VS_CONVEX_POLYHEDRON;
    a.mlp = learned ? static_cast<const void*>(mlp_packed(ctx)) : nullptr;
    a.mlp_stats = learned ? mlp_stats(ctx) : nullptr;
    cudaSetDevice(ctx->device);
    // plain SAT on a large polyhedron batch: pairs grouped by a geometric
    // class so that the thread-per-pair kernel's tiles are homogeneous
    const bool grouped = !learned && algorithm == RP3DG_ALGO_CONVEX_POLYHEDRON_VS_CONVEX_POLYHEDRON &&
                         p->n >= NP_GROUP_MIN_PAIRS;
    if (learned || grouped) {
        // an order key and a proposal byte per pair, in a buffer that grows
        // with the batch
        if (p->n > ctx->cap_proposals) {
            const uint32_t c = std::max(p->n, 2 * ctx->cap_proposals);
            cudaFree(ctx->d_proposals);
            ctx->d_proposals = nullptr;
            cudaError_t e = cudaMalloc(&ctx->d_proposals, 2 * size_t(c));
            if (e != cudaSuccess) { ctx->cap_proposals = 0; return cuda_fail(ctx, e, "cudaMalloc(proposals)"); }
            ctx->cap_proposals = c;
        }
        uint8_t* key = ctx->d_proposals;
        uint8_t* prop = ctx->d_proposals + p->n;
        cudaError_t e = rp3dg::launch_classify_pairs(a, key, learned ? prop : nullptr, ctx->num_sms, ctx->stream);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "pair classes");
        ctx->launches++;
        if (learned) a.proposals = prop;
        // tiles of one learned class each (the order only, not the results)
        if (p->n > ctx->cap_perm) {
            const uint32_t c = std::max(p->n, 2 * ctx->cap_perm);
            cudaFree(ctx->d_perm);
            ctx->d_perm = nullptr;
            e = cudaMalloc(&ctx->d_perm, (size_t(c) + 32) * sizeof(uint32_t));
            if (e != cudaSuccess) { ctx->cap_perm = 0; return cuda_fail(ctx, e, "cudaMalloc(pair order)"); }
            ctx->cap_perm = c;
        }
        e = rp3dg::launch_partition_by_class(a, key, ctx->d_perm + p->n, ctx->d_perm, ctx->stream);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "pair grouping");
        ctx->launches += 2;
        a.perm = ctx->d_perm;
    }
    int launched = 0;
    cudaError_t e = rp3dg::launch_narrowphase(algorithm, a, ctx->num_sms, ctx->stream, &launched);
    ctx->launches += uint64_t(launched);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "narrowphase launch");
    return 0;
}

int rp3dg_narrowphase_count_events(rp3dg_ctx* ctx, int algorithm, const rp3dg_pair_batch* p,
                                   const rp3dg_contact_batch* out, int clip_with_previous_axis,
                                   unsigned long long* events) {
    if (!events) return fail(ctx, RP3DG_EINVAL, "null events array");
    for (int k = 0; k < RP3DG_NP_EVENTS; k++) events[k] = 0;
    rp3dg::NpArgs a;
    const int rc = np_args(ctx, algorithm, p, out, clip_with_previous_axis, a);
    if (rc != 0) return rc > 0 ? 0 : rc;
    static_assert(RP3DG_NP_EVENTS == rp3dg::NP_EVENT_COUNT, "event array size");
    cudaSetDevice(ctx->device);
    cudaError_t e = cudaSuccess;
    if (!ctx->d_events) e = cudaMalloc(&ctx->d_events, RP3DG_NP_EVENTS * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemsetAsync(ctx->d_events, 0, RP3DG_NP_EVENTS * sizeof(unsigned long long), ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "event counters");
    a.events = ctx->d_events;
    int launched = 0;
    e = rp3dg_events_launch_narrowphase(algorithm, &a, ctx->num_sms, ctx->stream, &launched);
    ctx->launches += uint64_t(launched);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(events, ctx->d_events, RP3DG_NP_EVENTS * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                            ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "narrowphase (event counting)");
    return 0;
}

int rp3dg_reduce_contacts_device(rp3dg_ctx* ctx, const rp3dg_pair_batch* p, const rp3dg_contact_batch* c, uint8_t* kept) {
    if (!ctx || !p || !c) return fail(ctx, RP3DG_EINVAL, "null argument");
    if (p->n == 0) return 0;
    if (!p->rot1 || !c->is_colliding || !c->nb_contacts || !c->normal_depth || !c->local1 || !c->local2)
        return fail(ctx, RP3DG_EINVAL, "null array");
    if (c->max_contacts < 1 || c->max_contacts > RP3DG_MAX_CONTACTS_PER_PAIR)
        return fail(ctx, RP3DG_EINVAL, "max_contacts must be in 1..16");
    if (!aligned(p->rot1, 16) || !aligned(p->cache, 16) || !aligned(c->normal_depth, 16) || !aligned(c->local1, 16) ||
        !aligned(c->local2, 16) || !aligned(kept, 4))
        return fail(ctx, RP3DG_EINVAL, "misaligned device array (float4 arrays need 16 bytes, kept 4)");
    rp3dg::ReduceArgs a;
    a.n = p->n;
    a.max_contacts = c->max_contacts;
    a.rot1 = reinterpret_cast<const float4*>(p->rot1);
    a.cache = p->cache;
    a.is_colliding = c->is_colliding;
    a.nb_contacts = c->nb_contacts;
    a.normal_depth = reinterpret_cast<float4*>(c->normal_depth);
    a.local1 = reinterpret_cast<float4*>(c->local1);
    a.local2 = reinterpret_cast<float4*>(c->local2);
    a.kept = kept;
    cudaSetDevice(ctx->device);
    cudaError_t e = rp3dg::launch_contacts_reduce(a, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "contact reduction");
    ctx->launches++;
    return 0;
}

namespace {

// Host-array narrow phase through the staging buffer; with reduce set, the
// manifold reduction runs on the device before the copy back (kept: n x 4).
int narrowphase_host_impl(rp3dg_ctx* ctx, int algorithm, const rp3dg_pair_batch* p, const rp3dg_contact_batch* out,
                          int clip_with_previous_axis, bool reduce, uint8_t* kept) {
    if (!ctx || !p || !out) return fail(ctx, RP3DG_EINVAL, "null argument");
    if (p->n == 0) return 0;
    if (out->max_contacts < 1 || out->max_contacts > RP3DG_MAX_CONTACTS_PER_PAIR)
        return fail(ctx, RP3DG_EINVAL, "max_contacts must be in 1..16");
    const size_t n = p->n, mc = out->max_contacts;
    // staging layout: inputs then outputs, each array 256-byte aligned
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    size_t off = 0;
    const size_t o_s1 = off; off += al(n * 4);
    const size_t o_s2 = off; off += al(n * 4);
    const size_t o_p1 = off; off += al(n * 16);
    const size_t o_r1 = off; off += al(n * 16);
    const size_t o_p2 = off; off += al(n * 16);
    const size_t o_r2 = off; off += al(n * 16);
    const size_t o_rep = off; off += p->report_contacts ? al(n) : 0;
    const size_t o_cache = off; off += p->cache ? al(n * sizeof(rp3dg_lastframe)) : 0;
    const size_t o_col = off; off += al(n);
    const size_t o_nb = off; off += al(n);
    const size_t o_nd = off; off += al(n * mc * 16);
    const size_t o_l1 = off; off += al(n * mc * 16);
    const size_t o_l2 = off; off += al(n * mc * 16);
    const size_t o_kept = off; off += (reduce && kept) ? al(n * 4) : 0;
    cudaSetDevice(ctx->device);
    if (off > ctx->cap_stage) {
        cudaFree(ctx->d_stage);
        ctx->d_stage = nullptr;
        cudaError_t e = cudaMalloc(&ctx->d_stage, off);
        if (e != cudaSuccess) { ctx->cap_stage = 0; return cuda_fail(ctx, e, "cudaMalloc(staging)"); }
        ctx->cap_stage = off;
    }
    char* b = static_cast<char*>(ctx->d_stage);
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaSuccess;
    auto up = [&](size_t o, const void* src, size_t bytes) {
        if (e == cudaSuccess && src) e = cudaMemcpyAsync(b + o, src, bytes, cudaMemcpyHostToDevice, s);
    };
    up(o_s1, p->shape1, n * 4); up(o_s2, p->shape2, n * 4);
    up(o_p1, p->pos1, n * 16); up(o_r1, p->rot1, n * 16);
    up(o_p2, p->pos2, n * 16); up(o_r2, p->rot2, n * 16);
    up(o_rep, p->report_contacts, n);
    up(o_cache, p->cache, n * sizeof(rp3dg_lastframe));
    if (e != cudaSuccess) return cuda_fail(ctx, e, "upload batch");
    rp3dg_pair_batch dp;
    dp.n = p->n;
    dp.shape1 = reinterpret_cast<const int32_t*>(b + o_s1);
    dp.shape2 = reinterpret_cast<const int32_t*>(b + o_s2);
    dp.pos1 = reinterpret_cast<const rp3dg_float4*>(b + o_p1);
    dp.rot1 = reinterpret_cast<const rp3dg_float4*>(b + o_r1);
    dp.pos2 = reinterpret_cast<const rp3dg_float4*>(b + o_p2);
    dp.rot2 = reinterpret_cast<const rp3dg_float4*>(b + o_r2);
    dp.report_contacts = p->report_contacts ? reinterpret_cast<const uint8_t*>(b + o_rep) : nullptr;
    dp.cache = p->cache ? reinterpret_cast<rp3dg_lastframe*>(b + o_cache) : nullptr;
    rp3dg_contact_batch dout;
    dout.is_colliding = reinterpret_cast<uint8_t*>(b + o_col);
    dout.nb_contacts = reinterpret_cast<uint8_t*>(b + o_nb);
    dout.normal_depth = reinterpret_cast<rp3dg_float4*>(b + o_nd);
    dout.local1 = reinterpret_cast<rp3dg_float4*>(b + o_l1);
    dout.local2 = reinterpret_cast<rp3dg_float4*>(b + o_l2);
    dout.max_contacts = out->max_contacts;
    int rc = rp3dg_narrowphase_device(ctx, algorithm, &dp, &dout, clip_with_previous_axis);
    if (rc) return rc;
    if (reduce) {
        rc = rp3dg_reduce_contacts_device(ctx, &dp, &dout, kept ? reinterpret_cast<uint8_t*>(b + o_kept) : nullptr);
        if (rc) return rc;
    }
    auto down = [&](void* dst, size_t o, size_t bytes) {
        if (e == cudaSuccess && dst) e = cudaMemcpyAsync(dst, b + o, bytes, cudaMemcpyDeviceToHost, s);
    };
    if (reduce) down(kept, o_kept, n * 4);
    down(out->is_colliding, o_col, n);
    down(out->nb_contacts, o_nb, n);
    down(p->cache, o_cache, p->cache ? n * sizeof(rp3dg_lastframe) : 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "narrowphase (host arrays)");
    // copy back only the slots in use (slot-major: slot k of every pair is contiguous)
    uint32_t used = 0;
    for (size_t i = 0; i < n; i++) used = out->nb_contacts[i] > used ? out->nb_contacts[i] : used;
    down(out->normal_depth, o_nd, n * used * 16);
    down(out->local1, o_l1, n * used * 16);
    down(out->local2, o_l2, n * used * 16);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = cudaGetLastError();
    return e == cudaSuccess ? 0 : cuda_fail(ctx, e, "narrowphase (host arrays)");
}

}  // namespace

int rp3dg_narrowphase_host(rp3dg_ctx* ctx, int algorithm, const rp3dg_pair_batch* p, const rp3dg_contact_batch* out,
                           int clip_with_previous_axis) {
    return narrowphase_host_impl(ctx, algorithm, p, out, clip_with_previous_axis, false, nullptr);
}

int rp3dg_narrowphase_manifolds_host(rp3dg_ctx* ctx, int algorithm, const rp3dg_pair_batch* p,
                                     const rp3dg_contact_batch* out, int clip_with_previous_axis, uint8_t* kept) {
    return narrowphase_host_impl(ctx, algorithm, p, out, clip_with_previous_axis, true, kept);
}

int rp3dg_narrowphase_input_host(rp3dg_ctx* ctx, uint32_t nb, const int32_t* algos, const rp3dg_pair_batch* P,
                                 const rp3dg_contact_batch* O, int clip) {
    if (!ctx || (nb && (!algos || !P || !O))) return fail(ctx, RP3DG_EINVAL, "null argument");
    // device staging of a batch: its inputs, then one block of flags, counts,
    // group starts and the record count (copied to the host in one piece),
    // the slot-major contacts and the packed records; host staging: that
    // block and the cache, then the records.  A batch whose pair count is
    // the one of the same batch in the last call expects about as many
    // records as then: that many (plus an eighth and 64) are copied back
    // right after the flags, without waiting for the count; a batch with
    // more records, or none expected, is copied once its count is known.
    struct Lay {
        size_t s1, s2, p1, r1, p2, r2, rep, cache, col, nbc, ws, cnt, meta, nd, l1, l2, rec;
        size_t h_meta, h_cache, h_rec, h_spec;
        uint32_t groups, expect;
        bool spec;
    };
    std::vector<Lay> L(nb);
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    size_t off = 0, hoff = 0, hspec = 0;
    if (ctx->last_pairs.size() != nb) {
        ctx->last_pairs.assign(nb, 0);
        ctx->last_records.assign(nb, 0);
    }
    for (uint32_t b = 0; b < nb; b++) {
        const rp3dg_pair_batch& p = P[b];
        const rp3dg_contact_batch& o = O[b];
        if (p.n == 0) continue;
        if (!p.shape1 || !p.shape2 || !p.pos1 || !p.rot1 || !p.pos2 || !p.rot2)
            return fail(ctx, RP3DG_EINVAL, "null pair array");
        if (!o.is_colliding || !o.nb_contacts || !o.normal_depth || !o.local1 || !o.local2)
            return fail(ctx, RP3DG_EINVAL, "null contact array");
        if (o.max_contacts < 1 || o.max_contacts > RP3DG_MAX_CONTACTS_PER_PAIR)
            return fail(ctx, RP3DG_EINVAL, "max_contacts must be in 1..16");
        const size_t n = p.n, mc = o.max_contacts;
        Lay& l = L[b];
        l.groups = uint32_t((n + 31) / 32);
        l.s1 = off; off += al(n * 4);
        l.s2 = off; off += al(n * 4);
        l.p1 = off; off += al(n * 16);
        l.r1 = off; off += al(n * 16);
        l.p2 = off; off += al(n * 16);
        l.r2 = off; off += al(n * 16);
        l.rep = off; off += p.report_contacts ? al(n) : 0;
        l.cache = off; off += p.cache ? al(n * sizeof(rp3dg_lastframe)) : 0;
        l.col = off;
        l.nbc = l.col + al(n);
        l.ws = l.nbc + al(n);
        l.cnt = l.ws + al(size_t(l.groups) * 4);
        l.meta = l.cnt + 4 - l.col;
        off = l.col + al(l.meta);
        l.nd = off; off += al(n * mc * 16);
        l.l1 = off; off += al(n * mc * 16);
        l.l2 = off; off += al(n * mc * 16);
        l.rec = off; off += al(n * mc * 48);
        l.h_meta = hoff; hoff += al(l.meta);
        l.h_cache = hoff; hoff += p.cache ? al(n * sizeof(rp3dg_lastframe)) : 0;
        l.h_rec = 0;
        l.spec = false;
        l.expect = 0;
        if (ctx->last_pairs[b] == p.n && ctx->last_records[b])
            l.expect = uint32_t(std::min<size_t>(size_t(ctx->last_records[b]) + ctx->last_records[b] / 8 + 64, n * mc));
        l.h_spec = hspec;
        hspec += al(size_t(l.expect) * 48);
    }
    cudaSetDevice(ctx->device);
    int rc = grow(ctx, &ctx->d_istage, &ctx->cap_istage, std::max<size_t>(off, 256), "cudaMalloc(narrow-phase input)");
    if (!rc) rc = grow_pinned(ctx, &ctx->h_imeta, &ctx->cap_imeta, std::max<size_t>(hoff, 256), "cudaMallocHost(narrow-phase results)");
    if (!rc && hspec)
        rc = grow_pinned(ctx, &ctx->h_ispec, &ctx->cap_ispec, hspec, "cudaMallocHost(narrow-phase contacts)");
    if (rc) return rc;
    cudaError_t e = cudaSuccess;
    if (!ctx->s_up) e = cudaStreamCreateWithFlags(&ctx->s_up, cudaStreamNonBlocking);
    if (e == cudaSuccess && !ctx->s_pub) e = cudaStreamCreateWithFlags(&ctx->s_pub, cudaStreamNonBlocking);
    if (e == cudaSuccess && !ctx->s_rec) e = cudaStreamCreateWithFlags(&ctx->s_rec, cudaStreamNonBlocking);
    while (e == cudaSuccess && ctx->events.size() < 4 * size_t(nb)) {
        cudaEvent_t ev;
        e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e == cudaSuccess) ctx->events.push_back(ev);
    }
    if (e != cudaSuccess) return cuda_fail(ctx, e, "narrow-phase input streams");
    char* base = static_cast<char*>(ctx->d_istage);
    char* hmeta = static_cast<char*>(ctx->h_imeta);
    cudaEvent_t* ev_up = ctx->events.data();
    cudaEvent_t* ev_comp = ev_up + nb;
    cudaEvent_t* ev_meta = ev_comp + nb;
    cudaEvent_t* ev_rec = ev_meta + nb;
    // The batches are independent, so they go in order of decreasing
    // estimated kernel time: the long polyhedron batches compute while the
    // others upload.
    std::vector<uint32_t> order(nb);
    for (uint32_t b = 0; b < nb; b++) order[b] = b;
    auto cost = [&](uint32_t b) {
        static const double per_pair[7] = {0.0, 1.0, 1.0, 1.2, 4.0, 8.0, 20.0};
        const int a = algos[b];
        double c = (a >= 1 && a <= 6 ? per_pair[a] : 1.0) * double(P[b].n);
        // a polyhedron batch whose first pair has a convex mesh: hull work
        if (a == RP3DG_ALGO_CONVEX_POLYHEDRON_VS_CONVEX_POLYHEDRON && P[b].n) {
            const int32_t s1 = P[b].shape1[0], s2 = P[b].shape2[0];
            const size_t ns = ctx->host_shapes.size();
            if ((s1 >= 0 && size_t(s1) < ns && ctx->host_shapes[size_t(s1)].kind == RP3DG_SHAPE_CONVEX_MESH) ||
                (s2 >= 0 && size_t(s2) < ns && ctx->host_shapes[size_t(s2)].kind == RP3DG_SHAPE_CONVEX_MESH))
                c *= 3.0;
        }
        return c;
    };
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return cost(x) > cost(y); });
    // 1. every batch: upload (s_up), kernels and the packing of its contacts
    // (context stream), its flags / counts / group starts / record count and
    // cache to the host (s_pub); each stream waits on the stage before it
    uint32_t queued = 0;
    for (uint32_t ob = 0; ob < nb && rc == 0 && e == cudaSuccess; ob++) {
        const uint32_t b = order[ob];
        const rp3dg_pair_batch& p = P[b];
        const rp3dg_contact_batch& o = O[b];
        if (p.n == 0) continue;
        const Lay& l = L[b];
        const size_t n = p.n;
        auto up = [&](size_t at, const void* src, size_t bytes) {
            if (e == cudaSuccess && src) e = cudaMemcpyAsync(base + at, src, bytes, cudaMemcpyHostToDevice, ctx->s_up);
        };
        up(l.s1, p.shape1, n * 4); up(l.s2, p.shape2, n * 4);
        up(l.p1, p.pos1, n * 16); up(l.r1, p.rot1, n * 16);
        up(l.p2, p.pos2, n * 16); up(l.r2, p.rot2, n * 16);
        up(l.rep, p.report_contacts, n);
        up(l.cache, p.cache, n * sizeof(rp3dg_lastframe));
        if (e == cudaSuccess) e = cudaEventRecord(ev_up[b], ctx->s_up);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->stream, ev_up[b], 0);
        if (e != cudaSuccess) break;
        rp3dg_pair_batch dp;
        dp.n = p.n;
        dp.shape1 = reinterpret_cast<const int32_t*>(base + l.s1);
        dp.shape2 = reinterpret_cast<const int32_t*>(base + l.s2);
        dp.pos1 = reinterpret_cast<const rp3dg_float4*>(base + l.p1);
        dp.rot1 = reinterpret_cast<const rp3dg_float4*>(base + l.r1);
        dp.pos2 = reinterpret_cast<const rp3dg_float4*>(base + l.p2);
        dp.rot2 = reinterpret_cast<const rp3dg_float4*>(base + l.r2);
        dp.report_contacts = p.report_contacts ? reinterpret_cast<const uint8_t*>(base + l.rep) : nullptr;
        dp.cache = p.cache ? reinterpret_cast<rp3dg_lastframe*>(base + l.cache) : nullptr;
        rp3dg_contact_batch dout;
        dout.is_colliding = reinterpret_cast<uint8_t*>(base + l.col);
        dout.nb_contacts = reinterpret_cast<uint8_t*>(base + l.nbc);
        dout.normal_depth = reinterpret_cast<rp3dg_float4*>(base + l.nd);
        dout.local1 = reinterpret_cast<rp3dg_float4*>(base + l.l1);
        dout.local2 = reinterpret_cast<rp3dg_float4*>(base + l.l2);
        dout.max_contacts = o.max_contacts;
        rc = rp3dg_narrowphase_device(ctx, algos[b], &dp, &dout, clip);
        if (rc) break;
        rp3dg::CompactArgs ca;
        ca.n = p.n;
        ca.nb = dout.nb_contacts;
        ca.nd = reinterpret_cast<const float4*>(dout.normal_depth);
        ca.l1 = reinterpret_cast<const float4*>(dout.local1);
        ca.l2 = reinterpret_cast<const float4*>(dout.local2);
        ca.records = reinterpret_cast<float4*>(base + l.rec);
        ca.warp_start = reinterpret_cast<uint32_t*>(base + l.ws);
        ca.counter = reinterpret_cast<uint32_t*>(base + l.cnt);
        e = cudaMemsetAsync(ca.counter, 0, 4, ctx->stream);
        if (e == cudaSuccess) e = rp3dg::launch_compact_contacts(ca, ctx->stream);
        ctx->launches++;
        if (e == cudaSuccess) e = cudaEventRecord(ev_comp[b], ctx->stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->s_pub, ev_comp[b], 0);
        if (e == cudaSuccess) e = cudaMemcpyAsync(hmeta + l.h_meta, base + l.col, l.meta, cudaMemcpyDeviceToHost, ctx->s_pub);
        if (e == cudaSuccess && p.cache)
            e = cudaMemcpyAsync(hmeta + l.h_cache, base + l.cache, n * sizeof(rp3dg_lastframe), cudaMemcpyDeviceToHost,
                                ctx->s_pub);
        if (e == cudaSuccess && l.expect)
            e = cudaMemcpyAsync(static_cast<char*>(ctx->h_ispec) + l.h_spec, base + l.rec, size_t(l.expect) * 48,
                                cudaMemcpyDeviceToHost, ctx->s_pub);
        if (e == cudaSuccess) e = cudaEventRecord(ev_meta[b], ctx->s_pub);
        queued = ob + 1;
    }
    // 2. as each batch's count arrives: its records to the host (s_rec), and
    // the batches whose records are in scattered into the caller's arrays on
    // the host threads while the later batches are still on the GPU
    auto scatter = [&](uint32_t b) {
        const rp3dg_pair_batch& p = P[b];
        const rp3dg_contact_batch& o = O[b];
        const Lay& l = L[b];
        const size_t n = p.n;
        const uint8_t* col = reinterpret_cast<const uint8_t*>(hmeta + l.h_meta);
        const uint8_t* cnt = col + (l.nbc - l.col);
        const uint32_t* ws = reinterpret_cast<const uint32_t*>(col + (l.ws - l.col));
        // the caller's arrays need only 4-byte alignment: plain struct copies
        const rp3dg_float4* rec = reinterpret_cast<const rp3dg_float4*>(
            l.spec ? static_cast<char*>(ctx->h_ispec) + l.h_spec : static_cast<char*>(ctx->h_irec) + l.h_rec);
        std::memcpy(o.is_colliding, col, n);
        std::memcpy(o.nb_contacts, cnt, n);
        if (p.cache) std::memcpy(p.cache, hmeta + l.h_cache, n * sizeof(rp3dg_lastframe));
        rp3dg_float4* nd = o.normal_depth;
        rp3dg_float4* l1 = o.local1;
        rp3dg_float4* l2 = o.local2;
        const long groups = long(l.groups);
#pragma omp parallel for schedule(static) if (groups >= 2048)
        for (long g = 0; g < groups; g++) {
            size_t r = ws[g];
            const size_t i1 = std::min(n, size_t(g + 1) * 32);
            for (size_t i = size_t(g) * 32; i < i1; i++)
                for (uint32_t k = 0; k < cnt[i]; k++, r++) {
                    const size_t at = size_t(k) * n + i;
                    nd[at] = rec[3 * r];
                    l1[at] = rec[3 * r + 1];
                    l2[at] = rec[3 * r + 2];
                }
        }
    };
    std::vector<uint32_t> pending;   // records on their way, in order
    size_t rec_used = 0;
    for (uint32_t ob = 0; ob < queued && rc == 0 && e == cudaSuccess; ob++) {
        const uint32_t b = order[ob];
        if (P[b].n == 0) continue;
        Lay& l = L[b];
        e = cudaEventSynchronize(ev_meta[b]);
        if (e != cudaSuccess) break;
        uint32_t total = 0;
        std::memcpy(&total, hmeta + l.h_meta + (l.cnt - l.col), 4);
        if (size_t(total) > size_t(P[b].n) * O[b].max_contacts) {
            rc = fail(ctx, RP3DG_ECUDA, "narrow-phase contact count out of range");
            break;
        }
        ctx->last_pairs[b] = P[b].n;
        ctx->last_records[b] = total;
        l.spec = total <= l.expect;
        if (l.spec) {
            // the records came back with the flags
            scatter(b);
            continue;
        }
        const size_t need = al(size_t(total) * 48);
        if (rec_used + need > ctx->cap_irec) {
            // the pending batches are finished first; then the staging grows
            for (uint32_t q : pending) {
                e = cudaEventSynchronize(ev_rec[q]);
                if (e != cudaSuccess) break;
                scatter(q);
            }
            pending.clear();
            rec_used = 0;
            if (e != cudaSuccess) break;
            rc = grow_pinned(ctx, &ctx->h_irec, &ctx->cap_irec, std::max<size_t>(need, 256),
                             "cudaMallocHost(narrow-phase contacts)");
            if (rc) break;
        }
        l.h_rec = rec_used;
        rec_used += need;
        if (total)
            e = cudaMemcpyAsync(static_cast<char*>(ctx->h_irec) + l.h_rec, base + l.rec, size_t(total) * 48,
                                cudaMemcpyDeviceToHost, ctx->s_rec);
        if (e == cudaSuccess) e = cudaEventRecord(ev_rec[b], ctx->s_rec);
        if (e != cudaSuccess) break;
        while (!pending.empty()) {
            const cudaError_t q = cudaEventQuery(ev_rec[pending.front()]);
            if (q == cudaErrorNotReady) {
                (void)cudaGetLastError();   // not an error: the copy is still running
                break;
            }
            if (q != cudaSuccess) {
                e = q;
                break;
            }
            scatter(pending.front());
            pending.erase(pending.begin());
        }
        pending.push_back(b);
    }
    for (uint32_t q : pending) {
        if (rc || e != cudaSuccess) break;
        e = cudaEventSynchronize(ev_rec[q]);
        if (e == cudaSuccess) scatter(q);
    }
    // every stream drained before returning (also after an error)
    const cudaError_t e1 = cudaStreamSynchronize(ctx->s_up);
    const cudaError_t e2 = cudaStreamSynchronize(ctx->stream);
    const cudaError_t e3 = cudaStreamSynchronize(ctx->s_pub);
    const cudaError_t e4 = cudaStreamSynchronize(ctx->s_rec);
    if (rc) return rc;
    if (e == cudaSuccess) e = e1 != cudaSuccess ? e1 : (e2 != cudaSuccess ? e2 : (e3 != cudaSuccess ? e3 : e4));
    if (e == cudaSuccess) e = cudaGetLastError();
    return e == cudaSuccess ? 0 : cuda_fail(ctx, e, "narrow-phase input (host arrays)");
}

namespace {

int ensure_mlp(rp3dg_ctx* ctx) {
    if (ctx->d_mlp) return 0;
    cudaError_t e = cudaMalloc(&ctx->d_mlp, MLP_BLOCK_BYTES);
    if (e != cudaSuccess) { ctx->d_mlp = nullptr; return cuda_fail(ctx, e, "cudaMalloc(mlp)"); }
    e = cudaMemsetAsync(ctx->d_mlp, 0, MLP_BLOCK_BYTES, ctx->stream);
    return e == cudaSuccess ? 0 : cuda_fail(ctx, e, "clear mlp state");
}

int mlp_repack(rp3dg_ctx* ctx) {
    cudaError_t e = rp3dg::launch_mlp_pack(mlp_params(ctx), mlp_packed(ctx), ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "mlp pack");
    ctx->launches++;
    ctx->mlp_ready = true;
    return 0;
}

int mlp_pair_args(rp3dg_ctx* ctx, const rp3dg_pair_batch* p, rp3dg::MlpPairArgs& a) {
    if (!p->shape1 || !p->shape2 || !p->pos1 || !p->rot1 || !p->pos2 || !p->rot2) return fail(ctx, RP3DG_EINVAL, "null pair array");
    if (!ctx->d_shapes) return fail(ctx, RP3DG_EINVAL, "no shape table (rp3dg_set_shapes)");
    a.n = p->n;
    a.nb_shapes = ctx->nb_shapes;
    a.shapes = ctx->d_shapes;
    a.shape1 = p->shape1; a.shape2 = p->shape2;
    a.pos1 = reinterpret_cast<const float4*>(p->pos1); a.rot1 = reinterpret_cast<const float4*>(p->rot1);
    a.pos2 = reinterpret_cast<const float4*>(p->pos2); a.rot2 = reinterpret_cast<const float4*>(p->rot2);
    a.mesh_words = ctx->d_arena;
    a.box = nullptr;
    return 0;
}

int mlp_grads_into(rp3dg_ctx* ctx, const float* x, const uint8_t* y, uint32_t n, float* grads, float* loss) {
    const size_t need = size_t(n) * rp3dg::MLP_SCRATCH_ROW * sizeof(float);
    if (need > ctx->cap_mlp_scratch) {
        cudaFree(ctx->d_mlp_scratch);
        ctx->d_mlp_scratch = nullptr;
        cudaError_t e = cudaMalloc(&ctx->d_mlp_scratch, need);
        if (e != cudaSuccess) { ctx->cap_mlp_scratch = 0; return cuda_fail(ctx, e, "cudaMalloc(mlp scratch)"); }
        ctx->cap_mlp_scratch = need;
    }
    cudaError_t e = cudaMemsetAsync(mlp_loss(ctx), 0, sizeof(float), ctx->stream);
    if (e == cudaSuccess) e = rp3dg::launch_mlp_grads(mlp_params(ctx), x, y, n, ctx->d_mlp_scratch, grads, mlp_loss(ctx), ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "mlp gradients");
    ctx->launches += 2;
    if (loss) {
        float sum = 0.0f;
        e = cudaMemcpyAsync(&sum, mlp_loss(ctx), sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "read mlp loss");
        *loss = sum / float(n);
    }
    return 0;
}

}  // namespace

int rp3dg_axis_mlp_init(rp3dg_ctx* ctx, uint64_t seed) {
    if (!ctx) return RP3DG_EINVAL;
    cudaSetDevice(ctx->device);
    int rc = ensure_mlp(ctx);
    if (rc) return rc;
    // He-uniform weights from a splitmix64 stream, zero biases
    std::vector<float> p(RP3DG_MLP_NPARAMS, 0.0f);
    uint64_t st = seed;
    auto next = [&st]() {
        uint64_t z = (st += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return double((z ^ (z >> 31)) >> 11) * (1.0 / 9007199254740992.0);
    };
    auto fill = [&](int off, int fan_in, int count) {
        const double lim = std::sqrt(6.0 / fan_in);
        for (int k = 0; k < count; k++) p[off + k] = float((2.0 * next() - 1.0) * lim);
    };
    fill(rp3dg::MLP_OFF_W1, rp3dg::MLP_IN, rp3dg::MLP_IN * rp3dg::MLP_H);
    fill(rp3dg::MLP_OFF_W2, rp3dg::MLP_H, rp3dg::MLP_H * rp3dg::MLP_H);
    fill(rp3dg::MLP_OFF_W3, rp3dg::MLP_H, rp3dg::MLP_H * rp3dg::MLP_OUT);
    cudaError_t e = cudaMemcpyAsync(mlp_params(ctx), p.data(), MLP_PARAM_BYTES, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(mlp_m(ctx), 0, 2 * MLP_PARAM_BYTES, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "mlp init");
    ctx->mlp_step = 0;
    return mlp_repack(ctx);
}

int rp3dg_axis_mlp_get_params(rp3dg_ctx* ctx, float* params) {
    if (!ctx || !params) return fail(ctx, RP3DG_EINVAL, "null argument");
    if (!ctx->d_mlp) return fail(ctx, RP3DG_EINVAL, "mlp not initialised");
    cudaSetDevice(ctx->device);
    cudaError_t e = cudaMemcpyAsync(params, mlp_params(ctx), MLP_PARAM_BYTES, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    return e == cudaSuccess ? 0 : cuda_fail(ctx, e, "read mlp params");
}

int rp3dg_axis_mlp_set_params(rp3dg_ctx* ctx, const float* params) {
    if (!ctx || !params) return fail(ctx, RP3DG_EINVAL, "null argument");
    cudaSetDevice(ctx->device);
    int rc = ensure_mlp(ctx);
    if (rc) return rc;
    cudaError_t e = cudaMemcpyAsync(mlp_params(ctx), params, MLP_PARAM_BYTES, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "write mlp params");
    return mlp_repack(ctx);
}

int rp3dg_axis_features(rp3dg_ctx* ctx, const rp3dg_pair_batch* p, float* features) {
    if (!ctx || !p || !features) return fail(ctx, RP3DG_EINVAL, "null argument");
    rp3dg::MlpPairArgs a;
    int rc = mlp_pair_args(ctx, p, a);
    if (rc) return rc;
    cudaSetDevice(ctx->device);
    cudaError_t e = rp3dg::launch_axis_features(a, features, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "axis features");
    ctx->launches += p->n ? 1 : 0;
    return 0;
}

int rp3dg_axis_labels(rp3dg_ctx* ctx, const rp3dg_pair_batch* p, const uint8_t* is_colliding, uint8_t* labels) {
    if (!ctx || !p || !is_colliding || !labels || !p->cache) return fail(ctx, RP3DG_EINVAL, "null argument (labels need the cache)");
    rp3dg::MlpPairArgs a;
    int rc = mlp_pair_args(ctx, p, a);
    if (rc) return rc;
    cudaSetDevice(ctx->device);
    cudaError_t e = rp3dg::launch_axis_labels(a, is_colliding, p->cache, labels, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "axis labels");
    ctx->launches += p->n ? 1 : 0;
    return 0;
}

int rp3dg_axis_mlp_grads(rp3dg_ctx* ctx, const float* x, const uint8_t* y, uint32_t n, float* grads, float* loss) {
    if (!ctx || !x || !y || !grads || n == 0) return fail(ctx, RP3DG_EINVAL, "bad argument");
    if (!ctx->d_mlp) return fail(ctx, RP3DG_EINVAL, "mlp not initialised");
    cudaSetDevice(ctx->device);
    return mlp_grads_into(ctx, x, y, n, grads, loss);
}

int rp3dg_axis_mlp_grads_noalloc(rp3dg_ctx* ctx, const float* x, const uint8_t* y, uint32_t n, float* grads,
                                 float* loss) {
    if (!ctx || !x || !y || !grads || n == 0) return fail(ctx, RP3DG_EINVAL, "bad argument");
    if (n > rp3dg::MLP_NOALLOC_MAX_SAMPLES)
        return fail(ctx, RP3DG_ECAPACITY, "rp3dg_axis_mlp_grads_noalloc takes at most 4096 samples per call");
    if (!ctx->d_mlp) return fail(ctx, RP3DG_EINVAL, "mlp not initialised");
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e == cudaSuccess) e = rp3dg::launch_mlp_grads_noalloc(mlp_params(ctx), x, y, n, grads, loss, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "mlp gradients (no allocation)");
    ctx->launches += 2;
    return 0;
}

int rp3dg_axis_mlp_train_step(rp3dg_ctx* ctx, const float* x, const uint8_t* y, uint32_t n, float lr, float* loss) {
    if (!ctx || !x || !y || n == 0) return fail(ctx, RP3DG_EINVAL, "bad argument");
    if (!ctx->d_mlp) return fail(ctx, RP3DG_EINVAL, "mlp not initialised");
    cudaSetDevice(ctx->device);
    int rc = mlp_grads_into(ctx, x, y, n, mlp_g(ctx), loss);
    if (rc) return rc;
    ctx->mlp_step++;
    cudaError_t e = rp3dg::launch_mlp_adam(mlp_params(ctx), mlp_g(ctx), mlp_m(ctx), mlp_v(ctx), lr, ctx->mlp_step, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "mlp adam");
    ctx->launches++;
    return mlp_repack(ctx);
}

int rp3dg_axis_mlp_predict(rp3dg_ctx* ctx, const float* x, uint32_t n, uint8_t* classes) {
    if (!ctx || !x || !classes) return fail(ctx, RP3DG_EINVAL, "null argument");
    if (!ctx->mlp_ready) return fail(ctx, RP3DG_EINVAL, "mlp not initialised");
    cudaSetDevice(ctx->device);
    cudaError_t e = rp3dg::launch_mlp_predict(mlp_packed(ctx), x, n, classes, ctx->num_sms, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "mlp predict");
    ctx->launches += n ? 1 : 0;
    return 0;
}

int rp3dg_set_learned_axis(rp3dg_ctx* ctx, int enable) {
    if (!ctx) return RP3DG_EINVAL;
    if (enable && !ctx->mlp_ready) return fail(ctx, RP3DG_EINVAL, "mlp not initialised");
    ctx->learned_axis = enable != 0;
    return 0;
}

int rp3dg_learned_axis_stats(rp3dg_ctx* ctx, uint64_t* tested, uint64_t* confirmed, int clear) {
    if (!ctx || !tested || !confirmed) return fail(ctx, RP3DG_EINVAL, "null argument");
    if (!ctx->d_mlp) { *tested = *confirmed = 0; return 0; }
    cudaSetDevice(ctx->device);
    unsigned long long h[2] = {0, 0};
    cudaError_t e = cudaMemcpyAsync(h, mlp_stats(ctx), sizeof(h), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess && clear) e = cudaMemsetAsync(mlp_stats(ctx), 0, sizeof(h), ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "read learned-axis stats");
    *tested = h[0];
    *confirmed = h[1];
    return 0;
}

}  // extern "C"

namespace rp3dg {
// Triangle tests of one algorithm batch of the world step (device arrays,
// asynchronous): like rp3dg_narrowphase_device, with the TriangleShape of
// each test in tri (the triangle side has shape index -1).
int narrowphase_tri_device(rp3dg_ctx* ctx, int algorithm, const rp3dg_pair_batch* p, const rp3dg_contact_batch* out,
                           const float4* tri) {
    if (!ctx || !p || !out || !tri) return fail(ctx, RP3DG_EINVAL, "null argument");
    if (algorithm < RP3DG_ALGO_SPHERE_VS_CONVEX_POLYHEDRON || algorithm > RP3DG_ALGO_CONVEX_POLYHEDRON_VS_CONVEX_POLYHEDRON)
        return fail(ctx, RP3DG_EINVAL, "triangle tests need a convex-polyhedron algorithm");
    if (p->n == 0) return 0;
    if (!ctx->d_shapes) return fail(ctx, RP3DG_EINVAL, "no shape table (rp3dg_set_shapes)");
    NpArgs a;
    a.n = p->n;
    a.nb_shapes = ctx->nb_shapes;
    a.error = ctx->d_error;
    a.max_contacts = out->max_contacts;
    a.clip = 1;
    a.mesh_nwords = uint32_t(ctx->arena.size());
    a.mesh_words = ctx->d_arena;
    a.stage_mesh = (a.mesh_nwords > 0 && size_t(a.mesh_nwords) * 4 <= MESH_STAGE_MAX_BYTES) ? 1 : 0;
    a.shapes = ctx->d_shapes;
    a.shape1 = p->shape1; a.shape2 = p->shape2;
    a.pos1 = reinterpret_cast<const float4*>(p->pos1); a.rot1 = reinterpret_cast<const float4*>(p->rot1);
    a.pos2 = reinterpret_cast<const float4*>(p->pos2); a.rot2 = reinterpret_cast<const float4*>(p->rot2);
    a.report = p->report_contacts;
    a.cache = p->cache;
    a.is_colliding = out->is_colliding;
    a.nb_contacts = out->nb_contacts;
    a.normal_depth = reinterpret_cast<float4*>(out->normal_depth);
    a.local1 = reinterpret_cast<float4*>(out->local1);
    a.local2 = reinterpret_cast<float4*>(out->local2);
    a.mlp = nullptr;
    a.mlp_stats = nullptr;
    a.proposals = nullptr;
    a.tri = tri;
    a.perm = nullptr;
    cudaError_t e = launch_narrowphase_tri(algorithm, a, ctx->num_sms, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "triangle narrow-phase launch");
    ctx->launches++;
    return 0;
}
}  // namespace rp3dg

// ---- dynamics stage ------------------------------------------------------

namespace {

// Device scratch that only grows, doubling, so that a world whose sizes creep
// up step after step reallocates (a cudaFree waits for the device) rarely.
int grow(rp3dg_ctx* ctx, void** buf, size_t* cap, size_t need, const char* what) {
    if (need <= *cap) return 0;
    const size_t n = std::max(need, 2 * *cap);
    cudaFree(*buf);
    *buf = nullptr;
    cudaError_t e = cudaMalloc(buf, n);
    if (e != cudaSuccess) { *cap = 0; *buf = nullptr; return cuda_fail(ctx, e, what); }
    *cap = n;
    return 0;
}

// The same for page-locked host memory (old contents are not kept).
int grow_pinned(rp3dg_ctx* ctx, void** buf, size_t* cap, size_t need, const char* what) {
    if (need <= *cap) return 0;
    const size_t n = std::max(need, 2 * *cap);
    cudaFreeHost(*buf);
    *buf = nullptr;
    cudaError_t e = cudaMallocHost(buf, n);
    if (e != cudaSuccess) { *cap = 0; *buf = nullptr; return cuda_fail(ctx, e, what); }
    *cap = n;
    return 0;
}

int check_dynamics(rp3dg_ctx* ctx, const rp3dg_dynamics_params* pr, const rp3dg_bodies* b, const rp3dg_colliders* c,
                   const rp3dg_manifolds* m, const rp3dg_points* p, const rp3dg_islands* is) {
    if (!ctx || !pr || !b || !c || !m || !p || !is) return fail(ctx, RP3DG_EINVAL, "null argument");
    if (b->n_enabled > b->n || c->n_enabled > c->n) return fail(ctx, RP3DG_EINVAL, "n_enabled > n");
    if (!(pr->dt > 0.0f) || pr->velocity_iterations < 0) return fail(ctx, RP3DG_EINVAL, "bad dt or iterations");
    if (b->n && (!b->position || !b->orientation || !b->com_world || !b->com_local || !b->linear_velocity ||
                 !b->angular_velocity || !b->force || !b->torque || !b->inv_inertia_local || !b->inv_inertia_world ||
                 !b->mass || !b->linear_lock || !b->angular_lock || !b->gravity))
        return fail(ctx, RP3DG_EINVAL, "null body array");
    if (c->n && (!c->body || !c->local_position || !c->local_orientation || !c->world_position ||
                 !c->world_orientation || !c->material))
        return fail(ctx, RP3DG_EINVAL, "null collider array");
    if (m->n && (!m->ids || !m->point_start || !m->nb_points || !m->friction_vector1 || !m->friction_vector2 ||
                 !m->friction_impulse))
        return fail(ctx, RP3DG_EINVAL, "null manifold array");
    if (p->n && (!p->normal_depth || !p->local1 || !p->local2 || !p->penetration_impulse || !p->is_resting))
        return fail(ctx, RP3DG_EINVAL, "null point array");
    if (is->n && (!is->manifold_start || !is->manifold_count)) return fail(ctx, RP3DG_EINVAL, "null island array");
    if (m->n && (!b->n || !c->n || !p->n)) return fail(ctx, RP3DG_EINVAL, "manifolds without bodies, colliders or points");
    return 0;
}

}  // namespace

int rp3dg_dynamics_step_device(rp3dg_ctx* ctx, const rp3dg_dynamics_params* pr, const rp3dg_bodies* b,
                               const rp3dg_colliders* c, const rp3dg_manifolds* m, const rp3dg_points* p,
                               const rp3dg_islands* is) {
    return rp3dg::dynamics_step_flags(ctx, pr, b, c, m, p, is, nullptr, nullptr);
}

namespace rp3dg {
// The dynamics stage with the enabled bodies / colliders given as per-row
// flags (several worlds in one batch) instead of a leading range.
int dynamics_step_flags(rp3dg_ctx* ctx, const rp3dg_dynamics_params* pr, const rp3dg_bodies* b,
                        const rp3dg_colliders* c, const rp3dg_manifolds* m, const rp3dg_points* p,
                        const rp3dg_islands* is, const uint8_t* b_enabled, const uint8_t* c_enabled,
                        const DynJoints* joints, const DynTuning* tune, const DynSolver* solver) {
    int rc = check_dynamics(ctx, pr, b, c, m, p, is);
    if (rc) return rc;
    const void* f16[] = {b->position, b->orientation, b->com_world, b->com_local, b->linear_velocity,
                         b->angular_velocity, b->force, b->torque, b->inv_inertia_local, b->inv_inertia_world,
                         b->mass, b->linear_lock, b->angular_lock, c->local_position, c->local_orientation,
                         c->world_position, c->world_orientation, c->material, m->ids, m->friction_vector1,
                         m->friction_vector2, m->friction_impulse, p->normal_depth, p->local1, p->local2};
    for (const void* q : f16)
        if (!aligned(q, 16)) return fail(ctx, RP3DG_EINVAL, "misaligned device array (float4 / int4 arrays need 16 bytes)");
    const void* f4[] = {c->body, m->point_start, p->penetration_impulse, is->manifold_start, is->manifold_count};
    for (const void* q : f4)
        if (!aligned(q, 4)) return fail(ctx, RP3DG_EINVAL, "misaligned device array (32-bit arrays need 4 bytes)");
    cudaSetDevice(ctx->device);
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t vel_bytes = al(size_t(b->n) * 16);
    const size_t off_m = 4 * vel_bytes;
    const size_t off_p = off_m + al(size_t(m->n) * sizeof(rp3dg::DynManifoldRec));
    const size_t off_lev = off_p + al(size_t(p->n) * sizeof(rp3dg::DynPointRec));
    const size_t off_ord = off_lev + al(size_t(m->n) * 4);
    const size_t off_blev = off_ord + al(size_t(m->n) * 4);
    const size_t off_bslot = off_blev + al(size_t(b->n) * 4);
    const size_t off_cnt = off_bslot + al(size_t(b->n) * 4);
    const size_t off_list = off_cnt + 256;
    const size_t off_giant = off_list + al(size_t(is->n) * 4);
    size_t need = off_giant + al(size_t(is->n) * 4) + 256;
    // graph-coloured solver scratch
    const bool colored = solver && solver->colored;
    const size_t o_cstart = need; if (colored) need += al((size_t(b->n) + 1) * 4);
    const size_t o_cfill = need; if (colored) need += al(size_t(b->n) * 4);
    const size_t o_cadj = need; if (colored) need += al(size_t(m->n) * 8);
    const size_t o_ccol = need; if (colored) need += al(size_t(m->n));
    const size_t o_ctent = need; if (colored) need += al(size_t(m->n));
    const size_t o_ccnt = need; if (colored) need += al((rp3dg::COLOR_MAX + 2) * 4);
    const size_t o_coff = need; if (colored) need += al(rp3dg::COLOR_MAX * 4);
    const size_t o_cord = need; if (colored) need += al(size_t(m->n) * 4);
    rc = grow(ctx, &ctx->d_dyn, &ctx->cap_dyn, need, "cudaMalloc(dynamics scratch)");
    if (rc) return rc;
    char* s = static_cast<char*>(ctx->d_dyn);
    rp3dg::DynArgs a = {};
    a.b_enabled = b_enabled;
    a.c_enabled = c_enabled;
    if (joints && joints->nj) {
        a.nj = joints->nj; a.j_list = joints->j_list; a.j_rec = joints->j_rec;
        a.i_jstart = joints->i_jstart; a.i_jcount = joints->i_jcount;
        a.nji = joints->nji; a.ji_island = joints->ji_island; a.ji_bstart = joints->ji_bstart;
        a.ji_bcount = joints->ji_bcount; a.ji_rows = joints->ji_rows;
        a.xc = joints->xc; a.qc = joints->qc;
        a.position_iterations = joints->position_iterations;
    }
    a.dt = pr->dt; a.gx = pr->gravity[0]; a.gy = pr->gravity[1]; a.gz = pr->gravity[2];
    a.gravity_enabled = pr->gravity_enabled; a.iterations = pr->velocity_iterations; a.split = pr->split_impulse ? 1 : 0;
    a.restitution_threshold = pr->restitution_velocity_threshold;
    a.nb = b->n; a.nb_enabled = b->n_enabled;
    a.position = reinterpret_cast<float4*>(b->position);
    a.orientation = reinterpret_cast<float4*>(b->orientation);
    a.com_world = reinterpret_cast<float4*>(b->com_world);
    a.com_local = reinterpret_cast<const float4*>(b->com_local);
    a.lin_vel = reinterpret_cast<float4*>(b->linear_velocity);
    a.ang_vel = reinterpret_cast<float4*>(b->angular_velocity);
    a.force = reinterpret_cast<const float4*>(b->force);
    a.torque = reinterpret_cast<const float4*>(b->torque);
    a.iil = reinterpret_cast<const float4*>(b->inv_inertia_local);
    a.iiw = reinterpret_cast<float4*>(b->inv_inertia_world);
    a.mass = reinterpret_cast<const float4*>(b->mass);
    a.llock = reinterpret_cast<const float4*>(b->linear_lock);
    a.alock = reinterpret_cast<const float4*>(b->angular_lock);
    a.gravity = b->gravity;
    a.nc = c->n; a.nc_enabled = c->n_enabled;
    a.c_body = c->body;
    a.c_lpos = reinterpret_cast<const float4*>(c->local_position);
    a.c_lori = reinterpret_cast<const float4*>(c->local_orientation);
    a.c_wpos = reinterpret_cast<float4*>(c->world_position);
    a.c_wori = reinterpret_cast<float4*>(c->world_orientation);
    a.c_mat = reinterpret_cast<const float4*>(c->material);
    a.nm = m->n; a.np = p->n; a.ni = is->n;
    a.m_ids = reinterpret_cast<const int4*>(m->ids);
    a.m_pstart = m->point_start;
    a.m_npts = m->nb_points;
    a.m_fv1 = reinterpret_cast<float4*>(m->friction_vector1);
    a.m_fv2 = reinterpret_cast<float4*>(m->friction_vector2);
    a.m_fimp = reinterpret_cast<float4*>(m->friction_impulse);
    a.p_nd = reinterpret_cast<const float4*>(p->normal_depth);
    a.p_l1 = reinterpret_cast<const float4*>(p->local1);
    a.p_l2 = reinterpret_cast<const float4*>(p->local2);
    a.p_impulse = p->penetration_impulse;
    a.p_resting = p->is_resting;
    a.i_start = is->manifold_start;
    a.i_count = is->manifold_count;
    a.error = ctx->d_error;
    a.cv = reinterpret_cast<float4*>(s);
    a.cw = reinterpret_cast<float4*>(s + vel_bytes);
    a.sv = reinterpret_cast<float4*>(s + 2 * vel_bytes);
    a.sw = reinterpret_cast<float4*>(s + 3 * vel_bytes);
    a.mrec = reinterpret_cast<rp3dg::DynManifoldRec*>(s + off_m);
    a.prec = reinterpret_cast<rp3dg::DynPointRec*>(s + off_p);
    a.level = reinterpret_cast<uint32_t*>(s + off_lev);
    a.order = reinterpret_cast<uint32_t*>(s + off_ord);
    a.body_level = reinterpret_cast<uint32_t*>(s + off_blev);
    a.body_slot = reinterpret_cast<int32_t*>(s + off_bslot);
    a.counters = reinterpret_cast<uint32_t*>(s + off_cnt);
    a.large_list = reinterpret_cast<uint32_t*>(s + off_list);
    a.giant_list = reinterpret_cast<uint32_t*>(s + off_giant);
    const rp3dg::DynTuning tdef{};
    const rp3dg::DynTuning& tn = tune ? *tune : tdef;
    a.large_ctas = uint32_t(ctx->num_sms) * (tn.large_per_sm ? tn.large_per_sm : 1u);
    a.small_max = tn.small_max;
    a.giant_min = tn.giant_min;
    a.giant_ctas = uint32_t(ctx->num_sms);
    // the opt-in maximum less room for the kernel's static shared memory
    a.giant_smem = ctx->smem_optin > 2048 ? uint32_t(ctx->smem_optin - 1024) : 0u;
    rp3dg::ColorScratch cs{};
    if (colored) {
        cs.start = reinterpret_cast<uint32_t*>(s + o_cstart);
        cs.fill = reinterpret_cast<uint32_t*>(s + o_cfill);
        cs.adj = reinterpret_cast<uint32_t*>(s + o_cadj);
        cs.color = reinterpret_cast<uint8_t*>(s + o_ccol);
        cs.tent = reinterpret_cast<uint8_t*>(s + o_ctent);
        cs.count = reinterpret_cast<uint32_t*>(s + o_ccnt);
        cs.offset = reinterpret_cast<uint32_t*>(s + o_coff);
        cs.order = reinterpret_cast<uint32_t*>(s + o_cord);
        a.colored = 1;
        a.color = &cs;
    }
    a.stats = solver ? solver->stats : nullptr;
    cudaError_t e = rp3dg::launch_dynamics(a, ctx->stream, &ctx->launches);
    return e == cudaSuccess ? 0 : cuda_fail(ctx, e, "dynamics launch");
}
}  // namespace rp3dg


int rp3dg_dynamics_step_host(rp3dg_ctx* ctx, const rp3dg_dynamics_params* pr, const rp3dg_bodies* b,
                             const rp3dg_colliders* c, const rp3dg_manifolds* m, const rp3dg_points* p,
                             const rp3dg_islands* is) {
    int rc = check_dynamics(ctx, pr, b, c, m, p, is);
    if (rc) return rc;
    // every array goes to one staging buffer (256-byte aligned slots); the
    // ones the stage writes come back
    struct Arr { const void* host; void* out; size_t bytes; size_t off; };
    std::vector<Arr> arrs;
    size_t off = 0;
    auto add = [&](const void* host, size_t bytes, bool written) -> size_t {
        Arr r{host, written ? const_cast<void*>(host) : nullptr, host ? bytes : 0, off};
        off += (r.bytes + 255) & ~size_t(255);
        arrs.push_back(r);
        return arrs.size() - 1;
    };
    const size_t nb = b->n, nc = c->n, nm = m->n, np = p->n, ni = is->n;
    const size_t i_pos = add(b->position, nb * 16, true), i_ori = add(b->orientation, nb * 16, true);
    const size_t i_comw = add(b->com_world, nb * 16, true), i_coml = add(b->com_local, nb * 16, false);
    const size_t i_lv = add(b->linear_velocity, nb * 16, true), i_av = add(b->angular_velocity, nb * 16, true);
    const size_t i_f = add(b->force, nb * 16, false), i_t = add(b->torque, nb * 16, false);
    const size_t i_iil = add(b->inv_inertia_local, nb * 16, false), i_iiw = add(b->inv_inertia_world, nb * 48, true);
    const size_t i_mass = add(b->mass, nb * 16, false), i_ll = add(b->linear_lock, nb * 16, false);
    const size_t i_al = add(b->angular_lock, nb * 16, false), i_g = add(b->gravity, nb, false);
    const size_t i_cb = add(c->body, nc * 4, false), i_clp = add(c->local_position, nc * 16, false);
    const size_t i_clo = add(c->local_orientation, nc * 16, false), i_cwp = add(c->world_position, nc * 16, true);
    const size_t i_cwo = add(c->world_orientation, nc * 16, true), i_cm = add(c->material, nc * 16, false);
    const size_t i_mid = add(m->ids, nm * 16, false), i_mps = add(m->point_start, nm * 4, false);
    const size_t i_mnp = add(m->nb_points, nm, false), i_fv1 = add(m->friction_vector1, nm * 16, true);
    const size_t i_fv2 = add(m->friction_vector2, nm * 16, true), i_fi = add(m->friction_impulse, nm * 16, true);
    const size_t i_pnd = add(p->normal_depth, np * 16, false), i_pl1 = add(p->local1, np * 16, false);
    const size_t i_pl2 = add(p->local2, np * 16, false), i_pi = add(p->penetration_impulse, np * 4, true);
    const size_t i_pr = add(p->is_resting, np, true);
    const size_t i_is = add(is->manifold_start, ni * 4, false), i_ic = add(is->manifold_count, ni * 4, false);
    cudaSetDevice(ctx->device);
    rc = grow(ctx, &ctx->d_dyn_stage, &ctx->cap_dyn_stage, off + 256, "cudaMalloc(dynamics staging)");
    if (rc) return rc;
    char* d = static_cast<char*>(ctx->d_dyn_stage);
    cudaError_t e = cudaSuccess;
    for (const Arr& r : arrs)
        if (e == cudaSuccess && r.bytes) e = cudaMemcpyAsync(d + r.off, r.host, r.bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "upload dynamics arrays");
    auto D = [&](size_t i) { return arrs[i].bytes ? static_cast<void*>(d + arrs[i].off) : nullptr; };
    auto F = [&](size_t i) { return static_cast<rp3dg_float4*>(D(i)); };
    rp3dg_bodies db = *b;
    db.position = F(i_pos); db.orientation = F(i_ori); db.com_world = F(i_comw); db.com_local = F(i_coml);
    db.linear_velocity = F(i_lv); db.angular_velocity = F(i_av); db.force = F(i_f); db.torque = F(i_t);
    db.inv_inertia_local = F(i_iil); db.inv_inertia_world = F(i_iiw); db.mass = F(i_mass);
    db.linear_lock = F(i_ll); db.angular_lock = F(i_al); db.gravity = static_cast<const uint8_t*>(D(i_g));
    rp3dg_colliders dc = *c;
    dc.body = static_cast<const int32_t*>(D(i_cb)); dc.local_position = F(i_clp); dc.local_orientation = F(i_clo);
    dc.world_position = F(i_cwp); dc.world_orientation = F(i_cwo); dc.material = F(i_cm);
    rp3dg_manifolds dm = *m;
    dm.ids = static_cast<const int32_t*>(D(i_mid)); dm.point_start = static_cast<const uint32_t*>(D(i_mps));
    dm.nb_points = static_cast<const uint8_t*>(D(i_mnp)); dm.friction_vector1 = F(i_fv1);
    dm.friction_vector2 = F(i_fv2); dm.friction_impulse = F(i_fi);
    rp3dg_points dp = *p;
    dp.normal_depth = F(i_pnd); dp.local1 = F(i_pl1); dp.local2 = F(i_pl2);
    dp.penetration_impulse = static_cast<float*>(D(i_pi)); dp.is_resting = static_cast<uint8_t*>(D(i_pr));
    rp3dg_islands di = *is;
    di.manifold_start = static_cast<const uint32_t*>(D(i_is)); di.manifold_count = static_cast<const uint32_t*>(D(i_ic));
    rc = rp3dg_dynamics_step_device(ctx, pr, &db, &dc, &dm, &dp, &di);
    if (rc) return rc;
    for (const Arr& r : arrs)
        if (e == cudaSuccess && r.out && r.bytes) e = cudaMemcpyAsync(r.out, d + r.off, r.bytes, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    return e == cudaSuccess ? 0 : cuda_fail(ctx, e, "dynamics (host arrays)");
}

// ---- broad phase -----------------------------------------------------------

namespace {

int check_bp(rp3dg_ctx* ctx, const rp3dg_broadphase* bp) {
    if (!ctx || !bp) return fail(ctx, RP3DG_EINVAL, "null argument");
    if (bp->n_update > bp->n) return fail(ctx, RP3DG_EINVAL, "n_update > n");
    if (bp->nb_groups > 1 && !bp->group) return fail(ctx, RP3DG_EINVAL, "nb_groups > 1 needs group");
    if (bp->n && (!bp->fat_min || !bp->fat_max)) return fail(ctx, RP3DG_EINVAL, "null fat AABB array");
    if (!aligned(bp->fat_min, 16) || !aligned(bp->fat_max, 16) || !aligned(bp->world_position, 16) ||
        !aligned(bp->world_orientation, 16) || !aligned(bp->shape, 4) || !aligned(bp->body, 4) ||
        !aligned(bp->group, 4) || !aligned(bp->category, 2) || !aligned(bp->mask, 2))
        return fail(ctx, RP3DG_EINVAL, "misaligned device array (float4 arrays need 16 bytes)");
    return 0;
}

}  // namespace

int rp3dg_broadphase_update_device(rp3dg_ctx* ctx, const rp3dg_broadphase* bp) {
    return rp3dg::broadphase_update_flags(ctx, bp, nullptr);
}

namespace rp3dg {
// The fat-AABB update of the flagged rows of [0, n_update) only.
int broadphase_update_flags(rp3dg_ctx* ctx, const rp3dg_broadphase* bp, const uint8_t* enabled) {
    int rc = check_bp(ctx, bp);
    if (rc) return rc;
    if (bp->n_update == 0) return 0;
    if (!bp->shape || !bp->world_position || !bp->world_orientation || !bp->moved)
        return fail(ctx, RP3DG_EINVAL, "null collider array");
    if (!ctx->d_shapes || !ctx->d_shape_bounds) return fail(ctx, RP3DG_EINVAL, "no shape table (rp3dg_set_shapes)");
    rp3dg::BpArgs a = {};
    a.n = bp->n;
    a.n_update = bp->n_update;
    a.nb_shapes = ctx->nb_shapes;
    a.shapes = ctx->d_shapes;
    a.bounds = reinterpret_cast<const float4*>(ctx->d_shape_bounds);
    a.shape = bp->shape;
    a.wpos = reinterpret_cast<const float4*>(bp->world_position);
    a.wori = reinterpret_cast<const float4*>(bp->world_orientation);
    a.force = bp->force_reinsert;
    a.fat_min = reinterpret_cast<float4*>(bp->fat_min);
    a.fat_max = reinterpret_cast<float4*>(bp->fat_max);
    a.moved = bp->moved;
    a.enabled = enabled;
    a.error = ctx->d_error;
    cudaSetDevice(ctx->device);
    cudaError_t e = rp3dg::launch_bp_update(a, ctx->stream, &ctx->launches);
    return e == cudaSuccess ? 0 : cuda_fail(ctx, e, "broad-phase update");
}
}  // namespace rp3dg


int rp3dg_broadphase_pairs_device(rp3dg_ctx* ctx, const rp3dg_broadphase* bp, int axis, int32_t* pairs,
                                  uint32_t capacity, uint32_t* count) {
    int rc = check_bp(ctx, bp);
    if (rc) return rc;
    if (axis < RP3DG_BROADPHASE_LBVH || axis > 2) return fail(ctx, RP3DG_EINVAL, "axis must be -1 (LBVH), 0, 1 or 2");
    if (!count || (capacity && !pairs)) return fail(ctx, RP3DG_EINVAL, "null output");
    if (bp->n && !bp->body) return fail(ctx, RP3DG_EINVAL, "null body array");
    if (!aligned(pairs, 4) || !aligned(count, 4)) return fail(ctx, RP3DG_EINVAL, "misaligned output");
    const size_t n = bp->n;
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    size_t off = 0;
    const size_t o_keys = off; off += al(n * 8);
    const size_t o_keys2 = off; off += al(n * 8);
    const size_t o_vals = off; off += al(n * 4);
    const size_t o_vals2 = off; off += al(n * 4);
    const size_t o_hist = off; off += al(rp3dg::sort_scratch_words(uint32_t(n)) * 4);
    const size_t o_lo = off; off += al(n * 16);
    const size_t o_hi = off; off += al(n * 16);
    const size_t o_grp = off; off += al(n * 4);
    const size_t o_poff = off; off += al(n * 4 + 4);
    const bool lbvh = axis == RP3DG_BROADPHASE_LBVH;
    const size_t o_lb = off; off += lbvh ? al(8 * 4) : 0;
    const size_t o_lchild = off; off += lbvh ? al(n * 8) : 0;
    const size_t o_lrange = off; off += lbvh ? al(n * 8) : 0;
    const size_t o_lparent = off; off += lbvh ? al(2 * n * 4) : 0;
    const size_t o_lvisit = off; off += lbvh ? al(n * 4) : 0;
    const size_t o_lnlo = off; off += lbvh ? al(n * 16) : 0;
    const size_t o_lnhi = off; off += lbvh ? al(n * 16) : 0;
    cudaSetDevice(ctx->device);
    rc = grow(ctx, &ctx->d_bp, &ctx->cap_bp, off + 256, "cudaMalloc(broad-phase scratch)");
    if (rc) return rc;
    char* s = static_cast<char*>(ctx->d_bp);
    rp3dg::BpArgs a = {};
    a.n = bp->n;
    a.fat_min = reinterpret_cast<float4*>(bp->fat_min);
    a.fat_max = reinterpret_cast<float4*>(bp->fat_max);
    a.group = bp->nb_groups > 1 ? bp->group : nullptr;
    a.body = bp->body;
    a.category = bp->category;
    a.mask = bp->mask;
    int bits = 0;
    if (bp->nb_groups > 1) while (bits < 32 && (uint64_t(1) << bits) < bp->nb_groups) bits++;
    a.group_bits = bits;
    a.keys = reinterpret_cast<unsigned long long*>(s + o_keys);
    a.keys_tmp = reinterpret_cast<unsigned long long*>(s + o_keys2);
    a.vals = reinterpret_cast<uint32_t*>(s + o_vals);
    a.vals_tmp = reinterpret_cast<uint32_t*>(s + o_vals2);
    a.sort_hist = reinterpret_cast<uint32_t*>(s + o_hist);
    a.s_lo = reinterpret_cast<float4*>(s + o_lo);
    a.s_hi = reinterpret_cast<float4*>(s + o_hi);
    a.s_group = reinterpret_cast<int32_t*>(s + o_grp);
    a.pair_offset = reinterpret_cast<uint32_t*>(s + o_poff);
    a.pairs = pairs;
    a.capacity = capacity;
    a.pair_count = count;
    a.error = ctx->d_error;
    if (lbvh) {
        a.lbvh_bounds = reinterpret_cast<uint32_t*>(s + o_lb);
        a.lbvh_child = reinterpret_cast<int2*>(s + o_lchild);
        a.lbvh_range = reinterpret_cast<int2*>(s + o_lrange);
        a.lbvh_parent = reinterpret_cast<int32_t*>(s + o_lparent);
        a.lbvh_visits = reinterpret_cast<uint32_t*>(s + o_lvisit);
        a.lbvh_nlo = reinterpret_cast<float4*>(s + o_lnlo);
        a.lbvh_nhi = reinterpret_cast<float4*>(s + o_lnhi);
    }
    cudaError_t e = rp3dg::launch_bp_pairs(a, axis, ctx->stream, &ctx->launches);
    return e == cudaSuccess ? 0 : cuda_fail(ctx, e, "broad-phase pairs");
}

int rp3dg_broadphase_pairs_host(rp3dg_ctx* ctx, const rp3dg_broadphase* bp, int axis, int32_t* pairs,
                                uint32_t capacity, uint32_t* count) {
    if (!ctx || !bp || !count) return fail(ctx, RP3DG_EINVAL, "null argument");
    if (bp->nb_groups > 1 && !bp->group) return fail(ctx, RP3DG_EINVAL, "nb_groups > 1 needs group");
    const size_t n = bp->n;
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    size_t off = 0;
    const size_t o_min = off; off += al(n * 16);
    const size_t o_max = off; off += al(n * 16);
    const size_t o_body = off; off += al(n * 4);
    const size_t o_grp = off; off += al(n * 4);
    const size_t o_cat = off; off += al(n * 2);
    const size_t o_msk = off; off += al(n * 2);
    const size_t o_cnt = off; off += 256;
    const size_t o_pairs = off; off += al(size_t(capacity) * 8);
    cudaSetDevice(ctx->device);
    int rc = grow(ctx, &ctx->d_bp_stage, &ctx->cap_bp_stage, off + 256, "cudaMalloc(broad-phase staging)");
    if (rc) return rc;
    char* d = static_cast<char*>(ctx->d_bp_stage);
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaSuccess;
    auto up = [&](size_t o, const void* src, size_t bytes) {
        if (e == cudaSuccess && src && bytes) e = cudaMemcpyAsync(d + o, src, bytes, cudaMemcpyHostToDevice, s);
    };
    up(o_min, bp->fat_min, n * 16); up(o_max, bp->fat_max, n * 16);
    up(o_body, bp->body, n * 4);
    if (bp->nb_groups > 1) up(o_grp, bp->group, n * 4);
    up(o_cat, bp->category, n * 2); up(o_msk, bp->mask, n * 2);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "upload broad-phase arrays");
    rp3dg_broadphase dbp = *bp;
    dbp.fat_min = reinterpret_cast<rp3dg_float4*>(d + o_min);
    dbp.fat_max = reinterpret_cast<rp3dg_float4*>(d + o_max);
    dbp.body = reinterpret_cast<const int32_t*>(d + o_body);
    dbp.group = bp->nb_groups > 1 ? reinterpret_cast<const int32_t*>(d + o_grp) : nullptr;
    dbp.category = bp->category ? reinterpret_cast<const uint16_t*>(d + o_cat) : nullptr;
    dbp.mask = bp->mask ? reinterpret_cast<const uint16_t*>(d + o_msk) : nullptr;
    dbp.shape = nullptr; dbp.world_position = nullptr; dbp.world_orientation = nullptr;
    dbp.force_reinsert = nullptr; dbp.moved = nullptr;
    uint32_t* dcount = reinterpret_cast<uint32_t*>(d + o_cnt);
    int32_t* dpairs = reinterpret_cast<int32_t*>(d + o_pairs);
    rc = rp3dg_broadphase_pairs_device(ctx, &dbp, axis, dpairs, capacity, dcount);
    if (rc) return rc;
    e = cudaMemcpyAsync(count, dcount, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess && capacity && pairs) {
        const size_t got = *count < capacity ? *count : capacity;
        if (got) e = cudaMemcpyAsync(pairs, dpairs, got * 8, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    return e == cudaSuccess ? 0 : cuda_fail(ctx, e, "broad-phase pairs (host arrays)");
}
