"""FP32 work of the narrow phase: path events x a static op table.

rp3dg_narrowphase_count_events runs a batch through the event-counting build
of the kernels and returns how many times the pairs' code paths executed
each step of the reference's algorithms (face tests, Gauss-map tests, edge
distances, clipped vertices, GJK iterations, ...).  Each step is a fixed
piece of the reference's arithmetic; OPS below gives its FP32 operation
count, read off the reference source (additions, subtractions,
multiplications, divisions, square roots and comparisons of floats each
count 1; negations and copies count 0).  The FP32 work of a batch is then
sum(events[e] * OPS[e]): the operations the reference's own code performs
for those pairs, which is also the work the CPU baseline does.

The kernels do less than that where they can: the warp schedule evaluates
the polyhedron-1 half of each Gauss-map test once per edge instead of once
per edge pair, and against a box each Gauss-map dot product reduces to one
product (the other terms are exact zeros).  The fraction of the FP32 peak
achieved on the reference's operation count therefore measures useful work
per second in the reference's units.

Primitive costs (reference headers under include/reactphysics3d/mathematics):
  Quaternion * Vector3 (Quaternion.h:365-379)       41
  Transform * Vector3 (Transform.h:193-195)          44
  Transform::getInverse (Transform.h:162-165)        41
  Transform * Transform (Transform.h:198-220)        72
  dot 5, cross 9, vector add / sub 3, lengthSquare 5, getUnit 9 (length + 3 divisions)
"""
import numpy as np

QV, TV, TINV, TT = 41, 44, 41, 72
DOT, CROSS, SUB, LEN2, UNIT = 5, 9, 3, 5, 9

# event ids (csrc/rp3dg_internal.h NpEvent, the order of the C ABI array)
EVENTS = ["poly_setup", "face_test", "support_box", "support_vertex", "support_tri", "support_capsule", "edge1",
          "gauss", "edge_dist", "clip_setup", "antiparallel", "inc_vertex", "clip_plane", "clip_vertex",
          "clip_intersect", "clip_depth", "contact", "edge_contact", "gjk_setup", "gjk_iter", "sx_seg", "sx_tri",
          "sx_tet", "gjk_contact", "sphere_face", "sphere_poly_contact", "capsule_face", "capsule_edge",
          "capsule_edge_axis", "capsule_clip", "closed_form", "closed_form_contact", "capsule_gjk_face",
          "tri_smooth"]
NB_EVENTS = 40

# closest points of two segments, computeClosestPointBetweenTwoSegments
# (mathematics_functions.h:123-193): 3 differences, 5 dots, the denominator,
# the clamped parameters and the two points
SEGMENT_CLOSEST = 3 * SUB + 5 * DOT + 3 + 14 + 2 * 6

OPS = {
    # SATAlgorithm.cpp:502-503: shape2^-1 * shape1, then its inverse
    "poly_setup": TINV + TT + TINV,
    # testSingleFaceDirectionPolyhedronVsPolyhedron (:1087-1110) + the two
    # comparisons of testFacesDirectionPolyhedronVsPolyhedron (:1125-1138)
    "face_test": QV + TV + SUB + DOT + 2,
    "support_box": 3,                       # BoxShape.h:166-171: three sign tests
    "support_vertex": DOT + 1,              # ConvexMeshShape.cpp:80-102: one dot + compare per vertex
    "support_tri": 3 * DOT + 2,             # TriangleShape.cpp: three dots, getMaxAxis
    "support_capsule": 3,                   # CapsuleShape.h:191-206
    "edge1": 2 * TV + SUB,                  # SATAlgorithm.cpp:753-755
    # edge-2 direction (:764) + testEdgesBuildMinkowskiFace (:1146-1172: three
    # rotations, two differences) + testGaussMapArcsIntersect (:1180-1191:
    # four dots, three products, three comparisons)
    "gauss": SUB + 3 * QV + 2 * SUB + 4 * DOT + 6,
    # centroid (:776) + computeDistanceBetweenEdges (:1040-1083: parallel test,
    # cross, unit, two oriented dots, comparison) + the caller's comparisons
    # (:784, :801-802)
    "edge_dist": TV + (CROSS + LEN2 + 1) + CROSS + UNIT + (SUB + DOT) + 1 + (SUB + DOT) + 4,
    "clip_setup": 2 * QV,                   # :921, :924-925
    "antiparallel": DOT + 1,                # ConvexPolyhedronShape.h:105-123
    "inc_vertex": TV,                       # :945-948
    # side plane (:958-961) + clipPolygonWithPlane set-up (mathematics_functions.h:339-343)
    "clip_plane": SUB + CROSS + DOT + SUB + DOT,
    "clip_vertex": SUB + DOT + 2,           # mathematics_functions.h:351-376
    # computePlaneSegmentIntersection (mathematics_functions.h:226-238) + range
    # tests + interpolation (:362-363)
    "clip_intersect": (SUB + DOT + 1 + DOT + 1 + 1) + 2 + 9,
    "clip_depth": SUB + DOT + 1,            # :1000-1002
    "contact": TV + (SUB + DOT + 3 + SUB),  # :1007-1010, projectPointOntoPlane
    "edge_contact": SEGMENT_CLOSEST + TV + QV,   # :853-864
    # GJKAlgorithm.cpp:79-92: body2 to body1, rotation to body 2, margins
    "gjk_setup": TINV + TT + 28 + 2,
    # one iteration (:118-190) without the supports and the simplex: rotate
    # and transform the support, w, v.w tests, point-in-simplex, progress test,
    # affine dependence, |v|^2, termination tests
    "gjk_iter": QV + TV + SUB + DOT + 4 + 18 + 3 + 20 + LEN2 + 3 + 15,
    "sx_seg": 16 + 9 + 9 + SUB + 3,         # VoronoiSimplex.cpp:304-331 + the closest points (:188-205)
    "sx_tri": 70 + 15 + 15 + SUB,           # VoronoiSimplex.cpp:336-451 + the closest points (:207-229)
    "sx_tet": 4 * 27 + 2 * 78 + 2 * 21 + SUB,   # VoronoiSimplex.cpp:456-611, two faces outside on average
    # GJKAlgorithm.cpp:196-233: distance, the two points, the normal, the depth
    "gjk_contact": 1 + 7 + (TINV + 7 + TV) + (UNIT + QV) + 1 + 2 + LEN2 + 1,
    "sphere_face": SUB + DOT + 1 + 2,       # SATAlgorithm.cpp:147-162 + :90-95
    "sphere_poly_contact": 3 * QV + 6 + 6 + 1,   # :100-140
    # :197-211 with the capsule's support with margin (ConvexShape.cpp:40-56)
    "capsule_face": QV + (3 + LEN2 + 1 + UNIT + 6) + TV + SUB + DOT + 2,
    "capsule_edge": SUB + 3 * QV + 2 * DOT + 2,          # :218-230, isMinkowskiFaceCapsuleVsEdge :476-482
    "capsule_edge_axis": CROSS + LEN2 + 1 + 2 * TV + SUB + DOT + 1 + UNIT + 24 + SUB + DOT + 2,  # :322-354
    "capsule_clip": SUB + CROSS + 2 * (SUB + DOT) + 2 + 13,   # clipSegmentWithPlanes per plane
    "closed_form": None,                    # per algorithm, below
    "closed_form_contact": None,
    # CapsuleVsConvexPolyhedronAlgorithm.cpp:104-160: rotate the normal, the
    # direction test, areOrthogonalVectors, areParallelVectors
    "capsule_gjk_face": QV + DOT + 1 + (DOT + 1) + (CROSS + LEN2 + 1),
    "tri_smooth": 150,                      # TriangleShape.h:309-365 (not in the microbenchmark)
}

# whole-pair costs of the closed forms, by algorithm id (rp3dg.h)
CLOSED_FORM = {
    # SphereVsSphereAlgorithm.cpp:52-63: distance test
    1: (SUB + LEN2 + 1 + 1 + 1 + 3,
        # :70-100: two inverses, two transforms, three unit vectors, scales
        2 * TINV + 2 * TV + 3 * UNIT + 6 + 1),
    # SphereVsCapsuleAlgorithm.cpp:55-75: relative transform, closest point on
    # the segment, distance test
    2: (TINV + TT + 25 + SUB + LEN2 + 5,
        1 + 3 + TINV + TV + 6 + 6 + QV + 2),
    # CapsuleVsCapsuleAlgorithm.cpp:52-76, :158-180: relative transform, both
    # segments, parallel test, closest points, distance test
    3: (TINV + TT + 2 * TV + 2 * SUB + 1 + (CROSS + LEN2 + 1) + SEGMENT_CLOSEST + SUB + LEN2 + 2,
        1 + 3 + TINV + TV + 6 + 6 + QV + 2),
}


def op_table(algo):
    """Per-event FP32 operation counts (length NB_EVENTS) for a batch of the
    given algorithm id."""
    t = np.zeros(NB_EVENTS, dtype=np.float64)
    for k, name in enumerate(EVENTS):
        v = OPS[name]
        if name == "closed_form":
            v = CLOSED_FORM.get(int(algo), (0, 0))[0]
        elif name == "closed_form_contact":
            v = CLOSED_FORM.get(int(algo), (0, 0))[1]
        t[k] = v
    return t


def fp32_ops(algo, events):
    """FP32 operations of a batch's reference code paths."""
    ev = np.asarray(events, dtype=np.float64)[:NB_EVENTS]
    return float(ev @ op_table(algo))


def named(events):
    """{event name: count} of the non-zero events."""
    return {name: int(events[k]) for k, name in enumerate(EVENTS) if int(events[k])}
