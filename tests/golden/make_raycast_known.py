"""Known-answer raycast cases read from the reference's own raycast test.

Parses test/tests/collision/TestRaycast.h of the reference (as text) for the
box, sphere, capsule, convex-mesh, concave-mesh and height-field tests: the body and shape
transforms of the test fixture, the shapes, every ray the tests cast through
PhysicsWorld::raycast (endpoints in the shape's local space, the ray's
maxFraction) with the expected outcome (hit or miss) and, where the test
checks them, the expected hit fraction and hit point.  Writes
tests/golden/raycast_known.json.

    python tests/golden/make_raycast_known.py [path/to/reference]

(the path defaults to the RP3D_REFERENCE environment variable)
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("RP3D_REFERENCE", "")
SRC = os.path.join(REF, "test", "tests", "collision", "TestRaycast.h")
TESTS = {"box": "testBox", "sphere": "testSphere", "capsule": "testCapsule",
         "convex_mesh": "testConvexMesh", "concave_mesh": "testConcaveMesh", "heightfield": "testHeightField"}

NUM = r"-?\d+(?:\.\d+)?"


def nums(s):
    return [float(x) for x in re.findall(NUM, s.replace("decimal", ""))]


def body(text, name):
    start = text.index(f"void {name}()")
    nxt = text.find("void test", start + 10)
    return text[start:nxt if nxt > 0 else len(text)]


def parse_test(src):
    points, rays, cases = {}, {}, []
    for m in re.finditer(r"Vector3 (\w+) = mLocalShapeToWorld \* Vector3\(([^;]*)\);", src):
        points[m.group(1)] = nums(m.group(2))
    for m in re.finditer(r"Ray (\w+)\((\w+), (\w+)\);", src):
        rays[m.group(1)] = (points[m.group(2)], points[m.group(3)])
    for m in re.finditer(r"Ray (ray\d+)\(mLocalShapeToWorld \* Vector3\(([^)]*)\), "
                         r"mLocalShapeToWorld \* Vector3\(([^)]*)\)\);", src):
        rays[m.group(1)] = (nums(m.group(2)), nums(m.group(3)))
    # statements in order: world raycasts, their hit test, and the checks of
    # the callback's hit fraction and hit point that follow them
    stmt = re.compile(r"mWorld->raycast\((.*?), &mCallback\);|rp3d_test\((!?)mCallback\.isHit\);|"
                      r"approxEqual\(mCallback\.raycastInfo\.hitFraction, (?:decimal\()?(" + NUM + r")\)?, epsilon\)|"
                      r"approxEqual\(mCallback\.raycastInfo\.worldPoint\.x, (\w+)\.x, epsilon\)")
    cur = None
    for m in stmt.finditer(src):
        if m.group(1) is not None:
            expr = m.group(1)
            k = re.match(r"Ray\((\w+)\.point1, (\w+)\.point2, decimal\((" + NUM + r")\)\)", expr)
            name, maxf = (k.group(1), float(k.group(3))) if k else (expr.strip(), 1.0)
            p1, p2 = rays[name]
            cur = {"ray": name, "p1": p1, "p2": p2, "max_fraction": maxf, "hit": None}
            cases.append(cur)
        elif m.group(2) is not None and cur is not None and cur["hit"] is None:
            cur["hit"] = m.group(2) != "!"
        elif m.group(3) is not None and cur is not None:
            cur["fraction"] = float(m.group(3))
        elif m.group(4) is not None and cur is not None:
            cur["hit_point"] = points[m.group(4)]
    return [c for c in cases if c["hit"] is not None]


def main():
    with open(SRC) as fh:
        text = fh.read()
    setup = text[text.index("Body transform"):text.index("mBoxShape = ")]
    pos = nums(re.search(r"Vector3 position\(([^)]*)\)", setup).group(1))
    shape_pos = nums(re.search(r"Vector3 shapePosition\(([^)]*)\)", setup).group(1))
    shapes = text[text.index("mBoxShape = "):text.index("Compound shape")]
    verts = {int(i): float(v) for i, v in re.findall(r"mConvexMeshVertices\[(\d+)\] = (" + NUM + r");", shapes)}
    idx = {int(i): int(v) for i, v in re.findall(r"mConvexMeshIndices\[(\d+)\] = (\d+);", shapes)}
    v = [verts[i] for i in range(len(verts))]
    ix = [idx[i] for i in range(len(idx))]
    cverts = [nums(m) for m in re.findall(r"mConcaveMeshVertices\.push_back\(Vector3\(([^)]*)\)\);", text)]
    cidx = [int(m) for m in re.findall(r"mConcaveMeshIndices\.push_back\((\d+)\);", text)]
    hf = re.search(r"mHeightFieldData\[i\] = (" + NUM + r");", text)
    hfc = re.search(r"createHeightField\((\d+), (\d+),", text)
    out = {
        "source": "reference test/tests/collision/TestRaycast.h (setUp, testBox, testSphere, testCapsule, "
                  "testConvexMesh, testConcaveMesh, testHeightField), parsed by tests/golden/make_raycast_known.py",
        # Quaternion::fromEulerAngles arguments of the fixture (radians, as multiples of PI)
        "body_position": pos, "body_euler_pi": [1 / 5, 1 / 6, 1 / 7],
        "shape_position": shape_pos, "shape_euler_pi": [3 / 6, -1 / 8, 1 / 3],
        "box_half_extents": nums(re.search(r"createBoxShape\(Vector3\(([^)]*)\)\)", shapes).group(1)),
        "sphere_radius": nums(re.search(r"createSphereShape\(([^)]*)\)", shapes).group(1))[0],
        "capsule": nums(re.search(r"createCapsuleShape\(([^)]*)\)", shapes).group(1)),
        "convex_vertices": [v[3 * k:3 * k + 3] for k in range(len(v) // 3)],
        "convex_faces": [ix[4 * f:4 * f + 4] for f in range(len(ix) // 4)],
        "concave_vertices": cverts,
        "concave_triangles": [cidx[3 * t:3 * t + 3] for t in range(len(cidx) // 3)],
        "heightfield": {"columns": int(hfc.group(1)), "rows": int(hfc.group(2)), "height": float(hf.group(1))},
        "cases": {},
    }
    # the Euler angles as written in the fixture
    assert "fromEulerAngles(PI_RP3D / 5, PI_RP3D / 6, PI_RP3D / 7)" in setup
    assert "fromEulerAngles(3 * PI_RP3D / 6 , -PI_RP3D / 8, PI_RP3D / 3)" in setup
    for key, fn in TESTS.items():
        out["cases"][key] = parse_test(body(text, fn))
    with open(os.path.join(HERE, "raycast_known.json"), "w") as fh:
        json.dump(out, fh, indent=1)
    for key, cs in out["cases"].items():
        print(key, len(cs), "cases,", sum(c["hit"] for c in cs), "hits,",
              sum("fraction" in c for c in cs), "with a fraction")


if __name__ == "__main__":
    main()
