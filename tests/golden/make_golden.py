"""Generates the committed golden fixtures of tests/golden/ from the reference's
own test inputs.  Reads the reference checkout named by AVBD_REFERENCE_ROOT
(default /root/reference); the GPU box and the tests only read the JSON it
writes.

neohookean_element0.json -- the element used by test/test_neohookean_accumulate.cpp:
  tet 0 of resource/cube2.msh (gmsh MSH 4.1 ASCII, read directly because gmsh
  is not installed), lambda 1e7, mu 1e6, kd 10, V 5, dt 1e-3 and the vertex
  perturbations of :45-48.
"""
import json
import os

REF = os.environ.get("AVBD_REFERENCE_ROOT", "/root/reference")
HERE = os.path.dirname(os.path.abspath(__file__))


def read_msh41(path):
    lines = open(path).read().split("\n")
    i = 0
    nodes = {}
    tets = []
    while i < len(lines):
        if lines[i].strip() == "$Nodes":
            nblocks, nnodes, _, _ = map(int, lines[i + 1].split())
            i += 2
            for _ in range(nblocks):
                dim, tag, parametric, n = map(int, lines[i].split())
                tags = [int(lines[i + 1 + k]) for k in range(n)]
                coords = [list(map(float, lines[i + 1 + n + k].split()[:3])) for k in range(n)]
                for t, c in zip(tags, coords):
                    nodes[t] = c
                i += 1 + 2 * n
            continue
        if lines[i].strip() == "$Elements":
            nblocks = int(lines[i + 1].split()[0])
            i += 2
            for _ in range(nblocks):
                dim, tag, etype, n = map(int, lines[i].split())
                for k in range(n):
                    parts = list(map(int, lines[i + 1 + k].split()))
                    if etype == 4:
                        tets.append(parts[1:5])
                i += 1 + n
            continue
        i += 1
    return nodes, tets


def main():
    nodes, tets = read_msh41(os.path.join(REF, "resource", "cube2.msh"))
    t0 = tets[0]
    verts = [nodes[t] for t in t0]
    out = {
        "source": "resource/cube2.msh element 0, inputs of test/test_neohookean_accumulate.cpp:16-48",
        "element_node_tags": t0,
        "vertices": verts,
        "lambda": 1e7, "mu": 1e6, "kd": 10.0, "rest_volume": 5.0, "dt": 1e-3,
        "perturbations": [[0.3, 0.3, 0.3], [0.1, 0.2, 0.3], [-0.2, -0.3, -0.2], [-0.1, 0.1, 0.1]],
    }
    with open(os.path.join(HERE, "neohookean_element0.json"), "w") as f:
        json.dump(out, f, indent=1)
    cos = {
        "source": "test/test_cosserat_accumulate.cpp:10-23",
        "p1": [0, 0, 0], "euler1_deg": [0, 0, 0], "p2": [0.3, 0.4, 0.5], "euler2_deg": [60, -30, 20],
        "mass": 10, "inertia": [1, 1, 1], "stiffness": [2, 2, 3.5, 0.5, 0.5, 0.8], "rest_length": 0.2,
        "precurvature": [0, 0, 0], "dt": 1e-3, "fd_eps": 1e-6,
    }
    with open(os.path.join(HERE, "cosserat_pair.json"), "w") as f:
        json.dump(cos, f, indent=1)
    jnt = {
        "source": "test/test_one_sided_fixed_joint_accumulate.cpp:9-22",
        "p": [0, 0, 0], "mass": 10, "inertia": [1, 1, 1], "position_offset": [0.4, 0.6, 0.2],
        "rotation_offset_euler_deg": [60, -30, 20], "ref_position": [-0.3, -0.5, -0.2],
        "ref_rotation_euler_deg": [-60, 50, -20], "dt": 1e-3, "fd_eps": 1e-6,
    }
    with open(os.path.join(HERE, "joint.json"), "w") as f:
        json.dump(jnt, f, indent=1)
    lb = {
        "source": "test/test_lbvh.cpp:38-47 (codes) and :168-189 (triangles), :243-267 (spheres)",
        "karras_codes_by_slot": [0b11001, 0b00100, 0b00101, 0b00010, 0b11000, 0b00001, 0b10011, 0b11110],
        "triangles": [
            [[0.0, 0.0, 0.0], [1.0, 0.0, 0.5], [0.0, 1.0, 0.0]],
            [[1.0, 1.0, 1.0], [1.2, 1.0, 1.2], [1.4, 1.2, 1.2]],
            [[0.6, 0.8, 0.8], [0.4, 0.6, 0.6], [0.8, 0.4, 0.6]],
            [[0.7, 1.1, 1.3], [1.1, 1.2, 1.4], [0.6, 0.7, 0.7]]],
        "dt": 1e-3,
    }
    with open(os.path.join(HERE, "lbvh_inputs.json"), "w") as f:
        json.dump(lb, f, indent=1)
    print("wrote fixtures for element", t0)


if __name__ == "__main__":
    main()
