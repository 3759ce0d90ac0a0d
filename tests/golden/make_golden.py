"""Extract the reference's own known answers into small fixtures.

Reads, as text or raw bytes, the expected-output files that ship with the SNAC
tests (the reference tree is needed only when this script runs; the
fixtures it writes are committed and used by tests/ without it):

  Snac/libSnac/tests/test*-4-4-4.0of1.expected   ->  libsnac_known_answers.json
      tetra volumes / face areas / normals of a 100 m cube (element 0),
      element volume and min length scale, node gravity forces and the
      running |force| sums ("balance"), node masses of a 0.5 m mesh, and the
      velocities and coordinates after 10 iterations of the unit-cube pull test
  Snac/tests/test-basic.timeStep.0.expected       ->  basic_timestep.json
      the first dynamic dt of basic.xml
  Snac/tests/test-basic-velocity-completeForceCalc.vel.0.expected
                                                  ->  basic_velocity_vel.npz
      13 float32 velocity dumps of basic-velocity-completeForceCalc.xml

usage: python tests/golden/make_golden.py [/path/to/snac/source/tree]
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NUM = r"[-+]?(?:\d+\.?\d*|\.\d+)(?:[eE][-+]?\d+)?"


def lines(path):
    with open(path, encoding="latin-1") as f:
        return f.read().splitlines()


def main(root):
    T = os.path.join(root, "Snac", "libSnac", "tests")
    ka = {}

    def exp(name):
        return lines(os.path.join(T, f"{name}-4-4-4.0of1.expected"))

    # element 0 of the 100 m mesh: coordinates, tet volumes, face areas and normals
    for ln in exp("testTetrahedra-volume"):
        m = re.match(r"Element: 0, Coords: (.*)", ln)
        if m:
            ka["cube100_element0_coords"] = [[float(x) for x in grp.split()] for grp in re.findall(r"\(([^)]*)\)", m.group(1))]
    ka["cube100_tet_volume"] = [float(m.group(2)) for ln in exp("testTetrahedra-volume")
                                for m in [re.match(rf"Element: 0, Tetrahedra: (\d+), Volume: ({NUM})", ln)] if m]
    area = np.zeros((10, 4))
    for ln in exp("testTetrahedra-face-area"):
        m = re.match(rf"Element: 0, Tetrahedra: (\d+), Face: (\d+), Area: ({NUM})", ln)
        if m:
            area[int(m.group(1)), int(m.group(2))] = float(m.group(3))
    ka["cube100_face_area"] = area.tolist()
    nrm = np.zeros((10, 4, 3))
    for ln in exp("testTetrahedra-face-normal"):
        m = re.match(rf"Element: 0, Tetrahedra: (\d+), Face: (\d+), Normal: ({NUM}) ({NUM}) ({NUM})", ln)
        if m:
            nrm[int(m.group(1)), int(m.group(2))] = [float(m.group(k)) for k in (3, 4, 5)]
    ka["cube100_face_normal"] = nrm.tolist()
    for ln in exp("testUpdateElement-volume"):
        m = re.match(rf"Element: 0, volume: ({NUM})", ln)
        if m:
            ka["cube100_element_volume"] = float(m.group(1))
    for ln in exp("testUpdateElement-minLengthScale"):
        m = re.match(rf"Element: 0, minLengthScale: ({NUM})", ln)
        if m:
            ka["cube100_min_length_scale"] = float(m.group(1))

    # node force / balance (100 m mesh, gravity only) and mass (0.5 m mesh)
    def node_vals(name, key):
        out = {}
        for ln in exp(name):
            m = re.match(rf"\s*(Corner|Edge|Surface|Internal)\s+Node\s+(\d+) \((\d),(\d),(\d)\): {key}: \(?([^)]*)\)?", ln)
            if m:
                out[m.group(1).lower()] = {"node": int(m.group(2)),
                                           "ijk": [int(m.group(k)) for k in (3, 4, 5)],
                                           "value": [float(x) for x in m.group(6).split()]}
        return out

    ka["cube100_gravity_force"] = node_vals("testUpdateNode-force", "force")
    ka["cube100_gravity_balance"] = node_vals("testUpdateNode-balance", "balance")
    ka["cube05_mass"] = node_vals("testUpdateNode-mass", "mass")

    # unit-cube pull test after 10 iterations
    ka["pull_vx_after_10"] = {int(m.group(1)): float(m.group(2)) for ln in exp("testUpdateNode-velocity")
                              for m in [re.match(rf"After 10 iterations, Node (\d+) : vx = ({NUM})", ln)] if m}
    ka["pull_coord_after_10"] = {int(m.group(1)): [float(m.group(k)) for k in (2, 3, 4)]
                                 for ln in exp("testUpdateNode-coord")
                                 for m in [re.match(rf"Node (\d+) : coord = ({NUM}) ({NUM}) ({NUM})", ln)] if m}
    with open(os.path.join(HERE, "libsnac_known_answers.json"), "w") as f:
        json.dump(ka, f, indent=1, sort_keys=True)

    S = os.path.join(root, "Snac", "tests")
    rows = [ln.split() for ln in lines(os.path.join(S, "test-basic.timeStep.0.expected")) if ln.strip()]
    with open(os.path.join(HERE, "basic_timestep.json"), "w") as f:
        json.dump({"rows": [[float(x) for x in r] for r in rows]}, f, indent=1)

    raw = np.fromfile(os.path.join(S, "test-basic-velocity-completeForceCalc.vel.0.expected"), dtype="<f4")
    np.savez_compressed(os.path.join(HERE, "basic_velocity_vel.npz"), vel=raw.reshape(-1, 13 * 11 * 11, 3))
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    # the checkout that holds Snac/: the first argument, else the parent of $SNAC_REF,
    # else reference/ beside this repository
    default = os.path.dirname(os.environ["SNAC_REF"].rstrip("/")) if os.environ.get("SNAC_REF") else \
        os.path.normpath(os.path.join(HERE, "..", "..", "..", "reference"))
    main(sys.argv[1] if len(sys.argv) > 1 else default)
