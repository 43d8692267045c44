"""Extract the known-answer vectors of the reference's own JUnit tests into
reference_kats.json.

Run here, where the reference sources are readable:

    python tests/golden/make_reference_kats.py <path of the reference checkout>

It reads (as text) these test methods and records every expected gradient,
energy and displacement they assert, with the file:line of the assertion
call, next to the inputs the test constructs:

  test/readdy/impl/sim/core/pot/potentials/P2_HarmonicTest.java   testSetCoordinates_getGrad_getNrg
  test/readdy/impl/sim/core/pot/potentials/P1_DiskTest.java       testSetCoordinates_getGrad_getNrg
  test/readdy/impl/sim/core/bd/PotentialDisplacementComputerTest.java
        testComputeSingleDisplacement, testComputePairDisplacement

The potential parameters come from the tests' setUpClass blocks and the
fixtures they parse (test/testInputFiles/test_default/param_global.xml,
param_particles.xml, test/testInputFiles/test_potentials/tplgy_potentials.xml);
they are restated below with their line numbers.  The tests' tolerance is
assertEquals(..., 0.0001).
"""
import json
import os
import re
import sys

NUM = r"[-+0-9.eE]+"


def _arr(text):
    return [float(v) for v in re.findall(NUM, text)]


def _lines(path):
    with open(path) as f:
        return f.read().split("\n")


def harmonic(ref):
    rel = "test/readdy/impl/sim/core/pot/potentials/P2_HarmonicTest.java"
    L = _lines(os.path.join(ref, rel))
    # setUpClass (:58-91): spring/repulsive/attractive, forceConst 10
    pots = {"potSpring": "spring", "potRepulsive": "repulsive", "potAttractive": "attractive"}
    env = {}
    cases = []
    grad = nrg = None
    for no, line in enumerate(L, 1):
        m = re.search(r"IParticle (p\d) = new Particle\(\d+, \d+, new double\[\]\{(.*?)\}\)", line)
        if m:
            env[m.group(1)] = _arr(m.group(2))
        m = re.search(r"double (dist|radiusS|radiusL) = (" + NUM + ");", line)
        if m:
            env[m.group(1)] = float(m.group(2))
        m = re.search(r"expGrad = new double\[\]\{(.*?)\};", line)
        if m:
            grad = _arr(m.group(1))
        m = re.search(r"expNrg = (" + NUM + ");", line)
        if m:
            nrg = float(m.group(1))
        m = re.search(r"testPotential\((\w+), p1, p2, dist, (\w+), expGrad, expNrg\)", line)
        if m:
            cases.append({"where": f"{rel}:{no}", "subtype": pots[m.group(1)], "k": 10.0,
                          "x1": env["p1"], "x2": env["p2"], "dist": env["dist"],
                          "radius": env[m.group(2)], "grad": grad, "energy": nrg})
    return cases


def disk(ref):
    rel = "test/readdy/impl/sim/core/pot/potentials/P1_DiskTest.java"
    L = _lines(os.path.join(ref, rel))
    # setUpClass (:44-87): both disks forceConst 1, center [0,0,0],
    # normal [-1,1,1], radius 3, considerParticleRadius true
    pots = {"potAttractive": "attractive", "potRepulsive": "repulsive"}
    env = {}
    cases = []
    grad = nrg = None
    for no, line in enumerate(L, 1):
        m = re.search(r"IParticle (\w+) = new Particle\(\d+, \d+, new double\[\]\{(.*?)\}\)", line)
        if m:
            env[m.group(1)] = _arr(m.group(2))
        m = re.search(r"double (pRadius\w) = (" + NUM + ");", line)
        if m:
            env[m.group(1)] = float(m.group(2))
        m = re.search(r"expGrad = new double\[\]\{(.*?)\};", line)
        if m:
            grad = _arr(m.group(1))
        m = re.search(r"expNrg = (" + NUM + ");", line)
        if m:
            nrg = float(m.group(1))
        m = re.search(r"testPotential\((\w+), (\w+), (\w+), expGrad, expNrg\)", line)
        if m and m.group(1) in pots:
            cases.append({"where": f"{rel}:{no}", "subtype": pots[m.group(1)], "k": 1.0,
                          "center": [0.0, 0.0, 0.0], "normal": [-1.0, 1.0, 1.0], "radius": 3.0,
                          "x": env[m.group(2)], "p_radius": env[m.group(3)],
                          "grad": grad, "energy": nrg})
    return cases


def displacement(ref):
    rel = "test/readdy/impl/sim/core/bd/PotentialDisplacementComputerTest.java"
    L = _lines(os.path.join(ref, rel))
    single, pair = [], []
    env = {}
    grad = disp = None
    text = "\n".join(L)
    for no, line in enumerate(L, 1):
        m = re.search(r"(?:IParticle )?(\w+) = new Particle\((\d+), (\d+), new double\[\]\{(.*?)\}\)", line)
        if m:
            env[m.group(1)] = {"id": int(m.group(2)), "type": int(m.group(3)), "x": _arr(m.group(4))}
        m = re.search(r"double (pRadius\w|radius\w) = (" + NUM + ");", line)
        if m:
            env[m.group(1)] = float(m.group(2))
        m = re.search(r"expectedGradient = new double\[\]\{(.*?)\};", line)
        if m:
            grad = _arr(m.group(1))
        m = re.search(r"expectedDisplacement = new double\[\]\{(.*?)\};", line)
        if m:
            disp = _arr(m.group(1))
        m = re.search(r"testComputeSingleDisplacementOnDisk\((\w+), (\w+), expectedGradient", line)
        if m:
            p = env[m.group(1)]
            single.append({"where": f"{rel}:{no}", "type": p["type"], "x": p["x"],
                           "p_radius": env[m.group(2)], "grad": grad, "disp": disp})
        m = re.search(r"testComputePairDisplacementViaHarmonics\(p1, p2, (\w+), expDisplacement\)", line)
        if m:
            # the expDisplacement literal is the last new double[][]{...} before this line
            upto = "\n".join(L[:no])
            blk = upto[upto.rindex("expDisplacement = new double[][]"):]
            rows = re.findall(r"new double\[\]\{(.*?)\}", blk, re.S)
            r = m.group(1)
            radius = env[r] if r in env else float(r)
            pair.append({"where": f"{rel}:{no}", "p1": env["p1"], "p2": env["p2"],
                         "radius": radius, "disp1": _arr(rows[0]), "disp2": _arr(rows[1])})
    del text
    return single, pair


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_reference_kats.py <path of the reference checkout>")
    ref = sys.argv[1]
    single, pair = displacement(ref)
    out = {
        "source": "reference JUnit tests (assertEquals tolerance 1e-4)",
        "tolerance": 1e-4,
        "harmonic": harmonic(ref),
        "disk": disk(ref),
        # fixture parameters of PotentialDisplacementComputerTest:
        #  test/testInputFiles/test_default/param_global.xml: dt 1e-8 s, T 300 K,
        #    Kb 0.0083144621
        #  test/testInputFiles/test_default/param_particles.xml: D(A)=1e6,
        #    D(B)=0.5e6, D(ABcmplx)=0.75e6 nm^2/s (types 0,1,2)
        #  test/testInputFiles/test_potentials/tplgy_potentials.xml:
        #    DISK attractive k=100 center 0 normal z radius 30 on type 0;
        #    CYLINDER attractive k=100 center [0,0,10] normal z radius 30 height 20 on types 1,2;
        #    HARMONIC attractive k=3 on type pairs (1,1),(0,1);
        #    HARMONIC repulsive k=1 on particle-id pair (0,1);
        #    HARMONIC spring k=0.1 on type pair (2,2)
        "displacement_fixture": {
            "dt": 1e-8, "T": 300.0, "Kb": 0.0083144621,
            "D": [1e6, 0.5e6, 0.75e6],
            "disk": {"k": 100.0, "center": [0, 0, 0], "normal": [0, 0, 1], "radius": 30.0, "types": [0]},
            "cylinder": {"k": 100.0, "center": [0, 0, 10], "normal": [0, 0, 1], "radius": 30.0,
                         "height": 20.0, "types": [1, 2]},
            "harmonic_attractive": {"k": 3.0, "type_pairs": [[1, 1], [0, 1]]},
            "harmonic_repulsive_id": {"k": 1.0, "id_pairs": [[0, 1]]},
            "harmonic_spring": {"k": 0.1, "type_pairs": [[2, 2]]},
        },
        "single_displacement": single,
        "pair_displacement": pair,
    }
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_kats.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {dst}: {len(out['harmonic'])} harmonic, {len(out['disk'])} disk, "
          f"{len(single)} single, {len(pair)} pair cases")


if __name__ == "__main__":
    main()
