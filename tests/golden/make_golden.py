"""Regenerates the golden fixtures from the reference tree (run where the reference is present).

* heateq_mesh.npz -- the 2D mesh of fem/tests/heateq/Mesh (408 nodes, 734 linear
  triangles, 86 boundary elements), shared with fem/tests/linearsolvers.
* targets.json    -- the NRM targets those cases print (END TEST CASE ... Target NRM=...),
  parsed from the .sif files.

Usage: python tests/golden/make_golden.py /path/to/elmerfem
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from elmerfem_b200 import meshgen  # noqa: E402


def main(ref):
    tests = os.path.join(ref, "fem", "tests")
    m = meshgen.read_elmer_mesh(os.path.join(tests, "heateq", "Mesh"))
    np.savez_compressed(os.path.join(HERE, "heateq_mesh.npz"), coords=m.coords, elements=m.elements,
                        bnd_elements=m.bnd_elements, bnd_ids=m.bnd_ids)
    sif = open(os.path.join(tests, "heateq", "TempDist.sif")).read()
    heateq = float(re.search(r"Target NRM=([0-9.Ee+-]+)", sif).group(1))
    lin = open(os.path.join(tests, "linearsolvers", "TempDist.sif")).read()
    cases = {int(c): float(v) for c, v in re.findall(r"END TEST CASE (\d+): Taget NRM=([0-9.Ee+-]+)", lin)}
    json.dump({"heateq": {"nrm": heateq, "source": "fem/tests/heateq/TempDist.sif", "eps": 1e-5},
               "linearsolvers": {"nrm_by_case": cases, "source": "fem/tests/linearsolvers/TempDist.sif"}},
              open(os.path.join(HERE, "targets.json"), "w"), indent=1)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_golden.py <path of the reference checkout>")
    main(sys.argv[1])
