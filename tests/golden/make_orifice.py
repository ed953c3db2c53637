"""Writes tests/golden/orifice_compact.npz: the compact part of the
reference's own mesher output src/core/common/tests/assets/orifice.mles
(1056 cells, 5654 internal faces, 693 boundary faces in 6 zones), read by
this project's .mles reader (nextgen_b200.mles) and reduced to what the
solver's operator build takes (nextgen_b200.mles.CompactMesh).  The GPU
tests run the solver on it where the reference tree is not present.

  python tests/golden/make_orifice.py [reference root]
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from nextgen_b200.mles import CompactMesh, MlesMesh  # noqa: E402


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REFERENCE_ROOT", "/root/reference")
    m = MlesMesh(os.path.join(root, "src/core/common/tests/assets/orifice.mles"))
    c = CompactMesh.from_mles(m)
    out = os.path.join(HERE, "orifice_compact.npz")
    c.save(out)
    print("wrote %s: %d cells, %d faces, %d boundary faces, zones %s" % (out, c.ncv, c.nfa, c.nbf, c.zone_names))


if __name__ == "__main__":
    main()
