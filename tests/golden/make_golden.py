"""Extract the reference's golden data for the hot path into a small fixture.

Reads, from a NEMO-3D source tree (its NEMO_3D directory, given as the
argument or in NEMO3D_SRC):
  nemo3d/example/TestRun/GaAs_bulk.old_nd_Ek_ascii  (6400 eigenvalues, 40 k)
  nemo3d/example/TestRun/Si_Bulk.old_nd_Ek_ascii    (358 Lanczos eigenvalues)
  nemo3d/bin/Si_Bulk.nd_nbrIndx                      (8x4 neighbour table)
  nemo3d/example/TestRun/Si_Bulk.nd_Ek               (binary <HDR> file: its
                                                      header and first 16
                                                      records)
and writes tests/golden/reference_golden.npz.  Run it where the reference is
mounted; the fixture then travels with the repository.
"""
import os
import sys

import numpy as np

ROOT = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("NEMO3D_SRC", "")
if not ROOT:
    sys.exit("usage: make_golden.py <NEMO_3D directory of the reference> (or set NEMO3D_SRC)")
HERE = os.path.dirname(os.path.abspath(__file__))


def read_ek(path):
    return np.loadtxt(path, skiprows=5)


def read_nbr(path):
    raw = open(path, "rb").read()
    end = raw.index(b"<\\HDR>") + len(b"<\\HDR>")
    return np.frombuffer(raw[end:], dtype="<i4").reshape(-1, 4)


def main():
    tr = os.path.join(ROOT, "nemo3d", "example", "TestRun")
    gaas = read_ek(os.path.join(tr, "GaAs_bulk.old_nd_Ek_ascii"))
    si = read_ek(os.path.join(tr, "Si_Bulk.old_nd_Ek_ascii"))
    nbr = read_nbr(os.path.join(ROOT, "nemo3d", "bin", "Si_Bulk.nd_nbrIndx"))
    raw = open(os.path.join(tr, "Si_Bulk.nd_Ek"), "rb").read()
    head = raw[:raw.index(b"<\\HDR>") + 6 + 16 * 32]
    np.savez_compressed(os.path.join(HERE, "reference_golden.npz"),
                        gaas_bulk_kE=gaas, si_bulk_kE=si, si_bulk_nbr=nbr,
                        si_bulk_nd_ek_head=np.frombuffer(head, np.uint8))
    print("wrote", gaas.shape, si.shape, nbr.shape, len(head))


if __name__ == "__main__":
    main()
