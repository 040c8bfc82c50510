"""Reader of the reference's <HDR> result files.

A file is a text header -- ``<HDR>``, ``record format = {...}``, ``record
dimension i = n label``, ``user data i =text``, ``<\\HDR>`` (nemo3d/src/io/
fileformat.c:182-204) -- followed by native-endian binary records of the
listed fields (``real`` = 8-byte double, ``int`` = 4 bytes, ``float`` = 4
bytes).  ``nd_Ek`` holds {kx, ky, kz, E} per eigenvalue, ``nd_evec*`` holds
{wf.r, wf.i} per basis state.  The library writes them with
``tbgpu_write_eigenvalues`` / ``tbgpu_write_eigenvector``; this module reads
those and the reference's own files.
"""

from __future__ import annotations

import re

import numpy as np

_TYPES = {"real": np.float64, "int": np.int32, "float": np.float32}


def read(path: str):
    """Return (header dict, structured record array)."""
    raw = open(path, "rb").read()
    end = raw.index(b"<\\HDR>")
    text = raw[:end].decode("ascii", "replace")
    hdr = {"format": None, "dims": [], "dim_labels": [], "user": []}
    for line in text.splitlines():
        if "=" not in line:
            continue
        key, val = line.split("=", 1)
        key = key.strip()
        if key == "record format":
            hdr["format"] = val.strip()
        elif key.startswith("record dimension"):
            parts = val.split(None, 1)
            hdr["dims"].append(int(parts[0]))
            hdr["dim_labels"].append(parts[1].strip() if len(parts) > 1 else "")
        elif key.startswith("user data"):
            hdr["user"].append(val)
    fields = re.findall(r"(real|int|float)\s+([\w.]+)", hdr["format"] or "")
    dtype = np.dtype([(name, _TYPES[t]) for t, name in fields])
    body = raw[end + 6:]
    data = np.frombuffer(body[:len(body) // dtype.itemsize * dtype.itemsize], dtype=dtype)
    return hdr, data


def read_eigenvalues(path: str) -> np.ndarray:
    """nd_Ek file -> array [n, 4] of (kx, ky, kz, E)."""
    hdr, rec = read(path)
    n = hdr["dims"][0]
    return np.stack([rec[f] for f in rec.dtype.names], axis=1)[:n]


def read_eigenvector(path: str) -> np.ndarray:
    """nd_evec file -> complex vector [atoms * orbitals]."""
    hdr, rec = read(path)
    n = hdr["dims"][0] * hdr["dims"][1]
    return (rec["wf.r"] + 1j * rec["wf.i"])[:n]
