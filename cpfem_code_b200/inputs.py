"""fs3pre's input files: material property sets (``.fmt``) and Gauss-point
orientation lists (``.ori``).

A user of the reference prepares these for the pre-processor; reading them
here lets the same files drive :func:`cpfem_code_b200.generator.structured_cube`.

* ``.fmt`` (SETMATC, src/prepro/fs3p-matl.f90:75-108), list-directed: the
  number of plastic parameters, the number of slip systems ns, the 9
  compliances, ns reorientation angles (twins: |angle| > 1.5), ns lines of
  slip direction and plane normal, ns lines of plastic parameters, and ns
  lines of the latent-hardening matrix, line i holding column i.
* ``.ori`` (SETSTATE option 4, src/prepro/fs3p-gps.f90:227-236): one line
  per Gauss point, a leading value that is ignored and three Euler angles
  (phi1, Phi, phi2) in radians.
"""
from __future__ import annotations

import os

import numpy as np


def _numbers(path: str) -> list[float]:
    with open(path) as f:
        return [float(t) for t in f.read().replace(",", " ").split()]


def read_fmt(path: str) -> dict:
    """A material property set in the generator's material format."""
    v = _numbers(path)
    pos = 0

    def take(n):
        nonlocal pos
        if pos + n > len(v):
            raise ValueError(f"{path}: file ends early")
        out = np.array(v[pos:pos + n])
        pos += n
        return out

    nmpar = int(take(1)[0])
    ns = int(take(1)[0])
    if not (1 <= nmpar <= 10 and 1 <= ns <= 60):
        raise ValueError(f"{path}: {nmpar} plastic parameters, {ns} systems")
    e = take(9)
    ssang = take(ns)
    dn = take(6 * ns).reshape(ns, 6)
    ampar = np.zeros((ns, 10))
    ampar[:, :nmpar] = take(nmpar * ns).reshape(ns, nmpar)
    cols = take(ns * ns).reshape(ns, ns)          # line i = smatrx(1:ns, i)
    return dict(name=os.path.splitext(os.path.basename(path))[0], ns=ns, nmpar=nmpar, e=e, ssang=ssang,
                ab=dn[:, :3].copy(), an=dn[:, 3:].copy(), ampar=ampar, smatrx=cols.T.copy())


def read_ori(path: str, ngps: int | None = None) -> np.ndarray:
    """Euler angles [ngps, 3] (radians), one Gauss point per line."""
    rows = []
    with open(path) as f:
        for line in f:
            t = line.replace(",", " ").split()
            if not t:
                continue
            if len(t) < 4:
                raise ValueError(f"{path}: line {len(rows) + 1} has {len(t)} values")
            rows.append([float(t[1]), float(t[2]), float(t[3])])
            if ngps is not None and len(rows) == ngps:
                break
    out = np.array(rows, dtype=np.float64).reshape(-1, 3)
    if ngps is not None and len(out) < ngps:
        raise ValueError(f"{path}: {len(out)} orientations for {ngps} Gauss points")
    return out
