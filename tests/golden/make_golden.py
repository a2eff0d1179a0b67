"""Generate the known-answer fixtures in this folder from closed-form mathematics.

The reference ships no tests or golden vectors, and the Fortran reference
cannot be compiled here, so the oracle is pinned to values derived directly
from the formulas the reference implements (cited per entry), computed here
independently of the oracle:

  kat_kernels.json   W and dW/dq of the Wendland C6 (kernel.f90:498-508) and
                     the cubic spline (kernel.f90:324-340, restored with
                     factor 15/(7 pi) (scale_h/h)^2, default-real literals
                     2./3. and 1./6. in single precision) at chosen q
  kat_lattice.json   neighbour counts of an interior particle of a perfect
                     square lattice for SIMP support radii 2.4 dx and 3 dx
                     (pairs iff r <= (hsml_i + hsml_j) / 2, nnps.f90:281)
  kat_physics.json   free-drift speed of uniform ice under uniform wind with
                     quadratic air and water drag (wind_forcing.f90:41-49,
                     water_drag.f90:42-50) and the constants of
                     data_variables.f90:157-180

Run:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import math
import os
import struct

HERE = os.path.dirname(os.path.abspath(__file__))
PI = 3.1415926535897932


def real4(v: float) -> float:
    return struct.unpack("f", struct.pack("f", v))[0]


def c6(q: float, hij: float):
    """W and dW/dr * (1/r) factor pieces for Wendland C6 with scale_h = 1."""
    f = 78.0 / (7.0 * PI) * (1.0 / hij) ** 2
    w = f * (1 - q) ** 8 * (32 * q ** 3 + 25 * q ** 2 + 8 * q + 1)
    dwdq = f * (-22.0 * q * (1 - q) ** 7 * (16 * q ** 2 + 7 * q + 1))
    return w, dwdq / hij          # dW/dr = dwdq * scale_h / hij


def cubic(q: float, hij: float):
    sh = 2.0
    f = 15.0 / (7.0 * PI) * (sh / hij) ** 2
    c23, c16 = real4(2.0 / 3.0), real4(1.0 / 6.0)
    if q <= 1.0:
        w = f * (c23 - q ** 2 + 0.5 * q ** 3)
        g = f * (-2.0 * q + 1.5 * q ** 2)
    else:
        w = f * (c16 * (2.0 - q) ** 3)
        g = f * (-0.5 * (2.0 - q) ** 2)
    return w, g / hij * sh


def kernels():
    hij = 1000.0
    out = {"hsml_ij": hij, "wendland_c6": [], "cubic": []}
    for q in (0.05, 0.25, 0.5, 0.75, 0.95):
        w, g = c6(q, hij)
        out["wendland_c6"].append({"q": q, "r": q * hij, "w": w, "dwdr": g})
    for q in (0.1, 0.5, 1.0, 1.25, 1.5, 1.9):
        r = q * hij / 2.0
        w, g = cubic(q, hij)
        out["cubic"].append({"q": q, "r": r, "w": w, "dwdr": g})
    return out


def lattice():
    def count(support: float) -> int:
        n = 0
        R = int(math.ceil(support)) + 1
        for i in range(-R, R + 1):
            for j in range(-R, R + 1):
                if (i, j) != (0, 0) and math.hypot(i, j) <= support:
                    n += 1
        return n
    return {"support_over_dx": {"2.4": count(2.4), "3.0": count(3.0)}}


def physics():
    rho_air, c_air = real4(1.3), 1.2e-3
    rho_w, c_w = 1026.0, 5.5e-3
    s = math.sqrt(rho_air * c_air / (rho_w * c_w))
    U = 10.0
    # rho_a c_a (U-u)^2 = rho_w c_w u^2  ->  u = U s / (1 + s)
    return {"wind": U, "s": s, "free_drift_speed": U * s / (1.0 + s)}


def main():
    for name, obj in (("kat_kernels.json", kernels()), ("kat_lattice.json", lattice()),
                      ("kat_physics.json", physics())):
        with open(os.path.join(HERE, name), "w") as f:
            json.dump(obj, f, indent=1)
        print("wrote", name)


if __name__ == "__main__":
    main()
