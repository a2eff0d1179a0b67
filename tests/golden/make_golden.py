"""Generate the known-answer fixtures in this folder from closed-form mathematics.

The reference ships no tests or golden vectors, and the Fortran reference
cannot be compiled here, so the oracle is pinned to values derived directly
from the formulas the reference implements (cited per entry), computed here
independently of the oracle:

  kat_kernels.json   W and dW/dr of every reference kernel at chosen q: the
                     Wendland C6 (kernel.f90:498-508), the cubic spline
                     (kernel.f90:324-340, restored with factor 15/(7 pi)
                     (scale_h/h)^2, default-real literals 2./3. and 1./6. in
                     single precision), and quadratic, Gaussian, quintic,
                     Wendland C2 and C4, Marquis and Marquis2
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


def simple(key: str, q: float, hij: float):
    """W and dW/dr of the other reference kernels (kernel.f90, by subroutine),
    with their scale_h (initialize.f90:208-217)."""
    sh = {"quadratic": 2.0, "gaussian": 3.0, "quintic": 3.0, "wendland_c2": 1.0,
          "wendland_c4": 1.0, "marquis": 3.0, "marquis2": 3.0}[key]
    if key == "quadratic":                                  # :269-276
        f = 2.0 / PI * (sh / hij) ** 2
        w, g = f * (0.1875 * q * q - 0.75 * q + 0.75), f * (0.375 * q - 0.75)
    elif key == "gaussian":                                 # :136-144
        f = 1.0 / PI * (sh / hij) ** 2
        w, g = f * math.exp(-q * q), f * (-2.0 * q * math.exp(-q * q))
    elif key == "quintic":                                  # :193-219
        f = 7.0 / (478.0 * PI) * (sh / hij) ** 2
        t = [(3 - q, 1, -5), (2 - q, -6, 30), (1 - q, 15, -75)]
        w = f * sum(a * u ** 5 for u, a, _ in t if u > 0)
        g = f * sum(b * u ** 4 for u, _, b in t if u > 0)
    elif key == "wendland_c2":                              # :387-393
        f = 3.0 / (2.0 * PI) * (sh / hij) ** 2
        w, g = f * (1 - q) ** 4 * (1 + 4 * q), f * (-20.0 * q * (1 - q) ** 3)
    elif key == "wendland_c4":                              # :443-450
        f = 3.0 / PI * (sh / hij) ** 2
        w, g = f * (1 - q) ** 6 * (35 * q * q + 18 * q + 3), f * (-56 * q * (5 * q + 1) * (1 - q) ** 5)
    elif key == "marquis":                                  # :555-563
        f = 1.0 / PI * (sh / hij) ** 2
        w, g = f * (0.5 - 0.5 * math.tanh(300 * (q - 1))), f * (-150.0 / math.cosh(300 * (q - 1)) ** 2)
    else:                                                   # marquis2, :612-620
        c1, c2 = 10.0, 50.0
        l2 = real4(math.log(2.0))    # log of the default real 2.
        f = 1.0 / (real4(34.1558) * PI * hij ** 2)
        w = f * c2 * (math.log(math.cosh(c1 * (1 - q))) / c1 - q + 1 + l2 / c1)
        g = f * (-c2 * math.tanh(c1 * (1 - q)) - 1)
    return w, g / hij * sh


SIMPLE_Q = {"quadratic": (0.1, 0.7, 1.4, 1.9), "gaussian": (0.2, 0.9, 1.7, 2.8),
            "quintic": (0.3, 0.9, 1.2, 1.8, 2.4, 2.9), "wendland_c2": (0.1, 0.4, 0.8),
            "wendland_c4": (0.1, 0.4, 0.8), "marquis": (0.5, 0.995, 1.003, 2.0),
            "marquis2": (0.2, 0.9, 1.1, 2.5)}


def kernels():
    hij = 1000.0
    out = {"hsml_ij": hij, "wendland_c6": [], "cubic": []}
    for key, qs in SIMPLE_Q.items():
        sh = {"quadratic": 2.0, "wendland_c2": 1.0, "wendland_c4": 1.0}.get(key, 3.0)
        out[key] = []
        for q in qs:
            w, g = simple(key, q, hij)
            out[key].append({"q": q, "r": q * hij / sh, "w": w, "dwdr": g})
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
