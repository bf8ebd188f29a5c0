#!/usr/bin/env python3
"""Write rot_consts.cuh: exact constants of the rotations by j*2pi/48.

The register DFTs (radix 8, 12, 16) rotate by multiples of 2pi/48.  The
FP64 form needs (cos, sin); the FP32 form needs the lifting parameters
(t = tan(phi'/2), s = sin(phi'), g) of make_rotf().  They are computed here
in extended precision so that the device code holds literal constants.
"""
import math
import os
from decimal import Decimal, getcontext

import numpy as np

getcontext().prec = 40


def rotf(phi):
    pi = math.pi
    p = math.remainder(phi, 2 * pi)
    g = 1.0
    if p > 0.5 * pi:
        p -= pi
        g = -1.0
    elif p < -0.5 * pi:
        p += pi
        g = -1.0
    return float(np.float32(math.tan(0.5 * p))), float(np.float32(math.sin(p))), g


lines = ["// rot_consts.cuh -- generated by gen_consts.py; rotations by j*2pi/48.",
         "#pragma once", "namespace espec {", "namespace rc {",
         "ESPEC_HD constexpr double cd(int j) {", "  switch (j) {"]
for j in range(48):
    lines.append(f"    case {j}: return {math.cos(2 * math.pi * j / 48)!r};")
lines += ["  }", "  return 0.0;", "}", "ESPEC_HD constexpr double sd(int j) {", "  switch (j) {"]
for j in range(48):
    lines.append(f"    case {j}: return {math.sin(2 * math.pi * j / 48)!r};")
lines += ["  }", "  return 0.0;", "}"]
for name, idx in (("tf", 0), ("sf", 1), ("gf", 2)):
    lines += [f"ESPEC_HD constexpr float {name}(int j) {{", "  switch (j) {"]
    for j in range(48):
        v = rotf(2 * math.pi * j / 48)[idx]
        lines.append(f"    case {j}: return {np.float32(v)!r}f;".replace("np.float32(", "").replace(")f", "f"))
    lines += ["  }", "  return 0.0f;", "}"]
lines += ["}  // namespace rc", "}  // namespace espec", ""]
out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "rot_consts.cuh")
with open(out, "w") as f:
    f.write("\n".join(lines))
print("wrote", out)
