"""Pick list (.lst) -> RELION particle STAR file.

Replaces the reference's python_scripts/convert_my-lst_to_relion_mic.py
with the same command line

    python -m gisspa_b200.relion <input lstfile> <scale factor> <pixel size> <out star file> <micrographs dir>

and the same output, value for value: the micrograph name is the list
path's last component behind <micrographs dir> (:28-33), coordinates are the
centres times the integer scale (:47-48), DefocusU/V = (defocus -/+ dfdiff)
x 10^4 (:35-38), rot = fmod(az - 90, 360), tilt = alt, psi = fmod(phi + 90,
360) (:49), magnification 50000 / pixel size (:17), and the fixed columns of
the script.  Numbers are printed as the script's Python 2 `str` prints them:
12 significant digits, ".0" added to integral values.
"""
from __future__ import annotations

import math
import sys
from typing import List, Sequence

HEADER = ("# RELION; version 3.0-beta-2\n\ndata_\n\nloop_\n _rlnMicrographName #1 \n_rlnCoordinateX #2 \n"
          "_rlnCoordinateY #3 \n_rlnImageName #4 \n_rlnDefocusU #5 \n_rlnDefocusV #6 \n_rlnDefocusAngle #7 \n"
          "_rlnVoltage #8 \n_rlnSphericalAberration #9 \n_rlnAmplitudeContrast #10 \n_rlnMagnification #11 \n"
          "_rlnDetectorPixelSize #12 \n_rlnCtfFigureOfMerit #13 \n_rlnGroupNumber #14 \n_rlnAngleRot #15 \n"
          "_rlnAngleTilt #16 \n_rlnAnglePsi #17 \n_rlnOriginX #18 \n_rlnOriginY #19 \n_rlnClassNumber #20 \n"
          "_rlnNormCorrection #21 \n_rlnLogLikeliContribution #22 \n_rlnMaxValueProbDistribution #23 \n"
          "_rlnNrOfSignificantSamples #24\n")


def py2_float_str(x: float) -> str:
    """Python 2's str(float): %.12g, with '.0' added when the result has
    neither a point nor an exponent."""
    if math.isnan(x):
        return "nan"
    if math.isinf(x):
        return "inf" if x > 0 else "-inf"
    s = "%.12g" % x
    if not any(c in s for c in ".en"):
        s += ".0"
    return s


def star_line(line: str, scale: int, apix: float, mdir: str) -> str:
    f = line.split("\t")
    path = f[1]
    micro = mdir + path.split("/")[-1]
    df = float(f[2].split("=")[1]) * 10000
    dfdiff = float(f[3].split("=")[1]) * 10000
    dfang = float(f[4].split("=")[1])
    e = f[5].split("=")[1].split(",")
    alt, az, phi = float(e[0]), float(e[1]), float(e[2])
    c = f[6].split("=")[1].split(",")
    cx, cy = float(c[0]) * scale, float(c[1]) * scale
    mag = 50000 / apix
    s = py2_float_str
    return (micro + "\t" + s(cx) + "\t" + s(cy) + "\t000001@" + micro + "\t" + s(df - dfdiff) + "\t"
            + s(df + dfdiff) + "\t" + s(dfang) + "\t300.000000\t2.700000\t0.100000\t" + s(mag)
            + "\t5.000000\t0.140000\t1\t" + s(math.fmod(az - 90, 360)) + "\t" + s(alt) + "\t"
            + s(math.fmod(phi + 90, 360))
            + "\t0.000000\t0.000000\t1\t0.600000\t1.800000e+05\t1.000000\t1\n")


def lst_to_star(lines: Sequence[str], scale: int, apix: float, mdir: str) -> str:
    return HEADER + "".join(star_line(l, scale, apix, mdir) for l in lines)


def main(argv: List[str]) -> int:
    if len(argv) < 6:
        print("<input lstfile> <scale factor> <pixel size> <out star file> <micrographs dir>")
        return 1
    with open(argv[1]) as fh:
        lines = fh.readlines()
    with open(argv[4], "w") as fh:
        fh.write(lst_to_star(lines, int(argv[2]), float(argv[3]), argv[5]))
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
