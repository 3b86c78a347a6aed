"""Restatement of the reference's duplicate merging of pick lists
(python_scripts/remove_repeat_particles_from_list.py), float64 like the
script.

TEST INFRASTRUCTURE: only tests/ may import this module; the product never
does.

Lines are grouped into runs of consecutive lines with the same micrograph
path (remove_repeat_particles_from_list.py:22-35).  Inside a run, picks are
visited in order (:36-50); a pick already removed when its turn comes is
skipped, but a pick removed later in its own turn keeps comparing.  Pick j
(after i, not yet removed) is a duplicate of i when their centres are closer
than `center` (:53-57) and their orientations are closer than `euler_thres`
degrees, or than that modulo 180 (:131-135); then the lower score is removed
(ties remove i, :136-140).  The orientation distance is the rotation angle
of R_j^T-like product of the two Euler matrices (:59-94), taken from the
rotation's quaternion (:96-128) with the script's branch order: in the
non-positive-trace case the second branch always overrides the first, and
pairs whose square-root argument is negative or whose q0 leaves [-1, 1] are
not compared.
"""
from __future__ import annotations

import math
from typing import List, Optional, Sequence

PI = 3.14159265359  # the script's constant (:15)


def parse_line(line: str):
    f = line.split("\t")
    alt, az, phi = (float(v) for v in f[5].split("=")[1].split(",")[:3])
    x, y = (float(v) for v in f[6].split("=")[1].split(",")[:2])
    score = float(f[7].split("=")[1])
    return f[1], x, y, alt, az, phi, score


def euler_distance(a1: float, z1: float, p1: float, a2: float, z2: float, p2: float) -> Optional[float]:
    """Rotation angle (degrees) between orientations 1 and 2 (angles in
    degrees), or None where the script skips the pair."""
    alt, az, phi = a1 * PI / 180, z1 * PI / 180, p1 * PI / 180
    alt_o, az_o, phi_o = a2 * PI / 180, z2 * PI / 180, p2 * PI / 180
    c, s = math.cos, math.sin
    # matrix of orientation 2 (:62-70)
    mo = [c(phi_o) * c(az_o) - s(phi_o) * c(alt_o) * s(az_o),
          c(phi_o) * s(az_o) + s(phi_o) * c(alt_o) * c(az_o),
          s(phi_o) * s(alt_o),
          -s(phi_o) * c(az_o) - c(phi_o) * c(alt_o) * s(az_o),
          -s(phi_o) * s(az_o) + c(phi_o) * c(alt_o) * c(az_o),
          c(phi_o) * s(alt_o),
          s(alt_o) * s(az_o),
          -s(alt_o) * c(az_o),
          c(alt_o)]
    # matrix of orientation 1, transposed layout (:72-80)
    m = [c(phi) * c(az) - s(phi) * c(alt) * s(az),
         -s(phi) * c(az) - c(phi) * c(alt) * s(az),
         s(alt) * s(az),
         c(phi) * s(az) + s(phi) * c(alt) * c(az),
         -s(phi) * s(az) + c(phi) * c(alt) * c(az),
         -s(alt) * c(az),
         s(phi) * s(alt),
         c(phi) * s(alt),
         c(alt)]
    # relative rotation (:82-90)
    r = [m[0] * mo[0] + m[3] * mo[1] + m[6] * mo[2],
         mo[0] * m[1] + mo[1] * m[4] + mo[2] * m[7],
         mo[0] * m[2] + mo[1] * m[5] + mo[2] * m[8],
         mo[3] * m[0] + mo[4] * m[3] + mo[5] * m[6],
         mo[3] * m[1] + mo[4] * m[4] + mo[5] * m[7],
         mo[3] * m[2] + mo[4] * m[5] + mo[5] * m[8],
         mo[6] * m[0] + mo[7] * m[3] + mo[8] * m[6],
         mo[6] * m[1] + mo[7] * m[4] + mo[8] * m[7],
         mo[6] * m[2] + mo[7] * m[5] + mo[8] * m[8]]
    tr = r[0] + r[4] + r[8]
    q0 = None
    if tr > 0:
        t = math.sqrt(1 + tr) * 2
        if t == 0:
            return None
        q0 = 0.25 * t
    if tr <= 0:
        if r[0] >= r[4] and r[0] >= r[8]:
            t = math.sqrt(1 + r[0] - r[4] - r[8]) * 2
            if t == 0:
                return None
            q0 = (r[7] - r[5]) / t
        if r[4] > r[8]:
            if 1 - r[0] + r[4] - r[8] < 0:
                return None
            t = math.sqrt(1 - r[0] + r[4] - r[8]) * 2
            if t == 0:
                return None
            q0 = (r[2] - r[6]) / t
        else:
            if 1 - r[0] - r[4] + r[8] < 0:
                return None
            t = math.sqrt(1 - r[0] - r[4] + r[8]) * 2
            if t == 0:
                return None
            q0 = (r[3] - r[1]) / t
    if q0 > 1 or q0 < -1:
        return None
    return abs(math.acos(q0) * 2 * 180 / PI)


def is_duplicate(p, q, center: float, euler_thres: float) -> bool:
    _, x1, y1, a1, z1, f1, _ = p
    _, x2, y2, a2, z2, f2, _ = q
    dist = abs(math.sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1)))
    if not dist < center:
        return False
    ed = euler_distance(a1, z1, f1, a2, z2, f2)
    if ed is None:
        return False
    d2 = ed % 180
    if d2 > euler_thres + 1:
        d2 = 180 - d2
    return ed < euler_thres or d2 < euler_thres


def merge_keep(lines: Sequence[str], center: float, euler_thres: float) -> List[bool]:
    """keep flag per line."""
    recs = [parse_line(l) for l in lines]
    keep = [True] * len(recs)
    start = 0
    while start < len(recs):
        end = start
        while end < len(recs) and recs[end][0] == recs[start][0]:
            end += 1
        removed = [False] * (end - start)
        for i in range(start, end):
            if removed[i - start]:
                continue
            for j in range(i + 1, end):
                if removed[j - start]:
                    continue
                if is_duplicate(recs[i], recs[j], center, euler_thres):
                    if recs[i][6] > recs[j][6]:
                        removed[j - start] = True
                    else:
                        removed[i - start] = True
        for k in range(start, end):
            keep[k] = not removed[k - start]
        start = end
    return keep


def merge_lines(lines: Sequence[str], center: float, euler_thres: float) -> List[str]:
    return [l for l, k in zip(lines, merge_keep(lines, center, euler_thres)) if k]
