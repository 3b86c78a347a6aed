"""Reference-compatible file formats for the GisSPA search boundary.

Python mirror of the reference's readers and writer, used by the Python
wrapper, the tests and the synthetic-data generator.  The C++ driver
(``csrc/driver``) implements the same rules natively.

* config file: ``key = value`` lines, ``#`` comments
  (EMReader/DataReader.cpp:128-265);
* Euler file: ``alt az`` per line (DataReader.cpp:267-284);
* input list (EMAN ``#LST``): ``nn<TAB>path<TAB>defocus=..<TAB>dfdiff=..<TAB>dfang=..``
  with the path relative to the list's directory and the first line always
  consumed as a header (DataReader.cpp:318-388, main.cu:125-138);
* MRC images and stacks (EMReader/emdata_.cpp:384-617);
* output pick lines (main.cu:985-987).
"""
from __future__ import annotations

import os
import struct
from dataclasses import dataclass, field, fields
from typing import Dict, List, Optional, Tuple

import numpy as np

f32 = np.float32

MRC_HEADER_BYTES = 1024


# ---------------------------------------------------------------------------
# Config (DataReader.h:14-42 defaults, DataReader.cpp:128-265 parser)
# ---------------------------------------------------------------------------
@dataclass
class Config:
    inlst: str = "  "
    temp2d: str = "  "
    eulerf: str = "  "
    apix: float = -1.0
    phi_step: float = -1.0
    kk: float = -1.0
    energy: float = -1.0
    cs: float = -1.0
    highres: float = -1.0
    lowres: float = -1.0
    d_m: float = -1.0
    outlst: str = "./outlst"
    first: int = -1
    last: int = -1
    thres: float = 7.0
    device_id: int = 0
    padding_size: int = 320
    phase_flip: int = 0
    overlap: int = -1
    norm_type: int = 0
    invert: int = 0
    # keys of this implementation that the reference ignores
    precision: str = "fp32"
    unknown: List[str] = field(default_factory=list)


_KEYS = {
    "input": ("inlst", str), "template": ("temp2d", str), "eulerfile": ("eulerf", str),
    "kk": ("kk", float), "angpix": ("apix", float), "phistep": ("phi_step", float),
    "energy": ("energy", float), "cs": ("cs", float), "Highres": ("highres", float),
    "Lowres": ("lowres", float), "diameter": ("d_m", float), "output": ("outlst", str),
    "first": ("first", int), "last": ("last", int), "threshold": ("thres", float),
    "GPU_ID": ("device_id", int), "window_size": ("padding_size", int),
    "phase_flip": ("phase_flip", int), "overlap": ("overlap", int),
    "norm_type": ("norm_type", int), "invert": ("invert", int),
    "precision": ("precision", str),
}


def _atoi(s: str) -> int:
    s = s.strip()
    i = 0
    if i < len(s) and s[i] in "+-":
        i += 1
    while i < len(s) and s[i].isdigit():
        i += 1
    try:
        return int(s[:i])
    except ValueError:
        return 0


def _atof(s: str) -> float:
    s = s.strip()
    best = 0.0
    for k in range(len(s), 0, -1):
        try:
            best = float(s[:k])
            return float(f32(best))
        except ValueError:
            continue
    return 0.0


def parse_config_line(line: str, cfg: Config) -> None:
    """One ``key = value`` line, as DataReader.cpp:128-246 splits it: the key
    ends at the first ' ' or '=', the value starts after the following run of
    ' ' and '=' and runs to the end of the line."""
    i = 0
    while i < len(line) and line[i] not in " =":
        i += 1
    option = line[:i]
    while i < len(line) and line[i] in " =":
        i += 1
    value = line[i:]
    if option in _KEYS:
        name, typ = _KEYS[option]
        if typ is str:
            setattr(cfg, name, value)
        elif typ is int:
            setattr(cfg, name, _atoi(value))
        else:
            setattr(cfg, name, _atof(value))
    else:
        cfg.unknown.append(value)


def read_config(path: str) -> Config:
    cfg = Config()
    with open(path, "r") as fh:
        for raw in fh.read().split("\n"):
            if raw == "" or raw[0] == "#":
                continue
            parse_config_line(raw, cfg)
    return cfg


def missing_required(cfg: Config) -> List[str]:
    """checkRequestPara (DataReader.cpp:302-315)."""
    out = []
    if cfg.inlst.startswith(" "):
        out.append("input")
    if cfg.temp2d.startswith(" "):
        out.append("template")
    if cfg.eulerf.startswith(" "):
        out.append("eulerfile")
    for key, name in (("angpix", "apix"), ("phistep", "phi_step"), ("kk", "kk"),
                      ("energy", "energy"), ("cs", "cs"), ("Highres", "highres"),
                      ("Lowres", "lowres"), ("diameter", "d_m")):
        if getattr(cfg, name) < 0:
            out.append(key)
    return out


def write_config(path: str, items: Dict[str, object]) -> None:
    with open(path, "w") as fh:
        for k, v in items.items():
            fh.write("%s = %s\n" % (k, v))


# ---------------------------------------------------------------------------
# Euler file and input list
# ---------------------------------------------------------------------------
def read_euler(path: str) -> np.ndarray:
    """(N, 2) float32 of (alt, az) (DataReader.cpp:267-284)."""
    rows = []
    with open(path, "r") as fh:
        for raw in fh.read().split("\n"):
            if raw == "" or raw[0] == "#":
                continue
            parts = raw.split()
            vals = []
            for tok in parts[:2]:
                try:
                    vals.append(float(tok))
                except ValueError:
                    break
            while len(vals) < 2:
                vals.append(0.0)
            rows.append(vals)
    return np.asarray(rows, dtype=np.float32).reshape(-1, 2)


def write_euler(path: str, alt_az: np.ndarray) -> None:
    with open(path, "w") as fh:
        for alt, az in alt_az:
            fh.write("%f\t%f\t0\n" % (alt, az))


@dataclass
class LstEntry:
    nn: int
    path: str          # as written to the output: list-directory prefix + name
    defocus: float     # value as written in the list (positive underfocus, um)
    dfdiff: float
    dfang: float


def _parse_pairs(rest: str) -> Tuple[float, float, float]:
    defocus = dfdiff = dfang = 0.0
    for tok in rest.split():
        if tok.startswith("defocus="):
            try:
                defocus = float(f32(float(tok[8:])))
            except ValueError:
                pass
        elif tok.startswith("dfdiff="):
            try:
                dfdiff = float(f32(float(tok[7:])))
            except ValueError:
                pass
        elif tok.startswith("dfang="):
            try:
                dfang = float(f32(float(tok[6:])))
            except ValueError:
                pass
    return defocus, dfdiff, dfang


def read_lst_entry(inlst: str, n: int) -> Optional[LstEntry]:
    """Entry ``n`` of a plain EMAN list (DataReader.cpp:348-363): the first line
    is consumed unconditionally, then '#' lines are skipped.  The path gets the
    list's directory prefixed (main.cu:125-138)."""
    with open(inlst, "r") as fh:
        lines = fh.read().split("\n")
    if not lines:
        return None
    body = [ln for ln in lines[1:] if ln != "" and not ln.startswith("#")]
    if n < 0:
        n = 0
    if n >= len(body):
        return None
    parts = body[n].split(None, 2)
    nn = _atoi(parts[0]) if parts else 0
    name = parts[1] if len(parts) > 1 else ""
    rest = parts[2] if len(parts) > 2 else ""
    slash = inlst.rfind("/")
    prefix = inlst[:slash + 1] if slash >= 0 else ""
    d, dd, da = _parse_pairs(rest)
    return LstEntry(nn, prefix + name, d, dd, da)


def write_lst(path: str, entries: List[Tuple[int, str, float, float, float]]) -> None:
    with open(path, "w") as fh:
        fh.write("#LST\n")
        for nn, name, d, dd, da in entries:
            fh.write("%d\t%s\tdefocus=%g\tdfdiff=%g\tdfang=%g\n" % (nn, name, d, dd, da))


def format_pick_line(nn: int, path: str, defocus: float, dfdiff: float, dfang: float,
                     alt: float, az: float, phi: float, cx: float, cy: float,
                     score: float) -> str:
    """main.cu:985-987 (every value a float32 printed through %f)."""
    vals = tuple(float(f32(v)) for v in (defocus, dfdiff, dfang, alt, az, phi, cx, cy, score))
    return ("%d\t%s\tdefocus=%f\tdfdiff=%f\tdfang=%f\teuler=%f,%f,%f\tcenter=%f,%f\tscore=%f\n"
            % ((nn, path) + vals))


def parse_pick_line(line: str) -> Dict[str, object]:
    parts = line.rstrip("\n").split("\t")
    out: Dict[str, object] = {"nn": int(parts[0]), "path": parts[1]}
    for tok in parts[2:]:
        k, v = tok.split("=", 1)
        if k in ("euler", "center"):
            out[k] = tuple(float(x) for x in v.split(","))
        else:
            out[k] = float(v)
    return out


# ---------------------------------------------------------------------------
# MRC (EMReader/emdata_.cpp:384-617, header layout EMReader/ImgType.h mrcH)
# ---------------------------------------------------------------------------
def write_mrc(path: str, data: np.ndarray, apix: float = 1.0) -> None:
    """Little-endian mode-2 MRC; 2D image or (nz, ny, nx) stack."""
    a = np.asarray(data, dtype="<f4")
    if a.ndim == 2:
        a = a[None]
    nz, ny, nx = a.shape
    hdr = bytearray(MRC_HEADER_BYTES)
    struct.pack_into("<10i", hdr, 0, nx, ny, nz, 2, 0, 0, 0, nx, ny, nz)
    struct.pack_into("<6f", hdr, 40, nx * apix, ny * apix, nz * apix, 90.0, 90.0, 90.0)
    struct.pack_into("<3i", hdr, 64, 1, 2, 3)
    struct.pack_into("<3f", hdr, 76, float(a.min()), float(a.max()), float(a.mean()))
    struct.pack_into("<2i", hdr, 88, 0, 0)
    hdr[208:212] = b"MAP "
    hdr[212:216] = bytes([0x44, 0x44, 0x00, 0x00])
    struct.pack_into("<f", hdr, 216, float(a.std()))
    struct.pack_into("<i", hdr, 220, 1)
    label = b"gisspa_b200 synthetic"
    hdr[224:224 + len(label)] = label
    with open(path, "wb") as fh:
        fh.write(bytes(hdr))
        fh.write(a.tobytes())


def read_mrc_header(path: str) -> Dict[str, object]:
    with open(path, "rb") as fh:
        hdr = fh.read(MRC_HEADER_BYTES)
    if len(hdr) < MRC_HEADER_BYTES:
        raise IOError("short MRC header: %s" % path)
    big = hdr[0] == 0 and hdr[1] == 0
    e = ">" if big else "<"
    nx, ny, nz, mode = struct.unpack_from(e + "4i", hdr, 0)
    nsymbt = struct.unpack_from(e + "i", hdr, 92)[0]
    nlabl = struct.unpack_from(e + "i", hdr, 220)[0]
    return {"nx": nx, "ny": ny, "nz": nz, "mode": mode, "nsymbt": nsymbt,
            "nlabl": nlabl, "endian": e}


def read_mrc(path: str, section: int = -1) -> np.ndarray:
    """Section ``section`` of an MRC image/stack as float32 (ny, nx), or the
    whole (nz, ny, nx) volume for an out-of-range section, following
    readMRC's mode conversions (mode 0 as unsigned bytes /100 - 1.28, 1 int16,
    2 float32, 4 as float pairs, 6 uint16)."""
    h = read_mrc_header(path)
    nx, ny, nz, mode = h["nx"], h["ny"], h["nz"], h["mode"]
    if ny > 0xFFFF or nz > 0xFFFF or mode > 4 or h["nlabl"] > 11:
        raise IOError("invalid MRC file: %s" % path)
    if ny == 1:
        raise IOError("1D MRC file: %s" % path)
    if mode in (3, 4):
        nx *= 2
    if 0 <= section < nz:
        z0, zn = section, 1
    else:
        z0, zn = 0, nz
    e = h["endian"]
    dt = {0: np.dtype("u1"), 1: np.dtype(e + "i2"), 2: np.dtype(e + "f4"),
          3: np.dtype(e + "i2"), 4: np.dtype(e + "f4"), 6: np.dtype(e + "u2")}[mode]
    if mode == 3:
        raise IOError("short-complex MRC input is not supported: %s" % path)
    count = nx * ny * zn
    with open(path, "rb") as fh:
        fh.seek(MRC_HEADER_BYTES + h["nsymbt"] + z0 * nx * ny * dt.itemsize)
        raw = np.frombuffer(fh.read(count * dt.itemsize), dtype=dt)
    if raw.size != count:
        raise IOError("truncated MRC data: %s" % path)
    if mode == 0:
        out = (raw.astype(np.float64) / 100.0 - 1.28).astype(np.float32)
    else:
        out = raw.astype(np.float32)
    out = out.reshape(zn, ny, nx)
    return out[0] if zn == 1 else out
