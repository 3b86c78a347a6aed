"""gisspa_b200: B200-native GisSPA 2D template-matching search.

Thin ctypes binding of the C ABI in ``include/gisspa.h`` (the library
``gisspa_b200/lib/libgisspa_b200.so``, built by ``gisspa_b200.build``).
There is no CPU fallback: every call runs the CUDA kernels, and a missing
library or GPU raises.

Typical use mirrors the reference's driver (main.cu:1025-1269)::

    ctx = Context(device=0)
    ctx.set_templates(params, templates, first_ctf=(defocus, dfdiff, dfang))
    picks = ctx.search(micrograph, ctf=(defocus, dfdiff, dfang))
"""
from __future__ import annotations

import ctypes as C
import os
from typing import List, Optional, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libgisspa_b200.so")
DRIVER_PATH = os.path.join(HERE, "lib", "gisspa_main")

GS_OK = 0
GS_ERR_ARG, GS_ERR_OOM, GS_ERR_CUDA, GS_ERR_STATE, GS_ERR_UNSUPPORTED, GS_ERR_TIMEOUT, GS_ERR_IO = range(1, 8)
STATUS = {0: "ok", 1: "invalid argument", 2: "out of memory", 3: "CUDA error",
          4: "invalid call order", 5: "unsupported input", 6: "device wait timed out",
          7: "I/O error"}
# arithmetic of the correlation's DFT stages (gs_params.precision)
GS_PREC_FP32, GS_PREC_TC_BF16, GS_PREC_TC_FP16, GS_PREC_TC_FULL, GS_PREC_TC_FULL_1P = 0, 1, 2, 3, 4
# gs_set_option options (include/gisspa.h)
GS_OPT_GENERIC_FFT, GS_OPT_TWO_PASS, GS_OPT_WINDOW_BLOCK, GS_OPT_CORR_SLOTS, GS_OPT_CORR_LAG = 1, 2, 3, 4, 5
GS_OPT_CORR_CTAS, GS_OPT_GRAPH, GS_OPT_AUTOTUNE, GS_OPT_CORR_TILE, GS_OPT_ANGLES_PER_LAUNCH = 6, 7, 8, 9, 10


class GsParams(C.Structure):
    _fields_ = [("apix", C.c_float), ("phi_step", C.c_float), ("kk", C.c_float),
                ("energy", C.c_float), ("cs", C.c_float), ("highres", C.c_float),
                ("lowres", C.c_float), ("d_m", C.c_float), ("thres", C.c_float),
                ("window_size", C.c_int), ("overlap", C.c_int), ("phase_flip", C.c_int),
                ("norm_type", C.c_int), ("invert", C.c_int), ("ampconst", C.c_float),
                ("a", C.c_float), ("b", C.c_float), ("b2", C.c_float),
                ("bfactor", C.c_float), ("bfactor2", C.c_float), ("bfactor3", C.c_float),
                ("precision", C.c_int)]


class GsCtf(C.Structure):
    _fields_ = [("defocus", C.c_float), ("dfdiff", C.c_float), ("dfang", C.c_float)]


class GsPick(C.Structure):
    _fields_ = [("angle_index", C.c_int), ("phi", C.c_float), ("window_x", C.c_int),
                ("window_y", C.c_int), ("template_index", C.c_int), ("center_x", C.c_float),
                ("center_y", C.c_float), ("score", C.c_float)]


class GsGeometry(C.Structure):
    _fields_ = [("l", C.c_int), ("n_windows_x", C.c_int), ("n_windows_y", C.c_int),
                ("n_angles", C.c_int), ("n_templates", C.c_int)]


class GsStats(C.Structure):
    _fields_ = [("kernel_launches", C.c_ulonglong), ("searches", C.c_ulonglong),
                ("units", C.c_ulonglong)]


REFINE_PICK_DTYPE = np.dtype([("window", "<i4"), ("template_index", "<i4"), ("pos", "<i4"),
                              ("angle", "<f4"), ("dx", "<f4"), ("dy", "<f4"), ("defocus", "<f4"),
                              ("dfdiff", "<f4"), ("dfang", "<f4")])
REFINE_RESULT_DTYPE = np.dtype([("score", "<f4"), ("d_angle", "<f4"), ("d_dx", "<f4"), ("d_dy", "<f4"),
                                ("d_defocus", "<f4"), ("d_dfdiff", "<f4"), ("d_dfang", "<f4")])
UNIT_DTYPE = np.dtype([("score", "<f4"), ("pos", "<i4"), ("peak", "<f4"), ("sigma", "<f4")])
PICK_DTYPE = np.dtype([("angle_index", "<i4"), ("phi", "<f4"), ("window_x", "<i4"),
                       ("window_y", "<i4"), ("template_index", "<i4"), ("center_x", "<f4"),
                       ("center_y", "<f4"), ("score", "<f4")])

# every entry point declared in include/gisspa.h
EXPORTS = ("gs_status_string", "gs_version", "gs_params_default", "gs_ctx_create",
           "gs_ctx_destroy", "gs_ctx_last_error", "gs_set_templates", "gs_get_geometry",
           "gs_search", "gs_search_device", "gs_get_units", "gs_get_pixel_max", "gs_picks_free",
           "gs_get_timings",
           "gs_get_stats", "gs_set_kernel_timing", "gs_set_option",
           "gs_correlate_window_noalloc", "gs_search_batch", "gs_get_tuning", "gs_score_grad",
           "gs_refine", "gs_merge_duplicates", "gs_hdf_read_image", "gs_hdf_read_dataset",
           "gs_hdf_read_attribute", "gs_host_free")

_lib_handle = None


class GisspaError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__("%s (%d): %s" % (STATUS.get(status, "?"), status, msg))
        self.status = status


def load_library(path: Optional[str] = None) -> C.CDLL:
    """Load the C-ABI library (raises if it has not been built)."""
    global _lib_handle
    if _lib_handle is not None and path is None:
        return _lib_handle
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise FileNotFoundError("CUDA library not built: %s (run gisspa_b200.build)" % p)
    lib = C.CDLL(p)
    vp = C.c_void_p
    lib.gs_status_string.restype = C.c_char_p
    lib.gs_status_string.argtypes = [C.c_int]
    lib.gs_version.restype = C.c_int
    lib.gs_params_default.argtypes = [C.POINTER(GsParams)]
    lib.gs_ctx_create.argtypes = [C.c_int, C.POINTER(vp)]
    lib.gs_ctx_destroy.argtypes = [vp]
    lib.gs_ctx_last_error.restype = C.c_char_p
    lib.gs_ctx_last_error.argtypes = [vp]
    lib.gs_set_templates.argtypes = [vp, C.POINTER(GsParams), C.POINTER(C.c_float), C.c_int,
                                     C.c_int, C.c_int, C.POINTER(GsCtf)]
    lib.gs_get_geometry.argtypes = [vp, C.c_int, C.c_int, C.POINTER(GsGeometry)]
    lib.gs_search.argtypes = [vp, C.POINTER(C.c_float), C.c_int, C.c_int, C.POINTER(GsCtf),
                              C.POINTER(C.POINTER(GsPick)), C.POINTER(C.c_size_t)]
    lib.gs_search_device.argtypes = [vp, C.c_void_p, C.c_int, C.c_int, C.POINTER(GsCtf),
                                     C.POINTER(C.POINTER(GsPick)), C.POINTER(C.c_size_t)]
    lib.gs_get_units.argtypes = [vp, C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t)]
    lib.gs_get_pixel_max.argtypes = [vp, C.c_int, C.c_float, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.gs_picks_free.argtypes = [C.POINTER(GsPick)]
    lib.gs_picks_free.restype = None
    lib.gs_get_timings.argtypes = [vp, C.POINTER(C.c_float), C.c_int]
    lib.gs_set_kernel_timing.argtypes = [vp, C.c_int]
    lib.gs_set_option.argtypes = [vp, C.c_int, C.c_int]
    lib.gs_correlate_window_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                                C.c_float, C.c_void_p, C.c_void_p]
    lib.gs_get_stats.argtypes = [vp, C.POINTER(GsStats)]
    lib.gs_search_batch.argtypes = [vp, C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_int),
                                    C.POINTER(C.c_int), C.POINTER(GsCtf),
                                    C.POINTER(C.POINTER(GsPick)), C.POINTER(C.c_size_t),
                                    C.POINTER(C.c_size_t)]
    lib.gs_get_tuning.argtypes = [vp, C.POINTER(C.c_int), C.c_int]
    lib.gs_score_grad.argtypes = [vp, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    lib.gs_refine.argtypes = [vp, C.c_void_p, C.c_int, C.c_int, C.c_void_p]
    lib.gs_merge_duplicates.argtypes = [C.c_int, C.c_void_p, C.c_size_t, C.c_double, C.c_double,
                                        C.c_void_p]
    lib.gs_hdf_read_image.argtypes = [C.c_char_p, C.c_int, C.POINTER(C.POINTER(C.c_float)),
                                      C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                      C.c_char_p, C.c_size_t]
    lib.gs_hdf_read_dataset.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(C.POINTER(C.c_double)),
                                        C.POINTER(C.c_int64), C.POINTER(C.c_int), C.c_char_p, C.c_size_t]
    lib.gs_hdf_read_attribute.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.POINTER(C.c_double),
                                          C.c_size_t, C.POINTER(C.c_size_t), C.c_char_p, C.c_size_t,
                                          C.c_char_p, C.c_size_t]
    lib.gs_host_free.argtypes = [C.c_void_p]
    lib.gs_host_free.restype = None
    if path is None:
        _lib_handle = lib
    return lib


_HDF5_SIGNATURE = b"\x89HDF\r\n\x1a\n"


def is_hdf5(path: str) -> bool:
    """The file starts with the HDF5 signature (EMhdf::is_valid,
    EMReader/emhdf_.cpp:47-62)."""
    try:
        with open(path, "rb") as fh:
            return fh.read(8) == _HDF5_SIGNATURE
    except OSError:
        return False


def read_hdf_image(path: str, index: int = 0) -> np.ndarray:
    """Image ``index`` of an EMAN HDF5 file (old EMAN or EMAN2 layout) as
    float32, shape (ny, nx) or (nz, ny, nx), through gs_hdf_read_image."""
    lib = load_library()
    data = C.POINTER(C.c_float)()
    nx, ny, nz = C.c_int(), C.c_int(), C.c_int()
    err = C.create_string_buffer(512)
    st = lib.gs_hdf_read_image(path.encode(), int(index), C.byref(data), C.byref(nx), C.byref(ny),
                               C.byref(nz), err, len(err))
    if st != GS_OK:
        raise GisspaError(st, err.value.decode(errors="replace"))
    try:
        n = nx.value * ny.value * nz.value
        a = np.ctypeslib.as_array(data, (n,)).copy()
    finally:
        lib.gs_host_free(data)
    shape = (ny.value, nx.value) if nz.value == 1 else (nz.value, ny.value, nx.value)
    return a.reshape(shape)


def read_hdf_dataset(path: str, name: str) -> np.ndarray:
    """Any numeric dataset of an HDF5 file as float64 (gs_hdf_read_dataset)."""
    lib = load_library()
    data = C.POINTER(C.c_double)()
    dims = (C.c_int64 * 8)()
    rank = C.c_int()
    err = C.create_string_buffer(512)
    st = lib.gs_hdf_read_dataset(path.encode(), name.encode(), C.byref(data), dims, C.byref(rank), err,
                                 len(err))
    if st != GS_OK:
        raise GisspaError(st, err.value.decode(errors="replace"))
    try:
        shape = tuple(int(dims[k]) for k in range(rank.value))
        n = int(np.prod(shape)) if shape else 1
        a = np.ctypeslib.as_array(data, (n,)).copy() if n else np.zeros(0)
    finally:
        lib.gs_host_free(data)
    return a.reshape(shape)


def read_hdf_attribute(path: str, obj: str, name: str):
    """Attribute ``name`` of HDF5 object ``obj``: a float64 array, or a str for
    a fixed-length string (gs_hdf_read_attribute)."""
    lib = load_library()
    vals = (C.c_double * 64)()
    nv = C.c_size_t()
    text = C.create_string_buffer(1024)
    err = C.create_string_buffer(512)
    st = lib.gs_hdf_read_attribute(path.encode(), obj.encode(), name.encode(), vals, 64, C.byref(nv), text,
                                   len(text), err, len(err))
    if st != GS_OK:
        raise GisspaError(st, err.value.decode(errors="replace"))
    if nv.value == 0 and text.value:
        return text.value.decode(errors="replace")
    return np.array([vals[k] for k in range(min(nv.value, 64))])


def read_image(path: str, section: int = -1) -> np.ndarray:
    """emdata::readImage (EMReader/emdata_.cpp:174-205): image ``section`` of
    an EMAN HDF5 file, else section ``section`` of an MRC file (the whole
    stack for an out-of-range section)."""
    from . import formats
    if is_hdf5(path):
        return read_hdf_image(path, section)
    return formats.read_mrc(path, section)


def default_params(**kw) -> GsParams:
    """Reference defaults (DataReader.h:16-42) updated with ``kw``."""
    lib = load_library()
    p = GsParams()
    lib.gs_params_default(C.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


def params_from_config(cfg) -> GsParams:
    """GsParams from a :class:`gisspa_b200.formats.Config`."""
    return default_params(apix=cfg.apix, phi_step=cfg.phi_step, kk=cfg.kk, energy=cfg.energy,
                          cs=cfg.cs, highres=cfg.highres, lowres=cfg.lowres, d_m=cfg.d_m,
                          thres=cfg.thres, window_size=cfg.padding_size, overlap=cfg.overlap,
                          phase_flip=cfg.phase_flip, norm_type=cfg.norm_type, invert=cfg.invert)


def _ctf(c) -> GsCtf:
    if isinstance(c, GsCtf):
        return c
    d, dd, da = c
    return GsCtf(float(d), float(dd), float(da))


class Context:
    """One CUDA device + stream + the device buffers of a run (gs_ctx)."""

    def __init__(self, device: int = 0):
        self._lib = load_library()
        self._h = C.c_void_p()
        st = self._lib.gs_ctx_create(int(device), C.byref(self._h))
        if st != GS_OK:
            raise GisspaError(st, "gs_ctx_create(device=%d)" % device)

    def _check(self, st: int, what: str) -> None:
        if st != GS_OK:
            msg = self._lib.gs_ctx_last_error(self._h).decode(errors="replace")
            raise GisspaError(st, "%s: %s" % (what, msg))

    def close(self) -> None:
        if self._h:
            self._lib.gs_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_templates(self, params: GsParams, templates: np.ndarray, first_ctf) -> None:
        t = np.ascontiguousarray(templates, dtype=np.float32)
        if t.ndim != 3:
            raise ValueError("templates must be (N, ty, tx)")
        n, ty, tx = t.shape
        self._check(self._lib.gs_set_templates(self._h, C.byref(params),
                                               t.ctypes.data_as(C.POINTER(C.c_float)), n, tx, ty,
                                               C.byref(_ctf(first_ctf))), "gs_set_templates")
        self._keep = t

    def geometry(self, nx: int, ny: int) -> GsGeometry:
        g = GsGeometry()
        self._check(self._lib.gs_get_geometry(self._h, nx, ny, C.byref(g)), "gs_get_geometry")
        return g

    def _picks(self, ptr, n) -> np.ndarray:
        out = np.zeros(n, dtype=PICK_DTYPE)
        if n:
            buf = (GsPick * n).from_address(C.addressof(ptr.contents))
            out[:] = np.frombuffer(buf, dtype=PICK_DTYPE, count=n)
            self._lib.gs_picks_free(ptr)
        return out

    def search(self, micrograph: np.ndarray, ctf) -> np.ndarray:
        m = np.ascontiguousarray(micrograph, dtype=np.float32)
        ny, nx = m.shape
        ptr = C.POINTER(GsPick)()
        n = C.c_size_t()
        self._check(self._lib.gs_search(self._h, m.ctypes.data_as(C.POINTER(C.c_float)), nx, ny,
                                        C.byref(_ctf(ctf)), C.byref(ptr), C.byref(n)), "gs_search")
        return self._picks(ptr, n.value)

    def search_batch(self, micrographs, ctfs) -> List[np.ndarray]:
        """gs_search_batch: one search over several micrographs (sizes may
        differ); returns each micrograph's picks."""
        ms = [np.ascontiguousarray(m, dtype=np.float32) for m in micrographs]
        n = len(ms)
        if n == 0 or len(ctfs) != n:
            raise ValueError("need one CTF per micrograph")
        ptrs = (C.c_void_p * n)(*[m.ctypes.data for m in ms])
        nx = (C.c_int * n)(*[m.shape[1] for m in ms])
        ny = (C.c_int * n)(*[m.shape[0] for m in ms])
        cs = (GsCtf * n)(*[_ctf(c) for c in ctfs])
        per = (C.c_size_t * n)()
        ptr = C.POINTER(GsPick)()
        tot = C.c_size_t()
        self._check(self._lib.gs_search_batch(self._h, n, ptrs, nx, ny, cs, C.byref(ptr),
                                              C.byref(tot), per), "gs_search_batch")
        allp = self._picks(ptr, tot.value)
        out, k = [], 0
        for m in range(n):
            out.append(allp[k:k + per[m]].copy())
            k += per[m]
        return out

    def score_grad(self, picks: np.ndarray, with_gradient: bool = True,
                   template_gradients: bool = False):
        """gs_score_grad: objective (and gradient) of REFINE_PICK_DTYPE picks;
        returns REFINE_RESULT_DTYPE results (and, with template_gradients,
        d score / d template base as (n, l, l) float32)."""
        pk = np.ascontiguousarray(picks, dtype=REFINE_PICK_DTYPE)
        n = pk.shape[0]
        out = np.zeros(n, dtype=REFINE_RESULT_DTYPE)
        tg = None
        if template_gradients and with_gradient and n:
            l = self._l()
            tg = np.zeros((n, l, l), dtype=np.float32)
        self._check(self._lib.gs_score_grad(self._h, pk.ctypes.data, n, 1 if with_gradient else 0,
                                            out.ctypes.data, tg.ctypes.data if tg is not None else None),
                    "gs_score_grad")
        return (out, tg) if template_gradients else out

    def refine(self, picks: np.ndarray, steps: int = 20):
        """gs_refine: gradient ascent; returns (refined picks, final results)."""
        pk = np.array(picks, dtype=REFINE_PICK_DTYPE, copy=True)
        out = np.zeros(pk.shape[0], dtype=REFINE_RESULT_DTYPE)
        self._check(self._lib.gs_refine(self._h, pk.ctypes.data, pk.shape[0], int(steps), out.ctypes.data),
                    "gs_refine")
        return pk, out

    def _l(self) -> int:
        g = self.geometry(4096, 4096)
        return int(g.l)

    def set_graph(self, enable: bool) -> None:
        """Capture the angle loop as one CUDA graph (GS_OPT_GRAPH)."""
        self._check(self._lib.gs_set_option(self._h, GS_OPT_GRAPH, 1 if enable else 0), "gs_set_option")

    def set_autotune(self, enable: bool) -> None:
        """Tune the persistent kernel's scheduling on first use (GS_OPT_AUTOTUNE)."""
        self._check(self._lib.gs_set_option(self._h, GS_OPT_AUTOTUNE, 1 if enable else 0), "gs_set_option")

    def set_corr_ctas(self, per_sm: int) -> None:
        """Resident CTAs per SM of the persistent kernel (0 = as many as fit)."""
        self._check(self._lib.gs_set_option(self._h, GS_OPT_CORR_CTAS, int(per_sm)), "gs_set_option")

    def tuning(self) -> Tuple[int, int, int, int, int]:
        """(ring slots, lag, window block, CTAs per SM, tile width) of the last search."""
        t = (C.c_int * 5)()
        self._check(self._lib.gs_get_tuning(self._h, t, 5), "gs_get_tuning")
        return tuple(t[:])

    def set_angles_per_launch(self, angles: int) -> None:
        """In-plane angles per persistent correlation launch (GS_OPT_ANGLES_PER_LAUNCH;
        0 = chosen from the unit count)."""
        self._check(self._lib.gs_set_option(self._h, GS_OPT_ANGLES_PER_LAUNCH, int(angles)), "gs_set_option")

    def angles_per_launch(self) -> int:
        """In-plane angles per persistent launch of the last search."""
        t = (C.c_int * 6)()
        self._check(self._lib.gs_get_tuning(self._h, t, 6), "gs_get_tuning")
        return int(t[5])

    def set_corr_tile(self, vectors: int) -> None:
        """Tile width of the FP32 persistent kernel (16 or 8 vectors)."""
        self._check(self._lib.gs_set_option(self._h, GS_OPT_CORR_TILE, int(vectors)), "gs_set_option")

    def search_device(self, dev_ptr: int, nx: int, ny: int, ctf) -> np.ndarray:
        ptr = C.POINTER(GsPick)()
        n = C.c_size_t()
        self._check(self._lib.gs_search_device(self._h, C.c_void_p(int(dev_ptr)), nx, ny,
                                               C.byref(_ctf(ctf)), C.byref(ptr), C.byref(n)),
                    "gs_search_device")
        return self._picks(ptr, n.value)

    def units(self, shape: Optional[Tuple[int, int, int]] = None) -> np.ndarray:
        """Dense (n_angles, n_windows, n_templates) table of the last search."""
        n = C.c_size_t()
        self._check(self._lib.gs_get_units(self._h, None, 0, C.byref(n)), "gs_get_units")
        out = np.zeros(n.value, dtype=UNIT_DTYPE)
        self._check(self._lib.gs_get_units(self._h, out.ctypes.data, n.value, C.byref(n)),
                    "gs_get_units")
        return out.reshape(shape) if shape is not None else out

    def pixel_max(self, thres: float, shape: Tuple[int, int], micrograph: int = 0):
        """Per-pixel maximum of cc / sigma over (template, angle) of micrograph
        `micrograph` (shape (ny, nx)) of the last search (gs_get_pixel_max):
        (value, template_index, angle_index) arrays; value 0 and indices -1
        where no map reaches `thres`."""
        ny, nx = shape
        value = np.zeros((ny, nx), dtype=np.float32)
        tmpl = np.zeros((ny, nx), dtype=np.int32)
        ang = np.zeros((ny, nx), dtype=np.int32)
        self._check(self._lib.gs_get_pixel_max(self._h, micrograph, thres, value.ctypes.data,
                                               tmpl.ctypes.data, ang.ctypes.data), "gs_get_pixel_max")
        return value, tmpl, ang

    def stats(self) -> GsStats:
        st = GsStats()
        self._check(self._lib.gs_get_stats(self._h, C.byref(st)), "gs_get_stats")
        return st

    def timings(self) -> np.ndarray:
        """[prep, spectra, correlation, total, row-pass ms, row-pass launches,
        column-pass ms, column-pass launches] of the last search."""
        t = (C.c_float * 8)()
        self._check(self._lib.gs_get_timings(self._h, t, 8), "gs_get_timings")
        return np.array(t[:], dtype=np.float64)

    def set_generic_fft(self, enable: bool) -> None:
        """Force the generic mixed-radix kernels (cross-check of the fast path)."""
        self._check(self._lib.gs_set_option(self._h, GS_OPT_GENERIC_FFT, 1 if enable else 0), "gs_set_option")

    def set_two_pass(self, enable: bool) -> None:
        """Run the correlation as per-window row and column launches instead of
        one persistent launch per angle (cross-check of the persistent kernel)."""
        self._check(self._lib.gs_set_option(self._h, GS_OPT_TWO_PASS, 1 if enable else 0), "gs_set_option")

    def set_window_block(self, windows: int) -> None:
        """Windows per block of the persistent kernel's unit order."""
        self._check(self._lib.gs_set_option(self._h, GS_OPT_WINDOW_BLOCK, int(windows)), "gs_set_option")

    def set_corr_ring(self, slots: int, lag: int) -> None:
        """Scratch-map ring size and column-tile lag of the persistent kernel."""
        # order matters: each call checks slots > lag against the current other value
        if slots > self._lag_now():
            self._check(self._lib.gs_set_option(self._h, GS_OPT_CORR_SLOTS, int(slots)), "gs_set_option")
            self._check(self._lib.gs_set_option(self._h, GS_OPT_CORR_LAG, int(lag)), "gs_set_option")
        else:
            self._check(self._lib.gs_set_option(self._h, GS_OPT_CORR_LAG, int(lag)), "gs_set_option")
            self._check(self._lib.gs_set_option(self._h, GS_OPT_CORR_SLOTS, int(slots)), "gs_set_option")
        self._lag = int(lag)

    def _lag_now(self) -> int:
        return getattr(self, "_lag", 6)

    def set_kernel_timing(self, enable: bool) -> None:
        self._check(self._lib.gs_set_kernel_timing(self._h, 1 if enable else 0),
                    "gs_set_kernel_timing")


MERGE_ITEM_DTYPE = np.dtype([("x", "<f8"), ("y", "<f8"), ("alt", "<f8"), ("az", "<f8"),
                             ("phi", "<f8"), ("score", "<f8"), ("group", "<i8")])
MERGE_CLI_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "gisspa_merge")


def merge_duplicates(items: np.ndarray, center: float, euler_thres: float, device: int = 0) -> np.ndarray:
    """gs_merge_duplicates on MERGE_ITEM_DTYPE picks; returns the keep mask."""
    it = np.ascontiguousarray(items, dtype=MERGE_ITEM_DTYPE)
    keep = np.zeros(it.shape[0], dtype=np.uint8)
    st = load_library().gs_merge_duplicates(int(device), it.ctypes.data, it.shape[0], float(center),
                                            float(euler_thres), keep.ctypes.data)
    if st != GS_OK:
        raise GisspaError(st, "gs_merge_duplicates")
    return keep.astype(bool)


def merge_lines(lines, center: float, euler_thres: float, device: int = 0):
    """Duplicate merging of pick lines (the reference's
    remove_repeat_particles_from_list.py): the kept lines, in order."""
    from . import formats
    items = np.zeros(len(lines), dtype=MERGE_ITEM_DTYPE)
    group, prev = -1, None
    for k, line in enumerate(lines):
        d = formats.parse_pick_line(line)
        if d["path"] != prev:
            group += 1
            prev = d["path"]
        items[k] = (d["center"][0], d["center"][1], d["euler"][0], d["euler"][1], d["euler"][2],
                    d["score"], group)
    keep = merge_duplicates(items, center, euler_thres, device)
    return [l for l, k in zip(lines, keep) if k]


NOALLOC_SCRATCH_BYTES = 32 << 20
NOALLOC_MAX_WINDOW = 2012


def correlate_window_noalloc(d_window_spectrum: int, d_pair_spectra: int, n_templates: int,
                             l: int, d_m: float, d_units: int, stream: int = 0) -> None:
    """gs_correlate_window_noalloc on raw device pointers (no device
    allocation; work queued on ``stream``, the call does not wait)."""
    lib = load_library()
    st = lib.gs_correlate_window_noalloc(C.c_void_p(d_window_spectrum), C.c_void_p(d_pair_spectra),
                                         int(n_templates), int(l), float(d_m),
                                         C.c_void_p(d_units), C.c_void_p(stream or None))
    if st != GS_OK:
        raise GisspaError(st, "gs_correlate_window_noalloc(l=%d, n_templates=%d)" % (l, n_templates))


def run_config(config_path: str, device: Optional[int] = None, return_units: bool = False,
               precision: int = 0):
    """Python mirror of the drop-in driver (main.cu:1025-1269 behaviour) over
    the C ABI: returns the output lines (and optionally the dense per-unit
    tables, one per micrograph).  Paths resolve relative to the current
    directory, as in the reference.  ``precision`` selects the arithmetic of
    the correlation's DFT stage (GS_PREC_*, no config-file counterpart)."""
    from . import formats
    cfg = formats.read_config(config_path)
    missing = formats.missing_required(cfg)
    if missing:
        raise ValueError("missing required keys: %s" % ", ".join(missing))
    eul = formats.read_euler(cfg.eulerf)
    n = eul.shape[0]
    if is_hdf5(cfg.temp2d):
        # one image per template (readAndPaddingTemplate, main.cu:186-190)
        stack = np.stack([read_hdf_image(cfg.temp2d, J) for J in range(n)])
    else:
        whole = formats.read_mrc(cfg.temp2d, -1)
        if whole.ndim == 2:
            whole = whole[None]
        stack = np.stack([whole[J] if J < whole.shape[0] else whole[0] for J in range(n)])
    first = formats.read_lst_entry(cfg.inlst, cfg.first)
    if first is None:
        raise IOError("entry %d of %s not found" % (cfg.first, cfg.inlst))
    params = params_from_config(cfg)
    params.precision = precision
    lines = []
    tables = []
    with Context(cfg.device_id if device is None else device) as ctx:
        ctx.set_templates(params, stack, (first.defocus, first.dfdiff, first.dfang))
        for m in range(cfg.first, cfg.last):
            ent = formats.read_lst_entry(cfg.inlst, m)
            if ent is None:
                raise IOError("entry %d of %s not found" % (m, cfg.inlst))
            img = read_image(ent.path, ent.nn)
            if img.ndim == 3:
                img = img[0]
            picks = ctx.search(img, (ent.defocus, ent.dfdiff, ent.dfang))
            for pk in picks:
                J = int(pk["template_index"])
                lines.append(formats.format_pick_line(
                    ent.nn, ent.path, ent.defocus, ent.dfdiff, ent.dfang, float(eul[J, 0]),
                    float(eul[J, 1]), float(pk["phi"]), float(pk["center_x"]),
                    float(pk["center_y"]), float(pk["score"])))
            if return_units:
                g = ctx.geometry(img.shape[1], img.shape[0])
                tables.append(ctx.units((g.n_angles, g.n_windows_x * g.n_windows_y, g.n_templates)))
    return (lines, tables) if return_units else lines
