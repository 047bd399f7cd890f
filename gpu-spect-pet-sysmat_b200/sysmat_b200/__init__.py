"""sysmat_b200: ctypes binding of libsysmat_b200.so (B200 / sm_100a).

The C ABI is declared in ``include/sysmat_b200.h``.  This module mirrors it:

* :func:`PESysMatGen` -- the reference's entry point
  (``PEGen_RayTracing_CircularHole/PESysMatGen.h:4-9``): host tables, host
  ``dst`` of one z-slab, returns the number of voxels per row.
* :class:`Context`, :class:`Geometry` and :meth:`Geometry.pe` -- the
  status-returning API with explicit sub-sampling, row ranges, slabs, host or
  device outputs and caller streams.

There is no fallback: if the shared library is missing or no sm_100 device is
present, calls raise :class:`SysmatError`.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence, Tuple

import numpy as np

from . import params as params  # noqa: F401  (re-export)
from . import configs as configs  # noqa: F401

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libsysmat_b200.so")

SM_OK = 0
ERRORS = {-1: "SM_ERR_INVALID", -2: "SM_ERR_CAPACITY", -3: "SM_ERR_CUDA", -4: "SM_ERR_ALLOC",
          -5: "SM_ERR_IO", -6: "SM_ERR_TIMEOUT", -7: "SM_ERR_DEVICE"}


class SysmatError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__("%s (%d): %s" % (ERRORS.get(code, "SM_ERR"), code, message))
        self.code = code


class PeOptions(ctypes.Structure):
    _fields_ = [("sv", ctypes.c_int * 3), ("sc", ctypes.c_int * 3), ("tile_voxels", ctypes.c_int * 3),
                ("flags", ctypes.c_int), ("group", ctypes.c_int)]

    @staticmethod
    def make(sv=(1, 1, 1), sc=(8, 16, 8), tile_voxels=(0, 0, 0), autotune: bool = False, group: int = 0) -> "PeOptions":
        o = PeOptions()
        for i in range(3):
            o.sv[i], o.sc[i], o.tile_voxels[i] = int(sv[i]), int(sc[i]), int(tile_voxels[i])
        o.flags = 1 if autotune else 0
        o.group = int(group)
        return o


class ScatterOptions(ctypes.Structure):
    _fields_ = [("sp", ctypes.c_int * 3), ("parts", ctypes.c_int), ("flags", ctypes.c_int)]

    @staticmethod
    def make(sp=(1, 1, 1), parts: int = 3) -> "ScatterOptions":
        o = ScatterOptions()
        for i in range(3):
            o.sp[i] = int(sp[i])
        o.parts = int(parts)
        o.flags = 0
        return o


SCATTER_PARTS = {"crystal": 1, "collimator": 2, "both": 3}


class SurrogateOptions(ctypes.Structure):
    """sm_surrogate_options (include/sysmat_b200.h)."""
    _fields_ = [("sp", ctypes.c_int * 3), ("parts", ctypes.c_int), ("train_frac", ctypes.c_float),
                ("holdout_frac", ctypes.c_float), ("val_frac", ctypes.c_float), ("tol", ctypes.c_float),
                ("anchors", ctypes.c_int * 3), ("network", ctypes.c_int), ("layers", ctypes.c_int),
                ("width", ctypes.c_int), ("freqs", ctypes.c_int), ("emb", ctypes.c_int), ("steps", ctypes.c_int),
                ("batch", ctypes.c_int), ("lr", ctypes.c_float), ("seed", ctypes.c_uint64)]

    @staticmethod
    def make(**kw) -> "SurrogateOptions":
        o = SurrogateOptions()
        lib().sm_surrogate_options_default(ctypes.byref(o))
        for k, v in kw.items():
            if k in ("sp", "anchors"):
                for i in range(3):
                    getattr(o, k)[i] = int(v[i])
            elif k == "parts":
                o.parts = SCATTER_PARTS[v] if isinstance(v, str) else int(v)
            else:
                setattr(o, k, v)
        return o


class SurrogateStats(ctypes.Structure):
    """sm_surrogate_stats (include/sysmat_b200.h)."""
    _fields_ = [(n, ctypes.c_double) for n in ("ms_total", "ms_pairs", "ms_exact_subsets", "ms_baseline", "ms_transfer",
                                               "ms_train", "ms_correct", "ms_verify", "ms_recompute",
                                               "ms_collimator")] + \
               [(n, ctypes.c_int) for n in ("n_train_columns", "n_holdout_columns", "n_val_columns", "rows_corrected",
                                            "rows_recomputed")] + \
               [(n, ctypes.c_double) for n in ("holdout_median", "holdout_p90", "holdout_max",
                                               "baseline_holdout_median", "first_loss", "final_loss",
                                               "val_gain")]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}

_lib = None
_f32p = ctypes.POINTER(ctypes.c_float)
_i64p = ctypes.POINTER(ctypes.c_int64)
_i32p = ctypes.POINTER(ctypes.c_int32)
_vp = ctypes.c_void_p

# Prototypes of every exported function: (restype, argtypes).
PROTOTYPES = {
    "PESysMatGen": (ctypes.c_int, [_f32p, _f32p, _f32p, _f32p, ctypes.c_int]),
    "scatter": (ctypes.c_int, [_f32p, _f32p, _f32p, _f32p, _f32p, ctypes.c_char_p, ctypes.c_char_p, _f32p,
                               ctypes.c_int]),
    "sm_last_error": (ctypes.c_char_p, []),
    "sm_version": (ctypes.c_char_p, []),
    "sm_context_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_vp)]),
    "sm_context_destroy": (ctypes.c_int, [_vp]),
    "sm_context_sync": (ctypes.c_int, [_vp, _vp]),
    "sm_context_trim": (ctypes.c_int, [_vp]),
    "sm_geometry_create": (ctypes.c_int, [_vp, _f32p, ctypes.c_size_t, _f32p, ctypes.c_size_t, _f32p,
                                          ctypes.c_size_t, _f32p, ctypes.c_size_t, ctypes.POINTER(_vp)]),
    "sm_geometry_destroy": (ctypes.c_int, [_vp]),
    "sm_tables_check": (ctypes.c_int, [_f32p, ctypes.c_size_t, _f32p, ctypes.c_size_t, _f32p, ctypes.c_size_t,
                                       _f32p, ctypes.c_size_t, _i64p]),
    "sm_geometry_info": (ctypes.c_int, [_vp, _i64p]),
    "sm_pe_options_reference": (None, [ctypes.POINTER(PeOptions)]),
    "sm_pe_compute": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(PeOptions), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int64, ctypes.c_int, _vp]),
    "sm_pe_compute_static": (ctypes.c_int, [_f32p, ctypes.c_size_t, _f32p, ctypes.c_size_t, _f32p, ctypes.c_size_t,
                                            ctypes.POINTER(PeOptions), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int64, _vp]),
    "sm_pe_record_hits": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(PeOptions), ctypes.c_int, _i64p, _i64p,
                                         ctypes.c_int64, _i32p, ctypes.POINTER(ctypes.c_int)]),
    "sm_pe_set_counters": (ctypes.c_int, [_vp, ctypes.c_int]),
    "sm_pe_last_counters": (ctypes.c_int, [_vp, _i64p]),
    "sm_primitive_batch": (ctypes.c_int, [ctypes.c_int, _f32p, ctypes.c_int64, _f32p]),
    "sm_beam_metrics": (ctypes.c_int, [_vp, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_float, _vp, _vp,
                                       _vp, _vp, ctypes.c_int64, _vp, _vp]),
    "sm_pe_autotune": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(PeOptions), ctypes.c_int, ctypes.POINTER(PeOptions),
                                      ctypes.POINTER(ctypes.c_double)]),
    "sm_pe_batch_create": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(_vp), ctypes.POINTER(PeOptions),
                                          ctypes.POINTER(ctypes.c_int), ctypes.POINTER(_vp), _i64p, ctypes.POINTER(_vp)]),
    "sm_pe_batch_info": (ctypes.c_int, [_vp, _i64p]),
    "sm_pe_batch_run": (ctypes.c_int, [_vp, _vp]),
    "sm_pe_batch_destroy": (ctypes.c_int, [_vp]),
    "sm_gemm_bf16": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_int64, ctypes.c_int64, _vp,
                                    ctypes.c_int64, ctypes.c_int64, _vp, ctypes.c_int64, ctypes.c_float, _vp, _vp,
                                    ctypes.c_int, ctypes.c_int, _vp, _vp]),
    "sm_scatter_options_reference": (None, [ctypes.POINTER(ScatterOptions)]),
    "sm_scatter_bitmap_words": (ctypes.c_int, [_vp, _i64p]),
    "sm_scatter_bitmap_hashes": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_uint64)]),
    "sm_scatter_bitmaps": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_int, _vp]),
    "sm_scatter_compute": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(ScatterOptions), ctypes.c_int, _vp,
                                          ctypes.c_int64, ctypes.c_int, _vp, _vp, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, _vp, ctypes.c_int64, ctypes.c_int, _vp]),
    "sm_scatter_subset": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(ScatterOptions), ctypes.c_int, _vp, ctypes.c_int64,
                                         _i32p, ctypes.c_int, _i32p, ctypes.c_int, _vp, ctypes.c_int64, _vp]),
    "sm_scatter_transfer": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(ScatterOptions), ctypes.c_int, _vp, ctypes.c_int,
                                           _vp, ctypes.c_int64, _vp]),
    "sm_tc_wait_limit": (ctypes.c_int, [ctypes.c_int64, _i64p]),
    "sm_surrogate_options_default": (None, [ctypes.POINTER(SurrogateOptions)]),
    "sm_scatter_surrogate": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(SurrogateOptions), ctypes.c_int, _vp,
                                            ctypes.c_int64, _vp, ctypes.c_int64, _f32p, _i32p,
                                            ctypes.POINTER(SurrogateStats), _vp]),
    "sm_surrogate_columns": (ctypes.c_int, [_vp, ctypes.POINTER(SurrogateOptions), _i32p, ctypes.POINTER(ctypes.c_int),
                                            ctypes.POINTER(ctypes.c_int)]),
    "sm_surrogate_net_create": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                               ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                               ctypes.c_uint64, ctypes.POINTER(_vp)]),
    "sm_surrogate_net_layout": (ctypes.c_int, [_vp, _i64p, _i64p]),
    "sm_surrogate_net_get": (ctypes.c_int, [_vp, _f32p]),
    "sm_surrogate_net_set": (ctypes.c_int, [_vp, _f32p]),
    "sm_surrogate_net_loss_grad": (ctypes.c_int, [_vp, _i32p, _i32p, ctypes.c_int, _f32p, _f32p, ctypes.c_int64,
                                                  ctypes.POINTER(ctypes.c_double), _f32p]),
    "sm_surrogate_net_adam": (ctypes.c_int, [_vp, ctypes.c_float]),
    "sm_surrogate_net_predict": (ctypes.c_int, [_vp, _i32p, ctypes.c_int, _f32p]),
    "sm_surrogate_net_apply": (ctypes.c_int, [_vp, _i32p, ctypes.c_int, _f32p, _f32p]),
    "sm_surrogate_net_destroy": (ctypes.c_int, [_vp]),
    "sm_scatter_legacy": (ctypes.c_int, [ctypes.c_int, _f32p, _f32p, _f32p, _f32p, _f32p, ctypes.c_char_p,
                                         ctypes.c_char_p, _f32p, ctypes.c_int]),
}


def lib():
    """Load libsysmat_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise SysmatError(-7, "%s is missing: build it with `make -C gpu-spect-pet-sysmat_b200/csrc`" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(rc: int):
    if rc != SM_OK:
        raise SysmatError(rc, (lib().sm_last_error() or b"").decode(errors="replace"))


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(_f32p)


def _as_f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


# --------------------------------------------------------------------------
# Reference interface
# --------------------------------------------------------------------------

def PESysMatGen(parameter_Collimator, parameter_Detector, parameter_Image, dst: np.ndarray, cuda_id: int = 0) -> int:
    """Drop-in for the reference's ``int PESysMatGen(float*, float*, float*, float*, int)``.

    ``parameter_Image`` carries the slab side channel ([2] slab nz, [30] full
    nz, [31] z0, [20] rotation index) exactly as the reference's CLI sets it.
    ``dst`` (float32, C-contiguous) receives [N][nx*ny*Image[2]].  Tables must
    hold at least 80000 / 80000 / 100 floats.
    """
    col, det, img = _as_f32(parameter_Collimator), _as_f32(parameter_Detector), _as_f32(parameter_Image)
    if col.size < 80000 or det.size < 80000 or img.size < 100:
        raise SysmatError(-1, "PESysMatGen reads 80000 / 80000 / 100 floats")
    if not (dst.dtype == np.float32 and dst.flags.c_contiguous):
        raise SysmatError(-1, "dst must be a C-contiguous float32 array")
    return lib().PESysMatGen(_fptr(col), _fptr(det), _fptr(img), _fptr(dst), int(cuda_id))


# --------------------------------------------------------------------------
# Status-returning API
# --------------------------------------------------------------------------

def tables_check(collimator, detector, image, physics=None) -> dict:
    """``sm_tables_check``: the library's table validation without a device.
    Table lengths are the arrays' sizes; raises SysmatError naming the field
    at fault.  Returns crystals, holes, plates, grid and rotations."""
    col, det, img = _as_f32(collimator), _as_f32(detector), _as_f32(image)
    phy = _as_f32(physics) if physics is not None else np.zeros(0, np.float32)
    out = np.zeros(7, np.int64)
    _check(lib().sm_tables_check(_fptr(col), col.size, _fptr(det), det.size, _fptr(img), img.size,
                                 _fptr(phy) if phy.size else None, phy.size, out.ctypes.data_as(_i64p)))
    return {"crystals": int(out[0]), "holes": int(out[1]), "plates": int(out[2]),
            "grid": (int(out[3]), int(out[4]), int(out[5])), "rotations": int(out[6])}


class Context:
    def __init__(self, device: int = 0):
        h = _vp()
        _check(lib().sm_context_create(int(device), ctypes.byref(h)))
        self.handle = h
        self.device = device

    def close(self):
        if self.handle:
            lib().sm_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sync(self, stream: int = 0):
        _check(lib().sm_context_sync(self.handle, _vp(stream)))

    def trim(self):
        """Return the context's cached device workspaces to the device."""
        _check(lib().sm_context_trim(self.handle))

    def set_counters(self, enable: bool):
        _check(lib().sm_pe_set_counters(self.handle, 1 if enable else 0))

    def last_counters(self) -> Tuple[int, int, int, int]:
        out = np.zeros(4, dtype=np.int64)
        _check(lib().sm_pe_last_counters(self.handle, out.ctypes.data_as(_i64p)))
        return tuple(int(x) for x in out)


class Geometry:
    """Parsed, validated, device-resident geometry built from the four tables."""

    def __init__(self, ctx: Context, p):
        self.ctx = ctx
        self.params = p
        self._tables = [_as_f32(p.collimator), _as_f32(p.detector), _as_f32(p.image), _as_f32(p.physics)]
        col, det, img, phy = self._tables
        h = _vp()
        _check(lib().sm_geometry_create(ctx.handle, _fptr(col), col.size, _fptr(det), det.size, _fptr(img), img.size,
                                        _fptr(phy), phy.size, ctypes.byref(h)))
        self.handle = h
        info = np.zeros(7, dtype=np.int64)
        _check(lib().sm_geometry_info(h, info.ctypes.data_as(_i64p)))
        self.n_crystals, self.n_holes, self.n_plates, self.nx, self.ny, self.nz, self.n_rotations = map(int, info)

    def close(self):
        if self.handle:
            lib().sm_geometry_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def options(self, sv=None, sc=None, tile_voxels=(0, 0, 0)) -> PeOptions:
        sv = self.params.sv if sv is None else sv
        sc = self.params.sc if sc is None else sc
        return PeOptions.make(sv, sc, tile_voxels)

    def pe(self, rotation: int = 0, rows: Optional[Tuple[int, int]] = None, z: Optional[Tuple[int, int]] = None,
           opts: Optional[PeOptions] = None, out=None, ld: Optional[int] = None, stream: int = 0) -> np.ndarray:
        """Photoelectric sysmat block [rows][slab voxels].

        ``out`` may be None (a host array is returned), a host float32 array,
        or an integer device pointer (the call is then asynchronous on
        ``stream`` and returns None).
        """
        r0, r1 = rows if rows is not None else (0, self.n_crystals)
        z0, nz = z if z is not None else (0, self.nz)
        opts = opts if opts is not None else self.options()
        slab = self.nx * self.ny * nz
        ld = slab if ld is None else ld
        if out is None or isinstance(out, np.ndarray):
            host = np.zeros((r1 - r0, ld), dtype=np.float32) if out is None else out
            if host.dtype != np.float32 or not host.flags.c_contiguous or host.size < (r1 - r0) * ld:
                raise SysmatError(-1, "out must be C-contiguous float32 with rows*ld elements")
            _check(lib().sm_pe_compute(self.ctx.handle, self.handle, ctypes.byref(opts), int(rotation), int(r0),
                                       int(r1), int(z0), int(nz), _vp(host.ctypes.data), int(ld), 0, _vp(stream)))
            return host
        _check(lib().sm_pe_compute(self.ctx.handle, self.handle, ctypes.byref(opts), int(rotation), int(r0), int(r1),
                                   int(z0), int(nz), _vp(int(out)), int(ld), 1, _vp(stream)))
        return None

    # ---- primary-Compton scatter -------------------------------------------

    def bitmap_words(self) -> Tuple[int, int]:
        out = np.zeros(2, dtype=np.int64)
        _check(lib().sm_scatter_bitmap_words(self.handle, out.ctypes.data_as(_i64p)))
        return int(out[0]), int(out[1])

    def bitmap_hashes(self) -> Tuple[int, int]:
        """Geometry hashes of the crystal and collimator bitmaps (the .geohash values)."""
        out = (ctypes.c_uint64 * 2)()
        _check(lib().sm_scatter_bitmap_hashes(self.handle, out))
        return int(out[0]), int(out[1])

    def scatter_bitmaps(self) -> Tuple[np.ndarray, np.ndarray]:
        """The crystal and collimator bitmaps (uint32 words, the reference's file format)."""
        wc, wh = self.bitmap_words()
        c = np.zeros(max(wc, 1), dtype=np.uint32)
        h = np.zeros(max(wh, 1), dtype=np.uint32)
        _check(lib().sm_scatter_bitmaps(self.ctx.handle, self.handle, _vp(c.ctypes.data),
                                        _vp(h.ctypes.data) if wh > 0 else None, 0, None))
        return c[:wc], h[:wh]

    def scatter(self, pe=None, rotation: int = 0, sp=(1, 1, 1), parts="both", rows: Optional[Tuple[int, int]] = None,
                bitmaps: Optional[Tuple[np.ndarray, np.ndarray]] = None, out=None, ld: Optional[int] = None,
                pe_ld: Optional[int] = None, stream: int = 0) -> Optional[np.ndarray]:
        """Primary-Compton scatter sysmat block [rows][voxels].

        ``pe``: the rotation's PE sysmat, a host float32 array [N][V] or an
        integer device pointer (then ``pe_ld`` gives its row pitch).  ``out``:
        None (a host array is returned), a host array, or an integer device
        pointer (asynchronous on ``stream`` when ``pe`` is on the device).
        ``bitmaps``: optional host word arrays (crystal, collimator) as read
        from the reference's files; computed on the device when omitted.
        """
        opt = ScatterOptions.make(sp, SCATTER_PARTS[parts] if isinstance(parts, str) else parts)
        r0, r1 = rows if rows is not None else (0, self.n_crystals)
        V = self.nx * self.ny * self.nz
        ld = V if ld is None else ld
        pe_ptr, pe_dev, pe_ld_v = None, 0, V
        if pe is not None:
            if isinstance(pe, np.ndarray):
                pe_arr = np.ascontiguousarray(pe, dtype=np.float32)
                if pe_arr.size < self.n_crystals * V:
                    raise SysmatError(-1, "pe must hold N x V floats")
                pe_ptr, pe_ld_v = _vp(pe_arr.ctypes.data), pe_arr.size // self.n_crystals
            else:
                pe_ptr, pe_dev, pe_ld_v = _vp(int(pe)), 1, (V if pe_ld is None else int(pe_ld))
        bm_c = bm_h = None
        if bitmaps is not None:
            bc = np.ascontiguousarray(bitmaps[0], dtype=np.uint32)
            bh = np.ascontiguousarray(bitmaps[1], dtype=np.uint32)
            bm_c, bm_h = _vp(bc.ctypes.data), (_vp(bh.ctypes.data) if bh.size else None)
        if out is None or isinstance(out, np.ndarray):
            host = np.zeros((r1 - r0, ld), dtype=np.float32) if out is None else out
            if host.dtype != np.float32 or not host.flags.c_contiguous or host.size < (r1 - r0) * ld:
                raise SysmatError(-1, "out must be C-contiguous float32 with rows*ld elements")
            _check(lib().sm_scatter_compute(self.ctx.handle, self.handle, ctypes.byref(opt), int(rotation), pe_ptr,
                                            int(pe_ld_v), pe_dev, bm_c, bm_h, 0, int(r0), int(r1),
                                            _vp(host.ctypes.data), int(ld), 0, _vp(stream)))
            return host
        _check(lib().sm_scatter_compute(self.ctx.handle, self.handle, ctypes.byref(opt), int(rotation), pe_ptr,
                                        int(pe_ld_v), pe_dev, bm_c, bm_h, 0, int(r0), int(r1), _vp(int(out)),
                                        int(ld), 1, _vp(stream)))
        return None

    def scatter_subset(self, pe_ptr: int, rows: Sequence[int], out_ptr: int, cols=None, ld: Optional[int] = None,
                       rotation: int = 0, sp=(1, 1, 1), parts="crystal", pe_ld: Optional[int] = None,
                       stream: int = 0):
        """Exact scatter of the listed rows (distinct) into device ``out_ptr``:
        every voxel (``cols`` None, row i at out[i * ld + v]) or the voxel
        y-columns (x, z) = cols[c] (out[i * ld + c * ny + y]).  Device pointers;
        queued on ``stream``."""
        opt = ScatterOptions.make(sp, SCATTER_PARTS[parts] if isinstance(parts, str) else parts)
        V = self.nx * self.ny * self.nz
        r = np.ascontiguousarray(rows, dtype=np.int32)
        c = None if cols is None else np.ascontiguousarray(cols, dtype=np.int32).reshape(-1, 2)
        width = V if c is None else c.shape[0] * self.ny
        ld = width if ld is None else int(ld)
        _check(lib().sm_scatter_subset(self.ctx.handle, self.handle, ctypes.byref(opt), int(rotation),
                                       _vp(int(pe_ptr)) if pe_ptr else None, int(V if pe_ld is None else pe_ld),
                                       r.ctypes.data_as(_i32p), int(r.size),
                                       None if c is None else c.ctypes.data_as(_i32p), 0 if c is None else int(c.shape[0]),
                                       _vp(int(out_ptr)), ld, _vp(stream)))

    def scatter_transfer(self, vbar_ptr: int, k_ptr: int, n_anchors: int = 1, ldk: Optional[int] = None,
                         rotation: int = 0, sp=(1, 1, 1), stream: int = 0):
        """Crystal-scatter transfer matrices K[a][d][s] into device ``k_ptr`` for
        the device float32 [n_anchors][N][4] arrival points ``vbar_ptr``
        (fractional voxel indices, w > 0 in use); queued on ``stream``."""
        opt = ScatterOptions.make(sp, 1)
        _check(lib().sm_scatter_transfer(self.ctx.handle, self.handle, ctypes.byref(opt), int(rotation),
                                         _vp(int(vbar_ptr)), int(n_anchors), _vp(int(k_ptr)),
                                         int(self.n_crystals if ldk is None else ldk), _vp(stream)))

    def scatter_surrogate(self, pe_ptr: int, out_ptr: int, options: Optional["SurrogateOptions"] = None,
                          rotation: int = 0, ld: Optional[int] = None, pe_ld: Optional[int] = None,
                          stream: int = 0, **kw) -> dict:
        """Crystal (+ collimator) scatter sysmat [N][V] into device ``out_ptr``
        through the surrogate (physics baseline, learned correction, exact
        re-check and recompute); ``pe_ptr`` the rotation's device PE sysmat.
        Returns the run's statistics plus ``row_error`` (held-out error per
        row) and ``row_state`` (0 baseline, 1 corrected, 2 recomputed)."""
        o = options if options is not None else SurrogateOptions.make(**kw)
        V = self.nx * self.ny * self.nz
        st = SurrogateStats()
        err = np.zeros(self.n_crystals, dtype=np.float32)
        state = np.zeros(self.n_crystals, dtype=np.int32)
        _check(lib().sm_scatter_surrogate(self.ctx.handle, self.handle, ctypes.byref(o), int(rotation),
                                          _vp(int(pe_ptr)), int(V if pe_ld is None else pe_ld), _vp(int(out_ptr)),
                                          int(V if ld is None else ld), _fptr(err), state.ctypes.data_as(_i32p),
                                          ctypes.byref(st), _vp(stream)))
        out = st.as_dict()
        out["row_error"] = err
        out["row_state"] = state
        return out

    def surrogate_columns(self, options: Optional["SurrogateOptions"] = None, **kw):
        """(train, holdout): the (x, z) voxel columns a surrogate run computes exactly."""
        o = options if options is not None else SurrogateOptions.make(**kw)
        nt, nh = ctypes.c_int(0), ctypes.c_int(0)
        _check(lib().sm_surrogate_columns(self.handle, ctypes.byref(o), None, ctypes.byref(nt), ctypes.byref(nh)))
        xz = np.zeros((nt.value + nh.value, 2), dtype=np.int32)
        _check(lib().sm_surrogate_columns(self.handle, ctypes.byref(o), xz.ctypes.data_as(_i32p), ctypes.byref(nt),
                                          ctypes.byref(nh)))
        return xz[:nt.value], xz[nt.value:]

    def record_hits(self, rows: Sequence[int], voxels: Sequence[int], rotation: int = 0,
                    opts: Optional[PeOptions] = None) -> np.ndarray:
        """Per-ray hit records of entries (rows[i], voxels[i]); shape (n, rays, words)."""
        opts = opts if opts is not None else self.options()
        r = np.ascontiguousarray(rows, dtype=np.int64)
        v = np.ascontiguousarray(voxels, dtype=np.int64)
        rays = int(np.prod(opts.sv)) * int(np.prod(opts.sc))
        words = ctypes.c_int(0)
        out = np.zeros(r.size * rays * 64, dtype=np.int32)
        _check(lib().sm_pe_record_hits(self.ctx.handle, self.handle, ctypes.byref(opts), int(rotation),
                                       r.ctypes.data_as(_i64p), v.ctypes.data_as(_i64p), r.size,
                                       out.ctypes.data_as(_i32p), ctypes.byref(words)))
        w = words.value
        return out[:r.size * rays * w].reshape(r.size, rays, w)


def pe_compute_static(p, dst_ptr: int, ld: int, rotation: int = 0, rows: Optional[Tuple[int, int]] = None,
                      z: Optional[Tuple[int, int]] = None, opts: Optional[PeOptions] = None, stream: int = 0):
    """Photoelectric sysmat through ``sm_pe_compute_static``, the entry point
    that allocates no device memory (for callers that cannot call
    cudaMalloc).  ``dst_ptr`` is a device pointer to (rows) x ``ld`` float32 on
    the current device; the call returns when the block is written."""
    col, det, img = _as_f32(p.collimator), _as_f32(p.detector), _as_f32(p.image)
    nx, ny, nz_full = p.grid
    r0, r1 = rows if rows is not None else (0, p.n_crystals)
    z0, nz = z if z is not None else (0, nz_full)
    opts = opts if opts is not None else PeOptions.make(p.sv, p.sc)
    _check(lib().sm_pe_compute_static(_fptr(col), col.size, _fptr(det), det.size, _fptr(img), img.size,
                                      ctypes.byref(opts), int(rotation), int(r0), int(r1), int(z0), int(nz),
                                      _vp(int(dst_ptr)), int(ld), _vp(stream)))


def autotune(geo: "Geometry", opts: Optional[PeOptions] = None, rotation: int = 0):
    """Brick (tile_voxels) the autotuner picks for ``geo``; returns
    (options with that brick, ms per tile or -1 for a cached answer)."""
    opts = opts if opts is not None else geo.options()
    out = PeOptions()
    ms = ctypes.c_double(0)
    _check(lib().sm_pe_autotune(geo.ctx.handle, geo.handle, ctypes.byref(opts), int(rotation), ctypes.byref(out),
                                ctypes.byref(ms)))
    return out, ms.value


class PeBatch:
    """Whole PE sysmats of many geometries in one persistent launch (a CUDA
    graph after the first run).  ``outputs``: device pointers, one [N][ld]
    float32 buffer per geometry."""

    def __init__(self, ctx: Context, geometries: Sequence["Geometry"], opts: Sequence[PeOptions],
                 outputs: Sequence[int], lds: Sequence[int], rotations: Optional[Sequence[int]] = None):
        n = len(geometries)
        geos = (_vp * n)(*[g.handle for g in geometries])
        op = (PeOptions * n)(*opts)
        dst = (_vp * n)(*[_vp(int(o)) for o in outputs])
        ld = np.ascontiguousarray(lds, dtype=np.int64)
        rot = None if rotations is None else (ctypes.c_int * n)(*[int(r) for r in rotations])
        h = _vp()
        _check(lib().sm_pe_batch_create(ctx.handle, n, geos, op, rot, dst, ld.ctypes.data_as(_i64p), ctypes.byref(h)))
        self.handle, self.ctx, self._keep = h, ctx, (geos, op, dst, ld, rot, list(geometries))

    def info(self):
        out = np.zeros(3, dtype=np.int64)
        _check(lib().sm_pe_batch_info(self.handle, out.ctypes.data_as(_i64p)))
        return {"geometries": int(out[0]), "items": int(out[1]), "ctas": int(out[2])}

    def run(self, stream: int = 0):
        _check(lib().sm_pe_batch_run(self.handle, _vp(stream)))

    def close(self):
        if self.handle:
            lib().sm_pe_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gemm_bf16(m: int, n: int, k: int, a: int, a_strides, b: int, b_strides, c: int, ldc: int, alpha: float = 1.0,
              row_scale: int = 0, bias: int = 0, accumulate: bool = False, n_tile: int = 256, error: int = 0,
              stream: int = 0):
    """The surrogate's tcgen05 BF16 GEMM on device pointers (see sm_gemm_bf16)."""
    _check(lib().sm_gemm_bf16(int(m), int(n), int(k), _vp(a), int(a_strides[0]), int(a_strides[1]), _vp(b),
                              int(b_strides[0]), int(b_strides[1]), _vp(c), int(ldc), float(alpha),
                              _vp(row_scale) if row_scale else None, _vp(bias) if bias else None, 1 if accumulate else 0,
                              int(n_tile), _vp(error) if error else None, _vp(stream)))


def tc_wait_limit(polls: int) -> int:
    """sm_tc_wait_limit: sets the tensor-core GEMMs' bounded-wait limit
    (polls < 0 restores the default); returns the previous limit."""
    prev = ctypes.c_int64(0)
    _check(lib().sm_tc_wait_limit(int(polls), ctypes.byref(prev)))
    return int(prev.value)


class SurrogateNet:
    """The surrogate's coordinate MLP alone (sm_surrogate_net_*): parameters,
    loss and gradient of a batch, Adam steps and predictions, host buffers."""

    def __init__(self, ctx: "Context", n_crystals: int, grid, layers: int = 6, width: int = 256, freqs: int = 16,
                 emb: int = 64, seed: int = 1):
        self.ctx = ctx
        self.n_crystals = int(n_crystals)
        self.layers = int(layers)
        h = _vp()
        _check(lib().sm_surrogate_net_create(ctx.handle, self.n_crystals, int(grid[0]), int(grid[1]), int(grid[2]),
                                             self.layers, int(width), int(freqs), int(emb), int(seed),
                                             ctypes.byref(h)))
        self.handle = h
        n = ctypes.c_int64(0)
        offs = np.zeros(2 * self.layers + 3, dtype=np.int64)
        _check(lib().sm_surrogate_net_layout(self.handle, ctypes.byref(n), offs.ctypes.data_as(_i64p)))
        self.n_params = int(n.value)
        self.offsets = offs

    def get(self) -> np.ndarray:
        out = np.zeros(self.n_params, dtype=np.float32)
        _check(lib().sm_surrogate_net_get(self.handle, _fptr(out)))
        return out

    def set(self, params: np.ndarray):
        p = np.ascontiguousarray(params, dtype=np.float32)
        if p.size != self.n_params:
            raise SysmatError(-1, "expected %d parameters" % self.n_params)
        _check(lib().sm_surrogate_net_set(self.handle, _fptr(p)))

    def loss_grad(self, vox, col, rho: np.ndarray, wgt: np.ndarray):
        v = np.ascontiguousarray(vox, dtype=np.int32)
        c = np.ascontiguousarray(col, dtype=np.int32)
        r = np.ascontiguousarray(rho, dtype=np.float32)
        w = np.ascontiguousarray(wgt, dtype=np.float32)
        loss = ctypes.c_double(0.0)
        g = np.zeros(self.n_params, dtype=np.float32)
        _check(lib().sm_surrogate_net_loss_grad(self.handle, v.ctypes.data_as(_i32p), c.ctypes.data_as(_i32p), v.size,
                                                _fptr(r), _fptr(w), r.shape[1], ctypes.byref(loss), _fptr(g)))
        return loss.value, g

    def adam(self, lr: float):
        _check(lib().sm_surrogate_net_adam(self.handle, float(lr)))

    def predict(self, vox) -> np.ndarray:
        v = np.ascontiguousarray(vox, dtype=np.int32)
        out = np.zeros((self.n_crystals, v.size), dtype=np.float32)
        _check(lib().sm_surrogate_net_predict(self.handle, v.ctypes.data_as(_i32p), v.size, _fptr(out)))
        return out

    def apply(self, vox, values: np.ndarray, gate) -> np.ndarray:
        """values[d][j] * exp(gate[d] * rho(d, vox[j])): the surrogate's correction step."""
        v = np.ascontiguousarray(vox, dtype=np.int32)
        out = np.array(values, dtype=np.float32, order="C", copy=True)
        g = np.ascontiguousarray(gate, dtype=np.float32)
        if out.shape != (self.n_crystals, v.size) or g.size != self.n_crystals:
            raise SysmatError(-1, "values must be [N][len(vox)] and gate [N]")
        _check(lib().sm_surrogate_net_apply(self.handle, v.ctypes.data_as(_i32p), v.size, _fptr(g), _fptr(out)))
        return out

    def close(self):
        if self.handle:
            lib().sm_surrogate_net_destroy(self.handle)
            self.handle = None


def scatter_legacy(parts: str, collimator, detector, image, physics, pe: np.ndarray, geo_crystal: Optional[str],
                   geo_collimator: Optional[str], dst: np.ndarray, cuda_id: int = 0) -> int:
    """The reference's ``scatter`` host entry points (combined, crystal-only,
    collimator-only) through ``sm_scatter_legacy``; tables of at least
    80000 / 80000 / 100 / 100 floats, host ``pe`` and ``dst`` of [N][V]."""
    col = None if collimator is None else _as_f32(collimator)
    det, img, phy = _as_f32(detector), _as_f32(image), _as_f32(physics)
    pe_a = _as_f32(pe) if pe is not None else np.zeros(1, np.float32)
    if not (dst.dtype == np.float32 and dst.flags.c_contiguous):
        raise SysmatError(-1, "dst must be a C-contiguous float32 array")
    rc = lib().sm_scatter_legacy(SCATTER_PARTS[parts], None if col is None else _fptr(col), _fptr(det), _fptr(img),
                                 _fptr(phy), _fptr(pe_a), None if geo_crystal is None else geo_crystal.encode(),
                                 None if geo_collimator is None else geo_collimator.encode(), _fptr(dst), int(cuda_id))
    if rc < 0:
        raise SysmatError(rc, (lib().sm_last_error() or b"").decode(errors="replace"))
    return rc


def primitive_batch(kind: str, args: np.ndarray) -> np.ndarray:
    """Run the device ray primitives (``box``, ``inside``, ``cylinder``) on argument rows."""
    k = {"box": 0, "inside": 1, "cylinder": 2}[kind]
    a = _as_f32(args)
    n = a.shape[0]
    out = np.zeros(n, dtype=np.float32)
    _check(lib().sm_primitive_batch(k, _fptr(a), n, _fptr(out)))
    return out


def parse_records(rec: np.ndarray, n_holes_cap: int = 16):
    """Decode one entry's records (rays, words) into {ray: (plate_mask, holes, crystals)}."""
    out = {}
    for ray in range(rec.shape[0]):
        w = rec[ray]
        nh = int(w[1])
        holes = tuple(int(x) for x in w[2:2 + nh])
        nc = int(w[2 + n_holes_cap])
        crystals = tuple(int(x) for x in w[3 + n_holes_cap:3 + n_holes_cap + nc])
        out[ray] = (int(w[0]), holes, crystals)
    return out
