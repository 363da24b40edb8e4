"""Python binding of libpppm_b200 (the C ABI in include/pppm_b200.h) through ctypes.

`Solver` mirrors the reference's PPPMSolver (src/algorithm/pppm.h:11-165): construct with the
grid, `set_mesh`, `update_mesh` on motion frames, `update_grid_and_face(acc)` per step
(`step(acc_rows)` for many), listener cells read per step like the demo driver
(experiments/demo/main.cu:266).  Errors raise PPPMError; the CUDA library is required - a
missing library raises at its first use (ImportError), there is no CPU fallback.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_PKG = os.path.dirname(os.path.dirname(_HERE))
LIB_PATH = os.environ.get("PPPM_B200_LIB", os.path.join(_PKG, "lib", "libpppm_b200.so"))

OK, ERR_ARG, ERR_CUDA, ERR_CAPACITY, ERR_NAN, ERR_STATE, ERR_TIMEOUT, ERR_NOMEM = range(8)
PRECISION = {"fp32": 0, "fp64": 1}
WEIGHTS = {"ref32": 0, "fp64": 1}

DUMP = dict(grid_t=0, grid_tm1=1, grid_tm2=2, neumann=3, dirichlet=4, tri_geom=5, tri_cells=6, cell_counts=7,
            n3_cells=8, n3_tris=9, b4_cells=10, b4_tris=11, n4_tris=12, grid_cache=13, face_pairs=14,
            face_cache=15, interp=16, cell_type=17, cell_nearest=18, cell_ghost=19, cell_points=20, counts=21,
            ghost_cells=22, ghost_order=23, ghost_weights=24, ghost_iters=25)

# dtype of each dump (None: follows the handle precision; "rec": 72-byte weight records)
_DUMP_DTYPE = dict(grid_t=None, grid_tm1=None, grid_tm2=None, neumann=None, dirichlet=None, tri_geom=np.float32,
                   tri_cells=np.int32, cell_counts=np.int32, n3_cells=np.int32, n3_tris=np.int32,
                   b4_cells=np.int32, b4_tris=np.int32, n4_tris=np.int32, grid_cache="rec", face_pairs=np.int32,
                   face_cache="rec", interp=np.float32, cell_type=np.int32, cell_nearest=np.int32,
                   cell_ghost=np.int32, cell_points=np.float32, counts=np.int32, ghost_cells=np.int32,
                   ghost_order=np.int32, ghost_weights=np.float32, ghost_iters=np.int32)

# the reference's LayerWeightHalf record (bem.h:163-169)
RECORD = np.dtype([("s", "<f2", 16), ("ms", "<f4"), ("d", "<f2", 16), ("md", "<f4")])
assert RECORD.itemsize == 72


class PPPMError(RuntimeError):
    def __init__(self, status, where, message):
        super().__init__("%s: %s (%s)" % (where, message, status))
        self.status = status


class _Params(ctypes.Structure):
    _fields_ = [("res", ctypes.c_int), ("dl", ctypes.c_float), ("dt", ctypes.c_float),
                ("min_pos", ctypes.c_float * 3), ("pml_width", ctypes.c_int), ("reflect_coeff", ctypes.c_float),
                ("c", ctypes.c_float), ("rho", ctypes.c_float), ("precision", ctypes.c_int),
                ("weights", ctypes.c_int), ("device", ctypes.c_int), ("stream", ctypes.c_void_p),
                ("method", ctypes.c_int), ("ghost_threshold", ctypes.c_float)]


METHOD = dict(pppm=0, ghost=1)


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError("libpppm_b200.so not built (%s); run pppm-tdbem_b200/build.py" % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    vp, ip, fp, i, sz = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float), ctypes.c_int, ctypes.c_size_t
    sig = {
        "pppm_params_default": [ctypes.POINTER(_Params)],
        "pppm_create": [ctypes.POINTER(_Params), ctypes.POINTER(vp)],
        "pppm_destroy": [vp],
        "pppm_set_mesh": [vp, vp, i, vp, i],
        "pppm_update_mesh": [vp, vp, i],
        "pppm_step": [vp, vp, i, i],
        "pppm_add_listener": [vp, i, i, i],
        "pppm_clear_listeners": [vp],
        "pppm_listener_count": [vp, ip, ip],
        "pppm_read_listeners": [vp, i, i, fp],
        "pppm_rewind_listeners": [vp],
        "pppm_get_time": [vp, ip],
        "pppm_set_time": [vp, i],
        "pppm_reset_fields": [vp],
        "pppm_state_size": [vp, ctypes.POINTER(sz)],
        "pppm_save_state": [vp, vp, sz],
        "pppm_restore_state": [vp, vp, sz],
        "pppm_dump_size": [vp, i, ctypes.POINTER(sz)],
        "pppm_dump": [vp, i, vp, sz],
        "pppm_load": [vp, i, vp, sz],
        "pppm_import_grid_cache": [vp, vp, sz],
        "pppm_import_face_cache": [vp, vp, vp, i],
        "pppm_classify_cells": [vp, ip],
        "pppm_fill_fresh_cells": [vp, vp, vp, ip],
        "pppm_batch_create": [ctypes.POINTER(vp), i, ctypes.POINTER(vp)],
        "pppm_batch_destroy": [vp],
        "pppm_batch_run": [vp, ctypes.POINTER(vp), ip, i],
        "pppm_adjoint": [vp, vp, i, i, i, vp],
        "pppm_read_listeners_raw": [vp, i, i, vp, i],
        "pppm_get_stream": [vp, ctypes.POINTER(vp)],
        "pppm_launch_count": [vp, ctypes.POINTER(ctypes.c_longlong)],
        "pppm_enable_timing": [vp, i],
        "pppm_set_option": [vp, i, i],
        "pppm_get_option": [vp, i, ip],
        "pppm_autotune": [vp, i, fp, ip],
        "pppm_kernel_times": [vp, fp, fp, fp, ip],
        "pppm_kernel_profile": [vp, i, fp, ctypes.POINTER(ctypes.c_longlong)],
        "pppm_sync": [vp],
        "pppm_time_kernels": [vp, i, i, fp],
        "pppm_cache_state_size": [vp, ctypes.POINTER(sz)],
        "pppm_save_cache_state": [vp, vp, sz],
        "pppm_restore_cache_state": [vp, vp, sz],
        "pppm_checkpoint_push": [vp, ctypes.POINTER(i)],
        "pppm_checkpoint_rewind": [vp, i],
        "pppm_checkpoint_clear": [vp, i],
        "pppm_checkpoint_info": [vp, ctypes.POINTER(i), ctypes.POINTER(sz)],
    }
    fl = ctypes.c_float
    sig["pppm_tdbem_constants"] = [fl, fl, fl, fp, fp]
    sig["pppm_pair_weights"] = [i, fl, fl, fl, vp, i, vp, i, vp, vp, vp]
    sig["pppm_pair_weights_static"] = [i, vp, fl, fl, fl, vp, i, vp, i, vp, vp, vp]
    for name, args in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = ctypes.c_int
    lib.pppm_status_string.argtypes = [ctypes.c_int]
    lib.pppm_status_string.restype = ctypes.c_char_p
    lib.pppm_last_error_message.argtypes = []
    lib.pppm_last_error_message.restype = ctypes.c_char_p
    return lib


class _Lib:
    """libpppm_b200.so, mapped into the process at the first call through it.  Importing the
    package (for `scenes`, say) maps no native code; the first Solver, Batch or entry-point call
    loads the library and raises ImportError when it is not built."""

    _cdll = None

    def __getattr__(self, name):
        return getattr(load(), name)


def load():
    """Map libpppm_b200.so now (idempotent) and return the ctypes handle."""
    if _Lib._cdll is None:
        _Lib._cdll = _load()
    return _Lib._cdll


def loaded():
    """True once the native library is mapped into this process."""
    return _Lib._cdll is not None


lib = _Lib()


def check(status, where):
    if status != OK:
        msg = lib.pppm_last_error_message().decode() or lib.pppm_status_string(status).decode()
        raise PPPMError(status, where, msg)


def _ptr(a):
    """Host numpy array -> (pointer, on_device=0); torch CUDA tensor -> (data_ptr, 1)."""
    if hasattr(a, "data_ptr") and hasattr(a, "is_cuda"):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return ctypes.c_void_p(a.data_ptr()), 1 if a.is_cuda else 0
    return a.ctypes.data_as(ctypes.c_void_p), 0


def tdbem_constants(dt, dl, c=340.3):
    """lambda and the 16 wave numbers (complex) the library derives from dt and h (host only)."""
    lam = ctypes.c_float()
    w = np.zeros(32, np.float32)
    check(lib.pppm_tdbem_constants(float(dt), float(dl), float(c), ctypes.byref(lam),
                                   w.ctypes.data_as(ctypes.POINTER(ctypes.c_float))), "tdbem_constants")
    return lam.value, w.reshape(16, 2)


def pair_weights(dt, dl, verts, src, point=None, face=None, c=340.3, device=0):
    """16 + 16 TDBEM taps of one pair computed on the device with the caches' FP32 arithmetic."""
    v = np.ascontiguousarray(verts, np.float32).reshape(-1, 3)
    s = np.ascontiguousarray(src, np.int32)
    out = np.zeros(32, np.float32)
    if point is not None:
        pt = np.ascontiguousarray(point, np.float32)
        rc = lib.pppm_pair_weights(device, float(dt), float(dl), float(c), v.ctypes.data_as(ctypes.c_void_p), len(v),
                                   s.ctypes.data_as(ctypes.c_void_p), 1, None, pt.ctypes.data_as(ctypes.c_void_p),
                                   out.ctypes.data_as(ctypes.c_void_p))
    else:
        fc = np.ascontiguousarray(face, np.int32)
        rc = lib.pppm_pair_weights(device, float(dt), float(dl), float(c), v.ctypes.data_as(ctypes.c_void_p), len(v),
                                   s.ctypes.data_as(ctypes.c_void_p), 0, fc.ctypes.data_as(ctypes.c_void_p), None,
                                   out.ctypes.data_as(ctypes.c_void_p))
    check(rc, "pair_weights")
    return out


def pair_weights_static(dt, dl, verts, src, point=None, face=None, c=340.3, device=0, stream=None):
    """pair_weights without any device allocation: the library stages the vertex rows in its own
    static device array (at most STATIC_MAX_VERTS rows).  stream: a raw cudaStream_t as an int
    (None: the default stream)."""
    v = np.ascontiguousarray(verts, np.float32).reshape(-1, 3)
    s = np.ascontiguousarray(src, np.int32)
    out = np.zeros(32, np.float32)
    st = ctypes.c_void_p(stream) if stream else None
    if point is not None:
        pt = np.ascontiguousarray(point, np.float32)
        rc = lib.pppm_pair_weights_static(device, st, float(dt), float(dl), float(c),
                                          v.ctypes.data_as(ctypes.c_void_p), len(v), s.ctypes.data_as(ctypes.c_void_p),
                                          1, None, pt.ctypes.data_as(ctypes.c_void_p),
                                          out.ctypes.data_as(ctypes.c_void_p))
    else:
        fc = np.ascontiguousarray(face, np.int32)
        rc = lib.pppm_pair_weights_static(device, st, float(dt), float(dl), float(c),
                                          v.ctypes.data_as(ctypes.c_void_p), len(v), s.ctypes.data_as(ctypes.c_void_p),
                                          0, fc.ctypes.data_as(ctypes.c_void_p), None,
                                          out.ctypes.data_as(ctypes.c_void_p))
    check(rc, "pair_weights_static")
    return out


STATIC_MAX_VERTS = 65536  # PPPM_STATIC_MAX_VERTS


class Solver:
    """One scene: FDTD grid + TDBEM near-field correction (reference PPPMSolver)."""

    def __init__(self, res, dl, dt, min_pos=(0.0, 0.0, 0.0), pml_width=0, reflect_coeff=0.83, c=340.3,
                 rho=1.225, precision="fp32", weights="ref32", device=0, stream=None, method="pppm",
                 ghost_threshold=25.0):
        """method "pppm": FDTD + TDBEM near-field correction (PPPMSolver); "ghost": FDTD + ghost
        cells (GhostCellSolver) with the given condition-number threshold (0: first order)."""
        p = _Params()
        check(lib.pppm_params_default(ctypes.byref(p)), "params_default")
        p.res, p.dl, p.dt = int(res), float(dl), float(dt)
        for k in range(3):
            p.min_pos[k] = float(min_pos[k])
        p.pml_width, p.reflect_coeff, p.c, p.rho = int(pml_width), float(reflect_coeff), float(c), float(rho)
        p.precision, p.weights, p.device = PRECISION[precision], WEIGHTS[weights], int(device)
        p.stream = stream
        p.method, p.ghost_threshold = METHOD[method], float(ghost_threshold)
        self.h = ctypes.c_void_p()
        check(lib.pppm_create(ctypes.byref(p), ctypes.byref(self.h)), "pppm_create")
        self.res, self.dl, self.dt = int(res), float(dl), float(dt)
        self.precision = precision
        self.device = int(device)
        self.real = np.float64 if precision == "fp64" else np.float32
        self.nt = 0
        self.nv = 0

    # -- lifecycle
    def close(self):
        if self.h:
            lib.pppm_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- mesh
    def set_mesh(self, verts, tris):
        v = np.ascontiguousarray(verts, dtype=np.float32).reshape(-1, 3)
        f = np.ascontiguousarray(tris, dtype=np.int32).reshape(-1, 3)
        check(lib.pppm_set_mesh(self.h, v.ctypes.data_as(ctypes.c_void_p), len(v), f.ctypes.data_as(ctypes.c_void_p),
                                len(f)), "set_mesh")
        self.nv, self.nt = len(v), len(f)

    def update_mesh(self, verts):
        if hasattr(verts, "data_ptr"):
            ptr, dev = _ptr(verts)
            check(lib.pppm_update_mesh(self.h, ptr, dev), "update_mesh")
            return
        v = np.ascontiguousarray(verts, dtype=np.float32).reshape(-1, 3)
        if len(v) != self.nv:
            raise ValueError("vertex count changed")
        check(lib.pppm_update_mesh(self.h, v.ctypes.data_as(ctypes.c_void_p), 0), "update_mesh")

    # -- stepping
    def step(self, acc=None, nsteps=None):
        """acc: (nsteps, nt) host array or CUDA tensor; None only before set_mesh."""
        if acc is None:
            check(lib.pppm_step(self.h, None, 0, int(nsteps or 1)), "step")
            return
        if hasattr(acc, "data_ptr"):
            n = acc.shape[0] if acc.dim() == 2 else 1
            ptr, dev = _ptr(acc)
            check(lib.pppm_step(self.h, ptr, dev, n), "step")
            return
        a = np.ascontiguousarray(acc, dtype=np.float32)
        if a.ndim == 1:
            a = a.reshape(1, -1)
        check(lib.pppm_step(self.h, a.ctypes.data_as(ctypes.c_void_p), 0, a.shape[0]), "step")

    def sync(self):
        """Wait for the queued work (pppm_sync); raises PPPMError(ERR_NAN) once a non-finite
        Dirichlet value or listener sample has appeared."""
        check(lib.pppm_sync(self.h), "sync")

    def update_grid_and_face(self, acc):
        self.step(np.asarray(acc, dtype=np.float32).reshape(1, -1))

    update_step = update_grid_and_face

    # -- listeners
    def add_listener(self, x, y, z):
        check(lib.pppm_add_listener(self.h, int(x), int(y), int(z)), "add_listener")

    def listeners(self, first=0, count=None):
        n, nl = ctypes.c_int(), ctypes.c_int()
        check(lib.pppm_listener_count(self.h, ctypes.byref(n), ctypes.byref(nl)), "listener_count")
        if count is None:
            count = n.value - first
        out = np.zeros((count, nl.value), np.float32)
        if count and nl.value:
            check(lib.pppm_read_listeners(self.h, first, count, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))),
                  "read_listeners")
        return out

    @property
    def stream(self):
        """cudaStream_t (int) the solver queues its work on."""
        v = ctypes.c_void_p()
        check(lib.pppm_get_stream(self.h, ctypes.byref(v)), "get_stream")
        return v.value or 0

    @property
    def series_count(self):
        n, nl = ctypes.c_int(), ctypes.c_int()
        check(lib.pppm_listener_count(self.h, ctypes.byref(n), ctypes.byref(nl)), "listener_count")
        return n.value

    @property
    def n_listeners(self):
        n, nl = ctypes.c_int(), ctypes.c_int()
        check(lib.pppm_listener_count(self.h, ctypes.byref(n), ctypes.byref(nl)), "listener_count")
        return nl.value

    def series(self, first=0, count=None, out=None):
        """Listener samples [first, first + count) in the handle's precision: a host array, or
        written into `out` (a contiguous CUDA tensor of that dtype, queued on the solver's
        stream)."""
        if count is None:
            count = self.series_count - first
        nl = self.n_listeners
        if out is not None:
            if not out.is_contiguous() or out.numel() != count * nl or out.element_size() != np.dtype(self.real).itemsize:
                raise ValueError("out must be a contiguous (%d, %d) tensor of the handle's precision" % (count, nl))
            check(lib.pppm_read_listeners_raw(self.h, first, count, ctypes.c_void_p(out.data_ptr()), 1 if out.is_cuda else 0),
                  "read_listeners_raw")
            return out
        a = np.zeros((count, nl), self.real)
        if count and nl:
            check(lib.pppm_read_listeners_raw(self.h, first, count, a.ctypes.data_as(ctypes.c_void_p), 0),
                  "read_listeners_raw")
        return a

    def adjoint(self, dL_dsignal, fresh=True, out=None):
        """dL/dacc (nsteps, nt) for L = sum dL_dsignal * listener samples over the last nsteps
        steps differentiated (pppm_adjoint).  fresh=False continues the previous call's reverse
        sweep with the steps just before it.  Host arrays in, host array out; CUDA tensors in,
        CUDA tensor out (queued on the solver's stream)."""
        nl = self.n_listeners
        if hasattr(dL_dsignal, "data_ptr") and getattr(dL_dsignal, "is_cuda", False):
            import torch

            g = dL_dsignal.contiguous()
            if g.element_size() != np.dtype(self.real).itemsize:
                raise ValueError("gradient dtype must match the handle's precision")
            n = g.shape[0]
            if out is None:
                out = torch.empty((n, self.nt), dtype=g.dtype, device=g.device)
            check(lib.pppm_adjoint(self.h, ctypes.c_void_p(g.data_ptr()), n, 1, 1 if fresh else 0,
                                   ctypes.c_void_p(out.data_ptr())), "adjoint")
            return out
        g = np.ascontiguousarray(dL_dsignal, dtype=self.real).reshape(-1, nl)
        n = g.shape[0]
        res = np.zeros((n, self.nt), self.real)
        check(lib.pppm_adjoint(self.h, g.ctypes.data_as(ctypes.c_void_p), n, 0, 1 if fresh else 0,
                               res.ctypes.data_as(ctypes.c_void_p)), "adjoint")
        return res

    def rewind_listeners(self):
        check(lib.pppm_rewind_listeners(self.h), "rewind_listeners")

    # -- time and state
    @property
    def t(self):
        v = ctypes.c_int()
        check(lib.pppm_get_time(self.h, ctypes.byref(v)), "get_time")
        return v.value

    @t.setter
    def t(self, value):
        check(lib.pppm_set_time(self.h, int(value)), "set_time")

    def reset_fields(self):
        check(lib.pppm_reset_fields(self.h), "reset_fields")

    def save_state(self):
        n = ctypes.c_size_t()
        check(lib.pppm_state_size(self.h, ctypes.byref(n)), "state_size")
        buf = np.empty(n.value, np.uint8)
        check(lib.pppm_save_state(self.h, buf.ctypes.data_as(ctypes.c_void_p), n.value), "save_state")
        return buf

    def restore_state(self, buf):
        buf = np.ascontiguousarray(buf, dtype=np.uint8)
        check(lib.pppm_restore_state(self.h, buf.ctypes.data_as(ctypes.c_void_p), buf.size), "restore_state")

    def save_cache_state(self, on_device=False):
        """The motion-frame state of the weight caches (pppm_save_cache_state): a host uint8
        array, or with on_device=True a uint8 CUDA tensor on the handle's device (HBM-resident
        checkpoint)."""
        n = ctypes.c_size_t()
        check(lib.pppm_cache_state_size(self.h, ctypes.byref(n)), "cache_state_size")
        if on_device:
            import torch

            dev = torch.device("cuda", self.device)
            buf = torch.empty(n.value, dtype=torch.uint8, device=dev)
            torch.cuda.current_stream(dev).synchronize()  # the block may still be in use there
            ptr = ctypes.c_void_p(buf.data_ptr())
        else:
            buf = np.empty(n.value, np.uint8)
            ptr = buf.ctypes.data_as(ctypes.c_void_p)
        check(lib.pppm_save_cache_state(self.h, ptr, n.value), "save_cache_state")
        return buf

    def restore_cache_state(self, buf):
        """Restore a saved cache state (pppm_restore_cache_state), host array or CUDA tensor;
        update_mesh must follow."""
        if hasattr(buf, "data_ptr"):
            b = buf.contiguous()
            ptr, size = ctypes.c_void_p(b.data_ptr()), b.numel() * b.element_size()
        else:
            b = np.ascontiguousarray(buf, dtype=np.uint8)
            ptr, size = b.ctypes.data_as(ctypes.c_void_p), b.size
        check(lib.pppm_restore_cache_state(self.h, ptr, size), "restore_cache_state")

    def checkpoint_push(self):
        """A motion checkpoint of the current frame's caches, kept in device memory by the
        handle (pppm_checkpoint_push); returns its index."""
        i = ctypes.c_int()
        check(lib.pppm_checkpoint_push(self.h, ctypes.byref(i)), "checkpoint_push")
        return i.value

    def checkpoint_rewind(self, index):
        """Caches back to checkpoint `index`, later checkpoints dropped (pppm_checkpoint_rewind);
        update_mesh with that frame's vertices must follow."""
        check(lib.pppm_checkpoint_rewind(self.h, int(index)), "checkpoint_rewind")

    def checkpoint_clear(self, release=False):
        """Drop every checkpoint (pppm_checkpoint_clear); release=True frees their device memory
        too, else it is kept for the next checkpoints."""
        check(lib.pppm_checkpoint_clear(self.h, 1 if release else 0), "checkpoint_clear")

    def checkpoint_info(self):
        """(checkpoints held, device bytes their arena and logs use)"""
        n, b = ctypes.c_int(), ctypes.c_size_t()
        check(lib.pppm_checkpoint_info(self.h, ctypes.byref(n), ctypes.byref(b)), "checkpoint_info")
        return n.value, b.value

    # -- read-out
    def dump(self, what):
        code = DUMP[what]
        n = ctypes.c_size_t()
        check(lib.pppm_dump_size(self.h, code, ctypes.byref(n)), "dump_size(%s)" % what)
        raw = np.empty(n.value, np.uint8)
        if n.value:
            check(lib.pppm_dump(self.h, code, raw.ctypes.data_as(ctypes.c_void_p), n.value), "dump(%s)" % what)
        dt = _DUMP_DTYPE[what]
        if dt is None:
            dt = self.real
        if dt == "rec":
            if self.precision == "fp64":
                return raw.view(np.float64).reshape(-1, 16, 2)
            return raw.view(RECORD)
        return raw.view(dt)

    def grid(self, rel=0):
        return self.dump({0: "grid_t", -1: "grid_tm1", -2: "grid_tm2"}[rel]).reshape(self.res, self.res, self.res)

    def load(self, what, arr):
        a = np.ascontiguousarray(arr, dtype=self.real)
        check(lib.pppm_load(self.h, DUMP[what], a.ctypes.data_as(ctypes.c_void_p), a.nbytes), "load(%s)" % what)

    def import_grid_cache(self, records):
        r = np.ascontiguousarray(records)
        check(lib.pppm_import_grid_cache(self.h, r.ctypes.data_as(ctypes.c_void_p), r.nbytes), "import_grid_cache")

    def import_face_cache(self, pairs, records):
        p = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1, 2)
        r = np.ascontiguousarray(records)
        check(lib.pppm_import_face_cache(self.h, p.ctypes.data_as(ctypes.c_void_p), r.ctypes.data_as(ctypes.c_void_p),
                                         len(p)), "import_face_cache")

    def classify_cells(self):
        g = ctypes.c_int()
        check(lib.pppm_classify_cells(self.h, ctypes.byref(g)), "classify_cells")
        return g.value

    def fill_fresh_cells(self, acc, acc_old):
        a = np.ascontiguousarray(acc, dtype=np.float32)
        b = np.ascontiguousarray(acc_old, dtype=np.float32)
        n = ctypes.c_int()
        check(lib.pppm_fill_fresh_cells(self.h, a.ctypes.data_as(ctypes.c_void_p), b.ctypes.data_as(ctypes.c_void_p),
                                        ctypes.byref(n)), "fill_fresh_cells")
        return n.value

    def launch_count(self):
        v = ctypes.c_longlong()
        check(lib.pppm_launch_count(self.h, ctypes.byref(v)), "launch_count")
        return v.value

    OPTIONS = {"conv_pairs": 0, "face_threads": 1, "terms_pairs": 2, "split_stencil": 3, "graph_chunk": 4,
               "stencil_vec4": 5}
    TUNE_CANDIDATES = [(pairs, threads) for pairs in (0, 1) for threads in (64, 128, 256)]
    TUNE_CONFIGS = [(pairs, threads, terms) for pairs in (0, 1) for threads in (64, 128, 256) for terms in (0, 1)]

    def set_option(self, name, value):
        """Launch option of the recorded step graphs (pppm_set_option): conv_pairs (0: one pass
        per step, 1: two steps per pass), face_threads (64/128/256), terms_pairs (0/1),
        split_stencil (0/1), graph_chunk (steps per chunk graph of a long call; 0: one graph),
        stencil_vec4 (1: four interior cells per thread, 0: one, -1: by grid size)."""
        check(lib.pppm_set_option(self.h, self.OPTIONS[name], int(value)), "set_option")

    def get_option(self, name):
        v = ctypes.c_int()
        check(lib.pppm_get_option(self.h, self.OPTIONS[name], ctypes.byref(v)), "get_option")
        return v.value

    def autotune(self, reps=20):
        """Time the face-stage candidates on the current mesh (pppm_autotune) and keep the
        fastest.  Returns {"us": {(pairs, threads): us per two steps}, "launch_us":
        {(pairs, threads): (first kernel, second kernel) us per launch}, "best": (pairs, threads)}."""
        n = len(self.TUNE_CANDIDATES)
        us = (ctypes.c_float * (2 * (n + 2) + len(self.TUNE_CONFIGS)))()
        best = ctypes.c_int()
        check(lib.pppm_autotune(self.h, int(reps), us, ctypes.byref(best)), "autotune")
        per = [(float(us[2 * i]), float(us[2 * i + 1])) for i in range(n + 2)]
        step_us = [float(us[2 * (n + 2) + j]) for j in range(len(self.TUNE_CONFIGS))]
        chosen = (self.get_option("conv_pairs"), self.get_option("face_threads"))
        return {"us": {c: a + b for c, (a, b) in zip(self.TUNE_CANDIDATES, per)},
                "launch_us": dict(zip(self.TUNE_CANDIDATES, per)), "best": chosen,
                "finish_us": {"single": sum(per[n]), "pairs": sum(per[n + 1])},
                "finish_launch_us": {"single": per[n], "pairs": per[n + 1]},
                "step_us": dict(zip(self.TUNE_CONFIGS, step_us)) if any(step_us) else None,
                "terms_pairs": self.get_option("terms_pairs"), "stencil_vec4": self.get_option("stencil_vec4")}

    def enable_timing(self, on=True):
        check(lib.pppm_enable_timing(self.h, 1 if on else 0), "enable_timing")

    KERNEL_KINDS = ("stencil", "conv", "conv2", "fix", "finish", "finish1", "finish2", "near", "nwrite", "face",
                    "empty", "stencil_bulk", "stencil_corr")

    def kernel_profile(self):
        """{kind: (mean us per launch, launches)} of the kernels timed in measurement mode
        (pppm_kernel_profile), kinds with no launch left out."""
        n = len(self.KERNEL_KINDS)
        us = (ctypes.c_float * n)()
        cnt = (ctypes.c_longlong * n)()
        check(lib.pppm_kernel_profile(self.h, n, us, cnt), "kernel_profile")
        return {k: (float(us[i]), int(cnt[i])) for i, k in enumerate(self.KERNEL_KINDS) if cnt[i]}

    def time_kernels(self, reps=20):
        """{kind: us per launch} of every step kernel kind on the current mesh and state
        (pppm_time_kernels: reps back-to-back launches in one recorded graph); stepping continues
        unchanged afterwards."""
        n = len(self.KERNEL_KINDS)
        us = (ctypes.c_float * n)()
        check(lib.pppm_time_kernels(self.h, int(reps), n, us), "time_kernels")
        return {k: float(us[i]) for i, k in enumerate(self.KERNEL_KINDS) if us[i] > 0}

    def kernel_times(self):
        a, b, c, n = ctypes.c_float(), ctypes.c_float(), ctypes.c_float(), ctypes.c_int()
        check(lib.pppm_kernel_times(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ctypes.byref(n)),
              "kernel_times")
        return a.value, b.value, c.value, n.value


class Batch:
    """Scenes advanced together: one set of stage launches per step covers every scene
    (pppm_batch_*).  Each scene keeps its own state, listeners and series; results equal
    those of stepping each Solver alone."""

    def __init__(self, solvers):
        self.solvers = list(solvers)
        arr = (ctypes.c_void_p * len(self.solvers))(*[s.h for s in self.solvers])
        self.h = ctypes.c_void_p()
        check(lib.pppm_batch_create(arr, len(self.solvers), ctypes.byref(self.h)), "batch_create")

    def run(self, accs):
        """accs[i]: (nsteps_i, nt_i) float32 host arrays or CUDA tensors (all of one kind)."""
        n = len(self.solvers)
        if len(accs) != n:
            raise ValueError("one acceleration block per scene")
        def on_device(a):
            return bool(getattr(a, "is_cuda", False))

        on_dev = on_device(accs[0])
        keep = []
        ptrs = (ctypes.c_void_p * n)()
        steps = (ctypes.c_int * n)()
        for i, a in enumerate(accs):
            if on_device(a) != on_dev:
                raise ValueError("acceleration blocks must all be on the device or all on the host")
            if hasattr(a, "data_ptr"):  # torch tensor (CUDA, or host memory such as pinned buffers)
                if not a.is_contiguous() or a.dtype.itemsize != 4:
                    raise ValueError("tensor must be contiguous float32")
                if a.dim() == 2 and a.shape[0] and a.shape[1] != self.solvers[i].nt:
                    raise ValueError("scene %d: acceleration rows need %d values" % (i, self.solvers[i].nt))
                ptrs[i] = a.data_ptr()
                steps[i] = a.shape[0]
            else:
                a = np.ascontiguousarray(a, dtype=np.float32)
                if a.ndim != 2 or (a.shape[0] and a.shape[1] != self.solvers[i].nt):
                    raise ValueError("scene %d: accelerations must be (nsteps, %d)" % (i, self.solvers[i].nt))
                keep.append(a)
                ptrs[i] = a.ctypes.data
                steps[i] = a.shape[0]
        check(lib.pppm_batch_run(self.h, ptrs, steps, 1 if on_dev else 0), "batch_run")

    def close(self):
        if self.h:
            lib.pppm_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
