"""ctypes bindings of the checkers (TEST INFRASTRUCTURE - imported only by tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline / reference legs):

  Oracle     oracle/_build/liboracle.so, the plain-C restatement of the per-step hot path
             (oracle/pppm_oracle.c), FP32 reference arithmetic or FP64, OpenMP
  Reference  oracle/_ref/libpppm_ref.so, the reference solver itself compiled from its own
             sources (oracle/Makefile) with headless entry points (oracle/ref/ref_capi.cu);
             it runs on the GPU and is available only where it was built
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libpppm_ref.so")
REF_LIB_NDEBUG = os.path.join(HERE, "_ref", "libpppm_ref_ndebug.so")

RECORD = np.dtype([("s", "<f2", 16), ("ms", "<f4"), ("d", "<f2", 16), ("md", "<f4")])

_vp = ctypes.c_void_p
_i = ctypes.c_int
_f = ctypes.c_float


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _bind(lib, table):
    for name, (res, args) in table.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args


_olib = None


def oracle_lib():
    global _olib
    if _olib is None:
        if not os.path.exists(ORACLE_LIB):
            raise ImportError("oracle not built: make -C oracle oracle")
        lib = ctypes.CDLL(ORACLE_LIB)
        _bind(lib, {
            "orc_create": (_vp, [_i, _f, _f, _vp, _f, _f, _i, _i]),
            "orc_destroy": (None, [_vp]),
            "orc_set_mesh": (_i, [_vp, _vp, _i, _vp, _i]),
            "orc_set_mesh_cells": (_i, [_vp, _vp, _i, _vp, _i, _vp]),
            "orc_update_mesh": (_i, [_vp, _vp]),
            "orc_step": (_i, [_vp, _vp, _i, _vp, _i, _vp]),
            "orc_time": (_i, [_vp]),
            "orc_set_time": (_i, [_vp, _i]),
            "orc_read_grid": (_i, [_vp, _i, _vp]),
            "orc_write_grid": (_i, [_vp, _i, _vp]),
            "orc_read_history": (_i, [_vp, _vp, _vp]),
            "orc_write_history": (_i, [_vp, _vp, _vp]),
            "orc_counts": (_i, [_vp, _vp]),
            "orc_lists": (_i, [_vp, _vp, _vp, _vp, _vp, _vp]),
            "orc_face_pairs": (_i, [_vp, _vp]),
            "orc_triangles": (_i, [_vp, _vp, _vp]),
            "orc_interp": (_i, [_vp, _vp]),
            "orc_grid_weights": (_i, [_vp, _vp]),
            "orc_face_weights": (_i, [_vp, _vp]),
            "orc_grid_records": (_i, [_vp, _vp]),
            "orc_face_records": (_i, [_vp, _vp]),
            "orc_import_grid_cache": (_i, [_vp, _vp]),
            "orc_import_interp": (_i, [_vp, _vp]),
            "orc_import_face_cache": (_i, [_vp, _vp, _vp, _i]),
            "orc_laplace_weight": (_i, [_f, _f, _f, _vp, _vp, _i, _vp, _vp, _vp]),
            "orc_pair_integral": (_i, [_f, _vp, _vp, _i, _vp, _vp, ctypes.c_double, ctypes.c_double, _vp]),
            "orc_classify": (_i, [_vp, _vp, _vp, _vp, _vp, _vp]),
            "orc_fresh": (_i, [_vp, _vp, _vp, _vp]),
            "orc_threads": (_i, []),
        })
        _olib = lib
    return _olib


class Oracle:
    """CPU restatement of one scene (mirrors the product's Solver API)."""

    def __init__(self, res, dl, dt, min_pos=(0, 0, 0), reflect_coeff=0.83, c=340.3, pml_width=0, precision="fp32"):
        self.lib = oracle_lib()
        mn = np.asarray(min_pos, np.float32)
        self.prec = 1 if precision == "fp64" else 0
        self.real = np.float64 if self.prec else np.float32
        self.s = self.lib.orc_create(int(res), float(dl), float(dt), _p(mn), float(reflect_coeff), float(c),
                                     int(pml_width), self.prec)
        if not self.s:
            raise ValueError("orc_create failed")
        self.res, self.nt, self.nv = int(res), 0, 0

    def close(self):
        if self.s:
            self.lib.orc_destroy(self.s)
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ok(self, rc, what):
        if rc != 0:
            raise RuntimeError("oracle %s failed (%d)" % (what, rc))

    def set_mesh(self, verts, tris):
        v = np.ascontiguousarray(verts, np.float32).reshape(-1, 3)
        f = np.ascontiguousarray(tris, np.int32).reshape(-1, 3)
        self._ok(self.lib.orc_set_mesh(self.s, _p(v), len(v), _p(f), len(f)), "set_mesh")
        self.nv, self.nt = len(v), len(f)

    def set_mesh_cells(self, verts, tris, cells):
        """set_mesh with the triangles' grid / base cells given (n x 6)."""
        v = np.ascontiguousarray(verts, np.float32).reshape(-1, 3)
        f = np.ascontiguousarray(tris, np.int32).reshape(-1, 3)
        c = np.ascontiguousarray(cells, np.int32).reshape(-1, 6)
        self._ok(self.lib.orc_set_mesh_cells(self.s, _p(v), len(v), _p(f), len(f), _p(c)), "set_mesh_cells")
        self.nv, self.nt = len(v), len(f)

    def update_mesh(self, verts):
        v = np.ascontiguousarray(verts, np.float32).reshape(-1, 3)
        self._ok(self.lib.orc_update_mesh(self.s, _p(v)), "update_mesh")

    def step(self, acc=None, nsteps=None, listeners=()):
        if acc is None:
            n = int(nsteps or 1)
            a = np.zeros(1, np.float32)
        else:
            a = np.ascontiguousarray(acc, np.float32)
            if a.ndim == 1:
                a = a.reshape(1, -1)
            n = a.shape[0]
        lx = np.ascontiguousarray(np.asarray(listeners, np.int32).reshape(-1, 3))
        out = np.zeros((n, len(lx)), np.float32)
        self._ok(self.lib.orc_step(self.s, _p(a) if acc is not None else None, n, _p(lx), len(lx), _p(out)), "step")
        return out

    @property
    def t(self):
        return self.lib.orc_time(self.s)

    @t.setter
    def t(self, v):
        self.lib.orc_set_time(self.s, int(v))

    def grid(self, rel=0):
        out = np.zeros(self.res ** 3, self.real)
        self._ok(self.lib.orc_read_grid(self.s, rel, _p(out)), "read_grid")
        return out.reshape((self.res,) * 3)

    def write_grid(self, rel, arr):
        a = np.ascontiguousarray(arr, self.real)
        self._ok(self.lib.orc_write_grid(self.s, rel, _p(a)), "write_grid")

    def history(self):
        n = np.zeros((self.nt, 32), self.real)
        d = np.zeros((self.nt, 32), self.real)
        self._ok(self.lib.orc_read_history(self.s, _p(n), _p(d)), "read_history")
        return n, d

    def write_history(self, n, d):
        self._ok(self.lib.orc_write_history(self.s, _p(np.ascontiguousarray(n, self.real)),
                                            _p(np.ascontiguousarray(d, self.real))), "write_history")

    def counts(self):
        c = np.zeros(5, np.int32)
        self._ok(self.lib.orc_counts(self.s, _p(c)), "counts")
        return dict(n3=int(c[0]), p3=int(c[1]), b4=int(c[2]), p4=int(c[3]), pf=int(c[4]))

    def lists(self):
        c = self.counts()
        n3 = np.zeros((c["n3"], 4), np.int32)
        p3 = np.zeros(c["p3"], np.int32)
        b4 = np.zeros((c["b4"], 4), np.int32)
        p4 = np.zeros(c["p4"], np.int32)
        cc = np.zeros(self.res ** 3, np.int32)
        self._ok(self.lib.orc_lists(self.s, _p(n3), _p(p3), _p(b4), _p(p4), _p(cc)), "lists")
        return dict(n3_cells=n3, n3_tris=p3, b4_cells=b4, n4_tris=p4, cell_counts=cc)

    def face_pairs(self):
        out = np.zeros((self.counts()["pf"], 2), np.int32)
        self._ok(self.lib.orc_face_pairs(self.s, _p(out)), "face_pairs")
        return out

    def triangles(self):
        g = np.zeros((self.nt, 7), np.float32)
        c = np.zeros((self.nt, 6), np.int32)
        self._ok(self.lib.orc_triangles(self.s, _p(g), _p(c)), "triangles")
        return g, c

    def interp(self):
        out = np.zeros((self.nt, 8), np.float32)
        self._ok(self.lib.orc_interp(self.s, _p(out)), "interp")
        return out

    def grid_weights(self):
        out = np.zeros((self.nt, 54, 32), np.float64)
        self._ok(self.lib.orc_grid_weights(self.s, _p(out)), "grid_weights")
        return out

    def face_weights(self):
        out = np.zeros((self.counts()["pf"], 32), np.float64)
        self._ok(self.lib.orc_face_weights(self.s, _p(out)), "face_weights")
        return out

    def grid_records(self):
        out = np.zeros(self.nt * 54, RECORD)
        self._ok(self.lib.orc_grid_records(self.s, _p(out)), "grid_records")
        return out

    def face_records(self):
        out = np.zeros(self.counts()["pf"], RECORD)
        self._ok(self.lib.orc_face_records(self.s, _p(out)), "face_records")
        return out

    def import_grid_cache(self, records):
        r = np.ascontiguousarray(records)
        self._ok(self.lib.orc_import_grid_cache(self.s, _p(r)), "import_grid_cache")

    def import_interp(self, w):
        self._ok(self.lib.orc_import_interp(self.s, _p(np.ascontiguousarray(w, np.float32))), "import_interp")

    def import_face_cache(self, pairs, records):
        p = np.ascontiguousarray(pairs, np.int32)
        r = np.ascontiguousarray(records)
        self._ok(self.lib.orc_import_face_cache(self.s, _p(p), _p(r), len(p)), "import_face_cache")

    def classify(self):
        n = self.res ** 3
        t = np.zeros(n, np.int32)
        ne = np.zeros(n, np.int32)
        gh = np.zeros(n, np.int32)
        pts = np.zeros((n, 7), np.float32)
        g = ctypes.c_int()
        self._ok(self.lib.orc_classify(self.s, _p(t), _p(ne), _p(gh), _p(pts), ctypes.byref(g)), "classify")
        return dict(type=t, nearest=ne, ghost=gh, points=pts, ghost_count=g.value)

    def fresh(self, acc, acc_old):
        n = ctypes.c_int()
        self._ok(self.lib.orc_fresh(self.s, _p(np.ascontiguousarray(acc, np.float32)),
                                    _p(np.ascontiguousarray(acc_old, np.float32)), ctypes.byref(n)), "fresh")
        return n.value


def laplace_weight(dt, dl, verts, src, point=None, face=None, c=340.3):
    """Double-precision TDBEM weights of one pair: 16 single-layer then 16 double-layer taps."""
    lib = oracle_lib()
    v = np.ascontiguousarray(verts, np.float32)
    s = np.ascontiguousarray(src, np.int32)
    out = np.zeros(32, np.float64)
    if point is not None:
        pt = np.ascontiguousarray(point, np.float32)
        rc = lib.orc_laplace_weight(float(dt), float(dl), float(c), _p(v), _p(s), 1, None, _p(pt), _p(out))
    else:
        fc = np.ascontiguousarray(face, np.int32)
        rc = lib.orc_laplace_weight(float(dt), float(dl), float(c), _p(v), _p(s), 0, _p(fc), None, _p(out))
    if rc:
        raise RuntimeError("orc_laplace_weight failed")
    return out


def pair_integral(dl, verts, src, k, point=None, face=None):
    """Frequency-domain single / double layer integral of one pair at complex wave number k."""
    lib = oracle_lib()
    v = np.ascontiguousarray(verts, np.float32)
    s = np.ascontiguousarray(src, np.int32)
    out = np.zeros(4, np.float64)
    if point is not None:
        rc = lib.orc_pair_integral(float(dl), _p(v), _p(s), 1, None, _p(np.ascontiguousarray(point, np.float32)),
                                   float(np.real(k)), float(np.imag(k)), _p(out))
    else:
        rc = lib.orc_pair_integral(float(dl), _p(v), _p(s), 0, _p(np.ascontiguousarray(face, np.int32)), None,
                                   float(np.real(k)), float(np.imag(k)), _p(out))
    if rc:
        raise RuntimeError("orc_pair_integral failed")
    return complex(out[0], out[1]), complex(out[2], out[3])


def oracle_threads():
    return oracle_lib().orc_threads()


# ---------------------------------------------------------------- reference -----------
_rlibs = {}


def reference_available(ndebug=False):
    return os.path.exists(REF_LIB_NDEBUG if ndebug else REF_LIB)


def reference_lib(ndebug=False):
    path = REF_LIB_NDEBUG if ndebug else REF_LIB
    if path not in _rlibs:
        if not os.path.exists(path):
            raise ImportError("reference not built: make -C oracle ref")
        lib = ctypes.CDLL(path)
        _bind(lib, {
            "ref_abi_version": (_i, []),
            "ref_pppm_create": (_vp, [_i, _f, _f, _vp, _f]),
            "ref_pppm_destroy": (None, [_vp]),
            "ref_pppm_set_mesh": (_i, [_vp, _vp, _i, _vp, _i]),
            "ref_pppm_update_mesh": (_i, [_vp, _vp]),
            "ref_pppm_check_mesh": (_i, [_vp, _vp]),
            "ref_pppm_set_checks": (_i, [_vp, _i]),
            "ref_pppm_run": (_i, [_vp, _vp, _i, _vp, _i, _vp]),
            "ref_pppm_run_device": (_i, [_vp, _vp, _i, _i, _i, _i, _vp]),
            "ref_pppm_time": (_i, [_vp]),
            "ref_pppm_read_grid": (_i, [_vp, _i, _vp]),
            "ref_pppm_write_grid": (_i, [_vp, _i, _vp]),
            "ref_pppm_read_far": (_i, [_vp, _vp]),
            "ref_pppm_read_history": (_i, [_vp, _vp, _vp]),
            "ref_pppm_write_history": (_i, [_vp, _vp, _vp]),
            "ref_pppm_read_triangles": (_i, [_vp, _vp, _vp]),
            "ref_pppm_list_sizes": (_i, [_vp, _vp]),
            "ref_pppm_read_lists": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
            "ref_pppm_read_grid_cache": (_i, [_vp, _vp]),
            "ref_pppm_read_face_cache": (_i, [_vp, _vp, _vp, _i, _vp]),
            "ref_pppm_read_interp": (_i, [_vp, _vp]),
            "ref_pppm_direct_step": (_i, [_vp]),
            "ref_pppm_cached_correction_step": (_i, [_vp]),
            "ref_pppm_reset_fields": (_i, [_vp]),
            "ref_laplace_weight": (_i, [_f, _f, _vp, _i, _vp, _i, _vp, _vp, _vp]),
            "ref_laplace_spectrum": (_i, [_f, _f, _vp, _i, _vp, _i, _vp, _vp, _vp]),
            "ref_tdbem_init": (_i, [_f, _f, _vp, _vp]),
            "ref_fdtd_create": (_vp, [_i, _f, _f, _i]),
            "ref_fdtd_destroy": (None, [_vp]),
            "ref_fdtd_step": (_i, [_vp, _i]),
            "ref_fdtd_time": (_i, [_vp]),
            "ref_fdtd_read": (_i, [_vp, _i, _vp]),
            "ref_fdtd_write": (_i, [_vp, _i, _vp]),
            "ref_fdtd_read_pml": (_i, [_vp, _i, _vp]),
            "ref_cells_create": (_vp, [_i, _f, _f, _vp]),
            "ref_cells_destroy": (None, [_vp]),
            "ref_cells_set_mesh": (_i, [_vp, _vp, _i, _vp, _i, _vp]),
            "ref_cells_update_mesh": (_i, [_vp, _vp, _vp]),
            "ref_cells_read": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
            "ref_cells_write_grid": (_i, [_vp, _i, _vp]),
            "ref_cells_read_grid": (_i, [_vp, _i, _vp]),
            "ref_cells_fresh_error": (_i, [_vp]),
            "ref_ghost_create": (_vp, [_i, _f, _f, _vp, _f]),
            "ref_ghost_set_mesh": (_i, [_vp, _vp, _i, _vp, _i]),
            "ref_ghost_update_mesh": (_i, [_vp, _vp]),
            "ref_ghost_run": (_i, [_vp, _vp, _i, _vp, _i, _vp]),
            "ref_ghost_count": (_i, [_vp]),
            "ref_ghost_read": (_i, [_vp, _vp, _vp, _vp]),
        })
        _rlibs[path] = lib
    return _rlibs[path]


class ReferenceGhost:
    """The reference GhostCellSolver (compiled from source): labels, the ghost system from an
    8 x 8 SVD per ghost cell (cuSOLVER), BiCGSTAB-ILU0 per step (cuSPARSE)."""

    def __init__(self, res, dl, dt, min_pos=(0, 0, 0), threshold=25.0):
        self.lib = reference_lib()
        mn = np.asarray(min_pos, np.float32)
        self.h = self.lib.ref_ghost_create(int(res), float(dl), float(dt), _p(mn), float(threshold))
        if not self.h:
            raise RuntimeError("ref_ghost_create failed")
        self.res, self.nt = int(res), 0

    def close(self):
        if self.h:
            self.lib.ref_cells_destroy(self.h)
            self.h = None

    def _ok(self, rc, what):
        if rc != 0:
            raise RuntimeError("reference %s failed (%d)" % (what, rc))

    def set_mesh(self, verts, tris):
        v = np.ascontiguousarray(verts, np.float32).reshape(-1, 3)
        f = np.ascontiguousarray(tris, np.int32).reshape(-1, 3)
        self._ok(self.lib.ref_ghost_set_mesh(self.h, _p(v), len(v), _p(f), len(f)), "ghost set_mesh")
        self.nt = len(f)

    def update_mesh(self, verts):
        v = np.ascontiguousarray(verts, np.float32).reshape(-1, 3)
        self._ok(self.lib.ref_ghost_update_mesh(self.h, _p(v)), "ghost update_mesh")

    def run(self, acc, listeners):
        a = np.ascontiguousarray(acc, np.float32).reshape(-1, self.nt)
        lx = np.ascontiguousarray(np.asarray(listeners, np.int32).reshape(-1, 3))
        out = np.zeros((a.shape[0], len(lx)), np.float32)
        self._ok(self.lib.ref_ghost_run(self.h, _p(a), a.shape[0], _p(lx), len(lx), _p(out)), "ghost run")
        return out

    def ghosts(self):
        """(cells (g, 3), second_order (g,), weights (g, 8))"""
        g = self.lib.ref_ghost_count(self.h)
        c = np.zeros((max(g, 0), 3), np.int32)
        o = np.zeros(max(g, 0), np.int32)
        w = np.zeros((max(g, 0), 8), np.float32)
        if g > 0:
            self._ok(self.lib.ref_ghost_read(self.h, _p(c), _p(o), _p(w)), "ghost read")
        return c, o, w

    def grid(self, rel=0):
        out = np.zeros(self.res ** 3, np.float32)
        self._ok(self.lib.ref_cells_read_grid(self.h, rel, _p(out)), "read_grid")
        return out.reshape((self.res,) * 3)


class Reference:
    """The reference PPPMSolver (compiled from source) behind its headless entry points."""

    def __init__(self, res, dl, dt, min_pos=(0, 0, 0), reflect_coeff=0.83, ndebug=False):
        self.lib = reference_lib(ndebug)
        mn = np.asarray(min_pos, np.float32)
        self.h = self.lib.ref_pppm_create(int(res), float(dl), float(dt), _p(mn), float(reflect_coeff))
        if not self.h:
            raise RuntimeError("ref_pppm_create failed")
        self.res, self.nt, self.nv = int(res), 0, 0

    def close(self):
        if self.h:
            self.lib.ref_pppm_destroy(self.h)
            self.h = None

    def _ok(self, rc, what):
        if rc != 0:
            raise RuntimeError("reference %s failed (%d)" % (what, rc))

    def set_mesh(self, verts, tris):
        v = np.ascontiguousarray(verts, np.float32).reshape(-1, 3)
        f = np.ascontiguousarray(tris, np.int32).reshape(-1, 3)
        self._ok(self.lib.ref_pppm_set_mesh(self.h, _p(v), len(v), _p(f), len(f)), "set_mesh")
        self.nv, self.nt = len(v), len(f)

    def update_mesh(self, verts):
        v = np.ascontiguousarray(verts, np.float32).reshape(-1, 3)
        self._ok(self.lib.ref_pppm_update_mesh(self.h, _p(v)), "update_mesh")

    def check_mesh(self, verts):
        v = np.ascontiguousarray(verts, np.float32).reshape(-1, 3)
        self._ok(self.lib.ref_pppm_check_mesh(self.h, _p(v)), "check_mesh")

    def set_checks(self, on):
        self.lib.ref_pppm_set_checks(self.h, 1 if on else 0)

    def run_device(self, acc_ptr, nsteps, listener, out=None):
        """Steps driven by device-resident accelerations (acc_ptr: device pointer to
        nsteps x nt floats); the listener cell is read back every step like the demo."""
        o = out if out is not None else np.zeros(nsteps, np.float32)
        self._ok(self.lib.ref_pppm_run_device(self.h, ctypes.c_void_p(acc_ptr), int(nsteps), int(listener[0]),
                                              int(listener[1]), int(listener[2]), _p(o)), "run_device")
        return o

    def run(self, acc, listeners):
        a = np.ascontiguousarray(acc, np.float32).reshape(-1, self.nt)
        lx = np.ascontiguousarray(np.asarray(listeners, np.int32).reshape(-1, 3))
        out = np.zeros((a.shape[0], len(lx)), np.float32)
        self._ok(self.lib.ref_pppm_run(self.h, _p(a), a.shape[0], _p(lx), len(lx), _p(out)), "run")
        return out

    @property
    def t(self):
        return self.lib.ref_pppm_time(self.h)

    def grid(self, rel=0):
        out = np.zeros(self.res ** 3, np.float32)
        self._ok(self.lib.ref_pppm_read_grid(self.h, rel, _p(out)), "read_grid")
        return out.reshape((self.res,) * 3)

    def write_grid(self, rel, arr):
        self._ok(self.lib.ref_pppm_write_grid(self.h, rel, _p(np.ascontiguousarray(arr, np.float32))), "write_grid")

    def far(self):
        out = np.zeros(self.res ** 3, np.float32)
        self._ok(self.lib.ref_pppm_read_far(self.h, _p(out)), "read_far")
        return out.reshape((self.res,) * 3)

    def history(self):
        n = np.zeros((self.nt, 32), np.float32)
        d = np.zeros((self.nt, 32), np.float32)
        self._ok(self.lib.ref_pppm_read_history(self.h, _p(n), _p(d)), "read_history")
        return n, d

    def write_history(self, n, d):
        self._ok(self.lib.ref_pppm_write_history(self.h, _p(np.ascontiguousarray(n, np.float32)),
                                                 _p(np.ascontiguousarray(d, np.float32))), "write_history")

    def triangles(self):
        g = np.zeros((self.nt, 7), np.float32)
        c = np.zeros((self.nt, 6), np.int32)
        self._ok(self.lib.ref_pppm_read_triangles(self.h, _p(g), _p(c)), "read_triangles")
        return g, c

    def lists(self):
        sz = np.zeros(4, np.int32)
        self._ok(self.lib.ref_pppm_list_sizes(self.h, _p(sz)), "list_sizes")
        n3, p3, b4, p4 = (int(x) for x in sz)
        n3c = np.zeros((n3, 4), np.int32)
        p3t = np.zeros(p3, np.int32)
        b4c = np.zeros((b4, 4), np.int32)
        b4l = np.zeros(self.nt, np.int32)
        p4t = np.zeros(p4, np.int32)
        cc = np.zeros(self.res ** 3, np.int32)
        self._ok(self.lib.ref_pppm_read_lists(self.h, _p(n3c), _p(p3t), _p(b4c), _p(b4l), _p(p4t), _p(cc)), "read_lists")
        return dict(n3_cells=n3c, n3_tris=p3t, b4_cells=b4c, b4_tris=b4l, n4_tris=p4t, cell_counts=cc)

    def grid_cache(self):
        out = np.zeros(self.nt * 54, RECORD)
        self._ok(self.lib.ref_pppm_read_grid_cache(self.h, _p(out)), "read_grid_cache")
        return out

    def face_cache(self, pairs):
        p = np.ascontiguousarray(pairs, np.int32).reshape(-1, 2)
        c = np.ascontiguousarray(p[:, 0])
        n = np.ascontiguousarray(p[:, 1])
        out = np.zeros(len(p), RECORD)
        self._ok(self.lib.ref_pppm_read_face_cache(self.h, _p(c), _p(n), len(p), _p(out)), "read_face_cache")
        return out

    def interp(self):
        out = np.zeros((self.nt, 8), np.float32)
        self._ok(self.lib.ref_pppm_read_interp(self.h, _p(out)), "read_interp")
        return out

    def reset_fields(self):
        self._ok(self.lib.ref_pppm_reset_fields(self.h), "reset_fields")


def reference_weight(dt, dl, verts, src, point=None, face=None, ndebug=False):
    lib = reference_lib(ndebug)
    v = np.ascontiguousarray(verts, np.float32)
    s = np.ascontiguousarray(src, np.int32)
    out = np.zeros(32, np.float32)
    if point is not None:
        rc = lib.ref_laplace_weight(float(dt), float(dl), _p(v), len(v) // 3 if v.ndim == 1 else len(v), _p(s), 1,
                                    None, _p(np.ascontiguousarray(point, np.float32)), _p(out))
    else:
        rc = lib.ref_laplace_weight(float(dt), float(dl), _p(v), len(v) // 3 if v.ndim == 1 else len(v), _p(s), 0,
                                    _p(np.ascontiguousarray(face, np.int32)), None, _p(out))
    if rc:
        raise RuntimeError("ref_laplace_weight failed")
    return out


def reference_tdbem(dt, dl):
    lib = reference_lib()
    lam = ctypes.c_float()
    wn = np.zeros(32, np.float32)
    lib.ref_tdbem_init(float(dt), float(dl), ctypes.byref(lam), _p(wn))
    return lam.value, wn.reshape(16, 2)


class ReferenceFDTD:
    def __init__(self, res, dl, dt, pml_width=0):
        self.lib = reference_lib()
        self.h = self.lib.ref_fdtd_create(int(res), float(dl), float(dt), int(pml_width))
        self.res = res

    def close(self):
        if self.h:
            self.lib.ref_fdtd_destroy(self.h)
            self.h = None

    def step(self, n=1):
        if self.lib.ref_fdtd_step(self.h, int(n)):
            raise RuntimeError("ref_fdtd_step failed")

    @property
    def t(self):
        return self.lib.ref_fdtd_time(self.h)

    def grid(self, rel=0):
        out = np.zeros(self.res ** 3, np.float32)
        self.lib.ref_fdtd_read(self.h, rel, _p(out))
        return out.reshape((self.res,) * 3)

    def write(self, rel, arr):
        self.lib.ref_fdtd_write(self.h, rel, _p(np.ascontiguousarray(arr, np.float32)))


class ReferenceCells:
    def __init__(self, res, dl, dt, min_pos):
        self.lib = reference_lib()
        self.h = self.lib.ref_cells_create(int(res), float(dl), float(dt), _p(np.asarray(min_pos, np.float32)))
        self.res = res

    def close(self):
        if self.h:
            self.lib.ref_cells_destroy(self.h)
            self.h = None

    def set_mesh(self, verts, tris, acc=None):
        v = np.ascontiguousarray(verts, np.float32).reshape(-1, 3)
        f = np.ascontiguousarray(tris, np.int32).reshape(-1, 3)
        a = np.ascontiguousarray(acc if acc is not None else np.zeros(len(f)), np.float32)
        rc = self.lib.ref_cells_set_mesh(self.h, _p(v), len(v), _p(f), len(f), _p(a))
        if rc:
            raise RuntimeError("ref_cells_set_mesh failed (%d)" % rc)

    def update_mesh(self, verts, acc):
        rc = self.lib.ref_cells_update_mesh(self.h, _p(np.ascontiguousarray(verts, np.float32)),
                                            _p(np.ascontiguousarray(acc, np.float32)))
        if rc:
            raise RuntimeError("ref_cells_update_mesh failed (%d)" % rc)

    def read(self):
        n = self.res ** 3
        t = np.zeros(n, np.int32)
        ne = np.zeros(n, np.int32)
        gh = np.zeros(n, np.int32)
        npnt = np.zeros((n, 3), np.float32)
        rp = np.zeros((n, 3), np.float32)
        d = np.zeros(n, np.float32)
        self.lib.ref_cells_read(self.h, _p(t), _p(ne), _p(gh), _p(npnt), _p(rp), _p(d))
        return dict(type=t, nearest=ne, ghost=gh, nearest_point=npnt, reflect=rp, dist=d)

    def write_grid(self, rel, arr):
        self.lib.ref_cells_write_grid(self.h, rel, _p(np.ascontiguousarray(arr, np.float32)))

    def grid(self, rel=0):
        out = np.zeros(self.res ** 3, np.float32)
        self.lib.ref_cells_read_grid(self.h, rel, _p(out))
        return out.reshape((self.res,) * 3)
