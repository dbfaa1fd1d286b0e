"""ctypes binding of ``libdem_b200.so`` (declared in ``include/dem_b200.h``).

PyTorch is used only for device memory, pinned host staging buffers and the
current CUDA stream.  Every computation goes through the CUDA kernels of the
library; there is no CPU fallback: if the library or a CUDA device is missing
the classes raise instead of computing elsewhere.
"""

from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parents[1] / "libdem_b200.so"

DEM_OK = 0
DEM_E_INVALID = 1
DEM_E_CAPACITY = 2
DEM_E_CUDA = 3
DEM_E_DEVICE = 4
DEM_E_NOT_ALLOCATED = 5

PREC_FP64 = 0
PREC_MIXED = 1
PRECISIONS = {"fp64": PREC_FP64, "mixed": PREC_MIXED}

SCHED_AUTO = 0
SCHED_SPLIT = 1
SCHED_SYMMETRIC = 2
SCHED_SYMMETRIC_PLAIN = 3
SCHEDULES = {"auto": SCHED_AUTO, "split": SCHED_SPLIT, "symmetric": SCHED_SYMMETRIC,
             "symmetric_plain": SCHED_SYMMETRIC_PLAIN}

DEVERR_WAIT_TIMEOUT = 1
DEVERR_PAIR_OVERFLOW = 2
DEVERR_NODE_OVERFLOW = 4
DEVERR_NONFINITE = 8

# name -> (restype, argtypes); the C ABI in include/dem_b200.h
_i, _d, _vp, _i64 = C.c_int, C.c_double, C.c_void_p, C.c_int64
SIGNATURES = {
    "dem_version": (C.c_char_p, []),
    "dem_kernel_binary_version": (_i, [_i, C.POINTER(_i)]),
    "dem_launch_count": (C.c_ulonglong, []),
    "dem_count_replayed_launches": (None, [C.c_ulonglong]),
    "dem_ctx_create": (_i, [_i, _i, C.POINTER(_vp)]),
    "dem_ctx_destroy": (None, [_vp]),
    "dem_ctx_reserve": (_i, [_vp, _i]),
    "dem_ctx_capacity": (_i, [_vp]),
    "dem_last_error": (C.c_char_p, [_vp]),
    "dem_device_errors": (_i, [_vp, C.POINTER(C.c_uint32), _vp]),
    "dem_profile_enable": (_i, [_vp, _i]),
    "dem_profile_read": (_i, [_vp, C.c_char_p, C.POINTER(_d), C.POINTER(_i)]),
    "dem_profile_reset": (_i, [_vp]),
    "dem_direct_set_tuning": (_i, [_vp, _i, _i, _i, _d, _d, _i]),
    "dem_direct_get_tuning": (_i, [_vp, C.POINTER(_i), C.POINTER(_i), C.POINTER(_i), C.POINTER(_d), C.POINTER(_d),
                                   C.POINTER(_i)]),
    "dem_direct_plan": (_i, [_vp, _i, _i, C.POINTER(_i), C.POINTER(_i), C.POINTER(_i), C.POINTER(C.c_longlong),
                             C.POINTER(_i)]),
    "dem_direct_vjp": (_i, [_vp, _i] + [_vp] * 10 + [_d, _d, _d, _d, _i] + [_vp] * 7 + [_vp]),
    "dem_bh_create": (_i, [_vp, _i, C.POINTER(_vp)]),
    "dem_bh_destroy": (None, [_vp]),
    "dem_bh_build": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _d, _i, _i, _vp]),
    "dem_bh_forces": (_i, [_vp, _d, _d, _vp, _vp, _vp, _vp]),
    "dem_bh_velocity": (_i, [_vp, _vp, _vp, _vp, _d, _d, _d, _vp, _vp, _vp, _vp]),
    "dem_bh_stats": (_i, [_vp, C.POINTER(_i64)]),
    "dem_bh_set_window": (_i, [_vp, _i]),
    "dem_bh_set_correction": (_i, [_vp, _vp]),
    "dem_corr_create": (_i, [_vp, _i, _vp, _vp, _vp, _d, _d, _d, _d, _d, _d, C.POINTER(_vp)]),
    "dem_corr_destroy": (None, [_vp]),
    "dem_corr_info": (_i, [_vp, C.POINTER(_i), C.POINTER(_d), C.POINTER(_d)]),
    "dem_corr_gather_probe": (_i, [_vp, _i, _i, _vp, _vp]),
    "dem_direct_convection_corr": (_i, [_vp, _vp, _i] + [_vp] * 7 + [_d, _d, _i, _i, _vp, _vp, _vp, _vp]),
    "dem_batch_create": (_i, [_vp, _i, C.POINTER(_i64), C.POINTER(_d), _i, C.POINTER(_vp)]),
    "dem_batch_destroy": (None, [_vp]),
    "dem_batch_info": (_i, [_vp, C.POINTER(_i), C.POINTER(_i), C.POINTER(_i), C.POINTER(_i)]),
    "dem_batch_set_tuning": (_i, [_vp, _i, _i]),
    "dem_batch_get_tuning": (_i, [_vp, C.POINTER(_i), C.POINTER(_i)]),
    "dem_batch_forces": (_i, [_vp, _vp, _vp, _vp, _vp, _d, _vp, _vp, _vp, _vp]),
    "dem_batch_convection": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _d, _vp, _vp, _vp, _vp]),
    "dem_batch_step": (_i, [_vp, _vp, _vp, _vp, _vp, _d, _d, _d, _d, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "dem_batch_autotune": (_i, [_vp, _vp, _vp, _vp, _vp, _d, _d, _vp, _vp, _vp, _vp, _vp, _vp, _i, _vp,
                                C.POINTER(_d)]),
    "dem_batch_capture": (_i, [_vp, _vp, _vp, _vp, _vp, _d, _d, _d, _d, _vp, _vp, _vp, _vp, _vp, _vp]),
    "dem_batch_replay": (_i, [_vp, _i, _vp]),
    "dem_aos_to_soa": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _vp]),
    "dem_soa_to_aos": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _vp]),
    "dem_direct_forces": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _d, _d, _i, _i, _vp, _vp, _vp, _vp]),
    "dem_direct_convection": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _d, _d, _i, _i, _vp, _vp, _vp, _vp]),
    "dem_direct_forces_and_convection": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _d, _d, _d, _i, _i, _vp, _vp, _vp, _vp,
                                              _vp, _vp, _vp]),
    "dem_euler_update": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _d, _d, _d, _i, _vp, _vp, _vp, _vp]),
    "dem_euler_update_total": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _vp, _vp, _d, _d, _i, _vp, _vp, _vp, _vp]),
    "dem_hash_detect": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _d, _i, _i, _vp, _i64, _vp, _vp]),
    "dem_hash_detect_noalloc": (_i, [_i, _vp, _vp, _vp, _vp, _d, _i, _i, _vp, _i64, _vp, _vp]),
    "dem_overlap_pairs": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _d, _i, _i, _vp, _i64, _vp, _vp]),
    "dem_generate_droplets": (_i, [_vp, _i, C.c_ulonglong, _d, _d, _d, _d, _d, _i, _i, _vp, _vp, _vp, _vp,
                                   C.POINTER(_i), _vp]),
    "dem_merge": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "dem_tree_create": (_i, [_vp, _i, _i, C.POINTER(_vp)]),
    "dem_tree_destroy": (None, [_vp]),
    "dem_tree_build": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _d, _i, _i, _vp]),
    "dem_tree_forces": (_i, [_vp, _d, _d, _vp, _vp, _vp, _vp]),
    "dem_tree_propagate_forces": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "dem_tree_velocity": (_i, [_vp, _vp, _vp, _vp, _d, _d, _d, _vp, _vp, _vp, _vp]),
    "dem_tree_stats": (_i, [_vp, C.POINTER(_i64)]),
    "dem_tree_set_correction": (_i, [_vp, _vp]),
    "dem_tree_collision_matrix": (_i, [_vp, _vp, _i, _vp, _vp]),
    "dem_pair_bin_matrix": (_i, [_vp, _vp, _vp, _i64, _vp, _i, _vp, _vp]),
    "dem_tree_nodes": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "dem_tree_leaf_indices": (_i, [_vp, _vp, _vp]),
}

_lib = None
_lock = threading.Lock()


class DemError(RuntimeError):
    """A CUDA or device-side failure reported by libdem_b200."""


def lib():
    """Load the library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not LIB_PATH.exists():
                    raise ImportError(
                        f"{LIB_PATH} is missing: build it with `python particle-simulator_b200/build_native.py`"
                    )
                L = C.CDLL(str(LIB_PATH))
                for name, (res, args) in SIGNATURES.items():
                    fn = getattr(L, name)
                    fn.restype = res
                    fn.argtypes = args
                _lib = L
    return _lib


def exported_symbols():
    return sorted(SIGNATURES)


def version() -> str:
    return lib().dem_version().decode()


def kernel_binary_version(device: int = 0) -> int:
    """Binary version of the device code the runtime loads for this library's
    kernels (100 for sm_100a); needs a CUDA device."""
    v = _i()
    rc = lib().dem_kernel_binary_version(int(device), C.byref(v))
    if rc != DEM_OK:
        raise RuntimeError(f"dem_kernel_binary_version failed ({rc})")
    return v.value


def launch_count() -> int:
    """Kernels launched by the library in this process so far (host counter)."""
    return int(lib().dem_launch_count())


def count_replayed_launches(k: int) -> None:
    """Credit the counter with k library kernels replayed from a captured CUDA graph."""
    lib().dem_count_replayed_launches(int(k))


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("libdem_b200 needs a CUDA device (B200, sm_100a); none is available")
    return torch


def ptr(t) -> int | None:
    return None if t is None else t.data_ptr()


class Context:
    """One ``dem_ctx`` (device workspace) bound to a CUDA device."""

    def __init__(self, capacity: int, device=None):
        torch = _torch()
        self.torch = torch
        if device is None:
            device = torch.cuda.current_device()
        self.device = torch.device("cuda", torch.device(device).index if not isinstance(device, int) else device)
        self.handle = _vp()
        with torch.cuda.device(self.device):
            self._check(lib().dem_ctx_create(self.device.index, max(int(capacity), 1), C.byref(self.handle)), "create")

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value and _lib is not None:
            try:
                _lib.dem_ctx_destroy(h)
            except Exception:  # pragma: no cover - interpreter shutdown
                pass
            self.handle = None

    # -- errors -------------------------------------------------------------
    def _check(self, rc: int, what: str):
        if rc == DEM_OK:
            return
        msg = (lib().dem_last_error(self.handle).decode() if self.handle else "") or what
        if rc in (DEM_E_INVALID, DEM_E_CAPACITY):
            raise ValueError(msg)
        if rc == DEM_E_NOT_ALLOCATED:
            raise RuntimeError(msg)
        raise DemError(f"{what}: {msg} (code {rc})")

    def stream(self):
        return self.torch.cuda.current_stream(self.device).cuda_stream

    @property
    def capacity(self) -> int:
        return lib().dem_ctx_capacity(self.handle)

    def reserve(self, capacity: int):
        self._check(lib().dem_ctx_reserve(self.handle, int(capacity)), "reserve")

    def device_errors(self) -> int:
        out = C.c_uint32(0)
        self._check(lib().dem_device_errors(self.handle, C.byref(out), self.stream()), "device_errors")
        return int(out.value)

    def raise_device_errors(self):
        f = self.device_errors()
        if f & DEVERR_WAIT_TIMEOUT:
            raise DemError("a bounded device wait timed out")
        if f & DEVERR_NONFINITE:
            raise DemError("a kernel produced a non-finite value")
        return f

    # -- kernel timing ------------------------------------------------------
    def profile(self, enable: bool = True):
        self._check(lib().dem_profile_enable(self.handle, int(bool(enable))), "profile_enable")

    def profile_read(self, name: str):
        ms, k = _d(), _i()
        self._check(lib().dem_profile_read(self.handle, name.encode(), C.byref(ms), C.byref(k)), "profile_read")
        return float(ms.value), int(k.value)

    def profile_reset(self):
        self._check(lib().dem_profile_reset(self.handle), "profile_reset")

    # -- tuning -------------------------------------------------------------
    def set_tuning(self, i_per_thread=0, threads=0, j_splits=None, near_force=0.0, near_oseen=0.0, schedule=None):
        cur = self.get_tuning()
        if j_splits is None:
            j_splits = cur["j_splits"]
        if schedule is None:
            schedule = cur["schedule"]
        schedule = SCHEDULES.get(schedule, schedule)
        self._check(
            lib().dem_direct_set_tuning(self.handle, int(i_per_thread), int(threads), int(j_splits),
                                        float(near_force), float(near_oseen), int(schedule)),
            "set_tuning",
        )

    def get_tuning(self):
        a, b, c, g = _i(), _i(), _i(), _i()
        d, e = _d(), _d()
        self._check(lib().dem_direct_get_tuning(self.handle, C.byref(a), C.byref(b), C.byref(c), C.byref(d), C.byref(e),
                                                C.byref(g)), "get_tuning")
        return dict(i_per_thread=a.value, threads=b.value, j_splits=c.value, near_force=d.value, near_oseen=e.value,
                    schedule=g.value)

    def plan(self, n, periodic=True):
        """The plan the mixed passes run for n droplets: resolved schedule name,
        i-per-thread, threads per CTA, CTAs per pass, j-chunks (split only)."""
        sc, ipt, th, js = _i(), _i(), _i(), _i()
        ctas = C.c_longlong()
        self._check(lib().dem_direct_plan(self.handle, int(n), int(bool(periodic)), C.byref(sc), C.byref(ipt),
                                          C.byref(th), C.byref(ctas), C.byref(js)), "plan")
        names = {v: k for k, v in SCHEDULES.items()}
        return dict(schedule=names[sc.value], i_per_thread=ipt.value, threads=th.value, ctas=ctas.value,
                    j_splits=js.value)

    # -- thin wrappers over the C ABI (torch CUDA tensors in, no allocation) --
    def aos_to_soa(self, n, aos, soa):
        self._check(lib().dem_aos_to_soa(self.handle, n, ptr(aos), ptr(soa[0]), ptr(soa[1]), ptr(soa[2]), self.stream()),
                    "aos_to_soa")

    def soa_to_aos(self, n, soa, aos):
        self._check(lib().dem_soa_to_aos(self.handle, n, ptr(soa[0]), ptr(soa[1]), ptr(soa[2]), ptr(aos), self.stream()),
                    "soa_to_aos")

    def direct_forces(self, n, pos, r, m_const, L, periodic, precision, out):
        self._check(
            lib().dem_direct_forces(self.handle, n, ptr(pos[0]), ptr(pos[1]), ptr(pos[2]), ptr(r), float(m_const),
                                    float(L), int(periodic), int(precision), ptr(out[0]), ptr(out[1]), ptr(out[2]),
                                    self.stream()),
            "direct_forces",
        )

    def direct_convection(self, n, pos, r, F, eta_const, L, periodic, precision, out):
        self._check(
            lib().dem_direct_convection(self.handle, n, ptr(pos[0]), ptr(pos[1]), ptr(pos[2]), ptr(r), ptr(F[0]),
                                        ptr(F[1]), ptr(F[2]), float(eta_const), float(L), int(periodic),
                                        int(precision), ptr(out[0]), ptr(out[1]), ptr(out[2]), self.stream()),
            "direct_convection",
        )

    def direct_forces_and_convection(self, n, pos, r, m_const, eta_const, L, periodic, precision, F, V):
        self._check(
            lib().dem_direct_forces_and_convection(self.handle, n, ptr(pos[0]), ptr(pos[1]), ptr(pos[2]), ptr(r),
                                                   float(m_const), float(eta_const), float(L), int(periodic),
                                                   int(precision), ptr(F[0]), ptr(F[1]), ptr(F[2]), ptr(V[0]),
                                                   ptr(V[1]), ptr(V[2]), self.stream()),
            "direct_forces_and_convection",
        )

    def direct_convection_corr(self, corr: "Correction", n, pos, r, F, eta_const, L, periodic, precision, out):
        self._check(
            lib().dem_direct_convection_corr(self.handle, corr.handle, n, ptr(pos[0]), ptr(pos[1]), ptr(pos[2]),
                                             ptr(r), ptr(F[0]), ptr(F[1]), ptr(F[2]), float(eta_const), float(L),
                                             int(periodic), int(precision), ptr(out[0]), ptr(out[1]),
                                             ptr(out[2]), self.stream()),
            "direct_convection_corr",
        )

    def direct_vjp(self, n, pos, r, F, lam, m_const, eta_const, stokes, L, periodic, mu, g, gr):
        self._check(
            lib().dem_direct_vjp(self.handle, n, ptr(pos[0]), ptr(pos[1]), ptr(pos[2]), ptr(r), ptr(F[0]), ptr(F[1]),
                                 ptr(F[2]), ptr(lam[0]), ptr(lam[1]), ptr(lam[2]), float(m_const), float(eta_const),
                                 float(stokes), float(L), int(periodic), ptr(mu[0]), ptr(mu[1]), ptr(mu[2]),
                                 ptr(g[0]), ptr(g[1]), ptr(g[2]), ptr(gr), self.stream()),
            "direct_vjp",
        )

    def euler_update(self, n, pos, r, F, V, stokes, dt, L, periodic, out):
        self._check(
            lib().dem_euler_update(self.handle, n, ptr(pos[0]), ptr(pos[1]), ptr(pos[2]), ptr(r), ptr(F[0]), ptr(F[1]),
                                   ptr(F[2]), ptr(V[0]), ptr(V[1]), ptr(V[2]), float(stokes), float(dt), float(L),
                                   int(periodic), ptr(out[0]), ptr(out[1]), ptr(out[2]), self.stream()),
            "euler_update",
        )

    def euler_update_total(self, n, pos, V, dt, L, periodic, out):
        self._check(
            lib().dem_euler_update_total(self.handle, n, ptr(pos[0]), ptr(pos[1]), ptr(pos[2]), ptr(V[0]), ptr(V[1]),
                                         ptr(V[2]), float(dt), float(L), int(periodic), ptr(out[0]), ptr(out[1]),
                                         ptr(out[2]), self.stream()),
            "euler_update_total",
        )

    def hash_detect(self, n, pos, r, L, periodic, table_size, pairs, capacity, counts):
        self._check(
            lib().dem_hash_detect(self.handle, n, ptr(pos[0]), ptr(pos[1]), ptr(pos[2]), ptr(r), float(L),
                                  int(periodic), int(table_size), ptr(pairs), int(capacity), ptr(counts),
                                  self.stream()),
            "hash_detect",
        )

    def overlap_pairs(self, n, pos, r, L, periodic, table_size, pairs, capacity, counts):
        self._check(
            lib().dem_overlap_pairs(self.handle, n, ptr(pos[0]), ptr(pos[1]), ptr(pos[2]), ptr(r), float(L),
                                    int(periodic), int(table_size), ptr(pairs), int(capacity), ptr(counts),
                                    self.stream()),
            "overlap_pairs",
        )

    def generate_droplets(self, n, seed, lo, hi, rmin, rmax, minimum_distance, periodic, max_rounds, pos, r):
        rounds = _i(0)
        self._check(
            lib().dem_generate_droplets(self.handle, int(n), int(seed) & 0xFFFFFFFFFFFFFFFF, float(lo), float(hi),
                                        float(rmin), float(rmax), float(minimum_distance), int(bool(periodic)),
                                        int(max_rounds), ptr(pos[0]), ptr(pos[1]), ptr(pos[2]), ptr(r),
                                        C.byref(rounds), self.stream()),
            "generate_droplets",
        )
        return int(rounds.value)

    def pair_bin_matrix(self, pairs, num_pairs, capacity, bins, nbins, out):
        self._check(lib().dem_pair_bin_matrix(self.handle, ptr(pairs), ptr(num_pairs), int(capacity), ptr(bins),
                                              int(nbins), ptr(out), self.stream()), "pair_bin_matrix")

    def merge(self, n, pos, r, pairs, num_pairs, out_pos, out_r, n_out, merged=None):
        self._check(
            lib().dem_merge(self.handle, n, ptr(pos[0]), ptr(pos[1]), ptr(pos[2]), ptr(r), ptr(pairs), ptr(num_pairs),
                            ptr(out_pos[0]), ptr(out_pos[1]), ptr(out_pos[2]), ptr(out_r), ptr(n_out), ptr(merged),
                            self.stream()),
            "merge",
        )


class Correction:
    """One ``dem_corr``: a periodic-image correction grid on the device.

    Grids: (n, n, n) float64 host arrays (C order), nodes grid_min + k / inv_dx.
    Scalars as load_periodic_correction computes them."""

    def __init__(self, ctx: Context, grid_u, grid_v, grid_w, grid_min, inv_dx, Fz_inv, L_ratio, eta_ratio,
                 self_coeff):
        grids = [np.ascontiguousarray(g, dtype=np.float64) for g in (grid_u, grid_v, grid_w)]
        n = grids[0].shape[0] if grids[0].ndim == 3 else -1
        if any(g.shape != (n, n, n) for g in grids):
            raise ValueError("correction grids must be three (n, n, n) arrays")
        self.ctx = ctx  # the grid lives on ctx's device; keep the context alive
        self.n = n
        self.handle = _vp()
        ctx._check(lib().dem_corr_create(ctx.handle, n, grids[0].ctypes.data, grids[1].ctypes.data,
                                         grids[2].ctypes.data, float(grid_min), float(inv_dx), float(Fz_inv),
                                         float(L_ratio), float(eta_ratio), float(self_coeff),
                                         C.byref(self.handle)), "corr_create")

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value and _lib is not None:
            try:
                _lib.dem_corr_destroy(h)
            except Exception:  # pragma: no cover
                pass
            self.handle = None

    def gather_probe(self, ctas, per_thread, out):
        """Random 96-byte cell gathers from the FP32 table (see dem_corr_gather_probe)."""
        self.ctx._check(lib().dem_corr_gather_probe(self.handle, int(ctas), int(per_thread), ptr(out),
                                                    self.ctx.stream()), "corr_gather_probe")

    def info(self):
        n, c, g = _i(), _d(), _d()
        self.ctx._check(lib().dem_corr_info(self.handle, C.byref(n), C.byref(c), C.byref(g)), "corr_info")
        return dict(n=n.value, common=c.value, self_coeff=g.value)


class Tree:
    """One ``dem_tree`` (FP64 flat octree) owned by a Context."""

    def __init__(self, ctx: Context, capacity: int, max_nodes: int):
        self.ctx = ctx
        self.capacity = int(capacity)
        self.max_nodes = int(max_nodes)
        self.handle = _vp()
        ctx._check(lib().dem_tree_create(ctx.handle, self.capacity, self.max_nodes, C.byref(self.handle)),
                   "tree_create")

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value and _lib is not None:
            try:
                _lib.dem_tree_destroy(h)
            except Exception:  # pragma: no cover
                pass
            self.handle = None

    def build(self, n, pos, r, L, periodic, mpl):
        self.ctx._check(lib().dem_tree_build(self.handle, n, ptr(pos[0]), ptr(pos[1]), ptr(pos[2]), ptr(r), float(L),
                                             int(bool(periodic)), int(mpl), self.ctx.stream()), "tree_build")

    def forces(self, m_const, theta_sq, out):
        self.ctx._check(lib().dem_tree_forces(self.handle, float(m_const), float(theta_sq), ptr(out[0]), ptr(out[1]),
                                              ptr(out[2]), self.ctx.stream()), "tree_forces")

    def propagate_forces(self, F=None):
        a = (None, None, None) if F is None else (ptr(F[0]), ptr(F[1]), ptr(F[2]))
        self.ctx._check(lib().dem_tree_propagate_forces(self.handle, *a, self.ctx.stream()), "tree_propagate")

    def velocity(self, F, eta_const, theta_sq, stokes_factor, out):
        a = (None, None, None) if F is None else (ptr(F[0]), ptr(F[1]), ptr(F[2]))
        self.ctx._check(lib().dem_tree_velocity(self.handle, *a, float(eta_const), float(theta_sq),
                                                float(stokes_factor), ptr(out[0]), ptr(out[1]), ptr(out[2]),
                                                self.ctx.stream()), "tree_velocity")

    def collision_matrix(self, bins, nbins, out):
        self.ctx._check(lib().dem_tree_collision_matrix(self.handle, ptr(bins), int(nbins), ptr(out),
                                                        self.ctx.stream()), "tree_collision_matrix")

    def set_correction(self, corr: Correction | None):
        self._corr = corr  # the tree borrows the grid
        self.ctx._check(lib().dem_tree_set_correction(self.handle, None if corr is None else corr.handle),
                        "tree_set_correction")

    def stats(self):
        out = (_i64 * 8)()
        self.ctx._check(lib().dem_tree_stats(self.handle, out), "tree_stats")
        keys = ("node_count", "parent_count", "leaf_slot_count", "max_nodes", "n_levels", "num_particles",
                "pool_exhausted", "capacity")
        return {k: int(v) for k, v in zip(keys, out)}

    def nodes(self, count=None, first_child=None, next_=None, leaf_start=None, r3=None, fs=None):
        self.ctx._check(lib().dem_tree_nodes(self.handle, ptr(count), ptr(first_child), ptr(next_), ptr(leaf_start),
                                             ptr(r3), ptr(fs), self.ctx.stream()), "tree_nodes")

    def leaf_indices(self, out):
        self.ctx._check(lib().dem_tree_leaf_indices(self.handle, ptr(out), self.ctx.stream()), "tree_leaf_indices")


class MortonTree:
    """One ``dem_bh``: Barnes-Hut octree from Morton keys (FP32 walks)."""

    def __init__(self, ctx: Context, capacity: int):
        self.ctx = ctx
        self.capacity = int(capacity)
        self.handle = _vp()
        ctx._check(lib().dem_bh_create(ctx.handle, self.capacity, C.byref(self.handle)), "bh_create")

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value and _lib is not None:
            try:
                _lib.dem_bh_destroy(h)
            except Exception:  # pragma: no cover
                pass
            self.handle = None

    def build(self, n, pos, r, L, periodic, leaf_size):
        self.ctx._check(lib().dem_bh_build(self.handle, int(n), ptr(pos[0]), ptr(pos[1]), ptr(pos[2]), ptr(r),
                                           float(L), int(bool(periodic)), int(leaf_size), self.ctx.stream()),
                        "bh_build")

    def forces(self, m_const, theta, out):
        self.ctx._check(lib().dem_bh_forces(self.handle, float(m_const), float(theta), ptr(out[0]), ptr(out[1]),
                                            ptr(out[2]), self.ctx.stream()), "bh_forces")

    def velocity(self, F, eta_const, theta, stokes_factor, out):
        a = (None, None, None) if F is None else (ptr(F[0]), ptr(F[1]), ptr(F[2]))
        self.ctx._check(lib().dem_bh_velocity(self.handle, *a, float(eta_const), float(theta), float(stokes_factor),
                                              ptr(out[0]), ptr(out[1]), ptr(out[2]), self.ctx.stream()),
                        "bh_velocity")

    def set_window(self, window_level):
        self.ctx._check(lib().dem_bh_set_window(self.handle, int(window_level)), "bh_set_window")

    def set_correction(self, corr: Correction | None):
        self._corr = corr  # the tree borrows the grid
        self.ctx._check(lib().dem_bh_set_correction(self.handle, None if corr is None else corr.handle),
                        "bh_set_correction")

    def stats(self):
        out = (_i64 * 8)()
        self.ctx._check(lib().dem_bh_stats(self.handle, out), "bh_stats")
        keys = ("node_count", "levels", "num_particles", "max_nodes", "leaf_pairs", "node_terms", "leaf_size",
                "capacity")
        return {k: int(v) for k, v in zip(keys, out)}


class Batch:
    """One ``dem_batch``: independent boxes, droplets [offsets[b], offsets[b+1])."""

    def __init__(self, ctx: Context, offsets, L, periodic: bool):
        self.ctx = ctx
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        Ls = np.ascontiguousarray(L, dtype=np.float64)
        self.nbox = len(Ls)
        if len(off) != self.nbox + 1:
            raise ValueError("offsets must have one entry more than L")
        self.handle = _vp()
        ctx._check(lib().dem_batch_create(ctx.handle, self.nbox, off.ctypes.data_as(C.POINTER(_i64)),
                                          Ls.ctypes.data_as(C.POINTER(_d)), int(bool(periodic)),
                                          C.byref(self.handle)), "batch_create")

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value and _lib is not None:
            try:
                _lib.dem_batch_destroy(h)
            except Exception:  # pragma: no cover
                pass
            self.handle = None

    def info(self):
        a, b, c, d = _i(), _i(), _i(), _i()
        self.ctx._check(lib().dem_batch_info(self.handle, C.byref(a), C.byref(b), C.byref(c), C.byref(d)), "info")
        return dict(nbox=a.value, n=b.value, items_ipt2=c.value, items_ipt4=d.value)

    def set_tuning(self, i_per_thread=4, ctas=0):
        self.ctx._check(lib().dem_batch_set_tuning(self.handle, int(i_per_thread), int(ctas)), "batch_set_tuning")

    def get_tuning(self):
        a, b = _i(), _i()
        self.ctx._check(lib().dem_batch_get_tuning(self.handle, C.byref(a), C.byref(b)), "batch_get_tuning")
        return dict(i_per_thread=a.value, ctas=b.value)

    def forces(self, pos, r, m_const, out):
        self.ctx._check(lib().dem_batch_forces(self.handle, ptr(pos[0]), ptr(pos[1]), ptr(pos[2]), ptr(r),
                                               float(m_const), ptr(out[0]), ptr(out[1]), ptr(out[2]),
                                               self.ctx.stream()), "batch_forces")

    def convection(self, pos, r, F, eta_const, out):
        self.ctx._check(lib().dem_batch_convection(self.handle, ptr(pos[0]), ptr(pos[1]), ptr(pos[2]), ptr(r),
                                                   ptr(F[0]), ptr(F[1]), ptr(F[2]), float(eta_const), ptr(out[0]),
                                                   ptr(out[1]), ptr(out[2]), self.ctx.stream()), "batch_convection")

    def step(self, pos, r, m_const, eta_const, stokes, dt, F, V):
        self.ctx._check(lib().dem_batch_step(self.handle, ptr(pos[0]), ptr(pos[1]), ptr(pos[2]), ptr(r),
                                             float(m_const), float(eta_const), float(stokes), float(dt), ptr(F[0]),
                                             ptr(F[1]), ptr(F[2]), ptr(V[0]), ptr(V[1]), ptr(V[2]),
                                             self.ctx.stream()), "batch_step")

    def autotune(self, pos, r, m_const, eta_const, F, V, reps=3):
        best = _d()
        self.ctx._check(lib().dem_batch_autotune(self.handle, ptr(pos[0]), ptr(pos[1]), ptr(pos[2]), ptr(r),
                                                 float(m_const), float(eta_const), ptr(F[0]), ptr(F[1]), ptr(F[2]),
                                                 ptr(V[0]), ptr(V[1]), ptr(V[2]), int(reps), self.ctx.stream(),
                                                 C.byref(best)), "batch_autotune")
        return float(best.value)

    def capture(self, pos, r, m_const, eta_const, stokes, dt, F, V):
        self.ctx._check(lib().dem_batch_capture(self.handle, ptr(pos[0]), ptr(pos[1]), ptr(pos[2]), ptr(r),
                                                float(m_const), float(eta_const), float(stokes), float(dt),
                                                ptr(F[0]), ptr(F[1]), ptr(F[2]), ptr(V[0]), ptr(V[1]), ptr(V[2])),
                        "batch_capture")

    def replay(self, steps):
        self.ctx._check(lib().dem_batch_replay(self.handle, int(steps), self.ctx.stream()), "batch_replay")


class Buffers:
    """Growable device and pinned-host buffers owned by one calculator."""

    def __init__(self, device):
        import torch

        self.torch = torch
        self.device = device
        self._dev = {}
        self._host = {}

    def dev(self, name, shape, dtype=None):
        torch = self.torch
        dtype = dtype or torch.float64
        numel = int(np.prod(shape))
        t = self._dev.get(name)
        if t is None or t.numel() < numel or t.dtype != dtype:
            t = torch.empty(max(numel, 1), dtype=dtype, device=self.device)
            self._dev[name] = t
        return t[:numel].view(*shape)

    def host(self, name, shape, dtype=None):
        torch = self.torch
        dtype = dtype or torch.float64
        numel = int(np.prod(shape))
        t = self._host.get(name)
        if t is None or t.numel() < numel or t.dtype != dtype:
            t = torch.empty(max(numel, 1), dtype=dtype, pin_memory=True)
            self._host[name] = t
        return t[:numel].view(*shape)


def is_cuda_tensor(a) -> bool:
    try:
        import torch

        return isinstance(a, torch.Tensor) and a.is_cuda
    except Exception:  # pragma: no cover
        return False
