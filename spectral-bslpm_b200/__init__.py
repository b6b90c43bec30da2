"""B200-native backward semi-Lagrangian hot path of spectral-BSLPM.

Python binding of the C ABI in include/sbslpm.h (libsbslpm.so, built in-tree
by ``make -C spectral-bslpm_b200/csrc``).  The names mirror the reference's
C++ entry points (bve_back_rk4_step, upward_pass, bve_vel_interactions,
downward_pass_3, dual_tree_traversal, interp_init, ...).  Field arguments of
the device entry points are torch CUDA float64 tensors in the reference's
[panel][q] row-major layout; torch provides device memory and the stream,
every computation runs in this library's sm_100a kernels.

There is no CPU fallback: without the library or a GPU the calls raise.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

__all__ = [
    "SbslpmError", "Config", "Panel", "InteractPair", "FP64", "MIXED", "VEL_FMM", "VEL_DIRECT", "library_path",
    "FORCING_NONE", "FORCING_SSW", "FORCING_SSW2",
    "lib", "config_default", "read_run_config", "panel_count", "leaf_count", "cubed_sphere_panels_init",
    "interp_init", "cube_sphere_spec_points", "dual_tree_traversal", "dual_tree_traversal_flagged",
    "dual_tree_traversal_device_multi", "interp_vals_bli", "point_locate_panel",
    "Context", "direct_sum_bve", "direct_sum_inv_lap", "output_grid", "NcFile", "kernel_launches", "Grid",
    "build_grid",
]

HERE = os.path.dirname(os.path.abspath(__file__))
FP64, MIXED = 0, 1
FORCING_NONE, FORCING_SSW, FORCING_SSW2 = 0, 1, 2
VEL_FMM, VEL_DIRECT = 0, 1

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_VP = ctypes.c_void_p


class SbslpmError(RuntimeError):
    def __init__(self, status: int, where: str, message: str):
        super().__init__(f"{where}: status {status} ({message})")
        self.status = status


class Config(ctypes.Structure):
    """sbslpm_config: the hot-path fields of the reference's RunConfig."""

    _fields_ = [
        ("levels", ctypes.c_int),
        ("interp_degree", ctypes.c_int),
        ("fmm_theta", ctypes.c_double),
        ("kernel_eps", ctypes.c_double),
        ("omega", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("tracer_count", ctypes.c_int),
        ("velocity", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("exact_cc", ctypes.c_int),
        ("proxy_degree", ctypes.c_int),
        ("leaf_size", ctypes.c_int),
        ("g_over_a", ctypes.c_double),
        ("forcing", ctypes.c_int),
    ]


class Panel(ctypes.Structure):
    """sbslpm_panel: the reference's CubedSpherePanel."""

    _fields_ = [(n, ctypes.c_int) for n in (
        "id", "id_top_edge", "id_left_edge", "id_bot_edge", "id_right_edge", "face", "level", "parent_id",
        "child1", "child2", "child3", "child4", "is_leaf")] + [
        (n, ctypes.c_double) for n in ("min_xi", "max_xi", "min_eta", "max_eta", "radius", "area")] + [
        ("point_count", ctypes.c_int)]


class InteractPair(ctypes.Structure):
    _fields_ = [("target_panel", ctypes.c_int), ("source_panel", ctypes.c_int), ("interact_type", ctypes.c_int)]


def library_path() -> str:
    return os.path.join(HERE, "libsbslpm.so")


_lib = None


def lib() -> ctypes.CDLL:
    """The loaded C ABI library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `make -C {os.path.join(HERE, 'csrc')}`")
    L = ctypes.CDLL(path)
    L.sbslpm_status_string.restype = ctypes.c_char_p
    L.sbslpm_last_error.restype = ctypes.c_char_p
    L.sbslpm_kernel_launches.restype = ctypes.c_long
    L.sbslpm_point_locate_panel.restype = ctypes.c_int
    L.sbslpm_point_locate_panel.argtypes = [ctypes.POINTER(Panel), ctypes.c_double, ctypes.c_double, ctypes.c_double]
    L.sbslpm_interp_vals_bli.argtypes = [_D] + [ctypes.c_double] * 6 + [ctypes.c_int]
    L.sbslpm_dual_tree_traversal.argtypes = [ctypes.c_int, ctypes.POINTER(Panel), ctypes.c_double,
                                             ctypes.POINTER(InteractPair), ctypes.c_long,
                                             ctypes.POINTER(ctypes.c_long)]
    L.sbslpm_dual_tree_traversal_device.argtypes = L.sbslpm_dual_tree_traversal.argtypes
    L.sbslpm_dual_tree_traversal_flagged.argtypes = [ctypes.c_int, ctypes.POINTER(Panel), ctypes.c_double,
                                                     ctypes.POINTER(InteractPair), ctypes.c_char_p, ctypes.c_long,
                                                     ctypes.POINTER(ctypes.c_long)]
    L.sbslpm_dual_tree_traversal_device_multi.argtypes = [ctypes.c_int, ctypes.POINTER(Panel), ctypes.c_int, _D,
                                                          ctypes.POINTER(InteractPair), ctypes.c_char_p,
                                                          ctypes.c_long, ctypes.POINTER(ctypes.c_long)]
    L.sbslpm_batch_setup_times.argtypes = [_VP, _D]
    L.sbslpm_create.argtypes = [ctypes.POINTER(Config), ctypes.POINTER(_VP)]
    for name in ("sbslpm_destroy", "sbslpm_set_stream", "sbslpm_get_sizes", "sbslpm_get_panels",
                 "sbslpm_get_interactions"):
        getattr(L, name).argtypes = None
    L.sbslpm_bve_step.argtypes = [_VP] + [_VP] * 9 + [ctypes.c_double]
    L.sbslpm_bve_step_host.argtypes = [_VP] + [_VP] * 9 + [ctypes.c_double]
    L.sbslpm_pointer_on_device.argtypes = [_VP]
    L.sbslpm_pointer_on_device.restype = ctypes.c_int
    L.sbslpm_bve_run.argtypes = [_VP] + [_VP] * 9 + [ctypes.c_double, ctypes.c_int]
    L.sbslpm_upward_pass.argtypes = [_VP] * 4
    L.sbslpm_bve_vel_interactions.argtypes = [_VP] * 8
    L.sbslpm_downward_pass_3.argtypes = [_VP] * 7
    L.sbslpm_bve_departure.argtypes = [_VP] * 8 + [ctypes.c_double] + [_VP] * 3
    L.sbslpm_bve_remap.argtypes = [_VP] * 9
    L.sbslpm_direct_sum_bve.argtypes = [ctypes.c_long, _VP, _VP, _VP, ctypes.c_long, _VP, _VP, _VP, _VP,
                                        ctypes.c_double, ctypes.c_int, _VP, _VP, _VP, _VP]
    L.sbslpm_direct_sum_bve_noalloc.argtypes = L.sbslpm_direct_sum_bve.argtypes
    L.sbslpm_direct_sum_inv_lap.argtypes = [ctypes.c_long] + [_VP] * 7
    L.sbslpm_interp_to_latlon.argtypes = [_VP, _VP, ctypes.c_int, _VP, ctypes.c_int, _VP, _VP]
    L.sbslpm_poisson_fmm.argtypes = [_VP] * 4
    L.sbslpm_poisson_fmm_interactions.argtypes = [_VP] * 3
    L.sbslpm_downward_pass.argtypes = [_VP] * 3
    L.sbslpm_xyz_vel_to_uv_vel.argtypes = [_VP] * 9
    L.sbslpm_output_grid.argtypes = [ctypes.c_long, _D, _I, _I, _D, _D]
    _L = ctypes.POINTER(ctypes.c_long)
    L.sbslpm_nc_create.argtypes = [ctypes.c_char_p, ctypes.POINTER(_VP)]
    L.sbslpm_nc_def_dim.argtypes = [_VP, ctypes.c_char_p, ctypes.c_long, _I]
    L.sbslpm_nc_def_var.argtypes = [_VP, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, _I, _I]
    L.sbslpm_nc_put_att_text.argtypes = [_VP, ctypes.c_int, ctypes.c_char_p, ctypes.c_char_p]
    L.sbslpm_nc_put_att_int.argtypes = [_VP, ctypes.c_int, ctypes.c_char_p, ctypes.c_long, _I]
    L.sbslpm_nc_put_att_double.argtypes = [_VP, ctypes.c_int, ctypes.c_char_p, ctypes.c_long, _D]
    L.sbslpm_nc_enddef.argtypes = [_VP]
    L.sbslpm_nc_put_vara_double.argtypes = [_VP, ctypes.c_int, _L, _L, _D]
    L.sbslpm_nc_put_vara_int.argtypes = [_VP, ctypes.c_int, _L, _L, _I]
    L.sbslpm_nc_close.argtypes = [_VP]
    L.sbslpm_swe_step.argtypes = [_VP] + [_VP] * 14 + [ctypes.c_double]
    L.sbslpm_swe_run.argtypes = [_VP] + [_VP] * 14 + [ctypes.c_double, ctypes.c_int]
    L.sbslpm_swe_init.argtypes = [_VP] * 14
    L.sbslpm_swe_tendencies.argtypes = [_VP] * 14
    L.sbslpm_unify_boundary_vals.argtypes = [_VP] * 2
    L.sbslpm_swe_vel_interactions.argtypes = [_VP] * 9
    L.sbslpm_swe_tree_velocity.argtypes = [_VP] * 9
    L.sbslpm_cubed_sphere_2d_to_1d.argtypes = [ctypes.c_long, ctypes.c_int, _D, _D, _D, _I, _I,
                                               ctypes.POINTER(ctypes.c_long)]
    L.sbslpm_bve_adjoint_step.argtypes = [_VP] * 8
    L.sbslpm_direct_sum_bve_vjp.argtypes = [ctypes.c_long] + [_VP] * 6 + [ctypes.c_long] + [_VP] * 4 + [
        ctypes.c_double] + [_VP] * 5
    L.sbslpm_batch_create.argtypes = [ctypes.POINTER(Config), ctypes.c_int, _D, _I, ctypes.POINTER(_VP)]
    L.sbslpm_batch_destroy.argtypes = [_VP]
    L.sbslpm_batch_set_stream.argtypes = [_VP, _VP]
    L.sbslpm_batch_get_sizes.argtypes = [_VP, ctypes.POINTER(ctypes.c_long)]
    L.sbslpm_batch_step.argtypes = [_VP] + [_VP] * 6 + [ctypes.c_double]
    L.sbslpm_batch_run.argtypes = [_VP] + [_VP] * 6 + [ctypes.c_double, ctypes.c_int]
    L.sbslpm_batch_tuning.argtypes = [_VP, _I, _D]
    L.sbslpm_batch_pairs.argtypes = [_VP, _D, _D]
    L.sbslpm_batch_set_cc_mode.argtypes = [_VP, ctypes.c_int]
    L.sbslpm_batch_set_wait_test.argtypes = [_VP, ctypes.c_int]
    L.sbslpm_batch_cc_info.argtypes = [_VP, _I, _D, _D]
    L.sbslpm_batch_cc_groups.argtypes = [_VP, ctypes.c_int, _I, _I, _I, _D, _D, _D]
    L.sbslpm_batch_set_tuning.argtypes = [_VP, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.sbslpm_time_interactions.argtypes = [_VP, ctypes.c_int, _D, _D]
    L.sbslpm_set_near_tuning.argtypes = [_VP, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.sbslpm_near_tuning.argtypes = [_VP, _I, _D]
    L.sbslpm_set_cc_tuning.argtypes = [_VP, ctypes.c_int, ctypes.c_int]
    L.sbslpm_batch_set_stage0_shared.argtypes = [_VP, ctypes.c_int]
    L.sbslpm_cc_tuning.argtypes = [_VP, _I, _D]
    L.sbslpm_set_cc_tuning_direct.argtypes = [_VP, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.sbslpm_set_near_mutual.argtypes = [_VP, ctypes.c_int]
    L.sbslpm_set_cc_tuning_bulk.argtypes = [_VP, ctypes.c_int, ctypes.c_int]
    L.sbslpm_set_cc_tuning_warp.argtypes = [_VP, ctypes.c_int, ctypes.c_int]
    L.sbslpm_near_mutual.argtypes = [_VP, _I, _D]
    L.sbslpm_set_near_form.argtypes = [_VP, ctypes.c_int]
    L.sbslpm_near_form.argtypes = [_VP, _I]
    L.sbslpm_batch_set_near_form.argtypes = [_VP, ctypes.c_int]
    L.sbslpm_batch_near_form.argtypes = [_VP, _I]
    L.sbslpm_cc_form.argtypes = [_VP, _I]
    L.sbslpm_measure_fma_peak.argtypes = [ctypes.c_int, ctypes.c_double, _D]
    L.sbslpm_bve_velocity.argtypes = [_VP] * 9
    L.sbslpm_shard_unique_id.argtypes = [_VP]
    L.sbslpm_set_shard.argtypes = [_VP, ctypes.c_int, ctypes.c_int, _VP, ctypes.c_double]
    L.sbslpm_shard_range.argtypes = [_VP, ctypes.POINTER(ctypes.c_long), ctypes.POINTER(ctypes.c_long)]
    L.sbslpm_shard_release.argtypes = [_VP]
    _lib = L
    return L


def _check(status: int, where: str):
    if status != 0:
        L = lib()
        msg = L.sbslpm_last_error().decode() or L.sbslpm_status_string(status).decode()
        raise SbslpmError(status, where, msg)


def kernel_launches() -> int:
    return int(lib().sbslpm_kernel_launches())


def shard_unique_id() -> bytes:
    """A fresh NCCL unique id (128 bytes) for Context.shard (sbslpm_shard_unique_id)."""
    buf = (ctypes.c_ubyte * 128)()
    _check(lib().sbslpm_shard_unique_id(buf), "sbslpm_shard_unique_id")
    return bytes(buf)


def exchange_shard_id(group=None, make=shard_unique_id) -> bytes:
    """The id every rank of a torch.distributed group passes to Context.shard:
    made by the group's first rank (make()) and broadcast to the others -- the
    host side of the reference's MPI communicator set-up."""
    import torch.distributed as dist

    first = dist.get_global_rank(group, 0) if group is not None else 0
    obj = [make() if dist.get_rank(group) == 0 else None]
    dist.broadcast_object_list(obj, src=first, group=group)
    ident = obj[0]
    if not isinstance(ident, bytes) or len(ident) != 128:
        raise ValueError("a shard id is 128 bytes")
    return ident


def shard_slice(leaf_count: int, q: int, tree_leaves: int, rank: int, nranks: int):
    """(first, count) of rank's particles in a [leaf][q] field when tree_leaves
    tree leaves are split into nranks equal contiguous slices (sbslpm_shard_range)."""
    if nranks < 1 or not 0 <= rank < nranks or tree_leaves % nranks:
        raise ValueError("nranks must divide the tree's leaves and 0 <= rank < nranks")
    count = leaf_count * q // nranks
    return rank * count, count


# ---------------------------------------------------------------- config ----

def config_default(**overrides) -> Config:
    cfg = Config()
    _check(lib().sbslpm_config_default(ctypes.byref(cfg)), "sbslpm_config_default")
    for k, v in overrides.items():
        if not hasattr(cfg, k):
            raise AttributeError(f"unknown config field {k}")
        setattr(cfg, k, v)
    return cfg


def read_run_config(path: str, base: Config | None = None) -> Config:
    """read_run_config (src/io_utils.cpp:11-92) into a Config."""
    cfg = base if base is not None else config_default()
    _check(lib().sbslpm_read_run_config(path.encode(), ctypes.byref(cfg)), "sbslpm_read_run_config")
    return cfg


# ----------------------------------------------------------------- setup ----

def panel_count(levels: int) -> int:
    return 2 * (4**levels - 1)


def leaf_count(levels: int) -> int:
    return 6 * 4 ** (levels - 1)


def cubed_sphere_panels_init(levels: int):
    panels = (Panel * panel_count(levels))()
    _check(lib().sbslpm_cubed_sphere_panels_init(levels, panels), "sbslpm_cubed_sphere_panels_init")
    return panels


def interp_init(degree: int, exact_cc: bool = False) -> np.ndarray:
    out = np.zeros(((degree + 1) ** 2, 4))
    _check(lib().sbslpm_interp_init(degree, int(exact_cc), out.ctypes.data_as(_D)), "sbslpm_interp_init")
    return out


def cube_sphere_spec_points(levels: int, degree: int, panels, interp: np.ndarray):
    A, q = leaf_count(levels), (degree + 1) ** 2
    x, y, z, area = (np.zeros((A, q)) for _ in range(4))
    interp = np.ascontiguousarray(interp, dtype=np.float64)
    _check(lib().sbslpm_cube_sphere_spec_points(levels, degree, panels, interp.ctypes.data_as(_D),
                                                *[a.ctypes.data_as(_D) for a in (x, y, z, area)]),
           "sbslpm_cube_sphere_spec_points")
    return x, y, z, area


def dual_tree_traversal(levels: int, panels, theta: float, device: bool = False) -> np.ndarray:
    """Interaction list (I x 3 int32: target, source, type) in the reference's order,
    built on the host or (device=True) on the GPU."""
    fn = lib().sbslpm_dual_tree_traversal_device if device else lib().sbslpm_dual_tree_traversal
    n = ctypes.c_long(0)
    _check(fn(levels, panels, theta, None, 0, ctypes.byref(n)), "traversal")
    out = (InteractPair * max(n.value, 1))()
    _check(fn(levels, panels, theta, out, n.value, ctypes.byref(n)), "traversal")
    return np.ctypeslib.as_array(ctypes.cast(out, ctypes.POINTER(ctypes.c_int)), (max(n.value, 1), 3))[: n.value].copy()


def dual_tree_traversal_flagged(levels: int, panels, theta: float):
    """(list I x 3 int32, near I uint8): the treecode's traversal on the host,
    near = 1 for the leaf pairs that failed the MAC."""
    fn = lib().sbslpm_dual_tree_traversal_flagged
    n = ctypes.c_long(0)
    _check(fn(levels, panels, theta, None, None, 0, ctypes.byref(n)), "traversal")
    out = (InteractPair * max(n.value, 1))()
    near = ctypes.create_string_buffer(max(n.value, 1))
    _check(fn(levels, panels, theta, out, near, n.value, ctypes.byref(n)), "traversal")
    lst = np.ctypeslib.as_array(ctypes.cast(out, ctypes.POINTER(ctypes.c_int)), (max(n.value, 1), 3))[: n.value]
    return lst.copy(), np.frombuffer(near.raw, np.uint8)[: n.value].copy()


def dual_tree_traversal_device_multi(levels: int, panels, thetas):
    """One traversal per theta on the GPU in one launch series: a list of
    (list I x 3 int32, near I uint8) per theta."""
    th = np.ascontiguousarray(thetas, dtype=np.float64)
    fn = lib().sbslpm_dual_tree_traversal_device_multi
    counts = (ctypes.c_long * len(th))()
    _check(fn(levels, panels, len(th), th.ctypes.data_as(_D), None, None, 0, counts), "traversal")
    total = sum(counts)
    out = (InteractPair * max(total, 1))()
    near = ctypes.create_string_buffer(max(total, 1))
    _check(fn(levels, panels, len(th), th.ctypes.data_as(_D), out, near, total, counts), "traversal")
    allp = np.ctypeslib.as_array(ctypes.cast(out, ctypes.POINTER(ctypes.c_int)), (max(total, 1), 3))[:total]
    alln = np.frombuffer(near.raw, np.uint8)[:total]
    res, o = [], 0
    for c in counts:
        res.append((allp[o:o + c].copy(), alln[o:o + c].copy()))
        o += c
    return res


def interp_vals_bli(xi, eta, min_xi, max_xi, min_eta, max_eta, degree) -> np.ndarray:
    out = np.zeros((degree + 1) ** 2)
    _check(lib().sbslpm_interp_vals_bli(out.ctypes.data_as(_D), xi, eta, min_xi, max_xi, min_eta, max_eta, degree),
           "sbslpm_interp_vals_bli")
    return out


def cubed_sphere_2d_to_1d(x: np.ndarray, y: np.ndarray, z: np.ndarray, degree: int):
    """cubed_sphere_2d_to_1d (src/initialize_cubed_sphere.cpp:290-326) on host
    arrays [leaf][q]: (two_d_to_1d int32 [leaf][q], counts int32 [unique])."""
    x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z))
    A = x.shape[0]
    m = np.zeros(x.shape, np.int32)
    counts = np.zeros(A * degree * degree + 2, np.int32)
    u = ctypes.c_long(0)
    _check(lib().sbslpm_cubed_sphere_2d_to_1d(A, degree, *[a.ctypes.data_as(_D) for a in (x, y, z)],
                                              m.ctypes.data_as(_I), counts.ctypes.data_as(_I), ctypes.byref(u)),
           "sbslpm_cubed_sphere_2d_to_1d")
    return m, counts[: u.value].copy()


def point_locate_panel(panels, x, y, z) -> int:
    return int(lib().sbslpm_point_locate_panel(panels, x, y, z))


@dataclass
class Grid:
    """Leaf points of the cubed sphere (numpy, [leaf][q])."""

    levels: int
    degree: int
    panels: object
    interp: np.ndarray
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    area: np.ndarray


def build_grid(levels: int, degree: int, exact_cc: bool = True) -> Grid:
    panels = cubed_sphere_panels_init(levels)
    interp = interp_init(degree, exact_cc)
    x, y, z, area = cube_sphere_spec_points(levels, degree, panels, interp)
    return Grid(levels, degree, panels, interp, x, y, z, area)


# --------------------------------------------------------------- device ----

def _dev(t, name, shape=None):
    """Device pointer of a contiguous float64 CUDA tensor (None -> NULL)."""
    if t is None:
        return None
    import torch

    if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.float64 or not t.is_contiguous():
        raise TypeError(f"{name} must be a contiguous float64 CUDA tensor")
    if shape is not None and t.numel() != int(np.prod(shape)):
        raise ValueError(f"{name} has {t.numel()} elements, expected {shape}")
    return t.data_ptr()


def _host(a, name, shape=None, write=False):
    """Host pointer of a C-contiguous float64 numpy array or CPU torch tensor
    (pinned or pageable; None -> NULL)."""
    if a is None:
        return None
    if hasattr(a, "is_cuda"):
        import torch

        if a.is_cuda or a.dtype != torch.float64 or not a.is_contiguous():
            raise TypeError(f"{name} must be a contiguous float64 host tensor")
        n, ptr = a.numel(), a.data_ptr()
    else:
        if not isinstance(a, np.ndarray) or a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
            raise TypeError(f"{name} must be a C-contiguous float64 numpy array")
        if write and not a.flags["WRITEABLE"]:
            raise ValueError(f"{name} is read-only")
        n, ptr = a.size, a.ctypes.data
    if shape is not None and n != int(np.prod(shape)):
        raise ValueError(f"{name} has {n} elements, expected {shape}")
    return ptr


def pointer_on_device(p) -> int:
    """sbslpm_pointer_on_device: 1 device memory, 0 host memory, -1 unknown."""
    return int(lib().sbslpm_pointer_on_device(ctypes.c_void_p(p)))


def _stream():
    import torch

    return torch.cuda.current_stream().cuda_stream


class Context:
    """sbslpm_ctx: tree, interaction list, static geometry and workspace on one GPU."""

    def __init__(self, cfg: Config):
        self.cfg = cfg
        h = _VP()
        _check(lib().sbslpm_create(ctypes.byref(cfg), ctypes.byref(h)), "sbslpm_create")
        self._h = h
        sizes = (ctypes.c_long * 4)()
        _check(lib().sbslpm_get_sizes(self._h, sizes), "sbslpm_get_sizes")
        self.panel_count, self.leaf_count, self.q, self.interaction_count = (int(v) for v in sizes)

    def close(self):
        if getattr(self, "_h", None):
            lib().sbslpm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _sync_stream(self):
        _check(lib().sbslpm_set_stream(self._h, _VP(_stream())), "sbslpm_set_stream")

    def panels(self):
        out = (Panel * self.panel_count)()
        _check(lib().sbslpm_get_panels(self._h, out), "sbslpm_get_panels")
        return out

    def interactions(self) -> np.ndarray:
        n = max(self.interaction_count, 1)
        out = (InteractPair * n)()
        _check(lib().sbslpm_get_interactions(self._h, out), "sbslpm_get_interactions")
        arr = np.ctypeslib.as_array(ctypes.cast(out, ctypes.POINTER(ctypes.c_int)), (n, 3))
        return arr[: self.interaction_count].copy()

    # -- Poisson FMM ----------------------------------------------------
    def poisson_fmm(self, area, pots, soln):
        """The Poisson FMM driver's solve (executables/poisson_eq_fmm.cpp:128-160): soln written."""
        lq = (self.leaf_count, self.q)
        self._sync_stream()
        _check(lib().sbslpm_poisson_fmm(self._h, _dev(area, "area", lq), _dev(pots, "pots", lq),
                                        _dev(soln, "soln", lq)), "sbslpm_poisson_fmm")

    def poisson_fmm_interactions(self, source, target):
        """poisson_fmm_interactions (src/fmm_interactions/inverse_poisson.cpp:9-34): target += ..."""
        pq = (self.panel_count, self.q)
        self._sync_stream()
        _check(lib().sbslpm_poisson_fmm_interactions(self._h, _dev(source, "source", pq), _dev(target, "target", pq)),
               "sbslpm_poisson_fmm_interactions")

    def downward_pass(self, proxy_target, soln):
        """downward_pass (src/fmm_funcs.cpp:357-372): proxy_target updated, soln written."""
        self._sync_stream()
        _check(lib().sbslpm_downward_pass(self._h, _dev(proxy_target, "proxy_target", (self.panel_count, self.q)),
                                          _dev(soln, "soln", (self.leaf_count, self.q))), "sbslpm_downward_pass")

    # -- output path ----------------------------------------------------
    def interp_to_latlon(self, data, lats, lons, out=None):
        """interp_to_latlon_host (src/interp_funcs.hpp:22-77) on the device: the [leaf][q]
        field data at latitudes lats x longitudes lons (degrees, float64 CUDA tensors);
        returns out [len(lats)][len(lons)]."""
        import torch

        nlat, nlon = int(lats.numel()), int(lons.numel())
        if out is None:
            out = torch.empty((nlat, nlon), dtype=torch.float64, device=data.device)
        self._sync_stream()
        _check(lib().sbslpm_interp_to_latlon(self._h, _dev(data, "data", (self.leaf_count, self.q)), nlat,
                                             _dev(lats, "lats"), nlon, _dev(lons, "lons"),
                                             _dev(out, "out", (nlat, nlon))), "sbslpm_interp_to_latlon")
        return out

    def xyz_vel_to_uv_vel(self, xcos, ycos, zcos, vel_x, vel_y, vel_z, vel_u=None, vel_v=None):
        """xyz_vel_to_uv_vel (src/general_utils_impl.hpp:195-229): (vel_u, vel_v) of the grid."""
        import torch

        vel_u = torch.empty_like(vel_x) if vel_u is None else vel_u
        vel_v = torch.empty_like(vel_x) if vel_v is None else vel_v
        lq = (self.leaf_count, self.q)
        self._sync_stream()
        _check(lib().sbslpm_xyz_vel_to_uv_vel(self._h, *[_dev(t, n, lq) for t, n in (
            (xcos, "xcos"), (ycos, "ycos"), (zcos, "zcos"), (vel_x, "vel_x"), (vel_y, "vel_y"), (vel_z, "vel_z"),
            (vel_u, "vel_u"), (vel_v, "vel_v"))]), "sbslpm_xyz_vel_to_uv_vel")
        return vel_u, vel_v

    # -- the step -------------------------------------------------------
    def bve_back_rk4_step(self, xcos, ycos, zcos, area, vors, vel_x, vel_y, vel_z, tracers=None, time=0.0):
        """bve_back_rk4_step (src/bve_time_step.cpp:311-419): vors, vel_*, tracers in place."""
        lq = (self.leaf_count, self.q)
        self._sync_stream()
        _check(lib().sbslpm_bve_step(self._h, *[_dev(t, n, lq) for t, n in (
            (xcos, "xcos"), (ycos, "ycos"), (zcos, "zcos"), (area, "area"), (vors, "vors"), (vel_x, "vel_x"),
            (vel_y, "vel_y"), (vel_z, "vel_z"))], _dev(tracers, "tracers"), float(time)), "sbslpm_bve_step")

    def bve_back_rk4_step_host(self, xcos, ycos, zcos, area, vors, vel_x, vel_y, vel_z, tracers=None, time=0.0):
        """The step on host arrays (numpy or CPU torch, float64, C order):
        vors, vel_*, tracers in place (sbslpm_bve_step_host)."""
        lq = (self.leaf_count, self.q)
        self._sync_stream()
        ptrs = [_host(a, n, lq, w) for a, n, w in (
            (xcos, "xcos", False), (ycos, "ycos", False), (zcos, "zcos", False), (area, "area", False),
            (vors, "vors", True), (vel_x, "vel_x", True), (vel_y, "vel_y", True), (vel_z, "vel_z", True))]
        tr = _host(tracers, "tracers", lq + (self.cfg.tracer_count,), True) if tracers is not None else None
        _check(lib().sbslpm_bve_step_host(self._h, *ptrs, tr, float(time)), "sbslpm_bve_step_host")

    def bve_run(self, xcos, ycos, zcos, area, vors, vel_x, vel_y, vel_z, tracers=None, time=0.0, nsteps=1):
        """nsteps steps replayed from one captured CUDA graph."""
        lq = (self.leaf_count, self.q)
        self._sync_stream()
        _check(lib().sbslpm_bve_run(self._h, *[_dev(t, n, lq) for t, n in (
            (xcos, "xcos"), (ycos, "ycos"), (zcos, "zcos"), (area, "area"), (vors, "vors"), (vel_x, "vel_x"),
            (vel_y, "vel_y"), (vel_z, "vel_z"))], _dev(tracers, "tracers"), float(time), int(nsteps)),
            "sbslpm_bve_run")

    def bve_velocity(self, xcos, ycos, zcos, area, vors, vel_x, vel_y, vel_z):
        """The step's first-stage velocity of vors into vel_* (sbslpm_bve_velocity); a
        sharded context without a communicator writes only its own slice."""
        lq = (self.leaf_count, self.q)
        self._sync_stream()
        _check(lib().sbslpm_bve_velocity(self._h, *[_dev(t, n, lq) for t, n in (
            (xcos, "xcos"), (ycos, "ycos"), (zcos, "zcos"), (area, "area"), (vors, "vors"), (vel_x, "vel_x"),
            (vel_y, "vel_y"), (vel_z, "vel_z"))]), "sbslpm_bve_velocity")

    # -- one problem over several GPUs -----------------------------------
    def shard(self, rank: int, nranks: int, nccl_id: bytes = None, timeout: float = 300.0):
        """Make this context rank `rank` of `nranks` of one sharded treecode problem
        (sbslpm_set_shard).  With nccl_id (exchange_shard_id) every rank joins the
        communicator together and whole steps all-gather each stage's velocity;
        without it the context evaluates only its own slice (bve_velocity)."""
        ident = None
        if nccl_id is not None:
            if len(nccl_id) != 128:
                raise ValueError("a shard id is 128 bytes")
            ident = (ctypes.c_ubyte * 128).from_buffer_copy(nccl_id)
        self._sync_stream()
        _check(lib().sbslpm_set_shard(self._h, int(rank), int(nranks), ident, float(timeout)), "sbslpm_set_shard")

    def shard_over(self, group=None, timeout: float = 300.0):
        """Shard over the ranks of a torch.distributed group (one GPU per rank)."""
        import torch.distributed as dist

        nranks = dist.get_world_size(group)
        ident = exchange_shard_id(group) if nranks > 1 else None
        self.shard(dist.get_rank(group), nranks, ident, timeout)

    def shard_range(self):
        """(first, count): this rank's particles in a [leaf][q] field."""
        first, count = ctypes.c_long(), ctypes.c_long()
        _check(lib().sbslpm_shard_range(self._h, ctypes.byref(first), ctypes.byref(count)), "sbslpm_shard_range")
        return first.value, count.value

    def shard_release(self):
        """End the context's communicator (every rank together)."""
        _check(lib().sbslpm_shard_release(self._h), "sbslpm_shard_release")

    # -- shallow water (SWE v2) ------------------------------------------
    def swe_back_rk4_step_2(self, xcos, ycos, zcos, area, vors, divs, height, vel_x, vel_y, vel_z, tracers,
                            base_vor_tend, base_div_tend, base_h_tend, time=0.0):
        """swe_back_rk4_step_2 (src/swe_time_step_2.cpp:785-1035): vors, divs, height,
        vel_*, tracers in place."""
        lq = (self.leaf_count, self.q)
        self._sync_stream()
        _check(lib().sbslpm_swe_step(self._h, *[_dev(t, n, lq) for t, n in (
            (xcos, "xcos"), (ycos, "ycos"), (zcos, "zcos"), (area, "area"), (vors, "vors"), (divs, "divs"),
            (height, "height"), (vel_x, "vel_x"), (vel_y, "vel_y"), (vel_z, "vel_z"))], _dev(tracers, "tracers"),
            *[_dev(t, n, lq) for t, n in ((base_vor_tend, "base_vor_tend"), (base_div_tend, "base_div_tend"),
                                          (base_h_tend, "base_h_tend"))], float(time)), "sbslpm_swe_step")

    def swe_run(self, xcos, ycos, zcos, area, vors, divs, height, vel_x, vel_y, vel_z, tracers, base_vor_tend,
                base_div_tend, base_h_tend, time=0.0, nsteps=1):
        """nsteps of the driver loop (step + unify of vors, divs, height) from one CUDA graph."""
        lq = (self.leaf_count, self.q)
        self._sync_stream()
        _check(lib().sbslpm_swe_run(self._h, *[_dev(t, n, lq) for t, n in (
            (xcos, "xcos"), (ycos, "ycos"), (zcos, "zcos"), (area, "area"), (vors, "vors"), (divs, "divs"),
            (height, "height"), (vel_x, "vel_x"), (vel_y, "vel_y"), (vel_z, "vel_z"))], _dev(tracers, "tracers"),
            *[_dev(t, n, lq) for t, n in ((base_vor_tend, "base_vor_tend"), (base_div_tend, "base_div_tend"),
                                          (base_h_tend, "base_h_tend"))], float(time), int(nsteps)),
            "sbslpm_swe_run")

    def swe_init(self, xcos, ycos, zcos, area, vors, divs, height, vel_x, vel_y, vel_z, base_vor_tend,
                 base_div_tend, base_h_tend):
        """The driver's set-up: unified initial velocity and base tendencies (written)."""
        lq = (self.leaf_count, self.q)
        self._sync_stream()
        _check(lib().sbslpm_swe_init(self._h, *[_dev(t, "field", lq) for t in (
            xcos, ycos, zcos, area, vors, divs, height, vel_x, vel_y, vel_z, base_vor_tend, base_div_tend,
            base_h_tend)]), "sbslpm_swe_init")

    def swe_tendencies(self, xcos, ycos, zcos, vel_x, vel_y, vel_z, vors, divs, height, surface, vor_tend,
                       div_tend, h_tend):
        """swe_tendency_computation_2 over every leaf panel."""
        lq = (self.leaf_count, self.q)
        self._sync_stream()
        _check(lib().sbslpm_swe_tendencies(self._h, *[_dev(t, "field", lq) for t in (
            xcos, ycos, zcos, vel_x, vel_y, vel_z, vors, divs, height, surface, vor_tend, div_tend, h_tend)]),
            "sbslpm_swe_tendencies")

    def unify_boundary_vals(self, vals):
        """unify_boundary_vals (src/initialize_cubed_sphere.cpp:364-370), in place."""
        self._sync_stream()
        _check(lib().sbslpm_unify_boundary_vals(self._h, _dev(vals, "vals", (self.leaf_count, self.q))),
               "sbslpm_unify_boundary_vals")

    def swe_vel_interactions(self, disp_x, disp_y, disp_z, source_vor, source_div, t1, t2, t3):
        self._sync_stream()
        _check(lib().sbslpm_swe_vel_interactions(self._h, *[_dev(t, "field") for t in (
            disp_x, disp_y, disp_z, source_vor, source_div, t1, t2, t3)]), "sbslpm_swe_vel_interactions")

    def swe_tree_velocity(self, disp_x, disp_y, disp_z, w_vor, w_div, u_x, u_y, u_z):
        """Treecode SWE velocity at the grid: vorticity sources displaced by disp (strengths
        w_vor), divergence sources at the grid (strengths w_div); u_* written."""
        lq = (self.leaf_count, self.q)
        self._sync_stream()
        _check(lib().sbslpm_swe_tree_velocity(self._h, *[_dev(t, n, lq) for t, n in (
            (disp_x, "disp_x"), (disp_y, "disp_y"), (disp_z, "disp_z"), (w_vor, "w_vor"), (w_div, "w_div"),
            (u_x, "u_x"), (u_y, "u_y"), (u_z, "u_z"))]), "sbslpm_swe_tree_velocity")

    # -- adjoint -----------------------------------------------------------
    def bve_adjoint_step(self, xcos, ycos, zcos, area, vors, vors_bar_next, vors_bar):
        """One reverse step: vors_bar = (d step(vors) / d vors)^T vors_bar_next."""
        lq = (self.leaf_count, self.q)
        self._sync_stream()
        _check(lib().sbslpm_bve_adjoint_step(self._h, *[_dev(t, n, lq) for t, n in (
            (xcos, "xcos"), (ycos, "ycos"), (zcos, "zcos"), (area, "area"), (vors, "vors"),
            (vors_bar_next, "vors_bar_next"), (vors_bar, "vors_bar"))]), "sbslpm_bve_adjoint_step")

    def set_near_tuning(self, threads: int, targets_per_thread: int, splits: int):
        """Fix the treecode's near-field launch shape instead of autotuning it."""
        _check(lib().sbslpm_set_near_tuning(self._h, int(threads), int(targets_per_thread), int(splits)),
               "sbslpm_set_near_tuning")

    def near_tuning(self):
        """(threads, targets per thread, splits, candidates timed, ms per near launch)."""
        shape = (ctypes.c_int * 4)()
        ms = ctypes.c_double()
        _check(lib().sbslpm_near_tuning(self._h, shape, ctypes.byref(ms)), "sbslpm_near_tuning")
        return (*[int(v) for v in shape], ms.value)

    def set_cc_tuning(self, slots: int, chunk_len: int):
        """Fix the treecode's well-separated launch shape (chunk slots per block,
        list entries per chunk; 0, 0: one block per target panel) instead of
        autotuning it."""
        _check(lib().sbslpm_set_cc_tuning(self._h, int(slots), int(chunk_len)), "sbslpm_set_cc_tuning")

    def set_near_mutual(self, on: bool):
        """The first stage's two-sided near-field kernel on or off (mixed, 256-particle leaves)."""
        _check(lib().sbslpm_set_near_mutual(self._h, int(bool(on))), "sbslpm_set_near_mutual")

    def near_mutual(self):
        """(in use for stage 0, ms per launch of the two-sided kernel from the first-step timing)."""
        on, ms = ctypes.c_int(), ctypes.c_double()
        _check(lib().sbslpm_near_mutual(self._h, ctypes.byref(on), ctypes.byref(ms)), "sbslpm_near_mutual")
        return bool(on.value), ms.value

    def set_near_form(self, expanded: bool):
        """Mixed precision: the near-field pair arithmetic, expanded (8 float32
        operations per pair; needs kernel_eps > 0) or difference form (10)."""
        _check(lib().sbslpm_set_near_form(self._h, int(bool(expanded))), "sbslpm_set_near_form")

    def near_form(self) -> bool:
        """True when the near field runs the expanded pair form."""
        on = ctypes.c_int()
        _check(lib().sbslpm_near_form(self._h, ctypes.byref(on)), "sbslpm_near_form")
        return bool(on.value)

    def set_cc_tuning_direct(self, slots: int, chunk_len: int, targets_per_thread: int):
        """Fix the barrier-free form of the mixed-precision well-separated kernel
        (sources read through L1 from a pair-transposed copy) and its shape."""
        _check(lib().sbslpm_set_cc_tuning_direct(self._h, int(slots), int(chunk_len), int(targets_per_thread)),
               "sbslpm_set_cc_tuning_direct")

    def set_cc_tuning_bulk(self, slots: int, chunk_len: int):
        """Fix the bulk-copy form of the mixed-precision well-separated kernel (each slot's
        source panels copied into shared memory by cp.async.bulk, double-buffered)."""
        _check(lib().sbslpm_set_cc_tuning_bulk(self._h, int(slots), int(chunk_len)), "sbslpm_set_cc_tuning_bulk")

    def set_cc_tuning_warp(self, warps: int, chunk_len: int):
        """Fix the warp-per-chunk form of the mixed-precision well-separated kernel
        (ceil(q / 32) target proxies per lane, warp-private cp.async staging)."""
        _check(lib().sbslpm_set_cc_tuning_warp(self._h, int(warps), int(chunk_len)), "sbslpm_set_cc_tuning_warp")

    def cc_form(self) -> int:
        """0: sources staged in shared memory; 1 | 2: barrier-free, targets per thread; 3: bulk copies;
        4: warp per chunk."""
        t = ctypes.c_int()
        _check(lib().sbslpm_cc_form(self._h, ctypes.byref(t)), "sbslpm_cc_form")
        return t.value

    def cc_tuning(self):
        """(slots, chunk length, threads per block, candidates timed, ms per
        well-separated launch)."""
        shape = (ctypes.c_int * 4)()
        ms = ctypes.c_double()
        _check(lib().sbslpm_cc_tuning(self._h, shape, ctypes.byref(ms)), "sbslpm_cc_tuning")
        return (*[int(v) for v in shape], ms.value)

    def time_interactions(self, reps: int = 5):
        """(ms per launch, pair evaluations per launch) of the interaction kernel alone."""
        ms, pairs = ctypes.c_double(), ctypes.c_double()
        self._sync_stream()
        _check(lib().sbslpm_time_interactions(self._h, int(reps), ctypes.byref(ms), ctypes.byref(pairs)),
               "sbslpm_time_interactions")
        return ms.value, pairs.value

    # -- pieces ---------------------------------------------------------
    def upward_pass(self, area, pots, proxy_source):
        self._sync_stream()
        _check(lib().sbslpm_upward_pass(self._h, _dev(area, "area"), _dev(pots, "pots"),
                                        _dev(proxy_source, "proxy_source")), "sbslpm_upward_pass")

    def bve_vel_interactions(self, disp_x, disp_y, disp_z, source, t1, t2, t3):
        self._sync_stream()
        _check(lib().sbslpm_bve_vel_interactions(self._h, *[_dev(t, "field") for t in (
            disp_x, disp_y, disp_z, source, t1, t2, t3)]), "sbslpm_bve_vel_interactions")

    def downward_pass_3(self, t1, t2, t3, s1, s2, s3):
        self._sync_stream()
        _check(lib().sbslpm_downward_pass_3(self._h, *[_dev(t, "field") for t in (t1, t2, t3, s1, s2, s3)]),
               "sbslpm_downward_pass_3")

    def bve_departure(self, xcos, ycos, zcos, v0, v1, v2, v3, dt, dep_x, dep_y, dep_z):
        self._sync_stream()
        _check(lib().sbslpm_bve_departure(self._h, *[_dev(t, "field") for t in (xcos, ycos, zcos, v0, v1, v2, v3)],
                                          float(dt), *[_dev(t, "dep") for t in (dep_x, dep_y, dep_z)]),
               "sbslpm_bve_departure")

    def bve_remap(self, zcos, dep_x, dep_y, dep_z, vors, tracers, new_vors, new_tracers):
        self._sync_stream()
        _check(lib().sbslpm_bve_remap(self._h, *[_dev(t, "field") for t in (zcos, dep_x, dep_y, dep_z, vors)],
                                      _dev(tracers, "tracers"), _dev(new_vors, "new_vors"),
                                      _dev(new_tracers, "new_tracers")), "sbslpm_bve_remap")


class Batch:
    """sbslpm_batch: an ensemble of BVE problems on one particle grid, each
    member with its own vorticity, theta and treecode proxy degree."""

    def __init__(self, base: Config, theta, proxy_degree):
        theta = np.ascontiguousarray(theta, dtype=np.float64)
        deg = np.ascontiguousarray(proxy_degree, dtype=np.int32)
        if theta.shape != deg.shape or theta.ndim != 1:
            raise ValueError("theta and proxy_degree must be 1-D of equal length")
        self.cfg = base
        h = _VP()
        _check(lib().sbslpm_batch_create(ctypes.byref(base), len(theta), theta.ctypes.data_as(_D),
                                         deg.ctypes.data_as(_I), ctypes.byref(h)), "sbslpm_batch_create")
        self._h = h
        sizes = (ctypes.c_long * 4)()
        _check(lib().sbslpm_batch_get_sizes(self._h, sizes), "sbslpm_batch_get_sizes")
        self.members, self.leaf_count, self.q, self.particles = (int(v) for v in sizes)

    def close(self):
        if getattr(self, "_h", None):
            lib().sbslpm_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _sync_stream(self):
        _check(lib().sbslpm_batch_set_stream(self._h, _VP(_stream())), "sbslpm_batch_set_stream")

    def _ptrs(self, xcos, ycos, zcos, area, vors, vel):
        lq = (self.leaf_count, self.q)
        return ([_dev(t, n, lq) for t, n in ((xcos, "xcos"), (ycos, "ycos"), (zcos, "zcos"), (area, "area"))] +
                [_dev(vors, "vors", (self.members,) + lq), _dev(vel, "vel", (self.members, 3) + lq)])

    def step(self, xcos, ycos, zcos, area, vors, vel, time=0.0):
        """One step of every member: vors [members][leaf][q] in place,
        vel [members][3][leaf][q] receives the stage-0 velocities."""
        self._sync_stream()
        _check(lib().sbslpm_batch_step(self._h, *self._ptrs(xcos, ycos, zcos, area, vors, vel), float(time)),
               "sbslpm_batch_step")

    def run(self, xcos, ycos, zcos, area, vors, vel, time=0.0, nsteps=1):
        """nsteps steps of every member replayed from one captured CUDA graph."""
        self._sync_stream()
        _check(lib().sbslpm_batch_run(self._h, *self._ptrs(xcos, ycos, zcos, area, vors, vel), float(time),
                                      int(nsteps)), "sbslpm_batch_run")

    def tuning(self):
        """(threads per block, targets per thread, splits, candidates timed, ms per near launch)."""
        shape = (ctypes.c_int * 4)()
        ms = ctypes.c_double()
        _check(lib().sbslpm_batch_tuning(self._h, shape, ctypes.byref(ms)), "sbslpm_batch_tuning")
        return (*[int(v) for v in shape], ms.value)

    def set_tuning(self, threads: int, targets_per_thread: int, splits: int):
        _check(lib().sbslpm_batch_set_tuning(self._h, int(threads), int(targets_per_thread), int(splits)),
               "sbslpm_batch_set_tuning")

    def pairs(self):
        """(near-field, well-separated) pair evaluations of one velocity evaluation, all members."""
        a, b = ctypes.c_double(), ctypes.c_double()
        _check(lib().sbslpm_batch_pairs(self._h, ctypes.byref(a), ctypes.byref(b)), "sbslpm_batch_pairs")
        return a.value, b.value

    CC_AUTO, CC_CUDA_CORES, CC_TC_3XTF32, CC_TC_TF32, CC_SHARED = -1, 0, 1, 2, 3

    def set_stage0_shared(self, shared: bool):
        """Mixed precision: the first stage's near field shared by theta-sorted
        groups of members (True, the default) or run per member (False: bit-exact
        with single contexts)."""
        _check(lib().sbslpm_batch_set_stage0_shared(self._h, 1 if shared else 0), "sbslpm_batch_set_stage0_shared")

    def set_near_form(self, expanded: bool):
        """The members' near-field pair arithmetic (as Context.set_near_form)."""
        _check(lib().sbslpm_batch_set_near_form(self._h, int(bool(expanded))), "sbslpm_batch_set_near_form")

    def near_form(self) -> bool:
        on = ctypes.c_int()
        _check(lib().sbslpm_batch_near_form(self._h, ctypes.byref(on)), "sbslpm_batch_near_form")
        return bool(on.value)

    def set_cc_mode(self, mode: int):
        """Well-separated interactions: -1 autotuned per proxy-degree group (default for mixed
        precision), 0 CUDA-core pairs, 1 tensor-core 3xTF32 GEMM, 2 tensor-core single-pass TF32 GEMM."""
        _check(lib().sbslpm_batch_set_cc_mode(self._h, int(mode)), "sbslpm_batch_set_cc_mode")

    def setup_times(self) -> dict:
        """Wall time (s) of the creation's list build (every member's traversal on the GPU)."""
        t = ctypes.c_double()
        _check(lib().sbslpm_batch_setup_times(self._h, ctypes.byref(t)), "sbslpm_batch_setup_times")
        return {"lists_s": t.value}

    def set_wait_test(self, on: bool):
        """Test of the tensor-core kernel's bounded waits: with on, its steps
        in modes 1 and 2 report SBSLPM_ERR_TIMEOUT (sbslpm_batch_set_wait_test)."""
        _check(lib().sbslpm_batch_set_wait_test(self._h, int(bool(on))), "sbslpm_batch_set_wait_test")

    def cc_info(self):
        """(mode, union cluster pairs over the degree groups, MMA flops per velocity evaluation)."""
        mode = ctypes.c_int()
        up, fl = ctypes.c_double(), ctypes.c_double()
        _check(lib().sbslpm_batch_cc_info(self._h, ctypes.byref(mode), ctypes.byref(up), ctypes.byref(fl)),
               "sbslpm_batch_cc_info")
        return mode.value, up.value, fl.value

    def cc_groups(self):
        """Per proxy-degree group: dicts of degree, members, mode in use and the autotuner's
        timings (ms per launch) of the per-member CUDA-core, tensor-core 3xTF32 and
        shared-pair CUDA-core modes."""
        n = 16
        deg, mem, mode = (ctypes.c_int * n)(), (ctypes.c_int * n)(), (ctypes.c_int * n)()
        t0, t1, t3 = (ctypes.c_double * n)(), (ctypes.c_double * n)(), (ctypes.c_double * n)()
        _check(lib().sbslpm_batch_cc_groups(self._h, n, deg, mem, mode, t0, t1, t3), "sbslpm_batch_cc_groups")
        return [{"degree": deg[k], "members": mem[k], "mode": mode[k], "ms_cuda_cores": t0[k],
                 "ms_tensor_cores": t1[k], "ms_shared": t3[k]} for k in range(n) if mem[k] > 0]


def measure_fma_peak(kind: int = 0, ms: float = 50.0) -> float:
    """Measured CUDA-core FMA throughput in FLOP/s (kind 0 float32, 1 float64)."""
    out = ctypes.c_double()
    _check(lib().sbslpm_measure_fma_peak(int(kind), float(ms), ctypes.byref(out)), "sbslpm_measure_fma_peak")
    return out.value


def direct_sum_bve(tx, ty, tz, sx, sy, sz, strength, eps, precision=FP64, out=None):
    """Biot-Savart direct sum on the sphere; returns (ux, uy, uz) tensors."""
    import torch

    nt, ns = tx.numel(), sx.numel()
    if out is None:
        out = tuple(torch.empty(nt, dtype=torch.float64, device=tx.device) for _ in range(3))
    _check(lib().sbslpm_direct_sum_bve(nt, *[_dev(t, "target") for t in (tx, ty, tz)], ns,
                                       *[_dev(t, "source") for t in (sx, sy, sz, strength)], float(eps),
                                       int(precision), *[_dev(t, "out") for t in out], _VP(_stream())),
           "sbslpm_direct_sum_bve")
    return out


def direct_sum_bve_noalloc(tx, ty, tz, sx, sy, sz, strength, eps, precision=FP64, out=None):
    """direct_sum_bve through the entry point that allocates no device memory
    (fixed scratch inside the library; at most 699,050 targets)."""
    import torch

    nt, ns = tx.numel(), sx.numel()
    if out is None:
        out = tuple(torch.empty(nt, dtype=torch.float64, device=tx.device) for _ in range(3))
    _check(lib().sbslpm_direct_sum_bve_noalloc(nt, *[_dev(t, "target") for t in (tx, ty, tz)], ns,
                                               *[_dev(t, "source") for t in (sx, sy, sz, strength)], float(eps),
                                               int(precision), *[_dev(t, "out") for t in out], _VP(_stream())),
           "sbslpm_direct_sum_bve_noalloc")
    return out


def direct_sum_bve_vjp(tx, ty, tz, ubar, sx, sy, sz, strength, eps):
    """VJP of direct_sum_bve with respect to the sources: (strength_bar, (sx_bar, sy_bar, sz_bar))."""
    import torch

    nt, ns = tx.numel(), sx.numel()
    qb = torch.empty(ns, dtype=torch.float64, device=sx.device)
    yb = tuple(torch.empty(ns, dtype=torch.float64, device=sx.device) for _ in range(3))
    _check(lib().sbslpm_direct_sum_bve_vjp(nt, *[_dev(t, "target") for t in (tx, ty, tz)],
                                           *[_dev(t.contiguous(), "ubar") for t in ubar], ns,
                                           *[_dev(t, "source") for t in (sx, sy, sz, strength)], float(eps),
                                           _dev(qb, "out"), *[_dev(t, "out") for t in yb], _VP(_stream())),
           "sbslpm_direct_sum_bve_vjp")
    return qb, yb


def _autograd():
    """torch.autograd.Function wrappers (built on first use: torch is optional at import)."""
    import torch

    class DirectSumBVE(torch.autograd.Function):
        """u = direct_sum_bve(targets, sources, strength); gradients for the
        source positions and strengths (targets are treated as constants)."""

        @staticmethod
        def forward(ctx, tx, ty, tz, sx, sy, sz, strength, eps):
            ctx.save_for_backward(tx, ty, tz, sx, sy, sz, strength)
            ctx.eps = eps
            ux, uy, uz = direct_sum_bve(tx, ty, tz, sx, sy, sz, strength, eps)
            return torch.stack([ux, uy, uz])

        @staticmethod
        def backward(ctx, ubar):
            tx, ty, tz, sx, sy, sz, q = ctx.saved_tensors
            qb, (xb, yb, zb) = direct_sum_bve_vjp(tx, ty, tz, [ubar[0], ubar[1], ubar[2]], sx, sy, sz, q, ctx.eps)
            return None, None, None, xb, yb, zb, qb, None

    class BVERollout(torch.autograd.Function):
        """nsteps of bve_back_rk4_step from vors0 with per-step checkpoints of
        the vorticity; the backward pass runs the hand-written adjoint step
        in reverse order from the checkpoints."""

        @staticmethod
        def forward(ctx, vors0, context, xcos, ycos, zcos, area, nsteps):
            v = vors0.detach().clone().contiguous()
            vel = [torch.zeros_like(v) for _ in range(3)]
            ckpt = []
            for _ in range(int(nsteps)):
                ckpt.append(v.clone())
                context.bve_back_rk4_step(xcos, ycos, zcos, area, v, *vel)
            ctx.context = context
            ctx.fields = (xcos, ycos, zcos, area)
            ctx.ckpt = ckpt
            return v

        @staticmethod
        def backward(ctx, vbar):
            wbar = vbar.detach().clone().contiguous()
            out = torch.empty_like(wbar)
            for v in reversed(ctx.ckpt):
                ctx.context.bve_adjoint_step(*ctx.fields, v, wbar, out)
                wbar, out = out, wbar
            return wbar, None, None, None, None, None, None

    return DirectSumBVE, BVERollout


def direct_sum_bve_autograd(tx, ty, tz, sx, sy, sz, strength, eps):
    """direct_sum_bve as a differentiable torch function (gradients for the sources)."""
    return _autograd()[0].apply(tx, ty, tz, sx, sy, sz, strength, eps)


def bve_rollout(context, xcos, ycos, zcos, area, vors0, nsteps):
    """nsteps BVE steps as a differentiable torch function of the initial
    vorticity (a float64 direct-sum context, or a treecode context in float64
    or mixed precision), adjoint with per-step checkpoints."""
    return _autograd()[1].apply(vors0, context, xcos, ycos, zcos, area, int(nsteps))


def output_grid(point_count: int):
    """The drivers' output grid (executables/bve_time_evo.cpp:93-95, 206-211):
    (spacing in degrees, latitudes, longitudes) as float64 numpy arrays."""
    sp, nlat, nlon = ctypes.c_double(), ctypes.c_int(), ctypes.c_int()
    _check(lib().sbslpm_output_grid(int(point_count), ctypes.byref(sp), ctypes.byref(nlat), ctypes.byref(nlon),
                                    None, None), "sbslpm_output_grid")
    lats, lons = np.zeros(nlat.value), np.zeros(nlon.value)
    _check(lib().sbslpm_output_grid(int(point_count), ctypes.byref(sp), ctypes.byref(nlat), ctypes.byref(nlon),
                                    _dp(lats), _dp(lons)), "sbslpm_output_grid")
    return sp.value, lats, lons


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class NcFile:
    """netCDF classic (64-bit offset) writer with the netCDF library's call
    pattern (nc_def_dim, nc_def_var, nc_put_att_*, nc_enddef, nc_put_vara_*,
    nc_close) as the reference drivers use it.  Host arrays."""

    INT, DOUBLE, GLOBAL = 4, 6, -1

    def __init__(self, path: str):
        h = _VP()
        _check(lib().sbslpm_nc_create(str(path).encode(), ctypes.byref(h)), "sbslpm_nc_create")
        self._h = h

    def def_dim(self, name: str, length: int) -> int:
        d = ctypes.c_int()
        _check(lib().sbslpm_nc_def_dim(self._h, name.encode(), int(length), ctypes.byref(d)), "sbslpm_nc_def_dim")
        return d.value

    def def_var(self, name: str, nctype: int, dims) -> int:
        dims = (ctypes.c_int * max(len(dims), 1))(*dims)
        v = ctypes.c_int()
        _check(lib().sbslpm_nc_def_var(self._h, name.encode(), int(nctype), len(dims) if dims else 0, dims,
                                       ctypes.byref(v)), "sbslpm_nc_def_var")
        return v.value

    def put_att(self, varid: int, name: str, value):
        if isinstance(value, str):
            _check(lib().sbslpm_nc_put_att_text(self._h, varid, name.encode(), value.encode()), "sbslpm_nc_put_att")
            return
        arr = np.atleast_1d(value)
        if np.issubdtype(arr.dtype, np.integer):
            a = np.ascontiguousarray(arr, np.int32)
            _check(lib().sbslpm_nc_put_att_int(self._h, varid, name.encode(), a.size,
                                               a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))), "sbslpm_nc_put_att")
        else:
            a = np.ascontiguousarray(arr, np.float64)
            _check(lib().sbslpm_nc_put_att_double(self._h, varid, name.encode(), a.size, _dp(a)), "sbslpm_nc_put_att")

    def enddef(self):
        _check(lib().sbslpm_nc_enddef(self._h), "sbslpm_nc_enddef")

    def put_vara(self, varid: int, data, start=None):
        data = np.asarray(data)
        cl = ctypes.c_long * max(data.ndim, 1)
        st = cl(*(start if start is not None else [0] * data.ndim))
        cnt = cl(*data.shape)
        if np.issubdtype(data.dtype, np.integer):
            a = np.ascontiguousarray(data, np.int32)
            _check(lib().sbslpm_nc_put_vara_int(self._h, varid, st, cnt, a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))),
                   "sbslpm_nc_put_vara")
        else:
            a = np.ascontiguousarray(data, np.float64)
            _check(lib().sbslpm_nc_put_vara_double(self._h, varid, st, cnt, _dp(a)), "sbslpm_nc_put_vara")

    def close(self):
        if getattr(self, "_h", None):
            _check(lib().sbslpm_nc_close(self._h), "sbslpm_nc_close")
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def direct_sum_inv_lap(x, y, z, area, pots, soln):
    """direct_sum_inv_lap (src/direct_sum.cpp:8-15): soln accumulated in place."""
    _check(lib().sbslpm_direct_sum_inv_lap(x.numel(), *[_dev(t, "field") for t in (x, y, z, area, pots, soln)],
                                           _VP(_stream())), "sbslpm_direct_sum_inv_lap")
