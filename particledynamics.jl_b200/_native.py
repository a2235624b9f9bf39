"""ctypes binding of libpdb200.so (declarations mirror include/pdb200.h).

The shared object is built in-tree by ``build.py``.  Loading fails loudly when
it is missing: there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libpdb200.so"

PD_OK, PD_EINVAL, PD_ENOMEM, PD_ECAPACITY, PD_ENONFINITE, PD_ECUFFT, PD_ECUDA, PD_ESTATE, PD_ENOTSUP = range(9)
PD_LJ_NONE, PD_LJ_UNIFORM, PD_LJ_TABLE = 0, 1, 2
PD_MESH_SPME, PD_MESH_P3M_AD, PD_MESH_P3M_IK = 1, 2, 3
PD_MAX_POLY = 32
PD_MAX_TYPES = 16
PD_PAIR_LJ, PD_PAIR_WCA = 1, 2
PD_LEARNED_MAX_RADIAL = 8

_p = C.c_void_p
_fp = C.c_void_p   # device pointers are passed as integers


class ClusterParams(C.Structure):
    _fields_ = [
        ("n", C.c_int),
        ("rmax", C.c_double), ("skin", C.c_double), ("prune_buffer", C.c_double),
        ("lj_kind", C.c_int),
        ("lj_c6", C.c_float), ("lj_c12", C.c_float), ("lj_rc2", C.c_float), ("lj_esh", C.c_float),
        ("ntypes", C.c_int),
        ("lj_table", C.c_float * (PD_MAX_TYPES * PD_MAX_TYPES * 4)),
        ("coulomb", C.c_int),
        ("coul_C", C.c_float), ("coul_rc2", C.c_float), ("coul_sx", C.c_float), ("coul_eshift", C.c_float),
        ("coul_has_mesh", C.c_int),
        ("coul_ne", C.c_int), ("coul_nf", C.c_int),
        ("coul_pe", C.c_float * PD_MAX_POLY), ("coul_pf", C.c_float * PD_MAX_POLY),
        ("selfc", C.c_float),
        ("nstlist", C.c_int), ("nstprune", C.c_int),
    ]


class GsdIndexEntry(C.Structure):
    """pd_gsd_index_entry: one 32-byte GSD index entry (include/pdb200.h)."""
    _fields_ = [("frame", C.c_uint64), ("N", C.c_uint64), ("location", C.c_int64), ("M", C.c_uint32),
                ("id", C.c_uint16), ("type", C.c_uint8), ("flags", C.c_uint8)]


class SnapshotSrc(C.Structure):
    """pd_snapshot_src: one frame's per-particle device arrays (include/pdb200.h)."""
    _fields_ = [("n", C.c_int), ("dim", C.c_int)] + [(k, C.c_void_p) for k in (
        "x", "y", "z", "vx", "vy", "vz", "fx", "fy", "fz", "type", "vir")]


class SnapshotOffsets(C.Structure):
    _fields_ = [("position", C.c_uint64), ("velocity", C.c_uint64), ("force", C.c_uint64), ("typeid", C.c_uint64),
                ("virial", C.c_uint64), ("virial_columns", C.c_int), ("bytes", C.c_uint64)]


class ClusterStats(C.Structure):
    _fields_ = [
        ("superclusters", C.c_int), ("outer_entries", C.c_int), ("working_entries", C.c_int),
        ("error", C.c_int), ("required", C.c_int), ("capacity", C.c_int),
        ("builds", C.c_int), ("prunes", C.c_int), ("nsmax", C.c_int), ("nslot", C.c_int),
        ("last_build", C.c_int), ("last_prune", C.c_int),
        ("tile_bits", C.c_longlong),
        ("mask_entries", C.c_int), ("outside_pairs", C.c_int),
    ]


class MeshParams(C.Structure):
    _fields_ = [
        ("kind", C.c_int), ("order", C.c_int), ("alias_order", C.c_int),
        ("mesh", C.c_int * 3),
        ("alpha", C.c_double), ("C", C.c_double),
        ("background", C.c_int), ("qtotal", C.c_double),
        ("nmax", C.c_int),
    ]


PD_MESH_ESP, PD_MESH_ESP_DECONV = 4, 5
PD_PROLATE_MAX_QUAD, PD_PROLATE_MAX_DEG, PD_PROLATE_MAX_NODES = 256, 24, 8


class Prolate(C.Structure):
    """pd_prolate: the prolate split and window of an ESP mesh (include/pdb200.h)."""
    _fields_ = [
        ("cutoff", C.c_double), ("nquad", C.c_int),
        ("xq", C.c_double * PD_PROLATE_MAX_QUAD), ("wchi", C.c_double * PD_PROLATE_MAX_QUAD),
        ("background_coefficient", C.c_double), ("deg", C.c_int),
        ("poly", (C.c_double * PD_PROLATE_MAX_NODES) * (PD_PROLATE_MAX_DEG + 1)),
        ("table", C.c_void_p * 3),
    ]


class MDState(C.Structure):
    _fields_ = [
        ("n", C.c_int),
        ("x", _fp), ("y", _fp), ("z", _fp),
        ("vx", _fp), ("vy", _fp), ("vz", _fp),
        ("fx", _fp), ("fy", _fp), ("fz", _fp),
        ("q", _fp), ("type", _fp), ("inv_mass", _fp),
        ("inv_mass_uniform", C.c_float),
        ("epot", _fp), ("vir6", _fp), ("vglobal6", _fp),
    ]


class EllParams(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("n", C.c_int),
        ("cutoff", C.c_double), ("skin", C.c_double),
        ("cap", C.c_int), ("interval", C.c_int), ("model", C.c_int),
        ("eps", C.c_float), ("sigma", C.c_float), ("rc2", C.c_float), ("eshift", C.c_float),
        ("lanes", C.c_int),
    ]


class EllStats(C.Structure):
    _fields_ = [
        ("valid", C.c_int), ("error", C.c_int), ("requested", C.c_int),
        ("step", C.c_longlong), ("last_build", C.c_longlong), ("interval", C.c_longlong),
        ("checks", C.c_longlong), ("builds", C.c_longlong), ("required", C.c_longlong),
        ("cap", C.c_int), ("lanes", C.c_int), ("allpairs", C.c_int),
    ]


class BatchReplica(C.Structure):
    _fields_ = [
        ("box", C.c_double * 3), ("n", C.c_int), ("kind", C.c_int),
        ("eps", C.c_float), ("sigma", C.c_float), ("rc2", C.c_float), ("eshift", C.c_float),
    ]


class BatchCoulomb(C.Structure):
    """pd_batch_coulomb: the real-space Coulomb polynomial of charged replicas (include/pdb200.h)."""
    _fields_ = [
        ("C", C.c_float), ("rc2", C.c_float), ("sx", C.c_float), ("eshift", C.c_float),
        ("ne", C.c_int), ("nf", C.c_int),
        ("pe", C.c_float * PD_MAX_POLY), ("pf", C.c_float * PD_MAX_POLY),
        ("selfc", C.c_float),
    ]


class LearnedParams(C.Structure):
    _fields_ = [
        ("rcut", C.c_float), ("skin", C.c_float), ("cap", C.c_int),
        ("mu0", C.c_float), ("dmu", C.c_float), ("sigma", C.c_float),
        ("nb", C.c_int), ("nu0", C.c_float), ("dnu", C.c_float), ("tau", C.c_float),
        ("coef", C.c_float * PD_LEARNED_MAX_RADIAL),
    ]


# name: (restype, argtypes)
_SIGS = {
    "pd_version": (C.c_int, []),
    "pd_strerror": (C.c_char_p, [C.c_int]),
    "pd_last_error": (C.c_char_p, []),
    "pd_launch_count": (C.c_uint64, []),
    "pd_cluster_create": (C.c_int, [C.POINTER(_p), C.POINTER(ClusterParams), C.POINTER(C.c_double)]),
    "pd_cluster_destroy": (C.c_int, [_p]),
    "pd_cluster_setup": (C.c_int, [_p, C.POINTER(C.c_double)]),
    "pd_cluster_grow": (C.c_int, [_p]),
    "pd_cluster_set_pair_shape": (C.c_int, [_p, C.c_int, C.c_int]),
    "pd_cluster_pair_shape": (C.c_int, [_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "pd_cluster_request_build": (C.c_int, [_p, _p]),
    "pd_cluster_decide": (C.c_int, [_p, _fp, _fp, _fp, C.c_int, _p]),
    "pd_cluster_build": (C.c_int, [_p, _fp, _fp, _fp, _fp, _fp, C.c_int, _p]),
    "pd_cluster_pack": (C.c_int, [_p, _fp, _fp, _fp, _fp, _fp, _p]),
    "pd_cluster_prune": (C.c_int, [_p, _fp, _fp, _fp, C.c_int, _p]),
    "pd_cluster_pairs": (C.c_int, [_p, C.c_int, _p]),
    "pd_cluster_scatter": (C.c_int, [_p, _fp, _fp, _fp, _fp, _fp, _fp, C.c_int, C.c_int, _p]),
    "pd_cluster_compute": (C.c_int, [_p, _fp, _fp, _fp, _fp, _fp, _fp, _fp, _fp, _fp, _fp, C.c_int, _p]),
    "pd_cluster_compute_static": (C.c_int, [C.POINTER(ClusterParams), C.POINTER(C.c_double), _fp, _fp, _fp, _fp,
                                            _fp, _fp, _fp, _fp, _fp, _fp, C.c_int, _p]),
    "pd_cluster_status": (C.c_int, [_p, C.POINTER(ClusterStats), _p]),
    "pd_cluster_set_exceptions": (C.c_int, [_p, C.c_int, _p, _p, _p, C.c_int, _p, _p]),
    "pd_cluster_order": (_fp, [_p]),
    "pd_cluster_buffers": (C.c_int, [_p, C.POINTER(_p), C.POINTER(_p), C.POINTER(_p), C.POINTER(_p),
                                     C.POINTER(_p), C.POINTER(_p)]),
    "pd_md_set_schedule": (C.c_int, [_p, C.c_int]),
    "pd_mesh_create": (C.c_int, [C.POINTER(_p), C.POINTER(MeshParams), C.POINTER(C.c_double)]),
    "pd_mesh_create_prolate": (C.c_int, [C.POINTER(_p), C.POINTER(MeshParams), C.POINTER(Prolate),
                                         C.POINTER(C.c_double)]),
    "pd_mesh_destroy": (C.c_int, [_p]),
    "pd_mesh_set_box": (C.c_int, [_p, C.POINTER(C.c_double)]),
    "pd_mesh_transform": (C.c_int, [_p, _fp, _fp, _fp, _fp, _fp, C.c_int, C.c_int, _p]),
    "pd_mesh_gather": (C.c_int, [_p, _fp, _fp, _fp, _fp, _fp, C.c_int, _fp, _fp, _fp, _fp, _fp, C.c_int,
                                 C.c_int, _p]),
    "pd_mesh_energy": (C.c_int, [_p, C.POINTER(C.c_double), _p]),
    "pd_mesh_influence": (C.c_int, [_p, _p, _p]),
    "pd_mesh_dims": (C.c_int, [_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "pd_mesh_set_self_force_removal": (C.c_int, [_p, C.c_int]),
    "pd_mesh_self_force_table": (C.c_int, [_p, _p, C.POINTER(C.c_int)]),
    "pd_md_create": (C.c_int, [C.POINTER(_p), _p, _p, C.POINTER(MDState), C.POINTER(C.c_double)]),
    "pd_md_destroy": (C.c_int, [_p]),
    "pd_md_evaluate": (C.c_int, [_p, C.c_int, _p]),
    "pd_md_step": (C.c_int, [_p, C.c_int, C.c_float, C.c_int, C.c_int, _p]),
    "pd_md_step_host": (C.c_int, [_p, _p, _p, C.c_int, C.c_float, C.POINTER(C.c_double), _p]),
    "pd_ell_create": (C.c_int, [C.POINTER(_p), C.POINTER(EllParams), C.POINTER(C.c_double)]),
    "pd_ell_destroy": (C.c_int, [_p]),
    "pd_ell_update": (C.c_int, [_p, _fp, _fp, _fp, _p]),
    "pd_ell_request": (C.c_int, [_p, _p]),
    "pd_ell_forces": (C.c_int, [_p, _fp, _fp, _fp, _fp, _fp, _fp, _fp, _fp, C.c_int, _p]),
    "pd_ell_status": (C.c_int, [_p, C.POINTER(EllStats)]),
    "pd_ell_rows": (C.c_int, [_p, C.POINTER(_p), C.POINTER(_p)]),
    "pd_ell_resize": (C.c_int, [_p, C.c_int]),
    "pd_ell_md_create": (C.c_int, [C.POINTER(_p), _p, C.POINTER(MDState)]),
    "pd_ell_md_destroy": (C.c_int, [_p]),
    "pd_ell_md_evaluate": (C.c_int, [_p, C.c_int, _p]),
    "pd_ell_md_step": (C.c_int, [_p, C.c_int, C.c_float, C.c_int, C.c_int, _p]),
    "pd_ell_md_langevin": (C.c_int, [_p, C.c_int, C.c_float, C.c_float, C.c_float, C.c_ulonglong, C.c_int,
                                     C.c_int, _p]),
    "pd_ell_md_gjf": (C.c_int, [_p, C.c_int, C.c_float, C.c_float, C.c_float, C.c_ulonglong, C.c_int, C.c_int, _p]),
    "pd_ell_md_bookkeeping": (C.c_int, [_p, _fp, _fp, _fp]),
    "pd_ell_md_baoa": (C.c_int, [_p, C.c_int, C.c_float, C.c_float, C.c_float, C.c_ulonglong, C.c_int, C.c_int, _p]),
    "pd_mlp_param_count": (C.c_int, []),
    "pd_mlp_create": (C.c_int, [C.POINTER(_p)]),
    "pd_mlp_destroy": (C.c_int, [_p]),
    "pd_mlp_set_params": (C.c_int, [_p, _p]),
    "pd_mlp_get_params": (C.c_int, [_p, _p]),
    "pd_mlp_get_grads": (C.c_int, [_p, _p]),
    "pd_mlp_forward": (C.c_int, [_p, _fp, C.c_int, _fp, _fp, _fp, _p]),
    "pd_mlp_train": (C.c_int, [_p, _fp, _fp, C.c_int, C.c_float, _p]),
    "pd_mlp_adam": (C.c_int, [_p, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, _p]),
    "pd_mlp_loss": (C.c_int, [_p, C.POINTER(C.c_double), C.c_int]),
    "pd_mlp_zero_grads": (C.c_int, [_p, _p]),
    "pd_mlp_error": (C.c_int, [_p, C.POINTER(C.c_int)]),
    "pd_learned_create": (C.c_int, [C.POINTER(_p), C.POINTER(LearnedParams), C.c_int, C.POINTER(C.c_double)]),
    "pd_learned_destroy": (C.c_int, [_p]),
    "pd_learned_set_radial": (C.c_int, [_p, _p, C.c_int]),
    "pd_learned_descriptors": (C.c_int, [_p, _fp, _fp, _fp, _fp, _fp, _fp, _fp, _fp, _p]),
    "pd_learned_correction": (C.c_int, [_p, _p, _fp, _fp, _fp, _fp, _fp, _fp, _p]),
    "pd_learned_buffers": (C.c_int, [_p, C.POINTER(_p), C.POINTER(_p), C.POINTER(_p)]),
    "pd_learned_status": (C.c_int, [_p, C.POINTER(EllStats)]),
    "pd_learned_resize": (C.c_int, [_p, C.c_int]),
    "pd_md_set_learned": (C.c_int, [_p, _p, _p]),
    "pd_batch_create": (C.c_int, [C.POINTER(_p), C.POINTER(BatchReplica), C.c_int, C.c_float, C.c_int, C.c_int]),
    "pd_batch_destroy": (C.c_int, [_p]),
    "pd_batch_count": (C.c_int, [_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "pd_batch_set_lanes": (C.c_int, [_p, C.c_int]),
    "pd_batch_update": (C.c_int, [_p, _fp, _fp, _fp, _p]),
    "pd_batch_forces": (C.c_int, [_p, _fp, _fp, _fp, _fp, _fp, _fp, _fp, C.c_int, _p]),
    "pd_batch_status": (C.c_int, [_p, C.POINTER(EllStats)]),
    "pd_batch_rows": (C.c_int, [_p, C.POINTER(_p), C.POINTER(_p), C.POINTER(_p)]),
    "pd_batch_bind": (C.c_int, [_p, C.POINTER(MDState)]),
    "pd_batch_evaluate": (C.c_int, [_p, C.c_int, _p]),
    "pd_batch_step": (C.c_int, [_p, C.c_int, C.c_float, C.c_int, _p]),
    "pd_batch_set_coulomb": (C.c_int, [_p, C.POINTER(BatchCoulomb)]),
    "pd_batch_set_mesh": (C.c_int, [_p, C.c_int, C.c_int, C.c_double, C.c_double, C.POINTER(C.c_int)]),
    "pd_batch_set_spread_tile": (C.c_int, [_p, C.c_int, C.c_int]),
    "pd_batch_mesh_info": (C.c_int, [_p, C.POINTER(C.c_int), C.POINTER(C.c_longlong), C.POINTER(C.c_longlong),
                                     C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "pd_ewald_oracle": (C.c_int, [C.c_int, _fp, C.POINTER(C.c_double), C.c_double, C.c_double, C.c_double, C.c_int,
                                  _fp, C.POINTER(C.c_double)]),
    "pd_gsd_open": (C.c_int, [C.c_char_p, C.c_int, C.c_char_p, C.c_char_p, C.c_uint32, C.POINTER(_p)]),
    "pd_gsd_close": (C.c_int, [_p]),
    "pd_gsd_write_chunk": (C.c_int, [_p, C.c_char_p, C.c_int, C.c_uint64, C.c_uint32, _p]),
    "pd_gsd_end_frame": (C.c_int, [_p]),
    "pd_gsd_flush": (C.c_int, [_p]),
    "pd_gsd_nframes": (C.c_uint64, [_p]),
    "pd_gsd_header": (C.c_int, [_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.c_char_p, C.c_char_p]),
    "pd_gsd_find_chunk": (C.c_int, [_p, C.c_uint64, C.c_char_p, C.POINTER(GsdIndexEntry), C.POINTER(C.c_int)]),
    "pd_gsd_read_chunk": (C.c_int, [_p, C.POINTER(GsdIndexEntry), _p, C.c_uint64]),
    "pd_gsd_frame_entries": (C.c_int, [_p, C.c_uint64, C.POINTER(GsdIndexEntry), C.c_int, C.POINTER(C.c_int)]),
    "pd_gsd_name": (C.c_int, [_p, C.c_int, C.c_char_p, C.c_int]),
    "pd_snapshot_layout": (C.c_int, [C.POINTER(SnapshotSrc), C.POINTER(SnapshotOffsets)]),
    "pd_snapshot_pack": (C.c_int, [C.POINTER(SnapshotSrc), _fp, C.c_uint64, _p]),
}

EXPORTED = tuple(_SIGS)

_lib = None


class NativeError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where}: {msg} (status {code})")
        self.code = code


def lib() -> C.CDLL:
    """The loaded library (raises if libpdb200.so was not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python {HERE / '_build.py'}` (there is no CPU fallback)")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(code: int, where: str) -> None:
    if code != PD_OK:
        L = lib()
        msg = L.pd_last_error().decode() or L.pd_strerror(code).decode()
        raise NativeError(code, where, msg)


def call(name: str, *args) -> int:
    f = getattr(lib(), name)
    code = f(*args)
    if f.restype is C.c_int:
        check(code, name)
    return code


def dbl3(v) -> C.Array:
    return (C.c_double * 3)(*[float(a) for a in v])
