"""moleculardynamics_b200 -- B200-native moldyn force / neighbour / integrator path.

A thin Python binding over the C ABI in ``include/moldyn_b200.h`` (library:
``libmoldyn_b200.so`` next to this file).  Class and method names follow the
reference's C++ API (``moldyn::System``, ``CellList``, ``VerletList``,
``LennardJones``, ``VelocityVerlet``, ``LangevinBAOAB``, ``NoseHooverChain``) so
code and tests read like the reference's own.

There is no CPU fallback: importing works anywhere, but constructing a
``Context`` raises unless the CUDA library is built and a GPU is present.
Arrays cross the boundary in the caller's atom order as float64 numpy arrays of
shape (N, 3) (positions, velocities, forces) or (N,) (masses, charges).
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmoldyn_b200.so")

# C ABI constants (include/moldyn_b200.h)
MD_OK = 0
MD_ERR_INVALID_ARGUMENT = -1
MD_ERR_RUNTIME = -2
MD_ERR_CUDA = -3
MD_ERR_OUT_OF_MEMORY = -4
MD_ERR_DEVICE = -5
FIELD_X, FIELD_Y, FIELD_Z, FIELD_VX, FIELD_VY, FIELD_VZ = range(6)
FIELD_FX, FIELD_FY, FIELD_FZ, FIELD_MASS, FIELD_CHARGE = range(6, 11)
PRECISION_FP64, PRECISION_MIXED = 0, 1
MD_KERNEL_LJ_FORCE, MD_KERNEL_NEIGHBOR, MD_KERNEL_INTEGRATE = 0, 1, 2
MD_KERNEL_EWALD_REAL, MD_KERNEL_EWALD_RECIP = 3, 4


class Truncation:
    """forcefield/lennard_jones.hpp:11"""
    Truncated = 0
    LinearForceShift = 1


class MDError(RuntimeError):
    code = 0


class InvalidArgument(MDError, ValueError):
    """The reference's std::invalid_argument."""


class DeviceError(MDError):
    """A device status bit (neighbour overflow, constraint divergence, ...)."""


_ERRORS = {MD_ERR_INVALID_ARGUMENT: InvalidArgument, MD_ERR_RUNTIME: MDError,
           MD_ERR_CUDA: MDError, MD_ERR_OUT_OF_MEMORY: MemoryError, MD_ERR_DEVICE: DeviceError}

_lib = None
_vp = C.c_void_p
_d = C.POINTER(C.c_double)
_i64p = C.POINTER(C.c_int64)


def library_path() -> str:
    return LIB_PATH


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is not built; run `make -C moleculardynamics_b200/csrc` "
            "(or __graft_entry__.build()).  There is no CPU fallback.")
    L = C.CDLL(LIB_PATH)
    sig = {
        "md_last_error": (C.c_char_p, []),
        "md_abi_version": (C.c_int, []),
        "md_context_create": (C.c_int, [C.c_int, C.POINTER(_vp)]),
        "md_context_destroy": (C.c_int, [_vp]),
        "md_context_synchronize": (C.c_int, [_vp]),
        "md_context_status": (C.c_int, [_vp, C.POINTER(C.c_uint32), C.c_int]),
        "md_context_launch_count": (C.c_int, [_vp, _i64p]),
        "md_context_graph_captures": (C.c_int, [_vp, _i64p]),
        "md_context_set_timing": (C.c_int, [_vp, C.c_int]),
        "md_context_set_graphs": (C.c_int, [_vp, C.c_int]),
        "md_context_device_name": (C.c_int, [_vp, C.c_char_p, C.c_int]),
        "md_context_kernel_time": (C.c_int, [_vp, C.c_int, C.c_int, _d, _i64p]),
        "md_context_span_begin": (C.c_int, [_vp]),
        "md_context_span_end": (C.c_int, [_vp, _d]),
        "md_host_alloc": (C.c_void_p, [C.c_size_t]),
        "md_host_free": (C.c_int, [C.c_void_p]),
        "md_system_create": (C.c_int, [_vp, C.c_int64, _d, C.POINTER(_vp)]),
        "md_system_destroy": (C.c_int, [_vp]),
        "md_system_size": (C.c_int64, [_vp]),
        "md_system_box": (C.c_int, [_vp, _d]),
        "md_system_set": (C.c_int, [_vp, C.c_int, _d]),
        "md_system_get": (C.c_int, [_vp, C.c_int, _d]),
        "md_system_set_fields": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_int), C.POINTER(_d)]),
        "md_system_get_fields": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_int), C.POINTER(_d)]),
        "md_system_set_molecule_ids": (C.c_int, [_vp, _i64p]),
        "md_system_get_molecule_ids": (C.c_int, [_vp, _i64p]),
        "md_system_zero_forces": (C.c_int, [_vp]),
        "md_system_kinetic_energy": (C.c_int, [_vp, _d]),
        "md_system_total_momentum": (C.c_int, [_vp, _d]),
        "md_system_remove_com_motion": (C.c_int, [_vp]),
        "md_system_rescale_temperature": (C.c_int, [_vp, C.c_int64, C.c_double]),
        "md_system_last_energy": (C.c_int, [_vp, _d, _d]),
        "md_cells_create": (C.c_int, [_vp, _d, C.c_double, C.POINTER(_vp)]),
        "md_cells_destroy": (C.c_int, [_vp]),
        "md_cells_dims": (C.c_int, [_vp, C.POINTER(C.c_int)]),
        "md_cells_usable": (C.c_int, [_vp]),
        "md_cells_build": (C.c_int, [_vp, _vp]),
        "md_cells_pairs": (C.c_int, [_vp, _i64p, _i64p, C.c_int64, _i64p]),
        "md_verlet_create": (C.c_int, [_vp, _d, C.c_double, C.c_double, C.POINTER(_vp)]),
        "md_verlet_destroy": (C.c_int, [_vp]),
        "md_verlet_build": (C.c_int, [_vp, _vp]),
        "md_verlet_needs_rebuild": (C.c_int, [_vp, _vp, C.POINTER(C.c_int)]),
        "md_verlet_rebuild_if_needed": (C.c_int, [_vp, _vp, C.POINTER(C.c_int)]),
        "md_verlet_rebuild_count": (C.c_int, [_vp, _i64p]),
        "md_verlet_pairs": (C.c_int, [_vp, _i64p, _i64p, C.c_int64, _i64p]),
        "md_verlet_set_criterion": (C.c_int, [_vp, C.c_int]),
        "md_verlet_set_cell_width": (C.c_int, [_vp, C.c_double]),
        "md_verlet_cells_per_side": (C.c_int, [_vp, C.POINTER(C.c_int)]),
        "md_verlet_displacements": (C.c_int, [_vp, _vp, _d, _d]),
        "md_verlet_set_capacity": (C.c_int, [_vp, C.c_int, C.c_int]),
        "md_lj_create": (C.c_int, [C.c_double, C.c_double, C.c_double, C.c_int, C.c_int,
                                   C.POINTER(_vp)]),
        "md_lj_destroy": (C.c_int, [_vp]),
        "md_lj_energy_virial": (C.c_int, [_vp, _vp, _d, _d]),
        "md_lj_forces": (C.c_int, [_vp, _vp, _d, _d]),
        "md_lj_forces_cells": (C.c_int, [_vp, _vp, _vp, _d, _d]),
        "md_lj_forces_verlet": (C.c_int, [_vp, _vp, _vp, _d, _d]),
        "md_lj_lrc": (C.c_int, [_vp, C.c_int64, _d, _d, _d]),
        "md_lj_set_threads_per_atom": (C.c_int, [C.c_int]),
        "md_lj_set_unroll": (C.c_int, [C.c_int]),
        "md_lj_set_launch": (C.c_int, [_vp, C.c_int, C.c_int]),
        "md_lj_set_halo": (C.c_int, [_vp, C.c_int]),
        "md_lj_set_tile_threads": (C.c_int, [_vp, C.c_int]),
        "md_thermo_csv_open": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_int,
                                        C.c_int64, C.c_int64, C.POINTER(_vp)]),
        "md_thermo_csv_append": (C.c_int, [_vp, _vp, C.c_int64, _d, C.c_int64, C.c_int64,
                                          C.c_double, C.c_char_p, C.c_int64, _d, C.c_int64]),
        "md_thermo_csv_close": (C.c_int, [_vp]),
        "md_xyz_append": (C.c_int, [C.c_char_p, _vp, C.c_int64, C.c_double, C.c_char_p,
                                   C.c_char_p, C.c_char_p, C.c_char_p]),
        "md_checkpoint_save": (C.c_int, [_vp, _vp, C.c_char_p]),
        "md_checkpoint_load": (C.c_int, [_vp, C.c_char_p, C.POINTER(_vp), _vp]),
        "md_rdf_create": (C.c_int, [_vp, C.c_double, C.c_int64, C.POINTER(_vp)]),
        "md_rdf_destroy": (C.c_int, [_vp]),
        "md_rdf_accumulate": (C.c_int, [_vp, _vp]),
        "md_rdf_accumulate_subset": (C.c_int, [_vp, _vp, C.c_int64, C.c_int64]),
        "md_rdf_histogram": (C.c_int, [_vp, _d]),
        "md_rdf_g": (C.c_int, [_vp, _d]),
        "md_rdf_bin_centres": (C.c_int, [_vp, _d]),
        "md_rdf_frames": (C.c_int, [_vp, C.POINTER(C.c_int64)]),
        "md_msd_create": (C.c_int, [_vp, C.c_int64, C.c_int64, C.POINTER(_vp)]),
        "md_msd_destroy": (C.c_int, [_vp]),
        "md_msd_push": (C.c_int, [_vp, _vp]),
        "md_msd_values": (C.c_int, [_vp, _d]),
        "md_msd_diffusion": (C.c_int, [_vp, C.c_double, C.c_int64, C.c_int64, _d]),
        "md_vacf_create": (C.c_int, [_vp, C.c_int64, C.c_int64, C.POINTER(_vp)]),
        "md_vacf_destroy": (C.c_int, [_vp]),
        "md_vacf_push": (C.c_int, [_vp, _vp]),
        "md_vacf_values": (C.c_int, [_vp, C.c_int, _d]),
        "md_vacf_diffusion": (C.c_int, [_vp, C.c_double, _d]),
        "md_verlet_halo_tiles": (C.c_int, [_vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
        "md_verlet_set_halo": (C.c_int, [_vp, C.c_int]),
        "md_integrator_create_vv": (C.c_int, [C.c_double, C.POINTER(_vp)]),
        "md_integrator_create_baoab": (C.c_int, [C.c_double, C.c_double, C.c_double, C.c_uint64,
                                                 C.POINTER(_vp)]),
        "md_integrator_create_nhc": (C.c_int, [C.c_double, C.c_double, C.c_double, C.c_int,
                                               C.c_int64, C.POINTER(_vp)]),
        "md_integrator_destroy": (C.c_int, [_vp]),
        "md_integrator_pre_force": (C.c_int, [_vp, _vp]),
        "md_integrator_post_force": (C.c_int, [_vp, _vp]),
        "md_integrator_conserved": (C.c_int, [_vp, _d]),
        "md_integrator_set_noise": (C.c_int, [_vp, _d, C.c_int64]),
        "md_run_lj": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int64, _d]),
        "md_fcc_lattice": (C.c_int, [C.c_int, C.c_double, C.c_double, C.c_uint64] + [_d] * 8),
        "md_coulomb_prefactor": (C.c_double, []),
        "md_rng_normals": (C.c_int64, [C.c_uint64, C.c_int64, _d]),
        "md_lj_forces_static": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, _d,
                                          C.c_double, C.c_double, C.c_double, C.c_int,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p]),
        "md_ewald_create": (C.c_int, [_vp, C.c_double, C.c_int, C.c_double, C.POINTER(_vp)]),
        "md_ewald_destroy": (C.c_int, [_vp]),
        "md_ewald_set_skin": (C.c_int, [_vp, C.c_double]),
        "md_ewald_compute": (C.c_int, [_vp, _vp, C.c_int, _d, _d]),
        "md_ewald_alpha": (C.c_int, [_vp, _d]),
        "md_ewald_kvector_count": (C.c_int, [_vp, C.POINTER(C.c_int)]),
        "md_ewald_set_pme": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int]),
        "md_ewald_set_precision": (C.c_int, [_vp, C.c_int]),
        "md_ewald_pme_grid": (C.c_int, [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "md_spce_create": (C.c_int, [_vp, C.c_double, C.c_double, C.c_double, C.c_int, C.c_double,
                                     C.POINTER(_vp)]),
        "md_spce_compute": (C.c_int, [_vp, _vp, C.c_int, _d, _d]),
        "md_spce_set_lj_truncation": (C.c_int, [_vp, C.c_int]),
        "md_rigid_set_settle": (C.c_int, [_vp, C.c_int]),
        "md_rigid_create": (C.c_int, [C.c_double, C.c_double, C.c_double, C.c_int,
                                      C.POINTER(_vp)]),
        "md_rigid_destroy": (C.c_int, [_vp]),
        "md_rigid_distances": (C.c_int, [_vp, _d, _d]),
        "md_rigid_degrees_of_freedom": (C.c_int64, [C.c_int64, C.c_int]),
        "md_rigid_constrain_positions": (C.c_int, [_vp, _vp, _d, _d, _d, C.POINTER(C.c_int)]),
        "md_rigid_constrain_velocities": (C.c_int, [_vp, _vp, C.POINTER(C.c_int)]),
        "md_integrator_create_rattle": (C.c_int, [C.c_double, _vp, C.POINTER(_vp)]),
        "md_integrator_create_rattle_nhc": (C.c_int, [C.c_double, _vp, C.c_double, C.c_double,
                                                      C.c_int, C.c_int64, C.POINTER(_vp)]),
        "md_integrator_iterations": (C.c_int, [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "md_run_spce": (C.c_int, [_vp, _vp, _vp, C.c_int64, _d]),
        "md_water_rdf_run": (C.c_int, [_vp, _vp, _vp, _vp, C.c_double, C.c_int64, C.c_int64,
                                       C.c_int64, C.c_int64, C.c_int64, _d]),
        "md_batch_create": (C.c_int, [C.POINTER(_vp)]),
        "md_batch_destroy": (C.c_int, [_vp]),
        "md_batch_add": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.POINTER(C.c_int)]),
        "md_batch_size": (C.c_int, [_vp]),
        "md_batch_set_batched": (C.c_int, [_vp, C.c_int]),
        "md_batch_run": (C.c_int, [_vp, C.c_int64, _d]),
        "md_adjoint_create": (C.c_int, [_vp, C.POINTER(_vp)]),
        "md_adjoint_destroy": (C.c_int, [_vp]),
        "md_adjoint_forward": (C.c_int, [_vp, _vp, _vp, C.c_double, C.c_int64, C.c_int,
                                         C.c_double, _d]),
        "md_adjoint_backward": (C.c_int, [_vp, _d, _d, _d, _d]),
        "md_lj_hvp": (C.c_int, [_vp, _vp, _vp, _d, _d, _d]),
        "md_ewald_charge_gradient": (C.c_int, [_vp, _vp, _d]),
        "md_ewald_real_hvp": (C.c_int, [_vp, _vp, _d, _d]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def lib():
    return _load()


def _check(rc):
    if rc != MD_OK:
        msg = _load().md_last_error().decode(errors="replace")
        exc = _ERRORS.get(rc, MDError)(f"[{rc}] {msg}")
        if isinstance(exc, MDError):
            exc.code = rc
        raise exc
    return rc


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _ptr(a):
    return a.ctypes.data_as(_d)


# ---------------------------------------------------------------- context
_default_ctx = None


class Context:
    """One device, one stream, one device status word."""

    def __init__(self, device: int = 0):
        h = _vp()
        _check(_load().md_context_create(device, C.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    def synchronize(self):
        _check(lib().md_context_synchronize(self._h))

    def status(self, clear=False):
        st = C.c_uint32()
        _check(lib().md_context_status(self._h, C.byref(st), 1 if clear else 0))
        return st.value

    def launch_count(self):
        c = C.c_int64()
        _check(lib().md_context_launch_count(self._h, C.byref(c)))
        return c.value

    def graph_captures(self):
        """Step graphs fused loops have captured on this context."""
        c = C.c_int64()
        _check(lib().md_context_graph_captures(self._h, C.byref(c)))
        return c.value

    def device_name(self) -> str:
        buf = C.create_string_buffer(256)
        _check(lib().md_context_device_name(self._h, buf, 256))
        return buf.value.decode()

    def set_graphs(self, enable: bool):
        """Fused loops replay one captured CUDA graph per step (default) or launch
        every kernel from the host; results are identical."""
        _check(lib().md_context_set_graphs(self._h, 1 if enable else 0))

    def close(self):
        if getattr(self, "_h", None):
            lib().md_context_destroy(self._h)
            self._h = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


def require_gpu() -> None:
    """Raises unless the CUDA library loads and a device context can be created."""
    default_context()


# ---------------------------------------------------------------- system
class System:
    """core/system.hpp:11-60 on the device.  Arrays in the caller's atom order."""

    def __init__(self, n, box, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        box = _f64(box).reshape(3)
        h = _vp()
        _check(lib().md_system_create(self.ctx.handle, int(n), _ptr(box), C.byref(h)))
        self._h = h
        self.n = int(n)
        self.box = box.copy()

    @classmethod
    def _adopt(cls, h, ctx):
        """Wrap a system handle created by the library (checkpoint_load)."""
        s = cls.__new__(cls)
        s.ctx = ctx
        s._h = h
        s.n = int(lib().md_system_size(h))
        box = np.zeros(3)
        _check(lib().md_system_box(h, _ptr(box)))
        s.box = box
        return s

    @classmethod
    def from_arrays(cls, pos, box, vel=None, mass=None, charge=None, mol=None, ctx=None):
        pos = _f64(pos).reshape(-1, 3)
        s = cls(pos.shape[0], box, ctx)
        s.positions = pos
        if vel is not None:
            s.velocities = vel
        if mass is not None:
            s.masses = mass
        if charge is not None:
            s.charges = charge
        if mol is not None:
            s.molecule_ids = mol
        return s

    @property
    def handle(self):
        return self._h

    def size(self):
        return self.n

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.md_system_destroy(self._h)
            self._h = None

    def _get3(self, f0):
        out = np.empty((3, self.n))
        for k in range(3):
            _check(lib().md_system_get(self._h, f0 + k, _ptr(out[k])))
        return out.T.copy()

    def _set3(self, f0, a):
        a = _f64(a).reshape(self.n, 3)
        for k in range(3):
            col = np.ascontiguousarray(a[:, k])
            _check(lib().md_system_set(self._h, f0 + k, _ptr(col)))

    def _get1(self, f):
        out = np.empty(self.n)
        _check(lib().md_system_get(self._h, f, _ptr(out)))
        return out

    def _set1(self, f, a):
        a = _f64(a).reshape(self.n)
        _check(lib().md_system_set(self._h, f, _ptr(a)))

    positions = property(lambda s: s._get3(FIELD_X), lambda s, a: s._set3(FIELD_X, a))
    velocities = property(lambda s: s._get3(FIELD_VX), lambda s, a: s._set3(FIELD_VX, a))
    forces = property(lambda s: s._get3(FIELD_FX), lambda s, a: s._set3(FIELD_FX, a))
    masses = property(lambda s: s._get1(FIELD_MASS), lambda s, a: s._set1(FIELD_MASS, a))
    charges = property(lambda s: s._get1(FIELD_CHARGE), lambda s, a: s._set1(FIELD_CHARGE, a))

    @property
    def molecule_ids(self):
        out = np.empty(self.n, dtype=np.int64)
        _check(lib().md_system_get_molecule_ids(self._h, out.ctypes.data_as(_i64p)))
        return out

    @molecule_ids.setter
    def molecule_ids(self, ids):
        ids = np.ascontiguousarray(ids, dtype=np.int64).reshape(self.n)
        _check(lib().md_system_set_molecule_ids(self._h, ids.ctypes.data_as(_i64p)))

    def zero_forces(self):
        _check(lib().md_system_zero_forces(self._h))

    def kinetic_energy(self):
        v = C.c_double()
        _check(lib().md_system_kinetic_energy(self._h, C.byref(v)))
        return v.value

    def temperature(self, dof):
        """system.cpp:133-135"""
        return 2.0 * self.kinetic_energy() / float(dof)

    def total_momentum(self):
        p = np.zeros(3)
        _check(lib().md_system_total_momentum(self._h, _ptr(p)))
        return p

    def remove_center_of_mass_motion(self):
        _check(lib().md_system_remove_com_motion(self._h))

    def rescale_temperature(self, dof, target):
        """v *= sqrt(target / T), T = 2 KE / dof, if T > 0; on the device,
        asynchronous (apps/water_rdf.cpp:186-195)."""
        _check(lib().md_system_rescale_temperature(self._h, int(dof), float(target)))

    def volume(self):
        return float(self.box[0] * self.box[1] * self.box[2])

    def last_energy_virial(self):
        e = C.c_double()
        w = C.c_double()
        _check(lib().md_system_last_energy(self._h, C.byref(e), C.byref(w)))
        return e.value, w.value


# ---------------------------------------------------------------- neighbours
def _pairs(fn, h):
    cnt = C.c_int64()
    _check(fn(h, None, None, 0, C.byref(cnt)))
    n = cnt.value
    pi = np.zeros(max(n, 1), np.int64)
    pj = np.zeros(max(n, 1), np.int64)
    _check(fn(h, pi.ctypes.data_as(_i64p), pj.ctypes.data_as(_i64p), n, C.byref(cnt)))
    return np.stack([pi[:n], pj[:n]], 1)


class CellList:
    """neighbor/cell_list.hpp:26-37"""

    def __init__(self, box, cutoff, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        h = _vp()
        _check(lib().md_cells_create(self.ctx.handle, _ptr(_f64(box).reshape(3)), float(cutoff),
                                     C.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.md_cells_destroy(self._h)
            self._h = None

    def build(self, sys: System):
        _check(lib().md_cells_build(self._h, sys.handle))

    def cells_per_side(self, dim):
        d = (C.c_int * 3)()
        _check(lib().md_cells_dims(self._h, d))
        return d[dim]

    def usable(self):
        return bool(lib().md_cells_usable(self._h))

    def pairs(self):
        """Candidate pairs (i<j) of forEachPair, as an (M, 2) array (any order)."""
        return _pairs(lib().md_cells_pairs, self._h)


class VerletList:
    """neighbor/verlet_list.hpp:26-39"""

    def __init__(self, box, cutoff, skin, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        h = _vp()
        _check(lib().md_verlet_create(self.ctx.handle, _ptr(_f64(box).reshape(3)), float(cutoff),
                                      float(skin), C.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.md_verlet_destroy(self._h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def build(self, sys: System):
        _check(lib().md_verlet_build(self._h, sys.handle))

    def needs_rebuild(self, sys: System) -> bool:
        f = C.c_int()
        _check(lib().md_verlet_needs_rebuild(self._h, sys.handle, C.byref(f)))
        return bool(f.value)

    def rebuild_if_needed(self, sys: System) -> bool:
        f = C.c_int()
        _check(lib().md_verlet_rebuild_if_needed(self._h, sys.handle, C.byref(f)))
        return bool(f.value)

    def rebuild_count(self) -> int:
        c = C.c_int64()
        _check(lib().md_verlet_rebuild_count(self._h, C.byref(c)))
        return c.value

    def pairs(self):
        """Pairs (i<j) held in the list, sorted by (i, j)."""
        return _pairs(lib().md_verlet_pairs, self._h)

    def set_criterion(self, criterion: int):
        _check(lib().md_verlet_set_criterion(self._h, int(criterion)))

    def set_cell_width(self, width: float):
        """Cells at least `width` wide (>= cutoff + skin; 0: the reference's rule).
        The pair set is unchanged; the list must be built again."""
        _check(lib().md_verlet_set_cell_width(self._h, float(width)))

    def cells_per_side(self):
        d = (C.c_int * 3)()
        _check(lib().md_verlet_cells_per_side(self._h, d))
        return tuple(d)

    def set_capacity(self, capacity: int, fixed: bool = False):
        """Neighbours per atom the rows hold; host builds grow it on overflow
        unless fixed.  The list must be built again."""
        _check(lib().md_verlet_set_capacity(self._h, int(capacity), 1 if fixed else 0))

    def set_halo(self, on=True):
        """Keep halo tiles for the mixed-precision force kernel (built now and at
        every rebuild), or drop them.  Fused runs of large systems turn them on."""
        _check(lib().md_verlet_set_halo(self._h, 1 if on else 0))

    def halo_tiles(self):
        """(staged, total) halo tiles of this list ((0, 0) without tiles)."""
        a, b = C.c_int64(), C.c_int64()
        _check(lib().md_verlet_halo_tiles(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def displacements(self, sys: System):
        a = C.c_double()
        b = C.c_double()
        _check(lib().md_verlet_displacements(self._h, sys.handle, C.byref(a), C.byref(b)))
        return a.value, b.value


# ---------------------------------------------------------------- forces
class LennardJones:
    """forcefield/lennard_jones.hpp:24-100.  Energy-returning calls give
    (energy, virial) like EnergyVirial."""

    def __init__(self, sigma, epsilon, cutoff, truncation=Truncation.Truncated,
                 precision=PRECISION_FP64):
        h = _vp()
        _check(lib().md_lj_create(float(sigma), float(epsilon), float(cutoff), int(truncation),
                                  int(precision), C.byref(h)))
        self._h = h
        self.sigma, self.epsilon, self.cutoff = float(sigma), float(epsilon), float(cutoff)
        self.truncation = int(truncation)
        self.precision = int(precision)

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.md_lj_destroy(self._h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def _ev(self, fn, *args):
        e = C.c_double()
        w = C.c_double()
        _check(fn(self._h, *args, C.byref(e), C.byref(w)))
        return e.value, w.value

    def compute_energy_virial(self, sys: System):
        return self._ev(lib().md_lj_energy_virial, sys.handle)

    def compute_forces(self, sys: System, source=None):
        """Brute force (source None), a CellList or a VerletList."""
        if source is None:
            return self._ev(lib().md_lj_forces, sys.handle)
        if isinstance(source, CellList):
            return self._ev(lib().md_lj_forces_cells, sys.handle, source._h)
        return self._ev(lib().md_lj_forces_verlet, sys.handle, source.handle)

    def set_launch(self, tpa=0, unroll=0):
        """Threads per atom and gathers in flight of this object's Verlet force
        kernel (0 = library default); see moleculardynamics_b200.autotune."""
        _check(lib().md_lj_set_launch(self._h, int(tpa), int(unroll)))

    def set_tile_threads(self, tpa: int):
        """Threads per atom of the mixed tile kernel (2, 4 or 8; 0: the default)."""
        _check(lib().md_lj_set_tile_threads(self._h, int(tpa)))

    def set_halo(self, on=True):
        """Mixed precision: read neighbours through shared-memory halo tiles (the
        default) or gather them through the int32 rows; forces are identical."""
        _check(lib().md_lj_set_halo(self._h, 1 if on else 0))

    def hessian_vector_product(self, sys: System, verlet: VerletList, u):
        """(dF/dx)^T u for a per-atom field u (N, 3), and (u . dF/d epsilon,
        u . dF/d sigma).  FP64 over a built Verlet list."""
        u = _f64(u).reshape(sys.n, 3)
        out = np.zeros((sys.n, 3))
        th = np.zeros(2)
        _check(lib().md_lj_hvp(self._h, sys.handle, verlet.handle, _ptr(u), _ptr(out), _ptr(th)))
        return out, th

    def long_range_correction(self, sys: System):
        u = C.c_double()
        _check(lib().md_lj_lrc(self._h, sys.n, _ptr(_f64(sys.box)), C.byref(u), None))
        return u.value

    def long_range_correction_pressure(self, sys: System):
        p = C.c_double()
        _check(lib().md_lj_lrc(self._h, sys.n, _ptr(_f64(sys.box)), None, C.byref(p)))
        return p.value


def set_threads_per_atom(tpa: int):
    _check(lib().md_lj_set_threads_per_atom(int(tpa)))


def set_unroll(unroll: int):
    _check(lib().md_lj_set_unroll(int(unroll)))


def coulomb_prefactor() -> float:
    """e^2/(4 pi eps0 kB) in K*Angstrom/e^2 (forcefield/ewald.cpp:17-21)."""
    return lib().md_coulomb_prefactor()


class EwaldTerms(dict):
    """forcefield/ewald.hpp:24-31 (real, reciprocal, self, intra) as a dict."""

    def total(self):
        return self["real"] + self["reciprocal"] + self["self"] + self["intra"]


def fft_size(at_least):
    """The smallest n >= at_least whose prime factors are 2, 3, 5 and 7 (sizes
    the 3-D FFTs of PME handle fastest)."""
    n = max(1, math.ceil(at_least))
    while True:
        m = n
        for p in (2, 3, 5, 7):
            while m % p == 0:
                m //= p
        if m == 1:
            return n
        n += 1


class _PmeMixin:
    def set_pme(self, grid, order=6):
        """Smooth PME (Essmann et al. 1995) for the reciprocal term instead of
        the k-vector sums: grid is (kx, ky, kz) or one size for all axes; None
        or 0 returns to the k-vector sums."""
        if not grid:
            k = (0, 0, 0)
        elif np.isscalar(grid):
            k = (int(grid),) * 3
        else:
            k = tuple(int(v) for v in grid)
        _check(lib().md_ewald_set_pme(self._h, *k, int(order)))

    def set_pme_spacing(self, box, spacing=1.0, order=6):
        """PME with FFT-friendly grid sizes of at most `spacing` per grid cell."""
        self.set_pme([fft_size(math.ceil(float(L) / spacing)) for L in np.asarray(box)], order)

    def set_precision(self, precision):
        """PRECISION_FP64 (default) or PRECISION_MIXED: FP32 real-space pair
        terms with FP64 displacements and sums."""
        _check(lib().md_ewald_set_precision(self._h, int(precision)))

    def pme_grid(self):
        """((kx, ky, kz), order), or ((0, 0, 0), 0) with the k-vector sums."""
        k = (C.c_int * 3)()
        o = C.c_int()
        _check(lib().md_ewald_pme_grid(self._h, k, C.byref(o)))
        return tuple(k), o.value


class Ewald(_PmeMixin):
    """forcefield/ewald.hpp:49-68 plus alpha (<= 0: the reference's 5.6 / min L)."""

    def __init__(self, cutoff, kmax, alpha=0.0, ctx: Context | None = None, skin=1.0):
        self.ctx = ctx or default_context()
        h = _vp()
        _check(lib().md_ewald_create(self.ctx.handle, float(cutoff), int(kmax), float(alpha),
                                     C.byref(h)))
        self._h = h
        if skin != 1.0:
            _check(lib().md_ewald_set_skin(h, float(skin)))

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.md_ewald_destroy(self._h)
            self._h = None

    def _run(self, sys, mode):
        t = np.zeros(4)
        w = C.c_double()
        _check(lib().md_ewald_compute(self._h, sys.handle, mode, _ptr(t), C.byref(w)))
        self.last_virial = w.value
        return EwaldTerms(real=t[0], reciprocal=t[1], self=t[2], intra=t[3])

    def compute_energies(self, sys):
        return self._run(sys, 0)

    def compute_forces(self, sys):
        return self._run(sys, 1)

    def accumulate_forces(self, sys):
        return self._run(sys, 2)

    def charge_gradient(self, sys):
        """dE/dq_i of the Coulomb energy (real + reciprocal + self + intramolecular)."""
        out = np.zeros(sys.n)
        _check(lib().md_ewald_charge_gradient(self._h, sys.handle, _ptr(out)))
        return out

    def real_space_hvp(self, sys, u):
        """(dF_real/dx)^T u for a per-atom field u (N, 3)."""
        u = _f64(u).reshape(sys.n, 3)
        out = np.zeros((sys.n, 3))
        _check(lib().md_ewald_real_hvp(self._h, sys.handle, _ptr(u), _ptr(out)))
        return out

    def alpha(self):
        a = C.c_double()
        _check(lib().md_ewald_alpha(self._h, C.byref(a)))
        return a.value


class SpceParameters:
    """forcefield/spce.hpp:16-24"""
    qH = 0.42380
    sigmaO = 3.16555789
    epsilonO = 78.19743111
    rOH = 1.0
    angleHOH = 109.47
    massOxygen = 15.9994
    massHydrogen = 1.008


class SpceForceField(_PmeMixin):
    """forcefield/spce_forcefield.hpp:25-41 (+ alpha)."""

    def __init__(self, cutoff=10.0, kmax=5, alpha=0.0, params=SpceParameters,
                 ctx: Context | None = None, skin=1.0, truncation=Truncation.Truncated):
        """truncation applies to the O-O Lennard-Jones term: Truncated (the
        reference's, with the analytic tail) or LinearForceShift (no tail)."""
        self.ctx = ctx or default_context()
        h = _vp()
        _check(lib().md_spce_create(self.ctx.handle, params.sigmaO, params.epsilonO,
                                    float(cutoff), int(kmax), float(alpha), C.byref(h)))
        self._h = h
        if skin != 1.0:
            _check(lib().md_ewald_set_skin(h, float(skin)))
        if truncation != Truncation.Truncated:
            _check(lib().md_spce_set_lj_truncation(h, int(truncation)))
        self.parts = None

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.md_ewald_destroy(self._h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def _run(self, sys, forces):
        e = C.c_double()
        parts = np.zeros(8)
        _check(lib().md_spce_compute(self._h, sys.handle, 1 if forces else 0, C.byref(e),
                                     _ptr(parts)))
        self.parts = dict(disp=parts[0], lrc=parts[1], real=parts[2], reciprocal=parts[3],
                          self=parts[4], intra=parts[5], virial=parts[6], total=parts[7])
        return e.value

    def compute_forces(self, sys):
        return self._run(sys, True)

    def compute_energy(self, sys):
        return self._run(sys, False)


def build_spce_system(pos, types, box, params=SpceParameters, ctx=None):
    """forcefield/spce.cpp:8-40: O,H,H triples; molecule id = index / 3."""
    types = list(types)
    n = len(types)
    if n == 0 or n % 3 != 0:
        raise InvalidArgument("buildSpceSystem: atom count must be a positive multiple of 3")
    q = np.array([-2.0 * params.qH if t == "O" else params.qH for t in types])
    m = np.array([params.massOxygen if t == "O" else params.massHydrogen for t in types])
    for t in types:
        if t not in ("O", "H"):
            raise InvalidArgument(f"buildSpceSystem: unrecognised atom type '{t}'")
    return System.from_arrays(pos, box, mass=m, charge=q, mol=np.arange(n) // 3, ctx=ctx)


# ---------------------------------------------------------------- integrators
class _Integrator:
    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.md_integrator_destroy(self._h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def step(self, sys: System, compute_forces):
        """template<class ForceFn> step(System&, ForceFn&&): compute_forces(sys)
        is called exactly once, between the pre- and post-force halves."""
        _check(lib().md_integrator_pre_force(self._h, sys.handle))
        result = compute_forces(sys)
        _check(lib().md_integrator_post_force(self._h, sys.handle))
        return result

    def run(self, sys: System, verlet: VerletList, lj: LennardJones, steps: int, thermo=False):
        """Fused device loop with the moldyn_run ForceFn (rebuildIfNeeded + LJ).
        Returns a (steps, 4) array [energy, virial, kinetic, conserved] if thermo."""
        out = np.zeros((steps, 4)) if thermo and steps > 0 else None
        _check(lib().md_run_lj(self._h, sys.handle, verlet.handle, lj.handle, int(steps),
                               _ptr(out) if out is not None else None))
        return out

    def conserved_quantity_contribution(self):
        v = C.c_double()
        _check(lib().md_integrator_conserved(self._h, C.byref(v)))
        return v.value


class VelocityVerlet(_Integrator):
    """integrate/velocity_verlet.hpp:39-80"""

    def __init__(self, dt):
        h = _vp()
        _check(lib().md_integrator_create_vv(float(dt), C.byref(h)))
        self._h = h
        self.dt = float(dt)


class LangevinBAOAB(_Integrator):
    """integrate/langevin.hpp:27-97"""

    def __init__(self, dt, friction, temperature, seed):
        h = _vp()
        _check(lib().md_integrator_create_baoab(float(dt), float(friction), float(temperature),
                                                int(seed), C.byref(h)))
        self._h = h
        self.dt = float(dt)

    def set_noise(self, xi):
        """Replay caller-supplied normals (3N per step, atom-major x,y,z) instead of Philox."""
        if xi is None:
            _check(lib().md_integrator_set_noise(self._h, None, 0))
            return
        xi = _f64(xi).reshape(-1)
        _check(lib().md_integrator_set_noise(self._h, _ptr(xi), xi.size))


class NoseHooverChain(_Integrator):
    """integrate/nose_hoover.hpp:24-67"""

    def __init__(self, dt, temperature, tau, chain_length, dof):
        h = _vp()
        _check(lib().md_integrator_create_nhc(float(dt), float(temperature), float(tau),
                                              int(chain_length), int(dof), C.byref(h)))
        self._h = h
        self.dt = float(dt)


# ---------------------------------------------------------------- rigid water
class RigidWater:
    """constrain/rigid_water.hpp:29-67: SHAKE/RATTLE on O-H1, O-H2, H1-H2 of each
    consecutive (O, H, H) triple, one GPU thread per molecule."""

    def __init__(self, oh_distance, hoh_angle_degrees, tolerance=1e-12, max_iterations=500,
                 settle=False):
        h = _vp()
        _check(lib().md_rigid_create(float(oh_distance), float(hoh_angle_degrees),
                                     float(tolerance), int(max_iterations), C.byref(h)))
        self._h = h
        if settle:
            self.set_settle(True)

    def set_settle(self, on=True):
        """Closed-form SETTLE instead of SHAKE / RATTLE iterations (the same fixed
        point); integrators created afterwards inherit it."""
        _check(lib().md_rigid_set_settle(self._h, 1 if on else 0))

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.md_rigid_destroy(self._h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def _distances(self):
        oh, hh = C.c_double(), C.c_double()
        _check(lib().md_rigid_distances(self._h, C.byref(oh), C.byref(hh)))
        return oh.value, hh.value

    def oh_distance(self):
        return self._distances()[0]

    def hh_distance(self):
        return self._distances()[1]

    @staticmethod
    def degrees_of_freedom(molecules, com_removed):
        return int(lib().md_rigid_degrees_of_freedom(int(molecules), 1 if com_removed else 0))

    def constrain_positions(self, sys: System, reference) -> int:
        """Reset positions onto the constraint surface along the bonds of
        `reference` (an (N, 3) array in the system's atom order).  Returns the
        sweep count; raises MDError (std::runtime_error) on non-convergence."""
        ref = _f64(reference).reshape(-1, 3)
        if ref.shape[0] != sys.n:
            raise InvalidArgument("RigidWater: reference size differs from the system")
        cols = [np.ascontiguousarray(ref[:, k]) for k in range(3)]
        it = C.c_int()
        _check(lib().md_rigid_constrain_positions(self._h, sys.handle, *[_ptr(c) for c in cols],
                                                  C.byref(it)))
        return it.value

    def constrain_velocities(self, sys: System) -> int:
        it = C.c_int()
        _check(lib().md_rigid_constrain_velocities(self._h, sys.handle, C.byref(it)))
        return it.value


class ConstrainedVelocityVerlet(_Integrator):
    """integrate/constrained_velocity_verlet.hpp:22-66 (RATTLE form)."""

    def __init__(self, dt, constraint: RigidWater):
        h = _vp()
        _check(lib().md_integrator_create_rattle(float(dt), constraint.handle, C.byref(h)))
        self._h = h
        self.dt = float(dt)
        self.constraint = constraint

    def run(self, sys: System, ff: SpceForceField, steps: int, thermo=False):
        """Fused device loop with SPC/E forces.  Forces are recomputed on entry.
        Returns a (steps, 4) array [energy, virial, kinetic, conserved] if thermo."""
        out = np.zeros((steps, 4)) if thermo and steps > 0 else None
        _check(lib().md_run_spce(self._h, sys.handle, ff.handle, int(steps),
                                 _ptr(out) if out is not None else None))
        return out

    def iterations(self):
        """Largest (SHAKE, RATTLE) sweep counts seen so far."""
        a, b = C.c_int(), C.c_int()
        _check(lib().md_integrator_iterations(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value


class ConstrainedNoseHooverChain(ConstrainedVelocityVerlet):
    """A Nose-Hoover chain (integrate/nose_hoover.hpp) around the constrained
    step; the reference has no thermostatted rigid-water integrator.  dof is
    RigidWater.degrees_of_freedom(molecules, True) for a system at rest."""

    def __init__(self, dt, constraint: RigidWater, temperature, tau, chain_length, dof):
        h = _vp()
        _check(lib().md_integrator_create_rattle_nhc(float(dt), constraint.handle,
                                                     float(temperature), float(tau),
                                                     int(chain_length), int(dof), C.byref(h)))
        self._h = h
        self.dt = float(dt)
        self.constraint = constraint


# ---------------------------------------------------------------- adjoint
# ----------------------------------------------------------------- formats
def _b(x):
    return None if x is None else str(x).encode()


class ThermoCsv:
    """moldyn_run's thermo CSV (apps/moldyn_run.cpp:229-245, 497-511, 600-617):
    header on open, one row per thermo row of a fused run on append()."""

    def __init__(self, path, command_line="", revision=None, host=None, truncation=0,
                 dof_langevin=0, dof_nve=0):
        h = _vp()
        _check(lib().md_thermo_csv_open(_b(path), _b(command_line), _b(revision), _b(host),
                                        int(truncation), int(dof_langevin), int(dof_nve),
                                        C.byref(h)))
        self._h = h

    def append(self, lj, n, box, rows, first_step, dt, phase, dof, step_stride=1):
        rows = _f64(rows).reshape(-1, 4)
        _check(lib().md_thermo_csv_append(self._h, lj.handle, int(n), _ptr(_f64(box)),
                                          int(first_step), int(step_stride), float(dt),
                                          _b(phase), int(dof), _ptr(rows), len(rows)))

    def close(self):
        if getattr(self, "_h", None) and _lib is not None:
            h, self._h = self._h, None
            _check(_lib.md_thermo_csv_close(h))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def xyz_append(path, sys, step, time, phase, command_line="", revision=None, host=None):
    """One XYZ frame (moldyn_run.cpp:519-533) appended to path."""
    _check(lib().md_xyz_append(_b(path), sys.handle, int(step), float(time), _b(phase),
                               _b(revision), _b(host), _b(command_line)))


def checkpoint_save(sys, path, integrator=None):
    _check(lib().md_checkpoint_save(sys.handle, integrator.handle if integrator else None,
                                    _b(path)))


def checkpoint_load(path, integrator=None, ctx=None):
    """A System restored from a checkpoint (and the integrator's state, when given)."""
    ctx = ctx or default_context()
    h = _vp()
    _check(lib().md_checkpoint_load(ctx.handle, _b(path), C.byref(h),
                                    integrator.handle if integrator else None))
    return System._adopt(h, ctx)


# ---------------------------------------------------------------- analysis
class Rdf:
    """analyze/rdf.hpp:16-34: g(r) accumulated over frames, on the device."""

    def __init__(self, r_max, bins, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        self.bins = int(bins)
        h = _vp()
        _check(lib().md_rdf_create(self.ctx.handle, float(r_max), self.bins, C.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.md_rdf_destroy(self._h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def accumulate(self, sys: System, first=0, stride=1):
        """One frame; first/stride select the atoms with original index first,
        first + stride, ... (e.g. the oxygens of O, H, H water: 0, 3)."""
        if first == 0 and stride == 1:
            _check(lib().md_rdf_accumulate(self._h, sys.handle))
        else:
            _check(lib().md_rdf_accumulate_subset(self._h, sys.handle, int(first), int(stride)))

    def _vec(self, fn):
        out = np.zeros(self.bins)
        _check(fn(self._h, _ptr(out)))
        return out

    def histogram(self):
        """Pair counts per bin (i < j), summed over the frames."""
        return self._vec(lib().md_rdf_histogram)

    def g(self):
        return self._vec(lib().md_rdf_g)

    def bin_centres(self):
        return self._vec(lib().md_rdf_bin_centres)

    def frames(self) -> int:
        f = C.c_int64()
        _check(lib().md_rdf_frames(self._h, C.byref(f)))
        return f.value


class _Corr:
    _pre = ""

    def __init__(self, natoms, max_lag, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        self.max_lag = int(max_lag)
        h = _vp()
        _check(getattr(lib(), f"md_{self._pre}_create")(self.ctx.handle, int(natoms), self.max_lag,
                                                        C.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            getattr(_lib, f"md_{self._pre}_destroy")(self._h)
            self._h = None

    def push(self, sys: System):
        _check(getattr(lib(), f"md_{self._pre}_push")(self._h, sys.handle))


class Msd(_Corr):
    """analyze/msd.hpp:19-42: mean-squared displacement over all time origins."""
    _pre = "msd"

    def msd(self):
        out = np.zeros(self.max_lag + 1)
        _check(lib().md_msd_values(self._h, _ptr(out)))
        return out

    def diffusion_coefficient(self, dt, fit_from, fit_to):
        d = np.zeros(1)
        _check(lib().md_msd_diffusion(self._h, float(dt), int(fit_from), int(fit_to), _ptr(d)))
        return float(d[0])


class Vacf(_Corr):
    """analyze/vacf.hpp:151-174: velocity autocorrelation over all time origins."""
    _pre = "vacf"

    def vacf(self, normalised=True):
        out = np.zeros(self.max_lag + 1)
        _check(lib().md_vacf_values(self._h, 1 if normalised else 0, _ptr(out)))
        return out

    def diffusion_coefficient(self, dt):
        d = np.zeros(1)
        _check(lib().md_vacf_diffusion(self._h, float(dt), _ptr(d)))
        return float(d[0])


class AdjointTrajectory:
    """A differentiable FP64 velocity-Verlet LJ trajectory with a hand-written
    adjoint (no reference counterpart).  forward() saves the state every `every`
    steps and returns rows (steps, 3) = [U, W, KE] after each step; backward(g)
    with g = dL/d(rows) returns (dL/d epsilon, dL/d sigma, dL/dx0, dL/dv0)."""

    def __init__(self, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        h = _vp()
        _check(lib().md_adjoint_create(self.ctx.handle, C.byref(h)))
        self._h = h
        self.n = 0
        self.steps = 0
        self._sys = None

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.md_adjoint_destroy(self._h)
            self._h = None

    def forward(self, sys: System, lj: LennardJones, dt, steps, every=50, skin=1.0):
        rows = np.zeros((int(steps), 3))
        _check(lib().md_adjoint_forward(self._h, sys.handle, lj.handle, float(dt), int(steps),
                                        int(every), float(skin), _ptr(rows)))
        self.n, self.steps = sys.n, int(steps)
        self._sys = sys  # backward() replays on this system: keep it alive
        return rows

    def backward(self, grad_rows):
        g = _f64(grad_rows).reshape(self.steps, 3)
        th = np.zeros(2)
        gx = np.zeros((self.n, 3))
        gv = np.zeros((self.n, 3))
        _check(lib().md_adjoint_backward(self._h, _ptr(g), _ptr(th), _ptr(gx), _ptr(gv)))
        return th[0], th[1], gx, gv


# ---------------------------------------------------------------- batches
class Batch:
    """Independent LJ replicas stepped together (no reference counterpart).  Each
    replica is (integrator, system, Verlet list, LennardJones) with the system on
    its own Context; run() replays one CUDA graph per step over all replicas."""

    def __init__(self):
        h = _vp()
        _check(lib().md_batch_create(C.byref(h)))
        self._h = h
        self._keep = []

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.md_batch_destroy(self._h)
            self._h = None

    def add(self, integrator, sys: System, verlet: VerletList, lj: LennardJones) -> int:
        idx = C.c_int()
        _check(lib().md_batch_add(self._h, integrator.handle, sys.handle, verlet.handle,
                                  lj.handle, C.byref(idx)))
        self._keep.append((integrator, sys, verlet, lj))
        return idx.value

    def set_batched(self, on=True):
        """Stage kernels shared by all replicas (default) or a graph of
        per-replica kernels; every replica's trajectory is the same either way."""
        _check(lib().md_batch_set_batched(self._h, 1 if on else 0))

    def __len__(self):
        return lib().md_batch_size(self._h)

    def run(self, steps: int, thermo=False):
        """Returns a (replicas, steps, 4) array [energy, virial, kinetic, conserved]
        if thermo."""
        out = np.zeros((len(self), steps, 4)) if thermo and steps > 0 else None
        _check(lib().md_batch_run(self._h, int(steps), _ptr(out) if out is not None else None))
        return out


# ---------------------------------------------------------------- setup
class units:
    """core/units.hpp:33-40: the water side's time unit, tau = A sqrt(amu / kB)."""
    TAU_IN_PICOSECONDS = 1.0966875353

    @staticmethod
    def picoseconds(ps):
        return ps / units.TAU_IN_PICOSECONDS

    @staticmethod
    def femtoseconds(fs):
        return units.picoseconds(fs * 1.0e-3)

    @staticmethod
    def to_picoseconds(tau):
        return tau * units.TAU_IN_PICOSECONDS


def read_nist_config(path):
    """readNistConfig (io/nist_config.cpp:30-86): line 1 the box lengths, line 2
    a count (not trusted: the SPC/E files give molecules), then `index x y z
    [type]` lines until end of file, blank lines skipped.  Returns dict(pos,
    box, types); types is empty unless some line has the fifth column.  Raises
    MDError (std::runtime_error) on a missing file or a malformed line."""
    try:
        f = open(path)
    except OSError:
        raise MDError(f"readNistConfig: cannot open file {path}") from None
    with f:
        lines = f.read().split("\n")
    if lines and lines[-1] == "":
        lines.pop()
    if not lines:
        raise MDError(f"readNistConfig: empty file {path}")

    def numbers(text, count, conv):
        parts = text.split()
        if len(parts) < count:
            raise ValueError
        return [conv(x) for x in parts[:count]]

    try:
        box = np.array(numbers(lines[0], 3, float))
    except ValueError:
        raise MDError(f"readNistConfig: malformed box line in {path}") from None
    if len(lines) < 2:
        raise MDError(f"readNistConfig: missing count line in {path}")
    try:
        numbers(lines[1], 1, int)
    except ValueError:
        raise MDError(f"readNistConfig: malformed count line in {path}") from None
    pos, types, any_typed = [], [], False
    for line in lines[2:]:
        if not line.strip(" \t\r\n"):
            continue
        parts = line.split()
        try:
            int(parts[0])
            xyz = [float(v) for v in parts[1:4]]
            if len(xyz) < 3:
                raise ValueError
        except (ValueError, IndexError):
            raise MDError(f"readNistConfig: malformed atom line in {path}") from None
        pos.append(xyz)
        types.append(parts[4] if len(parts) > 4 else "")
        any_typed = any_typed or len(parts) > 4
    return dict(pos=np.array(pos).reshape(-1, 3), box=box, types=types if any_typed else [])


def water_lattice(per_side, box_length, seed, params=SpceParameters):
    """A simple cubic lattice of rigid SPC/E molecules (per_side^3 molecules in a
    cubic box of side box_length, oxygens at the cell centres, each molecule
    turned by a seeded random rotation); O, H, H order, rOH and the HOH angle of
    `params`.  Host-side setup, no reference counterpart (the reference reads
    its water from the NIST configuration files)."""
    rng = np.random.default_rng(seed)
    a = box_length / per_side
    half = 0.5 * np.radians(params.angleHOH)
    local = np.array([[0.0, 0.0, 0.0],
                      [params.rOH * np.sin(half), 0.0, params.rOH * np.cos(half)],
                      [-params.rOH * np.sin(half), 0.0, params.rOH * np.cos(half)]])
    m = per_side ** 3
    q = rng.normal(size=(m, 4))
    q /= np.linalg.norm(q, axis=1)[:, None]
    w, x, y, z = q.T
    rot = np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1)], 1)
    idx = np.arange(m)
    centre = (np.stack([idx % per_side, (idx // per_side) % per_side, idx // per_side ** 2], 1)
              + 0.5) * a - 0.5 * box_length
    pos = centre[:, None, :] + np.einsum("mij,kj->mki", rot, local)
    pos = pos.reshape(-1, 3)
    pos -= box_length * np.floor(pos / box_length + 0.5)
    types = ["O", "H", "H"] * m
    return dict(pos=pos, types=types, box=np.full(3, float(box_length)))


def fcc_lattice(cells, density, temperature, seed):
    """util/lattice.cpp:15-64 (host-side setup).  Returns dict(pos, vel, mass, box)."""
    n = 4 * int(cells) ** 3
    arrs = [np.zeros(n) for _ in range(7)]
    box = np.zeros(3)
    rc = lib().md_fcc_lattice(int(cells), float(density), float(temperature), int(seed),
                              *[_ptr(a) for a in arrs], _ptr(box))
    if rc < 0:
        _check(rc)
    x, y, z, vx, vy, vz, m = arrs
    return dict(pos=np.stack([x, y, z], 1), vel=np.stack([vx, vy, vz], 1), mass=m, box=box)
