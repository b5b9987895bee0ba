"""mahyco_b200 -- B200-native MaHyCo hydro cycle.

The compute path is ``libmahyco_b200.so`` (hand-written sm_100a kernels
behind the C ABI of ``include/mahyco_b200.h``).  This module is a thin
ctypes binding that mirrors the reference module interface
(``src/MahycoModule.h:164-349``): a :class:`Hydro` object exposes the
init and compute-loop entry points under the reference names.  There is no
CPU fallback: creating a case without the built library or without a CUDA
device raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .case import (CaseParams, EnvParams, add_bc, default_params, read_arc,  # noqa: F401
                   symmetry_bcs, CASE_SOD, CASE_SEDOV, CASE_TWO_STATE,
                   EOS_PERFECT_GAS, EOS_STIFFENED_GAS, EOS_MIE_GRUNEISEN,
                   MINMOD, SUPERBEE, VANLEER)

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmahyco_b200.so")

ST_NEG_VOLUME, ST_DT_UNDERFLOW, ST_NAN, ST_STOP = 1, 2, 4, 8
ST_OOM_ADMISSION, ST_TIMEOUT, ST_DAMAGE = 16, 32, 64
REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED = 0, 1, 2, 3

_lib = None

# exported symbols and their (restype, argtypes)
_SIGS = {
    "mhc_last_error": (C.c_char_p, []),
    "mhc_version": (C.c_char_p, []),
    "mhc_case_create": (C.c_int, [C.POINTER(CaseParams), C.POINTER(C.c_void_p)]),
    "mhc_case_destroy": (C.c_int, [C.c_void_p]),
    "mhc_case_stream": (C.c_void_p, [C.c_void_p]),
    "mhc_case_device_bytes": (C.c_longlong, [C.POINTER(CaseParams)]),
    "mhc_hydro_start_init": (C.c_int, [C.c_void_p]),
    "mhc_save_values_at_n": (C.c_int, [C.c_void_p]),
    "mhc_update_velocity": (C.c_int, [C.c_void_p]),
    "mhc_apply_boundary_condition": (C.c_int, [C.c_void_p]),
    "mhc_update_position": (C.c_int, [C.c_void_p]),
    "mhc_compute_geometric_values": (C.c_int, [C.c_void_p]),
    "mhc_update_density": (C.c_int, [C.c_void_p]),
    "mhc_compute_artificial_viscosity": (C.c_int, [C.c_void_p]),
    "mhc_update_elasticity_and_plasticity": (C.c_int, [C.c_void_p]),
    "mhc_update_energy_and_pressure": (C.c_int, [C.c_void_p]),
    "mhc_remap": (C.c_int, [C.c_void_p]),
    "mhc_compute_delta_t": (C.c_int, [C.c_void_p]),
    "mhc_cycle": (C.c_int, [C.c_void_p, C.c_int]),
    "mhc_cycle_graph": (C.c_int, [C.c_void_p, C.c_int]),
    "mhc_cycle_timed": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_longlong)]),
    "mhc_synchronize": (C.c_int, [C.c_void_p]),
    "mhc_get_scalars": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                  C.POINTER(C.c_longlong), C.POINTER(C.c_int)]),
    "mhc_get_field": (C.c_longlong, [C.c_void_p, C.c_char_p, C.c_int, C.POINTER(C.c_double), C.c_longlong]),
    "mhc_eos_apply": (C.c_int, [C.c_void_p, C.c_int]),
    "mhc_remap_apply": (C.c_int, [C.c_void_p]),
    "mhc_time_history": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "mhc_batch_create": (C.c_int, [C.POINTER(C.c_void_p)]),
    "mhc_batch_destroy": (C.c_int, [C.c_void_p]),
    "mhc_batch_stream": (C.c_void_p, [C.c_void_p]),
    "mhc_batch_add": (C.c_int, [C.c_void_p, C.POINTER(CaseParams), C.c_longlong, C.POINTER(C.c_int)]),
    "mhc_batch_init": (C.c_int, [C.c_void_p]),
    "mhc_batch_remove": (C.c_int, [C.c_void_p, C.c_int]),
    "mhc_batch_cycle": (C.c_int, [C.c_void_p, C.c_int]),
    "mhc_batch_cycle_graph": (C.c_int, [C.c_void_p, C.c_int]),
    "mhc_batch_cycle_timed": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_longlong)]),
    "mhc_batch_synchronize": (C.c_int, [C.c_void_p]),
    "mhc_batch_set_grid_scale": (C.c_int, [C.c_void_p, C.c_int]),
    "mhc_batch_set_stage_grid_scale": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "mhc_batch_launches": (C.c_longlong, [C.c_void_p]),
    "mhc_case_launches": (C.c_longlong, [C.c_void_p]),
    "mhc_batch_get_scalars": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                        C.POINTER(C.c_longlong), C.POINTER(C.c_int)]),
    "mhc_batch_get_field": (C.c_longlong, [C.c_void_p, C.c_int, C.c_char_p, C.c_int, C.POINTER(C.c_double),
                                           C.c_longlong]),
    "mhc_cfl_delta_t_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_double,
                                          C.c_double, C.c_double, C.c_double, C.c_void_p, C.c_void_p]),
    "mhc_noalloc_last_error": (C.c_char_p, []),
    "mhc_batch_detach": (C.c_int, [C.c_void_p, C.c_int]),
    "mhc_scalars_request": (C.c_int, [C.c_void_p]),
    "mhc_scalars_wait": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                   C.POINTER(C.c_longlong), C.POINTER(C.c_int)]),
    "mhc_case_checkpoint_bytes": (C.c_longlong, [C.c_void_p]),
    "mhc_case_checkpoint": (C.c_int, [C.c_void_p, C.c_void_p, C.c_longlong]),
    "mhc_case_restore": (C.c_int, [C.c_void_p, C.c_void_p, C.c_longlong]),
    "mhc_batch_checkpoint_bytes": (C.c_longlong, [C.c_void_p, C.c_int]),
    "mhc_batch_checkpoint": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_longlong]),
    "mhc_batch_restore": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_longlong]),
    "mhc_batch_poll": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_longlong), C.POINTER(C.c_int),
                                 C.POINTER(C.c_double)]),
    "mhc_server_create": (C.c_int, [C.c_longlong, C.POINTER(C.c_void_p)]),
    "mhc_server_destroy": (C.c_int, [C.c_void_p]),
    "mhc_server_stream": (C.c_void_p, [C.c_void_p, C.c_int]),
    "mhc_server_launches": (C.c_longlong, [C.c_void_p]),
    "mhc_server_submit": (C.c_int, [C.c_void_p, C.c_void_p, C.c_longlong, C.c_double, C.POINTER(C.c_longlong)]),
    "mhc_server_step": (C.c_int, [C.c_void_p, C.c_int]),
    "mhc_server_poll": (C.c_int, [C.c_void_p, C.c_longlong, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                  C.POINTER(C.c_longlong), C.POINTER(C.c_double)]),
    "mhc_server_times": (C.c_int, [C.c_void_p, C.c_longlong, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                   C.POINTER(C.c_double)]),
    "mhc_server_fetch": (C.c_longlong, [C.c_void_p, C.c_longlong, C.c_char_p, C.c_int, C.POINTER(C.c_double),
                                        C.c_longlong]),
    "mhc_server_release": (C.c_int, [C.c_void_p, C.c_longlong]),
    "mhc_server_stats": (C.c_int, [C.c_void_p, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong),
                                   C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    # field upload and the per-method service surface (IEquationOfState, IRemap)
    "mhc_case_params_default": (None, [C.POINTER(CaseParams)]),
    "mhc_case_params_size": (C.c_longlong, []),
    "mhc_batch_create_on_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "mhc_batch_poll_request": (C.c_int, [C.c_void_p]),
    "mhc_batch_set_sweep_layout": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "mhc_case_set_sweep_layout": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "mhc_case_set_stage_grid_scale": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "mhc_batch_poll_wait": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_longlong), C.POINTER(C.c_int),
                                      C.POINTER(C.c_double)]),
    "mhc_server_take_completed": (C.c_int, [C.c_void_p, C.POINTER(C.c_longlong), C.c_int]),
    "mhc_set_field": (C.c_longlong, [C.c_void_p, C.c_char_p, C.c_int, C.POINTER(C.c_double), C.c_longlong]),
    "mhc_case_set_initial_field": (C.c_longlong, [C.c_void_p, C.c_char_p, C.POINTER(C.c_double), C.c_longlong]),
    "mhc_eos_init": (C.c_int, [C.c_void_p, C.c_int]),
    "mhc_eos_reinit": (C.c_int, [C.c_void_p, C.c_int]),
    "mhc_eos_apply_one_cell": (C.c_int, [C.c_void_p, C.c_int, C.c_longlong, C.POINTER(C.c_double)]),
    "mhc_eos_endommagement": (C.c_int, [C.c_void_p, C.c_int]),
    "mhc_eos_get_adiabatic_cst": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double)]),
    "mhc_eos_get_density_damage_thresold": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double)]),
    "mhc_remap_appli_remap": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int]),
    "mhc_remap_sweeps": (C.c_int, [C.c_void_p]),
    "mhc_remap_variables": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int]),
    "mhc_remap_resize_remap_variables": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "mhc_remap_synchronize_uremap": (C.c_int, [C.c_void_p]),
    "mhc_remap_get_ordre_projection": (C.c_int, [C.c_void_p]),
    "mhc_remap_has_projection_pente_borne": (C.c_int, [C.c_void_p]),
    "mhc_remap_has_projection_simple_pente": (C.c_int, [C.c_void_p]),
    "mhc_remap_has_conservation_energie_totale": (C.c_int, [C.c_void_p]),
    "mhc_remap_is_euler": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int]),
}


class MahycoError(RuntimeError):
    pass


def load(path: str | None = None) -> C.CDLL:
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or os.environ.get("MAHYCO_B200_LIB") or LIB_PATH
    if not os.path.exists(p):
        raise MahycoError(f"{p} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'`")
    lib = C.CDLL(p)
    for name, (res, args) in _SIGS.items():
        f = getattr(lib, name)
        f.restype, f.argtypes = res, args
    if path is None:
        _lib = lib
    return lib


def _check(lib, code: int, what: str) -> int:
    if code < 0:
        raise MahycoError(f"{what} failed ({code}): {lib.mhc_last_error().decode()}")
    return code


class Hydro:
    """One MaHyCo case resident on the GPU (replaces the MahycoModule instance)."""

    CELL_FIELDS = ("Density", "Pressure", "InternalEnergy", "SoundSpeed", "PseudoViscosity",
                   "CellMass", "CellVolume", "FracVol", "MassFraction", "CaracteristicLength")

    def __init__(self, params: CaseParams, lib: C.CDLL | None = None):
        self.lib = lib or load()
        self.params = params
        h = C.c_void_p()
        _check(self.lib, self.lib.mhc_case_create(C.byref(params), C.byref(h)), "mhc_case_create")
        self.h = h
        self.ncell = params.ncell
        self.nnode = params.nnode

    @property
    def stream_handle(self) -> int:
        """cudaStream_t of the case (for torch.cuda.ExternalStream / events)"""
        return int(self.lib.mhc_case_stream(self.h))

    @property
    def launches(self) -> int:
        """Kernels this case has put on the GPU so far."""
        return int(self.lib.mhc_case_launches(self.h))

    def scalars_request(self) -> int:
        """Enqueue an asynchronous read-back of the scalars; returns its slot."""
        return _check(self.lib, self.lib.mhc_scalars_request(self.h), "mhc_scalars_request")

    def scalars_wait(self, slot: int) -> dict:
        """Scalars of an earlier scalars_request, once the copy has landed."""
        t, dt, it, st = C.c_double(), C.c_double(), C.c_longlong(), C.c_int()
        _check(self.lib, self.lib.mhc_scalars_wait(self.h, int(slot), C.byref(t), C.byref(dt), C.byref(it),
                                                   C.byref(st)), "mhc_scalars_wait")
        return {"time": t.value, "deltat": dt.value, "iteration": it.value, "status": st.value}

    def checkpoint(self) -> bytes:
        """Whole device state between iterations (protection)."""
        n = _check(self.lib, int(self.lib.mhc_case_checkpoint_bytes(self.h)), "checkpoint size")
        buf = C.create_string_buffer(n)
        _check(self.lib, self.lib.mhc_case_checkpoint(self.h, buf, n), "mhc_case_checkpoint")
        return buf.raw

    def restore(self, data: bytes) -> None:
        """Continue from a checkpoint of a case with identical parameters (reprise)."""
        buf = C.create_string_buffer(data, len(data))
        _check(self.lib, self.lib.mhc_case_restore(self.h, buf, len(data)), "mhc_case_restore")

    def close(self):
        if self.h:
            self.lib.mhc_case_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_initial_field(self, name: str, values) -> None:
        """Before hydroStartInit: NodeCoord of a mesh file (Lagrangian
        cases), Materiau / Density / Pressure of the EXTERNAL case model
        (mhc_case_set_initial_field)."""
        a = np.ascontiguousarray(values, dtype=np.float64)
        got = self.lib.mhc_case_set_initial_field(self.h, name.encode(), a.ctypes.data_as(C.POINTER(C.c_double)),
                                                  a.size)
        _check(self.lib, int(got), f"set_initial_field {name}")

    # -- init entry points (Mahyco.config:15-21)
    def hydroStartInit(self):
        return _check(self.lib, self.lib.mhc_hydro_start_init(self.h), "HydroStartInit")

    # -- compute-loop entry points (Mahyco.config:23-36)
    def saveValuesAtN(self): return _check(self.lib, self.lib.mhc_save_values_at_n(self.h), "SaveValuesAtN")
    def updateVelocity(self): return _check(self.lib, self.lib.mhc_update_velocity(self.h), "UpdateVelocity")
    def applyBoundaryCondition(self): return _check(self.lib, self.lib.mhc_apply_boundary_condition(self.h), "ApplyBoundaryCondition")
    def updatePosition(self): return _check(self.lib, self.lib.mhc_update_position(self.h), "UpdatePosition")
    def computeGeometricValues(self): return _check(self.lib, self.lib.mhc_compute_geometric_values(self.h), "ComputeGeometricValues")
    def updateDensity(self): return _check(self.lib, self.lib.mhc_update_density(self.h), "UpdateDensity")
    def computeArtificialViscosity(self): return _check(self.lib, self.lib.mhc_compute_artificial_viscosity(self.h), "ComputeArtificialViscosity")
    def updateElasticityAndPlasticity(self): return _check(self.lib, self.lib.mhc_update_elasticity_and_plasticity(self.h), "UpdateElasticityAndPlasticity")
    def updateEnergyAndPressure(self): return _check(self.lib, self.lib.mhc_update_energy_and_pressure(self.h), "UpdateEnergyAndPressure")
    def remap(self): return _check(self.lib, self.lib.mhc_remap(self.h), "Remap")
    def computeDeltaT(self): return _check(self.lib, self.lib.mhc_compute_delta_t(self.h), "ComputeDeltaT")

    def iterate(self):
        """One compute-loop iteration through the individual entry points."""
        for ep in (self.saveValuesAtN, self.updateVelocity, self.applyBoundaryCondition,
                   self.updatePosition, self.computeGeometricValues, self.updateDensity,
                   self.computeArtificialViscosity, self.updateElasticityAndPlasticity,
                   self.updateEnergyAndPressure, self.remap, self.computeDeltaT):
            ep()

    def cycle(self, n: int, graph: bool = False) -> None:
        f = self.lib.mhc_cycle_graph if graph else self.lib.mhc_cycle
        _check(self.lib, f(self.h, int(n)), "mhc_cycle")

    STAGES = ("lagrange_nodes", "lagrange_cells", "sweep_cells", "sweep_nodes",
              "finalize_cells", "finalize_nodes", "delta_t")

    def cycle_timed(self, n: int) -> dict:
        """n iterations with CUDA events around every kernel group (on the
        case stream); returns {stage: (total_ms, launches)}."""
        ms = (C.c_double * len(self.STAGES))()
        ln = (C.c_longlong * len(self.STAGES))()
        _check(self.lib, self.lib.mhc_cycle_timed(self.h, int(n), ms, ln), "mhc_cycle_timed")
        return {s: (ms[i], ln[i]) for i, s in enumerate(self.STAGES)}

    def synchronize(self) -> int:
        return _check(self.lib, self.lib.mhc_synchronize(self.h), "mhc_synchronize")

    def run(self, max_iter: int, chunk: int = 10) -> int:
        """Iterate until the final time (stop flag), an error flag or max_iter."""
        done = 0
        while done < max_iter:
            n = min(chunk, max_iter - done)
            for _ in range(n):
                self.cycle(1)
                st = self.synchronize()
                done += 1
                if st:
                    return st
        return self.synchronize()

    def scalars(self) -> dict:
        t, dt, it, st = C.c_double(), C.c_double(), C.c_longlong(), C.c_int()
        _check(self.lib, self.lib.mhc_get_scalars(self.h, C.byref(t), C.byref(dt), C.byref(it), C.byref(st)), "scalars")
        return {"time": t.value, "deltat": dt.value, "iteration": it.value, "status": st.value}

    def field(self, name: str, env: int = -1, out: np.ndarray | None = None) -> np.ndarray:
        """Copy a field to the host: a new array, or `out` (float64,
        contiguous, at least the field's size; page-locked memory is
        written by one direct copy)."""
        n = 3 * self.nnode if name in ("Velocity", "VelocityN", "NodeCoord") else (
            self.nnode if name == "NodeMass" else self.ncell)
        if out is None:
            out = np.empty(n, dtype=np.float64)
        elif out.dtype != np.float64 or not out.flags["C_CONTIGUOUS"] or out.size < n:
            raise MahycoError(f"field {name}: out must be a contiguous float64 array of >= {n} values")
        got = self.lib.mhc_get_field(self.h, name.encode(), int(env),
                                     out.ctypes.data_as(C.POINTER(C.c_double)), n)
        _check(self.lib, int(got), f"field {name}")
        return out

    def set_field(self, name: str, values: np.ndarray, env: int = -1) -> None:
        """Upload a field (mhc_set_field): same names, env semantics and
        layout as field()."""
        a = np.ascontiguousarray(values, dtype=np.float64)
        got = self.lib.mhc_set_field(self.h, name.encode(), int(env), a.ctypes.data_as(C.POINTER(C.c_double)), a.size)
        _check(self.lib, int(got), f"set_field {name}")

    # IEquationOfState (src/eos/IEquationOfState.h:38-65), per environment
    def set_sweep_layout(self, cell_layout: int, node_layout: int):
        """y / z sweep layouts: 0 by mesh size, 1 warp per line, 2 tile, 3 line chunks."""
        _check(self.lib, self.lib.mhc_case_set_sweep_layout(self.h, int(cell_layout), int(node_layout)),
               "sweep layout")

    def set_stage_grid_scale(self, stage: int | str, scale: int):
        st = Hydro.STAGES.index(stage) if isinstance(stage, str) else int(stage)
        _check(self.lib, self.lib.mhc_case_set_stage_grid_scale(self.h, st, int(scale)), "stage grid scale")

    def set_grid_scale(self, scale: int):
        for st in range(len(Hydro.STAGES)):
            self.set_stage_grid_scale(st, scale)

    def eos_apply(self, env: int) -> None:
        _check(self.lib, self.lib.mhc_eos_apply(self.h, int(env)), "applyEOS")

    def initEOS(self, env: int) -> None:
        _check(self.lib, self.lib.mhc_eos_init(self.h, int(env)), "initEOS")

    def ReinitEOS(self, env: int) -> None:
        _check(self.lib, self.lib.mhc_eos_reinit(self.h, int(env)), "ReinitEOS")

    def applyOneCellEOS(self, env: int, cell: int) -> float:
        """Pressure and sound speed of one cell of env in place; returns dp/de."""
        d = C.c_double()
        _check(self.lib, self.lib.mhc_eos_apply_one_cell(self.h, int(env), int(cell), C.byref(d)), "applyOneCellEOS")
        return d.value

    def Endommagement(self, env: int) -> None:
        _check(self.lib, self.lib.mhc_eos_endommagement(self.h, int(env)), "Endommagement")

    def getAdiabaticCst(self, env: int) -> float:
        d = C.c_double()
        _check(self.lib, self.lib.mhc_eos_get_adiabatic_cst(self.h, int(env), C.byref(d)), "getAdiabaticCst")
        return d.value

    def getdensityDamageThresold(self, env: int) -> float:
        d = C.c_double()
        _check(self.lib, self.lib.mhc_eos_get_density_damage_thresold(self.h, int(env), C.byref(d)),
               "getdensityDamageThresold")
        return d.value

    # IRemap (src/Remap/IRemap.h:44-63)
    def appliRemap(self, dimension: int, with_dual: int, nb_vars: int, nb_env: int) -> None:
        _check(self.lib, self.lib.mhc_remap_appli_remap(self.h, dimension, with_dual, nb_vars, nb_env), "appliRemap")

    def remapSweeps(self) -> None:
        _check(self.lib, self.lib.mhc_remap_sweeps(self.h), "remap sweeps")

    def remapVariables(self, dimension: int, with_dual: int, nb_vars: int, nb_env: int) -> None:
        _check(self.lib, self.lib.mhc_remap_variables(self.h, dimension, with_dual, nb_vars, nb_env),
               "remapVariables")

    def resizeRemapVariables(self, nb_vars: int, nb_env: int) -> None:
        _check(self.lib, self.lib.mhc_remap_resize_remap_variables(self.h, nb_vars, nb_env), "resizeRemapVariables")

    def synchronizeUremap(self) -> None:
        _check(self.lib, self.lib.mhc_remap_synchronize_uremap(self.h), "synchronizeUremap")

    def getOrdreProjection(self) -> int:
        return _check(self.lib, self.lib.mhc_remap_get_ordre_projection(self.h), "getOrdreProjection")

    def hasProjectionPenteBorne(self) -> bool:
        return bool(_check(self.lib, self.lib.mhc_remap_has_projection_pente_borne(self.h), "hasProjectionPenteBorne"))

    def hasProjectionSimplePente(self) -> bool:
        return bool(_check(self.lib, self.lib.mhc_remap_has_projection_simple_pente(self.h), "hasProjectionSimplePente"))

    def hasConservationEnergieTotale(self) -> bool:
        return bool(_check(self.lib, self.lib.mhc_remap_has_conservation_energie_totale(self.h),
                           "hasConservationEnergieTotale"))

    def isEuler(self) -> str:
        buf = C.create_string_buffer(8)
        _check(self.lib, self.lib.mhc_remap_is_euler(self.h, buf, 8), "isEuler")
        return buf.value.decode()

    def time_history(self) -> np.ndarray:
        out = np.empty(1 + 5 * self.params.nb_env, dtype=np.float64)
        _check(self.lib, self.lib.mhc_time_history(self.h, out.ctypes.data_as(C.POINTER(C.c_double))),
               "time history")
        return out


class Batch:
    """Many independent cases resident on the GPU, advanced together by one
    persistent launch per kernel phase (``mhc_batch_*`` of the C ABI)."""

    def __init__(self, lib: C.CDLL | None = None):
        self.lib = lib or load()
        b = C.c_void_p()
        _check(self.lib, self.lib.mhc_batch_create(C.byref(b)), "mhc_batch_create")
        self.b = b
        self.params = {}

    def close(self):
        if self.b:
            self.lib.mhc_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def stream_handle(self) -> int:
        return int(self.lib.mhc_batch_stream(self.b))

    def add(self, params: CaseParams, iteration_limit: int = 0) -> int:
        idx = C.c_int()
        _check(self.lib, self.lib.mhc_batch_add(self.b, C.byref(params), int(iteration_limit), C.byref(idx)),
               "mhc_batch_add")
        self.params[idx.value] = params
        return idx.value

    def init(self):
        _check(self.lib, self.lib.mhc_batch_init(self.b), "mhc_batch_init")

    def remove(self, idx: int):
        _check(self.lib, self.lib.mhc_batch_remove(self.b, int(idx)), "mhc_batch_remove")
        self.params.pop(idx, None)

    def cycle(self, n: int, graph: bool = False):
        f = self.lib.mhc_batch_cycle_graph if graph else self.lib.mhc_batch_cycle
        _check(self.lib, f(self.b, int(n)), "mhc_batch_cycle")

    def cycle_timed(self, n: int) -> dict:
        ms = (C.c_double * len(Hydro.STAGES))()
        ln = (C.c_longlong * len(Hydro.STAGES))()
        _check(self.lib, self.lib.mhc_batch_cycle_timed(self.b, int(n), ms, ln), "mhc_batch_cycle_timed")
        return {s: (ms[i], ln[i]) for i, s in enumerate(Hydro.STAGES)}

    def synchronize(self):
        _check(self.lib, self.lib.mhc_batch_synchronize(self.b), "mhc_batch_synchronize")

    def set_grid_scale(self, scale: int):
        _check(self.lib, self.lib.mhc_batch_set_grid_scale(self.b, int(scale)), "grid scale")

    def set_sweep_layout(self, cell_layout: int, node_layout: int):
        """y / z sweep layouts: 0 by mesh size, 1 warp per line, 2 tile, 3 line chunks."""
        _check(self.lib, self.lib.mhc_batch_set_sweep_layout(self.b, int(cell_layout), int(node_layout)),
               "sweep layout")

    @property
    def launches(self) -> int:
        """Kernels this batch has put on the GPU so far."""
        return int(self.lib.mhc_batch_launches(self.b))

    def set_stage_grid_scale(self, stage: int | str, scale: int):
        st = Hydro.STAGES.index(stage) if isinstance(stage, str) else int(stage)
        _check(self.lib, self.lib.mhc_batch_set_stage_grid_scale(self.b, st, int(scale)), "stage grid scale")

    def detach(self, idx: int):
        _check(self.lib, self.lib.mhc_batch_detach(self.b, int(idx)), "mhc_batch_detach")

    def poll(self) -> list[tuple[int, int, float]]:
        """(iteration, status, time) of every case index, from one read-back."""
        n = max(self.params) + 1 if self.params else 0
        it = (C.c_longlong * max(n, 1))()
        st = (C.c_int * max(n, 1))()
        tm = (C.c_double * max(n, 1))()
        _check(self.lib, self.lib.mhc_batch_poll(self.b, n, it, st, tm), "mhc_batch_poll")
        return [(it[i], st[i], tm[i]) for i in range(n)]

    def scalars(self, idx: int) -> dict:
        t, dt, it, st = C.c_double(), C.c_double(), C.c_longlong(), C.c_int()
        _check(self.lib, self.lib.mhc_batch_get_scalars(self.b, int(idx), C.byref(t), C.byref(dt), C.byref(it),
                                                        C.byref(st)), "batch scalars")
        return {"time": t.value, "deltat": dt.value, "iteration": it.value, "status": st.value}

    def field(self, idx: int, name: str, env: int = -1) -> np.ndarray:
        p = self.params[idx]
        n = 3 * p.nnode if name in ("Velocity", "VelocityN", "NodeCoord") else (p.nnode if name == "NodeMass" else p.ncell)
        out = np.empty(n, dtype=np.float64)
        got = self.lib.mhc_batch_get_field(self.b, int(idx), name.encode(), int(env),
                                           out.ctypes.data_as(C.POINTER(C.c_double)), n)
        _check(self.lib, int(got), f"batch field {name}")
        return out


class Server:
    """Request loop with continuous batching under an HBM budget
    (``mhc_server_*`` of the C ABI).  submit() queues a solve; step() admits
    what fits, advances every resident case and retires finished ones."""

    def __init__(self, hbm_budget_bytes: int = 0, lib: C.CDLL | None = None):
        self.lib = lib or load()
        s = C.c_void_p()
        _check(self.lib, self.lib.mhc_server_create(int(hbm_budget_bytes), C.byref(s)), "mhc_server_create")
        self.s = s
        self.params = {}

    def close(self):
        if self.s:
            self.lib.mhc_server_destroy(self.s)
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def stream_handle(self, size_class: int = 0) -> int:
        return int(self.lib.mhc_server_stream(self.s, int(size_class)) or 0)

    @property
    def launches(self) -> int:
        return int(self.lib.mhc_server_launches(self.s))

    def submit(self, params: CaseParams, iterations: int, timeout_s: float = 0.0) -> int:
        t = C.c_longlong()
        _check(self.lib, self.lib.mhc_server_submit(self.s, C.byref(params), int(iterations), float(timeout_s),
                                                    C.byref(t)), "mhc_server_submit")
        self.params[t.value] = params
        return t.value

    def step(self, cycles: int = 1) -> int:
        return _check(self.lib, self.lib.mhc_server_step(self.s, int(cycles)), "mhc_server_step")

    def take_completed(self, capacity: int = 4096) -> list[int]:
        """Tickets completed since the last call."""
        buf = (C.c_longlong * capacity)()
        n = _check(self.lib, self.lib.mhc_server_take_completed(self.s, buf, capacity), "mhc_server_take_completed")
        return list(buf[:n])

    def poll(self, ticket: int) -> dict:
        state, status, it, tm = C.c_int(), C.c_int(), C.c_longlong(), C.c_double()
        _check(self.lib, self.lib.mhc_server_poll(self.s, int(ticket), C.byref(state), C.byref(status), C.byref(it),
                                                  C.byref(tm)), "mhc_server_poll")
        return {"state": state.value, "status": status.value, "iteration": it.value, "time": tm.value}

    def times(self, ticket: int) -> dict:
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        _check(self.lib, self.lib.mhc_server_times(self.s, int(ticket), C.byref(a), C.byref(b), C.byref(c)),
               "mhc_server_times")
        return {"submit": a.value, "admit": b.value, "done": c.value}

    def fetch(self, ticket: int, name: str, env: int = -1) -> np.ndarray:
        p = self.params[ticket]
        n = 3 * p.nnode if name in ("Velocity", "VelocityN", "NodeCoord") else (p.nnode if name == "NodeMass" else p.ncell)
        out = np.empty(n, dtype=np.float64)
        got = self.lib.mhc_server_fetch(self.s, int(ticket), name.encode(), int(env),
                                        out.ctypes.data_as(C.POINTER(C.c_double)), n)
        _check(self.lib, int(got), f"server fetch {name}")
        return out

    def release(self, ticket: int):
        _check(self.lib, self.lib.mhc_server_release(self.s, int(ticket)), "mhc_server_release")
        self.params.pop(ticket, None)

    def stats(self) -> dict:
        q, r, b, g = C.c_longlong(), C.c_longlong(), C.c_longlong(), C.c_longlong()
        _check(self.lib, self.lib.mhc_server_stats(self.s, C.byref(q), C.byref(r), C.byref(b), C.byref(g)),
               "mhc_server_stats")
        return {"queued": q.value, "running": r.value, "bytes_in_use": b.value, "budget": g.value}
