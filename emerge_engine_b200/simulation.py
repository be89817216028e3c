"""`Simulation` on the CUDA backend, with the reference's method names.

Mirrors the public surface of the reference `Simulation` that the MLS-MPM step needs:
construction and builders (spacetime/solver/lifecycle.rs:26-214), `add_body`
(solver/particles.rs:355-423), `step` / `step_n` (solver/step.rs:23-60, 327-331),
`region_state` (solver/queries.rs:125-141), `particles()` and the last-step accessors.
Every call goes through the C ABI of libemerge_cuda.so; nothing is computed on the host
except scene bookkeeping (material registry, boundary list).
"""
from __future__ import annotations

import ctypes
from ctypes import byref, c_float, c_uint32, c_uint64, c_void_p

import numpy as np

from . import abi, lifecycle
from .abi import (PARTICLE_DTYPE, BodyStateC, MaterialParamsC, StepTimingC, check,
                  load_library)
from .config import BodyState, SimConfig, SlipBoundary, SpawnRegion
from .fields import Field, pack_fields
from .materials import DEVICE_MODELS, FallbackMaterial, Material, mixture_phase_of

MAX_MATERIAL_SLOTS = 64  # materials/registry.rs:6


class MaterialRegistry:
    """`MaterialRegistry` semantics (materials/registry.rs:12-112): contiguous ids from 0,
    at most 64 slots, slot 0 is the default."""

    def __init__(self, default: Material):
        self.materials = [default]

    def insert(self, material_id: int, material: Material) -> None:
        if material_id >= MAX_MATERIAL_SLOTS:
            raise ValueError(f"material_id {material_id} exceeds GPU limit of 64")
        if material_id < len(self.materials):
            self.materials[material_id] = material
        elif material_id == len(self.materials):
            self.materials.append(material)
        else:
            raise ValueError("material IDs must be registered contiguously starting at 0; "
                             f"expected id {len(self.materials)}, got {material_id}")

    def next_id(self) -> int:
        return len(self.materials)

    def set_default(self, material: Material) -> None:
        self.materials[0] = material

    def get(self, material_id: int) -> Material:
        if material_id < len(self.materials):
            return self.materials[material_id]
        return self.materials[0]

    def __len__(self):
        return len(self.materials)


class Simulation:
    """The reference `Simulation` API, stepped by the B200 kernels."""

    def __init__(self, config: SimConfig, device: int = 0, lib_path: str | None = None,
                 deterministic: bool = False):
        """`deterministic=True` selects the reference-order mode (EMERGE_OPT_DETERMINISTIC):
        every grid cell sums its contributions in the reference's particle index order."""
        config.validate()
        self._lib = load_library(lib_path)
        self.config = config.copy()
        cfg = config.to_c()
        ptr = c_void_p()
        check(self._lib, self._lib.emerge_cuda_create(byref(cfg), int(device), byref(ptr)))
        self._sim = ptr
        self.registry = MaterialRegistry(FallbackMaterial())
        self.boundaries = [SlipBoundary(config.boundary_thickness)]  # lifecycle.rs:29-30
        self.force_fields: list = []  # (name, field) in application order
        self.last_timing: dict | None = None
        if deterministic:
            self.set_option(abi.OPT_DETERMINISTIC, 1)

    # ---------------------------------------------------------------- lifecycle
    @classmethod
    def empty(cls, config: SimConfig, device: int = 0, **kw) -> "Simulation":
        return cls(config, device, **kw)

    @classmethod
    def new(cls, config: SimConfig, spawn: SpawnRegion, device: int = 0, **kw) -> "Simulation":
        """`Simulation::new` (lifecycle.rs:57-99)."""
        s = cls(config, device, **kw)
        if not spawn.fits_in_sim(config):
            raise ValueError("spawn region must stay inside the simulation domain")
        sp = spawn.to_c()
        s._check(s._lib.emerge_cuda_init_with_spawn(s._sim, byref(sp)))
        return s

    def close(self) -> None:
        if getattr(self, "_sim", None):
            self._lib.emerge_cuda_destroy(self._sim)
            self._sim = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, status: int) -> None:
        check(self._lib, status, self._sim)

    # ---------------------------------------------------------------- materials
    def _upload_materials(self) -> None:
        for k, m in enumerate(self.registry.materials):
            if m.constitutive_model() not in DEVICE_MODELS:
                raise abi.EmergeError(abi.ERR_UNSUPPORTED,
                                      f"material {k}: model {m.constitutive_model()} has no "
                                      "device implementation")
        arr = (MaterialParamsC * len(self.registry))(
            *[m.abi_params() for m in self.registry.materials])
        self._check(self._lib.emerge_cuda_set_materials(self._sim, arr, len(self.registry)))
        phases = (c_uint32 * len(self.registry))(*[mixture_phase_of(m) for m in self.registry.materials])
        self._check(self._lib.emerge_cuda_set_mixture_phases(self._sim, phases, len(self.registry)))

    def with_default_material(self, material: Material) -> "Simulation":
        """lifecycle.rs:107-111 (also re-runs init_particle on every particle)."""
        self.registry.set_default(material)
        self._upload_materials()
        return self

    def set_material(self, material_id: int, material: Material) -> None:
        self.registry.insert(material_id, material)
        self._upload_materials()

    def with_material(self, material_id: int, material: Material) -> "Simulation":
        self.set_material(material_id, material)
        return self

    def register_material(self, material: Material) -> int:
        mid = self.registry.next_id()
        self.set_material(mid, material)
        return mid

    # ---------------------------------------------------------------- multi-field contact
    def set_contact_grip(self, grip) -> None:
        """Simulation::with_contact_grip (lifecycle.rs:125-131); None removes the grip."""
        if grip is None:
            self._check(self._lib.emerge_cuda_set_contact_grip(self._sim, 0, 0.0, 0.0, 0.0, 0.0))
        else:
            self._check(self._lib.emerge_cuda_set_contact_grip(
                self._sim, 1, float(grip.mu_easy), float(grip.mu_resist),
                grip.easy_direction[0], grip.easy_direction[1]))

    def with_contact_grip(self, grip) -> "Simulation":
        self.set_contact_grip(grip)
        return self

    # ---------------------------------------------------------------- sleep partition
    def active_count(self) -> int:
        """Simulation::active_count (particles.rs:314)."""
        out = c_uint64()
        self._check(self._lib.emerge_cuda_active_count(self._sim, byref(out)))
        return int(out.value)

    def _replace(self, particles: np.ndarray, active: int) -> None:
        arr = np.ascontiguousarray(particles, dtype=PARTICLE_DTYPE)
        self._check(self._lib.emerge_cuda_replace_particles(
            self._sim, arr.ctypes.data_as(c_void_p), len(arr), int(active)))

    def wake_tag(self, tag: int) -> None:
        self._replace(*lifecycle.wake_tag(self.particles(), self.active_count(), int(tag)))

    def sleep_tag(self, tag: int) -> None:
        self._replace(*lifecycle.sleep_tag(self.particles(), self.active_count(), int(tag)))

    def remove_particles(self, predicate) -> int:
        """remove_particles (particles.rs:177-205); returns the number removed."""
        p, active, removed = lifecycle.remove_particles(self.particles(), self.active_count(), predicate)
        if removed:
            self._replace(p, active)
        return removed

    def retain_particles(self, predicate) -> None:
        """retain_particles (lifecycle.rs:237-253)."""
        self._replace(*lifecycle.retain_particles(self.particles(), self.active_count(), predicate))

    def split_particles(self, should_split, jitter: float) -> None:
        """split_particles (lifecycle.rs:271-310)."""
        self._replace(*lifecycle.split_particles(self.particles(), self.active_count(), should_split,
                                                 jitter))

    # ---------------------------------------------------------------- force fields
    def _upload_fields(self) -> None:
        table, data = pack_fields([f for _, f in self.force_fields])
        arr = (abi.ForceFieldC * max(len(table), 1))(*table)
        d = np.asarray(data if data else [0.0], dtype=np.float32)
        self._check(self._lib.emerge_cuda_set_force_fields(
            self._sim, arr, len(table), d.ctypes.data_as(ctypes.POINTER(c_float)), len(data)))

    def add_named_force_field(self, name: str, field: Field) -> None:
        """lifecycle.rs:374-377."""
        if not isinstance(field, Field):
            raise abi.EmergeError(abi.ERR_UNSUPPORTED,
                                  f"{type(field).__name__} has no device implementation")
        self.force_fields.append((str(name), field))
        self._upload_fields()

    def add_force_field(self, field: Field) -> None:
        """Anonymous field named force_field_N (lifecycle.rs:368-372)."""
        self.add_named_force_field(f"force_field_{len(self.force_fields)}", field)

    def with_force_field(self, field: Field) -> "Simulation":
        self.add_force_field(field)
        return self

    def with_named_force_field(self, name: str, field: Field) -> "Simulation":
        self.add_named_force_field(name, field)
        return self

    def remove_force_field(self, name: str) -> bool:
        """Removes the first field with this name (lifecycle.rs:380-387)."""
        for k, (n, _) in enumerate(self.force_fields):
            if n == name:
                del self.force_fields[k]
                self._upload_fields()
                return True
        return False

    def clear_force_fields(self) -> None:
        self.force_fields = []
        self._upload_fields()

    def force_field_names(self) -> list:
        return [n for n, _ in self.force_fields]

    def field_accelerations(self) -> np.ndarray:
        """(n, 2) float32: the fields' summed Field::acceleration per particle, reference index
        order, at the current state (the n-body tree built from the current positions)."""
        n = self.particle_count()
        out = np.zeros((max(n, 1), 2), dtype=np.float32)
        self._check(self._lib.emerge_cuda_field_accelerations(
            self._sim, out.ctypes.data_as(ctypes.POINTER(c_float)), n))
        return out[:n]

    # ---------------------------------------------------------------- boundaries
    def _upload_boundaries(self) -> None:
        arr = (c_uint64 * max(len(self.boundaries), 1))(*[b.thickness for b in self.boundaries])
        self._check(self._lib.emerge_cuda_set_slip_boundaries(self._sim, arr, len(self.boundaries)))

    def add_boundary_condition(self, boundary: SlipBoundary) -> None:
        if not isinstance(boundary, SlipBoundary):
            raise abi.EmergeError(abi.ERR_UNSUPPORTED, "only SlipBoundary is on the device path")
        self.boundaries.append(boundary)
        self._upload_boundaries()

    def with_boundary(self, boundary: SlipBoundary) -> "Simulation":
        self.add_boundary_condition(boundary)
        return self

    def set_boundary_condition(self, boundary: SlipBoundary) -> None:
        self.boundaries = []
        self.add_boundary_condition(boundary)

    def clear_boundaries(self) -> None:
        self.boundaries = []
        self._upload_boundaries()

    # ---------------------------------------------------------------- particles
    def add_body(self, spawn: SpawnRegion) -> int:
        """`add_body` (particles.rs:355-423); returns the group tag."""
        if not spawn.fits_in_sim(self.config):
            raise ValueError("spawn region must stay inside the simulation domain")
        sp = spawn.to_c()
        tag = c_uint32()
        self._check(self._lib.emerge_cuda_add_body(self._sim, byref(sp), byref(tag)))
        return int(tag.value)

    def add_particles(self, particles: np.ndarray, estimate_volumes: bool = False) -> None:
        arr = np.ascontiguousarray(particles, dtype=PARTICLE_DTYPE)
        self._check(self._lib.emerge_cuda_add_particles(
            self._sim, arr.ctypes.data_as(c_void_p), len(arr), 1 if estimate_volumes else 0))

    def particle_count(self) -> int:
        n = c_uint64()
        self._check(self._lib.emerge_cuda_particle_count(self._sim, byref(n)))
        return int(n.value)

    def particles(self) -> np.ndarray:
        """Copy of every particle in reference index order (structured array)."""
        n = self.particle_count()
        out = np.zeros(n, dtype=PARTICLE_DTYPE)
        if n:
            self._check(self._lib.emerge_cuda_read_particles(
                self._sim, out.ctypes.data_as(c_void_p), n))
        return out

    def set_particles(self, particles: np.ndarray) -> None:
        """Write-back of `particles_mut()` edits (lifecycle.rs:233)."""
        arr = np.ascontiguousarray(particles, dtype=PARTICLE_DTYPE)
        self._check(self._lib.emerge_cuda_write_particles(
            self._sim, arr.ctypes.data_as(c_void_p), len(arr)))

    # ---------------------------------------------------------------- stepping
    def step(self) -> None:
        self.step_n(1)

    def step_n(self, steps: int, timing: bool = False) -> None:
        if timing:
            t = StepTimingC()
            self._check(self._lib.emerge_cuda_step(self._sim, int(steps), byref(t)))
            self.last_timing = {name: int(getattr(t, name)) for name, _ in StepTimingC._fields_}
        else:
            self._check(self._lib.emerge_cuda_step(self._sim, int(steps), None))

    def synchronize(self) -> None:
        self._check(self._lib.emerge_cuda_synchronize(self._sim))

    def last_substeps(self) -> int:
        v = c_uint64()
        self._check(self._lib.emerge_cuda_last_substeps(self._sim, byref(v)))
        return int(v.value)

    def effective_dt(self) -> float:
        v = c_float()
        self._check(self._lib.emerge_cuda_effective_dt(self._sim, byref(v)))
        return float(v.value)

    def last_counters(self) -> tuple[int, int, float]:
        a, b, d = c_uint64(), c_uint64(), c_float()
        self._check(self._lib.emerge_cuda_last_counters(self._sim, byref(a), byref(b), byref(d)))
        return int(a.value), int(b.value), float(d.value)

    # ---------------------------------------------------------------- queries
    def region_state(self, center, radius: float) -> BodyState:
        out = BodyStateC()
        self._check(self._lib.emerge_cuda_region_state(
            self._sim, float(center[0]), float(center[1]), float(radius), byref(out)))
        return BodyState.from_c(out)

    # ---------------------------------------------------------------- tuning
    def set_option(self, option: int, value: int) -> None:
        self._check(self._lib.emerge_cuda_set_option(self._sim, int(option), int(value)))

    def sort_now(self, key_mode: int = 0) -> None:
        self._check(self._lib.emerge_cuda_sort_now(self._sim, int(key_mode)))

    def kernel_launches(self) -> int:
        v = c_uint64()
        self._check(self._lib.emerge_cuda_kernel_launches(self._sim, byref(v)))
        return int(v.value)

    def stream_handle(self) -> int:
        return int(self._lib.emerge_cuda_stream(self._sim) or 0)

    # ---------------------------------------------------------------- measurement
    def event_record(self, slot: int) -> None:
        self._check(self._lib.emerge_cuda_event_record(self._sim, int(slot)))

    def event_elapsed_ms(self, a: int, b: int) -> float:
        v = c_float()
        self._check(self._lib.emerge_cuda_event_elapsed(self._sim, int(a), int(b), byref(v)))
        return float(v.value)

    def flush_l2(self) -> None:
        self._check(self._lib.emerge_cuda_flush_l2(self._sim))

    def stats(self) -> dict:
        st = abi.StatsC()
        self._check(self._lib.emerge_cuda_stats(self._sim, byref(st)))
        return {name: int(getattr(st, name)) for name, _ in abi.StatsC._fields_}

    def write_particles_raw(self, ptr: int, n: int) -> None:
        """Upload `n` particles from host memory at address `ptr` (AoS, 128 B each)."""
        self._check(self._lib.emerge_cuda_write_particles(self._sim, c_void_p(ptr), int(n)))

    def read_particles_raw(self, ptr: int, n: int) -> None:
        """Read back `n` particles into host memory at address `ptr` (AoS, 128 B each)."""
        self._check(self._lib.emerge_cuda_read_particles(self._sim, c_void_p(ptr), int(n)))

    def read_particles_raw_async(self, ptr: int, n: int) -> None:
        """Enqueue the readback of `n` particles into host memory at `ptr` (AoS, 128 B each);
        the memory holds them after the next synchronize()."""
        self._check(self._lib.emerge_cuda_read_particles_async(self._sim, c_void_p(ptr), int(n)))

    # ---------------------------------------------------------------- learned closure
    # No counterpart in the reference: a network standing in for the smooth plastic branch
    # of the Drucker-Prager (model 0) and NACC (model 1) return mappings.
    def closure_log(self, capacity: int, stride: int = 1) -> None:
        """Log (inputs, targets) of the plain mapping during the following steps."""
        self._check(self._lib.emerge_cuda_closure_log(self._sim, int(capacity), int(stride)))

    def closure_train(self, model: int, epochs: int = 20, batch: int = 4096, lr: float = 2e-3,
                      lr_decay: float = 0.9, seed: int = 1, val_fraction: float = 0.1,
                      max_samples: int = 0, beta1: float = 0.9, beta2: float = 0.999,
                      eps: float = 1e-8) -> dict:
        cfg = abi.ClosureTrainConfigC(epochs=epochs, batch=batch, lr=lr, lr_decay=lr_decay,
                                      beta1=beta1, beta2=beta2, eps=eps, val_fraction=val_fraction,
                                      seed=seed, max_samples=max_samples)
        rep = abi.ClosureTrainReportC()
        self._check(self._lib.emerge_cuda_closure_train(self._sim, int(model), byref(cfg), byref(rep)))
        return {name: getattr(rep, name) for name, _ in abi.ClosureTrainReportC._fields_}

    def closure_enable(self, on: bool = True, judge_stride: int = 64) -> None:
        self._check(self._lib.emerge_cuda_closure_enable(self._sim, 1 if on else 0, int(judge_stride)))

    def closure_set_mode(self, defer: bool = True, judge_bar: float = 1e-3) -> None:
        """Deferred tensor-core evaluation (tile kernel) or evaluation inside the particle
        pass, and the judge's replacement bar (emerge_cuda_closure_set_mode)."""
        self._check(self._lib.emerge_cuda_closure_set_mode(self._sim, 1 if defer else 0, float(judge_bar)))

    def closure_stats(self, reset: bool = False) -> dict:
        st = abi.ClosureStatsC()
        self._check(self._lib.emerge_cuda_closure_stats(self._sim, byref(st), 1 if reset else 0))
        out = {name: getattr(st, name) for name, _ in abi.ClosureStatsC._fields_ if name != "pad_"}
        out["logged"] = [int(v) for v in st.logged]
        return out

    def closure_log_samples(self, model: int, max_samples: int = 1 << 20) -> tuple[np.ndarray, np.ndarray]:
        x = np.zeros((max_samples, 6), np.float32)
        t = np.zeros((max_samples, 3), np.float32)
        n = c_uint64()
        self._check(self._lib.emerge_cuda_closure_get_log(
            self._sim, int(model), x.ctypes.data_as(c_void_p), t.ctypes.data_as(c_void_p),
            int(max_samples), byref(n)))
        return x[:n.value].copy(), t[:n.value].copy()

    def closure_params(self, model: int) -> tuple[np.ndarray, np.ndarray]:
        params = np.zeros(abi.CLOSURE_NPARAMS, np.float32)
        norm = np.zeros(abi.CLOSURE_NNORM, np.float32)
        self._check(self._lib.emerge_cuda_closure_get_params(
            self._sim, int(model), params.ctypes.data_as(c_void_p), norm.ctypes.data_as(c_void_p)))
        return params, norm

    def set_closure_params(self, model: int, params: np.ndarray, norm: np.ndarray,
                           hull: np.ndarray) -> None:
        p = np.ascontiguousarray(params, np.float32)
        nm = np.ascontiguousarray(norm, np.float32)
        h = np.ascontiguousarray(hull, np.float32)
        assert p.size == abi.CLOSURE_NPARAMS and nm.size == abi.CLOSURE_NNORM and h.size == 12
        self._check(self._lib.emerge_cuda_closure_set_params(
            self._sim, int(model), p.ctypes.data_as(c_void_p), nm.ctypes.data_as(c_void_p),
            h.ctypes.data_as(c_void_p)))


class PinnedBuffer:
    """Page-locked host buffer from the CUDA library (cudaMallocHost)."""

    def __init__(self, nbytes: int):
        self._lib = load_library()
        ptr = c_void_p()
        check(self._lib, self._lib.emerge_cuda_host_alloc(int(nbytes), byref(ptr)))
        self.ptr = int(ptr.value)
        self.nbytes = int(nbytes)

    def as_particles(self, n: int) -> np.ndarray:
        buf = (ctypes.c_char * (n * PARTICLE_DTYPE.itemsize)).from_address(self.ptr)
        return np.frombuffer(buf, dtype=PARTICLE_DTYPE, count=n)

    def free(self) -> None:
        if self.ptr:
            self._lib.emerge_cuda_host_free(c_void_p(self.ptr))
            self.ptr = 0

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class DeterministicSimulation(Simulation):
    """`Simulation` in the reference-order mode (per-cell sums in particle index order)."""

    def __init__(self, config: SimConfig, device: int = 0, lib_path: str | None = None,
                 deterministic: bool = True):
        super().__init__(config, device, lib_path, deterministic=True)


# ---------------------------------------------------------------- closure test hooks
def mlp_loss_grad(params: np.ndarray, x: np.ndarray, t: np.ndarray) -> tuple[float, np.ndarray]:
    """Device loss and gradient of the closure MLP on one batch (normalised data)."""
    lib = load_library()
    p = np.ascontiguousarray(params, np.float32)
    xx = np.ascontiguousarray(x, np.float32)
    tt = np.ascontiguousarray(t, np.float32)
    loss = c_float()
    grad = np.zeros(abi.CLOSURE_NPARAMS, np.float32)
    check(lib, lib.emerge_cuda_mlp_loss_grad(p.ctypes.data_as(c_void_p), xx.ctypes.data_as(c_void_p),
                                             tt.ctypes.data_as(c_void_p), len(xx), byref(loss),
                                             grad.ctypes.data_as(c_void_p)))
    return float(loss.value), grad


def mlp_adam(params, m, v, grad, step, lr, beta1=0.9, beta2=0.999, eps=1e-8):
    """One device Adam step; returns updated (params, m, v)."""
    lib = load_library()
    p = np.array(params, np.float32)
    mm = np.array(m, np.float32)
    vv = np.array(v, np.float32)
    g = np.ascontiguousarray(grad, np.float32)
    check(lib, lib.emerge_cuda_mlp_adam(p.ctypes.data_as(c_void_p), mm.ctypes.data_as(c_void_p),
                                        vv.ctypes.data_as(c_void_p), g.ctypes.data_as(c_void_p),
                                        len(p), int(step), lr, beta1, beta2, eps))
    return p, mm, vv


def mlp_infer_tc(params: np.ndarray, x: np.ndarray) -> np.ndarray:
    """The closure MLP on normalised inputs as the closure's tile kernel evaluates it
    (tcgen05 tensor cores, 128 rows per tile)."""
    lib = load_library()
    p = np.ascontiguousarray(params, np.float32)
    xx = np.ascontiguousarray(x, np.float32)
    y = np.zeros((len(xx), 3), np.float32)
    check(lib, lib.emerge_cuda_mlp_infer_tc(p.ctypes.data_as(c_void_p), xx.ctypes.data_as(c_void_p),
                                            len(xx), y.ctypes.data_as(c_void_p)))
    return y


def silu_fast(x: np.ndarray) -> np.ndarray:
    """The closure tile kernel's SiLU (hardware tanh) on float32 values."""
    lib = load_library()
    xx = np.ascontiguousarray(x, np.float32).ravel()
    y = np.zeros_like(xx)
    check(lib, lib.emerge_cuda_silu_fast(xx.ctypes.data_as(c_void_p), len(xx), y.ctypes.data_as(c_void_p)))
    return y


def mlp_infer_bf16(params: np.ndarray, x: np.ndarray) -> np.ndarray:
    """The BF16 tensor-core inference of the closure MLP on normalised inputs."""
    lib = load_library()
    p = np.ascontiguousarray(params, np.float32)
    xx = np.ascontiguousarray(x, np.float32)
    y = np.zeros((len(xx), 3), np.float32)
    check(lib, lib.emerge_cuda_mlp_infer_bf16(p.ctypes.data_as(c_void_p), xx.ctypes.data_as(c_void_p),
                                              len(xx), y.ctypes.data_as(c_void_p)))
    return y


class Batch:
    """Many independent scenes advanced together (one launch per kernel per substep for
    all scenes).  Built from simulations set up with the single-scene API; their particles
    are copied, and they stay independent of the batch."""

    def __init__(self, sims):
        self._lib = load_library()
        arr = (c_void_p * len(sims))(*[s._sim for s in sims])
        ptr = c_void_p()
        st = self._lib.emerge_cuda_batch_create(arr, len(sims), byref(ptr))
        if st != abi.OK:
            raise abi.EmergeError(st, (self._lib.emerge_cuda_batch_last_error(None) or b"").decode())
        self._b = ptr
        self.n_scenes = len(sims)

    def _check(self, status: int) -> None:
        if status != abi.OK:
            raise abi.EmergeError(status, (self._lib.emerge_cuda_batch_last_error(self._b) or b"").decode())

    def close(self) -> None:
        if getattr(self, "_b", None):
            self._lib.emerge_cuda_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n: int = 1) -> None:
        self._check(self._lib.emerge_cuda_batch_step(self._b, int(n)))

    def time_steps(self, n: int, flush_l2: bool = True) -> float:
        """GPU milliseconds summed over n frames (CUDA events, optional L2 flush before each)."""
        ms = c_float()
        self._check(self._lib.emerge_cuda_batch_time_steps(self._b, int(n), 1 if flush_l2 else 0, byref(ms)))
        return float(ms.value)

    def particle_count(self, scene: int) -> int:
        n = c_uint64()
        self._check(self._lib.emerge_cuda_batch_particle_count(self._b, int(scene), byref(n)))
        return int(n.value)

    def particles(self, scene: int) -> np.ndarray:
        n = self.particle_count(scene)
        out = np.zeros(n, dtype=PARTICLE_DTYPE)
        self._check(self._lib.emerge_cuda_batch_read_particles(self._b, int(scene), out.ctypes.data_as(c_void_p), n))
        return out

    def region_state(self, scene: int, center, radius: float) -> BodyState:
        out = BodyStateC()
        self._check(self._lib.emerge_cuda_batch_region_state(
            self._b, int(scene), float(center[0]), float(center[1]), float(radius), byref(out)))
        return BodyState.from_c(out)

    def substeps(self) -> tuple[np.ndarray, np.ndarray]:
        """Per scene: substeps of the last frame and lifetime substeps."""
        last = np.zeros(self.n_scenes, np.uint64)
        total = np.zeros(self.n_scenes, np.uint64)
        self._check(self._lib.emerge_cuda_batch_substeps(self._b, last.ctypes.data_as(c_void_p),
                                                         total.ctypes.data_as(c_void_p)))
        return last, total

    def set_option(self, option: int, value: int) -> None:
        self._check(self._lib.emerge_cuda_batch_set_option(self._b, int(option), int(value)))

    def autotune(self, steps_per_trial: int = 2, cache_path: str | None = None) -> dict:
        """Tile shape, particles per CTA, sort interval and P2G aggregation for this batch
        (emerge_cuda_batch_autotune); `cache_path`: the tuning cache file (None = none)."""
        rep = abi.BatchTuneReportC()
        path = cache_path.encode() if cache_path else None
        self._check(self._lib.emerge_cuda_batch_autotune(self._b, int(steps_per_trial), path, byref(rep)))
        n = rep.n_trials
        return {"sort_interval": rep.sort_interval, "aggregate": rep.aggregate,
                "tile_shape": rep.tile_shape, "chunks_per_cta": rep.chunks_per_cta,
                "particles_per_cta": 256 * rep.chunks_per_cta, "from_cache": bool(rep.from_cache),
                "best_ms_per_step": rep.best_ms,
                "trials": [{"tile_shape": rep.trial_tile_shape[k], "chunks_per_cta": rep.trial_chunks[k],
                            "sort_interval": rep.trial_sort_interval[k], "aggregate": rep.trial_aggregate[k],
                            "ms_per_step": rep.trial_ms[k]} for k in range(n)]}
