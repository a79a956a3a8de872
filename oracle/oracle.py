"""Python side of the CPU parity oracle -- TEST INFRASTRUCTURE ONLY.

Only tests, the smoke check and the CPU-baseline leg of bench.py use this module, and only as the checker.

It restates the host orchestration of chadmv/plume's hot path (the Python around the Warp kernels) over numpy
arrays, calling the C++ restatement of each kernel in oracle/plume_oracle.cpp through ctypes:

    grid and fields        src/plume/sim/grid.py:36-94
    emitters               src/plume/sim/emitters.py:124-153
    forces, drag           src/plume/sim/forces.py:26-48
    vorticity confinement  src/plume/sim/vorticity.py:87-117
    turbulence             src/plume/sim/turbulence.py:59-67
    advection              src/plume/sim/advect.py:53-76
    projection             src/plume/sim/pressure.py:119-162, pressure_solver.py:9-13
    multigrid              src/plume/sim/multigrid.py:71-147
    smoke budget           src/plume/sim/conserve.py:33-52, reduce.py:28-38
    dissipation            src/plume/sim/dissipate.py:18-24
    CFL step cap           src/plume/sim/step_cap.py:22-66
    stepper, frame loop    src/plume/sim/stepper.py:17-60, run.py:22-85
    render                 src/plume/render/frame_renderer.py:16-94, light_volume.py:36-51,
                           normal_field.py:41-69

`precision="f32"` reproduces the reference's FP32 arithmetic (scalars are rounded to float32 where the
reference stores them in float32 struct fields or kernel arguments); `precision="f64"` runs the same
method in double precision.
"""

import ctypes
import math
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from plume_b200.recipe.schema import SHADE_LAYOUT

LIB_PATH = Path(__file__).resolve().parent / "libplume_oracle.so"
_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"the oracle library {LIB_PATH} is not built (run `make -C oracle`)")
        _lib = ctypes.CDLL(str(LIB_PATH))
        for name in ("oracle_total_f32", "oracle_total_f64", "oracle_abs_max_f32", "oracle_abs_max_f64"):
            getattr(_lib, name).restype = ctypes.c_double
    return _lib


def set_threads(count: int) -> int:
    return lib().oracle_threads(count)


class OInfo(ctypes.Structure):
    _fields_ = [("dims", ctypes.c_int * 3), ("cell_m", ctypes.c_double), ("origin_m", ctypes.c_double * 3),
                ("open_lo", ctypes.c_int * 3), ("open_hi", ctypes.c_int * 3), ("fill_hi", ctypes.c_double * 3),
                ("ghost_gap", ctypes.c_double)]


class OEmitter(ctypes.Structure):
    _fields_ = [("shape", ctypes.c_int), ("center_m", ctypes.c_double * 3), ("radius_m", ctypes.c_double),
                ("half_size_m", ctypes.c_double * 3), ("edge_softness", ctypes.c_double),
                ("start_s", ctypes.c_double), ("end_s", ctypes.c_double), ("smoke_per_s", ctypes.c_double),
                ("temperature_k", ctypes.c_double), ("velocity_mps", ctypes.c_double * 3),
                ("outward", ctypes.c_int), ("noise_scale_m", ctypes.c_double),
                ("noise_strength", ctypes.c_double), ("stream", ctypes.c_int)]


class OView(ctypes.Structure):
    _fields_ = [("right", ctypes.c_double * 3), ("up", ctypes.c_double * 3), ("toward", ctypes.c_double * 3),
                ("left_m", ctypes.c_double), ("top_m", ctypes.c_double), ("pixel_m", ctypes.c_double),
                ("perspective", ctypes.c_int), ("eye", ctypes.c_double * 3)]


class OLook(ctypes.Structure):
    _fields_ = [("opacity_per_density", ctypes.c_double), ("glow_start_k", ctypes.c_double),
                ("smoke_hides_heat", ctypes.c_double), ("normal_fade_thickness", ctypes.c_double),
                ("shade_layout", ctypes.c_int), ("shade_fill", ctypes.c_double)]


def _ptr(array: np.ndarray) -> ctypes.c_void_p:
    assert array.flags["C_CONTIGUOUS"]
    return ctypes.c_void_p(array.ctypes.data)


def _shape(array: np.ndarray):
    return (ctypes.c_int * 3)(*array.shape[:3])


def _d3(values):
    return (ctypes.c_double * 3)(*[float(v) for v in values])


class Precision:
    def __init__(self, name: str):
        assert name in ("f32", "f64")
        self.name = name
        self.dtype = np.float32 if name == "f32" else np.float64

    def round(self, value: float) -> float:
        """The value a float32 struct field or kernel argument holds (f32), or the value itself (f64)."""
        return float(np.float32(value)) if self.name == "f32" else float(value)

    def fn(self, stem: str):
        return getattr(lib(), f"oracle_{stem}_{self.name}")


U_FACE, V_FACE, W_FACE, CENTER = (0.0, 0.5, 0.5), (0.5, 0.0, 0.5), (0.5, 0.5, 0.0), (0.5, 0.5, 0.5)


class Field:
    """An advected quantity with MacCormack's scratch arrays (grid.py:36-51)."""

    def __init__(self, shape, offset, outside, uses_outside, dtype, initial=0.0):
        self.offset = offset
        self.outside = outside
        self.uses_outside = 1 if uses_outside else 0
        self.data = np.full(shape, initial, dtype=dtype)
        self.hat = np.zeros(shape, dtype=dtype)
        self.back = np.zeros(shape, dtype=dtype)
        self.next = np.zeros(shape, dtype=dtype)

    def swap(self):
        self.data, self.next = self.next, self.data


class Grid:
    def __init__(self, info: OInfo, cells, precision: Precision, ambient_k: float):
        self.info = info
        self.cells = tuple(cells)
        self.precision = precision
        dtype = precision.dtype
        nx, ny, nz = cells
        self.u = Field((nx + 1, ny, nz), U_FACE, 0.0, False, dtype)
        self.v = Field((nx, ny + 1, nz), V_FACE, 0.0, False, dtype)
        self.w = Field((nx, ny, nz + 1), W_FACE, 0.0, False, dtype)
        self.smoke = Field(cells, CENTER, 0.0, True, dtype)
        self.temperature = Field(cells, CENTER, precision.round(ambient_k), True, dtype,
                                 initial=precision.round(ambient_k))
        self.pressure = np.zeros(cells, dtype=dtype)
        self.divergence = np.zeros(cells, dtype=dtype)

    @property
    def cell_m(self) -> float:
        return self.info.cell_m

    def velocity_fields(self):
        return self.u, self.v, self.w


def make_info(cells, cell_m, origin_m, open_lo, open_hi, precision: Precision, fill_hi=(1.0, 1.0, 1.0),
              ghost_gap=0.5) -> OInfo:
    info = OInfo()
    info.dims = (ctypes.c_int * 3)(*cells)
    info.cell_m = precision.round(cell_m)
    info.origin_m = _d3(precision.round(o) for o in origin_m)
    info.open_lo = (ctypes.c_int * 3)(*open_lo)
    info.open_hi = (ctypes.c_int * 3)(*open_hi)
    info.fill_hi = _d3(precision.round(f) for f in fill_hi)
    info.ghost_gap = precision.round(ghost_gap)
    return info


def _is_open(kind: str) -> int:
    return 1 if kind == "open" else 0


def make_grid(derived, cell_m, faces, ambient_k, precision="f32") -> Grid:
    p = Precision(precision) if isinstance(precision, str) else precision
    info = make_info(derived.cells, cell_m, derived.domain_min_m,
                     [_is_open(k) for k in (faces.left, faces.bottom, faces.back)],
                     [_is_open(k) for k in (faces.right, faces.top, faces.front)], p)
    return Grid(info, derived.cells, p, ambient_k)


# ---- operators -------------------------------------------------------------------------------------------


def advect_semi_lagrangian(field: Field, velocity, grid: Grid, dt: float) -> None:
    u, v, w = velocity
    grid.precision.fn("semi_lagrangian")(
        ctypes.byref(grid.info), _shape(field.data), _ptr(field.data), _ptr(field.next), _ptr(u), _ptr(v),
        _ptr(w), ctypes.c_double(dt / grid.cell_m), _d3(field.offset), ctypes.c_double(field.outside),
        field.uses_outside)


def advect_maccormack(field: Field, velocity, grid: Grid, dt: float) -> None:
    u, v, w = velocity
    grid.precision.fn("maccormack")(
        ctypes.byref(grid.info), _shape(field.data), _ptr(field.data), _ptr(field.hat), _ptr(field.back),
        _ptr(field.next), _ptr(u), _ptr(v), _ptr(w), ctypes.c_double(dt / grid.cell_m), _d3(field.offset),
        ctypes.c_double(field.outside), field.uses_outside)


def emitter_params(emitters) -> ctypes.Array:
    out = (OEmitter * len(emitters))()
    for index, s in enumerate(emitters):
        e = out[index]
        e.shape = 0 if s.shape == "sphere" else 1
        e.center_m = _d3(s.center_m)
        e.radius_m = s.radius_m
        e.half_size_m = _d3(size / 2 for size in s.size_m)
        e.edge_softness = s.edge_softness
        e.start_s, e.end_s = s.start_s, s.end_s
        e.smoke_per_s = s.smoke_per_s
        e.temperature_k = s.temperature_k
        e.velocity_mps = _d3(s.velocity_mps)
        e.outward = 1 if s.velocity_mode == "outward" else 0
        e.noise_scale_m, e.noise_strength = s.noise.scale_m, s.noise.strength
        e.stream = index
    return out


def _rounded_emitters(params, precision: Precision):
    """Copies the emitters with every real rounded as the float32 struct fields hold it."""
    out = (OEmitter * len(params))()
    ctypes.memmove(out, params, ctypes.sizeof(out))
    if precision.name == "f32":
        for e in out:
            for name, kind in OEmitter._fields_:
                if kind is ctypes.c_double:
                    setattr(e, name, precision.round(getattr(e, name)))
                elif kind is ctypes.c_double * 3:
                    setattr(e, name, _d3(precision.round(x) for x in getattr(e, name)))
    return out


def emit(grid: Grid, params, seed: int, time_s: float, dt: float) -> None:
    rounded = _rounded_emitters(params, grid.precision)
    grid.precision.fn("emit")(
        ctypes.byref(grid.info), _ptr(grid.smoke.data), _ptr(grid.temperature.data), _ptr(grid.u.data),
        _ptr(grid.v.data), _ptr(grid.w.data), rounded, len(params), int(seed), ctypes.c_double(time_s),
        ctypes.c_double(dt))


def apply_buoyancy(grid: Grid, gravity, heat_buoyancy, smoke_weight, ambient_k, dt) -> None:
    grid.precision.fn("buoyancy")(
        ctypes.byref(grid.info), _ptr(grid.v.data), _ptr(grid.smoke.data), _ptr(grid.temperature.data),
        *(ctypes.c_double(x) for x in (gravity, heat_buoyancy, smoke_weight, ambient_k, dt)))


def apply_drag(grid: Grid, wind_mps, drag_per_s: float, dt: float) -> None:
    if drag_per_s == 0.0:
        return
    keep = math.exp(-drag_per_s * dt)
    for axis, field in enumerate(grid.velocity_fields()):
        grid.precision.fn("drag")(_shape(field.data), _ptr(field.data), ctypes.c_double(float(wind_mps[axis])),
                                  ctypes.c_double(keep))


class VorticityConfinement:
    def __init__(self, grid: Grid):
        shape = (*grid.cells, 3)
        self.center = np.zeros(shape, dtype=grid.precision.dtype)
        self.curl = np.zeros(shape, dtype=grid.precision.dtype)
        self.push = np.zeros(shape, dtype=grid.precision.dtype)

    def _run(self, grid: Grid, strength: float, dt: float, apply: int) -> None:
        grid.precision.fn("confinement")(
            ctypes.byref(grid.info), _ptr(grid.u.data), _ptr(grid.v.data), _ptr(grid.w.data), _ptr(self.center),
            _ptr(self.curl), _ptr(self.push), ctypes.c_double(strength), ctypes.c_double(dt), apply)

    def apply(self, grid: Grid, strength: float, dt: float) -> None:
        if strength == 0.0:
            return
        self._run(grid, strength, dt, 1)

    def measure_curl(self, grid: Grid) -> np.ndarray:
        self._run(grid, 0.0, 0.0, 0)
        return self.curl


def apply_turbulence(grid: Grid, seed, scale_m, strength_mps2, speed_mps, time_s, dt) -> None:
    if strength_mps2 == 0.0:
        return
    pattern_time = time_s * speed_mps / scale_m
    grid.precision.fn("turbulence")(
        ctypes.byref(grid.info), _ptr(grid.u.data), _ptr(grid.v.data), _ptr(grid.w.data), int(seed),
        *(ctypes.c_double(x) for x in (scale_m, strength_mps2, pattern_time, dt)))


def compute_divergence(grid: Grid) -> np.ndarray:
    grid.precision.fn("divergence")(ctypes.byref(grid.info), _ptr(grid.u.data), _ptr(grid.v.data),
                                    _ptr(grid.w.data), _ptr(grid.divergence))
    return grid.divergence


class GaussSeidel:
    RELAXATION = 1.5

    def __init__(self, iterations: int):
        self.iterations = iterations

    def __call__(self, grid: Grid) -> None:
        grid.precision.fn("red_black_sweeps")(ctypes.byref(grid.info), _ptr(grid.pressure), _ptr(grid.divergence),
                                              self.iterations, ctypes.c_double(self.RELAXATION))


@dataclass
class Level:
    info: OInfo
    cells: tuple
    q: np.ndarray
    rhs: np.ndarray
    residual: np.ndarray


def coarse_cells(cells):
    return tuple((n + 1) // 2 for n in cells)


class Multigrid:
    MIN_LEVEL_CELLS = 2
    MAX_LEVELS = 8

    def __init__(self, grid: Grid, cycles: int, sweeps: int):
        self.cycles, self.sweeps = cycles, sweeps
        p = grid.precision
        self.levels = [Level(grid.info, grid.cells, grid.pressure, grid.divergence,
                             np.zeros(grid.cells, dtype=p.dtype))]
        while min(self.levels[-1].cells) > self.MIN_LEVEL_CELLS and len(self.levels) < self.MAX_LEVELS:
            above = self.levels[-1]
            cells = coarse_cells(above.cells)
            scale = 2.0 ** len(self.levels)
            fill = [top / scale - (n - 1) for top, n in zip(grid.cells, cells)]
            info = make_info(cells, above.info.cell_m * 2.0, list(above.info.origin_m), list(above.info.open_lo),
                             list(above.info.open_hi), p, fill_hi=fill, ghost_gap=0.5 / scale)
            self.levels.append(Level(info, cells, *(np.zeros(cells, dtype=p.dtype) for _ in range(3))))

    def __call__(self, grid: Grid) -> None:
        self.levels[0].q = grid.pressure
        self.levels[0].rhs = grid.divergence
        n = len(self.levels)
        infos = (OInfo * n)(*[lv.info for lv in self.levels])
        arrays = [(ctypes.c_void_p * n)(*[lv_arr.ctypes.data for lv_arr in column])
                  for column in ([lv.q for lv in self.levels], [lv.rhs for lv in self.levels],
                                 [lv.residual for lv in self.levels])]
        grid.precision.fn("multigrid")(n, infos, *arrays, self.cycles, self.sweeps)

    def residual(self, grid: Grid) -> np.ndarray:
        top = self.levels[0]
        grid.precision.fn("residual")(ctypes.byref(top.info), _ptr(top.q), _ptr(top.rhs), _ptr(top.residual))
        return top.residual


def make_pressure_solve(grid: Grid, solver):
    if solver.pressure_solver == "gauss_seidel":
        return GaussSeidel(solver.pressure_iterations)
    return Multigrid(grid, solver.multigrid_cycles, solver.multigrid_sweeps)


def project(grid: Grid, solve) -> None:
    u, v, w = (f.data for f in grid.velocity_fields())
    grid.precision.fn("zero_closed_faces")(ctypes.byref(grid.info), _ptr(u), _ptr(v), _ptr(w))
    compute_divergence(grid)
    solve(grid)
    grid.precision.fn("subtract_gradient")(ctypes.byref(grid.info), _ptr(u), _ptr(v), _ptr(w), _ptr(grid.pressure))


def total(array: np.ndarray, precision: Precision) -> float:
    return precision.fn("total")(_shape(array), _ptr(array))


def held_total(before: float, semi_lagrangian: float, maccormack: float) -> float:
    return max(semi_lagrangian, min(maccormack, before))


class SmokeBudget:
    def __init__(self, grid: Grid):
        self.last_factor = 1.0

    def hold(self, grid: Grid) -> None:
        s, p = grid.smoke, grid.precision
        before, sl, mc = total(s.data, p), total(s.hat, p), total(s.next, p)
        target = held_total(before, sl, mc)
        self.last_factor = target / mc if mc > 0.0 else 1.0
        if self.last_factor != 1.0:
            p.fn("scale")(_shape(s.next), _ptr(s.next), ctypes.c_double(self.last_factor))


def dissipate(grid: Grid, smoke_per_s, cooling_per_s, ambient_k, dt) -> None:
    if smoke_per_s == 0.0 and cooling_per_s == 0.0:
        return
    grid.precision.fn("dissipate")(_shape(grid.smoke.data), _ptr(grid.smoke.data), _ptr(grid.temperature.data),
                                   ctypes.c_double(math.exp(-smoke_per_s * dt)),
                                   ctypes.c_double(math.exp(-cooling_per_s * dt)), ctypes.c_double(ambient_k))


class Stepper:
    def __init__(self, grid: Grid, recipe, before_step=None):
        """`before_step(grid, time_s, dt)`, when given, runs at the start of every substep (a test's source
        field, added before the emitters)."""
        self.grid, self.recipe = grid, recipe
        self.before_step = before_step
        self.emitters = emitter_params(recipe.emitter)
        self.pressure_solve = make_pressure_solve(grid, recipe.solver)
        self.smoke_budget = SmokeBudget(grid)
        self.confinement = VorticityConfinement(grid) if recipe.forces.vorticity_confinement > 0 else None

    def step(self, time_s: float, dt: float) -> None:
        grid, recipe = self.grid, self.recipe
        ambient = recipe.domain.ambient_k
        if self.before_step is not None:
            self.before_step(grid, time_s, dt)
        emit(grid, self.emitters, recipe.seed, time_s, dt)
        f = recipe.forces
        apply_buoyancy(grid, f.gravity_mps2, f.heat_buoyancy, f.smoke_weight, ambient, dt)
        if self.confinement is not None:
            self.confinement.apply(grid, f.vorticity_confinement, dt)
        t = f.turbulence
        apply_turbulence(grid, recipe.seed, t.scale_m, t.strength_mps2, t.speed_mps, time_s, dt)
        apply_drag(grid, f.wind_mps, f.drag_per_s, dt)
        fields = grid.velocity_fields()
        velocity = tuple(field.data for field in fields)
        for field in fields:
            advect_maccormack(field, velocity, grid, dt)
        for field in fields:
            field.swap()
        project(grid, self.pressure_solve)
        velocity = tuple(field.data for field in fields)
        advect_maccormack(grid.smoke, velocity, grid, dt)
        self.smoke_budget.hold(grid)
        grid.smoke.swap()
        advect_maccormack(grid.temperature, velocity, grid, dt)
        grid.temperature.swap()
        d = recipe.dissipation
        dissipate(grid, d.smoke_per_s, d.cooling_per_s, ambient, dt)


class RecipeCapError(Exception):
    pass


@dataclass(frozen=True)
class StepLog:
    warmup_steps: int
    steps_per_frame: tuple
    base_steps_per_frame: int
    base_warmup_steps: int

    @property
    def total_steps(self) -> int:
        return self.warmup_steps + sum(self.steps_per_frame)


class StepCap:
    def __init__(self, recipe):
        self.cell_m = recipe.domain.cell_m
        self.max_cells = recipe.solver.max_cells_per_step
        self.max_substeps = recipe.solver.max_substeps
        self.emitters = []
        for e in recipe.emitter:
            vel = np.asarray(e.velocity_mps, dtype=np.float64)
            speed = float(np.linalg.norm(vel)) if e.velocity_mode == "outward" else float(np.abs(vel).max())
            self.emitters.append((e.start_s, e.end_s, speed))

    @staticmethod
    def grid_speed(grid: Grid) -> float:
        return max(grid.precision.fn("abs_max")(_shape(f.data), _ptr(f.data)) for f in grid.velocity_fields())

    def plan(self, grid: Grid, start_s: float, length_s: float, base_steps: int, label: str) -> int:
        emitter = max([s for b, e, s in self.emitters if b < start_s + length_s and e > start_s], default=0.0)
        speed = max(self.grid_speed(grid), emitter)
        steps = max(base_steps, math.ceil(speed * length_s / (self.max_cells * self.cell_m)))
        if steps > max(self.max_substeps, base_steps):
            raise RecipeCapError(f"{label} needs {steps} steps; solver.max_substeps is {self.max_substeps}")
        return steps


def simulate_frames(recipe, derived, precision="f32"):
    grid = make_grid(derived, recipe.domain.cell_m, recipe.domain.faces, recipe.domain.ambient_k, precision)
    stepper = Stepper(grid, recipe)
    cap = StepCap(recipe)
    done = 0

    def run_block(base_steps: int, label: str) -> int:
        nonlocal done
        start_s, length_s = done * derived.dt_s, base_steps * derived.dt_s
        steps = cap.plan(grid, start_s, length_s, base_steps, label)
        for index in range(steps):
            if steps == base_steps:
                stepper.step((done + index) * derived.dt_s, derived.dt_s)
            else:
                stepper.step(start_s + index * length_s / steps, length_s / steps)
        done += base_steps
        return steps

    warmup, remaining = 0, derived.warmup_steps
    while remaining > 0:
        block = min(remaining, derived.steps_per_frame)
        warmup += run_block(block, "warmup")
        remaining -= block
    frames = []
    for frame in range(recipe.time.frames):
        frames.append(run_block(derived.steps_per_frame, f"frame {frame}"))
        yield frame, grid
    return StepLog(warmup, tuple(frames), derived.steps_per_frame, derived.warmup_steps)


def simulate(recipe, derived, capture, precision="f32") -> StepLog:
    frames = simulate_frames(recipe, derived, precision)
    while True:
        try:
            frame, grid = next(frames)
        except StopIteration as finished:
            return finished.value
        capture(frame, grid)


# ---- render ----------------------------------------------------------------------------------------------


def toward_light_world(camera, light_dir) -> np.ndarray:
    x, y, z = light_dir
    return x * camera.right + y * camera.up + z * camera.toward


def domain_view_params(view) -> OView:
    params = OView()
    params.right, params.up, params.toward = _d3(view.camera.right), _d3(view.camera.up), _d3(view.camera.toward)
    params.left_m, params.top_m, params.pixel_m = view.left_m, view.top_m, view.pixel_m
    params.perspective = 0
    params.eye = _d3((0.0, 0.0, 0.0))
    return params


def light_volume(smoke: np.ndarray, toward_light_world, cell_m: float, opacity: float, precision="f32") -> np.ndarray:
    """LightVolume.compute (light_volume.py:36-51) on a standalone smoke array."""
    p = Precision(precision) if isinstance(precision, str) else precision
    direction = np.asarray(toward_light_world, dtype=np.float64)
    light = np.zeros(smoke.shape, dtype=p.dtype)
    p.fn("light_volume")(_shape(smoke), _ptr(smoke), _d3(direction / np.linalg.norm(direction)),
                         ctypes.c_double(cell_m), ctypes.c_double(opacity), _ptr(light))
    return light


def gaussian_weights(sigma: float, radius: int) -> np.ndarray:
    if radius == 0:
        return np.ones(1, dtype=np.float64)
    offsets = np.arange(-radius, radius + 1, dtype=np.float64)
    weights = np.exp(-offsets**2 / (2.0 * sigma**2))
    return weights / weights.sum()


class FrameRenderer:
    def __init__(self, view, settings, cells, channels, precision="f32"):
        self.p = Precision(precision) if isinstance(precision, str) else precision
        dtype = self.p.dtype
        self.shade_layout = channels == SHADE_LAYOUT
        self.view_params = domain_view_params(view)
        look = OLook()
        look.opacity_per_density = settings.opacity_per_density
        look.glow_start_k = settings.glow_start_k
        look.smoke_hides_heat = settings.smoke_hides_heat
        look.normal_fade_thickness = settings.normal_fade_thickness
        look.shade_layout = 1 if self.shade_layout else 0
        look.shade_fill = settings.shade_fill
        self.look = look
        self.opacity = settings.opacity_per_density
        if self.shade_layout:
            direction = np.asarray(toward_light_world(view.camera, settings.light_dir), dtype=np.float64)
            self.toward_light = direction / np.linalg.norm(direction)
            self.light = np.zeros(cells, dtype=dtype)
            self.gradient = np.zeros((1, 1, 1, 3), dtype=dtype)
        else:
            self.radius = math.ceil(3.0 * settings.normal_blur_cells) if settings.normal_blur_cells > 0 else 0
            self.weights = gaussian_weights(settings.normal_blur_cells, self.radius)
            if self.p.name == "f32":
                self.weights = self.weights.astype(np.float32)
            self.blurred = np.zeros(cells, dtype=dtype)
            self.scratch = np.zeros(cells, dtype=dtype)
            self.gradient = np.zeros((*cells, 3), dtype=dtype)
            self.light = np.zeros((1, 1, 1), dtype=dtype)
        self.image = np.zeros((view.height_px, view.width_px, 5), dtype=dtype)

    def prepare(self, smoke: np.ndarray, cell_m: float) -> None:
        if self.shade_layout:
            self.p.fn("light_volume")(_shape(smoke), _ptr(smoke), _d3(self.toward_light), ctypes.c_double(cell_m),
                                      ctypes.c_double(self.opacity), _ptr(self.light))
        else:
            self.p.fn("normal_field")(_shape(smoke), _ptr(smoke), _ptr(self.blurred), _ptr(self.scratch),
                                      _ptr(self.gradient), _ptr(self.weights), self.radius)

    def march(self, smoke, temperature, info: OInfo, view: OView, image: np.ndarray) -> None:
        self.p.fn("raymarch")(ctypes.byref(info), _ptr(smoke), _ptr(temperature), _ptr(self.gradient),
                              _shape(self.gradient), _ptr(self.light), _shape(self.light), ctypes.byref(view),
                              ctypes.byref(self.look), _ptr(image), image.shape[0], image.shape[1])

    def render_fields(self, smoke, temperature, info: OInfo) -> np.ndarray:
        self.prepare(smoke, info.cell_m)
        self.march(smoke, temperature, info, self.view_params, self.image)
        return self.image.copy()

    def render(self, grid: Grid) -> np.ndarray:
        return self.render_fields(grid.smoke.data, grid.temperature.data, grid.info)
