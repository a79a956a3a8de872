"""Benchmark: the plain FP32 fluid step at 256 x 384 x 256 cells (seeded smoothed velocities, a masked smoke
sphere, temperature 1 + 0.8 smoke; the smoke-puff step with 4 multigrid V-cycles of 2+2 sweeps, buoyancy, drag,
vorticity confinement and a sphere emitter; dt = 1/96 s). The operator-level case at 128 x 192 x 128 is a
variant.

One step = one substep of the whole grid (Stepper.step -> plume_step, about 70 kernels, no host sync).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--cells NX,NY,NZ]

Multi-GPU: one process per GPU (torchrun); a single grid does not shard, so every rank steps its own
replica (weak scaling, no collective on the data path); rank 0 prints one JSON line with the max time over
ranks. `--impl reference` times the CPU restatement of the reference (the oracle, C++ with OpenMP on all host
cores) on the same workload; the reference itself is Python driving NVIDIA Warp, which is not installed here.
"""

import argparse
import datetime
import json
import math
import os
import shutil
import signal
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "Mcell-substeps/s"
# Algorithmic bytes per cell-substep of each phase (FP32, compulsory traffic, intermediates not counted):
# forces R s,T + R/W u,v,w = 32 (emission writes only the emitter's cells); velocity MacCormack R/W u,v,w = 24;
# divergence R u,v,w + W div = 16; multigrid 74 per top cell per V-cycle; gradient R q + R/W u,v,w = 28;
# scalar MacCormack + budget + dissipation R u,v,w,s,T + W s,T, then R/W s,T = 44.
PHASE_BYTES = {"forces": 32.0, "velocity advection": 24.0, "divergence": 16.0, "pressure solve": None,
               "gradient": 28.0, "scalar advection": 44.0}
MG_BYTES_PER_CYCLE = 74.0
# DRAM bytes (read + write) per top-level cell per V-cycle that ncu counted for the pressure-solve kernels of
# the 128x192x128 step (965.7 MB per substep at 4 cycles, every level in the natural layout); the solve's
# traffic scales with the level cells.
MG_TRAFFIC_PER_CYCLE = 965.7e6 / (128 * 192 * 128) / 4
# A top level in colour-split storage (levels of at least plume_split_min_cells cells), per top-level cell,
# from one ncu capture of each kernel at 256x384x256 (dram__bytes_read.sum + dram__bytes_write.sum): a colour
# pass 175.9 MB, the residual and restriction 219.3 MB, the prolongation 158.1 MB per V-cycle (8 passes per
# cycle at 2 + 2 sweeps); the three layout conversions 461.5 MB per solve. The levels below it are a natural
# hierarchy of one eighth the cells.
SPLIT_PASS_TRAFFIC = 175.9e6 / (256 * 384 * 256)
SPLIT_CYCLE_TRAFFIC = (219.3e6 + 158.1e6) / (256 * 384 * 256)
SPLIT_SOLVE_TRAFFIC = 461.5e6 / (256 * 384 * 256)


def solve_traffic(ncells: int, cycles: int, sweeps: int) -> float:
    """DRAM bytes of one multigrid solve per substep, from the measured per-cell figures above."""
    from plume_b200 import _native as N

    if ncells >= N.lib().plume_split_min_cells():
        top = cycles * (4 * sweeps * SPLIT_PASS_TRAFFIC + SPLIT_CYCLE_TRAFFIC) + SPLIT_SOLVE_TRAFFIC
        return ncells * (top + cycles * MG_TRAFFIC_PER_CYCLE / 8)
    return MG_TRAFFIC_PER_CYCLE * cycles * ncells


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=96)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--cells", default="256,384,256")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-variants", action="store_true", help="skip the mixed-storage and batched measurements")
    return ap.parse_args()


def peaks() -> tuple[float, str]:
    path = REPO / "MEASURED_PEAKS.json"
    if path.exists():
        return float(json.loads(path.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock and throttle samples for one GPU while the timed region runs.

    Each row carries nvidia-smi's own timestamp, and only the rows stamped between `mark_start()` and the exit
    of the `with` block count. nvidia-smi runs line-buffered (stdbuf) into a pipe that a thread reads, and it
    is stopped with SIGINT so that it flushes its last rows. With no row inside the region the summary says
    "unsampled" instead of reporting a clock taken outside it."""

    QUERY = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, uuid: str | None, command: list[str] | None = None, period_ms: int = 20):
        self.uuid = uuid
        self.command = command
        self.period_ms = period_ms
        self.proc = None
        self.thread = None
        self.rows: list[list[str]] = []
        self.lock = threading.Lock()
        self.start_s = self.end_s = None

    def _cmd(self) -> list[str]:
        if self.command is not None:
            return list(self.command)
        cmd = ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-lms", str(self.period_ms)]
        if self.uuid:
            cmd += ["-i", self.uuid]
        return (["stdbuf", "-oL"] if shutil.which("stdbuf") else []) + cmd

    def _read(self):
        for line in self.proc.stdout:
            cols = [c.strip() for c in line.split(",")]
            if len(cols) >= 10:
                with self.lock:
                    self.rows.append(cols)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(self._cmd(), stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True,
                                         bufsize=1)
        except OSError:
            self.proc = None
        if self.proc is not None:
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            deadline = time.perf_counter() + 3.0  # nvidia-smi takes a moment to start: wait for its first row
            while self.proc.poll() is None and time.perf_counter() < deadline:
                with self.lock:
                    if self.rows:
                        break
                time.sleep(0.01)
        self.mark_start()
        return self

    def mark_start(self):
        """The timed region starts now (wall clock, as nvidia-smi stamps its rows)."""
        self.start_s = time.time()

    def __exit__(self, *exc):
        self.end_s = time.time()
        if self.proc is not None:
            time.sleep(2 * self.period_ms / 1e3)  # let a row stamped inside the region reach the pipe
            try:
                self.proc.send_signal(signal.SIGINT)
                self.proc.wait(timeout=3)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.proc.wait()
            if self.thread is not None:
                self.thread.join(timeout=3)

    @staticmethod
    def _stamp(text: str) -> float | None:
        for fmt in ("%Y/%m/%d %H:%M:%S.%f", "%Y/%m/%d %H:%M:%S"):
            try:
                return datetime.datetime.strptime(text, fmt).timestamp()
            except ValueError:
                continue
        return None

    def summary(self) -> dict:
        with self.lock:
            rows = list(self.rows)
        inside = []
        for r in rows:
            t = self._stamp(r[0])
            if t is not None and self.start_s is not None and self.end_s is not None and \
                    self.start_s <= t <= self.end_s:
                inside.append(r)
        if not inside:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0,
                    "rows_outside_region": len(rows)}
        sm = [float(r[2]) for r in inside if r[2].replace(".", "").isdigit()]
        max_sm = [float(r[3]) for r in inside if r[3].replace(".", "").isdigit()]
        reasons = sorted({name for r in inside for name, flag in zip(self.REASONS, r[6:10]) if flag.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(max_sm) if max_sm else None,
                "reasons": reasons, "samples": len(inside), "rows_outside_region": len(rows) - len(inside)}


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def seeded_state(cells, ambient_k):
    from plume_b200.workloads import operator_fields

    return operator_fields(cells, 20261203, ambient_k)


def cpu_baseline(recipe, derived, fields, budget_s: float = 20.0) -> dict:
    """The oracle (C++ restatement of the reference, OpenMP on all host cores) on a bounded sample of the same
    workload: whole-grid substeps from the same seeded state, as many as fit in about `budget_s` seconds."""
    from oracle import oracle as O

    threads = O.set_threads(os.cpu_count() or 1)
    d = recipe.domain
    grid = O.make_grid(derived, d.cell_m, d.faces, d.ambient_k)
    for name, values in fields.items():
        getattr(grid, name).data[...] = values
    stepper = O.Stepper(grid, recipe)
    stepper.step(0.0, derived.dt_s)  # warm-up
    steps, start = 0, time.perf_counter()
    while True:
        stepper.step((steps + 1) * derived.dt_s, derived.dt_s)
        steps += 1
        elapsed = time.perf_counter() - start
        if elapsed > budget_s or steps >= 8:
            break
    cells = math.prod(derived.cells)
    return {"value": cells * steps / elapsed / 1e6, "unit": METRIC, "cores": threads, "kind": "port",
            "sample": f"{steps} whole-grid substeps of the {'x'.join(map(str, derived.cells))} plain step after 1 "
                      f"warm-up, oracle C++ FP32 with OpenMP on {threads} threads ({elapsed:.1f} s)"}


def batched_variant(device: str, count: int = 64, frames: int = 48) -> dict:
    """The batched uneven recipes (BASELINE C4): `count` instances from the sweep front-end, grids drawn among
    48^3, 64x96x64, 96x144x96 and 160x240x160, 48 frames with CFL-limited substeps. Three arms on the same
    instances: plain FP32 one instance after another, FP32 batched (all instances at once on their own
    streams) and BF16 batched. Each arm is built, run once (allocations, pressure-solve graph captures), reset
    and run again; the second run is timed with CUDA events. Each instance's last frame is rendered after the
    timed run: thickness differences of the BF16 arm from the FP32 arm (largest pixel difference, and the
    relative difference of the frame's total thickness), and whether the FP32 arms agree byte for byte."""
    import torch

    from plume_b200.recipe.derived import derive
    from plume_b200.render.camera import sheet_domain_view
    from plume_b200.render.frame_renderer import FrameRenderer
    from plume_b200.sim.batch import Batch
    from plume_b200.workloads import batched_recipes

    recipes = batched_recipes(count=count, frames=frames)
    arms = (("one_at_a_time_f32", torch.float32, True), ("batched_f32", torch.float32, False),
            ("batched_bf16", torch.bfloat16, False))
    out, last = {"instances": count, "frames": frames, "unit": METRIC}, {}
    for name, storage, sequential in arms:
        batch = Batch(recipes, device, storage=storage)
        batch.run(sequential=sequential)
        batch.reset()
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        wall = time.perf_counter()
        logs = batch.run(sequential=sequential)
        end.record()
        torch.cuda.synchronize()
        wall = time.perf_counter() - wall
        ms = start.elapsed_time(end)
        work = sum(math.prod(derive(r).cells) * log.total_steps for r, log in zip(recipes, logs))
        out[name] = {"value": work / (ms / 1e3) / 1e6, "device_ms": ms, "host_wall_s": wall,
                     "cell_substeps": work, "substeps": sum(log.total_steps for log in logs)}
        frames_out = []
        for recipe, grid in zip(recipes, batch.grids):
            derived = derive(recipe)
            view = sheet_domain_view(recipe, derived)
            renderer = FrameRenderer(view, recipe.render, derived.cells, recipe.output.channels, device)
            frames_out.append(renderer.render(grid)[..., 1].astype(np.float64))
        last[name] = frames_out
        del batch
        torch.cuda.empty_cache()
    base = out["one_at_a_time_f32"]["value"]
    out["ratio_bf16_batched_to_f32_one_at_a_time"] = out["batched_bf16"]["value"] / base
    out["ratio_f32_batched_to_f32_one_at_a_time"] = out["batched_f32"]["value"] / base
    out["f32_arms_identical"] = all(np.array_equal(a, b) for a, b in zip(last["one_at_a_time_f32"], last["batched_f32"]))
    pixel = [float(np.abs(a - b).max()) for a, b in zip(last["batched_bf16"], last["batched_f32"])]
    total = [abs(float(a.sum()) - float(b.sum())) / max(float(b.sum()), 1e-30)
             for a, b in zip(last["batched_bf16"], last["batched_f32"])]
    out["bf16_vs_f32_last_frame"] = {"max_pixel_thickness": max(pixel), "max_relative_total_thickness": max(total)}
    out["value"] = out["batched_bf16"]["value"]
    return out


def adjoint_variant(device: str) -> dict:
    """The differentiable step (BASELINE C3): 96 x 144 x 96 cells, 64 substeps (32 frames of 2), a 16^3 source
    field centred on cell (48, 8, 48), buoyancy 1.0, drag 0.2 and vorticity confinement 0.3, a checkpoint every 8
    substeps. FlowFit's gradient with respect to the source field, heat_buoyancy, drag_per_s and the confinement
    strength (the velocity path included) against the forward substep it differentiates: the forward is timed as plume_step substeps
    (the production step) and as FlowFit's taped forward; the adjoint is the backward pass (recomputing each
    segment, then every substep's adjoint). CUDA events around device-synchronised runs."""
    import torch

    from plume_b200.adjoint import FlowFit
    from plume_b200.recipe.derived import derive
    from plume_b200.sim.grid import make_grid
    from plume_b200.sim.stepper import Stepper
    from plume_b200.workloads import plain_step_recipe

    recipe = plain_step_recipe((96, 144, 96), cycles=4, frames=32, substeps=2)
    derived = derive(recipe)
    substeps = 64
    fit = FlowFit(recipe, (16, 16, 16), (40, 0, 40), substeps, device, checkpoint_every=8)
    source = torch.from_numpy(np.random.default_rng(3).uniform(0.0, 1.0, (16, 16, 16)).astype(np.float32)).to(device)
    target = torch.zeros((fit.view.height_px, fit.view.width_px), dtype=torch.float32, device=device)
    fit.loss_and_grad(source, target)  # warm-up: graph captures, allocations
    taped_ms = device_ms(lambda: fit.forward(source))
    total_ms = device_ms(lambda: fit.loss_and_grad(source, target))
    d = recipe.domain
    grid = make_grid(derived, d.cell_m, d.faces, d.ambient_k, device)
    stepper = Stepper(grid, recipe)
    stepper.step(0.0, derived.dt_s)
    step_ms = device_ms(lambda: [stepper.step(n * derived.dt_s, derived.dt_s) for n in range(substeps)])
    adjoint_ms = total_ms - taped_ms
    _, _, scalars, _ = fit.loss_and_grad(source, target)
    return {"cells": [96, 144, 96], "substeps": substeps, "checkpoint_every": 8,
            "parameters": ["source field 16^3", "heat_buoyancy", "drag_per_s", "vorticity_confinement"],
            "forward_step_ms_per_substep": step_ms / substeps,
            "forward_taped_ms_per_substep": taped_ms / substeps,
            "adjoint_ms_per_substep": adjoint_ms / substeps,
            "adjoint_over_forward": adjoint_ms / step_ms,
            "adjoint_over_taped_forward": adjoint_ms / taped_ms,
            "scalar_gradients": scalars}


def square_view(view, pixels: int):
    """The domain view re-sampled to pixels x pixels, the whole domain inside (the larger side fits)."""
    import dataclasses

    extent = max(view.width_px, view.height_px) * view.pixel_m
    return dataclasses.replace(view, pixel_m=extent / pixels, width_px=pixels, height_px=pixels)


def device_ms(fn) -> float:
    """Device time of fn() on the current stream (CUDA events, synchronised)."""
    import torch

    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record()
    fn()
    end.record()
    torch.cuda.synchronize()
    return start.elapsed_time(end)


def operators_variant(device: str) -> dict:
    """The operator-level case's single calls on its seeded fields: MacCormack advection of the five fields
    (dt = 1/96 s), buoyancy + vorticity confinement, a projection of the resulting divergence solved to
    relative residual 1e-6 by defect correction, and a 256 x 256 orthographic march (light volume + march);
    device milliseconds of each, the projection's corrections and residual ratios."""
    import torch

    from plume_b200.recipe.derived import derive
    from plume_b200.workloads import plain_step_recipe

    from plume_b200.render.camera import sheet_domain_view
    from plume_b200.render.frame_renderer import FrameRenderer
    from plume_b200.sim.advect import advect_maccormack
    from plume_b200.sim.forces import apply_buoyancy
    from plume_b200.sim.grid import make_grid
    from plume_b200.sim.multigrid import Multigrid
    from plume_b200.sim.pressure import project_refined
    from plume_b200.sim.vorticity import VorticityConfinement

    recipe = plain_step_recipe((128, 192, 128), cycles=4)
    derived = derive(recipe)
    d, f = recipe.domain, recipe.forces
    fields = seeded_state(derived.cells, d.ambient_k)
    grid = make_grid(derived, d.cell_m, d.faces, d.ambient_k, device)
    for name, values in fields.items():
        getattr(grid, name).data.copy_(torch.from_numpy(values))
    dt = derived.dt_s
    velocity = tuple(field.data for field in grid.velocity_fields())

    def advect():
        for name in ("u", "v", "w", "smoke", "temperature"):
            advect_maccormack(getattr(grid, name), velocity, grid, dt)

    confinement = VorticityConfinement(grid)

    def forces():
        apply_buoyancy(grid, f.gravity_mps2, f.heat_buoyancy, f.smoke_weight, d.ambient_k, dt)
        confinement.apply(grid, f.vorticity_confinement, dt)

    advect()  # warm-up (allocations)
    forces()
    advect_ms, forces_ms = device_ms(advect), device_ms(forces)
    multigrid = Multigrid(grid, recipe.solver.multigrid_cycles, recipe.solver.multigrid_sweeps)
    grid.pressure.zero_()
    torch.cuda.synchronize()
    start = time.perf_counter()
    refinement = project_refined(grid, multigrid, rel_tol=1e-6)
    torch.cuda.synchronize()
    project_ms = (time.perf_counter() - start) * 1e3
    view = square_view(sheet_domain_view(recipe, derived), 256)
    renderer = FrameRenderer(view, recipe.render, derived.cells, recipe.output.channels, device)
    renderer.render(grid)
    render_ms = device_ms(lambda: (renderer.prepare(grid.smoke.data, grid.info.cell_m),
                                   renderer.march(grid.smoke.data, grid.temperature.data, grid.info,
                                                  renderer.view_params, renderer.image)))
    return {"cells": list(derived.cells), "advect_five_fields_ms": advect_ms, "buoyancy_confinement_ms": forces_ms,
            "projection": {"rel_tol": 1e-6, "corrections": refinement.corrections, "ratio": refinement.ratio,
                           "ratios": list(refinement.ratios), "ms_with_host_syncs": project_ms},
            "march_256x256_ms": render_ms}


def mixed_variant(device: str, fields=None, steps: int = 8, frames: int = 2, pixels: int = 256) -> dict:
    """The large mixed-precision case (BASELINE C5) at 256 x 384 x 256 (dx = 1/128 m, emitter radius 24 cells):
    the seeded state stepped with velocity, smoke and temperature stored as FP32, BF16 and FP16 (FP32
    arithmetic), each timed over `steps` substeps (CUDA events), then restarted and run `frames` frames of 4
    substeps, each frame rendered (pixels x pixels, the normal-map layout: thickness and heat depend on smoke
    and temperature only). The same frames from an FP64 run of the plain method (the oracle in double, on the
    host cores) are the reference: per frame, the largest pixel difference of thickness and of heat (relative
    to the frame's largest heat), and the relative difference of the frame's total thickness. Also the
    projection refined to a relative residual of 1e-7 (FP32 multigrid with defect correction, FP64 norms and
    coarsest level) and a 512 x 512 march of the FP32 state."""
    import dataclasses

    import torch

    from oracle import oracle as O
    from plume_b200.recipe.derived import derive
    from plume_b200.render.camera import sheet_domain_view
    from plume_b200.render.frame_renderer import FrameRenderer
    from plume_b200.sim.grid import make_grid
    from plume_b200.sim.multigrid import Multigrid
    from plume_b200.sim.pressure import compute_divergence
    from plume_b200.sim.stepper import Stepper
    from plume_b200.workloads import plain_step_recipe

    cells = (256, 384, 256)
    recipe = plain_step_recipe(cells)
    derived = derive(recipe)
    d = recipe.domain
    if fields is None or tuple(fields["smoke"].shape) != cells:
        fields = seeded_state(cells, d.ambient_k)
    normal_layout = "heat,thickness,normal_x,normal_y"
    view = square_view(sheet_domain_view(recipe, derived), pixels)
    dt = derived.dt_s
    out = {"cells": list(cells), "frames": frames, "substeps_per_frame": 4, "frame_pixels": pixels}

    threads = O.set_threads(os.cpu_count() or 1)
    start = time.perf_counter()
    reference = O.make_grid(derived, d.cell_m, d.faces, d.ambient_k, "f64")
    for name, values in fields.items():
        getattr(reference, name).data[...] = values
    stepper64 = O.Stepper(reference, recipe)
    renderer64 = O.FrameRenderer(view, recipe.render, derived.cells, normal_layout, "f64")
    frames64 = []
    for frame in range(frames):
        for n in range(4):
            stepper64.step((4 * frame + n) * dt, dt)
        frames64.append(renderer64.render(reference).astype(np.float64))
    out["fp64_reference"] = {"kind": "oracle in double", "threads": threads, "seconds": time.perf_counter() - start}
    del reference, stepper64, renderer64

    for label, storage in (("f32", torch.float32), ("bf16", torch.bfloat16), ("f16", torch.float16)):
        grid = make_grid(derived, d.cell_m, d.faces, d.ambient_k, device, storage=storage)
        for name, values in fields.items():
            getattr(grid, name).data.copy_(torch.from_numpy(values))
        stepper = Stepper(grid, recipe)
        for n in range(3):  # warm-up: the solve's graph capture, allocations
            stepper.step(n * dt, dt)
        ms = device_ms(lambda: [stepper.step((3 + n) * dt, dt) for n in range(steps)])
        entry = {"value": math.prod(cells) * steps / (ms / 1e3) / 1e6, "unit": METRIC, "steps": steps}
        for name, values in fields.items():  # the frames restart from the seeded state
            getattr(grid, name).data.copy_(torch.from_numpy(values))
        grid.pressure.zero_()
        stepper = Stepper(grid, recipe)
        renderer = FrameRenderer(view, recipe.render, derived.cells, normal_layout, device)
        thickness_px, heat_px, total = [], [], []
        for frame in range(frames):
            for n in range(4):
                stepper.step((4 * frame + n) * dt, dt)
            image = renderer.render(grid).astype(np.float64)
            want = frames64[frame]
            heat_scale = max(float(np.abs(want[..., 0]).max()), 1e-30)
            thickness_px.append(float(np.abs(image[..., 1] - want[..., 1]).max()))
            heat_px.append(float(np.abs(image[..., 0] - want[..., 0]).max()) / heat_scale)
            total.append(abs(float(image[..., 1].sum()) - float(want[..., 1].sum())) / float(want[..., 1].sum()))
        entry.update({"thickness_max_pixel_vs_fp64": thickness_px, "heat_max_pixel_vs_fp64": heat_px,
                      "total_thickness_relative_vs_fp64": total})
        out[label] = entry
        if label == "f32":
            multigrid = Multigrid(grid, recipe.solver.multigrid_cycles, recipe.solver.multigrid_sweeps)
            compute_divergence(grid)
            grid.pressure.zero_()
            torch.cuda.synchronize()
            start = time.perf_counter()
            refinement = multigrid.refine(grid, rel_tol=1e-7)
            torch.cuda.synchronize()
            out["projection"] = {"rel_tol": 1e-7, "corrections": refinement.corrections, "ratio": refinement.ratio,
                                 "float_ratio": refinement.float_ratio,
                                 "ms_with_host_syncs": (time.perf_counter() - start) * 1e3}
            march = FrameRenderer(square_view(sheet_domain_view(recipe, derived), 512), recipe.render, derived.cells,
                                  recipe.output.channels, device)
            march.render(grid)
            out["march_512x512_ms"] = device_ms(lambda: (
                march.prepare(grid.smoke.data, grid.info.cell_m),
                march.march(grid.smoke.data, grid.temperature.data, grid.info, march.view_params, march.image)))
        del grid, stepper, renderer
        torch.cuda.empty_cache()
    for label in ("bf16", "f16"):
        out[label]["ratio_to_f32"] = out[label]["value"] / out["f32"]["value"]
    return out


def preview_run_variant(device: str) -> dict:
    """The smoke-puff preview (38 x 48 x 38 cells, 16 frames, 192 substeps) end to end on the device through
    plume_b200.run.run_recipe: simulate, render every frame, assemble the sheet, measure the numbers; wall
    seconds of a second run (the first warms the graphs and allocations), and frames per second."""
    import torch

    from plume_b200.recipe.load import load_recipe
    from plume_b200.run import run_recipe

    recipe = load_recipe(REPO / "tests" / "golden" / "smoke_puff.toml", preview=True)
    run_recipe(recipe, "recipes/smoke_puff.toml", device)
    torch.cuda.synchronize()
    start = time.perf_counter()
    run = run_recipe(recipe, "recipes/smoke_puff.toml", device)
    torch.cuda.synchronize()
    seconds = time.perf_counter() - start
    return {"cells": list(run.derived.cells), "frames": recipe.time.frames, "substeps": run.steps.total_steps,
            "seconds": seconds, "frames_per_s": recipe.time.frames / seconds,
            "mcell_substeps_per_s": math.prod(run.derived.cells) * run.steps.total_steps / seconds / 1e6}


def workload_name(derived, cycles: int) -> str:
    """The workload both arms time, by what it is and its sizes; what tells workloads apart comes first."""
    return (f"{'x'.join(map(str, derived.cells))} plain FP32 fluid step, {cycles} MG V-cycles 2+2, "
            f"confinement+drag+emitter, dt 1/96 s, seeded smoothed velocity, smoke ball")


def bench_config(derived, cycles: int, world: int) -> dict:
    """The `config` both arms print, identical for the same workload."""
    return {"workload": workload_name(derived, cycles), "cells": list(derived.cells),
            "parallelism": f"replicas x{world}",
            "l2": "no flush: every substep reads and writes the whole state, larger than the 126 MB L2"}


def run_reference(args, cells):
    """--impl reference: the oracle port of the reference's CPU path on the host cores."""
    world, rank, _ = dist_env()
    if rank != 0:
        return
    from oracle import oracle as O
    from plume_b200.recipe.derived import derive
    from plume_b200.workloads import plain_step_recipe

    recipe = plain_step_recipe(cells, cycles=4)
    derived = derive(recipe)
    threads = O.set_threads(os.cpu_count() or 1)
    d = recipe.domain
    grid = O.make_grid(derived, d.cell_m, d.faces, d.ambient_k)
    for name, values in seeded_state(derived.cells, d.ambient_k).items():
        getattr(grid, name).data[...] = values
    stepper = O.Stepper(grid, recipe)
    for n in range(args.warmup):
        stepper.step(n * derived.dt_s, derived.dt_s)
    budget_s, timed, start = 150.0, 0, time.perf_counter()
    for n in range(args.steps):
        stepper.step((args.warmup + n) * derived.dt_s, derived.dt_s)
        timed += 1
        if time.perf_counter() - start > budget_s:
            break
    elapsed = time.perf_counter() - start
    value = math.prod(derived.cells) * timed / elapsed / 1e6
    sample = (f"{timed} of {args.steps} whole-grid substeps (stopped at the {budget_s:.0f} s budget)" if timed < args.steps
              else f"{timed} whole-grid substeps") + f" after {args.warmup} warm-up, {threads} threads"
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": timed,
            "warmup": args.warmup, "ms_per_step": elapsed * 1e3 / timed, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "reference",
            "config": bench_config(derived, recipe.solver.multigrid_cycles, world),
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    cells = tuple(int(x) for x in args.cells.split(","))
    if args.impl == "reference":
        run_reference(args, cells)
        return
    import torch
    import torch.distributed as dist

    from plume_b200 import _native as N
    from plume_b200.recipe.derived import derive
    from plume_b200.render.camera import sheet_domain_view
    from plume_b200.render.frame_renderer import FrameRenderer
    from plume_b200.sim.grid import make_grid
    from plume_b200.sim.step_cap import StepCap
    from plume_b200.sim.stepper import Stepper
    from plume_b200.workloads import plain_step_recipe

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    device = f"cuda:{local}"
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device(device))
    recipe = plain_step_recipe(cells, cycles=4)
    derived = derive(recipe)
    d = recipe.domain
    fields = seeded_state(derived.cells, d.ambient_k)
    grid = make_grid(derived, d.cell_m, d.faces, d.ambient_k, device)
    for name, values in fields.items():
        getattr(grid, name).data.copy_(torch.from_numpy(values))
    stepper = Stepper(grid, recipe)
    dt = derived.dt_s
    stream = torch.cuda.current_stream()
    for n in range(args.warmup):
        stepper.step(n * dt, dt)
    torch.cuda.synchronize()
    resident_gb = torch.cuda.memory_allocated(local) / 1e9  # the grid and every scratch array of the step

    # timed region: K substeps, phase events recorded inside plume_step on the same stream
    phases = N.STEP_PHASES
    events = [[torch.cuda.Event(enable_timing=True) for _ in range(len(phases) + 1)] for _ in range(args.steps)]
    for row in events:  # torch creates an event on its first record; make every handle valid first
        for e in row:
            e.record(stream)
    torch.cuda.synchronize()
    handles = [(N.ctypes.c_void_p * (len(phases) + 1))(*[e.cuda_event for e in row]) for row in events]
    base_params = stepper._params
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        uuid = None
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches_before = N.launch_count()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(uuid) as clocks:
        start.record(stream)
        for n in range(args.steps):
            step = args.warmup + n
            params = base_params(step * dt, dt)
            params.phase_events = N.ctypes.cast(handles[n], N.ctypes.POINTER(N.ctypes.c_void_p))
            N.call("plume_step", stepper._state(), params, N.stream())
            for field in (*grid.velocity_fields(), grid.smoke, grid.temperature):
                field.swap()
        end.record(stream)
        torch.cuda.synchronize()
    launches = N.launch_count() - launches_before
    elapsed_ms = start.elapsed_time(end)
    timing = torch.tensor([elapsed_ms], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(timing, op=dist.ReduceOp.MAX)
    max_ms = float(timing.item())
    phase_ms = {name: sum(row[i].elapsed_time(row[i + 1]) for row in events) / args.steps
                for i, name in enumerate(phases)}

    # e2e: the public API frame loop (StepCap.plan readback, Stepper.step x substeps, FrameRenderer.render
    # copying the raw frame to the host) from a state uploaded from pinned host memory inside the timed region.
    # The synchronous render measured steadier and faster than FrameRenderer.render_async here (1426-1430 vs
    # 1205-1499 Mcell-substeps/s over three runs each): the overlapped frame competes with the substeps for SMs.
    pinned = {name: torch.from_numpy(values).pin_memory() for name, values in fields.items()}
    view = sheet_domain_view(recipe, derived)
    renderer = FrameRenderer(view, recipe.render, derived.cells, recipe.output.channels, device)
    cap = StepCap(recipe)
    substeps = derived.steps_per_frame
    frames = max(1, args.steps // substeps)
    grid2 = make_grid(derived, d.cell_m, d.faces, d.ambient_k, device)
    stepper2 = Stepper(grid2, recipe)
    renderer.render(grid2)  # warm the renderer
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e2e_start, e2e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_start.record(stream)
    for name, tensor in pinned.items():
        getattr(grid2, name).data.copy_(tensor, non_blocking=True)
    steps_run = 0
    for frame in range(frames):  # run_block of plume_b200.sim.run, one frame per block
        start_s, length_s = frame * substeps * dt, substeps * dt
        steps = cap.plan(grid2, start_s, length_s, substeps, f"frame {frame}").steps
        for index in range(steps):
            if steps == substeps:
                stepper2.step((frame * substeps + index) * dt, dt)
            else:
                stepper2.step(start_s + index * length_s / steps, length_s / steps)
        steps_run += steps
        renderer.render(grid2)
    e2e_end.record(stream)
    torch.cuda.synchronize()
    e2e_ms = torch.tensor([e2e_start.elapsed_time(e2e_end)], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(e2e_ms, op=dist.ReduceOp.MAX)
    e2e_ms = float(e2e_ms.item())

    ncells = math.prod(derived.cells)
    value = world * ncells * args.steps / (max_ms / 1e3) / 1e6
    e2e_value = world * ncells * steps_run / (e2e_ms / 1e3) / 1e6
    h2d = sum(t.numel() * 4 for t in pinned.values()) / steps_run
    d2h = (renderer.image.numel() * 4 + 4) * frames / steps_run

    peak, peak_kind = peaks()
    cycles = recipe.solver.multigrid_cycles
    phase_bytes = dict(PHASE_BYTES)
    phase_bytes["pressure solve"] = MG_BYTES_PER_CYCLE * cycles
    phase_gbs = {name: (phase_bytes[name] * ncells / (ms / 1e3) / 1e9 if ms > 0 else None)
                 for name, ms in phase_ms.items()}
    dominant = max(phase_ms, key=phase_ms.get)
    achieved = phase_gbs[dominant]
    step_bytes = sum(phase_bytes.values())
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": bench_config(derived, cycles, world),
        "resident_gb_per_grid": resident_gb,
        "roofline": {"bound": "hbm", "kernel": f"{dominant} phase of plume_step", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak if achieved else None,
                     "traffic": (solve_traffic(ncells, cycles, recipe.solver.multigrid_sweeps)
                                 if dominant == "pressure solve" else None),
                     "peak_kind": peak_kind},
        "step_roofline": {"bytes_per_cell_substep": step_bytes,
                          "achieved": step_bytes * ncells * args.steps / (max_ms / 1e3) / 1e9,
                          "frac": step_bytes * ncells * args.steps / (max_ms / 1e3) / 1e9 / peak},
        "phases_ms": phase_ms, "phases_gbs": phase_gbs,
        "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": steps_run, "frames": frames},
        "gpu_launches": launches,
        "clocks": clocks.summary(),
    }
    if not args.no_variants:
        line["variants"] = {"mixed": mixed_variant(device, fields), "batched": batched_variant(device),
                            "adjoint": adjoint_variant(device), "operators": operators_variant(device),
                            "preview_run": preview_run_variant(device)}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(recipe, derived, fields)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
