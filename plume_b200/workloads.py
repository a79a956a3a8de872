"""Synthetic workloads: seeded fields and recipes with the shapes and value distributions of the benchmark
configurations (no dataset is involved; everything is generated from a seed).

- `operator_fields`: the operator-level case -- u, v, w ~ U(-1, 1) m/s smoothed by three 3x3x3 box-filter
  passes with edge clamp; smoke ~ U(0, 1) masked to a sphere of radius 40/128 of the x extent at the grid
  centre; temperature = ambient + 0.8 * smoke (ambient 1).
- `plain_step_recipe`: the plain smoke-puff step at a given grid: dx = 1/64 m scaled to the grid, buoyancy
  f_y = 1.0 T - 0.05 density with ambient 1, drag 0.2/s, vorticity confinement 0.3, closed floor and open
  sides and ceiling, multigrid 4 V-cycles of 2+2 sweeps, a sphere emitter of radius 12/128 of the x extent
  near the floor holding temperature 2 and adding smoke at 1/s, dt = 1/96 s.
- `smoke_puff_recipe`: the 64 x 96 x 64 puff run (24 fps x 48 frames, CFL 1, at most 4 substeps).
"""

import numpy as np

from plume_b200.recipe.load import resolve_table

DEFAULT_SEED = 20261203


def box_filter(field: np.ndarray, passes: int = 3) -> np.ndarray:
    """`passes` 3x3x3 box-filter passes with edge clamp, in float64. Each pass runs as three 3-tap sums, one
    per axis (the 27-cell box is their product, edge replication included), then divides by 27."""
    out = field.astype(np.float64)
    for _ in range(passes):
        for axis in range(3):
            n = out.shape[axis]
            pad = [(1, 1) if a == axis else (0, 0) for a in range(3)]
            padded = np.pad(out, pad, mode="edge")

            def window(start):
                return padded[tuple(slice(start, start + n) if a == axis else slice(None) for a in range(3))]

            out = window(0) + window(1)
            out += window(2)
        out /= 27.0
    return out


def operator_fields(cells, seed: int = DEFAULT_SEED, ambient_k: float = 1.0) -> dict:
    nx, ny, nz = cells
    rng = np.random.default_rng(seed)
    fields = {
        "u": box_filter(rng.uniform(-1.0, 1.0, (nx + 1, ny, nz))).astype(np.float32),
        "v": box_filter(rng.uniform(-1.0, 1.0, (nx, ny + 1, nz))).astype(np.float32),
        "w": box_filter(rng.uniform(-1.0, 1.0, (nx, ny, nz + 1))).astype(np.float32),
    }
    smoke = rng.uniform(0.0, 1.0, cells)
    centre = [np.arange(n, dtype=np.float64) + 0.5 - n / 2.0 for n in cells]
    dist2 = centre[0][:, None, None] ** 2 + centre[1][None, :, None] ** 2 + centre[2][None, None, :] ** 2
    radius = 40.0 * nx / 128.0
    fields["smoke"] = np.where(dist2 <= radius * radius, smoke, 0.0).astype(np.float32)
    del smoke, dist2
    fields["temperature"] = (ambient_k + 0.8 * fields["smoke"].astype(np.float64)).astype(np.float32)
    return fields


def device_operator_fields(cells, seed: int = DEFAULT_SEED, ambient_k: float = 1.0, device: str = "cuda:0") -> dict:
    """operator_fields' distributions generated on the device (torch's generator, float32 box filters): for
    grids too large to fill quickly on the host. The values differ from operator_fields'."""
    import torch
    import torch.nn.functional as F

    generator = torch.Generator(device=device).manual_seed(seed)
    nx, ny, nz = cells

    def smoothed(shape):
        x = torch.rand(shape, generator=generator, device=device) * 2.0 - 1.0
        for _ in range(3):
            x = F.avg_pool3d(F.pad(x[None, None], (1, 1, 1, 1, 1, 1), mode="replicate"), 3, stride=1)[0, 0]
        return x.contiguous()

    fields = {"u": smoothed((nx + 1, ny, nz)), "v": smoothed((nx, ny + 1, nz)), "w": smoothed((nx, ny, nz + 1))}
    idx = [torch.arange(n, device=device, dtype=torch.float32) + 0.5 - n / 2.0 for n in cells]
    dist2 = idx[0][:, None, None] ** 2 + idx[1][None, :, None] ** 2 + idx[2][None, None, :] ** 2
    radius = 40.0 * nx / 128.0
    smoke = torch.rand(cells, generator=generator, device=device)
    fields["smoke"] = torch.where(dist2 <= radius * radius, smoke, torch.zeros_like(smoke))
    fields["temperature"] = ambient_k + 0.8 * fields["smoke"]
    return fields


def plain_step_recipe(cells=(128, 192, 128), cycles: int = 4, frames: int = 24, substeps: int = 4):
    nx, ny, nz = cells
    cell_m = (128.0 / nx) / 64.0
    table = {
        "seed": 7,
        "domain": {"size_m": [nx * cell_m, ny * cell_m, nz * cell_m], "cell_m": cell_m, "ambient_k": 1.0},
        "time": {"duration_s": frames / 24.0, "frames": frames, "substeps": substeps},
        "emitter": [{"name": "source", "center_m": [0.0, 16.0 * (nx / 128.0) * cell_m, 0.0],
                     "radius_m": 12.0 * (nx / 128.0) * cell_m, "edge_softness": 0.0, "end_s": 1.0e6,
                     "smoke_per_s": 1.0, "temperature_k": 2.0}],
        "forces": {"gravity_mps2": 1.0, "heat_buoyancy": 1.0, "smoke_weight": 0.05, "drag_per_s": 0.2,
                   "vorticity_confinement": 0.3},
        "solver": {"multigrid_cycles": cycles, "multigrid_sweeps": 2, "max_cells_per_step": 1.0,
                   "max_substeps": 32},
        "render": {"glow_start_k": 1.0, "light_dir": [0.5, 0.8, 0.3]},
        "output": {"frame_px": 128},
    }
    return resolve_table(table, "plain_step")


def smoke_puff_recipe(cells=(64, 96, 64), frames: int = 48):
    """The 64 x 96 x 64 puff: dx = 1/32 m, sphere of radius 6 cells at cell (32, 8, 32) adding density 1/s and
    holding temperature 2 (ambient 1) for the first 0.5 s, 24 fps, CFL 1 with at most 4 substeps."""
    nx, ny, nz = cells
    cell_m = 1.0 / 32.0 * (64.0 / nx)
    table = {
        "seed": 7,
        "domain": {"size_m": [nx * cell_m, ny * cell_m, nz * cell_m], "cell_m": cell_m, "ambient_k": 1.0},
        "time": {"duration_s": frames / 24.0, "frames": frames, "substeps": 1},
        "emitter": [{"name": "puff", "center_m": [0.0, 8.0 * (nx / 64.0) * cell_m, 0.0],
                     "radius_m": 6.0 * (nx / 64.0) * cell_m, "edge_softness": 0.0, "end_s": 0.5,
                     "smoke_per_s": 1.0, "temperature_k": 2.0}],
        "forces": {"gravity_mps2": 1.0, "heat_buoyancy": 1.0, "smoke_weight": 0.05, "drag_per_s": 0.2,
                   "vorticity_confinement": 0.3},
        "solver": {"multigrid_cycles": 4, "multigrid_sweeps": 2, "max_cells_per_step": 1.0, "max_substeps": 4},
        "render": {"glow_start_k": 1.0, "light_dir": [0.5, 0.8, 0.3]},
        "output": {"frame_px": 128},
    }
    return resolve_table(table, "smoke_puff_c1")


def run_plain_steps(cells=(128, 192, 128), substeps: int = 1, device: str = "cuda:0", render: bool = False,
                    storage: str = "f32"):
    """Steps the seeded operator-level state `substeps` times through Stepper.step (and renders one frame when
    `render`), for profiling single kernels on a small case; `storage` ("f32", "bf16" or "f16") is the element
    type of the stored fields."""
    import torch

    from plume_b200.recipe.derived import derive
    from plume_b200.render.camera import sheet_domain_view
    from plume_b200.render.frame_renderer import FrameRenderer
    from plume_b200.sim.grid import make_grid
    from plume_b200.sim.stepper import Stepper

    recipe = plain_step_recipe(tuple(cells))
    derived = derive(recipe)
    d = recipe.domain
    dtype = {"f32": torch.float32, "bf16": torch.bfloat16, "f16": torch.float16}[storage]
    grid = make_grid(derived, d.cell_m, d.faces, d.ambient_k, device, storage=dtype)
    for name, values in operator_fields(derived.cells, DEFAULT_SEED, d.ambient_k).items():
        getattr(grid, name).data.copy_(torch.from_numpy(values).to(dtype))
    stepper = Stepper(grid, recipe)
    for n in range(substeps):
        stepper.step(n * derived.dt_s, derived.dt_s)
    if render:
        view = sheet_domain_view(recipe, derived)
        FrameRenderer(view, recipe.render, derived.cells, recipe.output.channels, device).render(grid)
    torch.cuda.synchronize()
    return grid


if __name__ == "__main__":
    import argparse

    ap = argparse.ArgumentParser(description="run the plain step on the seeded operator-level state")
    ap.add_argument("--cells", default="128,192,128")
    ap.add_argument("--substeps", type=int, default=1)
    ap.add_argument("--render", action="store_true")
    ap.add_argument("--storage", choices=("f32", "bf16", "f16"), default="f32")
    args = ap.parse_args()
    run_plain_steps(tuple(int(x) for x in args.cells.split(",")), args.substeps, render=args.render,
                    storage=args.storage)
    print("ok")


BATCH_GRIDS = ((48, 48, 48), (64, 96, 64), (96, 144, 96), (160, 240, 160))


def batch_base_table(frames: int = 48) -> dict:
    """The batched runs' base recipe: the 64 x 96 x 64 smoke puff in a 2 m wide domain, 24 fps, CFL 1 with up to
    16 substeps per frame; every instance overrides its grid, emitter and forces."""
    cell_m = 2.0 / 64.0
    return {
        "seed": 7,
        "domain": {"size_m": [2.0, 3.0, 2.0], "cell_m": cell_m, "ambient_k": 1.0},
        "time": {"duration_s": frames / 24.0, "frames": frames, "substeps": 1},
        "emitter": [{"name": "puff", "center_m": [0.0, 0.25, 0.0], "radius_m": 6.0 * cell_m, "edge_softness": 0.0,
                     "end_s": 0.5, "smoke_per_s": 1.0, "temperature_k": 2.0}],
        "forces": {"gravity_mps2": 1.0, "heat_buoyancy": 1.0, "smoke_weight": 0.05, "drag_per_s": 0.2,
                   "vorticity_confinement": 0.3},
        "solver": {"multigrid_cycles": 4, "multigrid_sweeps": 2, "max_cells_per_step": 1.0, "max_substeps": 16},
        "render": {"glow_start_k": 1.0, "light_dir": [0.5, 0.8, 0.3]},
        "output": {"frame_px": 128},
    }


def batch_variations(count: int = 64, seed: int = DEFAULT_SEED, grids=BATCH_GRIDS) -> list:
    """The `--set` overrides of each batched instance (a parameter sweep): its grid drawn from `grids` by seed
    in the same 2 m wide domain (larger grids are finer and need more CFL substeps), emitter radius U(4, 10)
    cells, the emitter's position jittered by up to 10% of the domain, heat buoyancy U(0.5, 1.5), drag
    U(0, 0.5)/s, vorticity confinement U(0.1, 0.5)."""
    rng = np.random.default_rng(seed)
    variations = []
    for index in range(count):
        nx, ny, nz = grids[int(rng.integers(len(grids)))]
        cell_m = 2.0 / nx
        size = [nx * cell_m, ny * cell_m, nz * cell_m]
        radius = float(rng.uniform(4.0, 10.0)) * cell_m
        jitter = rng.uniform(-0.1, 0.1, 3) * np.array(size)
        center = [float(jitter[0]), float(8.0 * (nx / 64.0) * cell_m + abs(jitter[1]) * 0.5), float(jitter[2])]
        buoyancy, drag = float(rng.uniform(0.5, 1.5)), float(rng.uniform(0.0, 0.5))
        confinement = float(rng.uniform(0.1, 0.5))
        variations.append([f"seed={7 + index}", f"domain.size_m={size!r}", f"domain.cell_m={cell_m!r}",
                           f"emitter.puff.radius_m={radius!r}", f"emitter.puff.center_m={center!r}",
                           f"forces.heat_buoyancy={buoyancy!r}", f"forces.drag_per_s={drag!r}",
                           f"forces.vorticity_confinement={confinement!r}"])
    return variations


def batched_recipes(count: int = 64, frames: int = 48, seed: int = DEFAULT_SEED, grids=BATCH_GRIDS):
    """`count` uneven smoke-puff recipes: the base recipe swept over `batch_variations` through the recipe
    front-end's `sweep_table`, so every instance passes the recipe checks."""
    from plume_b200.recipe.variation import sweep_table

    return sweep_table(batch_base_table(frames), batch_variations(count, seed, grids), "batch")
