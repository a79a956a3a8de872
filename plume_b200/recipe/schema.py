"""Recipe tables the hot path reads, as frozen dataclasses.

Key names, nesting and defaults follow chadmv/plume src/plume/recipe/schema.py:60-247 so that a recipe written
for the reference loads here unchanged (a recipe is a file format: its keys have to match). Only the tables
the simulation, the render, the sheet geometry and the viewer's look use are modelled (the contact sheets'
`look.backgrounds` is accepted and ignored).
"""

from dataclasses import dataclass, field

Vec3 = tuple[float, float, float]

SEED_MAX = 2**31 - 1
SHADE_LAYOUT = "heat,thickness,shade,unused"
NORMAL_LAYOUT = "heat,thickness,normal_x,normal_y"
CHANNEL_LAYOUTS = (SHADE_LAYOUT, NORMAL_LAYOUT)
FACE_KINDS = ("closed", "open")


@dataclass(frozen=True, kw_only=True)
class FaceSettings:
    bottom: str = "closed"
    top: str = "open"
    left: str = "open"
    right: str = "open"
    back: str = "open"
    front: str = "open"


@dataclass(frozen=True, kw_only=True)
class DomainSettings:
    size_m: Vec3
    cell_m: float
    ambient_k: float = 293.0
    faces: FaceSettings = field(default_factory=FaceSettings)


@dataclass(frozen=True, kw_only=True)
class TimeSettings:
    duration_s: float
    frames: int = 64
    substeps: int = 3
    warmup_s: float = 0.0


@dataclass(frozen=True, kw_only=True)
class NoiseSettings:
    scale_m: float = 0.1
    strength: float = 0.0


@dataclass(frozen=True, kw_only=True)
class EmitterSettings:
    name: str
    center_m: Vec3
    end_s: float
    shape: str = "sphere"
    radius_m: float = 0.0
    size_m: Vec3 = (0.0, 0.0, 0.0)
    edge_softness: float = 0.3
    start_s: float = 0.0
    smoke_per_s: float = 0.0
    temperature_k: float = -1.0
    velocity_mps: Vec3 = (0.0, 0.0, 0.0)
    velocity_mode: str = "fixed"
    noise: NoiseSettings = field(default_factory=NoiseSettings)


@dataclass(frozen=True, kw_only=True)
class TurbulenceSettings:
    scale_m: float = 0.3
    strength_mps2: float = 0.0
    speed_mps: float = 0.2


@dataclass(frozen=True, kw_only=True)
class ForceSettings:
    gravity_mps2: float = 9.81
    heat_buoyancy: float = 1.0
    smoke_weight: float = 0.0
    wind_mps: Vec3 = (0.0, 0.0, 0.0)
    drag_per_s: float = 0.0
    vorticity_confinement: float = 0.0
    turbulence: TurbulenceSettings = field(default_factory=TurbulenceSettings)


@dataclass(frozen=True, kw_only=True)
class DissipationSettings:
    smoke_per_s: float = 0.0
    cooling_per_s: float = 0.0


@dataclass(frozen=True, kw_only=True)
class SolverSettings:
    pressure_solver: str = "multigrid"
    pressure_iterations: int = 60
    multigrid_cycles: int = 2
    multigrid_sweeps: int = 2
    max_cells_per_step: float = 1.0
    max_substeps: int = 32


@dataclass(frozen=True, kw_only=True)
class CameraSettings:
    elevation_deg: float = 0.0
    azimuth_deg: float = 0.0
    seat: str = ""


@dataclass(frozen=True, kw_only=True)
class RenderSettings:
    px_per_cell: float = 2.0
    opacity_per_density: float = 4.0
    glow_start_k: float = 600.0
    smoke_hides_heat: float = 1.0
    normal_blur_cells: float = 1.5
    normal_fade_thickness: float = 0.1
    light_dir: Vec3 = (-0.5, 0.7, 0.5)
    shade_fill: float = 0.25
    shade_fade_thickness: float = 0.1
    shade_neighborhood_px: float = 4.0
    soften_px: float = 0.75
    crop_margin: float = 0.04


@dataclass(frozen=True, kw_only=True)
class OutputSettings:
    name: str = ""
    frame_px: int = 256
    columns: int = 0
    channels: str = SHADE_LAYOUT


@dataclass(frozen=True, kw_only=True)
class PreviewSettings:
    longest_axis_cells: int = 48
    frames: int = 16
    frame_px: int = 128


ColorStop = tuple[float, str]


@dataclass(frozen=True, kw_only=True)
class LookSettings:
    """How the contact sheets and the viewer light a sheet frame (chadmv/plume recipe/schema.py:214-225)."""

    ambient: float = 0.65
    shade_depth: float = 0.75
    smoke_ramp: tuple[ColorStop, ...] = ((0.0, "#aea193"), (0.4, "#bc9c84"), (0.75, "#dca07a"), (1.0, "#f5b47e"))
    emission_ramp: tuple[ColorStop, ...] = ((0.0, "#000000"), (0.2, "#3a0c04"), (0.5, "#c4441a"), (0.8, "#ff9a3a"),
                                            (1.0, "#fff2c2"))
    contact_px: int = 128


@dataclass(frozen=True, kw_only=True)
class Recipe:
    emitter: tuple[EmitterSettings, ...]
    domain: DomainSettings
    time: TimeSettings
    seed: int = 0
    extends: str = ""
    forces: ForceSettings = field(default_factory=ForceSettings)
    dissipation: DissipationSettings = field(default_factory=DissipationSettings)
    solver: SolverSettings = field(default_factory=SolverSettings)
    camera: CameraSettings = field(default_factory=CameraSettings)
    render: RenderSettings = field(default_factory=RenderSettings)
    output: OutputSettings = field(default_factory=OutputSettings)
    preview: PreviewSettings = field(default_factory=PreviewSettings)
    look: LookSettings = field(default_factory=LookSettings)
