"""Simulation parameters for the B200 leapfrog path.

The field names, defaults and validation rules match the reference's
``SimulationConfig`` (lfm/config.py:145-347) so that a config object from
either package drives :class:`lfm_b200.Evolver`.  Only the parameters that
reach the time-step kernels, the boundary sponge and the report metrics are
kept; the Planck-unit metadata and the physical-scale auto-selection of the
reference are outside this path.

Constants follow lfm/constants.py:33-142 (all derived from chi0 = 19).
"""

from __future__ import annotations

import enum
import math
from dataclasses import dataclass, field

# --- constants (lfm/constants.py) -------------------------------------------
D = 3
D_ST = D + 1
CHI0 = float(3**D - 2**D)  # 19.0
N_COLORS = 3
KAPPA = 1.0 / (4**D - 1)  # 1/63
LAMBDA_H = D_ST / (2 * D_ST**2 - 1)  # 4/31
EPSILON_W = 2.0 / (CHI0 + 1)  # 0.1
ALPHA_S = 2.0 / (CHI0 - 2)  # 2/17
KAPPA_C = KAPPA / N_COLORS  # 1/189
EPSILON_CC = ALPHA_S
BETA_0 = int(CHI0) - 12
SA_GAMMA = EPSILON_W
SA_L = BETA_0
SA_D = SA_GAMMA * SA_L**2  # 4.9
Z2_COORD = 2 * D_ST**2
RANK_SU3 = N_COLORS - 1
KAPPA_TUBE = (Z2_COORD - RANK_SU3) * KAPPA  # 30/63
KAPPA_STRING = KAPPA_C
DT_DEFAULT = 0.02
C_DEFAULT = 1.0
E0_SQ_DEFAULT = 0.0
BOUNDARY_FRACTION_DEFAULT = 0.3
STENCIL_FACE_WEIGHT = 1.0 / 3.0
STENCIL_EDGE_WEIGHT = 1.0 / 6.0
STENCIL_CENTER_WEIGHT = -4.0
WELL_THRESHOLD = 17.0
VOID_THRESHOLD = 18.0
# Default soliton amplitude per grid size when e_amplitude is left at 0.
E_AMPLITUDE_BY_GRID = {32: 12.0, 64: 6.0, 128: 3.6, 256: 1.8, 512: 0.9}


# Physical radius of the observable universe in Planck lengths: the default
# box_planck_radius (metadata only; lfm/constants.py:238-254).
PLANCK_TIME_SEC = 5.391e-44
AGE_UNIVERSE_GYR = 13.8
SEC_PER_GYR = 1e9 * 365.25 * 24 * 3600
OBSERVABLE_RADIUS_PLANCK = (AGE_UNIVERSE_GYR * SEC_PER_GYR) / PLANCK_TIME_SEC


class ChiMode(enum.Enum):
    """GOV-02 update rule named by the config (lfm/config.py:49-67).  The step
    kernels implement WAVE, the full second-order chi equation."""

    WAVE = "wave"
    MEMORY = "memory"
    STATIC = "static"


class PhysicsScale(enum.Enum):
    """Named physical scale (lfm/config.py:70-129); setting one on the config
    selects the field level, chi mode and couplings below."""

    PLANCK = "planck"
    NUCLEAR = "nuclear"
    ATOMIC = "atomic"
    MOLECULAR = "molecular"
    CLASSICAL = "classical"
    SOLAR = "solar"
    GALACTIC = "galactic"
    COSMIC = "cosmic"


class FieldLevel(enum.IntEnum):
    """Field representation: real E, one complex Psi, or three colour components."""

    REAL = 0
    COMPLEX = 1
    COLOR = 2


class BoundaryType(enum.Enum):
    """Recorded for checkpoint compatibility.

    The step kernels always apply the cos^2 sponge, whatever this says: the
    reference's backends never read it (lfm/core/evolver.py:201-279).
    """

    FROZEN = "frozen"
    PERIODIC = "periodic"
    ABSORBING = "absorbing"


_SCALE_DEFAULTS = {
    PhysicsScale.PLANCK: (FieldLevel.COLOR, ChiMode.WAVE, LAMBDA_H, KAPPA_C),
    PhysicsScale.NUCLEAR: (FieldLevel.COLOR, ChiMode.WAVE, LAMBDA_H, KAPPA_C),
    PhysicsScale.ATOMIC: (FieldLevel.COMPLEX, ChiMode.WAVE, 0.0, 0.0),
    PhysicsScale.MOLECULAR: (FieldLevel.COMPLEX, ChiMode.WAVE, 0.0, 0.0),
    PhysicsScale.CLASSICAL: (FieldLevel.REAL, ChiMode.WAVE, 0.0, 0.0),
    PhysicsScale.SOLAR: (FieldLevel.REAL, ChiMode.WAVE, 0.0, 0.0),
    PhysicsScale.GALACTIC: (FieldLevel.REAL, ChiMode.MEMORY, 0.0, 0.0),
    PhysicsScale.COSMIC: (FieldLevel.REAL, ChiMode.MEMORY, 0.0, 0.0),
}


@dataclass
class SimulationConfig:
    """Parameters of one lattice run (names and defaults as lfm/config.py:153-247)."""

    grid_size: int = 128
    chi0: float = CHI0
    kappa: float = KAPPA
    lambda_self: float = 0.0
    epsilon_w: float = EPSILON_W
    kappa_c: float = 0.0
    epsilon_cc: float = 0.0
    kappa_string: float = 0.0
    kappa_tube: float = 0.0
    sa_gamma: float = SA_GAMMA
    sa_d: float = SA_D
    e0_sq: float = E0_SQ_DEFAULT
    dt: float = DT_DEFAULT
    c: float = C_DEFAULT
    field_level: FieldLevel = FieldLevel.REAL
    n_colors: int = N_COLORS
    boundary_type: BoundaryType = BoundaryType.FROZEN
    boundary_fraction: float = BOUNDARY_FRACTION_DEFAULT
    e_amplitude: float = 0.0
    blob_sigma_factor: float = 12.0
    phase1_steps: int = 10_000
    phase1_omega: float = 38.0
    phase1_amplitude: float = 0.3
    random_seed: int = 42
    report_interval: int = 5000
    box_planck_radius: float = OBSERVABLE_RADIUS_PLANCK
    physical_scale: PhysicsScale | None = None
    chi_mode: ChiMode = ChiMode.WAVE
    dx: float = field(init=False, default=1.0)
    sigma: float = field(init=False, default=0.0)

    def __post_init__(self) -> None:
        if self.physical_scale is not None:
            self.physical_scale = PhysicsScale(self.physical_scale)
            fl, cm, ls, kc = _SCALE_DEFAULTS[self.physical_scale]
            self.field_level, self.chi_mode, self.lambda_self, self.kappa_c = fl, cm, ls, kc
        if not isinstance(self.chi_mode, ChiMode):
            self.chi_mode = ChiMode(self.chi_mode)
        self.field_level = FieldLevel(int(self.field_level))
        if not isinstance(self.boundary_type, BoundaryType):
            self.boundary_type = BoundaryType(self.boundary_type)
        self._validate()
        self.dx = 1.0
        self.sigma = self.grid_size / self.blob_sigma_factor
        if self.e_amplitude == 0.0:
            self.e_amplitude = E_AMPLITUDE_BY_GRID.get(self.grid_size, 3.6)

    def _validate(self) -> None:
        # Same checks and messages as lfm/config.py:306-334.
        if self.grid_size < 8:
            raise ValueError(f"grid_size must be >= 8, got {self.grid_size}")
        if self.dt <= 0:
            raise ValueError(f"dt must be positive, got {self.dt}")
        cfl_limit = 1.0 / math.sqrt(16.0 / 3.0 + self.chi0**2)
        if self.dt > cfl_limit:
            raise ValueError(
                f"dt={self.dt} exceeds CFL limit {cfl_limit:.4f} "
                f"for 19-point stencil with χ₀={self.chi0}"
            )
        if self.chi0 <= 0:
            raise ValueError(f"chi0 must be > 0, got {self.chi0}")
        if self.kappa < 0:
            raise ValueError(f"kappa must be >= 0, got {self.kappa}")
        if self.lambda_self < 0:
            raise ValueError(f"lambda_self must be >= 0, got {self.lambda_self}")
        if not 0 < self.boundary_fraction < 1:
            raise ValueError(f"boundary_fraction must be in (0, 1), got {self.boundary_fraction}")
        if self.field_level == FieldLevel.COLOR and self.n_colors < 1:
            raise ValueError(f"n_colors must be >= 1, got {self.n_colors}")

    @property
    def sa_enabled(self) -> bool:
        """True when the S_a Helmholtz fields are active (kappa_tube > 0)."""
        return self.kappa_tube > 0.0


def gravity_only(grid_size: int = 64, **overrides: object) -> SimulationConfig:
    """REAL level, gravity only (lfm/config_presets.py:29-40)."""
    params: dict[str, object] = dict(
        grid_size=grid_size, field_level=FieldLevel.REAL, boundary_type=BoundaryType.FROZEN
    )
    params.update(overrides)
    return SimulationConfig(**params)  # type: ignore[arg-type]


def gravity_em(grid_size: int = 64, **overrides: object) -> SimulationConfig:
    """COMPLEX level with the Mexican hat on (lfm/config_presets.py:43-56)."""
    params: dict[str, object] = dict(
        grid_size=grid_size,
        field_level=FieldLevel.COMPLEX,
        boundary_type=BoundaryType.FROZEN,
        lambda_self=LAMBDA_H,
    )
    params.update(overrides)
    return SimulationConfig(**params)  # type: ignore[arg-type]


def full_physics(grid_size: int = 64, **overrides: object) -> SimulationConfig:
    """COLOR level with every coupling on (lfm/config_presets.py:59-79)."""
    params: dict[str, object] = dict(
        grid_size=grid_size,
        field_level=FieldLevel.COLOR,
        boundary_type=BoundaryType.FROZEN,
        lambda_self=LAMBDA_H,
        kappa_c=KAPPA_C,
        epsilon_cc=EPSILON_CC,
        kappa_string=KAPPA_STRING,
        kappa_tube=KAPPA_TUBE,
        sa_gamma=SA_GAMMA,
        sa_d=SA_D,
    )
    params.update(overrides)
    return SimulationConfig(**params)  # type: ignore[arg-type]
