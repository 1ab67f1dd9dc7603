"""Scheme axes: SchemeConfig (src/scheme/SchemeConfig.jl:15-77)."""
from __future__ import annotations

from dataclasses import dataclass


@dataclass(frozen=True)
class SchemeConfig:
    """Solution points (gl|gll), numerical flux (rusanov|hllc), time (ssp_rk3|ssp_rk2)."""

    points: str = "gl"
    flux: str = "rusanov"
    time: str = "ssp_rk3"

    def __post_init__(self):
        # SchemeConfig.jl:26-29: ArgumentError on unknown axes
        if self.points not in ("gl", "gll"):
            raise ValueError(f"points must be :gl or :gll, got {self.points}")
        if self.flux not in ("rusanov", "hllc"):
            raise ValueError(f"flux must be :rusanov or :hllc, got {self.flux}")
        if self.time not in ("ssp_rk3", "ssp_rk2"):
            raise ValueError(f"time must be :ssp_rk3 or :ssp_rk2, got {self.time}")


DEFAULT_SCHEME = SchemeConfig("gl", "rusanov", "ssp_rk3")


def parse_scheme(points: str = "gl", flux: str = "rusanov", time: str = "ssp_rk3") -> SchemeConfig:
    """Case-insensitive CLI axes (SchemeConfig.jl:57-66)."""
    return SchemeConfig(points.lower(), flux.lower(), time.lower().replace("-", "_"))


def scheme_dict(s: SchemeConfig) -> dict:
    """JSON-friendly record (SchemeConfig.jl:40-50)."""
    return {
        "points": "GL" if s.points == "gl" else "GLL",
        "flux": "Rusanov" if s.flux == "rusanov" else "HLLC",
        "time": "SSP-RK3" if s.time == "ssp_rk3" else "SSP-RK2",
        "points_symbol": s.points, "flux_symbol": s.flux, "time_symbol": s.time,
    }
