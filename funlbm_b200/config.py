"""Configuration objects with the reference's JSON keys and parsing rules.

Mirrors funlbm's ``config/base.py`` (BoundaryCondition, BaseConfig, Boundary,
BoundaryConfig, FileConfig).  Every value is read as ``lookup or default``
like the reference (config/base.py:99 and every ``_from_json``), so a value of
0 / 0.0 / "" silently falls back to the default -- a reference quirk kept for
drop-in compatibility.
"""
from __future__ import annotations

import json
import os
from enum import Enum
from typing import Any, Dict, Optional, Union


def deep_get(obj, key, default=None):
    """Dictionary lookup; a dotted key walks nested dictionaries."""
    if obj is None:
        return default
    cur = obj
    for part in str(key).split("."):
        if isinstance(cur, dict) and part in cur:
            cur = cur[part]
        else:
            return default
    return cur


class BoundaryCondition(Enum):
    """Face codes of config/base.py:9-45 (values kept: they travel to the C ABI)."""

    PERIODICAL = 11000
    WALL = 1200
    WALL_WITH_SPEED = 1201
    FAR_FIELD = 1300
    NON_EQUILIBRIUM = 1400
    NON_EQUILIBRIUM_EXREAPOLATION = 1500
    FULL_DEVELOPMENT = 1600

    @classmethod
    def find(cls, code: Union[int, str]) -> "BoundaryCondition":
        """By value or name; anything unknown becomes WALL (config/base.py:29-45)."""
        try:
            if isinstance(code, int):
                return next(bc for bc in cls if bc.value == code)
            return cls[str(code)]
        except (StopIteration, KeyError):
            return cls.WALL


class BaseConfig:
    """JSON-backed configuration (config/base.py:48-103)."""

    def __init__(self, *args, **kwargs) -> None:
        self.expand: Dict[str, Any] = kwargs.copy()

    def _from_json(self, config_json: Dict[str, Any], **kwargs) -> None:
        pass

    def from_file(self, path: str) -> "BaseConfig":
        with open(path) as fh:
            self.from_json(json.load(fh))
        return self

    def from_json(self, config_json: Dict[str, Any], **kwargs) -> "BaseConfig":
        self.expand.update(kwargs)
        self.expand.update(config_json)
        self._from_json(config_json, **kwargs)
        return self

    def get(self, key: str, default: Any = None) -> Any:
        return deep_get(self.expand, key) or default

    def to_json(self) -> Dict[str, Any]:
        return self.expand


class Boundary(BaseConfig):
    """One face (config/base.py:106-137).  ``uw`` (wall velocity of a
    WALL_WITH_SPEED face) is read as a 3-vector; the reference's own lookup of
    it fails for every value (``x or default`` on a list/tensor)."""

    def __init__(self, condition: BoundaryCondition = BoundaryCondition.WALL, *args, **kwargs):
        super().__init__(*args, **kwargs)
        self.condition: BoundaryCondition = condition
        self.poiseuille: Optional[Any] = None

    def is_condition(self, condition: BoundaryCondition) -> bool:
        return self.condition == condition

    def _from_json(self, config_json: Dict[str, Any], **kwargs) -> None:
        self.condition = BoundaryCondition.find(deep_get(config_json, "code") or "WALL")
        self.poiseuille = deep_get(config_json, "poiseuille")

    def wall_velocity(self):
        uw = deep_get(self.expand, "uw")
        if uw is None:
            return (0.0, 0.0, 0.0)
        if isinstance(uw, (int, float)):
            return (float(uw), 0.0, 0.0)
        vals = [float(v) for v in uw]
        if len(vals) != 3:
            raise ValueError("uw must have three components, got %r" % (uw,))
        return tuple(vals)


FACES = ("input", "output", "back", "forward", "bottom", "top")


class BoundaryConfig(BaseConfig):
    """The six faces (config/base.py:140-156): input/output are x = 0 / x = max,
    back/forward y = 0 / max, bottom/top z = 0 / max."""

    def __init__(self, *args, **kwargs) -> None:
        super().__init__(*args, **kwargs)
        for face in FACES:
            setattr(self, face, Boundary(BoundaryCondition.WALL))

    def _from_json(self, config_json: Dict[str, Any], **kwargs) -> None:
        for face in FACES:
            getattr(self, face).from_json(deep_get(config_json, face) or {})

    def codes(self):
        return [getattr(self, face).condition.value for face in FACES]


class FileConfig(BaseConfig):
    """Output locations (config/base.py:159-195)."""

    def __init__(self, *args, **kwargs) -> None:
        super().__init__(*args, **kwargs)
        self.cache_dir: str = "./data"
        self.per_steps: int = 100

    def _path(self, sub):
        path = os.path.join(self.cache_dir, sub)
        os.makedirs(path, exist_ok=True)
        return path

    @property
    def vtk_path(self) -> str:
        return self._path("vtk")

    @property
    def tecplot_path(self) -> str:
        return self._path("tecplot")

    @property
    def checkpoint_path(self) -> str:
        return self._path("checkpoint")

    def _from_json(self, config_json: Dict[str, Any], **kwargs) -> None:
        self.cache_dir = deep_get(config_json, "cache_dir") or self.cache_dir
        self.per_steps = deep_get(config_json, "per_steps") or self.per_steps
