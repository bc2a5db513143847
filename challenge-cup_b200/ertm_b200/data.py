"""``.npz`` wire format for models, shot records and images (data.py of the
reference, data.py:33-297).

Files written here load in the reference and the reference's files load
here: the same output tree (``logs models shots images reports``), the same
array keys and dtypes, and the same ``meta`` entry — one JSON object stored
as a 0-d unicode array, with the same keys in the same order.  A shot keeps
its named components as ``component_<i>`` plus ``component_names``.
"""

from __future__ import annotations

import json
from pathlib import Path
from typing import Any

import numpy as np

from .exceptions import DataError
from .types import ElasticModel, GridSpec, ImageResult, ReceiverSpec, ShotRecord, SourceSpec

OUTPUT_SUBDIRS = ("logs", "models", "shots", "images", "reports")


def ensure_output_dirs(root: str | Path) -> dict[str, Path]:
    """The output tree under ``root``; returns ``{"root": …, "<subdir>": …}`` (data.py:33-54)."""
    base = Path(root).expanduser()
    dirs = {"root": base}
    for sub in ("",) + OUTPUT_SUBDIRS:
        path = base / sub if sub else base
        try:
            path.mkdir(parents=True, exist_ok=True)
        except OSError as exc:
            raise DataError(f"cannot create output directory {path}: {exc}") from exc
        if not path.is_dir():
            raise DataError(f"output path is not a directory: {path}")
        if sub:
            dirs[sub] = path
    return dirs


def _meta_array(meta: dict[str, Any]) -> np.ndarray:
    try:
        return np.array(json.dumps(meta, ensure_ascii=False, default=str))
    except (TypeError, ValueError) as exc:
        raise DataError(f"metadata is not JSON-serialisable: {exc}") from exc


def _meta_dict(array: np.ndarray) -> dict[str, Any]:
    try:
        value = json.loads(str(array.item()))
    except (ValueError, TypeError) as exc:
        raise DataError(f"metadata is not valid JSON: {exc}") from exc
    if not isinstance(value, dict):
        raise DataError("metadata must be a JSON object")
    return value


def _grid_meta(grid) -> dict[str, Any]:
    return {"nx": grid.nx, "nz": grid.nz, "dx": grid.dx, "dz": grid.dz, "x0": grid.x0, "z0": grid.z0}


def _grid_from(meta: dict[str, Any]) -> GridSpec:
    g = meta["grid"]
    return GridSpec(nx=int(g["nx"]), nz=int(g["nz"]), dx=float(g["dx"]), dz=float(g["dz"]),
                    x0=float(g.get("x0", 0.0)), z0=float(g.get("z0", 0.0)))


class NumpyDataStore:
    """``.npz`` store rooted at an output directory (data.py:73-297)."""

    name = "numpy-data-store"

    def __init__(self, root: str | Path) -> None:
        self.dirs = ensure_output_dirs(root)
        self.root = self.dirs["root"]

    def _write(self, path: Path, what: str, **arrays: Any) -> Path:
        try:
            np.savez_compressed(path, **arrays)
        except OSError as exc:
            raise DataError(f"cannot save {what}: {path}: {exc}") from exc
        return path

    # ------------------------------------------------------------------ model
    def save_model(self, model: ElasticModel, name: str = "model") -> Path:
        model.validate()
        meta = {"kind": "elastic_model", "name": model.name, "grid": _grid_meta(model.grid),
                "model_meta": model.meta, "units": {"length": "m", "velocity": "m/s", "density": "kg/m3"}}
        return self._write(self.dirs["models"] / f"{name}.npz", "model", vp=model.vp, vs=model.vs, rho=model.rho,
                           qp=model.qp, qs=model.qs, meta=_meta_array(meta))

    def load_model(self, path: str | Path) -> ElasticModel:
        path = Path(path)
        try:
            with np.load(path, allow_pickle=False) as z:
                meta = _meta_dict(z["meta"])
                model = ElasticModel(grid=_grid_from(meta), vp=np.asarray(z["vp"]), vs=np.asarray(z["vs"]),
                                     rho=np.asarray(z["rho"]), qp=np.asarray(z["qp"]), qs=np.asarray(z["qs"]),
                                     name=str(meta.get("name", path.stem)), meta=dict(meta.get("model_meta", {})))
        except (OSError, KeyError, ValueError) as exc:
            raise DataError(f"cannot load model: {path}: {exc}") from exc
        try:
            return model.validate()
        except ValueError as exc:
            raise DataError(f"invalid model file: {path}: {exc}") from exc

    # ------------------------------------------------------------------- shot
    def save_shot(self, shot: ShotRecord, name: str = "shot") -> Path:
        shot.validate()
        src = shot.source
        meta = {"kind": "shot_record", "dt": shot.dt, "component": shot.receivers.component,
                "components": list(shot.component_names),
                "source": {"x": src.x, "z": src.z, "f0": src.f0, "kind": src.kind, "amplitude": src.amplitude,
                           "delay": src.delay, "mechanism": src.mechanism},
                "shot_meta": shot.meta, "units": {"time": "s", "amplitude": "a.u."}}
        arrays: dict[str, Any] = {"data": shot.data, "t": shot.t, "rx": shot.receivers.x, "rz": shot.receivers.z,
                                  "meta": _meta_array(meta)}
        arrays.update({f"component_{i}": a for i, a in enumerate(shot.components.values())})
        arrays["component_names"] = np.array(list(shot.components), dtype=str)
        return self._write(self.dirs["shots"] / f"{name}.npz", "shot record", **arrays)

    def load_shot(self, path: str | Path) -> ShotRecord:
        path = Path(path)
        try:
            with np.load(path, allow_pickle=False) as z:
                meta = _meta_dict(z["meta"])
                s = meta["source"]
                source = SourceSpec(x=float(s["x"]), z=float(s["z"]), f0=float(s["f0"]), kind=str(s["kind"]),
                                    amplitude=float(s["amplitude"]), delay=float(s["delay"]),
                                    mechanism=str(s.get("mechanism", "explosive")))
                receivers = ReceiverSpec(x=np.asarray(z["rx"], dtype=float), z=np.asarray(z["rz"], dtype=float),
                                         component=str(meta.get("component", "vz")))
                components: dict[str, np.ndarray] = {}
                if "component_names" in z:
                    for i, cname in enumerate(str(v) for v in np.asarray(z["component_names"])):
                        if f"component_{i}" in z:
                            components[cname] = np.asarray(z[f"component_{i}"], dtype=np.float32)
                shot = ShotRecord(data=np.asarray(z["data"]), dt=float(meta["dt"]),
                                  t=np.asarray(z["t"], dtype=float), receivers=receivers, source=source,
                                  meta=dict(meta.get("shot_meta", {})), components=components)
        except (OSError, KeyError, ValueError) as exc:
            raise DataError(f"cannot load shot record: {path}: {exc}") from exc
        try:
            return shot.validate()
        except ValueError as exc:
            raise DataError(f"invalid shot record file: {path}: {exc}") from exc

    # ------------------------------------------------------------------ image
    def save_image(self, image: ImageResult, name: str = "image") -> Path:
        image.validate()
        meta = {"kind": "image_result", "mode": image.mode, "grid": _grid_meta(image.grid),
                "image_meta": image.meta, "units": {"length": "m", "amplitude": "a.u."}}
        return self._write(self.dirs["images"] / f"{name}.npz", "image", image=image.image, meta=_meta_array(meta))

    def load_image(self, path: str | Path) -> ImageResult:
        path = Path(path)
        try:
            with np.load(path, allow_pickle=False) as z:
                meta = _meta_dict(z["meta"])
                image = ImageResult(image=np.asarray(z["image"]), grid=_grid_from(meta),
                                    mode=str(meta.get("mode", "pp")), meta=dict(meta.get("image_meta", {})))
        except (OSError, KeyError, ValueError) as exc:
            raise DataError(f"cannot load image: {path}: {exc}") from exc
        try:
            return image.validate()
        except ValueError as exc:
            raise DataError(f"invalid image file: {path}: {exc}") from exc

    # ------------------------------------------------------------------- json
    def save_json(self, payload: Any, name: str, subdir: str = "reports") -> Path:
        if subdir not in self.dirs:
            raise DataError(f"unknown output subdirectory: {subdir}")
        path = self.dirs[subdir] / f"{name}.json"
        try:
            path.write_text(json.dumps(payload, ensure_ascii=False, indent=2, default=str) + "\n", encoding="utf-8")
        except (OSError, TypeError, ValueError) as exc:
            raise DataError(f"cannot save JSON: {path}: {exc}") from exc
        return path
