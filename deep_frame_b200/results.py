"""Result and checkpoint files of the optimisation runs, in the reference's formats.

* ``fields.npz`` — boolean ``allowed`` / ``preserve`` / ``forbidden`` masks, the
  physical ``density`` and (when present) ``design_density``
  (deep_frame/topology_pipeline.py:214-219);
* ``result.json`` — the outcome dict of ``optimize_topology`` without its array
  values, NumPy scalars and arrays converted to plain JSON, NaN rejected, written
  through a temporary file that replaces the target (:44-71, :309);
* artifact records ``{"path", "sha256", "size_bytes"}`` and their validation
  (:192-212);
* ``checkpoint(path)`` / ``keep_best(out)`` callbacks of the MMA runs
  (tools/formulation_study.py:1216-1227): ``design``, ``level``, ``iteration``
  and the best-feasible keys;
* ``design.npz`` with a ``design`` array next to a ``result.json`` that holds
  the ``grid`` (the start-design pair tools/formulation_study.py:1066,1109 reads);
* the MMA state (iteration, previous iterates, asymptotes) of
  topology_optimizers.py:75-77, saved and restored so that an interrupted
  SIMP + MMA run resumes with the same asymptotes.
All files are host-side; device tensors are copied to the host first.
"""
import hashlib
import json
from pathlib import Path

import numpy as np


def _host(value):
    if hasattr(value, "detach") and hasattr(value, "cpu"):
        return value.detach().cpu().numpy()
    return value


_LEAF = ((np.ndarray, lambda v: v.tolist()), (np.generic, lambda v: v.item()), (Path, str))


def jsonable(value):
    """Plain-JSON copy: dict keys as strings, arrays and tensors as lists, NumPy scalars as Python numbers."""
    value = _host(value)
    for kind, convert in _LEAF:
        if isinstance(value, kind):
            return convert(value)
    if isinstance(value, dict):
        return {str(key): jsonable(item) for key, item in value.items()}
    if isinstance(value, (tuple, list)):
        return list(map(jsonable, value))
    return value


def save_json(path, value):
    """Write ``value`` as JSON so that readers see the old file or the complete new one, never a part:
    the text goes to a sibling temporary file that then replaces the target.  NaN and infinities
    raise ValueError (and leave the target untouched)."""
    target = Path(path)
    target.parent.mkdir(parents=True, exist_ok=True)
    text = json.dumps(jsonable(value), indent=2, allow_nan=False)
    staging = target.with_name(target.name + ".tmp")
    staging.write_text(text, encoding="utf-8")
    staging.replace(target)


def read_json(path):
    return json.loads(Path(path).read_text(encoding="utf-8"))


def file_digest(path):
    return hashlib.sha256(Path(path).read_bytes()).hexdigest()


def artifact(path, directory):
    path = Path(path)
    return {"path": str(path.relative_to(directory)).replace("\\", "/"), "sha256": file_digest(path), "size_bytes": path.stat().st_size}


def valid_artifacts(record, directory):
    """True when every artifact of ``record`` that names a digest is a file under ``directory`` with
    that SHA-256."""
    root = Path(directory)
    listed = [item for item in record.get("artifacts", {}).values() if isinstance(item, dict) and "sha256" in item]
    return all((root / item["path"]).is_file() and file_digest(root / item["path"]) == item["sha256"] for item in listed)


def save_fields(path, domain, result):
    """fields.npz: the domain masks and the result's physical (and, if present, design) density."""
    arrays = {"density": np.asarray(_host(result["density"]), dtype=float)}
    if result.get("design_density") is not None:
        arrays["design_density"] = np.asarray(_host(result["design_density"]), dtype=float)
    arrays.update({name: np.asarray(domain[name], dtype=bool) for name in ("allowed", "preserve", "forbidden")})
    Path(path).parent.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(path, **arrays)


def write_outcome(directory, domain, outcome, name="run"):
    """fields.npz + result.json of one optimisation outcome; returns the artifact record."""
    directory = Path(directory)
    directory.mkdir(parents=True, exist_ok=True)
    save_fields(directory / "fields.npz", domain, outcome)
    save_json(directory / "result.json", {key: value for key, value in outcome.items() if not isinstance(_host(value), np.ndarray)})
    return {"name": name, "status": outcome["status"],
            "artifacts": {"fields": artifact(directory / "fields.npz", directory), "result": artifact(directory / "result.json", directory)}}


def read_outcome(directory, record=None):
    """The outcome written by ``write_outcome`` with its density arrays restored; None when an artifact changed."""
    directory = Path(directory)
    if record is not None and not valid_artifacts(record, directory):
        return None
    result = read_json(directory / "result.json")
    with np.load(directory / "fields.npz", allow_pickle=False) as fields:
        result["density"] = fields["density"].copy()
        if "design_density" in fields:
            result["design_density"] = fields["design_density"].copy()
    return result


def save_design(directory, design, grid, extra=None):
    """design.npz (key ``design``) and result.json with the ``grid`` record: a start design for another run."""
    directory = Path(directory)
    directory.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(directory / "design.npz", design=np.asarray(_host(design), dtype=float))
    save_json(directory / "result.json", {"grid": grid, **(extra or {})})


def load_design(directory):
    directory = Path(directory)
    with np.load(directory / "design.npz", allow_pickle=False) as data:
        design = data["design"].copy()
    return design, read_json(directory / "result.json")["grid"]


def checkpoint(path):
    """Callback save(x, history, levels): the design, the level of the last history row and the iteration count."""
    def save(x, history, levels):
        np.savez_compressed(path, design=np.asarray(_host(x), dtype=float), level=history[-1].get("level", 0), iteration=len(history))
    return save


def keep_best(out):
    """Callback save(x, best): best_beta{beta}.npz with the design and the best-feasible record."""
    out = Path(out)

    def save(x, best):
        np.savez_compressed(out / f"best_beta{best['beta']:g}.npz", design=np.asarray(_host(x), dtype=float),
                            **{key: best[key] for key in ("iteration", "level", "beta", "f0", "mass_g", "max_violation")})
    return save


MMA_STATE_KEYS = ("old1", "old2", "low", "upp")


def save_mma_state(path, x, state, history=None):
    """Design, MMA iteration counter, previous iterates and asymptotes (+ the run's objective scale)."""
    arrays = {key: np.asarray(_host(state[key]), dtype=float) for key in MMA_STATE_KEYS}
    extra = {"objective_scale": float(state["objective_scale"])} if state.get("objective_scale") is not None else {}
    np.savez_compressed(path, design=np.asarray(_host(x), dtype=float), iteration=int(state["iteration"]),
                        history=json.dumps(jsonable(history or []), allow_nan=False), **arrays, **extra)


def load_mma_state(path):
    """(design, state, history) written by ``save_mma_state``."""
    with np.load(path, allow_pickle=False) as data:
        state = {key: data[key].copy() for key in MMA_STATE_KEYS}
        state["iteration"] = int(data["iteration"])
        if "objective_scale" in data:
            state["objective_scale"] = float(data["objective_scale"])
        return data["design"].copy(), state, json.loads(str(data["history"]))
