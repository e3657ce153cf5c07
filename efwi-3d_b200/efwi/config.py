"""The reference's para and survey JSON files.

Para file (written by fwi_utils.paraGen_3d, read by Parameter.cpp:15-185):
``nz, nx, ny`` (padded sizes), ``dz, dx, dy, nSteps, dt, f0, nPoints_pml,
survey_fname, data_dir_name`` and the optional ``if_win, filter,
if_src_update, scratch_dir_name, if_cross_misfit``.

Survey file (fwi_utils.surveyGen_3d, read by Src_Rec.cu:20-206):
``nShots`` and ``shot{i}: {z_src, x_src, y_src, nrec, z_rec[], x_rec[],
y_rec[]}`` with optional ``win_start[], win_end[], weights[], src_weight``.
Coordinates are model-relative; nPoints_pml is added here, as the reference
does (Src_Rec.cu:78-118).

Parsing is strict where the reference asserts: a missing key raises
:class:`ConfigError` instead of ending the process.
"""
from __future__ import annotations

import json
import os
from dataclasses import dataclass
from typing import Dict, List, Optional

import numpy as np

from .engine import Grid, Shot


class ConfigError(ValueError):
    pass


@dataclass
class Para:
    grid: Grid
    survey_fname: str
    data_dir_name: str
    scratch_dir_name: Optional[str] = None
    if_win: bool = False
    filter: Optional[list] = None
    if_src_update: bool = False
    if_cross_misfit: bool = False


def _need(d: dict, key: str, where: str):
    if key not in d:
        raise ConfigError(f"{where}: missing key '{key}'")
    return d[key]


def _int(d, key, where):
    v = _need(d, key, where)
    if isinstance(v, bool) or not isinstance(v, int):
        raise ConfigError(f"{where}: '{key}' must be an integer")
    return v


def _num(d, key, where):
    v = _need(d, key, where)
    if isinstance(v, bool) or not isinstance(v, (int, float)):
        raise ConfigError(f"{where}: '{key}' must be a number")
    return float(v)


def _load_json(path: str) -> dict:
    if not os.path.exists(path):
        raise ConfigError(f"cannot open {path}")
    with open(path) as fp:
        try:
            d = json.load(fp)
        except json.JSONDecodeError as e:
            raise ConfigError(f"{path}: invalid JSON ({e})") from None
    if not isinstance(d, dict):
        raise ConfigError(f"{path}: not a JSON object")
    return d


def read_para(path: str) -> Para:
    d = _load_json(path)
    w = os.path.basename(path)
    grid = Grid(nz=_int(d, "nz", w), nx=_int(d, "nx", w), ny=_int(d, "ny", w),
                npml=_int(d, "nPoints_pml", w), nt=_int(d, "nSteps", w), dz=_num(d, "dz", w),
                dx=_num(d, "dx", w), dy=_num(d, "dy", w), dt=_num(d, "dt", w),
                f0=_num(d, "f0", w))
    p = Para(grid=grid, survey_fname=str(_need(d, "survey_fname", w)),
             data_dir_name=str(_need(d, "data_dir_name", w)))
    if "scratch_dir_name" in d:
        p.scratch_dir_name = str(d["scratch_dir_name"])
    for key in ("if_win", "if_src_update", "if_cross_misfit"):
        if key in d:
            if not isinstance(d[key], bool):
                raise ConfigError(f"{w}: '{key}' must be a boolean")
            setattr(p, key, d[key])
    if "filter" in d:
        p.filter = list(d["filter"])
    return p


def read_survey(path: str, npml: int, if_win: bool = False) -> List[Shot]:
    d = _load_json(path)
    w = os.path.basename(path)
    nshots = _int(d, "nShots", w)
    shots = []
    for i in range(nshots):
        key = f"shot{i}"
        if key not in d:
            # Only shots that are used are read by the reference; keep a
            # placeholder so that indices stay aligned.
            shots.append(None)
            continue
        s = d[key]
        nrec = _int(s, "nrec", key)
        z = np.asarray(_need(s, "z_rec", key), dtype=np.int64) + npml
        x = np.asarray(_need(s, "x_rec", key), dtype=np.int64) + npml
        y = np.asarray(_need(s, "y_rec", key), dtype=np.int64) + npml
        if not (len(z) == len(x) == len(y) == nrec):
            raise ConfigError(f"{key}: nrec={nrec} but receiver arrays have {len(z)}/{len(x)}/{len(y)}")
        shot = Shot(src=(_int(s, "z_src", key) + npml, _int(s, "x_src", key) + npml,
                         _int(s, "y_src", key) + npml), z_rec=z, x_rec=x, y_rec=y)
        if if_win:
            shot.win_start = np.asarray(_need(s, "win_start", key), dtype=np.float32)
            shot.win_end = np.asarray(_need(s, "win_end", key), dtype=np.float32)
        if "weights" in s:
            shot.weights = np.asarray(s["weights"], dtype=np.float32)
        if "src_weight" in s:
            shot.src_weight = float(s["src_weight"])
        shots.append(shot)
    return shots


def shot_file(data_dir: str, comp: str, shot_id: int) -> str:
    """Observed-data file of one component (libCUFD.cu:277-279, 709-720)."""
    return os.path.join(data_dir, f"Shot_{comp}{shot_id}.bin")


def read_shot_data(data_dir: str, shot_id: int, nrec: int, nt: int) -> np.ndarray:
    """[3][nrec][nt] float32 from Shot_{x,y,z}{id}.bin."""
    out = np.empty((3, nrec, nt), np.float32)
    for c, comp in enumerate("xyz"):
        fn = shot_file(data_dir, comp, shot_id)
        if not os.path.exists(fn):
            raise ConfigError(f"Attempted to read {fn}: file reading error")
        a = np.fromfile(fn, dtype=np.float32, count=nrec * nt)
        if a.size != nrec * nt:
            raise ConfigError(f"{fn}: {a.size} samples, expected {nrec * nt}")
        out[c] = a.reshape(nrec, nt)
    return out


def write_shot_data(data_dir: str, shot_id: int, traces: np.ndarray, prefix: str = "Shot_") -> None:
    os.makedirs(data_dir, exist_ok=True)
    for c, comp in enumerate("xyz"):
        np.ascontiguousarray(traces[c], np.float32).tofile(
            os.path.join(data_dir, f"{prefix}{comp}{shot_id}.bin"))


def write_problem(dirpath: str, grid, shots, traces=None, shot_ids=None) -> str:
    """Writes the para JSON, the survey JSON and (optionally) observed data
    Shot_{x,y,z}{id}.bin of a problem into `dirpath`, in the formats the
    reference reads (Parameter.cpp, Src_Rec.cu, libCUFD.cu:277-279): padded
    sizes in the para file, model-relative indices in the survey.  `traces`
    is a list of [3][nrec][nt] arrays of the shots `shot_ids`.  Returns the
    para file's path."""
    import fwi_utils as ft
    para = os.path.join(dirpath, "para_file.json")
    survey = os.path.join(dirpath, "survey_file.json")
    data = os.path.join(dirpath, "Data")
    g = grid
    ft.paraGen_3d(g.nz, g.nx, g.ny, g.dz, g.dx, g.dy, g.nt, g.dt, g.f0, g.npml, para, survey, data)
    sv = {"nShots": len(shots)}
    for k, s in enumerate(shots):
        sv[f"shot{k}"] = {"z_src": int(s.src[0]) - g.npml, "x_src": int(s.src[1]) - g.npml,
                          "y_src": int(s.src[2]) - g.npml, "nrec": s.nrec,
                          "z_rec": (np.asarray(s.z_rec) - g.npml).tolist(),
                          "x_rec": (np.asarray(s.x_rec) - g.npml).tolist(),
                          "y_rec": (np.asarray(s.y_rec) - g.npml).tolist()}
    with open(survey, "w") as fp:
        json.dump(sv, fp)
    if traces is not None:
        for k, t in zip(shot_ids, traces):
            write_shot_data(data, k, np.asarray(t))
    return para
