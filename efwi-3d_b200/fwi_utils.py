"""Drop-in for the reference's Ops/FWI/fwi_utils.py.

Same function names, arguments and file formats, so that the reference's
drivers run unchanged with ``sys.path.append("efwi-3d_b200")``:

* padding_3d   replicate padding by nPml on every face (fwi_utils.py:9-20)
* paraGen_3d   writes the para JSON read by the solver (fwi_utils.py:22-60)
* surveyGen_3d writes the survey JSON (fwi_utils.py:63-88)
* sourceGene   integrated Ricker wavelet (fwi_utils.py:90-105)
"""
from __future__ import annotations

import json
import os

import numpy as np
import torch
import torch.nn.functional as F


def padding_3d(cp, cs, den, nz, nx, ny, nPml):
    """Replicate-pads three [nz, nx, ny] volumes by nPml cells per face."""
    p = int(nPml)
    shape = (int(nz) + 2 * p, int(nx) + 2 * p, int(ny) + 2 * p)

    def pad(v):
        v5 = v.reshape(1, 1, int(nz), int(nx), int(ny))
        return F.pad(v5, pad=(p, p, p, p, p, p), mode="replicate").reshape(shape)

    return pad(cp), pad(cs), pad(den)


def paraGen_3d(nz, nx, ny, dz, dx, dy, nSteps, dt, f0, nPml, para_fname, survey_fname,
               data_dir_name, if_win=False, filter_para=None, if_src_update=False,
               scratch_dir_name='', if_cross_misfit=False):
    """Writes the para JSON (one line).  nz, nx, ny are the padded sizes."""
    para = {"nz": int(nz), "nx": int(nx), "ny": int(ny), "dz": float(dz), "dx": float(dx),
            "dy": float(dy), "nSteps": int(nSteps), "dt": float(dt), "f0": float(f0),
            "nPoints_pml": int(nPml)}
    if if_win:
        para["if_win"] = True
    if filter_para is not None:
        para["filter"] = filter_para
    if if_src_update:
        para["if_src_update"] = True
    para["survey_fname"] = survey_fname
    para["data_dir_name"] = data_dir_name
    os.makedirs(data_dir_name, exist_ok=True)
    if if_cross_misfit:
        para["if_cross_misfit"] = True
    if scratch_dir_name != '':
        para["scratch_dir_name"] = scratch_dir_name
        os.makedirs(scratch_dir_name, exist_ok=True)
    d = os.path.dirname(para_fname)
    if d:
        os.makedirs(d, exist_ok=True)
    with open(para_fname, "w") as fp:
        json.dump(para, fp)


def surveyGen_3d(z_src, x_src, y_src, z_rec, x_rec, y_rec, survey_fname, Windows=None,
                 Weights=None, Src_Weights=None, Src_rxz=None, Rec_rxz=None):
    """Writes the survey JSON.  Source arrays are 2-D [n_src_x, n_src_y];
    shot i takes element (i % n_src_x, i // n_src_x); every shot records on
    the same receivers (model-relative indices)."""
    xs, zs, ys = (np.asarray(a).tolist() for a in (x_src, z_src, y_src))
    xr, zr, yr = (np.asarray(a).tolist() for a in (x_rec, z_rec, y_rec))
    n0 = len(xs)
    nsrc = n0 * len(xs[0])
    survey = {"nShots": nsrc}
    for i in range(nsrc):
        a, b = i % n0, i // n0
        survey[f"shot{i}"] = {"z_src": zs[a][b], "x_src": xs[a][b], "y_src": ys[a][b],
                              "nrec": len(xr), "z_rec": zr, "x_rec": xr, "y_rec": yr}
    d = os.path.dirname(survey_fname)
    if d:
        os.makedirs(d, exist_ok=True)
    with open(survey_fname, "w") as fp:
        json.dump(survey, fp)


def sourceGene(f, nStep, delta_t):
    """Ricker wavelet of peak frequency f delayed by 1.2/f, integrated in
    time (running sum times delta_t)."""
    e = np.pi * np.pi * f * f
    t = delta_t * np.arange(nStep) - 1.2 / f
    ricker = (1.0 - 2.0 * e * t ** 2) * np.exp(-e * t ** 2)
    return np.cumsum(ricker) * delta_t
