"""The reference-facing API end to end: paraGen_3d / surveyGen_3d files,
FWI_obscalc writing Shot_*.bin, FWI_3d + FWIFunction returning the misfit and
vp gradients through autograd, and fwi_ops.forward.  Checked against the FP64
oracle run on the same inputs."""
import numpy as np
import pytest
import torch

import oracle
from helpers import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _ready():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    oracle.build()


def _setup(tmp_path, nz=14, nx=16, ny=12, npml=5, nt=100):
    import fwi_utils as ft
    exp = tmp_path / "exp"
    para = str(exp / "para_file.json")
    survey = str(exp / "survey_file.json")
    data = str(exp / "Data")
    dt, dx = 1e-3, 10.0
    ft.paraGen_3d(nz + 2 * npml, nx + 2 * npml, ny + 2 * npml, dx, dx, dx, nt, dt, 12.0, npml,
                  para, survey, data)
    src_x = np.array([[3, 3], [10, 10]])
    src_y = np.array([[3, 8], [3, 8]])
    src_z = np.full((2, 2), 2)
    rx = np.arange(1, nx - 1, 3)
    ry = np.arange(1, ny - 1, 3)
    X, Y = np.meshgrid(rx, ry, indexing="ij")
    ft.surveyGen_3d(src_z, src_x, src_y, np.full(X.size, 1), X.ravel(), Y.ravel(), survey)
    stf = torch.tensor(ft.sourceGene(12.0, nt, dt), dtype=torch.float32).repeat(4, 1)
    opt = {"nz": nz, "nx": nx, "ny": ny, "nPml": npml, "para_fname": para}
    rng = np.random.default_rng(0)
    z = np.arange(nz)[:, None, None] * np.ones((1, nx, ny))
    vp_true = np.where(z < nz // 2, 2000.0, 2500.0) + 30 * rng.standard_normal((nz, nx, ny))
    vp_init = np.where(z < nz // 2, 2000.0, 2400.0) + 0 * z
    return opt, stf, vp_true.astype(np.float32), vp_init.astype(np.float32)


def test_obscalc_then_fwi3d_gradient(tmp_path):
    import FWI_ops_3d as F
    from efwi import config
    opt, stf, vp_true, vp_init = _setup(tmp_path)
    nz, nx, ny = opt["nz"], opt["nx"], opt["ny"]
    ids = torch.tensor([0, 1, 2, 3], dtype=torch.int32)
    vs_t = torch.tensor(vp_true / 1.8)
    rho_t = torch.full((nz, nx, ny), 2.3)
    F.FWI_obscalc(torch.tensor(vp_true), vs_t, rho_t, stf, opt)(ids, ngpu=1)
    p = config.read_para(opt["para_fname"])
    shots = config.read_survey(p.survey_fname, p.grid.npml)
    for k in range(4):
        d = config.read_shot_data(p.data_dir_name, k, shots[k].nrec, p.grid.nt)
        assert np.abs(d).max() > 0

    vp = torch.tensor(vp_init, requires_grad=True)
    model = F.FWI_3d(vp, torch.tensor(vp_init / 1.8), torch.full((nz, nx, ny), 2300.0), stf, opt)
    loss = model(ids, ngpu=1)
    loss.backward()
    g_vp = model.Vp.grad.detach().numpy()

    # same chain with the oracle: lambda, mu, rho -> reference gradients
    import fwi_utils as ft
    Vp, Vs, Rho = ft.padding_3d(torch.tensor(vp_init, dtype=torch.float64),
                                torch.tensor(vp_init / 1.8, dtype=torch.float64),
                                torch.full((nz, nx, ny), 2300.0, dtype=torch.float64),
                                nz, nx, ny, opt["nPml"])
    Vp.requires_grad_(True)
    rho = Rho / 1e3
    lam = (Vp ** 2 - 2 * Vs ** 2) * rho
    mu = Vs ** 2 * rho
    g = p.grid
    obs = [config.read_shot_data(p.data_dir_name, k, shots[k].nrec, g.nt).astype(np.float64)
           for k in range(4)]
    case = oracle.Case(g.nz, g.nx, g.ny, g.npml, g.nt, g.dz, g.dx, g.dy,
                       float(np.float32(g.dt)), g.f0, lam.detach().numpy(), mu.detach().numpy(),
                       rho.detach().numpy(), [tuple(s.src) for s in shots],
                       [(s.z_rec, s.x_rec, s.y_rec) for s in shots],
                       stf.numpy().astype(np.float64), None)
    J, gl, gm, gr, _ = oracle.port().gradient(case, obs, mode=0)
    assert abs(loss.item() - J) / J < 1e-4
    (lam * torch.from_numpy(gl) + mu * torch.from_numpy(gm) + rho * torch.from_numpy(gr)).sum().backward()
    # interior only: the reference gradient is zero in the padding
    assert rel_l2(g_vp, Vp.grad.numpy()[5:-5, 5:-5, 5:-5]) < 1e-4

    # calc_id 0 entry point returns the same misfit
    with torch.no_grad():
        Vp_p, Vs_p, Rho_p = ft.padding_3d(torch.tensor(vp_init), torch.tensor(vp_init / 1.8),
                                          torch.full((nz, nx, ny), 2300.0), nz, nx, ny, opt["nPml"])
        r = Rho_p / 1e3
        out = F.fwi_ops.forward((Vp_p ** 2 - 2 * Vs_p ** 2) * r, Vs_p ** 2 * r, r, stf, 0, ids,
                                opt["para_fname"])
    assert abs(out[0].item() - loss.item()) / loss.item() < 1e-6


def test_fwi3d_vs_and_rho_gradients(tmp_path):
    """Full elastic parametrisation end to end: dJ/dvs and dJ/drho through
    FWI_3d's autograd chain against the FP64 oracle's reference gradients
    carried through the same chain (interior cells, rel-L2 1e-4)."""
    import FWI_ops_3d as F
    import fwi_utils as ft
    from efwi import config
    opt, stf, vp_true, vp_init = _setup(tmp_path)
    nz, nx, ny, npml = opt["nz"], opt["nx"], opt["ny"], opt["nPml"]
    ids = torch.tensor([0, 1, 2, 3], dtype=torch.int32)
    F.FWI_obscalc(torch.tensor(vp_true), torch.tensor(vp_true / 1.8),
                  torch.full((nz, nx, ny), 2300.0), stf, opt)(ids, ngpu=1)
    vs0 = vp_init / 1.75
    rho0 = np.full((nz, nx, ny), 2250.0, np.float32)
    vp = torch.tensor(vp_init, requires_grad=True)
    vs = torch.tensor(vs0, requires_grad=True)
    rho = torch.tensor(rho0, requires_grad=True)
    model = F.FWI_3d(vp, vs, rho, stf, opt)
    loss = model(ids, ngpu=1)
    loss.backward()

    p = config.read_para(opt["para_fname"])
    shots = config.read_survey(p.survey_fname, p.grid.npml)
    g = p.grid
    Vp, Vs, Rho = ft.padding_3d(torch.tensor(vp_init, dtype=torch.float64),
                                torch.tensor(vs0, dtype=torch.float64),
                                torch.tensor(rho0, dtype=torch.float64), nz, nx, ny, npml)
    for t in (Vp, Vs, Rho):
        t.requires_grad_(True)
    r = Rho / 1e3
    lam = (Vp ** 2 - 2 * Vs ** 2) * r
    mu = Vs ** 2 * r
    obs = [config.read_shot_data(p.data_dir_name, k, shots[k].nrec, g.nt).astype(np.float64)
           for k in range(4)]
    case = oracle.Case(g.nz, g.nx, g.ny, g.npml, g.nt, g.dz, g.dx, g.dy,
                       float(np.float32(g.dt)), g.f0, lam.detach().numpy(), mu.detach().numpy(),
                       r.detach().numpy(), [tuple(s.src) for s in shots],
                       [(s.z_rec, s.x_rec, s.y_rec) for s in shots],
                       stf.numpy().astype(np.float64), None)
    J, gl, gm, gr, _ = oracle.port().gradient(case, obs, mode=0)
    assert abs(loss.item() - J) / J < 1e-4
    (lam * torch.from_numpy(gl) + mu * torch.from_numpy(gm) + r * torch.from_numpy(gr)).sum().backward()
    s = slice(npml, -npml)
    assert rel_l2(model.Vs.grad.numpy(), Vs.grad.numpy()[s, s, s]) < 1e-4
    assert rel_l2(model.Rho.grad.numpy(), Rho.grad.numpy()[s, s, s]) < 1e-4
    assert rel_l2(model.Vp.grad.numpy(), Vp.grad.numpy()[s, s, s]) < 1e-4


def test_scratch_dumps(tmp_path):
    """scratch_dir_name in the para file: Residual/Syn/CondObs_Shot_{x,y,z}{id}.bin
    (libCUFD.cu:660-700); the residual equals the FP64 oracle's adjoint
    source (3e-4) and residual = window * (CondObs - Syn) at every sample."""
    import json
    import os
    import FWI_ops_3d as F
    import fwi_utils as ft
    from efwi import config
    opt, stf, vp_true, vp_init = _setup(tmp_path)
    nz, nx, ny, npml = opt["nz"], opt["nx"], opt["ny"], opt["nPml"]
    ids = torch.tensor([0, 1, 2, 3], dtype=torch.int32)
    F.FWI_obscalc(torch.tensor(vp_true), torch.tensor(vp_true / 1.8),
                  torch.full((nz, nx, ny), 2300.0), stf, opt)(ids, ngpu=1)
    scratch = str(tmp_path / "scratch")
    with open(opt["para_fname"]) as f:
        d = json.load(f)
    d["scratch_dir_name"] = scratch
    with open(opt["para_fname"], "w") as f:
        json.dump(d, f)
    Vp, Vs, Rho = ft.padding_3d(torch.tensor(vp_init), torch.tensor(vp_init / 1.8),
                                torch.full((nz, nx, ny), 2300.0), nz, nx, ny, npml)
    r = Rho / 1e3
    lam, mu = (Vp ** 2 - 2 * Vs ** 2) * r, Vs ** 2 * r
    F.fwi_ops.backward(lam, mu, r, stf, 1, ids, opt["para_fname"])
    p = config.read_para(opt["para_fname"])
    shots = config.read_survey(p.survey_fname, p.grid.npml)
    g = p.grid
    obs = [config.read_shot_data(p.data_dir_name, k, shots[k].nrec, g.nt).astype(np.float64)
           for k in range(4)]
    case = oracle.Case(g.nz, g.nx, g.ny, g.npml, g.nt, g.dz, g.dx, g.dy,
                       float(np.float32(g.dt)), g.f0, lam.double().numpy(), mu.double().numpy(),
                       r.double().numpy(), [tuple(s.src) for s in shots],
                       [(s.z_rec, s.x_rec, s.y_rec) for s in shots],
                       stf.numpy().astype(np.float64), None)
    _, _, _, _, res = oracle.port().gradient(case, obs, mode=0)
    for k in range(4):
        nr = shots[k].nrec
        got = {}
        for prefix in ("Residual", "Syn", "CondObs"):
            got[prefix] = np.stack([np.fromfile(os.path.join(scratch, f"{prefix}_Shot_{c}{k}.bin"),
                                                np.float32).reshape(nr, g.nt) for c in "xyz"])
        assert rel_l2(got["Residual"], res[k]) < 3e-4
        diff = (got["CondObs"] - got["Syn"]).astype(np.float64)
        diff[..., 0] = 0.0
        # residual = w^2 (CondObs - Syn) with the same w^2 that conditioned obs
        w2 = np.divide(got["CondObs"], obs[k], out=np.zeros_like(obs[k]), where=np.abs(obs[k]) > 1e-20)
        m = np.abs(obs[k]) > 1e-6 * np.abs(obs[k]).max()
        assert np.allclose(got["Residual"][m], (w2 * diff)[m], rtol=1e-3, atol=1e-6 * np.abs(diff).max())
