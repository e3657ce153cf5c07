"""ctypes front end of the CPU checkers (test infrastructure only)."""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "_build", "libefwi_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libefwi_ref.so")


def build(quiet: bool = True) -> None:
    """Compile the FP64 port, and the reference kernels where the reference
    tree is present (oracle/Makefile)."""
    out = subprocess.run(["make", "-s", "-f", os.path.join(HERE, "Makefile"), "all"],
                         capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def ref_available() -> bool:
    return os.path.exists(REF_SO)


@dataclass
class Case:
    """One propagation problem on the padded grid (all indices padded)."""
    nz: int
    nx: int
    ny: int
    npml: int
    nt: int
    dz: float
    dx: float
    dy: float
    dt: float
    f0: float
    lam: np.ndarray
    mu: np.ndarray
    rho: np.ndarray
    src: Sequence[Sequence[int]]                 # per shot (z, x, y)
    rec: Sequence[Sequence[np.ndarray]]          # per shot (z_rec, x_rec, y_rec)
    stf: np.ndarray                              # [nshot, nt] untapered
    win: Optional[Sequence[tuple]] = None        # per shot (start, end, weights, src_weight)

    @property
    def nshot(self) -> int:
        return len(self.src)

    def nrec(self, k: int) -> int:
        return len(self.rec[k][0])

    def trace_sizes(self) -> List[int]:
        return [3 * self.nrec(k) * self.nt for k in range(self.nshot)]


def split_traces(case: Case, flat: np.ndarray) -> List[np.ndarray]:
    out, off = [], 0
    for k in range(case.nshot):
        n = 3 * case.nrec(k) * case.nt
        out.append(flat[off:off + n].reshape(3, case.nrec(k), case.nt))
        off += n
    return out


def join_traces(case: Case, traces: Sequence[np.ndarray], dtype) -> np.ndarray:
    return np.ascontiguousarray(np.concatenate([np.asarray(t, dtype).ravel() for t in traces]))


class _Lib:
    real = C.c_double
    npdtype = np.float64

    def __init__(self, path: str, prefix: str):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (run oracle.build())")
        self.lib = C.CDLL(path)
        self.prefix = prefix
        self._keep = []

    def _grid(self, case: Case):
        R = self.real

        class Grid(C.Structure):
            _fields_ = [("nz", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("npml", C.c_int),
                        ("nt", C.c_int), ("dz", R), ("dx", R), ("dy", R), ("dt", R), ("f0", R)]
        return Grid(case.nz, case.nx, case.ny, case.npml, case.nt, case.dz, case.dx, case.dy,
                    case.dt, case.f0)

    def _shots(self, case: Case):
        R = self.real

        class Shot(C.Structure):
            _fields_ = [("z_src", C.c_int), ("x_src", C.c_int), ("y_src", C.c_int),
                        ("nrec", C.c_int), ("z_rec", C.POINTER(C.c_int)),
                        ("x_rec", C.POINTER(C.c_int)), ("y_rec", C.POINTER(C.c_int)),
                        ("win_start", C.POINTER(R)), ("win_end", C.POINTER(R)),
                        ("weights", C.POINTER(R)), ("src_weight", R)]
        arr = (Shot * case.nshot)()
        keep = []
        for k in range(case.nshot):
            zr, xr, yr = [np.ascontiguousarray(a, np.int32) for a in case.rec[k]]
            keep += [zr, xr, yr]
            s = arr[k]
            s.z_src, s.x_src, s.y_src = [int(v) for v in case.src[k]]
            s.nrec = len(zr)
            s.z_rec = zr.ctypes.data_as(C.POINTER(C.c_int))
            s.x_rec = xr.ctypes.data_as(C.POINTER(C.c_int))
            s.y_rec = yr.ctypes.data_as(C.POINTER(C.c_int))
            s.src_weight = 1.0
            if case.win is not None and case.win[k] is not None:
                w0, w1, wt, sw = case.win[k]
                w0 = np.ascontiguousarray(w0, self.npdtype)
                w1 = np.ascontiguousarray(w1, self.npdtype)
                wt = np.ascontiguousarray(wt if wt is not None else np.ones(len(zr)), self.npdtype)
                keep += [w0, w1, wt]
                s.win_start = w0.ctypes.data_as(C.POINTER(R))
                s.win_end = w1.ctypes.data_as(C.POINTER(R))
                s.weights = wt.ctypes.data_as(C.POINTER(R))
                s.src_weight = float(sw)
        self._keep = keep
        return arr

    def _p(self, a):
        return a.ctypes.data_as(C.POINTER(self.real))

    def _model(self, case: Case):
        return [np.ascontiguousarray(a, self.npdtype) for a in (case.lam, case.mu, case.rho)]

    def set_threads(self, n: int) -> None:
        getattr(self.lib, self.prefix + "set_threads")(int(n))

    def num_threads(self) -> int:
        return int(getattr(self.lib, self.prefix + "num_threads")())

    def forward(self, case: Case) -> List[np.ndarray]:
        g, shots = self._grid(case), self._shots(case)
        lam, mu, rho = self._model(case)
        stf = np.ascontiguousarray(case.stf, self.npdtype)
        out = np.zeros(sum(case.trace_sizes()), self.npdtype)
        rc = getattr(self.lib, self.prefix + "forward")(
            C.byref(g), self._p(lam), self._p(mu), self._p(rho), case.nshot, shots, self._p(stf),
            self._p(out))
        assert rc == 0
        return split_traces(case, out)


class _Port(_Lib):
    def __init__(self):
        super().__init__(PORT_SO, "oracle_")

    def gradient(self, case: Case, obs: Sequence[np.ndarray], mode: int = 0,
                 if_win: bool = False):
        g, shots = self._grid(case), self._shots(case)
        lam, mu, rho = self._model(case)
        stf = np.ascontiguousarray(case.stf, np.float64)
        ob = join_traces(case, obs, np.float64)
        n = case.nz * case.nx * case.ny
        gl, gm, gr = (np.zeros(n) for _ in range(3))
        res = np.zeros_like(ob)
        J = C.c_double(0.0)
        rc = self.lib.oracle_gradient(C.byref(g), self._p(lam), self._p(mu), self._p(rho),
                                      case.nshot, shots, self._p(stf), self._p(ob), int(mode),
                                      int(if_win), C.byref(J), self._p(gl), self._p(gm),
                                      self._p(gr), self._p(res))
        assert rc == 0
        shp = (case.nz, case.nx, case.ny)
        return (J.value, gl.reshape(shp), gm.reshape(shp), gr.reshape(shp),
                split_traces(case, res))

    def cpml(self, n: int, npml: int, dh: float, f0: float, dt: float) -> np.ndarray:
        out = np.zeros(6 * n)
        self.lib.oracle_cpml(n, npml, C.c_double(dh), C.c_double(f0), C.c_double(dt),
                             self._p(out))
        return out.reshape(6, n)

    def taper_stf(self, stf: np.ndarray, dt: float) -> np.ndarray:
        s = np.ascontiguousarray(stf, np.float64)
        out = np.zeros_like(s)
        self.lib.oracle_taper_stf(self._p(s), len(s), C.c_double(dt), self._p(out))
        return out

    def illumination(self, case: Case):
        """Diagonal pseudo-Hessian (source illumination) of lambda, mu, rho."""
        g, shots = self._grid(case), self._shots(case)
        lam, mu, rho = self._model(case)
        stf = np.ascontiguousarray(case.stf, np.float64)
        out = [np.zeros(lam.shape, np.float64) for _ in range(3)]
        rc = self.lib.oracle_illumination(C.byref(g), self._p(lam), self._p(mu), self._p(rho),
                                          case.nshot, shots, self._p(stf), *[self._p(o) for o in out])
        assert rc == 0
        return tuple(out)

    def step(self, case: Case, state: np.ndarray, amp: float = 0.0, src=(0, 0, 0)) -> np.ndarray:
        g = self._grid(case)
        lam, mu, rho = self._model(case)
        st = np.ascontiguousarray(state, np.float64).copy()
        self.lib.oracle_step(C.byref(g), self._p(lam), self._p(mu), self._p(rho), int(src[0]),
                             int(src[1]), int(src[2]), C.c_double(amp), self._p(st))
        return st

    def step_T(self, case: Case, astate: np.ndarray) -> np.ndarray:
        g = self._grid(case)
        lam, mu, rho = self._model(case)
        st = np.ascontiguousarray(astate, np.float64).copy()
        self.lib.oracle_step_T(C.byref(g), self._p(lam), self._p(mu), self._p(rho), self._p(st))
        return st


class _Ref(_Lib):
    real = C.c_float
    npdtype = np.float32

    def __init__(self):
        super().__init__(REF_SO, "ref_")

    def gradient(self, case: Case, obs: Sequence[np.ndarray], if_win: bool = False):
        g, shots = self._grid(case), self._shots(case)
        lam, mu, rho = self._model(case)
        stf = np.ascontiguousarray(case.stf, np.float32)
        ob = join_traces(case, obs, np.float32)
        n = case.nz * case.nx * case.ny
        gl, gm, gr = (np.zeros(n, np.float32) for _ in range(3))
        res = np.zeros_like(ob)
        J = C.c_double(0.0)
        rc = self.lib.ref_gradient(C.byref(g), self._p(lam), self._p(mu), self._p(rho),
                                   case.nshot, shots, self._p(stf), self._p(ob), int(if_win),
                                   C.byref(J), self._p(gl), self._p(gm), self._p(gr),
                                   self._p(res))
        assert rc == 0
        shp = (case.nz, case.nx, case.ny)
        return (J.value, gl.reshape(shp), gm.reshape(shp), gr.reshape(shp),
                split_traces(case, res))

    def cpml(self, n: int, npml: int, dh: float, f0: float, dt: float) -> np.ndarray:
        out = np.zeros(6 * n, np.float32)
        self.lib.ref_cpml(n, npml, C.c_float(dh), C.c_float(f0), C.c_float(dt), self._p(out))
        return out.reshape(6, n)

    def taper_stf(self, stf: np.ndarray, dt: float) -> np.ndarray:
        s = np.ascontiguousarray(stf, np.float32)
        out = np.zeros_like(s)
        self.lib.ref_taper_stf(self._p(s), len(s), C.c_float(dt), self._p(out))
        return out


_port = None
_ref = None


def port() -> _Port:
    global _port
    if _port is None:
        _port = _Port()
    return _port


def ref() -> _Ref:
    global _ref
    if _ref is None:
        _ref = _Ref()
    return _ref
