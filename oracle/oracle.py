"""ORACLE — test infrastructure only (tests/, __graft_entry__.smoke(), and the
CPU-baseline leg of bench.py). The product library never imports this module.

ctypes bindings for the CPU oracle libraries built by ``oracle/Makefile``:

* ``Oracle(precision="f32")`` — the restated algorithm (``lbm_oracle.c``) in
  float, IEEE op-for-op with FlowCraft's ``LbmReference`` (LbmReference.cpp:241-469);
* ``Oracle(precision="f64")`` — the same restatement in double, the FP64 error
  reference;
* ``Oracle(precision="ref")`` / ``"ref_fast"`` — FlowCraft's own
  ``LbmReference.cpp`` compiled from its sources (``oracle/_ref/``), when
  present.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {
    "f32": (os.path.join(HERE, "liblbm_oracle32.so"), "oracle32_"),
    "f64": (os.path.join(HERE, "liblbm_oracle64.so"), "oracle64_"),
    "ref": (os.path.join(HERE, "_ref", "libfcref.so"), "ref_"),
    "ref_fast": (os.path.join(HERE, "_ref", "libfcref_fast.so"), "ref_"),
}


class OracleParams(ctypes.Structure):
    _fields_ = [
        ("tau", ctypes.c_float),
        ("inlet_velocity", ctypes.c_float),
        ("reverse_flow", ctypes.c_int32),
        ("free_slip_y", ctypes.c_int32),
        ("free_slip_z", ctypes.c_int32),
        ("smagorinsky_cs", ctypes.c_float),
    ]


class OracleStats(ctypes.Structure):
    _fields_ = [
        ("avg_density", ctypes.c_double),
        ("min_density", ctypes.c_double),
        ("max_density", ctypes.c_double),
        ("avg_speed", ctypes.c_double),
        ("max_speed", ctypes.c_double),
        ("force_x", ctypes.c_double),
        ("force_y", ctypes.c_double),
        ("force_z", ctypes.c_double),
        ("max_stress", ctypes.c_double),
        ("total_mass", ctypes.c_double),
        ("has_nan", ctypes.c_int32),
        ("fluid_count_lo", ctypes.c_int32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


def reference_tree() -> str:
    """The FlowCraft source tree oracle/_ref is compiled from: $FLOWCRAFT_REF,
    else the directory `reference` beside this repository's root."""
    env = os.environ.get("FLOWCRAFT_REF")
    return os.path.abspath(env) if env else os.path.abspath(os.path.join(HERE, "..", "..", "reference"))


def build(force: bool = False) -> None:
    """Compile the oracle libraries (and oracle/_ref when the reference tree exists)."""
    need = force or not all(os.path.exists(_LIBS[k][0]) for k in ("f32", "f64"))
    ref = reference_tree()
    if need or (os.path.isdir(ref) and not os.path.exists(_LIBS["ref"][0])):
        subprocess.run(["make", "-s", "-C", HERE, f"REF={ref}"], check=True)


def available(precision: str) -> bool:
    return os.path.exists(_LIBS[precision][0])


_loaded: dict = {}


def _lib(precision: str):
    if precision in _loaded:
        return _loaded[precision]
    path, prefix = _LIBS[precision]
    if not os.path.exists(path):
        if precision in ("f32", "f64"):
            build()
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle library missing: {path}")
    lib = ctypes.CDLL(path)
    vp, c_int, c_size = ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t
    fptr = ctypes.POINTER(ctypes.c_float)

    def fn(name, res, *args):
        f = getattr(lib, prefix + name)
        f.restype = res
        f.argtypes = list(args)
        return f

    is_ref = prefix == "ref_"
    create_args = [c_int, c_int, c_int, c_int, ctypes.POINTER(ctypes.c_uint8), fptr, c_size,
                   ctypes.POINTER(OracleParams), c_int]
    if not is_ref:
        create_args.append(c_int)
    api = {
        "create": fn("create", vp, *create_args),
        "destroy": fn("destroy", None, vp),
        "reset": fn("reset", None, vp, c_int),
        "reset_from_field": fn("reset_from_field", c_int, vp, fptr, c_size),
        "set_params": fn("set_params", None, vp, ctypes.POINTER(OracleParams)),
        "step": fn("step", None, vp, c_int),
        "has_diverged": fn("has_diverged", c_int, vp),
        "readback_field": fn("readback_field", None, vp, fptr),
        "stats": fn("stats", None, vp, ctypes.POINTER(OracleStats)),
        "is_ref": is_ref,
    }
    if not is_ref:
        u8p = ctypes.POINTER(ctypes.c_uint8)
        api["set_closure"] = fn("set_closure", c_int, vp, fptr, fptr, fptr, fptr, fptr, ctypes.c_float, ctypes.c_float,
                                fptr, fptr, fptr, fptr, ctypes.c_float, u8p, ctypes.c_float, ctypes.c_float)
        api["closure_eval"] = fn("closure_eval", None, vp, fptr, c_size, fptr)
        api["wall_distance"] = fn("wall_distance", None, c_int, c_int, c_int, u8p, u8p)
        api["readback_field_f64"] = fn("readback_field_f64", None, vp, ctypes.POINTER(ctypes.c_double))
        api["get_populations"] = fn("get_populations", None, vp, fptr, ctypes.POINTER(ctypes.c_double))
    _loaded[precision] = api
    return api


@dataclass
class Params:
    """Mirror of LbmReference::Params (LbmReference.h:41-52), same defaults."""
    tau: float = 0.8
    inlet_velocity: float = 0.05
    reverse_flow: bool = False
    free_slip_y: bool = True
    free_slip_z: bool = True
    smagorinsky_cs: float = 0.12

    def c(self) -> OracleParams:
        return OracleParams(self.tau, self.inlet_velocity, int(self.reverse_flow), int(self.free_slip_y),
                            int(self.free_slip_z), self.smagorinsky_cs)


class Oracle:
    """One CPU lattice (restated oracle or the reference build)."""

    def __init__(self, solid: np.ndarray, sdf: np.ndarray | None, q: int, params: Params,
                 seed_mid: bool = False, precision: str = "f32", threads: int = 0):
        self.api = _lib(precision)
        self.precision = precision
        solid = np.ascontiguousarray(solid, dtype=np.uint8)
        nz, ny, nx = solid.shape
        self.shape = (nz, ny, nx)
        self.q = q
        self.n = nx * ny * nz
        self._solid = solid
        sdf_ptr, sdf_n = None, 0
        if sdf is not None:
            self._sdf = np.ascontiguousarray(sdf, dtype=np.float32)
            sdf_ptr = self._sdf.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
            sdf_n = self._sdf.size
        p = params.c()
        args = [nx, ny, nz, q, solid.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), sdf_ptr, sdf_n,
                ctypes.byref(p), int(seed_mid)]
        if not self.api["is_ref"]:
            args.append(threads)
        self.h = self.api["create"](*args)
        if not self.h:
            raise RuntimeError("oracle create failed")

    def close(self):
        if self.h:
            self.api["destroy"](self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reset(self, seed_mid: bool = False):
        self.api["reset"](self.h, int(seed_mid))

    def reset_from_field(self, field: np.ndarray) -> int:
        field = np.ascontiguousarray(field, dtype=np.float32).ravel()
        return self.api["reset_from_field"](self.h, field.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), field.size)

    def set_params(self, params: Params):
        p = params.c()
        self.api["set_params"](self.h, ctypes.byref(p))

    def step(self, n: int = 1):
        self.api["step"](self.h, n)

    def has_diverged(self) -> bool:
        return bool(self.api["has_diverged"](self.h))

    def set_closure(self, cw, wall=None):
        """Installs a learned closure (an object with the fields of
        flowcraft_b200.closure.ClosureWeights), or None for Smagorinsky."""
        fp = ctypes.POINTER(ctypes.c_float)
        if cw is None:
            self.api["set_closure"](self.h, None, None, None, None, None, 0.0, 0.0, None, None, None, None, 0.0, None,
                                    0.0, 0.0)
            return
        self._closure_keep = [np.ascontiguousarray(a, dtype=np.float32) for a in
                              (cw.w1, cw.b1, cw.w2, cw.b2, cw.w3, cw.mean, cw.std, cw.lo, cw.hi)]
        k = [a.ctypes.data_as(fp) for a in self._closure_keep]
        wl = None
        if wall is not None:
            self._wall = np.ascontiguousarray(wall, dtype=np.uint8).ravel()
            wl = self._wall.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
        self.api["set_closure"](self.h, k[0], k[1], k[2], k[3], k[4], float(cw.b3), float(cw.out_scale), k[5], k[6],
                                k[7], k[8], float(cw.filter_width), wl, float(getattr(cw, "wall_min", 0.0)),
                                float(getattr(cw, "trust", 0.0)))

    def closure_eval(self, inputs) -> np.ndarray:
        """nu_t (-1 outside the training range) for rows of inputs 0-3."""
        x = np.ascontiguousarray(inputs, dtype=np.float32).reshape(-1, 4)
        out = np.empty(len(x), dtype=np.float32)
        fp = ctypes.POINTER(ctypes.c_float)
        self.api["closure_eval"](self.h, x.ctypes.data_as(fp), len(x), out.ctypes.data_as(fp))
        return out

    def readback_field(self) -> np.ndarray:
        out = np.empty(self.n * 4, dtype=np.float32)
        self.api["readback_field"](self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
        return out

    def readback_field_f64(self) -> np.ndarray:
        out = np.empty(self.n * 4, dtype=np.float64)
        self.api["readback_field_f64"](self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return out

    def populations(self) -> np.ndarray:
        out = np.empty(self.q * self.n, dtype=np.float32)
        self.api["get_populations"](self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), None)
        return out.reshape(self.q, self.n)

    def stats(self) -> dict:
        s = OracleStats()
        self.api["stats"](self.h, ctypes.byref(s))
        return s.as_dict()


def wall_distance(solid) -> np.ndarray:
    """The closure's wall-distance input (3x3x3 chamfer, 1/16 cells, cap 255)."""
    solid = np.ascontiguousarray(solid, dtype=np.uint8)
    nz, ny, nx = solid.shape
    out = np.empty_like(solid)
    u8p = ctypes.POINTER(ctypes.c_uint8)
    _lib("f32")["wall_distance"](nx, ny, nz, solid.ctypes.data_as(u8p), out.ctypes.data_as(u8p))
    return out


# ---- voxelizer oracle (voxel_oracle.c) and the reference's Voxelizer ----
def _vox_lib(kind: str):
    key = "vox_" + kind
    if key in _loaded:
        return _loaded[key]
    if kind == "oracle":
        path = os.path.join(HERE, "libvoxel_oracle.so")
        if not os.path.exists(path):
            build()
        lib = ctypes.CDLL(path)
        lib.voxo_grid_for_mesh.restype = ctypes.c_int
        lib.voxo_grid_for_mesh.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_float,
                                           ctypes.c_float, ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_void_p]
        lib.voxo_voxelize.restype = ctypes.c_int
        lib.voxo_voxelize.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t,
                                      ctypes.c_void_p, ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_void_p]
    else:
        lib = ctypes.CDLL(_LIBS["ref"][0])
        lib.ref_voxelize.restype = ctypes.c_void_p
        lib.ref_voxelize.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_size_t,
                                     ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_float]
        lib.ref_voxels_info.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        lib.ref_voxels_copy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        lib.ref_voxels_free.argtypes = [ctypes.c_void_p]
    _loaded[key] = lib
    return lib


def grid_for_mesh(positions, target_resolution=640, padding=(0.3, 1.0, 0.5)):
    """Voxelizer::Voxelize's grid for a mesh: ((nx, ny, nz), cell_size, origin)."""
    lib = _vox_lib("oracle")
    pos = np.ascontiguousarray(positions, dtype=np.float32)
    dims = np.zeros(3, dtype=np.int32)
    cell = np.zeros(1, dtype=np.float32)
    origin = np.zeros(3, dtype=np.float32)
    rc = lib.voxo_grid_for_mesh(pos.ctypes.data, len(pos), int(target_resolution), *[float(p) for p in padding],
                                dims.ctypes.data, cell.ctypes.data, origin.ctypes.data)
    if rc != 0:
        raise ValueError("empty mesh")
    return tuple(int(d) for d in dims), float(cell[0]), origin


def voxelize(positions, indices, dims, cell_size, origin, impl: str = "oracle"):
    """(solid u8 (nz,ny,nx), sdf f32 (nz,ny,nx)) on the given grid."""
    pos = np.ascontiguousarray(positions, dtype=np.float32)
    idx = np.ascontiguousarray(indices, dtype=np.uint32)
    nx, ny, nz = dims
    solid = np.empty(nx * ny * nz, dtype=np.uint8)
    sdf = np.empty(nx * ny * nz, dtype=np.float32)
    d = np.asarray(dims, dtype=np.int32)
    o = np.ascontiguousarray(origin, dtype=np.float32)
    lib = _vox_lib("oracle")
    rc = lib.voxo_voxelize(pos.ctypes.data, len(pos), idx.ctypes.data, idx.size, d.ctypes.data, float(cell_size),
                           o.ctypes.data, solid.ctypes.data, sdf.ctypes.data)
    if rc != 0:
        raise MemoryError("voxelizer oracle failed")
    return solid.reshape(nz, ny, nx), sdf.reshape(nz, ny, nx)


def voxelize_reference(positions, indices, target_resolution=640, padding=(0.3, 1.0, 0.5)):
    """FlowCraft's own Voxelizer::Voxelize (oracle/_ref): (dims, cell, origin, solid, sdf)."""
    lib = _vox_lib("ref")
    pos = np.ascontiguousarray(positions, dtype=np.float32)
    idx = np.ascontiguousarray(indices, dtype=np.uint32)
    h = lib.ref_voxelize(pos.ctypes.data, len(pos), idx.ctypes.data, idx.size, int(target_resolution),
                         *[float(p) for p in padding])
    dims = np.zeros(3, dtype=np.int32)
    cell = np.zeros(1, dtype=np.float32)
    origin = np.zeros(3, dtype=np.float32)
    lib.ref_voxels_info(h, dims.ctypes.data, cell.ctypes.data, origin.ctypes.data)
    nx, ny, nz = (int(v) for v in dims)
    solid = np.empty(nx * ny * nz, dtype=np.uint8)
    sdf = np.empty(nx * ny * nz, dtype=np.float32)
    lib.ref_voxels_copy(h, solid.ctypes.data, sdf.ctypes.data)
    lib.ref_voxels_free(h)
    return (nx, ny, nz), float(cell[0]), origin, solid.reshape(nz, ny, nx), sdf.reshape(nz, ny, nx)


# ---- aerodynamic forces (FieldOverlay::ComputeAerodynamicForces) ----
def aero_forces(solid, field, cell_size=1.0, origin=(0.0, 0.0, 0.0)) -> dict:
    """Restatement of FieldOverlay::ComputeAerodynamicForces
    (FlowCraft/FieldOverlay.cpp:469-621) over a 4-float-per-cell field:
    FP64 sums of the solid cells' momentum-exchange force, the lift-weighted
    (|Fz|) centre of pressure with the force-weighted and geometric
    fallbacks, the stress range over loaded skin cells and the lift arrow's
    base above the top skin. The sums are float64 like the reference's; their
    order differs (numpy pairwise), so results agree to rounding."""
    solid = np.asarray(solid, dtype=np.uint8)
    nz, ny, nx = solid.shape
    f = np.asarray(field, dtype=np.float32).reshape(nz, ny, nx, 4)
    zz, yy, xx = np.nonzero(solid)
    cs = np.float32(cell_size)
    org = np.asarray(origin, dtype=np.float32)
    # VoxelGrid::CellCenter in float: world x from grid y, world y from grid x
    px = (org[0] + (yy.astype(np.float32) + np.float32(0.5)) * cs).astype(np.float64)
    py = (org[1] + (xx.astype(np.float32) + np.float32(0.5)) * cs).astype(np.float64)
    pz = (org[2] + (zz.astype(np.float32) + np.float32(0.5)) * cs).astype(np.float64)
    v = f[zz, yy, xx]
    finite = np.isfinite(v).all(axis=1)
    out = {"has_nan": bool((~finite).any())}
    v64 = v[finite].astype(np.float64)
    fx, fy, fz = v64[:, 1], v64[:, 2], v64[:, 3]
    pxf, pyf, pzf = px[finite], py[finite], pz[finite]
    out["force_sum"] = (fx.sum(), fy.sum(), fz.sum())
    out["force"] = tuple(float(np.float32(s)) for s in out["force_sum"])
    wl = np.abs(fz)
    wf = np.sqrt(fx * fx + fy * fy + fz * fz)
    stress = v[finite][:, 0]
    loaded = stress[stress > 0]
    hi = float(loaded.max()) if loaded.size else None
    out["min_stress"] = 0.0
    out["max_stress"] = float(np.float32(1e-6)) if hi is None else (hi if hi > 0.0 else float(np.float32(1e-6)))
    if wl.sum() > 1e-9:
        s = wl.sum()
        cp = ((wl * pxf).sum() / s, (wl * pyf).sum() / s, (wl * pzf).sum() / s)
    elif wf.sum() > 1e-9:
        s = wf.sum()
        cp = ((wf * pxf).sum() / s, (wf * pyf).sum() / s, (wf * pzf).sum() / s)
    elif zz.size:
        cp = (px.mean(), py.mean(), pz.mean())
    else:
        cp = (0.0, 0.0, 0.0)
    cp = np.asarray(cp, dtype=np.float64).astype(np.float32)
    out["center_of_pressure"] = tuple(float(c) for c in cp)
    out["lift_weight_sum"] = float(wl.sum())
    out["force_weight_sum"] = float(wf.sum())
    out["solid_cells"] = int(zz.size)
    gx = int(np.clip(np.floor((cp[1] - org[1]) / cs), 0, max(nx - 1, 0)))
    gy = int(np.clip(np.floor((cp[0] - org[0]) / cs), 0, max(ny - 1, 0)))
    top = -1
    for dy in range(-2, 3):
        y = int(np.clip(gy + dy, 0, max(ny - 1, 0)))
        for dx in range(-2, 3):
            x = int(np.clip(gx + dx, 0, max(nx - 1, 0)))
            col = np.nonzero(solid[:, y, x])[0]
            if col.size:
                top = max(top, int(col.max()))
    eff = top if top >= 0 else max(int(zz.max()) if zz.size else -1, 0)
    out["lift_arrow_base"] = (out["center_of_pressure"][0], out["center_of_pressure"][1],
                              float(org[2] + (np.float32(eff) + np.float32(1.0)) * cs))
    return out


class _RefAero(ctypes.Structure):
    _fields_ = [("force", ctypes.c_float * 3), ("min_stress", ctypes.c_float), ("max_stress", ctypes.c_float),
                ("center_of_pressure", ctypes.c_float * 3), ("lift_arrow_base", ctypes.c_float * 3),
                ("has_nan", ctypes.c_int32)]


def aero_forces_reference(solid, field, cell_size=1.0, origin=(0.0, 0.0, 0.0)) -> dict:
    """FlowCraft's own FieldOverlay::ComputeAerodynamicForces (oracle/_ref)."""
    lib = _vox_lib("ref")
    if not hasattr(lib, "_aero_bound"):
        lib.ref_aero_forces.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(_RefAero)]
        lib._aero_bound = True
    solid = np.ascontiguousarray(solid, dtype=np.uint8)
    nz, ny, nx = solid.shape
    field = np.ascontiguousarray(field, dtype=np.float32)
    org = np.ascontiguousarray(origin, dtype=np.float32)
    r = _RefAero()
    lib.ref_aero_forces(nx, ny, nz, float(cell_size), org.ctypes.data, solid.ctypes.data, field.ctypes.data,
                        ctypes.byref(r))
    return {"force": tuple(r.force), "min_stress": r.min_stress, "max_stress": r.max_stress,
            "center_of_pressure": tuple(r.center_of_pressure), "lift_arrow_base": tuple(r.lift_arrow_base),
            "has_nan": bool(r.has_nan)}
