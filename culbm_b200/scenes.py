"""Init-state scenes in the reference's ``flag.dat``/``rho.dat``/``vx.dat``...
format, and the seeded synthetic workloads this solver is measured on.

Format (reference ``Simulator::Data::initFlag``/``initRhoU``,
src/simulator/single_dev_expt/simulator_expt_platform.cu:95-228): raw
little-endian arrays of nx*ny*nz values, x fastest (numpy shape (nz, ny, nx));
``flag.dat`` is uint32, the others float32.  ``flag.dat`` is mandatory,
missing ``rho``/``vx``/``vy``/``vz`` default to 1/0/0/0.

Scene builders:

* :func:`reference_channel`, :func:`reference_channel_cube` — the two helpers
  of the reference's scripts/state_initialization.ipynb (channel with
  bounce-back side walls, equilibrium inlet/outlet, optional cube obstacle);
* :func:`correctness_case` — the scene of analysis/correctness/generate.py
  (any size);
* :func:`sphere_channel` — channel with seeded spheres (the benchmark
  workloads: 64^3 with one sphere, 288x272x280 with 40 spheres, 512x512x256
  with 120 spheres and its 128x128x64 scaled copy);
* :func:`soft_obstacle_field` — clipped sum of seeded Gaussian bumps, the
  per-cell partial-bounce-back field of the adjoint workloads.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field
from typing import Optional, Tuple

import numpy as np

LOAD, EQU, COLLIDE, BOUNCE_BACK, STORE = 1 << 0, 1 << 1, 1 << 2, 1 << 3, 1 << 4
DUMP_RHO, DUMP_VX, DUMP_VY, DUMP_VZ = 1 << 27, 1 << 28, 1 << 29, 1 << 30
DUMP_ALL = DUMP_RHO | DUMP_VX | DUMP_VY | DUMP_VZ

FLUID = LOAD | COLLIDE | STORE | DUMP_ALL
WALL = LOAD | BOUNCE_BACK | STORE
EQUILIBRIUM = EQU | STORE


@dataclass
class Scene:
    """One init state; arrays have numpy shape (nz, ny, nx)."""

    flag: np.ndarray
    rho: np.ndarray
    vx: np.ndarray
    vy: np.ndarray
    vz: np.ndarray
    meta: dict = field(default_factory=dict)

    @property
    def shape(self) -> Tuple[int, int, int]:
        nz, ny, nx = self.flag.shape
        return nx, ny, nz

    @property
    def n(self) -> int:
        return int(self.flag.size)

    def solid_fraction(self) -> float:
        """Fraction of cells that are bounce-back (walls and obstacles)."""
        return float(np.count_nonzero(self.flag & BOUNCE_BACK)) / self.n

    def arrays(self):
        """(flag, rho, vx, vy, vz) flattened, x fastest."""
        return tuple(np.ascontiguousarray(a).reshape(-1) for a in (self.flag, self.rho, self.vx, self.vy, self.vz))


def _empty(nx, ny, nz) -> Scene:
    shape = (nz, ny, nx)
    return Scene(np.zeros(shape, np.uint32), np.ones(shape, np.float32), np.zeros(shape, np.float32),
                 np.zeros(shape, np.float32), np.zeros(shape, np.float32))


def default_scene(nx, ny, nz) -> Scene:
    """The state the reference uses without --initStateFolder: fluid everywhere, rho=1, u=0."""
    s = _empty(nx, ny, nz)
    s.flag[:] = FLUID
    return s


def reference_channel(nx=32, ny=32, nz=32, left_vel=0.05) -> Scene:
    """leftInletRightOutlet of scripts/state_initialization.ipynb: fluid interior,
    bounce-back y/z faces, equilibrium inlet (vx=left_vel) at x=0 and outlet at x=nx-1."""
    s = _empty(nx, ny, nz)
    f = s.flag
    f[1:-1, 1:-1, 1:-1] = FLUID
    f[:, 0, :] = WALL
    f[:, -1, :] = WALL
    f[0, 1:-1, :] = WALL
    f[-1, 1:-1, :] = WALL
    f[1:-1, 1:-1, 0] = EQUILIBRIUM
    f[1:-1, 1:-1, -1] = EQUILIBRIUM
    s.vx[1:-1, 1:-1, 0] = left_vel
    s.meta = {"kind": "reference_channel", "left_vel": left_vel}
    return s


def reference_channel_cube(nx=288, ny=272, nz=280, left_vel=0.05, cube=None) -> Scene:
    """leftInletRightOutletCubeObs of scripts/state_initialization.ipynb; the default
    cube spans the middle third of each axis as in the notebook's last cell."""
    s = reference_channel(nx, ny, nz, left_vel)
    if cube is None:
        cube = (nx // 2 - nx // 6, ny // 2 - ny // 6, nz // 2 - nz // 6,
                nx // 2 + nx // 6, ny // 2 + ny // 6, nz // 2 + nz // 6)
    x0, y0, z0, x1, y1, z1 = cube
    s.flag[z0:z1, y0:y1, x0:x1] = WALL
    s.meta = {"kind": "reference_channel_cube", "left_vel": left_vel, "cube": list(cube)}
    return s


def correctness_case(nx=768, ny=384, nz=384, left_vel=0.05, cube=None) -> Scene:
    """The scene of analysis/correctness/generate.py at any size (default: its own
    768x384x384 with the cube [128:256]^3)."""
    s = _empty(nx, ny, nz)
    f = s.flag
    f[:] = FLUID
    f[:, :, (0, -1)] = EQUILIBRIUM
    if cube is None:
        cube = (128, 128, 128, 256, 256, 256)
    x0, y0, z0, x1, y1, z1 = cube
    f[z0:z1, y0:y1, x0:x1] = WALL
    f[:, (0, -1), :] = WALL
    f[(0, -1), :, :] = WALL
    s.vx[:, :, 0] = left_vel
    s.vx[:, (0, -1), :] = 0.0
    s.vx[(0, -1), :, :] = 0.0
    s.meta = {"kind": "correctness_case", "left_vel": left_vel, "cube": list(cube)}
    return s


def _channel(nx, ny, nz, u_in, profile="uniform") -> Scene:
    """Fluid channel: equilibrium inlet at x=0 (vx=u_in, or a parabolic profile
    of peak u_in), equilibrium outlet rho=1, u=0 at x=nx-1, bounce-back y/z
    faces including their edges (the order of analysis/correctness/generate.py)."""
    s = _empty(nx, ny, nz)
    f = s.flag
    f[:] = FLUID
    f[:, :, (0, -1)] = EQUILIBRIUM
    f[:, (0, -1), :] = WALL
    f[(0, -1), :, :] = WALL
    if profile == "uniform":
        s.vx[:, :, 0] = u_in
    elif profile == "parabolic":
        y = (np.arange(ny) - 0.5) / (ny - 2)   # walls at y=0 and y=ny-1, fluid centred between
        z = (np.arange(nz) - 0.5) / (nz - 2)
        py = np.clip(4.0 * y * (1.0 - y), 0.0, None)
        pz = np.clip(4.0 * z * (1.0 - z), 0.0, None)
        s.vx[:, :, 0] = (u_in * pz[:, None] * py[None, :]).astype(np.float32)
    else:
        raise ValueError(profile)
    s.vx[:, (0, -1), :] = 0.0
    s.vx[(0, -1), :, :] = 0.0
    return s


def sphere_channel(nx, ny, nz, u_in, centers, radii) -> Scene:
    """Channel with solid spheres: a cell is solid when |p - c|^2 < r^2."""
    s = _channel(nx, ny, nz, u_in)
    z, y, x = np.ogrid[0:nz, 0:ny, 0:nx]
    for (cx, cy, cz), r in zip(centers, radii):
        m = (x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2 < r * r
        s.flag[m] = WALL
    s.vx[s.flag == WALL] = 0.0
    s.meta = {"kind": "sphere_channel", "u_in": u_in, "spheres": len(radii)}
    return s


def random_spheres(nx, ny, nz, count, rmin, rmax, seed, margin=0.1):
    """Seeded sphere set: centres uniform in the interior box that leaves
    `margin` of each axis free at both ends, radii uniform in [rmin, rmax]."""
    rng = np.random.default_rng(seed)
    lo = np.array([margin * nx, margin * ny, margin * nz])
    hi = np.array([(1 - margin) * nx, (1 - margin) * ny, (1 - margin) * nz])
    centers = rng.uniform(lo, hi, size=(count, 3))
    radii = rng.uniform(rmin, rmax, size=count)
    return centers, radii


def sphere_64() -> Scene:
    """64^3, inlet vx=0.02, outlet rho=1, walls on y/z faces, one sphere r=8 at (16,32,32)."""
    s = sphere_channel(64, 64, 64, 0.02, [(16, 32, 32)], [8])
    s.meta["config"] = "64^3 sphere r=8"
    return s


def spheres_288(seed=12345) -> Scene:
    """288x272x280 channel, inlet vx=0.05, 40 seeded spheres with radii in [4,12]."""
    c, r = random_spheres(288, 272, 280, 40, 4.0, 12.0, seed)
    s = sphere_channel(288, 272, 280, 0.05, c, r)
    s.meta.update({"config": "288x272x280, 40 spheres r in [4,12]", "seed": seed})
    return s


def spheres_512(seed=2024, scale=1.0) -> Scene:
    """512x512x256 channel with 120 seeded spheres, radii in [6,18]; `scale`
    shrinks the domain and the spheres together (0.25 gives the 128x128x64 copy)."""
    nx, ny, nz = int(512 * scale), int(512 * scale), int(256 * scale)
    c, r = random_spheres(512, 512, 256, 120, 6.0, 18.0, seed)
    s = sphere_channel(nx, ny, nz, 0.05, c * scale, r * scale)
    s.meta.update({"config": f"{nx}x{ny}x{nz}, 120 spheres r in [{6 * scale},{18 * scale}]", "seed": seed,
                   "scale": scale})
    return s


def soft_obstacle_field(nx, ny, nz, bumps=16, sigma=(3.0, 8.0), seed=7, margin=0.15) -> np.ndarray:
    """s(p) = clip(sum_k exp(-|p - c_k|^2 / (2 sigma_k^2)), 0, 1), centres uniform
    in the interior, sigma_k uniform in `sigma`; float32, shape (nz, ny, nx)."""
    rng = np.random.default_rng(seed)
    lo = np.array([margin * nx, margin * ny, margin * nz])
    hi = np.array([(1 - margin) * nx, (1 - margin) * ny, (1 - margin) * nz])
    centers = rng.uniform(lo, hi, size=(bumps, 3))
    sig = rng.uniform(sigma[0], sigma[1], size=bumps)
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    acc = np.zeros((nz, ny, nx), np.float64)
    for (cx, cy, cz), sk in zip(centers, sig):
        acc += np.exp(-((x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2) / (2.0 * sk * sk))
    return np.clip(acc, 0.0, 1.0).astype(np.float32)


def adjoint_channel(nx=128, ny=64, nz=64, u_peak=0.04, bumps=16, seed=7) -> Tuple[Scene, np.ndarray]:
    """Channel with a parabolic inlet of peak u_peak and a soft-obstacle field."""
    s = _channel(nx, ny, nz, u_peak, profile="parabolic")
    soft = soft_obstacle_field(nx, ny, nz, bumps=bumps, seed=seed)
    soft[s.flag != FLUID] = 0.0
    s.meta = {"kind": "adjoint_channel", "u_peak": u_peak, "bumps": bumps, "seed": seed}
    return s, soft


# ------------------------------------------------------------------ files ---

def write_folder(scene: Scene, folder: str, fields=("flag", "rho", "vx", "vy", "vz")) -> None:
    os.makedirs(folder, exist_ok=True)
    for name in fields:
        arr = getattr(scene, name)
        dt = "<u4" if name == "flag" else "<f4"
        np.ascontiguousarray(arr, dtype=dt).tofile(os.path.join(folder, f"{name}.dat"))


def read_folder(folder: str, nx: int, ny: int, nz: int) -> Scene:
    shape = (nz, ny, nx)
    flag = np.fromfile(os.path.join(folder, "flag.dat"), dtype="<u4").reshape(shape)
    s = _empty(nx, ny, nz)
    s.flag = flag.astype(np.uint32)
    for name, dflt in (("rho", 1.0), ("vx", 0.0), ("vy", 0.0), ("vz", 0.0)):
        p = os.path.join(folder, f"{name}.dat")
        if os.path.exists(p):
            setattr(s, name, np.fromfile(p, dtype="<f4").reshape(shape).astype(np.float32))
    return s


def read_dump(folder: str, field_name: str, step: int, nx: int, ny: int, nz: int) -> np.ndarray:
    """A dump file <folder>/<field>_<step>.dat as shape (nz, ny, nx)."""
    return np.fromfile(os.path.join(folder, f"{field_name}_{step}.dat"), dtype="<f4").reshape((nz, ny, nx))


# -------------------------------------------------------------------- CLI ---

_KINDS = ("default", "channel", "channel-cube", "correctness", "spheres", "sphere64", "spheres288", "spheres512",
          "adjoint-channel")


def build_scene(kind: str, domain=None, u_in=0.05, spheres=40, radii=(4.0, 12.0), seed=12345, bumps=16,
                scale=1.0) -> Tuple[Scene, Optional[np.ndarray]]:
    """A scene by name (see :data:`_KINDS`), and the soft-obstacle field for
    ``adjoint-channel`` (None otherwise)."""
    soft = None
    if kind == "sphere64":
        return sphere_64(), None
    if kind == "spheres288":
        return spheres_288(seed), None
    if kind == "spheres512":
        return spheres_512(seed, scale), None
    if domain is None:
        raise ValueError(f"--domain is required for {kind}")
    nx, ny, nz = (int(v) for v in domain)
    if kind == "default":
        s = default_scene(nx, ny, nz)
    elif kind == "channel":
        s = reference_channel(nx, ny, nz, u_in)
    elif kind == "channel-cube":
        s = reference_channel_cube(nx, ny, nz, u_in)
    elif kind == "correctness":
        s = correctness_case(nx, ny, nz, u_in, cube=(nx // 6, ny // 3, nz // 3, nx // 3, 2 * ny // 3, 2 * nz // 3))
    elif kind == "spheres":
        c, r = random_spheres(nx, ny, nz, spheres, radii[0], radii[1], seed)
        s = sphere_channel(nx, ny, nz, u_in, c, r)
    elif kind == "adjoint-channel":
        s, soft = adjoint_channel(nx, ny, nz, u_peak=u_in, bumps=bumps, seed=seed)
    else:
        raise ValueError(f"unknown scene kind {kind!r}; one of {', '.join(_KINDS)}")
    return s, soft


def main(argv=None) -> int:
    """Writes an init-state folder (flag.dat, rho.dat, vx.dat, vy.dat, vz.dat;
    soft.dat for adjoint-channel) for single_dev_expt_main --initStateFolder."""
    import argparse
    import json
    ap = argparse.ArgumentParser(prog="python -m culbm_b200.scenes", description=main.__doc__)
    ap.add_argument("kind", choices=_KINDS)
    ap.add_argument("out", help="output folder")
    ap.add_argument("--domain", type=int, nargs=3, metavar=("NX", "NY", "NZ"))
    ap.add_argument("--u-in", type=float, default=0.05, help="inlet velocity (peak for adjoint-channel)")
    ap.add_argument("--spheres", type=int, default=40)
    ap.add_argument("--radii", type=float, nargs=2, default=(4.0, 12.0))
    ap.add_argument("--seed", type=int, default=12345)
    ap.add_argument("--bumps", type=int, default=16)
    ap.add_argument("--scale", type=float, default=1.0, help="spheres512 only")
    args = ap.parse_args(argv)
    s, soft = build_scene(args.kind, args.domain, args.u_in, args.spheres, tuple(args.radii), args.seed, args.bumps,
                          args.scale)
    write_folder(s, args.out)
    if soft is not None:
        np.ascontiguousarray(soft, dtype="<f4").tofile(os.path.join(args.out, "soft.dat"))
    nz, ny, nx = s.flag.shape
    print(json.dumps({"folder": args.out, "domainDim": [nx, ny, nz], "cells": int(s.flag.size),
                      "solid_fraction": round(s.solid_fraction(), 5), **{k: v for k, v in s.meta.items()
                                                                          if isinstance(v, (int, float, str))}}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
