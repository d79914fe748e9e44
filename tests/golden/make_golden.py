"""Generates the golden fixtures of tests/golden/ from the reference itself.

The fixtures are outputs of the reference's own lbm_core routines
(src/lbm_core/device_function.hpp: calcEqu<27>, calcRhoU<27>, collision2<27>)
compiled for the host by oracle/Makefile into oracle/_ref/libref_lbm_core.so,
driven by the pull loop of StaticD3Q27PullKernel
(src/simulator/single_dev_expt/kernel.cu:2489-2735).  The reference ships no
golden vectors of its own, so these pin both the C oracle and the CUDA path.

    make -C oracle ref-cpu && python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle as O  # noqa: E402
from culbm_b200 import scenes  # noqa: E402


def unit_vectors(R, rng):
    n = 256
    rho = (1.0 + 0.05 * rng.standard_normal(n)).astype(np.float32)
    u = (0.08 * rng.standard_normal((n, 3))).astype(np.float32)
    equ = np.zeros((n, 27), np.float32)
    for k in range(n):
        R.ref_equ_f32(rho[k], u[k, 0], u[k, 1], u[k, 2], equ[k])
    f = (0.02 * rng.standard_normal((n, 27))).astype(np.float32)
    inv_tau = rng.uniform(0.3, 1.95, n).astype(np.float32)
    col = f.copy()
    mom = np.zeros((n, 4), np.float32)
    import ctypes as C
    for k in range(n):
        row = np.ascontiguousarray(col[k])
        R.ref_collide_f32(inv_tau[k], row)
        col[k] = row
        out = [C.c_float() for _ in range(4)]
        R.ref_rhou_f32(np.ascontiguousarray(f[k]), *[C.byref(o) for o in out])
        mom[k] = [o.value for o in out]
    np.savez_compressed(os.path.join(HERE, "unit_vectors.npz"), rho=rho, u=u, equ=equ, f=f, inv_tau=inv_tau,
                        collide=col, moments=mom)


def random_flags(rng, n, all_store=True):
    combos = [
        O.LOAD | O.COLLIDE | O.STORE | O.DUMP_ALL,                 # fluid
        O.LOAD | O.BOUNCE_BACK | O.STORE,                          # wall
        O.EQU | O.STORE,                                           # inlet/outlet
        O.LOAD | O.STORE | O.DUMP_RHO | O.DUMP_VZ,                 # streaming only
        O.LOAD | O.EQU | O.COLLIDE | O.STORE | O.DUMP_VX,          # load, overwrite, collide
        O.LOAD | O.BOUNCE_BACK | O.COLLIDE | O.STORE | O.DUMP_ALL,  # bounce then collide
    ]
    p = [0.6, 0.12, 0.08, 0.08, 0.06, 0.06]
    if not all_store:
        combos.append(O.LOAD | O.COLLIDE)                          # no store
        p = [0.55, 0.12, 0.08, 0.08, 0.06, 0.06, 0.05]
    return rng.choice(np.array(combos, np.uint32), n, p=p)


def stepped_case(name, scene, inv_tau, nsteps, state0):
    a = np.ascontiguousarray(state0, np.float32).copy()
    b = a.copy()
    for _ in range(nsteps):
        O.ref_step(scene, inv_tau, a, b)
        a, b = b, a
    mom = O.ref_moments(scene, a)
    np.savez_compressed(os.path.join(HERE, name), nx=scene.nx, ny=scene.ny, nz=scene.nz, flag=scene.flag,
                        rho=scene.rho, vx=scene.vx, vy=scene.vy, vz=scene.vz, inv_tau=np.float32(inv_tau),
                        nsteps=nsteps, state0=np.ascontiguousarray(state0, np.float32), state=a,
                        pulled=O.pulled(scene, a), d_rho=mom[0], d_vx=mom[1], d_vy=mom[2], d_vz=mom[3])


def main():
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libref_lbm_core.so missing: run `make -C oracle ref-cpu` first")
    R = O.ref()
    rng = np.random.default_rng(20261203)
    unit_vectors(R, rng)

    # random flag field, random start state, all cells STORE
    nx, ny, nz = 13, 11, 9
    n = nx * ny * nz
    sc = O.Scene(nx, ny, nz, random_flags(rng, n),
                 rho=(1 + 0.02 * rng.standard_normal(n)).astype(np.float32),
                 vx=(0.03 * rng.standard_normal(n)).astype(np.float32),
                 vy=(0.03 * rng.standard_normal(n)).astype(np.float32),
                 vz=(0.03 * rng.standard_normal(n)).astype(np.float32))
    stepped_case("random_13x11x9.npz", sc, 0.6, 15, (0.01 * rng.standard_normal(27 * n)).astype(np.float32))

    # the reference notebook's channel, from rest
    ch = scenes.reference_channel(16, 12, 10, 0.05)
    f, r, ux, uy, uz = ch.arrays()
    sc = O.Scene(16, 12, 10, f, r, ux, uy, uz)
    stepped_case("channel_16x12x10.npz", sc, 0.5, 30, O.rest_state(sc.n))

    # streaming only: payload = cell index, a pure permutation
    nx, ny, nz = 9, 7, 5
    n = nx * ny * nz
    sc = O.Scene(nx, ny, nz, np.full(n, O.LOAD | O.STORE | O.DUMP_ALL, np.uint32))
    payload = (np.arange(27 * n) % 4093).astype(np.float32) * np.float32(1.0 / 4096)
    stepped_case("stream_9x7x5.npz", sc, 0.5, 3, payload)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
