"""Generate the golden fixtures in tests/golden/ by running the REFERENCE's own code.

The reference (mrnorman/awflCloud) is C++ on the YAKL library, which is an absent
submodule in its repository; ``oracle/Makefile`` builds its unmodified headers on
project-written stand-ins for YAKL / yaml-cpp / netCDF into oracle/_ref/. This script
drives that build through ``oracle.pyoracle.RefHarness`` and stores:

* ``tables_o{5,9}.npz``  -- the constant tables the reference's init builds
                            (Spatial_euler3d_cons_expl_cart_fv_Agrid.h:274-315);
* ``probes_o{5,9}.npz``  -- coefs_to_tv and compute_weno_coefs on seeded inputs;
* ``case_<name>.npz``    -- per configuration: background, initial state, CFL dt,
                            tendencies of every split of steps 1-2, the state after
                            each split of step 1 and after every step;
* ``tracers_init.npz``   -- initTracers of the driver's tracers on three grids;
* ``tracer_transport.npz`` -- state and tracers after each split of the reference's own
                            tracer transport (its NO_TRACERS code compiled in);
* ``output_fields.npz``  -- everything the reference's output() writes (coordinates,
                            hydrostatic profiles, the six fields, the tracer fields).

Needs the reference's source tree (``--ref DIR`` or $AWFL_REFERENCE_DIR) and g++ with OpenMP.
Run from the repository root:  python tests/golden/make_golden.py --ref DIR
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import pyoracle  # noqa: E402
from oracle.pyoracle import RefHarness  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
SEED = 20261203

# name: (ord, nx, ny, nz, bc, weno_scalars, weno_winds, data, bubble, noise, nsteps)
BUBBLE_COS = (1, 10000.0, 10000.0, 2000.0, 2000.0, 2000.0, 2000.0, 3.0, 1.0)
CASES = {
    "o5_pw_thermal":     (5, 10, 8, 6, (0, 0, 1), True, True, "thermal", None, 0.01, 4),
    "o5_walls":          (5, 10, 8, 6, (1, 1, 1), True, True, "thermal", None, 0.01, 3),
    "o5_periodic":       (5, 10, 8, 6, (0, 0, 0), True, True, "thermal", None, 0.01, 3),
    "o5_linear":         (5, 10, 8, 6, (0, 0, 1), False, False, "thermal", None, 0.01, 3),
    "o5_mixedweno":      (5, 10, 8, 6, (0, 1, 1), False, True, "thermal", None, 0.01, 3),
    "o5_sim2d":          (5, 12, 1, 8, (0, 0, 1), True, True, "thermal", None, 0.01, 3),
    "o5_bubble_cos":     (5, 12, 12, 8, (0, 0, 1), True, True, "thermal", BUBBLE_COS, 0.01, 2),
    "o5_igw":            (5, 10, 8, 6, (0, 0, 1), True, True, "igw", None, None, 2),
    "o5_collision":      (5, 10, 8, 6, (0, 0, 1), True, True, "collision", None, None, 1),
    "o5_straka":         (5, 10, 8, 6, (0, 0, 1), True, True, "straka", None, None, 1),
    "o9_pw_thermal":     (9, 10, 8, 6, (0, 0, 1), True, True, "thermal", None, 0.01, 3),
    "o9_walls_mixed":    (9, 10, 8, 6, (1, 1, 1), True, False, "thermal", None, 0.01, 2),
    # wall directions shorter than the halo width: the stencil reaches past the line's far
    # end into halo cells that hold wall copies
    "o5_thin_walls":     (5, 1, 8, 6, (1, 0, 1), True, True, "thermal", None, 0.01, 3),
    "o5_flat_z":         (5, 10, 8, 1, (0, 1, 1), True, True, "thermal", None, 0.01, 3),
}


def make_case(name, spec):
    ord_, nx, ny, nz, bc, ws, ww, data, bubble, noise, nsteps = spec
    R = RefHarness(nx, ny, nz, bc=bc, weno_scalars=ws, weno_winds=ww, data=data, ord_=ord_)
    R.init_state()
    if bubble is not None:
        R.set_bubble(*bubble)
    if noise is not None:
        R.add_theta_noise(SEED, noise)
    out = {"config": np.array([ord_, nx, ny, nz, bc[0], bc[1], bc[2], int(ws), int(ww)]),
           "data": np.array(data), "state0": R.get_state()}
    if bubble is not None:
        out["bubble"] = np.array(bubble, dtype=np.float64)
    if noise is not None:
        out["noise"] = np.array([SEED, noise], dtype=np.float64)
    for k, v in R.background().items():
        out[k] = v
    dt = R.compute_dt(0.8)
    out["dt"] = np.array(dt)
    h = R.hs
    for step in range(nsteps):
        if step < 2:
            for spl in range(3):
                tend = R.compute_tendencies(dt, spl)
                st = R.get_state()  # halos were filled in place
                st[:, h:h + nz, h:h + ny, h:h + nx] += dt * tend
                R.set_state(st)
                out["tend_s%d_p%d" % (step, spl)] = tend
                if step == 0:
                    out["state_s0_p%d" % spl] = st
        else:
            R.time_step(dt)
        out["state_s%d" % step] = R.get_state()
    path = os.path.join(OUT, "case_%s.npz" % name)
    np.savez_compressed(path, **out)
    return path


def make_tables(ord_):
    R = RefHarness(10, 8, 6, ord_=ord_)
    np.savez_compressed(os.path.join(OUT, "tables_o%d.npz" % ord_), **R.tables())


def make_probes(ord_):
    R = RefHarness(10, 8, 6, ord_=ord_)
    rng = np.random.default_rng(SEED + ord_)
    hs = (ord_ - 1) // 2
    tv_lo_in = rng.standard_normal((64, hs + 1)) * 10.0 ** rng.integers(-6, 3, (64, 1))
    tv_hi_in = rng.standard_normal((64, ord_)) * 10.0 ** rng.integers(-6, 3, (64, 1))
    tv_lo = np.array([R.coefs_to_tv(a) for a in tv_lo_in])
    tv_hi = np.array([R.coefs_to_tv(a) for a in tv_hi_in])
    x = np.arange(ord_) - hs
    sten = [np.zeros(ord_), np.ones(ord_), 1.0 + 0.1 * x, 0.3 * x ** 2 - x, (x > 0).astype(float),
            np.where(x >= 1, 5.0, -2.0), 1e-9 * np.cos(x)]
    sten += list(rng.standard_normal((57, ord_)) * 10.0 ** rng.integers(-8, 2, (57, 1)))
    sten = np.array(sten)
    weno = np.array([R.weno_coefs(s) for s in sten])
    np.savez_compressed(os.path.join(OUT, "probes_o%d.npz" % ord_), tv_lo_in=tv_lo_in,
                        tv_lo=tv_lo, tv_hi_in=tv_hi_in, tv_hi=tv_hi, weno_in=sten, weno=weno)


# initTracers (Spatial_euler3d_cons_expl_cart_fv_Agrid.h:505-560) with the driver's three
# tracers plus one more: (ord, nx, ny, nz, bc, data)
TRACER_CASES = {
    "o5_3d": (5, 20, 20, 10, (0, 0, 1), "thermal"),
    "o5_sim2d": (5, 30, 1, 20, (0, 0, 1), "thermal"),
    "o9_walls": (9, 20, 10, 10, (1, 1, 1), "collision"),
}


def make_tracers():
    out = {}
    for name, (ord_, nx, ny, nz, bc, data) in TRACER_CASES.items():
        R = RefHarness(nx, ny, nz, bc=bc, data=data, ord_=ord_, ntracers=4)
        R.init_state()
        R.init_tracers()
        out[name + "_config"] = np.array([ord_, nx, ny, nz, bc[0], bc[1], bc[2]])
        out[name + "_data"] = np.array(data)
        out[name + "_tracers"] = R.get_tracers()
    path = os.path.join(OUT, "tracers_init.npz")
    np.savez_compressed(path, **out)
    return path


# Tracer transport by the reference's own tracer code (its Spatial header with NO_TRACERS
# blanked, built serially: oracle/Makefile): name -> (ord, nx, ny, nz, bc, pos, splits,
# crpow). Each case starts from the reference's state and tracers after two time steps of
# the noisy thermal with the driver's three tracers (initTracers), then records every
# split of `splits` (directions, in order). Positive-definite tracers are limited only in
# x and z: the reference's y limiter indexes tracerFlux(tr,k,j,ind_j) for v < 0
# (Spatial...h:1285-1286), faces of another direction that the y split never writes.
TRANSPORT_CASES = {
    "o5_pw_steps_nopos":  (5, 10, 8, 6, (0, 0, 1), (0, 0, 0), (0, 1, 2, 2, 1, 0), True),
    "o5_walls_steps_nopos": (5, 10, 8, 6, (1, 1, 1), (0, 0, 0), (0, 1, 2, 2, 1, 0), True),
    "o5_pw_xz_pos":       (5, 10, 8, 6, (0, 0, 1), (1, 1, 1), (0, 2, 2, 0), True),
    "o5_walls_xz_pos":    (5, 10, 8, 6, (1, 1, 1), (1, 1, 1), (0, 2, 2, 0), True),
    "o5_mixed_pos":       (5, 10, 8, 6, (0, 1, 1), (1, 0, 1), (0, 2), True),
    "o5_sim2d_steps_pos": (5, 12, 1, 8, (0, 0, 1), (1, 1, 1), (0, 2, 2, 0), True),
    "o9_pw_xz_pos":       (9, 10, 8, 6, (0, 0, 1), (1, 1, 1), (0, 2), True),
    "o5_pw_glibc_pos":    (5, 10, 8, 6, (0, 0, 1), (1, 1, 1), (0, 2), False),
}


def make_transport():
    out = {}
    for name, (ord_, nx, ny, nz, bc, pos, splits, crpow) in TRANSPORT_CASES.items():
        R = RefHarness(nx, ny, nz, bc=bc, ord_=ord_, crpow=crpow, ntracers=3, tracer_transport=True,
                       pos=list(pos))
        assert R.has_tracer_transport
        R.init_state()
        R.add_theta_noise(SEED, 0.01)
        R.init_tracers()
        dt = R.compute_dt(0.8 if ord_ == 5 else 0.4)
        for _ in range(2):
            R.time_step(dt)
        out[name + "_config"] = np.array([ord_, nx, ny, nz, bc[0], bc[1], bc[2], int(crpow)])
        out[name + "_pos"] = np.array(pos)
        out[name + "_splits"] = np.array(splits)
        out[name + "_dt"] = np.array(dt)
        out[name + "_state0"] = R.get_state()
        out[name + "_tracers0"] = R.get_tracers()
        for s, d in enumerate(splits):
            R.dimswitch = 1  # split index d is direction d
            R.split(dt, d)
            out[name + "_tracers%d" % (s + 1)] = R.get_tracers()
        out[name + "_state_end"] = R.get_state()
    path = os.path.join(OUT, "tracer_transport.npz")
    np.savez_compressed(path, **out)
    return path


# Spatial::output (Spatial...h:1705-1791) by the reference's own code, its netCDF writes
# recorded by the stand-in (oracle/shim/YAKL_netcdf.h): name -> (ord, nx, ny, nz, bc,
# crpow). For each case: the first record (etime 0: coordinates, hydrostatic profiles and
# the fields of the initial state with the driver's three tracers) and a later one after
# three time steps.
OUTPUT_CASES = {
    "o5_crpow": (5, 10, 8, 6, (0, 0, 1), True),
    "o5_glibc": (5, 10, 8, 6, (0, 0, 1), False),
    "o9_walls_crpow": (9, 12, 10, 8, (1, 1, 1), True),
}


def make_output():
    out = {}
    for name, (ord_, nx, ny, nz, bc, crpow) in OUTPUT_CASES.items():
        R = RefHarness(nx, ny, nz, bc=bc, ord_=ord_, crpow=crpow, ntracers=3)
        R.init_state()
        R.add_theta_noise(SEED, 0.01)
        R.init_tracers()
        dt = R.compute_dt(0.8 if ord_ == 5 else 0.4)
        out[name + "_config"] = np.array([ord_, nx, ny, nz, bc[0], bc[1], bc[2], int(crpow)])
        for rec, nsteps in ((0, 0), (1, 3)):
            for _ in range(nsteps):
                R.time_step(dt)
            etime = nsteps * dt
            out["%s_r%d_state" % (name, rec)] = R.get_state()
            out["%s_r%d_tracers" % (name, rec)] = R.get_tracers()
            for var, val in R.output(etime).items():
                out["%s_r%d_%s" % (name, rec, var)] = val
    path = os.path.join(OUT, "output_fields.npz")
    np.savez_compressed(path, **out)
    return path


def main():
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("AWFL_REFERENCE_DIR"),
                    help="the reference's source tree (mrnorman/awflCloud)")
    a = ap.parse_args()
    if not a.ref:
        ap.error("--ref or AWFL_REFERENCE_DIR is required")
    pyoracle.build(ref=True, ref_dir=a.ref)
    print("wrote", make_tracers())
    print("wrote", make_transport())
    print("wrote", make_output())
    for o in (5, 9):
        make_tables(o)
        make_probes(o)
    for name, spec in CASES.items():
        print("wrote", make_case(name, spec))


if __name__ == "__main__":
    main()
