"""Build the reference's unmodified driver.cpp against the drop-in operator headers.

driver.cpp (mrnorman/awflCloud) includes "const.h", "Spatial_euler3d_cons_expl_cart_fv_
Agrid.h" and "Temporal_ader.h" with quotes. It is compiled from standard input so that those
quote includes resolve to awflcloud_b200/dropin/ (the drop-in headers) and not to the copies
next to driver.cpp; the binary links libawfl.so. Output: awflcloud_b200/dropin/bin/
driver_o{5,9}. The reference source is read in place and never copied.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
DROPIN = os.path.join(HERE, "dropin")
BIN = os.path.join(DROPIN, "bin")


def cxx() -> str:
    return shutil.which("g++") or "/usr/bin/g++"


def build(ref_dir: str, orders=((5, 3), (9, 5))) -> list:
    from . import build as libbuild
    lib = libbuild.build()
    driver = os.path.join(ref_dir, "driver.cpp")
    if not os.path.exists(driver):
        raise FileNotFoundError(driver)
    os.makedirs(BIN, exist_ok=True)
    outs = []
    for o, g in orders:
        out = os.path.join(BIN, "driver_o%d" % o)
        cmd = [cxx(), "-std=c++17", "-O2", "-DORD=%d" % o, "-DNGLL=%d" % g, "-I" + DROPIN,
               "-I" + os.path.join(ROOT, "include"), "-x", "c++", "-", "-x", "none",
               "-L" + os.path.dirname(lib), "-lawfl", "-Wl,-rpath,$ORIGIN/../../lib", "-o", out]
        with open(driver, "rb") as src:
            subprocess.run(cmd, stdin=src, check=True)
        outs.append(out)
    return outs


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("AWFL_REFERENCE_DIR")
    if not ref:
        sys.exit("usage: python -m awflcloud_b200.dropin_build <reference source tree> "
                 "(or set AWFL_REFERENCE_DIR)")
    print(build(ref))
