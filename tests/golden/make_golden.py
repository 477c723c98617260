"""Generate the golden fixtures under tests/golden/ from the reference tree.

Run here (where the reference tree and oracle/_ref/libltref.so exist); the outputs are
committed so the GPU tests never read the reference tree.

  kat_dpie95.npz   the reference's known-answer test: 95 dPIE halos and one image point
                   with the deflection computed by Lenstool
                   (Benchmarks/GradientBenchmark/setup.cpp:19-44, SOA set-up :120-193),
                   plus the reference's own SoA gradient at that point.
  par_<name>.npz   catalogues read from Benchmarks/ConfigFiles/<name>.par (one per
                   profile: 90Pot81 = dPIE, 90Pot = PIEMD, 90PotSIS = SIS, MarkusBenchmark =
                   702 SIS) with the reference's outputs on a small grid over the file's
                   frame: deflection (gradient_grid_CPU) for every file; Hessian
                   (gradient2_grid_CPU), amplif_grid_CPU mode 5, the GPU Hessian and Kmap
                   kernels and the potential kernel (run on the host) for the dPIE file.

Usage:  python tests/golden/make_golden.py --reference <reference tree>
        (or with the tree in $LT_REFERENCE_TREE)
"""
from __future__ import annotations

import argparse
import importlib.util
import math
import os
import pathlib
import re
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent


def _load_pkg():
    spec = importlib.util.spec_from_file_location(
        "lenstool_hpc_b200", ROOT / "lenstool-hpc_b200" / "__init__.py",
        submodule_search_locations=[str(ROOT / "lenstool-hpc_b200")])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["lenstool_hpc_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def parse_c_array(text: str, name: str) -> np.ndarray:
    m = re.search(r"\b" + re.escape(name) + r"\s*\[\s*\]\s*=\s*\{([^}]*)\}", text)
    if not m:
        raise ValueError(f"array {name} not found")
    return np.array([float(v) for v in m.group(1).replace("\n", " ").split(",") if v.strip()])


def parse_c_scalar(text: str, name: str) -> float:
    m = re.search(r"\b" + re.escape(name) + r"\s*=\s*([-+0-9.eE]+)\s*;", text)
    if not m:
        raise ValueError(f"scalar {name} not found")
    return float(m.group(1))


def kat(ref_tree: pathlib.Path, out: pathlib.Path, catalog, reflib):
    src = (ref_tree / "Benchmarks" / "GradientBenchmark" / "setup.cpp").read_text()
    arr = {k: parse_c_array(src, k) for k in ("pos_x", "pos_y", "theta", "epot", "rcore", "rcut", "b0")}
    types = parse_c_array(src, "lense_type").astype(np.int32)
    n = int(parse_c_scalar(src, "num_lenses"))
    assert all(a.shape[0] == n for a in arr.values()) and types.shape[0] == n
    cs = np.array([math.cos(t) for t in arr["theta"]])
    sn = np.array([math.sin(t) for t in arr["theta"]])
    cat = catalog.HaloCatalog(type=types, position_x=arr["pos_x"], position_y=arr["pos_y"], b0=arr["b0"],
                              ellipticity_angle=arr["theta"], anglecos=cs, anglesin=sn,
                              ellipticity_potential=arr["epot"], rcore=arr["rcore"], rcut=arr["rcut"],
                              dlsds=np.ones(n), z=0.4)
    px, py = parse_c_scalar(src, "x_c"), parse_c_scalar(src, "y_c")
    gx, gy = parse_c_scalar(src, "grad_x"), parse_c_scalar(src, "grad_y")
    rx, ry = reflib.grad_points(cat, np.array([px]), np.array([py]))
    np.savez(out / "kat_dpie95.npz", **cat.arrays(), px=px, py=py, lenstool_grad=np.array([gx, gy]),
             reference_grad=np.array([rx[0], ry[0]]))
    print(f"kat: lenstool {gx:.15g} {gy:.15g}  reference SoA {rx[0]:.15g} {ry[0]:.15g}")


def parse_par(path: pathlib.Path, catalog):
    """Potential sections and frame of a Lenstool .par file, following
    module_readParameters_PotentialSOA_direct (src/module_readParameters.cpp:2234-2485) for
    the keys these fixtures use (radii in arcsec, angle_pos in degrees)."""
    dtr = math.acos(-1.) / 180.
    lines = path.read_text().splitlines()
    halos, frame = [], {}
    i = 0
    while i < len(lines):
        tok = lines[i].split()
        i += 1
        if not tok:
            continue
        if tok[0].startswith("potent"):
            h = dict(type=0, x=0., y=0., e=0., angle=0., vdisp=0., rcut=0., rcore=0., z=0.)
            while i < len(lines):
                t2 = lines[i].split()
                i += 1
                if not t2:
                    continue
                key, val = t2[0], (t2[1] if len(t2) > 1 else "")
                if key == "end":
                    break
                if key in ("profil", "profile"):
                    h["type"] = int(val)
                elif key in ("x_centre", "x_center"):
                    h["x"] = float(val)
                elif key in ("y_centre", "y_center"):
                    h["y"] = float(val)
                elif key in ("ellipticitymass", "ellipticity", "ellipticite"):
                    h["e"] = float(val)
                elif key in ("ellipticity_angle", "angle_pos"):
                    h["angle"] = float(val) * dtr
                elif key in ("rcore", "core_radius"):
                    h["rcore"] = float(val)
                elif key in ("rcut", "cut_radius"):
                    h["rcut"] = float(val)
                elif key == "z_lens":
                    h["z"] = float(val)
                elif key == "v_disp":
                    h["vdisp"] = float(val)
                elif key in ("core_radius_kpc", "cut_radius_kpc"):
                    raise ValueError("kpc radii need the cosmology; not used by these fixtures")
            halos.append(h)
        elif tok[0] == "frame":
            while i < len(lines):
                t2 = lines[i].split()
                i += 1
                if not t2:
                    continue
                if t2[0] == "end":
                    break
                if t2[0] in ("xmin", "xmax", "ymin", "ymax"):
                    frame[t2[0]] = float(t2[1])
    t = np.array([h["type"] for h in halos], np.int32)
    cat = catalog.make_catalog(t, [h["x"] for h in halos], [h["y"] for h in halos], [h["vdisp"] for h in halos],
                               [h["e"] for h in halos], [h["angle"] for h in halos], [h["rcore"] for h in halos],
                               [h["rcut"] for h in halos], z=halos[0]["z"])
    # anglecos/anglesin as the reader computes them (libm cos/sin)
    cat.anglecos = np.array([math.cos(a) for a in cat.ellipticity_angle])
    cat.anglesin = np.array([math.sin(a) for a in cat.ellipticity_angle])
    return cat, frame


def par_fixture(ref_tree, out, name, catalog, reflib, n=33):
    cat, frame = parse_par(ref_tree / "Benchmarks" / "ConfigFiles" / f"{name}.par", catalog)
    g = catalog.Grid(frame["xmin"], frame["xmax"], frame["ymin"], frame["ymax"], n, n)
    ax, ay = reflib.grad_grid(cat, g)
    extra = {}
    if np.all(cat.type == 81):
        extra["hess"] = np.stack(reflib.hess_grid(cat, g))
        extra["amplif5"] = reflib.amplif5_grid(cat, g)
        extra["gpu_hess"] = np.stack(reflib.gpu_kernel_grid("hess", cat, g))
        extra["pot"] = reflib.gpu_kernel_grid("pot", cat, g)
        # Kmap: two source planes, the second half of the halos at a different D_LS/D_OS
        kcat = catalog.HaloCatalog(**{**cat.arrays(), "z": cat.z})
        kcat.dlsds = np.where(np.arange(cat.n) < cat.n // 2, 0.7, 0.45)
        extra["kmap_dlsds"] = kcat.dlsds
        extra["kmap"] = np.stack(reflib.gpu_kernel_grid("kmap", kcat, g))
    np.savez(out / f"par_{name}.npz", **cat.arrays(), grid=np.array([g.xmin, g.xmax, g.ymin, g.ymax, n, n]),
             grad=np.stack([ax, ay]), **extra)
    print(f"{name}: {cat.n} halos, types {sorted(set(cat.type.tolist()))}, keys {sorted(extra)}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("LT_REFERENCE_TREE"),
                    help="the reference source tree (default: $LT_REFERENCE_TREE)")
    args = ap.parse_args()
    if not args.reference:
        ap.error("give --reference or set LT_REFERENCE_TREE")
    os.environ["LT_REFERENCE_TREE"] = args.reference
    ref_tree = pathlib.Path(args.reference)
    pkg = _load_pkg()
    from lenstool_hpc_b200 import catalog  # noqa: E402
    sys.path.insert(0, str(ROOT))
    import oracle  # noqa: E402
    oracle.build(with_reference=True)
    reflib = oracle.RefLib()
    kat(ref_tree, HERE, catalog, reflib)
    for name in ("90Pot81", "90Pot", "90PotSIS", "MarkusBenchmark"):
        par_fixture(ref_tree, HERE, name, catalog, reflib)
    del pkg


if __name__ == "__main__":
    main()
