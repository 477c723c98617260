"""Halo catalogues in the reference's Potential_SOA layout, and the seeded generators of
the benchmark workloads.

Field meaning follows ``struct Potential_SOA`` (src/structure_hpc.hpp:257-287): halos are
sorted into contiguous runs of equal profile type (src/module_readParameters.cpp:2289-2293
and :2455-2477), angles are in radians with ``anglecos``/``anglesin`` precomputed
(:2470-2471), and ``b0``/``ellipticity_potential`` are derived from the velocity
dispersion and mass ellipticity by module_readParameters_calculatePotentialparameter
(src/module_readParameters.cpp:2808-2871).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

# pi / c^2 in arcsec per (km/s)^2, src/structure_hpc.hpp:62
PI_C2 = 7.209970e-06

SIS, PIEMD, DPIE = 5, 8, 81
SUPPORTED_TYPES = (SIS, PIEMD, DPIE)

FIELDS = ("position_x", "position_y", "b0", "ellipticity_angle", "anglecos", "anglesin",
          "ellipticity_potential", "rcore", "rcut", "dlsds")


@dataclasses.dataclass
class HaloCatalog:
    """Structure of arrays, one entry per halo, float64 except ``type`` (int32)."""
    type: np.ndarray
    position_x: np.ndarray
    position_y: np.ndarray
    b0: np.ndarray
    ellipticity_angle: np.ndarray
    anglecos: np.ndarray
    anglesin: np.ndarray
    ellipticity_potential: np.ndarray
    rcore: np.ndarray
    rcut: np.ndarray
    dlsds: np.ndarray
    z: float = 0.35

    @property
    def n(self) -> int:
        return int(self.type.shape[0])

    def arrays(self) -> dict:
        out = {"type": self.type}
        for f in FIELDS:
            out[f] = getattr(self, f)
        return out

    def contiguous(self) -> "HaloCatalog":
        kw = {"type": np.ascontiguousarray(self.type, dtype=np.int32), "z": self.z}
        for f in FIELDS:
            kw[f] = np.ascontiguousarray(getattr(self, f), dtype=np.float64)
        return HaloCatalog(**kw)

    def subset(self, idx) -> "HaloCatalog":
        kw = {"type": self.type[idx], "z": self.z}
        for f in FIELDS:
            kw[f] = getattr(self, f)[idx]
        return HaloCatalog(**kw).contiguous()

    def sorted_by_type(self) -> "HaloCatalog":
        """Stable sort into runs of equal type, ascending type id (the reference fills
        the SoA by type index, src/module_readParameters.cpp:2455-2477)."""
        order = np.argsort(self.type, kind="stable")
        return self.subset(order)


def potential_parameters(ptype, vdisp, ellipticity):
    """b0 and ellipticity_potential from v_disp and the mass ellipticity,
    module_readParameters_calculatePotentialparameter, src/module_readParameters.cpp:2808-2871.
    """
    ptype = np.asarray(ptype)
    vdisp = np.asarray(vdisp, dtype=np.float64)
    e = np.asarray(ellipticity, dtype=np.float64)
    b0 = np.where(ptype == SIS, 4 * PI_C2 * vdisp * vdisp, 6. * PI_C2 * vdisp * vdisp)
    with np.errstate(divide="ignore", invalid="ignore"):
        epot_piemd = np.where(e == 0., 0.00001, (1. - np.sqrt(1 - e * e)) / np.where(e == 0., 1., e))
    epot = np.where(ptype == SIS, e / 3, epot_piemd)
    return b0, epot


def make_catalog(ptype, x, y, vdisp, ellipticity, angle, rcore, rcut, z=0.35, dlsds=None) -> HaloCatalog:
    ptype = np.asarray(ptype, dtype=np.int32)
    b0, epot = potential_parameters(ptype, vdisp, ellipticity)
    angle = np.asarray(angle, dtype=np.float64)
    n = ptype.shape[0]
    cat = HaloCatalog(
        type=ptype, position_x=np.asarray(x, np.float64), position_y=np.asarray(y, np.float64), b0=b0,
        ellipticity_angle=angle, anglecos=np.cos(angle), anglesin=np.sin(angle),
        ellipticity_potential=epot, rcore=np.asarray(rcore, np.float64), rcut=np.asarray(rcut, np.float64),
        dlsds=np.ones(n) if dlsds is None else np.asarray(dlsds, np.float64), z=z)
    return cat.sorted_by_type()


def cluster_galaxy_catalog(n_cluster: int, n_galaxy: int, seed: int, cluster_type: int = DPIE,
                           z: float = 0.35) -> HaloCatalog:
    """The synthetic cluster + galaxy catalogue of the benchmark workloads.

    Cluster-scale halos: sigma0 ~ U(800, 1200) km/s, rcore ~ U(5, 15)", rcut = 800",
    e ~ U[0, 0.6], theta ~ U[0, pi), centres ~ U(+-20")^2.
    Galaxy-scale halos (cut dPIE, type 81): sigma0 log-uniform in (80, 300) km/s,
    rcore ~ U(0.05, 0.2)", rcut ~ U(5, 50)", e ~ U[0, 0.5], theta ~ U[0, pi),
    centres ~ U(+-90")^2.  Draws use numpy PCG64 with the given seed.
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    nc, ng = n_cluster, n_galaxy
    c_sig = rng.uniform(800., 1200., nc)
    c_rc = rng.uniform(5., 15., nc)
    c_rcut = np.full(nc, 800.)
    c_e = rng.uniform(0., 0.6, nc)
    c_th = rng.uniform(0., math.pi, nc)
    c_x = rng.uniform(-20., 20., nc)
    c_y = rng.uniform(-20., 20., nc)
    g_sig = np.exp(rng.uniform(math.log(80.), math.log(300.), ng))
    g_rc = rng.uniform(0.05, 0.2, ng)
    g_rcut = rng.uniform(5., 50., ng)
    g_e = rng.uniform(0., 0.5, ng)
    g_th = rng.uniform(0., math.pi, ng)
    g_x = rng.uniform(-90., 90., ng)
    g_y = rng.uniform(-90., 90., ng)
    ptype = np.concatenate([np.full(nc, cluster_type), np.full(ng, DPIE)])
    return make_catalog(ptype, np.concatenate([c_x, g_x]), np.concatenate([c_y, g_y]),
                        np.concatenate([c_sig, g_sig]), np.concatenate([c_e, g_e]),
                        np.concatenate([c_th, g_th]), np.concatenate([c_rc, g_rc]),
                        np.concatenate([c_rcut, g_rcut]), z=z)


def perturb_catalog(base: HaloCatalog, rng: np.random.Generator, rel: float = 0.05) -> HaloCatalog:
    """A posterior-sample-like catalogue: every continuous parameter p -> p (1 + rel N(0,1)),
    positions move by rel (|x| + 1") N(0,1), ellipticity_potential clipped to [1e-5, 0.95],
    rcore < rcut enforced.  b0 is perturbed directly (it is the sample's impact parameter)."""
    n = base.n
    def jitter(a):
        return a * (1. + rel * rng.standard_normal(n))
    x = base.position_x + rel * (np.abs(base.position_x) + 1.) * rng.standard_normal(n)
    y = base.position_y + rel * (np.abs(base.position_y) + 1.) * rng.standard_normal(n)
    b0 = np.abs(jitter(base.b0))
    epot = np.clip(jitter(base.ellipticity_potential), 1e-5, 0.95)
    ang = jitter(base.ellipticity_angle)
    rc = np.abs(jitter(base.rcore))
    rcut = np.abs(jitter(base.rcut))
    rcut = np.maximum(rcut, rc * 1.5)
    return HaloCatalog(type=base.type.copy(), position_x=x, position_y=y, b0=b0, ellipticity_angle=ang,
                       anglecos=np.cos(ang), anglesin=np.sin(ang), ellipticity_potential=epot, rcore=rc,
                       rcut=rcut, dlsds=base.dlsds.copy(), z=base.z).contiguous()


@dataclasses.dataclass
class HaloParameters:
    """The physical parameters a posterior sample varies, in catalogue (type-sorted) order:
    the inputs of lt_catalog_update (Catalog.update)."""
    type: np.ndarray
    position_x: np.ndarray
    position_y: np.ndarray
    vdisp: np.ndarray
    ellipticity: np.ndarray
    ellipticity_angle: np.ndarray
    rcore: np.ndarray
    rcut: np.ndarray

    def catalog(self, z: float = 0.35) -> HaloCatalog:
        if np.any(np.diff(self.type) < 0):
            raise ValueError("parameters must be sorted by profile type")
        return make_catalog(self.type, self.position_x, self.position_y, self.vdisp, self.ellipticity,
                            self.ellipticity_angle, self.rcore, self.rcut, z=z)

    def perturbed(self, rng: np.random.Generator, rel: float = 0.05) -> "HaloParameters":
        """p -> p (1 + rel N(0,1)) for vdisp, ellipticity (clipped to [0, 0.95]), angle,
        rcore and rcut (kept >= 1.5 rcore); positions move by rel (|x| + 1") N(0,1)."""
        n = self.type.shape[0]

        def jitter(a):
            return a * (1. + rel * rng.standard_normal(n))
        x = self.position_x + rel * (np.abs(self.position_x) + 1.) * rng.standard_normal(n)
        y = self.position_y + rel * (np.abs(self.position_y) + 1.) * rng.standard_normal(n)
        sig = np.abs(jitter(self.vdisp))
        e = np.clip(jitter(self.ellipticity), 0., 0.95)
        th = jitter(self.ellipticity_angle)
        rc = np.abs(jitter(self.rcore))
        rcut = np.maximum(np.abs(jitter(self.rcut)), 1.5 * rc)
        return HaloParameters(self.type.copy(), x, y, sig, e, th, rc, rcut)

    def update_args(self):
        """The arguments of Catalog.update, with the host's cos/sin of the angle."""
        return (self.position_x, self.position_y, self.vdisp, self.ellipticity, self.ellipticity_angle, self.rcore,
                self.rcut, np.cos(self.ellipticity_angle), np.sin(self.ellipticity_angle))


def cluster_galaxy_parameters(n_cluster: int, n_galaxy: int, seed: int, cluster_type: int = DPIE) -> HaloParameters:
    """The physical parameters behind cluster_galaxy_catalog (same draws, same order)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nc, ng = n_cluster, n_galaxy
    c_sig = rng.uniform(800., 1200., nc)
    c_rc = rng.uniform(5., 15., nc)
    c_rcut = np.full(nc, 800.)
    c_e = rng.uniform(0., 0.6, nc)
    c_th = rng.uniform(0., math.pi, nc)
    c_x = rng.uniform(-20., 20., nc)
    c_y = rng.uniform(-20., 20., nc)
    g_sig = np.exp(rng.uniform(math.log(80.), math.log(300.), ng))
    g_rc = rng.uniform(0.05, 0.2, ng)
    g_rcut = rng.uniform(5., 50., ng)
    g_e = rng.uniform(0., 0.5, ng)
    g_th = rng.uniform(0., math.pi, ng)
    g_x = rng.uniform(-90., 90., ng)
    g_y = rng.uniform(-90., 90., ng)
    ptype = np.concatenate([np.full(nc, cluster_type), np.full(ng, DPIE)]).astype(np.int32)
    cat = lambda a, b: np.concatenate([a, b])  # noqa: E731
    return HaloParameters(ptype, cat(c_x, g_x), cat(c_y, g_y), cat(c_sig, g_sig), cat(c_e, g_e), cat(c_th, g_th),
                          cat(c_rc, g_rc), cat(c_rcut, g_rcut))


@dataclasses.dataclass
class Grid:
    """A pixel grid with both endpoints included: x_i = xmin + (i + istart) dx with
    dx = (xmax - xmin)/(n - 1) (src/grid_gradient_CPU.cpp:33-63), stored row-major at
    j*nx + i."""
    xmin: float
    xmax: float
    ymin: float
    ymax: float
    nx: int
    ny: int
    istart: int = 0
    jstart: int = 0
    dx: float = 0.
    dy: float = 0.

    def __post_init__(self):
        if not self.dx:
            self.dx = (self.xmax - self.xmin) / (self.nx - 1)
        if not self.dy:
            self.dy = (self.ymax - self.ymin) / (self.ny - 1)

    @classmethod
    def square(cls, half_width: float, n: int) -> "Grid":
        return cls(-half_width, half_width, -half_width, half_width, n, n)

    @property
    def npix(self) -> int:
        return self.nx * self.ny

    def coords(self, index=None):
        """Pixel coordinates computed with the reference's arithmetic (one multiply,
        one add, no fused multiply-add)."""
        if index is None:
            index = np.arange(self.npix, dtype=np.int64)
        index = np.asarray(index, dtype=np.int64)
        ii = index % self.nx
        jj = index // self.nx
        px = self.xmin + (ii + self.istart).astype(np.float64) * self.dx
        py = self.ymin + (jj + self.jstart).astype(np.float64) * self.dy
        return px, py


# Workload definitions (sizes of the benchmark configurations).
WORKLOADS = {
    "grad_200h_1024": dict(n_cluster=2, n_galaxy=198, half=100., n=1024, seed=20261203),
    "maps_1000h_4096": dict(n_cluster=4, n_galaxy=996, half=150., n=4096, seed=20261204),
}


def workload(name: str, cluster_type: int = DPIE):
    w = WORKLOADS[name]
    cat = cluster_galaxy_catalog(w["n_cluster"], w["n_galaxy"], w["seed"], cluster_type=cluster_type)
    return cat, Grid.square(w["half"], w["n"])
