"""bayes.dat posterior samples: the file reader, the meaning of its columns, and the model
their rows perturb (applied on the device by Context.bayes / lt_bayes_apply).

Reference: module_readParameters_preparebayes / _bayesmodels read the file
(src/module_readParameters.cpp:53-110: every '#' line names one column, every other line
holds one sample); module_readParameters_setbayesmapmodels (:132-227) walks the halos in
parameter-file order and takes, for each free parameter, the next column in the order
x, y, ellipticity_potential, ellipticity, theta (degrees), rcore, vdisp, rcut, z, after
two leading columns (Nsample, ln(Lhood)); then skips the image-redshift columns and
takes each potfile's cut and sigma."""
from __future__ import annotations

import dataclasses
import math
import re
from typing import Dict, Iterable, List, Optional, Sequence, Tuple

import numpy as np

SKIP, X, Y, EPOT, EMASS, THETA, RCORE, VDISP, RCUT, Z, POT_CUT, POT_SIGMA = range(12)
FIELD_NAMES = {X: "x", Y: "y", EPOT: "epot", EMASS: "emass", THETA: "theta", RCORE: "rcore", VDISP: "vdisp",
               RCUT: "rcut", Z: "z", POT_CUT: "pot_cut", POT_SIGMA: "pot_sigma"}
# the per-halo order of setbayesmapmodels (src/module_readParameters.cpp:142-188)
HALO_ORDER = (X, Y, EPOT, EMASS, THETA, RCORE, VDISP, RCUT, Z)
# column labels of the bayes.dat files the reference ships
_HALO_LABELS = {"x (arcsec)": X, "y (arcsec)": Y, "emass": EMASS, "theta (deg)": THETA, "rc (arcsec)": RCORE,
                "sigma (km/s)": VDISP, "rcut (arcsec)": RCUT}
_POT_LABELS = {"rcut (arcsec)": POT_CUT, "sigma (km/s)": POT_SIGMA}


def read_bayes(path) -> Tuple[List[str], np.ndarray]:
    """The column names ('#' lines, without the '#') and the samples (nvalues x nparam),
    as module_readParameters_preparebayes / _bayesmodels read them."""
    names: List[str] = []
    rows: List[List[float]] = []
    with open(path) as f:
        for line in f:
            if line.startswith("#"):
                names.append(line[1:].rstrip("\n"))
                continue
            vals = line.split()
            if not vals:
                continue
            if len(vals) < len(names):
                raise ValueError(f"{path}: a sample has {len(vals)} values, {len(names)} columns are named")
            rows.append([float(v) for v in vals[:len(names)]])
    return names, np.asarray(rows, np.float64).reshape(len(rows), len(names))


def columns_from_names(names: Sequence[str], halo_index=None, potfile_index=None) -> np.ndarray:
    """Column meanings (int32 pairs field, target) from bayes.dat column names:
    'O<k> : <label>' addresses halo halo_index(k) (default k - 1), 'Pot<k> <label>'
    potfile potfile_index(k) (default k); every other column (Nsample, ln(Lhood),
    'Redshift of ...', Chi2) is skipped.  A halo label that setbayesmapmodels does not read
    (e.g. an external shear's gamma) raises: it would shift every later column."""
    halo_index = halo_index or (lambda k: k - 1)
    potfile_index = potfile_index or (lambda k: k)
    out = np.zeros((len(names), 2), np.int32)
    for c, name in enumerate(names):
        m = re.match(r"\s*O(\d+)\s*:\s*(.*?)\s*$", name)
        if m:
            label = m.group(2)
            if label not in _HALO_LABELS:
                raise ValueError(f"column {c} '{name}': parameter '{label}' is not read by the map path")
            out[c] = (_HALO_LABELS[label], halo_index(int(m.group(1))))
            continue
        m = re.match(r"\s*Pot(\d+)\s+(.*?)\s*$", name)
        if m:
            label = m.group(2)
            if label not in _POT_LABELS:
                raise ValueError(f"column {c} '{name}': potfile parameter '{label}' is not read by the map path")
            out[c] = (_POT_LABELS[label], potfile_index(int(m.group(1))))
    return out


def columns_from_free(free: Sequence[Iterable[int]], n_z_param: int = 0,
                      potfile_free: Sequence[Tuple[bool, bool]] = (), soa_index=None) -> np.ndarray:
    """The column layout setbayesmapmodels assumes: 2 leading columns, then for halo i (in
    parameter-file order) its free fields in HALO_ORDER, addressed to soa_index[i] (the
    catalogue position; default i), then n_z_param redshift columns, then per potfile its
    cut (if free) and sigma (if free)."""
    cols = [(SKIP, 0), (SKIP, 0)]
    for i, fields in enumerate(free):
        fs = set(fields)
        bad = fs - set(HALO_ORDER)
        if bad:
            raise ValueError(f"halo {i}: unknown fields {sorted(bad)}")
        tgt = int(soa_index[i]) if soa_index is not None else i
        cols += [(f, tgt) for f in HALO_ORDER if f in fs]
    cols += [(SKIP, 0)] * n_z_param
    for k, (cut, sigma) in enumerate(potfile_free):
        if cut:
            cols.append((POT_CUT, k))
        if sigma:
            cols.append((POT_SIGMA, k))
    return np.asarray(cols, np.int32).reshape(-1, 2)


@dataclasses.dataclass
class Potfile:
    """One potfile's scaling relations (setScalingRelations,
    src/module_readParameters.cpp:1539-1656, ftype 1): galaxies first .. first+count-1
    of the model; lengths in arcsec."""
    first: int
    count: int
    mag0: float
    sigma: float
    cut: float
    core: float
    vdslope: float = 4.0
    slope: float = 4.0


@dataclasses.dataclass
class BayesModel:
    """The Potential_SOA state bayes.dat rows perturb, in catalogue (type-sorted) order."""
    type: np.ndarray
    position_x: np.ndarray
    position_y: np.ndarray
    ellipticity_potential: np.ndarray
    ellipticity: np.ndarray
    ellipticity_angle: np.ndarray  # radians
    rcore: np.ndarray
    vdisp: np.ndarray
    rcut: np.ndarray
    mag: Optional[np.ndarray] = None

    @property
    def n(self) -> int:
        return int(np.asarray(self.type).shape[0])

    def arrays(self):
        f64 = lambda a: np.ascontiguousarray(a, np.float64)  # noqa: E731
        return (np.ascontiguousarray(self.type, np.int32), f64(self.position_x), f64(self.position_y),
                f64(self.ellipticity_potential), f64(self.ellipticity), f64(self.ellipticity_angle), f64(self.rcore),
                f64(self.vdisp), f64(self.rcut), None if self.mag is None else f64(self.mag))


def model_from_parameters(p, epot=None) -> BayesModel:
    """A BayesModel from catalog.HaloParameters (ellipticity_potential 0 unless given:
    the potential-parameter step derives it from the mass ellipticity)."""
    n = p.type.shape[0]
    return BayesModel(p.type.copy(), p.position_x.copy(), p.position_y.copy(),
                      np.zeros(n) if epot is None else np.asarray(epot, np.float64).copy(), p.ellipticity.copy(),
                      p.ellipticity_angle.copy(), p.rcore.copy(), p.vdisp.copy(), p.rcut.copy())


def synthetic_rows(model: BayesModel, columns: np.ndarray, n_rows: int, rng: np.random.Generator,
                   rel: float = 0.05, potfiles: Sequence[Potfile] = ()) -> np.ndarray:
    """Seeded bayes-like samples for `columns`: each free value is the model's value times
    (1 + rel N(0,1)) (positions move by rel (|x| + 1") N(0,1); theta in degrees; emass
    clipped to [0, 0.95]; rcut kept above 1.5 rcore); skipped columns hold the sample index
    (column 0) or 0."""
    rows = np.zeros((n_rows, columns.shape[0]))
    rows[:, 0] = np.arange(1, n_rows + 1)
    for c, (f, t) in enumerate(columns):
        g = rng.standard_normal(n_rows)
        if f in (X, Y):
            v = (model.position_x if f == X else model.position_y)[t]
            rows[:, c] = v + rel * (abs(v) + 1.) * g
        elif f == EMASS:
            rows[:, c] = np.clip(model.ellipticity[t] * (1. + rel * g), 0., 0.95)
        elif f == EPOT:
            rows[:, c] = np.clip(model.ellipticity_potential[t] * (1. + rel * g), 1e-5, 0.95)
        elif f == THETA:
            rows[:, c] = np.degrees(model.ellipticity_angle[t]) * (1. + rel * g)
        elif f == RCORE:
            rows[:, c] = abs(model.rcore[t] * (1. + rel * g))
        elif f == VDISP:
            rows[:, c] = abs(model.vdisp[t] * (1. + rel * g))
        elif f == RCUT:
            rows[:, c] = abs(model.rcut[t] * (1. + rel * g))
        elif f == POT_CUT:
            rows[:, c] = abs(potfiles[t].cut * (1. + rel * g))
        elif f == POT_SIGMA:
            rows[:, c] = abs(potfiles[t].sigma * (1. + rel * g))
    # rcut > 1.5 rcore for halos with both free
    for t in np.unique(columns[(columns[:, 0] == RCUT), 1]):
        cc = np.where((columns[:, 0] == RCUT) & (columns[:, 1] == t))[0][0]
        rcs = np.where((columns[:, 0] == RCORE) & (columns[:, 1] == t))[0]
        rc = rows[:, rcs[0]] if rcs.size else np.full(n_rows, model.rcore[t])
        rows[:, cc] = np.maximum(rows[:, cc], 1.5 * rc)
    return rows


def reference_state(model: BayesModel, potfiles: Sequence[Potfile], columns: np.ndarray, row: np.ndarray) -> Dict:
    """A pure-numpy statement of one row applied to the model (setbayesmapmodels +
    setScalingRelations + the potential-parameter step), for tests: the Potential_SOA
    fields the records are packed from (x, y, b0, epot, cos, sin, rcore, rcut)."""
    n = model.n
    st = {k: np.array(getattr(model, k), np.float64) for k in (
        "position_x", "position_y", "ellipticity_potential", "ellipticity", "rcore", "vdisp", "rcut")}
    # the C library's cos/sin/pow (math), as the reference's host code calls them
    cs = np.array([math.cos(a) for a in model.ellipticity_angle])
    sn = np.array([math.sin(a) for a in model.ellipticity_angle])
    t = np.asarray(model.type)
    for _ in range(3):
        _calc(t, st)
    dtr = math.acos(-1.) / 180.
    for c, (f, tg) in enumerate(columns):
        v = row[c]
        if f in (X, Y, EPOT, EMASS, RCORE, VDISP, RCUT):
            key = {X: "position_x", Y: "position_y", EPOT: "ellipticity_potential", EMASS: "ellipticity",
                   RCORE: "rcore", VDISP: "vdisp", RCUT: "rcut"}[f]
            st[key][tg] = v
        elif f == THETA:
            cs[tg], sn[tg] = math.cos(float(v) * dtr), math.sin(float(v) * dtr)
    for k, p in enumerate(potfiles):
        sig = next((row[c] for c, (f, tg) in enumerate(columns) if f == POT_SIGMA and tg == k), p.sigma)
        cut = next((row[c] for c, (f, tg) in enumerate(columns) if f == POT_CUT and tg == k), p.cut)
        for i in range(p.first, p.first + p.count):
            mag = float(model.mag[i])
            if mag != 0:
                st["rcore"][i] = p.core * math.pow(10., 0.4 * (p.mag0 - mag) / 2.)
                st["vdisp"][i] = float(sig) * math.pow(10., 0.4 * (p.mag0 - mag) / p.vdslope)
                st["rcut"][i] = float(cut) * math.pow(10., 0.4 * (p.mag0 - mag) * 2. / p.slope)
    b0 = _calc(t, st)
    return {"x": st["position_x"], "y": st["position_y"], "b0": b0, "epot": st["ellipticity_potential"],
            "cos": cs, "sin": sn, "rcore": st["rcore"], "rcut": st["rcut"]}


def base_state(model: BayesModel, potfiles: Sequence[Potfile] = ()) -> Dict:
    """The model's own state (no column applied; potfiles at their own sigma and cut)."""
    return reference_state(model, potfiles, np.zeros((0, 2), np.int32), np.zeros(0))


def catalog_from_state(model: BayesModel, st: Dict, dlsds=None):
    """The HaloCatalog (lt_catalog_upload's input) of a state from reference_state."""
    from .catalog import HaloCatalog
    n = model.n
    return HaloCatalog(type=np.asarray(model.type, np.int32).copy(), position_x=st["x"].copy(),
                       position_y=st["y"].copy(), b0=st["b0"].copy(), ellipticity_angle=np.arctan2(st["sin"], st["cos"]),
                       anglecos=st["cos"].copy(), anglesin=st["sin"].copy(), ellipticity_potential=st["epot"].copy(),
                       rcore=st["rcore"].copy(), rcut=st["rcut"].copy(),
                       dlsds=np.ones(n) if dlsds is None else np.asarray(dlsds, np.float64).copy()).contiguous()


def _calc(t, st):
    pi_c2 = 7.209970e-06
    v, em, ep = st["vdisp"], st["ellipticity"], st["ellipticity_potential"]
    b0 = np.where(t == 5, 4. * pi_c2 * v * v, 6. * pi_c2 * v * v)
    for i in range(t.shape[0]):
        if t[i] == 5:
            if em[i] == 0. and ep[i] != 0.:
                ep[i] = em[i] / 3
            else:
                em[i] = ep[i] * 3
        elif em[i] == 0. and ep[i] != 0.:
            em[i] = 2. * ep[i] / (1. + ep[i] * ep[i])
        elif em[i] == 0. and ep[i] == 0.:
            ep[i] = 0.00001
        else:
            ep[i] = (1. - np.sqrt(1 - em[i] * em[i])) / em[i]
    return b0
