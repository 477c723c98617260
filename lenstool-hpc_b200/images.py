"""Multiple-image systems: the strong-lensing constraints of the chi2 path.

A system is a set of observed images of one source, with the source's lens efficiency
dr = D_LS/D_OS (the reference's galaxy.dr, src/structure_hpc.hpp:167-177).  Images are
stored concatenated, system by system, as in the reference's image arrays
(src/chi_CPU_barycenter.cpp:180-214 walks them with a running index).

`generate_systems` makes the synthetic constraints of the delensing + chi2 workload:
seeded sources near the lens centre, their images found by forward ray-shooting through
the true model (barycentric delensing on a fine grid, the same inversion the chi2 uses),
kept when a source has 3 to 5 images, plus Gaussian position noise.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class ImageSystems:
    nimg: np.ndarray                  # int32 [nsys], images per system
    x: np.ndarray                     # float64 [sum(nimg)], observed image positions (arcsec)
    y: np.ndarray
    dr: np.ndarray                    # float64 [nsys], D_LS/D_OS of each system's source
    source_x: np.ndarray = field(default=None)  # true source positions (generation only)
    source_y: np.ndarray = field(default=None)

    @property
    def nsys(self) -> int:
        return int(self.nimg.shape[0])

    @property
    def nimages(self) -> int:
        return int(self.nimg.sum())

    def contiguous(self) -> "ImageSystems":
        return ImageSystems(np.ascontiguousarray(self.nimg, np.int32), np.ascontiguousarray(self.x, np.float64),
                            np.ascontiguousarray(self.y, np.float64), np.ascontiguousarray(self.dr, np.float64),
                            self.source_x, self.source_y)


def generate_systems(delense, nsys: int, seed: int, dr: float = 0.6, centre=(0., 0.), source_radius: float = 6.,
                     min_images: int = 3, max_images: int = 5, noise: float = 0.05, max_draws: int = 20000,
                     batch: int = 64) -> ImageSystems:
    """Draw sources uniformly in a disc of `source_radius` around `centre` (numpy PCG64,
    `seed`) until `nsys` of them have between min_images and max_images images.

    delense(bx, by, dr) -> (nfound[k], fx[k, m], fy[k, m]): the predicted images of k
    sources through the true model (e.g. the library's lt_delense on a fine grid)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    xs, ys, nimg, sx, sy = [], [], [], [], []
    draws = 0
    while len(nimg) < nsys and draws < max_draws:
        r = source_radius * np.sqrt(rng.uniform(0., 1., batch))
        t = rng.uniform(0., 2. * np.pi, batch)
        bx = centre[0] + r * np.cos(t)
        by = centre[1] + r * np.sin(t)
        draws += batch
        nf, fx, fy = delense(bx, by, np.full(batch, dr))
        for k in range(batch):
            if len(nimg) == nsys:
                break
            if min_images <= nf[k] <= max_images:
                nimg.append(int(nf[k]))
                xs.append(fx[k, :nf[k]] + noise * rng.standard_normal(nf[k]))
                ys.append(fy[k, :nf[k]] + noise * rng.standard_normal(nf[k]))
                sx.append(bx[k])
                sy.append(by[k])
    if len(nimg) < nsys:
        raise RuntimeError(f"only {len(nimg)} of {nsys} sources gave {min_images}-{max_images} images "
                           f"in {draws} draws")
    return ImageSystems(np.asarray(nimg, np.int32), np.concatenate(xs), np.concatenate(ys),
                        np.full(nsys, dr), np.asarray(sx), np.asarray(sy))
