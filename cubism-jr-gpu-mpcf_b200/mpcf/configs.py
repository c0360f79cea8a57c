"""The five benchmark workloads: bubble clouds in a stiffened-gas liquid.

Material data: liquid gamma=6.59, pc=4096, rho=1000, p=100 (p=1000 in the
precision study); gas gamma=1.4, pc=0, rho=1, p=0.0234.  Interface
tanh-smoothed over 1.5 cells, velocity noise U(-1e-3, 1e-3), absorbing
boundaries, CFL 0.3.  Bubble centres uniform in [0.2, 0.8]^3 (times the
domain extent), seeded rejection sampling of non-overlapping spheres.
Synthetic inputs: no dataset is involved.
"""
import numpy as np

from ._lib import IcParams
from .solver import bubbles as _place

CFL = 0.3


def ic_params(p_liquid=100.0, seed=1234):
    return IcParams(rho_l=1000.0, p_l=p_liquid, gamma_l=6.59, pc_l=4096.0,
                    rho_g=1.0, p_g=0.0234, gamma_g=1.4, pc_g=0.0,
                    noise=1e-3, width=1.5, seed=seed)


def extents(dims):
    m = max(dims)
    return tuple(d / m for d in dims)


def config(name, seed=1234, placer=None):
    """Return dict(dims=[...], bubbles=[array], params=IcParams, steps, precision, ...).

    ``placer(seed, n, rmin, rmax, lo, hi)`` places the bubbles (default: the
    library's seeded rejection sampling, ``mpcf_bubbles``); any placer with
    the same rules gives the same workload."""
    _bubbles = placer or _place
    if name == "c1_64":
        dims = [(64, 64, 64)]
        bub = [np.array([[0.5, 0.5, 0.5, 0.15]])]
        return dict(name=name, dims=dims, bubbles=bub, params=ic_params(100.0, seed), steps=1,
                    precision="fp32_ref", desc="64^3, one bubble R=0.15 at the centre, 1 step")
    if name == "c2_256":
        dims = [(256, 256, 256)]
        bub = [_bubbles(seed, 50, 0.02, 0.06)]
        return dict(name=name, dims=dims, bubbles=bub, params=ic_params(100.0, seed), steps=100,
                    precision="fp32", desc="256^3, 50 bubbles R~U[0.02,0.06], 100 steps")
    if name == "c3_512":
        dims = [(512, 512, 512)]
        bub = [_bubbles(seed, 200, 0.02, 0.06)]
        return dict(name=name, dims=dims, bubbles=bub, params=ic_params(1000.0, seed), steps=20,
                    precision="mixed", desc="512^3, 200 bubbles R~U[0.02,0.06], liquid p=1000, 20 steps")
    if name == "c3_slab128":
        # the lower quarter of configuration 3's domain (512 x 512 x 128
        # cells, its cloud and liquid): a few-GB case of the same kernel and
        # tiling for hardware-counter captures
        dims = [(512, 512, 128)]
        bub = [_bubbles(seed, 200, 0.02, 0.06)]
        return dict(name=name, dims=dims, bubbles=bub, params=ic_params(1000.0, seed), steps=20,
                    precision="mixed", desc="512x512x128, the lower quarter of the 512^3 200-bubble cloud, liquid p=1000")
    if name == "c4_ensemble":
        rng = np.random.default_rng(seed)
        edges = (32, 48, 64, 96, 128)
        dims, bub = [], []
        for d in range(64):
            dd = tuple(int(e) for e in rng.choice(edges, size=3))
            dims.append(dd)
            ext = extents(dd)
            nb = int(rng.integers(1, 9))
            edge = min(ext)
            lo = tuple(0.2 * e for e in ext)
            hi = tuple(0.8 * e for e in ext)
            bub.append(_bubbles(seed + 17 * d + 1, nb, 0.05 * edge, 0.2 * edge, lo, hi))
        return dict(name=name, dims=dims, bubbles=bub, params=ic_params(100.0, seed), steps=50,
                    precision="mixed", desc="64 domains, edges in {32,48,64,96,128}, 1-8 bubbles each, 50 steps")
    if name == "c5_1024":
        dims = [(1024, 1024, 1024)]
        bub = [_bubbles(seed, 1000, 0.005, 0.02)]
        return dict(name=name, dims=dims, bubbles=bub, params=ic_params(100.0, seed), steps=10,
                    precision="mixed", desc="1024^3, 1000 bubbles R~U[0.005,0.02], 10 steps")
    raise KeyError(name)


def small_cloud(dims, nb=3, seed=7, p_liquid=100.0):
    """A small cloud for tests of any domain shape."""
    ext = extents(dims)
    edge = min(ext)
    lo = tuple(0.2 * e for e in ext)
    hi = tuple(0.8 * e for e in ext)
    return ic_params(p_liquid, seed), _place(seed, nb, 0.08 * edge, 0.2 * edge, lo, hi)
