"""Seeded synthetic basins (meshes, layers, forcing, initial state).

SHYFEM reads a basin from a `.bas` file made by `shypre` from a `.grd` mesh and a
`.str` parameter file (src/shyfem/shyfem_subs.f90:326-327).  No dataset ships
with the reference for the semi-implicit step, so every workload here is a
seeded synthetic basin of the named shape:

* `channel_case`   -- 2D barotropic tidal channel, 61 x 13 nodes, 10 km x 2 km,
                      M2 elevation on the x=0 boundary, quadratic friction.
* `basin3d_case`   -- 3D baroclinic basin, ~20k nodes on 50 km x 30 km, 20
                      z-layers 1..5 m thick, Gaussian-bump bathymetry 5..60 m,
                      T/S linear in depth plus seeded noise, 10 m/s wind, M2 0.3 m.
* `shelf_case`     -- tidal shelf on z-layers with three 1 m surface layers
                      and an M2 of 1.5 m, for z-adaptive layers (nzadapt).
* `ensemble_cases` -- independent basins with log-uniform node counts.

All arrays use the reference's layouts: Fortran column-major `(nlv, nel)` /
`(nlv, nkn)` stored here as C arrays `[nel][nlv]` (layer index fastest), node
and element numbers 1-based in `nen3v` like `basin :: nen3v(3,nel)`.

The structure of a case follows the reference's module state:
`basin` (nkn, nel, nen3v, xgv, ygv, hm3v), `levels` (nlv, hlv, hldv, ilhv,
ilhkv), boundary tables (`bnd_admin.f90`: ibtyp=1 level boundaries with
`ampli/period/phase/zref`), forcing (`mod_meteo`: tauxnv, tauynv, ppv) and
parameters under their `.str` names (`def_para.f90`).
"""
from __future__ import annotations

import math
import numpy as np

M2_PERIOD = 44714.0   # s, principal lunar semidiurnal
S2_PERIOD = 43200.0   # s, principal solar semidiurnal

# default parameters under their SHYFEM names (src/shyfem/def_para.f90)
DEFAULT_PARAMS = dict(
    dt=60.0,            # time step [s]
    azpar=0.5, ampar=0.5, afpar=0.5,   # def_para.f90:666-668
    atpar=1.0, adpar=1.0, aapar=1.0,   # def_para.f90:684-686
    grav=9.81, rowass=1025.0,          # def_para.f90:782-784
    vismol=1.0e-6, difmol=1.0e-6,      # def_para.f90:993-995
    ireib=5, czdef=2.5e-3,             # quadratic friction, cd const (chezy.f90:330)
    hzoff=0.05,                        # def_para.f90:745
    ahpar=0.0,                         # horizontal viscosity (def_para.f90:1023)
    ibarcl=0,                          # baroclinic terms (def_para.f90:1132)
    ilin=1,                            # linear momentum (def_para.f90:584)
    rstol=1.0,                         # transport Courant limit (def_para.f90:1055)
    thpar=0.0, shpar=0.0, chpar=0.0,   # horizontal diffusivity of T, S, tracers
    itemp=0, isalt=0, nconz=0,
    icor=0,
)


def _smooth_field(x, y, rng, n_modes=6, scale=1.0):
    """Sum of seeded low-wavenumber sinusoids normalised to [-scale, scale]."""
    lx = x.max() - x.min() + 1e-9
    ly = y.max() - y.min() + 1e-9
    f = np.zeros_like(x)
    for _ in range(n_modes):
        kx = rng.integers(1, 4) * math.pi / lx
        ky = rng.integers(1, 4) * math.pi / ly
        ph1, ph2 = rng.uniform(0, 2 * math.pi, 2)
        f += rng.uniform(0.5, 1.0) * np.sin(kx * x + ph1) * np.cos(ky * y + ph2)
    m = np.abs(f).max()
    return f * (scale / m if m > 0 else 0.0)


def structured_triangles(nx, ny, lx, ly, jitter, seed):
    """Regular nx x ny node grid, interior nodes jittered by +-jitter*spacing,
    each quad split on a seeded random diagonal.  Nodes are numbered row by
    row (x fastest), which keeps the sparsity band narrow like `shypre`'s
    bandwidth-reducing renumbering.  Returns x, y, nen3v (1-based, (3,nel)
    counter-clockwise), and the node (i, j) grid indices."""
    rng = np.random.default_rng(seed)
    dx = lx / (nx - 1)
    dy = ly / (ny - 1)
    jj, ii = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    x = (ii * dx).astype(np.float64).ravel()
    y = (jj * dy).astype(np.float64).ravel()
    interior = ((ii > 0) & (ii < nx - 1) & (jj > 0) & (jj < ny - 1)).ravel()
    x[interior] += rng.uniform(-jitter, jitter, interior.sum()) * dx
    y[interior] += rng.uniform(-jitter, jitter, interior.sum()) * dy
    node = lambda i, j: j * nx + i
    tris = []
    diag = rng.integers(0, 2, size=(ny - 1, nx - 1))
    for j in range(ny - 1):
        for i in range(nx - 1):
            a, b, c, d = node(i, j), node(i + 1, j), node(i + 1, j + 1), node(i, j + 1)
            if diag[j, i]:
                tris.append((a, b, c)); tris.append((a, c, d))
            else:
                tris.append((a, b, d)); tris.append((b, c, d))
    nen3v = np.asarray(tris, dtype=np.int32) + 1     # 1-based like the reference
    return x, y, nen3v, ii.ravel(), jj.ravel()


def z_layers(thick):
    """hldv (nominal thickness) and hlv (bottom depth of each layer)."""
    hldv = np.asarray(thick, dtype=np.float64)
    hlv = np.cumsum(hldv)
    return hlv, hldv


def layer_counts(nen3v, hm3v, hlv, hldv, nkn):
    """Layers per element (`ilhv`) and per node (`ilhkv`).  The bottom layer
    of an element must have positive thickness at every vertex
    (`hlast = htot - hlv(lmax-1) > 0`, elems_dealing.f90:1045-1047), and a
    bottom layer thinner than a quarter of its nominal thickness is merged
    into the layer above (the intent of `hlvmin`, def_para.f90:942)."""
    nlv = len(hlv)
    hmin = hm3v.min(axis=1)
    lmax = 1 + np.searchsorted(hlv, hmin, side="left")
    lmax = np.minimum(lmax, nlv)
    for _ in range(2):
        hl_prev = np.where(lmax > 1, hlv[np.maximum(lmax - 2, 0)], 0.0)
        thin = (lmax > 1) & ((hmin - hl_prev) < 0.25 * hldv[lmax - 1])
        lmax = np.where(thin, lmax - 1, lmax)
    ilhv = lmax.astype(np.int32)
    ilhkv = np.zeros(nkn, dtype=np.int32)
    np.maximum.at(ilhkv, nen3v.ravel() - 1, np.repeat(ilhv, 3))
    return ilhv, ilhkv


def _finish(case):
    """Fill derived defaults shared by all cases."""
    nkn, nel, nlv = case["nkn"], case["nel"], case["nlv"]
    p = dict(DEFAULT_PARAMS)
    p.update(case.get("params", {}))
    case["params"] = p
    case.setdefault("czv", np.full(nel, p["czdef"], np.float32))
    case.setdefault("fcorv", np.zeros(nel, np.float32))
    case.setdefault("visv", np.zeros((nkn, nlv + 1), np.float32))
    case.setdefault("difv", np.zeros((nkn, nlv + 1), np.float32))
    case.setdefault("tauxnv", np.zeros(nkn, np.float32))
    case.setdefault("tauynv", np.zeros(nkn, np.float32))
    case.setdefault("ppv", np.zeros(nkn, np.float32))
    case.setdefault("rqv", np.zeros(nkn, np.float32))
    case.setdefault("znv", np.zeros(nkn, np.float32))
    case.setdefault("utlnv", np.zeros((nel, nlv), np.float32))
    case.setdefault("vtlnv", np.zeros((nel, nlv), np.float32))
    case.setdefault("tempv", np.zeros((nkn, nlv), np.float32))
    case.setdefault("saltv", np.zeros((nkn, nlv), np.float32))
    nc = p["nconz"]
    case.setdefault("conzv", np.zeros((max(nc, 0), nkn, nlv), np.float32))
    for k in ("hlv", "hldv", "hm3v", "xgv", "ygv"):
        case[k] = np.ascontiguousarray(case[k], dtype=np.float32)
    case["nen3v"] = np.ascontiguousarray(case["nen3v"], dtype=np.int32)
    return case


def channel_case(nx=61, ny=13, lx=10.0e3, ly=2.0e3, seed=1, dt=60.0,
                 ampli=0.5, depth=10.0, ddepth=2.0):
    """2D barotropic tidal channel (one layer, FP64 reference run)."""
    x, y, nen3v, ii, jj = structured_triangles(nx, ny, lx, ly, 0.2, seed)
    rng = np.random.default_rng(seed + 101)
    hk = depth + _smooth_field(x, y, rng, scale=ddepth)
    nkn, nel = x.size, nen3v.shape[0]
    hm3v = hk[nen3v - 1]
    hlv, hldv = np.array([1.0e4]), np.array([1.0e4])   # one layer covering all depths
    ilhv = np.ones(nel, np.int32)
    ilhkv = np.ones(nkn, np.int32)
    bnd = np.zeros(nkn, np.int32)
    bnd[ii == 0] = 1                                  # ibtyp=1 level boundary at x=0
    tide = np.array([[[ampli, M2_PERIOD, 0.0, 0.0]]], np.float32)   # (nbnd, ntide, 4)
    case = dict(name=f"channel2d_{nkn}", nkn=nkn, nel=nel, nlv=1, nen3v=nen3v,
                xgv=x, ygv=y, hm3v=hm3v, hlv=hlv, hldv=hldv, ilhv=ilhv, ilhkv=ilhkv,
                bnd_index=bnd, tide=tide, seed=seed,
                params=dict(dt=dt))
    return _finish(case)


def basin3d_case(nkn_target=20000, lx=50.0e3, ly=30.0e3, seed=2, dt=120.0,
                 nlv=20, ampli=0.3, wind=10.0, baroclinic=True, ts=True):
    """3D baroclinic basin with z-layers, wind, M2 boundary and T/S."""
    ny = max(3, int(round(math.sqrt(nkn_target * ly / lx))))
    nx = max(3, int(round(nkn_target / ny)))
    x, y, nen3v, ii, jj = structured_triangles(nx, ny, lx, ly, 0.2, seed)
    rng = np.random.default_rng(seed + 202)
    nkn, nel = x.size, nen3v.shape[0]
    # Gaussian-bump bathymetry spanning 5..60 m
    h = np.zeros(nkn)
    for _ in range(8):
        cx, cy = rng.uniform(0, lx), rng.uniform(0, ly)
        s = rng.uniform(0.1, 0.3) * min(lx, ly)
        h += rng.uniform(0.3, 1.0) * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * s * s))
    h = 5.0 + 55.0 * (h - h.min()) / (h.max() - h.min())
    thick = np.linspace(1.0, 5.0, nlv)
    thick *= 60.0 / thick.sum()
    hlv, hldv = z_layers(thick)
    hlv[-1] = max(hlv[-1], h.max() + 1.0)
    hm3v = h[nen3v - 1]
    ilhv, ilhkv = layer_counts(nen3v, hm3v, hlv, hldv, nkn)
    bnd = np.zeros(nkn, np.int32)
    bnd[ii == 0] = 1
    tide = np.array([[[ampli, M2_PERIOD, 0.0, 0.0]]], np.float32)
    params = dict(dt=dt, ibarcl=1 if baroclinic else 0,
                  itemp=1 if ts else 0, isalt=1 if ts else 0)
    # uniform wind stress, normalised by water density as in mod_meteo (tauxnv = tau/rho0)
    rhoair, cd = 1.225, 2.5e-3
    taux = rhoair / 1025.0 * cd * wind * wind
    zc = np.zeros((nkn, nlv))
    # layer-centre depth at each node for T/S initialisation
    zc[:] = (hlv - 0.5 * hldv)[None, :]
    noise = np.random.default_rng(seed + 303)
    tempv = 20.0 - 10.0 * zc / 60.0 + 0.2 * noise.standard_normal((nkn, nlv))
    saltv = 30.0 + 8.0 * zc / 60.0 + 0.2 * noise.standard_normal((nkn, nlv))
    case = dict(name=f"basin3d_{nkn}x{nlv}", nkn=nkn, nel=nel, nlv=nlv, nen3v=nen3v,
                xgv=x, ygv=y, hm3v=hm3v, hlv=hlv, hldv=hldv, ilhv=ilhv, ilhkv=ilhkv,
                bnd_index=bnd, tide=tide, seed=seed, params=params,
                tauxnv=np.full(nkn, taux, np.float32),
                tempv=tempv.astype(np.float32), saltv=saltv.astype(np.float32))
    return _finish(case)


def lagoon_case(nkn_target=3000, lx=12.0e3, ly=6.0e3, seed=7, dt=30.0, nlv=30, ntracer=3,
                hmin=1.5, hmax=30.0):
    """Tidal lagoon on pure sigma layers (the large-lagoon config's vertical
    grid): a jittered triangle mesh deepening from `hmin` at the closed end
    to `hmax` at the open boundary with seeded smooth relief, `nlv` equal
    sigma layers (hlv = -l/nlv, nsigma = nlv), an M2 + S2 level boundary of
    0.8 m total amplitude, and `ntracer` passive tracers starting from
    seeded Gaussian patches.  Barotropic (sigma layers without baroclinic
    terms)."""
    ny = max(3, int(round(math.sqrt(nkn_target * ly / lx))))
    nx = max(3, int(round(nkn_target / ny)))
    x, y, nen3v, ii, jj = structured_triangles(nx, ny, lx, ly, 0.2, seed)
    rng = np.random.default_rng(seed + 404)
    nkn, nel = x.size, nen3v.shape[0]
    ramp = 1.0 - x / lx                               # deep at x = 0 (open boundary)
    h = hmin + (hmax - hmin) * ramp ** 1.5 + _smooth_field(x, y, rng, scale=0.3 * hmin)
    h = np.maximum(h, hmin)
    hm3v = h[nen3v - 1]
    hlv = -np.arange(1, nlv + 1, dtype=np.float64) / nlv
    hldv = np.full(nlv, -1.0 / nlv)
    ilhv = np.full(nel, nlv, np.int32)
    ilhkv = np.full(nkn, nlv, np.int32)
    bnd = np.zeros(nkn, np.int32)
    bnd[ii == 0] = 1
    tide = np.array([[[0.5, M2_PERIOD, 0.0, 0.0], [0.3, S2_PERIOD, 3600.0, 0.0]]], np.float32)
    conz = np.zeros((ntracer, nkn, nlv), np.float32)
    for t in range(ntracer):
        cx, cy = rng.uniform(0.3 * lx, 0.9 * lx), rng.uniform(0.2 * ly, 0.8 * ly)
        s = rng.uniform(0.05, 0.15) * lx
        conz[t] = (10.0 * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * s * s)))[:, None]
    params = dict(dt=dt, nsigma=nlv, hsigma=10000.0, nconz=ntracer, chpar=0.0)
    case = dict(name=f"lagoon_sigma_{nkn}x{nlv}", nkn=nkn, nel=nel, nlv=nlv, nen3v=nen3v,
                xgv=x, ygv=y, hm3v=hm3v, hlv=hlv, hldv=hldv, ilhv=ilhv, ilhkv=ilhkv,
                bnd_index=bnd, tide=tide, seed=seed, params=params, conzv=conz,
                tauxnv=np.full(nkn, 1.0e-4, np.float32))
    return _finish(case)


def hybrid_lagoon_case(nkn_target=900, nsigma=6, hsigma=8.0, dz=3.0, seed=7, dt=30.0, ntracer=3,
                       hmin=1.5, hmax=30.0):
    """The lagoon on hybrid layers: `nsigma` equal sigma layers down to
    `hsigma`, z-layers of `dz` below (hlv(nsigma) = hsigma, as the
    reference's level set-up makes it, initialize.f90:550-558).  Elements
    deeper than hsigma on average get a flat bottom at their mean depth
    (flatten_hm3v, depth_util.f90:603-629); an element has the nsigma
    sigma layers, plus the z-layers down to its depth when it is deeper than
    hsigma (set_ilhv, initialize.f90:787-836)."""
    c = lagoon_case(nkn_target=nkn_target, seed=seed, dt=dt, nlv=nsigma, ntracer=ntracer,
                    hmin=hmin, hmax=hmax)
    nkn, nel = c["nkn"], c["nel"]
    hm3v = np.asarray(c["hm3v"], np.float64).copy()
    hev = hm3v.mean(axis=1)
    deep = hev > hsigma
    hm3v[deep] = hev[deep][:, None]
    nz = int(math.ceil((hev.max() - hsigma) / dz)) if deep.any() else 0
    nlv = nsigma + nz
    hlv = np.r_[-np.arange(1, nsigma, dtype=np.float64) / nsigma, hsigma, hsigma + dz * np.arange(1, nz + 1)]
    hldv = np.r_[np.full(nsigma, -1.0 / nsigma), np.full(nz, dz)]
    ilhv = np.full(nel, nsigma, np.int32)
    for e in np.nonzero(deep)[0]:
        ilhv[e] = nsigma + int(np.argmax(hlv[nsigma:] >= hev[e])) + 1
    ilhkv = np.zeros(nkn, np.int32)
    np.maximum.at(ilhkv, c["nen3v"].ravel() - 1, np.repeat(ilhv, 3))
    conz = np.repeat(c["conzv"][:, :, :1], nlv, axis=2)
    c.update(name=f"lagoon_hybrid_{nkn}x{nlv}", nlv=nlv, hm3v=hm3v.astype(np.float32), hlv=hlv, hldv=hldv,
             ilhv=ilhv, ilhkv=ilhkv, conzv=conz)
    c["params"] = dict(c["params"], nsigma=nsigma, hsigma=hsigma)
    for k in ("visv", "difv", "tempv", "saltv", "znv", "utlnv", "vtlnv"):
        c.pop(k, None)
    return _finish(c)


def flat_case(nx=41, ny=9, lx=8.0e3, ly=1.6e3, seed=9, dt=60.0, nlv=1, ampli=1.0,
              hdeep=3.0, hshallow=-0.6):
    """Tidal flat for wetting and drying: a channel deepening linearly from
    `hshallow` (negative: land above the rest level) at the closed end to
    `hdeep` at the open boundary, M2 of `ampli`, `nlv` z-layers: the first
    `ampli` + 0.5 m thick (a surface layer must stay thicker than the tide
    takes away), then 1 m, the last one reaching the bottom.  The flat
    dries at low water and floods at high water (setweg)."""
    x, y, nen3v, ii, jj = structured_triangles(nx, ny, lx, ly, 0.2, seed)
    rng = np.random.default_rng(seed + 505)
    nkn, nel = x.size, nen3v.shape[0]
    h = hdeep + (hshallow - hdeep) * x / lx + _smooth_field(x, y, rng, scale=0.15)
    hm3v = h[nen3v - 1]
    if nlv == 1:
        hlv, hldv = np.array([1.0e4]), np.array([1.0e4])
        ilhv = np.ones(nel, np.int32)
        ilhkv = np.ones(nkn, np.int32)
    else:
        hlv, hldv = z_layers(np.r_[ampli + 0.5, np.ones(nlv - 1)])
        hlv[-1] = max(hlv[-1], h.max() + 1.0)
        ilhv, ilhkv = layer_counts(nen3v, np.maximum(hm3v, 0.1), hlv, hldv, nkn)
    bnd = np.zeros(nkn, np.int32)
    bnd[ii == 0] = 1
    tide = np.array([[[ampli, M2_PERIOD, 0.0, 0.0]]], np.float32)   # from the rest level, rising
    case = dict(name=f"flat_{nkn}x{nlv}", nkn=nkn, nel=nel, nlv=nlv, nen3v=nen3v,
                xgv=x, ygv=y, hm3v=hm3v, hlv=hlv, hldv=hldv, ilhv=ilhv, ilhkv=ilhkv,
                bnd_index=bnd, tide=tide, seed=seed, params=dict(dt=dt, wetdry=1))
    return _finish(case)


def shelf_case(nkn_target=1500, lx=20.0e3, ly=8.0e3, seed=11, dt=60.0, nzadapt=3, ampli=1.5,
               hmin=5.0, hmax=40.0, ntracer=1, closed=False, wind=8.0):
    """Tidal shelf on z-layers with thin surface layers for z-adaptive
    layers (nzadapt, zadaptutil.f90): three 1 m layers on top, then 2, 3,
    5, 8, 10 and 12 m; depth rising from `hmin` at the closed end to
    `hmax` at the open boundary; M2 of `ampli` that falls first (phase of
    half a period), so the level drops below the first layers' bottoms
    within a quarter period: plain z-layers (nzadapt = 0) lose their first
    layer there (setdepth stops), z-adaptive ones stretch.  `closed`
    removes the boundary (a wind-driven closed basin); `ntracer` passive
    tracers start as a front across the shelf."""
    ny = max(3, int(round(math.sqrt(nkn_target * ly / lx))))
    nx = max(3, int(round(nkn_target / ny)))
    x, y, nen3v, ii, jj = structured_triangles(nx, ny, lx, ly, 0.2, seed)
    rng = np.random.default_rng(seed + 606)
    nkn, nel = x.size, nen3v.shape[0]
    h = hmax + (hmin - hmax) * x / lx + _smooth_field(x, y, rng, scale=1.0)
    hm3v = h[nen3v - 1]
    hlv, hldv = z_layers([1.0, 1.0, 1.0, 2.0, 3.0, 5.0, 8.0, 10.0, 12.0])
    hlv[-1] = max(hlv[-1], h.max() + 1.0)
    nlv = len(hlv)
    ilhv, ilhkv = layer_counts(nen3v, hm3v, hlv, hldv, nkn)
    bnd = np.zeros(nkn, np.int32)
    if not closed:
        bnd[ii == 0] = 1
    tide = np.array([[[ampli, M2_PERIOD, 0.5 * M2_PERIOD, 0.0]]], np.float32)
    rhoair, cd = 1.225, 2.5e-3
    tau = rhoair / 1025.0 * cd * wind * wind
    conzv = np.zeros((ntracer, nkn, nlv), np.float32)
    for t in range(ntracer):
        front = 0.5 * (1.0 + np.tanh((x - lx * (0.3 + 0.2 * t)) / (0.05 * lx)))
        conzv[t] = (front[:, None] * (1.0 + 0.1 * np.arange(nlv))[None, :]).astype(np.float32)
    case = dict(name=f"shelf_{nkn}x{nlv}_za{nzadapt}", nkn=nkn, nel=nel, nlv=nlv, nen3v=nen3v,
                xgv=x, ygv=y, hm3v=hm3v, hlv=hlv, hldv=hldv, ilhv=ilhv, ilhkv=ilhkv,
                bnd_index=bnd, tide=tide, seed=seed,
                params=dict(dt=dt, nzadapt=nzadapt, nconz=ntracer),
                tauxnv=np.full(nkn, 0.6 * tau, np.float32), tauynv=np.full(nkn, 0.8 * tau, np.float32),
                conzv=conzv)
    return _finish(case)


def seiche_case(lx=50.0, ly=10.0, nx=21, ny=5, depth=25.0, nlv=10, ampli=0.01, dt=0.1, inohyd=1,
                seed=13, jitter=0.1):
    """Standing wave in a deep closed basin, for the non-hydrostatic
    pressure (nohydro.f90): a flat `depth` m basin `lx` m long, `nlv`
    equal z-layers, no friction, no wind, linear momentum, the initial
    level `ampli` cos(pi x / lx).  With k = pi / lx and k H near pi/2 the
    hydrostatic period 2 pi / (k sqrt(g H)) and the non-hydrostatic one
    2 pi / sqrt(g k tanh(k H)) differ by a quarter."""
    x, y, nen3v, ii, jj = structured_triangles(nx, ny, lx, ly, jitter, seed)
    x[ii == 0] = 0.0
    x[ii == nx - 1] = lx
    nkn, nel = x.size, nen3v.shape[0]
    hm3v = np.full((nel, 3), depth, np.float32)
    hlv, hldv = z_layers(np.full(nlv, depth / nlv))
    hlv[-1] = depth + 1.0
    hldv[-1] = hlv[-1] - (hlv[-2] if nlv > 1 else 0.0)
    ilhv, ilhkv = layer_counts(nen3v, hm3v, hlv, hldv, nkn)
    znv = (ampli * np.cos(np.pi * x / lx)).astype(np.float32)
    case = dict(name=f"seiche_{nkn}x{nlv}_nh{inohyd}", nkn=nkn, nel=nel, nlv=nlv, nen3v=nen3v,
                xgv=x, ygv=y, hm3v=hm3v, hlv=hlv, hldv=hldv, ilhv=ilhv, ilhkv=ilhkv,
                bnd_index=np.zeros(nkn, np.int32), tide=np.zeros((0, 1, 4), np.float32), seed=seed,
                params=dict(dt=dt, ireib=0, inohyd=inohyd), znv=znv)
    return _finish(case)


def nh_basin_case(nkn_target=1500, lx=300.0, ly=150.0, seed=2, dt=0.5, nlv=12, hmin=5.0, hmax=30.0,
                  sigma=True, wind=10.0, ts=True):
    """Small closed basin for the non-hydrostatic pressure: `lx` x `ly` m,
    Gaussian-bump bathymetry from `hmin` to `hmax` m, `nlv` sigma layers
    (or z-layers of 1 to 5 m), uniform wind, T/S linear in depth plus seeded
    noise (transported, no baroclinic terms), dt of half a second: the
    horizontal scale of the flow is the depth's, where the pressure
    matters."""
    c = basin3d_case(nkn_target=nkn_target, lx=lx, ly=ly, seed=seed, dt=dt, nlv=nlv, ampli=0.0, wind=wind,
                     baroclinic=False, ts=ts)
    c["bnd_index"][:] = 0
    c["tide"] = np.zeros((0, 1, 4), np.float32)
    h = c["hm3v"].astype(np.float64)
    c["hm3v"] = (hmin + (h - 5.0) * (hmax - hmin) / 55.0).astype(np.float32)
    if sigma:
        c["hlv"] = (-np.arange(1, nlv + 1) / nlv).astype(np.float32)
        c["hldv"] = np.full(nlv, -1.0 / nlv, np.float32)
        c["ilhv"][:] = nlv
        c["ilhkv"][:] = nlv
        c["params"] = dict(c["params"], nsigma=nlv)
    else:
        hlv, hldv = z_layers(np.linspace(1.0, 5.0, nlv) * hmax / np.linspace(1.0, 5.0, nlv).sum())
        hlv[-1] = hmax + 1.0
        c["hlv"], c["hldv"] = hlv.astype(np.float32), hldv.astype(np.float32)
        c["ilhv"], c["ilhkv"] = layer_counts(c["nen3v"], c["hm3v"], hlv, hldv, c["nkn"])
    c["params"] = dict(c["params"], inohyd=1)
    c["name"] = f"nhbasin_{c['nkn']}x{nlv}_{'sigma' if sigma else 'z'}"
    return c


def stratified_basin_case(nkn_target=1500, lx=30.0e3, ly=15.0e3, nlv=12, sigma=True, hmin=5.0, hmax=60.0,
                          wind=0.0, noise=0.0, dt=60.0, seed=2):
    """Closed basin on sigma layers (or z-layers) over Gaussian bumps from
    `hmin` to `hmax` m, stably stratified: temperature 20 degC at the
    surface falling by 10 degC over 60 m of depth (plus seeded noise of
    `noise` degC), salinity 35, baroclinic pressure on, optional uniform
    wind.  At rest, a horizontal stratification over a sloping bottom is
    where sigma layers need the density gradient taken on horizontal
    surfaces (set_barocl_new_interface's bsigadjust)."""
    c = nh_basin_case(nkn_target=nkn_target, lx=lx, ly=ly, seed=seed, dt=dt, nlv=nlv, hmin=hmin, hmax=hmax,
                      sigma=sigma, wind=wind, ts=True)
    c["params"] = dict(c["params"], inohyd=0, ibarcl=1)
    nkn = c["nkn"]
    hk = np.zeros(nkn)
    cnt = np.zeros(nkn)
    np.add.at(hk, c["nen3v"].ravel() - 1, c["hm3v"].ravel())
    np.add.at(cnt, c["nen3v"].ravel() - 1, 1)
    hk /= cnt
    if sigma:
        zc = (np.arange(nlv)[None, :] + 0.5) / nlv * hk[:, None]
    else:
        hlv, hld = c["hlv"].astype(float), c["hldv"].astype(float)
        zc = np.broadcast_to(hlv - 0.5 * hld, (nkn, nlv)).copy()
    rng = np.random.default_rng(seed + 404)
    c["tempv"] = (20.0 - 10.0 * zc / 60.0 + noise * rng.standard_normal((nkn, nlv))).astype(np.float32)
    c["saltv"] = np.full((nkn, nlv), 35.0, np.float32)
    c["name"] = f"stratified_{nkn}x{nlv}_{'sigma' if sigma else 'z'}"
    return c


def ensemble_member_case(nkn_target, aspect, seed, wind, dt=60.0, nlv=10, spacing=100.0,
                         ampli=0.5, depth=10.0, ddepth=2.0, top=2.0):
    """One member of the batched ensemble, made as the 2D channel is: a
    jittered triangle mesh of `spacing` (100 m) on a rectangle of the given
    aspect ratio, each quad split on a seeded diagonal, depth 10 m plus a
    seeded smooth perturbation of +-2 m, M2 of 0.5 m on the x = 0 boundary,
    quadratic friction; then `nlv` z-layers (a `top` m surface layer, wide
    enough for the tide and the wind set-down, 1 m layers below, the last
    one reaching the bottom) and a uniform wind of speed `wind` along x."""
    ny = max(3, int(round(math.sqrt(nkn_target / aspect))))
    nx = max(3, int(round(nkn_target / ny)))
    lx, ly = (nx - 1) * spacing, (ny - 1) * spacing
    x, y, nen3v, ii, jj = structured_triangles(nx, ny, lx, ly, 0.2, seed)
    rng = np.random.default_rng(seed + 101)
    hk = depth + _smooth_field(x, y, rng, scale=ddepth)
    nkn, nel = x.size, nen3v.shape[0]
    hm3v = hk[nen3v - 1]
    hlv, hldv = z_layers(np.r_[top, np.ones(nlv - 1)])
    hlv[-1] = max(hlv[-1], hk.max() + 1.0)
    hldv[-1] = hlv[-1] - hlv[-2]
    ilhv, ilhkv = layer_counts(nen3v, hm3v, hlv, hldv, nkn)
    bnd = np.zeros(nkn, np.int32)
    bnd[ii == 0] = 1
    tide = np.array([[[ampli, M2_PERIOD, 0.0, 0.0]]], np.float32)
    rhoair, cd = 1.225, 2.5e-3
    taux = rhoair / 1025.0 * cd * wind * abs(wind)
    case = dict(name=f"member_{nkn}x{nlv}", nkn=nkn, nel=nel, nlv=nlv, nen3v=nen3v,
                xgv=x, ygv=y, hm3v=hm3v, hlv=hlv, hldv=hldv, ilhv=ilhv, ilhkv=ilhkv,
                bnd_index=bnd, tide=tide, seed=seed, params=dict(dt=dt),
                tauxnv=np.full(nkn, taux, np.float32))
    return _finish(case)


def ensemble_cases(n, nkn_lo=5000, nkn_hi=100000, nlv=10, seed=4, dt=60.0, first=None, only=None):
    """The batched ensemble: `n` independent basins with node counts
    log-uniform in [nkn_lo, nkn_hi], each made like the 2D channel
    (`ensemble_member_case`: 100 m jittered mesh, depth 10 +- 2 m, M2 0.5 m)
    at a seeded aspect ratio in [2, 6], with 10 z-layers and a seeded wind
    of 10 m/s plus a perturbation of sigma 3 m/s.  `first` builds only the
    first members of the same ensemble, `only` the members of the given
    indices (in that order)."""
    draws = ensemble_draws(n, nkn_lo, nkn_hi, seed)
    idx = list(range(n if first is None else min(first, n))) if only is None else list(only)
    return [ensemble_member_case(draws[m][0], draws[m][1], seed * 1000 + m, draws[m][2], dt=dt, nlv=nlv)
            for m in idx]


def ensemble_draws(n, nkn_lo=5000, nkn_hi=100000, seed=4):
    """The seeded (node count, aspect ratio, wind speed) of each member."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nk = int(math.exp(rng.uniform(math.log(nkn_lo), math.log(nkn_hi))))
        aspect = rng.uniform(2.0, 6.0)
        wind = 10.0 + 3.0 * rng.standard_normal()
        out.append((nk, aspect, wind))
    return out


def serve_requests(n, rate_per_min=20.0, nkn_lo=2000, nkn_hi=200000, nlv=10, seed=5, dt=60.0,
                   horizon_steps=2880):
    """A forecast request stream: Poisson arrivals at `rate_per_min`, basins
    with log-uniform node counts, 10 z-layers, a 48 h horizon at dt = 60 s,
    and per-request seeded M2 boundary tides (amplitude 0.1..0.5 m, random
    phase) and winds (10 m/s, sigma 3 m/s).  Aspect ratios 1.5..3 keep the
    largest basins well short of quarter-wave resonance with M2, so the
    2 m surface layer stays wet over the horizon.  Returns [(arrival_s,
    case, nsteps)]."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for m in range(n):
        t += rng.exponential(60.0 / rate_per_min)
        nk = int(math.exp(rng.uniform(math.log(nkn_lo), math.log(nkn_hi))))
        aspect = rng.uniform(1.5, 3.0)
        ly = 2.0e3 * math.sqrt(nk / 793.0)
        c = basin3d_case(nkn_target=nk, lx=aspect * ly, ly=ly, seed=seed * 1000 + m, dt=dt, nlv=nlv,
                         ampli=float(rng.uniform(0.1, 0.5)), wind=10.0 + 3.0 * rng.standard_normal(),
                         baroclinic=False, ts=False)
        c["tide"][..., 2] = float(rng.uniform(0.0, M2_PERIOD))   # phase [s]
        c["name"] = f"request{m}_{c['nkn']}"
        out.append((t, c, horizon_steps))
    return out
