"""Seeded synthetic SHOC windows for the tracer-transport workloads.

A window is built the way SHOC's preprocessor lays it out (sparse wet cells,
lateral ghosts, sediment cells; see csrc/shoc_grid.c), and given

  * face volume fluxes u1flux3d / u2flux3d from a depth-integrated transport
    streamfunction (so every column's integrated divergence is zero to
    round-off and the free surface stays put), plus a seeded baroclinic part
    whose depth integral over each face is zero,
  * face velocities u1 / u2 = flux / (face thickness * face length),
  * w from continuity (the vel_w_update restatement in csrc/shoc_grid.c),
  * Kz at cell bottom faces and initial tracer fields.

Workloads (sizes from the transport benchmark description):

  basin64    64x64, 1 km, 20 layers, depth 10-50 m, no land, 1 Gaussian
             tracer, solid-body-like rotation <= 0.5 m/s, Kz 1e-2 -> 1e-5
  drop512    512x512, 40 layers, depth 2-200 m, 30% land, 10 log-normal
             tracers, streamfunction flow <= 1.5 m/s, Kz log-uniform
             1e-6..1e-1
  batch2048  2048x1024 curvilinear (cells 200 m - 2 km), 50 layers, 35% land,
             24 tracers at magnitudes 1e-3..1e2
  stiff2048  batch2048 with 0.5 m surface layers and Kz 1e-6..1
  small      a few-thousand-cell basin with land for quick parity tests

All random numbers come from numpy's PCG64 with the seed recorded in the case.
"""
import ctypes as C
import os

import numpy as np

from . import _abi
from ._abi import Geom, dptr, iptr

_HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None


class _GridSpec(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("layers", _abi.DP), ("bathy", _abi.DP), ("land", C.POINTER(C.c_ubyte)),
        ("h1acell", _abi.DP), ("h2acell", _abi.DP), ("h1au1", _abi.DP),
        ("h2au1", _abi.DP), ("h1au2", _abi.DP), ("h2au2", _abi.DP),
    ]


class _Grid(C.Structure):
    _fields_ = [
        ("geom", Geom),
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("nwet", C.c_int), ("ncol", C.c_int), ("nghost", C.c_int),
        ("kbot", _abi.IP), ("map_top", _abi.IP), ("is_wet", _abi.IP),
    ] + [(n, _abi.IP) for n in (
        "w3_t", "w2_t", "bot_t", "w3_e1", "w3_e2", "xp1", "xm1", "yp1", "ym1",
        "zp1", "zm1", "m2d", "s2i", "s2j", "s2k", "bpt", "bin")] + [
        (n, _abi.DP) for n in (
            "h1au1", "h2au2", "h1au2", "h2au1", "h1acell", "h2acell", "cellarea",
            "botz", "gridz")]


_lib_path = None


def use_grid_lib(path):
    """Build windows with the window-builder library at `path` (another build
    of csrc/shoc_grid.c) instead of the package's own; call before the first
    window is built."""
    global _lib_path
    if _lib is not None and path != _lib_path:
        raise RuntimeError("the window builder is already loaded from %s" % _lib_path)
    _lib_path = path


def lib():
    global _lib, _lib_path
    if _lib is None:
        path = _lib_path
        if path is None:
            from . import _build
            path = os.path.join(_HERE, "_lib", "libshoc_grid.so")
            if not os.path.exists(path):
                _build.grid_lib()
            _lib_path = path
        L = C.CDLL(path)
        L.shoc_grid_build.argtypes = [C.POINTER(_GridSpec), C.POINTER(_Grid)]
        L.shoc_grid_build.restype = C.c_int
        L.shoc_grid_free.argtypes = [C.POINTER(_Grid)]
        L.shoc_grid_init_surface.argtypes = [C.POINTER(_Grid), _abi.DP, _abi.IP, _abi.IP]
        L.shoc_grid_w_from_continuity.argtypes = [
            C.POINTER(_Grid), _abi.IP, _abi.DP, _abi.DP, _abi.DP]
        L.shoc_synth_flow.argtypes = [C.POINTER(_Grid), _abi.DP, _abi.DP, _abi.DP, C.c_double] + \
            [_abi.DP] * 6
        L.shoc_synth_flow.restype = C.c_int
        L.shoc_synth_kz_exp.argtypes = [C.POINTER(_Grid), C.c_double, C.c_double, _abi.DP]
        L.shoc_synth_kz_logu.argtypes = [C.POINTER(_Grid), C.c_ulonglong, C.c_double,
                                         C.c_double, _abi.DP]
        L.shoc_synth_tracers_logn.argtypes = [C.POINTER(_Grid), C.c_ulonglong, C.c_int,
                                              C.c_double, C.c_double, _abi.DP, _abi.DP]
        _lib = L
    return _lib


def _view_i(ptr, n):
    return np.ctypeslib.as_array(ptr, shape=(n,))


class Window:
    """A built SHOC window: geometry (owned by the C builder) + numpy views."""

    def __init__(self, nx, ny, nz, layers, bathy, land, h1acell, h2acell,
                 h1au1, h2au1, h1au2, h2au2):
        self._keep = dict(layers=np.ascontiguousarray(layers, np.float64),
                          bathy=np.ascontiguousarray(bathy, np.float64),
                          land=np.ascontiguousarray(land, np.uint8))
        for k, v in dict(h1acell=h1acell, h2acell=h2acell, h1au1=h1au1, h2au1=h2au1,
                         h1au2=h1au2, h2au2=h2au2).items():
            self._keep[k] = np.ascontiguousarray(v, np.float64)
        K = self._keep
        spec = _GridSpec(nx, ny, nz, dptr(K["layers"]), dptr(K["bathy"]),
                         K["land"].ctypes.data_as(C.POINTER(C.c_ubyte)),
                         dptr(K["h1acell"]), dptr(K["h2acell"]), dptr(K["h1au1"]),
                         dptr(K["h2au1"]), dptr(K["h1au2"]), dptr(K["h2au2"]))
        self._g = _Grid()
        rc = lib().shoc_grid_build(C.byref(spec), C.byref(self._g))
        if rc != 0:
            raise _abi.StatusError("shoc_grid_build", rc)
        g = self._g.geom
        self.geom = g
        self.nx, self.ny, self.nz = nx, ny, nz
        self.sgsiz, self.sgsizS = g.sgsiz, g.sgsizS
        self.nwet = self._g.nwet
        self.ncol = self._g.ncol
        S, S2 = g.sgsiz, g.sgsizS
        for n in ("xp1", "xm1", "yp1", "ym1", "zp1", "zm1", "m2d", "s2i", "s2j", "s2k"):
            setattr(self, n, _view_i(getattr(g, n), S))
        self.is_wet = _view_i(self._g.is_wet, S)
        self.w3_t = _view_i(g.w3_t, g.n3_t + 1)
        self.w2_t = _view_i(g.w2_t, g.n2_t + 1)
        self.bot_t = _view_i(g.bot_t, g.b2_t + 1)
        self.bpt = _view_i(g.bpt, g.nbpt + 1)
        self.bin = _view_i(g.bin, g.nbpt + 1)
        self.kbot = _view_i(self._g.kbot, nx * ny).reshape(ny, nx)
        self.map_top = _view_i(self._g.map_top, nx * ny).reshape(ny, nx)
        for n in ("h1au1", "h2au2", "h1au2", "h2au1", "h1acell", "h2acell",
                  "cellarea", "botz"):
            setattr(self, n, np.ctypeslib.as_array(getattr(g, n), shape=(S2,)))
        self.gridz = np.ctypeslib.as_array(g.gridz, shape=(S,))
        self.layers = K["layers"]

    def __del__(self):
        try:
            if getattr(self, "_g", None) is not None and lib() is not None:
                lib().shoc_grid_free(C.byref(self._g))
                self._g = None
        except Exception:
            pass

    def init_surface(self, eta):
        g = self.geom
        sur = np.zeros(g.b2_t + 1, np.int32)
        nsur = np.zeros(g.a2_t + 1, np.int32)
        lib().shoc_grid_init_surface(C.byref(self._g), dptr(eta), iptr(sur), iptr(nsur))
        return sur, nsur

    def w_from_continuity(self, sur_t, u1flux3d, u2flux3d):
        w = np.zeros(self.sgsiz, np.float64)
        lib().shoc_grid_w_from_continuity(C.byref(self._g), iptr(sur_t), dptr(u1flux3d),
                                          dptr(u2flux3d), dptr(w))
        return w

    # --- helpers over wet cells -------------------------------------------
    def wet_cells(self):
        return self.w3_t[1:self.geom.a3_t + 1]

    def cell_top(self, eta):
        """z of the top face of every wet cell (eta for the surface cell)."""
        c = self.wet_cells()
        top = np.zeros(self.sgsiz)
        zp1 = self.zp1[c]
        is_top = zp1 == c
        top[c] = np.where(is_top, 0.0, self.gridz[zp1])
        top[c[is_top]] = eta[self.m2d[c[is_top]]]
        # cells whose upper neighbour is above the free surface stop at eta
        top[c] = np.minimum(top[c], eta[self.m2d[c]])
        return top

    def cell_bot(self):
        c = self.wet_cells()
        bot = np.zeros(self.sgsiz)
        bot[c] = self.gridz[c]
        zm1 = self.zm1[c]
        is_bot = ~self.is_wet[zm1].astype(bool)
        bot[c[is_bot]] = self.botz[self.m2d[c[is_bot]]]
        return bot


def _smooth(rng, ny, nx, nmodes=8, kmax=4.0):
    """Smooth seeded field in [0, 1]: a sum of random low-wavenumber waves."""
    y = (np.arange(ny) + 0.5)[:, None] / ny
    x = (np.arange(nx) + 0.5)[None, :] / nx
    f = np.zeros((ny, nx))
    for _ in range(nmodes):
        kx, ky = rng.uniform(0.3, kmax, 2)
        px, py = rng.uniform(0, 2 * np.pi, 2)
        a = rng.uniform(0.5, 1.0)
        f += a * np.cos(2 * np.pi * kx * x + px) * np.cos(2 * np.pi * ky * y + py)
    f -= f.min()
    return f / max(f.max(), 1e-300)


def _metrics(h1c, h2c):
    """Face metrics on an (ny+1) x (nx+1) array from cell-centre sizes."""
    ny, nx = h1c.shape
    H1 = np.empty((ny + 1, nx + 1))
    H2 = np.empty((ny + 1, nx + 1))
    H1[:ny, :nx] = h1c
    H2[:ny, :nx] = h2c
    H1[ny, :] = H1[ny - 1, :]
    H2[ny, :] = H2[ny - 1, :]
    H1[:, nx] = H1[:, nx - 1]
    H2[:, nx] = H2[:, nx - 1]
    h1au1 = H1.copy()
    h2au1 = H2.copy()
    h1au1[:, 1:] = 0.5 * (H1[:, 1:] + H1[:, :-1])
    h2au1[:, 1:] = 0.5 * (H2[:, 1:] + H2[:, :-1])
    h1au2 = H1.copy()
    h2au2 = H2.copy()
    h1au2[1:, :] = 0.5 * (H1[1:, :] + H1[:-1, :])
    h2au2[1:, :] = 0.5 * (H2[1:, :] + H2[:-1, :])
    return H1, H2, h1au1, h2au1, h1au2, h2au2


def _snap_bathy(bathy, layers, minfrac=0.3):
    """Keep partial bottom cells at least minfrac of their layer thick."""
    k = np.searchsorted(layers, bathy, side="right") - 1
    k = np.clip(k, 0, len(layers) - 2)
    lo, hi = layers[k], layers[k + 1]
    frac = (hi - bathy) / (hi - lo)
    return np.where(frac < minfrac, hi - minfrac * (hi - lo), bathy)


class Case:
    """A complete tracer-transport problem on one window."""

    def __init__(self, name, win, ntr, dt, u1, u2, w, u1flux3d, u2flux3d, Kz, eta,
                 oldeta, tr, trasc=_abi.QUICKEST, ultimate=1, stab=_abi.SUB_STEP,
                 hmin=0.07, mintr=None, maxtr=None, seed=0, nsteps=1, dzu1=None,
                 dzu2=None, u1kh=None, u2kh=None, diffuse=None):
        self.name = name
        self.win = win
        self.ntr = ntr
        self.dt = float(dt)
        self.u1, self.u2, self.w = u1, u2, w
        self.u1flux3d, self.u2flux3d, self.Kz = u1flux3d, u2flux3d, Kz
        self.eta, self.oldeta = eta, oldeta
        self.tr = tr                       # (ntr, sgsiz) float64
        self.trasc, self.ultimate, self.stab, self.hmin = trasc, ultimate, stab, hmin
        self.mintr = np.full(ntr, -1e35) if mintr is None else np.asarray(mintr, np.float64)
        self.maxtr = np.full(ntr, 1e35) if maxtr is None else np.asarray(maxtr, np.float64)
        self.seed = seed
        self.nsteps = nsteps
        S = win.sgsiz
        self.dzu1 = np.zeros(S) if dzu1 is None else dzu1
        self.dzu2 = np.zeros(S) if dzu2 is None else dzu2
        self.u1kh = np.zeros(S) if u1kh is None else u1kh
        self.u2kh = np.zeros(S) if u2kh is None else u2kh
        self.diffuse = np.zeros(ntr, np.int32) if diffuse is None else np.asarray(diffuse, np.int32)
        # tracers per water column (None: all); see shoc_tr_opts.ntr2d
        self.ntr2d = None
        self.sur_t, self.nsur_t = win.init_surface(oldeta)

    @property
    def nwet(self):
        return self.win.nwet

    def copy_state(self):
        """Fresh copies of the mutable per-run state (tracers, surface vectors)."""
        return self.tr.copy(), self.sur_t.copy(), self.nsur_t.copy()

    def opts_arrays(self):
        n = self.ntr
        return dict(tbdy=np.arange(n, dtype=np.int32), tdif_v=np.arange(n, dtype=np.int32),
                    advect=np.ones(n, np.int32), diffuse=self.diffuse,
                    mintr=np.ascontiguousarray(self.mintr), maxtr=np.ascontiguousarray(self.maxtr))

    def make_opts(self, keep):
        a = self.opts_arrays()
        keep.append(a)
        return _abi.Opts(self.trasc, self.ultimate, self.stab, self.hmin,
                         len(a["tbdy"]), iptr(a["tbdy"]), len(a["tdif_v"]), iptr(a["tdif_v"]),
                         iptr(a["advect"]), iptr(a["diffuse"]), dptr(a["mintr"]),
                         dptr(a["maxtr"]), iptr(self.ntr2d))

    def make_state(self, tr, sur_t, nsur_t, keep):
        """shoc_tr_state over caller-owned arrays (tr: (ntr, sgsiz) float64)."""
        assert tr.dtype == np.float64 and tr.flags.c_contiguous
        rows = (_abi.DP * self.ntr)(*[tr[n].ctypes.data_as(_abi.DP) for n in range(self.ntr)])
        keep.append(rows)
        return _abi.State(self.ntr, C.cast(rows, C.POINTER(_abi.DP)), iptr(sur_t), iptr(nsur_t),
                          dptr(self.u1), dptr(self.u2), dptr(self.w), dptr(self.u1flux3d),
                          dptr(self.u2flux3d), dptr(self.Kz), dptr(self.dzu1), dptr(self.dzu2),
                          dptr(self.u1kh), dptr(self.u2kh), dptr(self.eta), dptr(self.oldeta),
                          self.dt)

    def cell_tracers(self):
        """Tracer values a step updates: wet cells x tracers, or with per-
        column tracer counts (ntr2d) the sum of each wet cell's count."""
        if self.ntr2d is None:
            return self.nwet * self.ntr
        return int(self.ntr2d[self.win.m2d[self.win.wet_cells()]].sum())

    def bytes_per_step(self, fp64=True):
        """Algorithmic HBM bytes of one step: one read + one write of every
        tracer value and one read of five per-cell fields (u1flux3d, u2flux3d,
        w, Kz, dz) per wet cell."""
        s = 8 if fp64 else 4
        return self.cell_tracers() * 2 * s + self.nwet * 5 * s


def _coast_taper(land, width):
    """0 on land and at corners touching land/edge, rising to 1 inland."""
    ny, nx = land.shape
    wet = np.zeros((ny + 2, nx + 2), bool)
    wet[1:-1, 1:-1] = land == 0
    # corner (i, j) touches cells (i-1..i, j-1..j)
    corner_wet = wet[:-1, :-1] & wet[1:, :-1] & wet[:-1, 1:] & wet[1:, 1:]
    dist = np.where(corner_wet, np.inf, 0.0)
    # cheap distance transform (chessboard) by repeated erosion
    d = np.zeros_like(dist)
    cur = corner_wet.copy()
    for step in range(1, width + 1):
        d[cur] = step
        nxt = cur.copy()
        nxt[1:, :] &= cur[:-1, :]
        nxt[:-1, :] &= cur[1:, :]
        nxt[:, 1:] &= cur[:, :-1]
        nxt[:, :-1] &= cur[:, 1:]
        cur = nxt
    d[cur] = width + 1
    return np.clip((d - 1) / width, 0.0, 1.0)


def build_case(name, nx, ny, layers, *, seed, ntr, dt=60.0, depth=(10.0, 50.0),
               land_frac=0.0, cell=(1000.0, 1000.0), curvilinear=False, umax=0.5,
               baroclinic=0.2, kz=("exp", 1e-2, 1e-5), tracers="gauss", nsteps=1,
               trasc=_abi.QUICKEST, ultimate=1, stab=_abi.SUB_STEP, hmin=0.07,
               mintr=None, maxtr=None, eta_offset=None, hdiff=None, bathy_land=None):
    rng = np.random.default_rng(seed)
    layers = np.asarray(layers, np.float64)
    nz = len(layers) - 1
    if bathy_land is None:
        f = _smooth(rng, ny, nx)
        bathy = -(depth[0] + (depth[1] - depth[0]) * f)
        bathy = np.maximum(bathy, layers[0])
        bathy = _snap_bathy(bathy, layers)
        land = np.zeros((ny, nx), np.uint8)
        if land_frac > 0:
            g = _smooth(rng, ny, nx, nmodes=10, kmax=6.0)
            land = (g < np.quantile(g, land_frac)).astype(np.uint8)
    else:
        bathy, land = bathy_land
    if curvilinear:
        h1c = cell[0] + (cell[1] - cell[0]) * _smooth(rng, ny, nx, nmodes=6, kmax=2.0)
        h2c = cell[0] + (cell[1] - cell[0]) * _smooth(rng, ny, nx, nmodes=6, kmax=2.0)
    else:
        h1c = np.full((ny, nx), float(cell[0]))
        h2c = np.full((ny, nx), float(cell[1]))
    H1, H2, h1au1, h2au1, h1au2, h2au2 = _metrics(h1c, h2c)
    win = Window(nx, ny, nz, layers, bathy, land, H1, H2, h1au1, h2au1, h1au2, h2au2)
    S, S2 = win.sgsiz, win.sgsizS
    eta = np.zeros(S2)
    oldeta = np.zeros(S2)
    if eta_offset is not None:
        eta[1:] = eta_offset[0] * (np.cos(np.arange(1, S2) * 0.37) )
        oldeta[1:] = eta_offset[1] * (np.sin(np.arange(1, S2) * 0.23))
    # transport streamfunction at corners: gyre x coastal taper
    yc = np.arange(ny + 1)[:, None] / ny
    xc = np.arange(nx + 1)[None, :] / nx
    psi = np.sin(np.pi * xc) * np.sin(np.pi * yc)
    psi = psi * (0.6 + 0.4 * _smooth(rng, ny + 1, nx + 1, nmodes=5, kmax=3.0))
    psi = psi * _coast_taper(land, width=3)
    bc = baroclinic * (2 * _smooth(rng, ny, nx, nmodes=5, kmax=3.0) - 1)
    u1, u2, u1flux3d, u2flux3d, dzu1, dzu2 = (np.zeros(S) for _ in range(6))
    psi = np.ascontiguousarray(psi)
    bc = np.ascontiguousarray(bc)
    rc = lib().shoc_synth_flow(C.byref(win._g), dptr(psi), dptr(bc), dptr(oldeta), umax,
                               dptr(u1), dptr(u2), dptr(u1flux3d), dptr(u2flux3d), dptr(dzu1),
                               dptr(dzu2))
    if rc:
        raise _abi.StatusError("shoc_synth_flow", rc)
    sur_t, _ = win.init_surface(oldeta)
    w = win.w_from_continuity(sur_t, u1flux3d, u2flux3d)
    # vertical diffusivity at bottom faces
    c = win.wet_cells()
    Kz = np.zeros(S)
    if kz[0] == "exp":
        lib().shoc_synth_kz_exp(C.byref(win._g), kz[1], kz[2], dptr(Kz))
    else:
        lib().shoc_synth_kz_logu(C.byref(win._g), seed, kz[1], kz[2], dptr(Kz))
    tr = np.zeros((ntr, S))
    if tracers not in ("gauss", "step"):
        sm = np.ascontiguousarray(np.stack([_smooth(rng, ny, nx, nmodes=6, kmax=5.0)
                                            for _ in range(ntr)]))
        lib().shoc_synth_tracers_logn(C.byref(win._g), seed, ntr, tracers[1], tracers[2],
                                      dptr(sm), dptr(tr))
        tracers = "done"
    ii, jj, kk = win.s2i[c], win.s2j[c], win.s2k[c]
    if tracers == "gauss":
        # centre off the cell grid in every direction, so no two cells are
        # mirror images and the limiter never sees exactly equal neighbours
        sig = 5.0
        x0, y0, z0 = nx / 2 - 0.37, ny / 2 - 0.21, nz / 2 - 0.33
        for n in range(ntr):
            r2 = ((ii - x0) ** 2 + (jj - y0) ** 2 + (kk - z0) ** 2)
            tr[n, c] = np.exp(-r2 / (2 * sig * sig))
    elif tracers == "step":
        for n in range(ntr):
            tr[n, c] = np.where((ii + jj + n) % 7 < 3, 1.0 + n, 0.0)

    # horizontal diffusion (hor_diffuse): hdiff = (Kh in m^2/s, per-tracer
    # on/off); Kh on the wet cells' u1 and u2 faces
    u1kh = u2kh = diffuse = None
    if hdiff is not None:
        u1kh = np.zeros(S)
        u1kh[c] = hdiff[0]
        u2kh = u1kh.copy()
        diffuse = np.asarray(hdiff[1], np.int32)
        assert len(diffuse) == ntr

    # ghost / above-surface values are filled by the step itself
    return Case(name, win, ntr, dt, u1, u2, w, u1flux3d, u2flux3d, Kz, eta, oldeta, tr,
                trasc=trasc, ultimate=ultimate, stab=stab, hmin=hmin, seed=seed,
                nsteps=nsteps, dzu1=dzu1, dzu2=dzu2, mintr=mintr, maxtr=maxtr,
                u1kh=u1kh, u2kh=u2kh, diffuse=diffuse)


# Uneven batch of independent basins (horizontal size, layers, tracers): the
# sizes, layer counts and tracer counts of the multi-basin configuration.
BATCH8 = ((128, 128, 20, 4), (256, 256, 26, 8), (384, 256, 31, 12), (512, 512, 37, 16),
          (768, 512, 43, 20), (1024, 1024, 49, 24), (1536, 768, 54, 28),
          (2048, 1024, 60, 32))


def batch_partition(basins, parts):
    """Basins (indices) of each of `parts` ranks: largest first (cells x
    tracers), each to the rank with the least work so far."""
    order = sorted(range(len(basins)), key=lambda b: -np.prod(basins[b], dtype=np.float64))
    load, out = [0.0] * parts, [[] for _ in range(parts)]
    for b in order:
        r = int(np.argmin(load))
        out[r].append(b)
        load[r] += float(np.prod(basins[b], dtype=np.float64))
    return [sorted(o) for o in out]


def build_batch(name, basins, *, seed, scale=1.0, gap=3, nz=60, depth=250.0, which=None, **kw):
    """One window holding independent basins side by side, separated by
    `gap` land columns, each with its own seeded bathymetry (its own deepest
    layer count and 30 % land) and tracer count (shoc_tr_opts.ntr2d).  The
    streamfunction vanishes at every coast, so no water or tracer crosses
    between basins and each steps as it would alone.  which: the indices of
    the basins to build (default all), each with the bathymetry and land it
    has in the whole batch (the seeded draws of the others are made and
    dropped)."""
    rng = np.random.default_rng(seed)
    layers = uniform_layers(nz, depth)
    dims = [(max(8, int(round(bx * scale))), max(8, int(round(by * scale))), L, T)
            for bx, by, L, T in basins]
    keep = list(range(len(dims))) if which is None else sorted(which)
    # the bathymetry and land draws of every basin, in order
    draws = []
    for bx, by, L, T in dims:
        f = _smooth(rng, by, bx)
        g = _smooth(rng, by, bx, nmodes=10, kmax=6.0)
        draws.append((f, g))
    dims = [dims[b] for b in keep]
    draws = [draws[b] for b in keep]
    nx = sum(d[0] for d in dims) + gap * (len(dims) + 1)
    ny = max(d[1] for d in dims) + 2 * gap
    bathy = np.full((ny, nx), layers[-2])
    land = np.ones((ny, nx), np.uint8)
    tr_of = np.zeros((ny, nx), np.int32)
    x0 = gap
    for (bx, by, L, T), (f, g) in zip(dims, draws):
        dmax = depth * L / nz
        b = -(2.0 + (dmax - 2.0) * f)
        b = np.maximum(b, layers[0])
        ld = (g < np.quantile(g, 0.3)).astype(np.uint8)
        bathy[gap:gap + by, x0:x0 + bx] = _snap_bathy(b, layers)
        land[gap:gap + by, x0:x0 + bx] = ld
        tr_of[gap:gap + by, x0:x0 + bx] = T
        x0 += bx + gap
    ntr = max(d[3] for d in dims)
    d = dict(layers=layers, seed=seed, ntr=ntr, cell=(150.0, 150.0), umax=1.5,
             kz=("logu", 1e-6, 1e-1), tracers=("logn", 1.0, 1.0), nsteps=500)
    d.update(kw)
    case = build_case(name, nx, ny, bathy_land=(bathy, land), **d)
    # tracers carried per water column: the basin's count
    win = case.win
    c2 = np.arange(1, win.sgsizS)
    ntr2d = np.zeros(win.sgsizS, np.int32)
    ok = c2 < len(win.s2i)
    i, j = win.s2i[c2[ok]], win.s2j[c2[ok]]
    inb = (i >= 0) & (i < nx) & (j >= 0) & (j < ny)
    ntr2d[c2[ok][inb]] = tr_of[j[inb], i[inb]]
    case.ntr2d = ntr2d
    case.basins = dims
    # basin of every 2D cell (-1: land between the basins)
    bid = np.full((ny, nx), -1, np.int32)
    x0 = gap
    for b, (bx, by, L, T) in enumerate(dims):
        bid[gap:gap + by, x0:x0 + bx] = b
        x0 += bx + gap
    basin2d = np.full(win.sgsizS, -1, np.int32)
    basin2d[c2[ok][inb]] = bid[j[inb], i[inb]]
    case.basin2d = basin2d
    return case


def uniform_layers(nz, depth):
    return np.linspace(-depth, 0.0, nz + 1)


def stiff_layers(nz, depth, nthin=10, thin=0.5):
    top = np.linspace(-nthin * thin, 0.0, nthin + 1)
    rest = np.linspace(-depth, -nthin * thin, nz - nthin + 1)
    return np.concatenate([rest[:-1], top])


WORKLOADS = ("small", "basin64", "drop512", "batch2048", "stiff2048", "batch8", "batch8small")


def make(name, seed=None, **kw):
    """Build one of the named workloads (see module docstring)."""
    if name == "small":
        d = dict(nx=20, ny=14, layers=uniform_layers(6, 30.0), seed=11, ntr=3,
                 depth=(3.0, 30.0), land_frac=0.2, cell=(500.0, 800.0), curvilinear=True,
                 umax=0.8, kz=("logu", 1e-5, 1e-1), tracers=("logn", 1e-2, 10.0), nsteps=10)
    elif name == "basin64":
        d = dict(nx=64, ny=64, layers=uniform_layers(20, 50.0), seed=64, ntr=1,
                 depth=(10.0, 50.0), umax=0.5, kz=("exp", 1e-2, 1e-5), tracers="gauss",
                 nsteps=100)
    elif name == "drop512":
        d = dict(nx=512, ny=512, layers=uniform_layers(40, 200.0), seed=512, ntr=10,
                 depth=(2.0, 200.0), land_frac=0.3, cell=(150.0, 150.0), umax=1.5,
                 kz=("logu", 1e-6, 1e-1), tracers=("logn", 1.0, 1.0), nsteps=500)
    elif name == "batch2048":
        d = dict(nx=2048, ny=1024, layers=uniform_layers(50, 250.0), seed=2048, ntr=24,
                 depth=(2.0, 250.0), land_frac=0.35, cell=(200.0, 2000.0), curvilinear=True,
                 umax=1.0, kz=("logu", 1e-6, 1e-1), tracers=("logn", 1e-3, 1e2), nsteps=1000)
    elif name in ("batch8", "batch8small"):
        kw = dict(kw)
        sc = kw.pop("scale", 1.0 if name == "batch8" else 1.0 / 16)
        return build_batch(name, BATCH8, seed=2048 if seed is None else seed, scale=sc, **kw)
    elif name == "stiff2048":
        d = dict(nx=2048, ny=1024, layers=stiff_layers(50, 250.0), seed=2048, ntr=24,
                 depth=(2.0, 250.0), land_frac=0.35, cell=(200.0, 2000.0), curvilinear=True,
                 umax=1.0, baroclinic=0.05, kz=("logu", 1e-6, 1.0),
                 tracers=("logn", 1e-3, 1e2), nsteps=1000)
    else:
        raise KeyError(name)
    if seed is not None:
        d["seed"] = seed
    d.update(kw)
    nx, ny = d.pop("nx"), d.pop("ny")
    return build_case(name, nx, ny, d.pop("layers"), **d)
