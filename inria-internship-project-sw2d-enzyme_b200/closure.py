"""The learned momentum-exchange closure: a small MLP on the tensor cores (C ABI sw2d_mlp_*).

``MLP`` owns a network of 10 features -> 64 -> 64 -> 2 outputs (GELU) on one GPU: inference,
loss and gradient, Adam steps, all in the library's tcgen05 kernels (BF16 operands, FP32
accumulation).  ``reference_forward`` / ``reference_loss_grad`` restate the same network in
numpy FP64 with the kernels' BF16 roundings, for the tests' gradient checks.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Tuple

import numpy as np

from . import capi

N_IN, N_HID, N_OUT = 10, 64, 2
SHAPES = [("W1", (N_HID, N_IN)), ("b1", (N_HID,)), ("W2", (N_HID, N_HID)), ("b2", (N_HID,)),
          ("W3", (N_OUT, N_HID)), ("b3", (N_OUT,))]


def init_params(seed: int = 0) -> np.ndarray:
    """He-style initialisation of the parameter vector (layout of sw2d_mlp_create)."""
    rng = np.random.default_rng(seed)
    out = []
    for name, shape in SHAPES:
        if name.startswith("W"):
            out.append(rng.normal(0.0, np.sqrt(2.0 / shape[1]), size=shape).reshape(-1))
        else:
            out.append(np.zeros(shape))
    return np.concatenate(out).astype(np.float32)


def unpack(p: np.ndarray):
    out, k = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(p[k:k + n], dtype=np.float64).reshape(shape)
        k += n
    return out


def bf16(a) -> np.ndarray:
    """Round to bfloat16 (nearest even), returned as float64."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def gelu(x):
    k0, k1 = 0.7978845608028654, 0.044715
    return 0.5 * x * (1.0 + np.tanh(k0 * (x + k1 * x ** 3)))


def gelu_grad(x):
    k0, k1 = 0.7978845608028654, 0.044715
    t = np.tanh(k0 * (x + k1 * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * k0 * (1.0 + 3.0 * k1 * x * x)


def reference_forward(p: np.ndarray, norm: np.ndarray, x: np.ndarray, rounding: bool = True):
    """FP64 forward with the kernels' BF16 roundings (inputs, weights, hidden activations), or
    without any rounding (rounding=False, for finite-difference checks of the formulas)."""
    rd = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    w = unpack(p)
    xm, xs, ym, ys = norm[:N_IN], norm[N_IN:2 * N_IN], norm[2 * N_IN:2 * N_IN + N_OUT], norm[2 * N_IN + N_OUT:]
    xn = rd(((np.asarray(x, np.float32) - xm.astype(np.float32)) / xs.astype(np.float32)))
    z1 = xn @ rd(w["W1"]).T + w["b1"]
    h1 = rd(gelu(z1))
    z2 = h1 @ rd(w["W2"]).T + w["b2"]
    h2 = rd(gelu(z2))
    yn = h2 @ rd(w["W3"]).T + w["b3"]
    return dict(xn=xn, z1=z1, h1=h1, z2=z2, h2=h2, yn=yn, y=yn * ys + ym)


def reference_loss_grad(p: np.ndarray, norm: np.ndarray, x: np.ndarray, t: np.ndarray,
                        rounding: bool = True) -> Tuple[float, np.ndarray]:
    """Loss (mean squared error of the normalised outputs) and its FP64 gradient, with the
    kernels' BF16 roundings of dY, dZ2 and dZ1 (or none: rounding=False)."""
    rd = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    w = unpack(p)
    f = reference_forward(p, norm, x, rounding)
    ym, ys = norm[2 * N_IN:2 * N_IN + N_OUT], norm[2 * N_IN + N_OUT:]
    tn = ((np.asarray(t, np.float32) - ym.astype(np.float32)) / ys.astype(np.float32)).astype(np.float64)
    n = x.shape[0]
    d = f["yn"] - tn
    loss = float(np.sum(d * d) / (n * N_OUT))
    dy = rd(2.0 * d / (n * N_OUT))
    dz2 = rd((dy @ rd(w["W3"])) * gelu_grad(f["z2"]))
    dz1 = rd((dz2 @ rd(w["W2"])) * gelu_grad(f["z1"]))
    g = dict(W3=dy.T @ f["h2"], b3=dy.sum(0), W2=dz2.T @ f["h1"], b2=dz2.sum(0), W1=dz1.T @ f["xn"],
             b1=dz1.sum(0))
    return loss, np.concatenate([g[name].reshape(-1) for name, _ in SHAPES])


class MLP:
    """The closure network on one GPU (the library's tcgen05 kernels)."""

    def __init__(self, params: Optional[np.ndarray] = None, norm: Optional[np.ndarray] = None, device: int = 0):
        self.lib = capi.load_library()
        n = self.lib.sw2d_mlp_param_count()
        p = init_params() if params is None else np.asarray(params, dtype=np.float32)
        if p.size != n:
            raise ValueError(f"expected {n} parameters")
        if norm is None:
            norm = np.concatenate([np.zeros(N_IN), np.ones(N_IN), np.zeros(N_OUT), np.ones(N_OUT)])
        self.norm = np.ascontiguousarray(norm, dtype=np.float32)
        self.h = ctypes.c_void_p()
        fp = ctypes.POINTER(ctypes.c_float)
        st = self.lib.sw2d_mlp_create(int(device), np.ascontiguousarray(p).ctypes.data_as(fp),
                                      self.norm.ctypes.data_as(fp), ctypes.byref(self.h))
        if st != 0:
            raise RuntimeError(f"sw2d_mlp_create failed ({st})")

    def _fp(self, a):
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))

    def _check(self, st):
        if st != 0:
            raise RuntimeError(f"sw2d_mlp error {st}: {self.lib.sw2d_mlp_last_error(self.h).decode()}")

    @property
    def params(self) -> np.ndarray:
        out = np.empty(self.lib.sw2d_mlp_param_count(), dtype=np.float32)
        self._check(self.lib.sw2d_mlp_get_params(self.h, self._fp(out)))
        return out

    def infer(self, x, layers: bool = False):
        x = np.ascontiguousarray(x, dtype=np.float32)
        n = x.shape[0]
        y = np.empty((n, N_OUT), dtype=np.float32)
        lay = np.empty((4, n, N_HID), dtype=np.float32) if layers else None
        self._check(self.lib.sw2d_mlp_infer(self.h, self._fp(x), n, self._fp(y),
                                            self._fp(lay) if layers else None))
        return (y, lay) if layers else y

    def loss_grad(self, x, t):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        loss = ctypes.c_double()
        g = np.empty(self.lib.sw2d_mlp_param_count(), dtype=np.float32)
        self._check(self.lib.sw2d_mlp_loss_grad(self.h, self._fp(x), self._fp(t), x.shape[0], ctypes.byref(loss),
                                                self._fp(g)))
        return loss.value, g

    def adam_step(self, lr: float) -> None:
        self._check(self.lib.sw2d_mlp_adam_step(self.h, float(lr)))

    def set_wait_polls(self, polls: int) -> None:
        """Poll limit of the first tensor-core wait of each chunk (< 0: the default)."""
        self._check(self.lib.sw2d_mlp_set_wait_polls(self.h, int(polls)))

    def train(self, x, t, epochs: int = 10, batch: int = 4096, lr: float = 2e-3, seed: int = 0):
        """Mini-batch Adam over seeded shuffles; returns the per-epoch mean losses."""
        rng = np.random.default_rng(seed)
        n = x.shape[0]
        hist = []
        for _ in range(epochs):
            order = rng.permutation(n)
            tot, cnt = 0.0, 0
            for s in range(0, n, batch):
                idx = order[s:s + batch]
                loss, _ = self.loss_grad(x[idx], t[idx])
                self.adam_step(lr)
                tot += loss * idx.size
                cnt += idx.size
            hist.append(tot / max(cnt, 1))
        return hist

    def close(self):
        if self.h:
            self.lib.sw2d_mlp_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------------------------------
# Training data from the solver itself: fine-mesh plain shallow-water runs over a building
# layout (buildings as holes in the mesh), averaged onto coarse dual-integral-porosity cells.
# ------------------------------------------------------------------------------------------
def building_layout(lx: float, ly: float, size=(5.0, 30.0), coverage: float = 0.3, seed: int = 0,
                    margin: float = 10.0) -> np.ndarray:
    """Seeded axis-aligned rectangular buildings [k x 4] = (x0, y0, x1, y1), sides U[size],
    placed (overlaps allowed) until the covered fraction of the domain reaches `coverage`
    (estimated on a 1 m raster); a margin along x = 0 and x = lx stays free."""
    rng = np.random.default_rng(seed)
    nxr, nyr = int(np.ceil(lx)), int(np.ceil(ly))
    covered = np.zeros((nyr, nxr), dtype=bool)
    out = []
    while covered.mean() < coverage:
        w, h = rng.uniform(size[0], size[1], 2)
        x0 = rng.uniform(margin, lx - margin - w)
        y0 = rng.uniform(0.0, ly - h)
        out.append((x0, y0, x0 + w, y0 + h))
        covered[int(y0):int(np.ceil(y0 + h)), int(x0):int(np.ceil(x0 + w))] = True
        if len(out) > 100000:
            break
    return np.array(out, dtype=np.float64).reshape(-1, 4)


def inside_buildings(x, y, blds: np.ndarray) -> np.ndarray:
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    ins = np.zeros(x.shape, dtype=bool)
    for x0, y0, x1, y1 in blds:
        ins |= (x > x0) & (x < x1) & (y > y0) & (y < y1)
    return ins


def _codes_for(lx):
    def codes(mx, my):
        c = np.full(mx.shape, -1, dtype=np.int32)
        c[mx < 1e-9] = -2
        c[mx > lx - 1e-9] = -3
        return c
    return codes


def urban_cases(lx: float = 200.0, ly: float = 100.0, dx_fine: float = 1.0, coarse_factor: int = 8,
                coverage: float = 0.3, h0: float = 0.5, h_in: float = 1.5, h_out: float = 0.5, n_manning: float = 0.02,
                seed: int = 0, t_max: float = 1.0e9):
    """(fine SP case, coarse DIP case, averager): the fine mesh resolves the buildings as holes
    (dx_fine triangles), the coarse mesh is a regular grid coarse_factor times coarser carrying
    the storage porosity phiW (fluid fraction of the cell, from the fine cells it contains) and
    the connectivity porosity phiG (fluid fraction of each edge, sampled along it, not above the
    adjacent cells' phiW).  Inflow: prescribed depth h_in on x = 0; outflow: depth h_out on
    x = lx; walls elsewhere and around the buildings.  Flat bed, Manning n, water at rest at
    depth h0."""
    from .case import BoundarySeries, Case
    from .mesh import jittered_triangles, mesh_from_triangles

    blds = building_layout(lx, ly, coverage=coverage, seed=seed)
    nxf, nyf = int(round(lx / dx_fine)), int(round(ly / dx_fine))
    x, y, z, tri = jittered_triangles(nxf, nyf, lx, ly, jitter=0.2, seed=seed + 1)
    cxf, cyf = x[tri].mean(1), y[tri].mean(1)
    keep = ~inside_buildings(cxf, cyf, blds)
    fine_mesh = mesh_from_triangles(x, y, z, tri[keep], _codes_for(lx))
    nxc, nyc = nxf // coarse_factor, nyf // coarse_factor
    xc, yc, zc, tric = jittered_triangles(nxc, nyc, lx, ly, jitter=0.0, seed=seed + 2)
    coarse_mesh = mesh_from_triangles(xc, yc, zc, tric, _codes_for(lx))
    av = Averager(fine_mesh, coarse_mesh, xc, yc, tric, nxc, nyc, lx, ly)
    # fine cells are assigned by centroid, so a coarse cell can collect a little more than its
    # area: the storage porosity is clipped to [0.05, 1]
    phiW = np.clip(av.fluid_fraction(), 0.05, 1.0)
    m = coarse_mesh

    def edge_fraction(ax, ay, bx, by, k=64):
        s = (np.arange(k) + 0.5) / k
        px = ax[:, None] + (bx - ax)[:, None] * s[None, :]
        py = ay[:, None] + (by - ay)[:, None] * s[None, :]
        return 1.0 - inside_buildings(px, py, blds).mean(1)

    # edge end points from the coarse triangles: an edge of length L, normal n, midpoint m runs
    # from m - L/2 t to m + L/2 t with t = (-n_y, n_x)
    def ends(mx, my, nx, ny, L):
        tx, ty = -ny, nx
        return mx - 0.5 * L * tx, my - 0.5 * L * ty, mx + 0.5 * L * tx, my + 0.5 * L * ty

    L, R = m.edge_int_cells[:, 0], m.edge_int_cells[:, 1]
    gi = edge_fraction(*ends(m.edge_int_mx, m.edge_int_my, m.edge_int_nx, m.edge_int_ny, m.edge_int_length))
    # the DIP specific force stops on phiG < 1e-16 (swDip.cpp:1524-1528): a blocked edge keeps a
    # small opening
    gi = np.minimum(np.maximum(gi, 0.01), np.minimum(phiW[L], phiW[R]))
    gb = edge_fraction(*ends(m.edge_bnd_mx, m.edge_bnd_my, m.edge_bnd_nx, m.edge_bnd_ny, m.edge_bnd_length))
    gb = np.minimum(np.maximum(gb, 0.01), phiW[m.edge_bnd_cell])
    bc = BoundarySeries(codes=[-1, -2, -3], types=["q", "h", "h"], times=np.array([0.0, 1.0e9]),
                        values=np.array([[0.0, 0.0], [h_in, h_in], [h_out, h_out]]))
    base = {"num_scheme": "godunov", "topo_discretization": "discontinuous", "model_friction": "manning",
            "cfl_max": 0.8, "dt_max": 1.0, "dt_map": 1.0e9, "h_min": 1e-5, "t_max": t_max, "fr_max": 10.0,
            "store_flag": "none", "output_format": "txt"}
    nf, nc = fine_mesh.cell_nb, m.cell_nb
    fine = Case(mesh=fine_mesh, opts=dict(base, model_hyperb="sp"), h0=np.full(nf, h0), q0=np.zeros(nf),
                r0=np.zeros(nf), phi=np.ones(nf), boussinesq=np.ones(nf),
                friction=np.stack([np.full(nf, n_manning), np.full(nf, n_manning), np.zeros(nf)]), bc=bc,
                extra={"name": "urban_fine", "buildings": blds})
    coarse = Case(mesh=m, opts=dict(base, model_hyperb="dip"), h0=np.full(nc, h0), q0=np.zeros(nc), r0=np.zeros(nc),
                  phi=phiW, boussinesq=np.ones(nc),
                  friction=np.stack([np.full(nc, n_manning), np.full(nc, n_manning), np.zeros(nc)]), bc=bc,
                  phi_g_int=gi, phi_g_bnd=gb, extra={"name": "urban_coarse"})
    return fine, coarse, av


class Averager:
    """Fine cells -> the coarse cells containing their centroids: the fluid fraction of each
    coarse cell and area-weighted averages of fine fields over its fluid part."""

    def __init__(self, fine_mesh, coarse_mesh, xc, yc, tric, nxc, nyc, lx, ly):
        fx, fy = fine_mesh.cell_x, fine_mesh.cell_y
        i = np.clip((fx / (lx / nxc)).astype(np.int64), 0, nxc - 1)
        j = np.clip((fy / (ly / nyc)).astype(np.int64), 0, nyc - 1)
        q = j * nxc + i
        cand = np.stack([2 * q, 2 * q + 1], 1)
        owner = np.full(fx.shape, -1, dtype=np.int64)
        for k in range(2):
            t = tric[cand[:, k]]
            ax, ay = xc[t[:, 0]], yc[t[:, 0]]
            bx, by = xc[t[:, 1]], yc[t[:, 1]]
            cx, cy = xc[t[:, 2]], yc[t[:, 2]]
            d1 = (fx - bx) * (ay - by) - (ax - bx) * (fy - by)
            d2 = (fx - cx) * (by - cy) - (bx - cx) * (fy - cy)
            d3 = (fx - ax) * (cy - ay) - (cx - ax) * (fy - ay)
            neg = (d1 < 0) | (d2 < 0) | (d3 < 0)
            pos = (d1 > 0) | (d2 > 0) | (d3 > 0)
            ins = ~(neg & pos)
            owner = np.where((owner < 0) & ins, cand[:, k], owner)
        owner = np.where(owner < 0, cand[:, 0], owner)  # on an edge of the quad's diagonal
        self.owner = owner
        self.nc = coarse_mesh.cell_nb
        self.fine_area = fine_mesh.cell_area
        self.coarse_area = coarse_mesh.cell_area
        self.fluid_area = np.bincount(owner, weights=self.fine_area, minlength=self.nc)

    def fluid_fraction(self) -> np.ndarray:
        return self.fluid_area / self.coarse_area

    def average(self, field: np.ndarray) -> np.ndarray:
        s = np.bincount(self.owner, weights=field * self.fine_area, minlength=self.nc)
        return np.where(self.fluid_area > 0, s / np.maximum(self.fluid_area, 1e-300), 0.0)


def phig_min_of(case) -> np.ndarray:
    """Smallest connectivity porosity of each cell's internal edges (1 where it has none)."""
    m = case.mesh
    out = np.ones(m.cell_nb)
    np.minimum.at(out, m.edge_int_cells[:, 0], case.phi_g_int)
    np.minimum.at(out, m.edge_int_cells[:, 1], case.phi_g_int)
    return out


def features(s0, s1, phiw, phig_min, dt) -> np.ndarray:
    """The ten closure features (float32) of every cell from the state at the start of a step
    (s0 = h, q, r) and after its flux balance (s1), as the step's update kernel forms them
    (the kernel's own record, SpModel.closure_record, is what the generators below use)."""
    h0, q0, r0 = (np.asarray(a, dtype=np.float64) for a in s0)
    h1, q1, r1 = (np.asarray(a, dtype=np.float64) for a in s1)
    f = np.stack([h0, q0, r0, h1 - h0, q1 - q0, r1 - r0, np.asarray(phiw, np.float64), np.asarray(phig_min, np.float64),
                  np.full(h0.shape, float(dt)), np.sqrt(q0 * q0 + r0 * r0) / np.maximum(h0, 1e-3)], 1)
    return f.astype(np.float32)


def recorder(device: int = 0) -> "MLP":
    """A network whose outputs are zero: attached with an empty hull it only records features."""
    n = np.concatenate([np.zeros(N_IN), np.ones(N_IN), np.zeros(N_OUT), np.ones(N_OUT)])
    return MLP(np.zeros_like(init_params()), n, device)


EMPTY_HULL = (np.ones(N_IN, np.float32), np.zeros(N_IN, np.float32))


def _in_hull(f, hull):
    return np.all((f >= hull[0]) & (f <= hull[1]), 1)


def generate_samples(fine, coarse, av, t_start: float, n_samples: int, spacing: float, device: int = 0,
                     min_depth: float = 1e-3):
    """One-step training pairs.  The fine run (buildings resolved) is brought to t_start, then
    for each sample: its state averaged onto the coarse cells is one coarse DIP step (without
    correction; features from the update kernel's record); the fine run is brought to exactly
    the same end time (t_max clip) and averaged again.  Targets: the averaged fine unit
    discharges minus the coarse step's.  Cells with fluid and depth above min_depth only.
    Returns (X [n x 10], Y [n x 2], times)."""
    from .solver import SpModel

    fm = SpModel(fine, device)
    cm = SpModel(coarse, device)
    rec = recorder(device)
    cm.set_closure(rec, *EMPTY_HULL)
    cm.set_option("closure_record", 1)
    wet_cells = av.fluid_area > 0
    X, Y, T = [], [], []
    fm.set_t_max(t_start)
    fm.execute()
    t = fm.t
    for _ in range(n_samples):
        s0 = tuple(av.average(a) for a in fm.state())
        cm.set_state(*s0)
        cm.set_time(t, 0.0)
        cm.set_t_max(1.0e9)
        cm.step(1)
        f = cm.closure_record()[:, :N_IN]
        s1 = cm.state()
        fm.set_t_max(cm.t)
        fm.execute()
        st = tuple(av.average(a) for a in fm.state())
        keep = wet_cells & (s0[0] > min_depth)
        X.append(f[keep])
        Y.append(np.stack([st[1] - s1[1], st[2] - s1[2]], 1)[keep].astype(np.float32))
        T.append(t)
        t = fm.t
        fm.set_t_max(t + spacing)
        fm.execute()
        t = fm.t
    fm.close()
    cm.close()
    rec.close()
    return np.concatenate(X), np.concatenate(Y), np.array(T)


def generate_trajectory_samples(fine, coarse, av, starts, window: float, tau: float, every: int = 4,
                                net=None, hull=None, device: int = 0, min_depth: float = 1e-3):
    """On-trajectory training pairs with nudging targets.  From each start time the coarse model
    runs freely from the averaged fine state for `window` seconds, with the network `net`
    attached (its hull, plain closure outside) or with none; every `every`-th step samples each
    cell: the features the update kernel formed, and as target the correction that would have
    moved the step's result a fraction dt / tau of the way to the fine run averaged at the same
    time: Y = c + (fine - coarse) dt / tau, c the correction applied in that step (zero without
    a network).  The coarse model thus learns, from its own states, the local mean of its error
    relative to the fine run; tau sets how fast it is corrected.  Returns (X, Y)."""
    from .solver import SpModel

    own = net is None
    if own:
        net, hull = recorder(device), EMPTY_HULL
    wet_cells = av.fluid_area > 0
    X, Y = [], []
    for ts in starts:
        fm = SpModel(fine, device)
        fm.set_t_max(ts)
        fm.execute()
        cm = SpModel(coarse, device)
        cm.set_state(*(av.average(a) for a in fm.state()))
        cm.set_time(fm.t, 0.0)
        cm.set_t_max(1.0e9)
        cm.set_closure(net, hull[0], hull[1])
        cm.set_option("closure_record", 1)
        t_end = fm.t + window
        while cm.t < t_end:
            if every > 1:
                cm.step(every - 1)
            h_before = cm.state()[0]
            cm.step(1)
            r = cm.closure_record()
            f, y = r[:, :N_IN], r[:, N_IN:].astype(np.float64)
            c = np.where(_in_hull(f, hull)[:, None], y, 0.0)
            s1 = cm.state()
            fm.set_t_max(cm.t)
            fm.execute()
            fa = tuple(av.average(a) for a in fm.state())
            keep = wet_cells & (h_before > min_depth)
            g = cm.dt / tau
            X.append(f[keep])
            Y.append((c + np.stack([fa[1] - s1[1], fa[2] - s1[2]], 1) * g)[keep].astype(np.float32))
        fm.close()
        cm.close()
    if own:
        net.close()
    return np.concatenate(X), np.concatenate(Y)


def train_closure(X, Y, epochs: int = 30, batch: int = 4096, lr: float = 2e-3, seed: int = 0, device: int = 0,
                  hull_margin: float = 0.0):
    """Trains the network on (X, Y) with the library's kernels; returns (net, hull_lo, hull_hi,
    loss history).  The hull is the per-feature range of the training features."""
    norm = np.concatenate([X.mean(0), np.maximum(X.std(0), 1e-6), Y.mean(0), np.maximum(Y.std(0), 1e-9)])
    net = MLP(init_params(seed), norm, device)
    hist = net.train(X, Y, epochs=epochs, batch=batch, lr=lr, seed=seed)
    span = X.max(0) - X.min(0)
    return net, X.min(0) - hull_margin * span, X.max(0) + hull_margin * span, hist


def train_on_layouts(layouts, tau: float = 16.0, starts=(4.0, 14.0, 24.0), window: float = 10.0, every: int = 8,
                     epochs: int = 20, batch: int = 8192, lr: float = 2e-3, seed: int = 0, device: int = 0):
    """The closure's training protocol: on-trajectory samples with nudging targets
    (generate_trajectory_samples) from every (fine, coarse, averager) layout, then Adam on the
    tensor cores.  Returns (net, hull_lo, hull_hi, loss history, number of samples)."""
    D = [generate_trajectory_samples(*lay, starts=starts, window=window, tau=tau, every=every, device=device)
         for lay in layouts]
    X = np.concatenate([d[0] for d in D])
    Y = np.concatenate([d[1] for d in D])
    net, lo, hi, hist = train_closure(X, Y, epochs=epochs, batch=batch, lr=lr, seed=seed, device=device)
    return net, lo, hi, hist, int(X.shape[0])


def evaluate(fine, coarse, av, t0: float, t1: float, net=None, hull=None, mus=(0.1, 0.3), device: int = 0,
             scales=(1.0,)):
    """Coarse DIP runs from the fine state averaged at t0 to t1 with (a) no closure, (b) the plain
    closure (uniform mu tensor, for each value in mus), (c) the learned closure with the plain one
    (mus[0]) as fallback out of its hull; each is judged against the fine run averaged at t1.
    Returns {run: (relative L2 error of h, of (q, r))} over the cells with fluid."""
    import copy
    from .solver import SpModel

    fm = SpModel(fine, device)
    fm.set_t_max(t0)
    fm.execute()
    s0 = tuple(av.average(a) for a in fm.state())
    fm.set_t_max(t1)
    fm.execute()
    truth = tuple(av.average(a) for a in fm.state())
    fm.close()
    wet = av.fluid_area > 0
    n = coarse.mesh.cell_nb

    def with_mu(mu):
        c = copy.copy(coarse)
        c.opts = dict(coarse.opts, model_momentum_dissipation="active")
        c.mu = np.stack([np.full(n, mu), np.full(n, mu), np.zeros(n)])
        return c

    def run(case, attach, scale=1.0):
        cm = SpModel(case, device)
        cm.set_state(*s0)
        cm.set_time(t0, 0.0)
        cm.set_t_max(t1)
        if attach:
            cm.set_closure(net, hull[0], hull[1], scale)
        cm.execute()
        out = cm.state()
        cm.close()
        eh = np.linalg.norm((out[0] - truth[0])[wet]) / max(np.linalg.norm(truth[0][wet]), 1e-30)
        dq = np.concatenate([(out[1] - truth[1])[wet], (out[2] - truth[2])[wet]])
        tq = np.concatenate([truth[1][wet], truth[2][wet]])
        return float(eh), float(np.linalg.norm(dq) / max(np.linalg.norm(tq), 1e-30))

    res = {"none": run(coarse, False)}
    for mu in mus:
        res[f"plain_mu{mu:g}"] = run(with_mu(mu), False)
    if net is not None:
        for sc in scales:
            res["learned" if sc == 1.0 else f"learned_x{sc:g}"] = run(with_mu(mus[0]), True, sc)
    return res
