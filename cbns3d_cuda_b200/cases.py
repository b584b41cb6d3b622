"""Synthetic test cases and the reference's file formats.

Formats (kept byte-compatible with the reference):
  * ASCII Plot3D single block: "IM JM KM" then x, y, z with i fastest
    (src/Block3d.cpp:151-202);
  * binary checkpoint: float64 t_cur, uint32 IM_G, JM_G, KM_G, then the AoS
    ghosted state Q[n + 5*(i + IM_G*(j + JM_G*k))] (src/Block3d.cpp:411-474);
  * input.txt: the 17 positional values python/parser_ini.py writes from an
    .ini (src/Block3d.cpp:33-93).

Cases (grids in the reference's non-dimensional units: rho_inf = 1, |u_inf| = 1,
p_inf = 1/(gamma M^2)).  Initial states are evaluated at every node of the
ghosted box, the grid being extended linearly into the ghost layers.
"""
from __future__ import annotations

import configparser
import dataclasses
import struct
from pathlib import Path

import numpy as np

NG = 2
NEQ = 5

INPUT_ORDER = ["grid_fname", "checkpoint_fname", "CFL", "t_cur", "t_end", "Pr", "Pr_t", "gamma", "Mach", "Re",
               "T_inf", "angle_attack", "nstep_max", "checkpoint_freq", "i_begin", "i_end", "is_restart"]


# ---------------------------------------------------------------- file formats
def write_plot3d(path, x, y, z):
    KM, JM, IM = x.shape
    with open(path, "w") as f:
        f.write(f"{IM} {JM} {KM}\n")
        for a in (x, y, z):
            np.ascontiguousarray(a, dtype=np.float64).reshape(-1).tofile(f, sep="\n", format="%.17g")
            f.write("\n")


def read_plot3d(path):
    with open(path) as f:
        IM, JM, KM = (int(v) for v in f.readline().split())
        data = np.fromfile(f, sep=" ", count=3 * IM * JM * KM)
    n = IM * JM * KM
    return [data[m * n:(m + 1) * n].reshape(KM, JM, IM) for m in range(3)]


def write_checkpoint(path, t_cur, Q):
    """Q: (KM_G, JM_G, IM_G, 5) float64."""
    KG, JG, IG, _ = Q.shape
    with open(path, "wb") as f:
        f.write(struct.pack("<d3I", float(t_cur), IG, JG, KG))
        f.write(np.ascontiguousarray(Q, dtype="<f8").tobytes())


def read_checkpoint(path):
    with open(path, "rb") as f:
        t, IG, JG, KG = struct.unpack("<d3I", f.read(20))
        Q = np.frombuffer(f.read(), dtype="<f8").reshape(KG, JG, IG, NEQ).copy()
    return t, Q


def read_vtk(path):
    """Legacy VTK STRUCTURED_GRID as the driver writes it (ASCII or BINARY):
    returns (dims (IM, JM, KM), points (n, 3), {name: array (n,)})."""
    data = Path(path).read_bytes()
    pos = 0

    def line():
        nonlocal pos
        e = data.index(b"\n", pos)
        s = data[pos:e].decode()
        pos = e + 1
        return s

    line()
    line()
    binary = line().strip() == "BINARY"
    line()
    dims = tuple(int(v) for v in line().split()[1:4])
    n = int(line().split()[1])

    def values(count):
        nonlocal pos
        if binary:
            a = np.frombuffer(data[pos:pos + 8 * count], dtype=">f8").astype(np.float64)
            pos += 8 * count + 1  # the newline after the block
            return a
        out = []
        while len(out) < count:
            out.extend(float(v) for v in line().split())
        return np.array(out)

    pts = values(3 * n).reshape(n, 3)
    line()  # POINT_DATA
    nf = int(line().split()[2])
    fields = {}
    for _ in range(nf):
        name = line().split()[0]
        fields[name] = values(n)
    return dims, pts, fields


def read_plot3d_binary(xyz_path, q_path):
    """The driver's binary Plot3D pair: returns (x, y, z, (Mach, alpha, Re, t), q (5, KM, JM, IM))."""
    with open(xyz_path, "rb") as f:
        IM, JM, KM = struct.unpack("<3i", f.read(12))
        g = np.frombuffer(f.read(), dtype="<f8").reshape(3, KM, JM, IM)
    with open(q_path, "rb") as f:
        assert struct.unpack("<3i", f.read(12)) == (IM, JM, KM)
        head = struct.unpack("<4d", f.read(32))
        q = np.frombuffer(f.read(), dtype="<f8").reshape(5, KM, JM, IM)
    return g[0], g[1], g[2], head, q


def write_input(path, **v):
    missing = [k for k in INPUT_ORDER if k not in v]
    if missing:
        raise ValueError(f"input.txt needs {missing}")
    with open(path, "w") as f:
        for k in INPUT_ORDER:
            val = v[k]
            if isinstance(val, bool):
                val = int(val)
            f.write(f"{val!r}\n" if isinstance(val, float) else f"{val}\n")


def parse_ini(ini_path, out_path="input.txt"):
    """The reference's python/parser_ini.py: every value of the .ini, in
    section order, one per line."""
    cfg = configparser.ConfigParser()
    cfg.optionxform = str
    cfg.read(ini_path)
    with open(out_path, "w") as f:
        for sec in cfg.sections():
            for key in cfg[sec]:
                f.write(cfg[sec][key])
                f.write("\n")


# ---------------------------------------------------------------- helpers
def ghost_extend(a):
    """Extend a (KM, JM, IM) coordinate array by NG layers on every side by
    linear extrapolation."""
    return np.pad(a, NG, mode="reflect", reflect_type="odd")


def conservative(rho, u, v, w, p, gamma):
    """Primitive -> AoS conservative (src/conservative_kernel.cu:13-48)."""
    E = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w)
    return np.stack([rho, rho * u, rho * v, rho * w, E], axis=-1)


def primitive(Q, gamma):
    r = Q[..., 0]
    u, v, w = Q[..., 1] / r, Q[..., 2] / r, Q[..., 3] / r
    p = (gamma - 1.0) * (Q[..., 4] - 0.5 * r * (u * u + v * v + w * w))
    return r, u, v, w, p


@dataclasses.dataclass
class Case:
    name: str
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    params: dict            # keyword arguments of cbns3d_cuda_b200.make_params
    Q0: np.ndarray | None   # ghosted AoS initial state, or None for the free-stream start
    t_end: float
    nsteps: int

    @property
    def shape(self):
        KM, JM, IM = self.x.shape
        return IM, JM, KM

    def write(self, workdir, nsteps=None, checkpoint_freq=None, grid_name="grid.xyz",
              checkpoint_name="checkpoint.dat"):
        """Write grid, checkpoint and input.txt for the reference/driver executables."""
        wd = Path(workdir)
        wd.mkdir(parents=True, exist_ok=True)
        write_plot3d(wd / grid_name, self.x, self.y, self.z)
        if self.Q0 is not None:
            write_checkpoint(wd / checkpoint_name, 0.0, self.Q0)
        n = self.nsteps if nsteps is None else nsteps
        p = self.params
        write_input(wd / "input.txt", grid_fname=grid_name, checkpoint_fname=checkpoint_name,
                    CFL=float(p.get("CFL", 0.5)), t_cur=0.0, t_end=float(self.t_end), Pr=float(p.get("Pr", 0.72)),
                    Pr_t=float(p.get("Pr_t", 0.9)), gamma=float(p.get("gamma", 1.4)), Mach=float(p["Mach"]),
                    Re=float(p.get("Re", 1.0e4)), T_inf=float(p.get("T_inf", 288.15)),
                    angle_attack=float(p.get("angle_attack", 0.0)), nstep_max=int(n),
                    checkpoint_freq=int(checkpoint_freq if checkpoint_freq else max(n, 1)),
                    i_begin=int(p.get("i_begin", 1)), i_end=int(p.get("i_end", 0)),
                    is_restart=0 if self.Q0 is not None else 1)
        return wd


# ---------------------------------------------------------------- grids
def perturbed_box(IM, JM, KM, L=(10.0, 5.0, 2.5), amp=0.1):
    """x = i dx + amp sin(2 pi j/JM) sin(2 pi k/KM), and the analogous
    perturbation of y (in i, k) and z (in i, j)."""
    k, j, i = np.meshgrid(np.arange(KM), np.arange(JM), np.arange(IM), indexing="ij")
    dx, dy, dz = L[0] / (IM - 1), L[1] / (JM - 1), L[2] / (KM - 1)
    tp = 2.0 * np.pi
    x = i * dx + amp * np.sin(tp * j / JM) * np.sin(tp * k / KM)
    y = j * dy + amp * np.sin(tp * i / IM) * np.sin(tp * k / KM)
    z = k * dz + amp * np.sin(tp * i / IM) * np.sin(tp * j / JM)
    return x.astype(np.float64), y.astype(np.float64), z.astype(np.float64)


def stretched_skewed_box(IM, JM, KM, half=(1.0, 1.0, 1.0), stretch=1.5, skew=0.05):
    """Box [-h, h]^3 clustered toward the centre by the inverse-tanh map
    x = atanh(tanh(s) (2 xi - 1)) / s, then skewed by
    x += skew * h * sin(pi y/h) sin(pi z/h) (and cyclically for y, z)."""
    def axis(n, h):
        e = np.linspace(-1.0, 1.0, n)
        return h * np.arctanh(np.tanh(stretch) * e) / stretch
    ax = axis(IM, half[0])
    ay = axis(JM, half[1])
    az = axis(KM, half[2])
    z0, y0, x0 = np.meshgrid(az, ay, ax, indexing="ij")
    hx, hy, hz = half
    x = x0 + skew * hx * np.sin(np.pi * y0 / hy) * np.sin(np.pi * z0 / hz)
    y = y0 + skew * hy * np.sin(np.pi * z0 / hz) * np.sin(np.pi * x0 / hx)
    z = z0 + skew * hz * np.sin(np.pi * x0 / hx) * np.sin(np.pi * y0 / hy)
    return x, y, z


def skewed_channel(IM, JM, KM, L=(1.0, 1.0, 0.5), skew=0.05):
    """Uniform box [0,Lx]x[0,Ly]x[0,Lz] with a 5% sinusoidal skew."""
    k, j, i = np.meshgrid(np.linspace(0, 1, KM), np.linspace(0, 1, JM), np.linspace(0, 1, IM), indexing="ij")
    x = L[0] * (i + skew * np.sin(2 * np.pi * j) * np.sin(np.pi * k))
    y = L[1] * (j + skew * np.sin(2 * np.pi * i) * np.sin(np.pi * k))
    z = L[2] * (k + skew * np.sin(np.pi * i) * np.sin(np.pi * j))
    return x, y, z


def naca0012_ogrid(IM, JM, KM, first=1.0e-5, far=20.0, span=0.1):
    """O-grid around a closed-trailing-edge NACA 0012 of unit chord.  i runs from
    just below the trailing edge along the lower, then the upper surface
    (parameter angles offset by half a cell so i = 0 and IM-1 are distinct points
    either side of the edge); j runs outward along straight surface normals with
    geometric spacing, first cell `first` chords, last point `far` chords out;
    k is spanwise.  The profile is convex, so the normals never cross and the
    grid is right-handed (J > 0)."""
    dth = 2.0 * np.pi / IM
    th = np.linspace(0.5 * dth, 2.0 * np.pi - 0.5 * dth, IM)

    def surf(t):
        xs = 0.5 * (1.0 + np.cos(t))
        yt = 5 * 0.12 * (0.2969 * np.sqrt(xs) - 0.1260 * xs - 0.3516 * xs ** 2 + 0.2843 * xs ** 3
                         - 0.1036 * xs ** 4)
        return xs, np.where(t <= np.pi, -yt, yt)

    xs, ys = surf(th)
    h = 1e-6
    xa, ya = surf(th - h)
    xb, yb = surf(th + h)
    tx, ty = xb - xa, yb - ya
    nrm = np.hypot(tx, ty)
    nx, ny = -ty / nrm, tx / nrm  # outward normal for this orientation
    # geometric ratio r with first * (r^(JM-1) - 1)/(r - 1) = far
    lo, hi = 1.0 + 1e-9, 2.0
    for _ in range(200):
        r = 0.5 * (lo + hi)
        if first * (r ** (JM - 1) - 1) / (r - 1) > far:
            hi = r
        else:
            lo = r
    d = first * (r ** np.arange(JM) - 1) / (r - 1)
    x2 = xs[None, :] + d[:, None] * nx[None, :]
    y2 = ys[None, :] + d[:, None] * ny[None, :]
    zk = np.linspace(0.0, span, KM)
    x = np.broadcast_to(x2, (KM, JM, IM)).copy()
    y = np.broadcast_to(y2, (KM, JM, IM)).copy()
    z = np.broadcast_to(zk[:, None, None], (KM, JM, IM)).copy()
    return x, y, z, r


def naca0012_ogrid_blend(P, JM, KM, first=1.0e-5, far=20.0, span=0.1):
    """Periodic O-grid around the closed-trailing-edge NACA 0012 for the
    wrap-around boundary mode: P points around the profile at the parameter
    angles of naca0012_ogrid, each j line running straight from the surface
    point to the point at the same angle on the circle of radius `far` about
    mid-chord, with the geometric spacing of naca0012_ogrid (first cell
    `first` of the line length).  Unlike surface normals, which turn by almost
    180 degrees between the last and the first point at the trailing edge,
    these lines stay nearly parallel across the seam, so the cells there are as
    regular as elsewhere."""
    dth = 2.0 * np.pi / P
    th = np.linspace(0.5 * dth, 2.0 * np.pi - 0.5 * dth, P)
    xs = 0.5 * (1.0 + np.cos(th))
    yt = 5 * 0.12 * (0.2969 * np.sqrt(xs) - 0.1260 * xs - 0.3516 * xs ** 2 + 0.2843 * xs ** 3 - 0.1036 * xs ** 4)
    ys = np.where(th <= np.pi, -yt, yt)
    xf, yf = 0.5 + far * np.cos(th), -far * np.sin(th)
    lo, hi = 1.0 + 1e-9, 2.0
    for _ in range(200):
        r = 0.5 * (lo + hi)
        if first * (r ** (JM - 1) - 1) / (r - 1) > far:
            hi = r
        else:
            lo = r
    f = (r ** np.arange(JM) - 1) / (r ** (JM - 1) - 1)
    x2 = xs[None, :] + f[:, None] * (xf - xs)[None, :]
    y2 = ys[None, :] + f[:, None] * (yf - ys)[None, :]
    zk = np.linspace(0.0, span, KM)
    x = np.broadcast_to(x2, (KM, JM, P)).copy()
    y = np.broadcast_to(y2, (KM, JM, P)).copy()
    z = np.broadcast_to(zk[:, None, None], (KM, JM, P)).copy()
    return x, y, z


def _naca_half_thickness(x):
    return 5 * 0.12 * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x ** 2 + 0.2843 * x ** 3 - 0.1036 * x ** 4)


def _naca_half_thickness_dx(x):
    return 5 * 0.12 * (0.14845 / np.sqrt(x) - 0.1260 - 0.7032 * x + 0.8529 * x ** 2 - 0.4144 * x ** 3)


def naca0012_rounded_surface(P, te_radius=2.0e-3, cluster=0.9):
    """P points around the NACA 0012 whose sharp trailing edge is replaced by
    the circular arc of radius te_radius tangent to both surfaces (centre on
    the chord line, tangent where yt * sqrt(1 + yt'^2) = te_radius).  Point 0
    sits on the rounded edge; the points run along the lower surface to the
    leading edge and back along the upper one, spaced in arc length s(u) =
    S (u - cluster sin(4 pi u) / (4 pi)), u = i/P, so the spacing at both
    edges is 1 - cluster of the mean."""
    lo, hi = 0.9, 1.0 - 1e-12
    for _ in range(200):  # tangency abscissa
        m = 0.5 * (lo + hi)
        if _naca_half_thickness(m) * np.sqrt(1 + _naca_half_thickness_dx(m) ** 2) > te_radius:
            lo = m
        else:
            hi = m
    xt = lo
    xc = xt + _naca_half_thickness(xt) * _naca_half_thickness_dx(xt)
    phi = np.arctan2(_naca_half_thickness(xt), xt - xc)
    beta = np.linspace(0.0, np.pi, 20001)
    xs = 0.5 * (1.0 - np.cos(beta)) * xt
    arc = np.linspace(0.0, phi, 400)
    lower_arc = np.stack([xc + te_radius * np.cos(arc), -te_radius * np.sin(arc)], 1)
    lower = np.stack([xs[::-1][1:], -_naca_half_thickness(xs[::-1][1:])], 1)
    upper = np.stack([xs[1:], _naca_half_thickness(xs[1:])], 1)
    upper_arc = np.stack([xc + te_radius * np.cos(arc[::-1][1:]), te_radius * np.sin(arc[::-1][1:])], 1)
    closed = np.vstack([lower_arc, lower, upper, upper_arc])  # ends back on the edge point
    s = np.concatenate([[0.0], np.cumsum(np.hypot(*np.diff(closed, axis=0).T))])
    u = np.arange(P) / P
    st = s[-1] * (u - cluster * np.sin(4 * np.pi * u) / (4 * np.pi))
    return np.interp(st, s, closed[:, 0]), np.interp(st, s, closed[:, 1])


def naca0012_ogrid_marched(P, JM, KM, first=1.0e-5, far=20.0, span=0.1, te_radius=2.0e-3, smooth=0.3):
    """Periodic O-grid around the NACA 0012 with a rounded trailing edge
    (naca0012_rounded_surface), marched outward layer by layer: each layer
    steps along its own unit normals (central differences around the closed
    line), smoothed along the layer by 2 + 2j Jacobi sweeps of weight
    `smooth`, with the geometric spacing of naca0012_ogrid (first cell
    `first`, `far` chords in all).  The lines leave the wall within a few
    degrees of its normal; outward the smoothing fans them out evenly around
    the trailing edge, so
    the Jacobian stays positive at the full 384 x 128 size, where straight
    normal lines from the rounded edge give negative Jacobians in the wake
    fan."""
    x0, y0 = naca0012_rounded_surface(P, te_radius)
    lo, hi = 1.0 + 1e-9, 2.0
    for _ in range(200):
        r = 0.5 * (lo + hi)
        if first * (r ** (JM - 1) - 1) / (r - 1) > far:
            hi = r
        else:
            lo = r
    d = first * (r ** np.arange(JM) - 1) / (r - 1)
    X = np.zeros((JM, P))
    Y = np.zeros((JM, P))
    X[0], Y[0] = x0, y0
    for j in range(JM - 1):
        tx = np.roll(X[j], -1) - np.roll(X[j], 1)
        ty = np.roll(Y[j], -1) - np.roll(Y[j], 1)
        n = np.hypot(tx, ty)
        nx, ny = -ty / n, tx / n
        for _ in range(2 + 2 * j):
            nx = nx + smooth * (np.roll(nx, 1) + np.roll(nx, -1) - 2 * nx)
            ny = ny + smooth * (np.roll(ny, 1) + np.roll(ny, -1) - 2 * ny)
            n = np.hypot(nx, ny)
            nx, ny = nx / n, ny / n
        X[j + 1] = X[j] + (d[j + 1] - d[j]) * nx
        Y[j + 1] = Y[j] + (d[j + 1] - d[j]) * ny
    zk = np.linspace(0.0, span, KM)
    x = np.broadcast_to(X, (KM, JM, P)).copy()
    y = np.broadcast_to(Y, (KM, JM, P)).copy()
    z = np.broadcast_to(zk[:, None, None], (KM, JM, P)).copy()
    return x, y, z


def ogrid_wrap(a, wrap=4):
    """The block layout of the O-grid boundary mode (bc_mode = 3): the
    periodic line of P points along i (last axis) stored with `wrap` copies of
    the points across the seam on either side, P + 2*wrap points in all."""
    return np.concatenate([a[..., -wrap:], a, a[..., :wrap]], axis=-1)


# ---------------------------------------------------------------- initial states
def isentropic_vortex(xg, yg, Mach, beta, xc, yc, R, gamma=1.4, u_dir=(1.0, 0.0)):
    """Isentropic vortex of strength beta (in units of the free-stream sound
    speed) and Gaussian radius R advected by a free stream of Mach number Mach,
    returned in the reference's units (|u_inf| = 1, p_inf = 1/(gamma M^2))."""
    dx, dy = (xg - xc) / R, (yg - yc) / R
    r2 = dx * dx + dy * dy
    f = np.exp(0.5 * (1.0 - r2))
    U = Mach * np.sqrt(gamma)  # free-stream speed in sound-speed units (c_inf = sqrt(gamma), p_inf = rho_inf = 1)
    ua = U * u_dir[0] - beta / (2 * np.pi) * dy * f
    va = U * u_dir[1] + beta / (2 * np.pi) * dx * f
    T = 1.0 - (gamma - 1.0) * beta ** 2 / (8.0 * gamma * np.pi ** 2) * np.exp(1.0 - r2)
    rho = T ** (1.0 / (gamma - 1.0))
    p = rho * T
    return rho, ua / U, va / U, np.zeros_like(rho), p / (U * U)


def case_vortex(IM=64, JM=32, KM=16, nsteps=100, CFL=0.5, Mach=0.5):
    """Isentropic vortex case: isentropic vortex (strength 5, centre (3, 2.5), radius 1) at
    Mach 0.5 on the perturbed 10 x 5 x 2.5 box; 100 steps at CFL 0.5.  Reference
    boundary mode: i faces pressure-reset extrapolation, j faces held at the
    initial state (i_begin = 1, i_end = 0), k faces zero-gradient."""
    x, y, z = perturbed_box(IM, JM, KM)
    xg, yg = ghost_extend(x), ghost_extend(y)
    g = 1.4
    rho, u, v, w, p = isentropic_vortex(xg, yg, Mach, 5.0, 3.0, 2.5, 1.0, g)
    Q = conservative(rho, u, v, w, p, g)
    params = dict(CFL=CFL, Mach=Mach, gamma=g, i_begin=1, i_end=0, Re=1.0e4, Pr=0.72, T_inf=288.15)
    return Case("vortex", x, y, z, params, Q, t_end=100.0, nsteps=nsteps)


def case_naca(IM=384, JM=128, KM=4, nsteps=2000, CFL=0.8, first=1.0e-5):
    """NACA 0012 case: viscous NACA 0012 O-grid, M 0.8, AoA 1.25 deg, Re 5e4, Pr 0.72,
    Sutherland with T_inf = 288.15 K, free-stream start.  Reference boundary
    mode: wall on the whole j = 0 face (i_begin = 1, i_end = IM).  Small test
    grids use a larger first cell: with 1e-5 chords and few points around the
    profile, the impulsive start blows up at the leading edge within ~10 steps
    in the reference build and in the oracle alike."""
    x, y, z, _ = naca0012_ogrid(IM, JM, KM, first=first)
    params = dict(CFL=CFL, Mach=0.8, angle_attack=1.25, Re=5.0e4, Pr=0.72, Pr_t=0.9, T_inf=288.15, gamma=1.4,
                  i_begin=1, i_end=IM, viscous=True)
    return Case("naca", x, y, z, params, None, t_end=1.0e6, nsteps=nsteps)


def case_naca_ogrid(P=384, JM=128, KM=4, nsteps=2000, CFL=0.8, first=1.0e-5, viscous=True, grid="blend",
                    start="freestream"):
    """NACA 0012 case with its own boundaries (bc_mode = 3, BC_OGRID): an
    O-grid of P points around the profile, wrapped periodically in i (stored
    with 4 copied points either side, IM = P + 8), adiabatic no-slip wall on
    j = 0 (slip when inviscid), characteristic far field on j = JM-1; M 0.8,
    AoA 1.25 deg, Re 5e4.  grid "blend": naca0012_ogrid_blend (sharp edge,
    straight lines to a far circle; regular on small grids with a coarse first
    cell), "marched": naca0012_ogrid_marched (rounded edge, wall-normal
    marched lines; valid at the full 384 x 128 size with a 1e-5 first cell).
    start "freestream": the reference's impulsive start (Q0 None: the free
    stream everywhere); "potential": the started flow of naca_started_state,
    with the viscous divergence taken at the node (vis_divergence 1) and the
    full viscous time-step limit (dt_viscous 1).  On the wall-resolved grid the
    impulsive start expands to vacuum round the rounded trailing edge within
    ~15 steps, the reference's shifted divergence placement grows a
    grid-scale oscillation along the wall within ~40, and the reference's
    viscous time-step term vanishes where the flow is at rest."""
    gen = {"blend": naca0012_ogrid_blend, "marched": naca0012_ogrid_marched}[grid]
    x, y, z = (ogrid_wrap(a) for a in gen(P, JM, KM, first=first))
    params = dict(CFL=CFL, Mach=0.8, angle_attack=1.25, Re=5.0e4, Pr=0.72, Pr_t=0.9, T_inf=288.15, gamma=1.4,
                  i_begin=1, i_end=P + 8, viscous=viscous, bc_mode=3)
    Q0 = None
    if start == "potential":
        Q0 = naca_started_state(x, y, params["Mach"], params["angle_attack"], params["gamma"])
        if viscous:
            params.update(vis_divergence=1, dt_viscous=1)
    elif start != "freestream":
        raise ValueError(f"unknown start {start!r}")
    return Case("naca_ogrid", x, y, z, params, Q0, t_end=1.0e6, nsteps=nsteps)


def case_blast(IM=384, JM=384, KM=384, t_end=0.05, CFL=0.5):
    """Blast case: spherical blast (p = 10 inside r < 0.1, 0.1 outside, rho = 1,
    at rest) on the centre-clustered (stretch 1.5), 5%-skewed [-1,1]^3 box.
    Mach is chosen so that p_inf = 1/(gamma M^2) = 0.1, the ambient pressure
    the i-face boundary resets to."""
    x, y, z = stretched_skewed_box(IM, JM, KM)
    xg, yg, zg = ghost_extend(x), ghost_extend(y), ghost_extend(z)
    g = 1.4
    r2 = xg * xg + yg * yg + zg * zg
    p = np.where(r2 < 0.01, 10.0, 0.1)
    rho = np.ones_like(p)
    zero = np.zeros_like(p)
    Q = conservative(rho, zero, zero, zero, p, g)
    Mach = float(np.sqrt(1.0 / (g * 0.1)))
    params = dict(CFL=CFL, Mach=Mach, gamma=g, i_begin=1, i_end=0)
    return Case("blast", x, y, z, params, Q, t_end=t_end, nsteps=100000)


def case_batch(nblocks=64, seed=0, size_lo=(32, 32, 32), size_hi=(128, 64, 64), viscous=True, CFL=0.5):
    """Batched-blocks case: independent blocks for the batched form.  Per block (seeded
    draw): grid points uniform in size_lo..size_hi per dimension, free-stream
    Mach uniform in [0.3, 2.0], Reynolds number uniform in [1e3, 1e5], an
    isentropic vortex of strength uniform in [1, 5] at a random position of
    the middle half of the perturbed 10 x 5 x 2.5 box; viscous by default.
    Far-field boundaries on every face (bc_mode = 1, BC_FARFIELD: boundary and
    ghost nodes hold the initial state), as the configuration asks.
    Returns the list of Cases and the draw."""
    rng = np.random.default_rng(seed)
    out, draw = [], []
    for b in range(nblocks):
        IM, JM, KM = (int(rng.integers(lo, hi + 1)) for lo, hi in zip(size_lo, size_hi))
        Mach = float(rng.uniform(0.3, 2.0))
        Re = float(rng.uniform(1.0e3, 1.0e5))
        beta = float(rng.uniform(1.0, 5.0))
        xc, yc = float(rng.uniform(2.5, 7.5)), float(rng.uniform(1.25, 3.75))
        x, y, z = perturbed_box(IM, JM, KM)
        xg, yg = ghost_extend(x), ghost_extend(y)
        g = 1.4
        Q = conservative(*isentropic_vortex(xg, yg, Mach, beta, xc, yc, 1.0, g), g)
        params = dict(CFL=CFL, Mach=Mach, gamma=g, i_begin=1, i_end=0, Re=Re, Pr=0.72, T_inf=288.15,
                      viscous=viscous, bc_mode=1)
        out.append(Case(f"batch{b}", x, y, z, params, Q, t_end=1.0e30, nsteps=500))
        draw.append(dict(shape=(IM, JM, KM), Mach=Mach, Re=Re, beta=beta, centre=(xc, yc)))
    return out, draw


def case_shock_vortex(IM=256, JM=256, KM=128, nsteps=100, CFL=0.5, Ms=1.2, eps=0.3, rc=0.075):
    """Shock/vortex case: a stationary Mach 1.2 normal shock at x = 0.5 of the 5%-skewed
    [0,1]x[0,1]x[0,0.5] box, with an isentropic vortex (strength 0.3, radius
    0.075, centre (0.25, 0.5)) in the upstream flow moving into it."""
    x, y, z = skewed_channel(IM, JM, KM)
    xg, yg = ghost_extend(x), ghost_extend(y)
    g = 1.4
    # upstream (reference units): rho = 1, u = 1, p = 1/(gamma Ms^2)
    p1 = 1.0 / (g * Ms * Ms)
    r21 = ((g + 1) * Ms * Ms) / ((g - 1) * Ms * Ms + 2)
    p21 = 1 + 2 * g / (g + 1) * (Ms * Ms - 1)
    rho2, u2, p2 = r21, 1.0 / r21, p1 * p21
    # vortex: u_theta = eps * c1 * tau * exp(a (1 - tau^2)), Jiang & Shu form, a = 0.204
    a = 0.204
    xc, yc = 0.25, 0.5
    dx, dy = xg - xc, yg - yc
    rr = np.sqrt(dx * dx + dy * dy)
    tau = rr / rc
    c1 = np.sqrt(g * p1 / 1.0)
    ut = eps * c1 * tau * np.exp(a * (1.0 - tau * tau))
    with np.errstate(invalid="ignore", divide="ignore"):
        sn = np.where(rr > 0, dy / rr, 0.0)
        cs = np.where(rr > 0, dx / rr, 0.0)
    T1 = p1 / 1.0
    T = T1 - (g - 1) * (eps * c1) ** 2 / (4 * a * g) * np.exp(2 * a * (1 - tau * tau)) * (1.0 / 1.0)
    rho_v = (T / T1) ** (1 / (g - 1))
    p_v = p1 * (T / T1) ** (g / (g - 1))
    up = xg < 0.5
    rho = np.where(up, rho_v, rho2)
    u = np.where(up, 1.0 - ut * sn, u2)
    v = np.where(up, ut * cs, 0.0)
    w = np.zeros_like(rho)
    p = np.where(up, p_v, p2)
    Q = conservative(rho, u, v, w, p, g)
    params = dict(CFL=CFL, Mach=Ms, gamma=g, i_begin=1, i_end=0)
    return Case("shock_vortex", x, y, z, params, Q, t_end=1.0e6, nsteps=nsteps)


# ---------------------------------------------------------------- started flow
def panel_flow(xs, ys, alpha_deg):
    """Incompressible potential flow of unit free-stream speed at angle
    alpha_deg past the closed polygon (xs, ys) (points in clockwise order, the
    trailing edge at point 0), by the Hess-Smith panel method: a constant
    source density per panel and one vortex density shared by all panels,
    fixed by zero normal velocity at the panel midpoints and the Kutta
    condition (equal and opposite tangential velocity on the two panels that
    meet at the trailing edge).  Returns a function (x, y) -> (u, v) for points
    off the surface."""
    P = len(xs)
    x0, y0 = np.asarray(xs, float), np.asarray(ys, float)
    x1, y1 = np.roll(x0, -1), np.roll(y0, -1)
    th = np.arctan2(y1 - y0, x1 - x0)
    ct, st = np.cos(th), np.sin(th)
    xm, ym = 0.5 * (x0 + x1), 0.5 * (y0 + y1)
    al = np.deg2rad(alpha_deg)
    ua, va = np.cos(al), np.sin(al)

    def unit(px, py):
        """Velocities at points (px, py) (shape (n,)) induced by unit source
        and unit vortex density on every panel: (us, vs, uv, vv), each (n, P)."""
        rsx, rsy = x0[None, :] - px[:, None], y0[None, :] - py[:, None]
        rex, rey = x1[None, :] - px[:, None], y1[None, :] - py[:, None]
        beta = np.arctan2(rsx * rey - rsy * rex, rsx * rex + rsy * rey)
        lg = 0.5 * np.log((rsx * rsx + rsy * rsy) / (rex * rex + rey * rey))
        # panel frame: source (lg, beta)/(2 pi), vortex (beta, -lg)/(2 pi) rotated
        # by +90 degrees from it (clockwise circulation positive)
        sl, sn = lg / (2 * np.pi), beta / (2 * np.pi)
        us, vs = sl * ct - sn * st, sl * st + sn * ct
        uv, vv = sn * ct + sl * st, sn * st - sl * ct
        return us, vs, uv, vv

    us, vs, uv, vv = unit(xm, ym)
    idx = np.arange(P)
    # self-influence at a panel's own midpoint, outer side: beta = pi
    us[idx, idx], vs[idx, idx] = -0.5 * st, 0.5 * ct
    uv[idx, idx], vv[idx, idx] = 0.5 * ct, 0.5 * st
    nx, ny = -st, ct
    A = np.zeros((P + 1, P + 1))
    A[:P, :P] = us * nx[:, None] + vs * ny[:, None]
    A[:P, P] = (uv * nx[:, None] + vv * ny[:, None]).sum(1)
    b = np.zeros(P + 1)
    b[:P] = -(ua * nx + va * ny)
    for i in (0, P - 1):  # Kutta: tangential velocities on panels 0 and P-1 sum to zero
        A[P, :P] += us[i] * ct[i] + vs[i] * st[i]
        A[P, P] += (uv[i] * ct[i] + vv[i] * st[i]).sum()
        b[P] -= ua * ct[i] + va * st[i]
    sol = np.linalg.solve(A, b)
    q, g = sol[:P], sol[P]

    def velocity(px, py):
        px, py = np.asarray(px, float).ravel(), np.asarray(py, float).ravel()
        u = np.empty_like(px)
        v = np.empty_like(px)
        for s in range(0, px.size, 4096):
            e = slice(s, s + 4096)
            a, bb, c, d = unit(px[e], py[e])
            u[e] = ua + a @ q + g * c.sum(1)
            v[e] = va + bb @ q + g * d.sum(1)
        return u, v

    return velocity


def naca_started_state(x, y, Mach, alpha_deg, gamma=1.4, wrap=4):
    """Started-flow initial state of the wrapped NACA O-grid block (x, y of
    shape (KM, JM, P + 2 wrap), j = 0 the wall): the compressible free stream
    replaced by the incompressible potential flow past the profile with the
    Kutta condition (panel_flow over the j = 0 line), density and pressure from
    the isentropic relations of the local speed (T / T_inf = 1 + (gamma-1)/2
    M^2 (1 - |u|^2), floored at 0.5).  Nodes closer to the wall than half the
    local surface spacing take the tangential velocity of the first node along
    their j line that is not; the wall nodes take zero (the no-slip boundary
    condition sets them anyway).  Returns the ghosted AoS state (ghost layers
    copied from the nearest node; every boundary mode rewrites them)."""
    xs, ys = x[0, 0, wrap:-wrap], y[0, 0, wrap:-wrap]
    vel = panel_flow(xs, ys, alpha_deg)
    X, Y = x[0], y[0]
    JM, IM = X.shape
    u, v = vel(X[1:], Y[1:])
    u, v = u.reshape(JM - 1, IM), v.reshape(JM - 1, IM)
    # surface spacing at each i and the first usable node of each j line
    sx, sy = X[0], Y[0]
    ds = 0.5 * (np.hypot(np.roll(sx, -1) - sx, np.roll(sy, -1) - sy) +
                np.hypot(sx - np.roll(sx, 1), sy - np.roll(sy, 1)))
    d = np.hypot(X - sx[None, :], Y - sy[None, :])
    tx, ty = np.roll(sx, -1) - np.roll(sx, 1), np.roll(sy, -1) - np.roll(sy, 1)
    tn = np.hypot(tx, ty)
    tx, ty = tx / tn, ty / tn
    for i in range(IM):
        jf = int(np.argmax(d[1:, i] >= 0.5 * ds[i]))  # index into rows 1..JM-1
        ut = u[jf, i] * tx[i] + v[jf, i] * ty[i]
        u[:jf, i], v[:jf, i] = ut * tx[i], ut * ty[i]
    U = np.zeros((JM, IM))
    V = np.zeros((JM, IM))
    U[1:], V[1:] = u, v
    T = np.maximum(1.0 + 0.5 * (gamma - 1.0) * Mach ** 2 * (1.0 - (U * U + V * V)), 0.5)
    rho = T ** (1.0 / (gamma - 1.0))
    p = T ** (gamma / (gamma - 1.0)) / (gamma * Mach ** 2)
    KM = x.shape[0]
    f = [np.broadcast_to(a, (KM, JM, IM)) for a in (rho, U, V, np.zeros_like(U), p)]
    Q = conservative(*f, gamma)
    return np.pad(Q, ((NG, NG), (NG, NG), (NG, NG), (0, 0)), mode="edge")
