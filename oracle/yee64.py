"""FP64 host reference of the Yee branch (test infrastructure: the checker of
the library's Yee step, never part of the product).

Restates, in float64 numpy, MaxwellSimulation::step_at
(include/pic/simulation_maxwell.hpp:52-110) for the periodic feature set
(no delta-f, no relativistic push, uniform B0, no boundaries, no antenna):

  1. B half step, k_faraday (yee2d.hpp:70-81):  B -= dt/2 curl E
  2. staggered CIC gather of E (+ pump) and B (+ B0), Boris kick-rotate-kick,
     x1 = x0 + u dt / dx                          (yee2d.hpp:99-112, 141-305)
  3. Esirkepov current over the 4 x 4 union stencil {ib-1..ib+2} x {jb-1..jb+2},
     ib = floor(min(x0, x1)), node shapes S = max(0, 1 - |x - p|):
       Jx(i+1/2, j) = -(q w / (dt dy)) prefix_i sum DSx(i) (Sy0 + DSy/2)
       Jy(i, j+1/2) = -(q w / (dt dx)) prefix_j sum DSy(j) (Sx0 + DSx/2)
       Jz(i, j)     =  (q w vz / (dx dy)) (Sx0 Sy0 + (DSx Sy0 + Sx0 DSy)/2 + DSx DSy/3)
                                                  (yee2d.hpp:17-29, 307-355)
     then the periodic wrap of the positions (Particles::migrate), and jfilter
     passes of the binomial current filter
  4. B half step
  5. E full step, k_ampere (yee2d.hpp:84-97): E += dt (c^2 curl B - J)  (eps0 = 1)

Staggering (yee2d.hpp:8-11): Ex(i+1/2, j), Ey(i, j+1/2), Ez(i, j),
Bx(i, j+1/2), By(i+1/2, j), Bz(i+1/2, j+1/2); arrays [ny][nx], periodic.
"""
import numpy as np

# gather offsets (ox, oy) in cells of each component's lattice
OFFSETS = {"Ex": (0.5, 0.0), "Ey": (0.0, 0.5), "Ez": (0.0, 0.0),
           "Bx": (0.0, 0.5), "By": (0.5, 0.0), "Bz": (0.5, 0.5)}


class YeeCase:
    def __init__(self, nx, ny, Lx, Ly, dt, c, qm=-1.0, B0=(0.0, 0.0, 0.0), jfilter=0):
        """jfilter: passes of the binomial current filter [1,2,1] x [1,2,1] / 16
        after the deposit (k_binomial3x3, yee2d.hpp:471-487;
        simulation_maxwell.hpp:78-92)."""
        self.jfilter = jfilter
        self.nx, self.ny = nx, ny
        self.dx, self.dy = Lx / nx, Ly / ny
        self.dt, self.c2, self.qm = dt, c * c, qm
        self.B0 = np.asarray(B0, np.float64)
        self.f = {k: np.zeros((ny, nx)) for k in OFFSETS}
        self.J = {k: np.zeros((ny, nx)) for k in ("Jx", "Jy", "Jz")}

    # ---- fields ---------------------------------------------------------------
    def faraday(self, dt2):
        f = self.f
        ez_xp, ez_yp = np.roll(f["Ez"], -1, 1), np.roll(f["Ez"], -1, 0)
        ex_yp, ey_xp = np.roll(f["Ex"], -1, 0), np.roll(f["Ey"], -1, 1)
        f["Bx"] = f["Bx"] - dt2 * (ez_yp - f["Ez"]) / self.dy
        f["By"] = f["By"] + dt2 * (ez_xp - f["Ez"]) / self.dx
        f["Bz"] = f["Bz"] - dt2 * ((ey_xp - f["Ey"]) / self.dx - (ex_yp - f["Ex"]) / self.dy)

    def ampere(self):
        f, J, dt, c2 = self.f, self.J, self.dt, self.c2
        bz_ym, bz_xm = np.roll(f["Bz"], 1, 0), np.roll(f["Bz"], 1, 1)
        bx_ym, by_xm = np.roll(f["Bx"], 1, 0), np.roll(f["By"], 1, 1)
        f["Ex"] = f["Ex"] + dt * (c2 * (f["Bz"] - bz_ym) / self.dy - J["Jx"])
        f["Ey"] = f["Ey"] + dt * (-c2 * (f["Bz"] - bz_xm) / self.dx - J["Jy"])
        f["Ez"] = f["Ez"] + dt * (c2 * ((f["By"] - by_xm) / self.dx - (f["Bx"] - bx_ym) / self.dy) - J["Jz"])

    # ---- particles ------------------------------------------------------------
    def gather(self, name, x, y):
        ox, oy = OFFSETS[name]
        xs, ys = x - ox, y - oy
        i0, j0 = np.floor(xs).astype(np.int64), np.floor(ys).astype(np.int64)
        fx, fy = xs - i0, ys - j0
        a = self.f[name]
        i0, j0 = i0 % self.nx, j0 % self.ny
        i1, j1 = (i0 + 1) % self.nx, (j0 + 1) % self.ny
        return ((1 - fx) * (1 - fy) * a[j0, i0] + fx * (1 - fy) * a[j0, i1] + (1 - fx) * fy * a[j1, i0]
                + fx * fy * a[j1, i1])

    @staticmethod
    def shape4(x, b):
        """S over the nodes b-1 .. b+2: [4][n]."""
        p = b[None, :] - 1 + np.arange(4)[:, None]
        d = np.abs(x[None, :] - p)
        return np.where(d < 1.0, 1.0 - d, 0.0)

    def push_deposit(self, p):
        x0, y0 = p["x"].astype(np.float64), p["y"].astype(np.float64)
        E = [self.gather(k, x0, y0) for k in ("Ex", "Ey", "Ez")]
        B = [self.gather(k, x0, y0) + self.B0[d] for d, k in enumerate(("Bx", "By", "Bz"))]
        qmh = self.qm * 0.5 * self.dt
        u = [p[k].astype(np.float64) + qmh * E[d] for d, k in enumerate(("ux", "uy", "uz"))]
        t = [qmh * b for b in B]
        s = [2.0 * tt / (1.0 + t[0] ** 2 + t[1] ** 2 + t[2] ** 2) for tt in t]
        up = [u[0] + (u[1] * t[2] - u[2] * t[1]), u[1] + (u[2] * t[0] - u[0] * t[2]),
              u[2] + (u[0] * t[1] - u[1] * t[0])]
        u = [u[0] + (up[1] * s[2] - up[2] * s[1]), u[1] + (up[2] * s[0] - up[0] * s[2]),
             u[2] + (up[0] * s[1] - up[1] * s[0])]
        u = [u[d] + qmh * E[d] for d in range(3)]
        x1 = x0 + u[0] * self.dt / self.dx
        y1 = y0 + u[1] * self.dt / self.dy
        qw = self.qm * p["w"].astype(np.float64)
        self.esirkepov(x0, y0, x1, y1, qw, u[2])
        q = dict(p)
        q["ux"], q["uy"], q["uz"] = u
        q["x"], q["y"] = np.mod(x1, self.nx), np.mod(y1, self.ny)
        return q

    def esirkepov(self, x0, y0, x1, y1, qw, vz):
        nx, ny = self.nx, self.ny
        ib = np.floor(np.minimum(x0, x1)).astype(np.int64)
        jb = np.floor(np.minimum(y0, y1)).astype(np.int64)
        Sx0, Sx1 = self.shape4(x0, ib), self.shape4(x1, ib)
        Sy0, Sy1 = self.shape4(y0, jb), self.shape4(y1, jb)
        DSx, DSy = Sx1 - Sx0, Sy1 - Sy0
        cJx = -qw / (self.dt * self.dy)
        cJy = -qw / (self.dt * self.dx)
        cJz = qw * vz / (self.dx * self.dy)
        J = {k: np.zeros(ny * nx) for k in ("Jx", "Jy", "Jz")}
        wx = np.cumsum(DSx[:, None, :] * (Sy0 + 0.5 * DSy)[None, :, :], axis=0)     # [ni][nj][n]
        wy = np.cumsum(DSy[None, :, :] * (Sx0 + 0.5 * DSx)[:, None, :], axis=1)
        wz = (Sx0[:, None, :] * Sy0[None, :, :] + 0.5 * (DSx[:, None, :] * Sy0[None, :, :]
                                                         + Sx0[:, None, :] * DSy[None, :, :])
              + (1.0 / 3.0) * DSx[:, None, :] * DSy[None, :, :])
        for ni in range(4):
            for nj in range(4):
                cell = ((jb - 1 + nj) % ny) * nx + (ib - 1 + ni) % nx
                J["Jx"] += np.bincount(cell, cJx * wx[ni, nj], minlength=nx * ny)
                J["Jy"] += np.bincount(cell, cJy * wy[ni, nj], minlength=nx * ny)
                J["Jz"] += np.bincount(cell, cJz * wz[ni, nj], minlength=nx * ny)
        self.J = {k: v.reshape(ny, nx) for k, v in J.items()}

    @staticmethod
    def binomial(a):
        """One pass of [1,2,1] x [1,2,1] / 16, periodic: sum w_di w_dj a(i+di, j+dj)."""
        w = (0.25, 0.5, 0.25)
        r = np.zeros_like(a)
        for dj in (-1, 0, 1):
            for di in (-1, 0, 1):
                r += w[di + 1] * w[dj + 1] * np.roll(np.roll(a, -dj, 0), -di, 1)
        return r

    # ---- step -----------------------------------------------------------------
    def step(self, p):
        self.faraday(0.5 * self.dt)
        p = self.push_deposit(p)
        for _ in range(self.jfilter):
            self.J = {k: self.binomial(v) for k, v in self.J.items()}
        self.faraday(0.5 * self.dt)
        self.ampere()
        return p

    def rho(self, x, y, w):
        """CIC node charge q w S / (dx dy) (k_rho_nodes, yee2d.hpp:489-507)."""
        nx, ny = self.nx, self.ny
        i0, j0 = np.floor(x).astype(np.int64), np.floor(y).astype(np.int64)
        fx, fy = x - i0, y - j0
        q = self.qm * w / (self.dx * self.dy)
        r = np.zeros(ny * nx)
        for di, wx in ((0, 1 - fx), (1, fx)):
            for dj, wy in ((0, 1 - fy), (1, fy)):
                r += np.bincount(((j0 + dj) % ny) * nx + (i0 + di) % nx, q * wx * wy, minlength=nx * ny)
        return r.reshape(ny, nx)
