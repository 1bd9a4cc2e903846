"""FP64 host reference for the gradient of the electrostatic step (test
infrastructure: the checker of aw_grad_es, never part of the product).

The reference has no adjoint. This module restates, in float64 and without the
fixed-point quantisation, the ES step the library runs, and its discrete
adjoint, so that the library's FP32 gradient has an FP64 reference, and the
FP64 reference itself is checked against central finite differences.

Forward (the reference's ES step, Simulation<Cfg>::step):
  rho   = CIC deposit of q_p = qm w_p / (dx dy)      include/pic/depositor.hpp:35-58
  E     = spectral Poisson, E_k = -i k rho_k/(eps0 k^2), k = 0 and Nyquist zeroed
                                                      include/pic/solver_es.hpp:40-78
  u'    = Boris: half kick, rotation about B0, half kick   include/pic/pusher.hpp:47-80
  x'    = wrap(x + u' dt/dx)                          include/pic/pusher.hpp:126-127,
                                                      include/pic/particles.hpp:294-315
  init: the field of x^0 and the half-step rollback u(-dt/2)
                                                      include/pic/simulation.hpp:56-70
Loss: 0.5 eps0 dx dy sum E^2 of the last step's field (Diagnostics ee,
include/pic/diagnostics.hpp:58-108).
"""
import numpy as np


class Case:
    def __init__(self, nx, ny, Lx, Ly, dt, qm=-1.0, eps0=1.0, B0=(0.0, 0.0, 0.0)):
        self.nx, self.ny, self.Lx, self.Ly = nx, ny, Lx, Ly
        self.dx, self.dy = Lx / nx, Ly / ny
        self.dt, self.qm, self.eps0 = dt, qm, eps0
        self.B0 = np.asarray(B0, np.float64)
        kx = 2.0 * np.pi / Lx * np.arange(nx // 2 + 1)
        m = np.arange(ny)
        m = np.where(m <= ny // 2, m, m - ny)
        ky = 2.0 * np.pi / Ly * m
        KX, KY = np.meshgrid(kx, ky)                     # [ny][nkx]
        k2 = KX * KX + KY * KY
        gr = np.where(k2 > 0, 1.0 / np.where(k2 > 0, eps0 * k2, 1.0), 0.0)
        nyq = np.zeros_like(k2, bool)
        if nx % 2 == 0:
            nyq[:, nx // 2] = True
        if ny % 2 == 0:
            nyq[ny // 2, :] = True
        keep = (~nyq).astype(np.float64)
        self.Kx = -1j * KX * gr * keep                   # E_d,k = K_d rho_k
        self.Ky = -1j * KY * gr * keep

    # ---- CIC ------------------------------------------------------------------
    def stencil(self, x, y):
        i0 = np.floor(x).astype(np.int64)
        j0 = np.floor(y).astype(np.int64)
        fx, fy = x - i0, y - j0
        i0 %= self.nx
        j0 %= self.ny
        i1, j1 = (i0 + 1) % self.nx, (j0 + 1) % self.ny
        return i0, j0, i1, j1, fx, fy

    def deposit(self, x, y, q):
        i0, j0, i1, j1, fx, fy = self.stencil(x, y)
        g = np.zeros(self.ny * self.nx)
        nx = self.nx
        np.add.at(g, j0 * nx + i0, q * (1 - fx) * (1 - fy))
        np.add.at(g, j0 * nx + i1, q * fx * (1 - fy))
        np.add.at(g, j1 * nx + i0, q * (1 - fx) * fy)
        np.add.at(g, j1 * nx + i1, q * fx * fy)
        return g.reshape(self.ny, self.nx)

    def gather(self, G, x, y):
        i0, j0, i1, j1, fx, fy = self.stencil(x, y)
        return ((1 - fx) * (1 - fy) * G[j0, i0] + fx * (1 - fy) * G[j0, i1]
                + (1 - fx) * fy * G[j1, i0] + fx * fy * G[j1, i1])

    def gather_grad(self, G, x, y):
        """(dG/dx, dG/dy) of the CIC interpolant at the particles (cell units)."""
        i0, j0, i1, j1, fx, fy = self.stencil(x, y)
        g00, g10, g01, g11 = G[j0, i0], G[j0, i1], G[j1, i0], G[j1, i1]
        ddx = (1 - fy) * (g10 - g00) + fy * (g11 - g01)
        ddy = (1 - fx) * (g01 - g00) + fx * (g11 - g10)
        return ddx, ddy

    # ---- solve and its transpose ------------------------------------------------
    def solve(self, rho):
        rk = np.fft.rfft2(rho)
        s = (self.ny, self.nx)
        return np.fft.irfft2(self.Kx * rk, s=s), np.fft.irfft2(self.Ky * rk, s=s)

    def solve_T(self, lEx, lEy):
        s = (self.ny, self.nx)
        return np.fft.irfft2(np.conj(self.Kx) * np.fft.rfft2(lEx) + np.conj(self.Ky) * np.fft.rfft2(lEy), s=s)

    # ---- Boris -------------------------------------------------------------------
    def rot_ts(self, qmh):
        t = qmh * self.B0
        s = 2.0 * t / (1.0 + t @ t)
        return t, s

    def boris(self, u, ex, ey, qmh):
        a = np.stack([qmh * ex, qmh * ey, np.zeros_like(ex)], axis=1)
        u1 = u + a
        t, s = self.rot_ts(qmh)
        up = u1 + np.cross(u1, t)
        u2 = u1 + np.cross(up, s)
        return u2 + a

    def rot_T(self, lam, qmh):
        """R^T lam for the rotation u -> u + (u + u x t) x s."""
        t, s = self.rot_ts(qmh)
        ls = np.cross(lam, s)
        return lam - ls + np.cross(ls, t)

    # ---- forward / backward ----------------------------------------------------------
    def forward(self, x, y, u, w, nsteps):
        """Initial state (x, y in cell units, u [n][3], w) -> (loss, trajectory)."""
        x, y, u = np.array(x, np.float64), np.array(y, np.float64), np.array(u, np.float64)
        q = self.qm / (self.dx * self.dy) * np.asarray(w, np.float64)
        qmh = self.qm * 0.5 * self.dt
        qmh_b = self.qm * 0.5 * (-0.5 * self.dt)
        ex, ey = self.solve(self.deposit(x, y, q))
        u = self.boris(u, self.gather(ex, x, y), self.gather(ey, x, y), qmh_b)
        traj = []
        for _ in range(nsteps):
            ex, ey = self.solve(self.deposit(x, y, q))
            traj.append((x.copy(), y.copy(), ex, ey))
            u = self.boris(u, self.gather(ex, x, y), self.gather(ey, x, y), qmh)
            x = np.mod(x + u[:, 0] * self.dt / self.dx, self.nx)
            y = np.mod(y + u[:, 1] * self.dt / self.dy, self.ny)
        ex, ey = traj[-1][2], traj[-1][3]
        loss = 0.5 * self.eps0 * self.dx * self.dy * float(np.sum(ex * ex + ey * ey))
        return loss, traj, q

    def gradient(self, x, y, u, w, nsteps):
        """(loss, dloss/du0 [n][3]) by the discrete adjoint of forward()."""
        loss, traj, q = self.forward(x, y, u, w, nsteps)
        n = len(q)
        qmh = self.qm * 0.5 * self.dt
        qmh_b = self.qm * 0.5 * (-0.5 * self.dt)
        cx, cy = self.dt / self.dx, self.dt / self.dy
        lx, ly, lu = np.zeros(n), np.zeros(n), np.zeros((n, 3))
        ext = self.eps0 * self.dx * self.dy
        for s in range(nsteps - 1, -1, -1):
            xs, ys, ex, ey = traj[s]
            lu3 = lu.copy()
            lu3[:, 0] += cx * lx
            lu3[:, 1] += cy * ly
            lu1 = self.rot_T(lu3, qmh)
            lEx = qmh * (lu3[:, 0] + lu1[:, 0])
            lEy = qmh * (lu3[:, 1] + lu1[:, 1])
            dxx, dxy = self.gather_grad(ex, xs, ys)
            dyx, dyy = self.gather_grad(ey, xs, ys)
            lx = lx + lEx * dxx + lEy * dyx
            ly = ly + lEx * dxy + lEy * dyy
            lu = lu1
            gEx = self.deposit(xs, ys, lEx)
            gEy = self.deposit(xs, ys, lEy)
            if s == nsteps - 1:
                gEx = gEx + ext * ex
                gEy = gEy + ext * ey
            lrho = self.solve_T(gEx, gEy)
            ddx, ddy = self.gather_grad(lrho, xs, ys)
            lx = lx + q * ddx
            ly = ly + q * ddy
        return loss, self.rot_T(lu, qmh_b)


def loss_at(case, x, y, u, w, nsteps):
    return case.forward(x, y, u, w, nsteps)[0]


def central_difference(case, x, y, u, w, nsteps, direction, h):
    """(L(u + h d) - L(u - h d)) / 2h in float64."""
    lp = loss_at(case, x, y, u + h * direction, w, nsteps)
    lm = loss_at(case, x, y, u - h * direction, w, nsteps)
    return (lp - lm) / (2.0 * h)
