"""FP64 host reference for the gradient of the Darwin step (test
infrastructure: the checker of aw_grad_darwin, never part of the product).

The reference has no adjoint. This module restates, in float64 and without the
fixed-point quantisation, the Darwin step the library runs, and its discrete
adjoint, so that the library's FP32 gradient has an FP64 reference; the FP64
reference itself is checked against central finite differences.

Forward step n (include/pic/simulation.hpp:80-84, 103-119; cell units, t = n dt):
  rho = D(x) q, J_d = D(x) (q u_d), amu_m = D(x) (q a_m(u))   depositor.hpp:161-270
        a(u) = (0.5 (ux^2 - uy^2), ux uy, uz ux, uz uy), q = qm w / (dx dy)
  E_L = -i k rho_k / (eps0 k^2), B = i (k x J_k) / (eps0 c^2 k^2)
                                                     solver_darwin.hpp:38-75
  Btot = B + B0                                      pump.hpp:59-66
  Fd = E_L + P(t)     (P: the pump, 1D in x)         pump.hpp:27-54
  dcu = D(x) (c_p (G(Fd)(x) + u x G(Btot)(x))), c_p = qm q_p
                                                     depositor.hpp:276-324
  E_T = -(dcu_k - i S(amu)_k)_T / (eps0 c^2 k^2 + n0),
        S = (kx a0 + ky a1, kx a1 - ky a0, kx a2 + ky a3)
                                                     solver_darwin.hpp:83-129
  E = E_L + E_T + P(t)                               solver_darwin.hpp:220-231
  push: Boris with e = G(E)(x), b = G(Btot)(x); x' = wrap(x + u' dt/dx)
                                                     pusher.hpp:103-109, 212-258
k = 0 and the Nyquist modes are zeroed in every solve. No half-step rollback
(the reference's Darwin init has none).
Loss: 0.5 eps0 dx dy sum (Ex^2 + Ey^2) of the last step's E (the ee
diagnostic of the run, diagnostics.hpp:58-108).
The pump amplitude enters as P = a P_nom; dL/da is taken at a = 1.
"""
import numpy as np


class DarwinCase:
    def __init__(self, nx, ny, Lx, Ly, dt, qm=-1.0, eps0=1.0, c=1.0, n0=1.0, B0=(0.0, 0.0, 0.0), pump=None):
        self.nx, self.ny, self.Lx, self.Ly = nx, ny, Lx, Ly
        self.dx, self.dy = Lx / nx, Ly / ny
        self.dt, self.qm, self.eps0, self.c, self.n0 = dt, qm, eps0, c, n0
        self.B0 = np.asarray(B0, np.float64)
        self.pump = pump
        kx = 2.0 * np.pi / Lx * np.arange(nx // 2 + 1)
        m = np.arange(ny)
        m = np.where(m <= ny // 2, m, m - ny)
        ky = 2.0 * np.pi / Ly * m
        KX, KY = np.meshgrid(kx, ky)                     # [ny][nkx]
        k2 = KX * KX + KY * KY
        pos = k2 > 0
        safe = np.where(pos, k2, 1.0)
        keep = np.ones_like(k2)
        if nx % 2 == 0:
            keep[:, nx // 2] = 0.0
        if ny % 2 == 0:
            keep[ny // 2, :] = 0.0
        keep = keep * pos
        self.KX, self.KY, self.k2, self.keep = KX, KY, safe, keep
        gE = keep / (eps0 * safe)
        gB = keep / (eps0 * c * c * safe)
        gT = keep / (eps0 * c * c * safe + n0)
        self.gE, self.gB, self.gT = gE, gB, gT

    # ---- CIC (the ES oracle's conventions) ---------------------------------------
    def stencil(self, x, y):
        i0 = np.floor(x).astype(np.int64)
        j0 = np.floor(y).astype(np.int64)
        fx, fy = x - i0, y - j0
        i0 %= self.nx
        j0 %= self.ny
        i1, j1 = (i0 + 1) % self.nx, (j0 + 1) % self.ny
        r0, r1 = j0 * self.nx, j1 * self.nx
        return (r0 + i0, r0 + i1, r1 + i0, r1 + i1), fx, fy

    def deposit(self, st, v):
        (c00, c10, c01, c11), fx, fy = st
        m = self.ny * self.nx
        gx, gy = 1.0 - fx, 1.0 - fy
        g = np.bincount(c00, v * gx * gy, minlength=m)
        g += np.bincount(c10, v * fx * gy, minlength=m)
        g += np.bincount(c01, v * gx * fy, minlength=m)
        g += np.bincount(c11, v * fx * fy, minlength=m)
        return g.reshape(self.ny, self.nx)

    def gather(self, G, st):
        (c00, c10, c01, c11), fx, fy = st
        G = G.reshape(-1)
        gx, gy = 1.0 - fx, 1.0 - fy
        return gx * gy * G[c00] + fx * gy * G[c10] + gx * fy * G[c01] + fx * fy * G[c11]

    def gather_grad(self, G, st):
        (c00, c10, c01, c11), fx, fy = st
        G = G.reshape(-1)
        g00, g10, g01, g11 = G[c00], G[c10], G[c01], G[c11]
        return (1.0 - fy) * (g10 - g00) + fy * (g11 - g01), (1.0 - fx) * (g01 - g00) + fx * (g11 - g10)

    # ---- spectral operators and their transposes -----------------------------------
    def _r2c(self, f):
        return np.fft.rfft2(f)

    def _c2r(self, F):
        return np.fft.irfft2(F, s=(self.ny, self.nx))

    def solve_elb(self, rho, J):
        rk = self._r2c(rho)
        Jk = [self._r2c(a) for a in J]
        elx = self._c2r(-1j * self.KX * self.gE * rk)
        ely = self._c2r(-1j * self.KY * self.gE * rk)
        bx = self._c2r(1j * self.gB * self.KY * Jk[2])
        by = self._c2r(-1j * self.gB * self.KX * Jk[2])
        bz = self._c2r(1j * self.gB * (self.KX * Jk[1] - self.KY * Jk[0]))
        return (elx, ely), (bx, by, bz)

    def solve_elb_T(self, lel, lb):
        """(lambda rho, lambda J) from (lambda E_L, lambda B): the transpose of
        solve_elb (irfft(conj(K) rfft(.)) per term)."""
        Lx, Ly = self._r2c(lel[0]), self._r2c(lel[1])
        Bx, By, Bz = (self._r2c(a) for a in lb)
        lrho = self._c2r(np.conj(-1j * self.KX * self.gE) * Lx + np.conj(-1j * self.KY * self.gE) * Ly)
        ljx = self._c2r(np.conj(-1j * self.gB * self.KY) * Bz)
        ljy = self._c2r(np.conj(1j * self.gB * self.KX) * Bz)
        ljz = self._c2r(np.conj(1j * self.gB * self.KY) * Bx + np.conj(-1j * self.gB * self.KX) * By)
        return lrho, (ljx, ljy, ljz)

    def solve_et(self, dcu, amu):
        d = [self._r2c(a) for a in dcu]
        a = [self._r2c(v) for v in amu]
        KX, KY = self.KX, self.KY
        S = (KX * a[0] + KY * a[1], KX * a[1] - KY * a[0], KX * a[2] + KY * a[3])
        Jp = [d[k] - 1j * S[k] for k in range(3)]
        kd = (KX * Jp[0] + KY * Jp[1]) / self.k2
        JT = (Jp[0] - KX * kd, Jp[1] - KY * kd, Jp[2])
        return tuple(self._c2r(-self.gT * v) for v in JT)

    def solve_et_T(self, let):
        """(lambda dcu, lambda amu) from lambda E_T (transpose of solve_et)."""
        L = [self._r2c(v) for v in let]
        KX, KY = self.KX, self.KY
        # E_T = -gT P (dcu - i S), P the transverse projection (symmetric), S linear in amu
        Lp = [-self.gT * v for v in L]
        kd = (KX * Lp[0] + KY * Lp[1]) / self.k2
        PL = (Lp[0] - KX * kd, Lp[1] - KY * kd, Lp[2])          # P^T = P
        ldcu = tuple(self._c2r(v) for v in PL)
        # d/d amu of -i S . PL: S_x = kx a0 + ky a1, S_y = kx a1 - ky a0, S_z = kx a2 + ky a3
        W = [np.conj(-1j) * v for v in PL]                          # conj(-i) PL
        la0 = self._c2r(KX * W[0] - KY * W[1])
        la1 = self._c2r(KY * W[0] + KX * W[1])
        la2 = self._c2r(KX * W[2])
        la3 = self._c2r(KY * W[2])
        return ldcu, (la0, la1, la2, la3)

    # ---- pump ------------------------------------------------------------------------
    def pump_field(self, t):
        """The pump at every cell (cell column i at x = i dx), or zeros."""
        z = np.zeros((self.ny, self.nx))
        p = self.pump
        if not p or t >= p["toff"]:
            return z, z.copy(), z.copy()
        if t < p["trmp"]:
            r = t / p["trmp"]
        elif t > p["toff"] - p["trmp"]:
            r = (p["toff"] - t) / p["trmp"]
        else:
            r = 1.0
        th = p["k0"] * np.arange(self.nx) * self.dx - p["w0"] * t
        row = np.ones((self.ny, 1))
        return (row * (p["ex"] * np.cos(th) * r), row * (-p["ey"] * np.sin(th) * r),
                row * (p["ez"] * np.cos(th) * r))

    # ---- Boris with per-particle B ------------------------------------------------------
    @staticmethod
    def _cross(a, b):
        return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])

    def boris_parts(self, u, e, b, h):
        u1 = tuple(u[d] + h * e[d] for d in range(3))
        t = tuple(h * b[d] for d in range(3))
        t2 = t[0] * t[0] + t[1] * t[1] + t[2] * t[2]
        s = tuple(2.0 * t[d] / (1.0 + t2) for d in range(3))
        c1 = self._cross(u1, t)
        up = tuple(u1[d] + c1[d] for d in range(3))
        c2 = self._cross(up, s)
        u2 = tuple(u1[d] + c2[d] for d in range(3))
        u3 = tuple(u2[d] + h * e[d] for d in range(3))
        return u1, t, t2, s, up, u3

    def boris_T(self, lam3, u, e, b, h):
        """(lambda u, lambda e, lambda b) of u3 = Boris(u, e, b) given lambda u3."""
        u1, t, t2, s, up, _ = self.boris_parts(u, e, b, h)
        le = [h * lam3[d] for d in range(3)]
        l2 = lam3
        lup = self._cross(s, l2)                       # d(up x s) wrt up
        ls = self._cross(l2, up)                       # d(up x s) wrt s
        l1 = [l2[d] + lup[d] for d in range(3)]
        tl = self._cross(t, lup)                       # d(u1 x t) wrt u1
        l1 = [l1[d] + tl[d] for d in range(3)]
        lt = list(self._cross(lup, u1))                # d(u1 x t) wrt t
        den = 1.0 + t2
        sdt = ls[0] * t[0] + ls[1] * t[1] + ls[2] * t[2]
        for d in range(3):
            lt[d] = lt[d] + 2.0 / den * ls[d] - 4.0 * sdt / (den * den) * t[d]
        lb = [h * lt[d] for d in range(3)]
        le = [le[d] + h * l1[d] for d in range(3)]
        return l1, le, lb

    # ---- forward / backward ------------------------------------------------------------
    def sources(self, st, q, u):
        a = (0.5 * (u[0] * u[0] - u[1] * u[1]), u[0] * u[1], u[2] * u[0], u[2] * u[1])
        return (self.deposit(st, q), tuple(self.deposit(st, q * u[d]) for d in range(3)),
                tuple(self.deposit(st, q * a[m]) for m in range(4)))

    def step(self, x, y, u, q, n, keep=None):
        st = self.stencil(x, y)
        rho, J, amu = self.sources(st, q, u)
        (elx, ely), B = self.solve_elb(rho, J)
        Bt = tuple(B[d] + self.B0[d] for d in range(3))
        P = self.pump_field(n * self.dt)
        Fd = (elx + P[0], ely + P[1], P[2])
        cq = self.qm * q
        g_fd = [self.gather(Fd[d], st) for d in range(3)]
        g_b = [self.gather(Bt[d], st) for d in range(3)]
        uxb = self._cross(u, g_b)
        dcu = tuple(self.deposit(st, cq * (g_fd[d] + uxb[d])) for d in range(3))
        et = self.solve_et(dcu, amu)
        E = (elx + et[0] + P[0], ely + et[1] + P[1], et[2] + P[2])
        e = [self.gather(E[d], st) for d in range(3)]
        h = self.qm * 0.5 * self.dt
        u3 = self.boris_parts(u, e, g_b, h)[5]
        xn = np.mod(x + u3[0] * (self.dt / self.dx), self.nx)
        yn = np.mod(y + u3[1] * (self.dt / self.dy), self.ny)
        if keep is not None:
            keep.append(dict(x=x.copy(), y=y.copy(), u=u, E=E, Bt=Bt, Fd=Fd, P=P))
        return xn, yn, u3, E

    def forward(self, x, y, u, w, nsteps, keep=True):
        x, y = np.array(x, np.float64), np.array(y, np.float64)
        u = tuple(np.array(u[:, d], np.float64) for d in range(3))
        q = self.qm / (self.dx * self.dy) * np.asarray(w, np.float64)
        traj = [] if keep else None
        E = None
        for n in range(nsteps):
            x, y, u, E = self.step(x, y, u, q, n, traj)
        loss = 0.5 * self.eps0 * self.dx * self.dy * float(np.sum(E[0] * E[0] + E[1] * E[1]))
        return loss, traj, q

    def gradient(self, x, y, u, w, nsteps):
        """(loss, dloss/du0 [n][3], dloss/d(pump amplitude)) by the discrete adjoint."""
        loss, traj, q = self.forward(x, y, u, w, nsteps)
        n = len(q)
        h = self.qm * 0.5 * self.dt
        cx, cy = self.dt / self.dx, self.dt / self.dy
        lx, ly = np.zeros(n), np.zeros(n)
        lu = [np.zeros(n), np.zeros(n), np.zeros(n)]
        ext = self.eps0 * self.dx * self.dy
        dpump = 0.0
        cq = self.qm * q
        for s in range(nsteps - 1, -1, -1):
            T = traj[s]
            st = self.stencil(T["x"], T["y"])
            u = T["u"]
            # push: move, Boris with gathered e, b
            lam3 = [lu[0] + cx * lx, lu[1] + cy * ly, lu[2]]
            e = [self.gather(T["E"][d], st) for d in range(3)]
            b = [self.gather(T["Bt"][d], st) for d in range(3)]
            lun, le, lb = self.boris_T(lam3, u, e, b, h)
            for d in range(3):
                gx_, gy_ = self.gather_grad(T["E"][d], st)
                lx = lx + le[d] * gx_
                ly = ly + le[d] * gy_
                gx_, gy_ = self.gather_grad(T["Bt"][d], st)
                lx = lx + lb[d] * gx_
                ly = ly + lb[d] * gy_
            lE = [self.deposit(st, le[d]) for d in range(3)]
            lBt = [self.deposit(st, lb[d]) for d in range(3)]
            if s == nsteps - 1:
                lE[0] = lE[0] + ext * T["E"][0]
                lE[1] = lE[1] + ext * T["E"][1]
            dpump += sum(float(np.sum(lE[d] * T["P"][d])) for d in range(3))
            # E = E_L + E_T + P
            ldcu, lamu = self.solve_et_T(lE)
            # dcu = D(c (G(Fd) + u x G(Bt)))
            g = [self.gather(ldcu[d], st) for d in range(3)]
            gfd = [self.gather(T["Fd"][d], st) for d in range(3)]
            uxb = self._cross(u, b)
            dcu_p = [cq * (gfd[d] + uxb[d]) for d in range(3)]
            for d in range(3):
                gx_, gy_ = self.gather_grad(ldcu[d], st)
                lx = lx + dcu_p[d] * gx_
                ly = ly + dcu_p[d] * gy_
            lfd_p = [cq * g[d] for d in range(3)]
            gxu = self._cross(g, u)
            lbt_p = [cq * gxu[d] for d in range(3)]
            bxg = self._cross(b, g)
            for d in range(3):
                lun[d] = lun[d] + cq * bxg[d]
                gx_, gy_ = self.gather_grad(T["Fd"][d], st)
                lx = lx + lfd_p[d] * gx_
                ly = ly + lfd_p[d] * gy_
                gx_, gy_ = self.gather_grad(T["Bt"][d], st)
                lx = lx + lbt_p[d] * gx_
                ly = ly + lbt_p[d] * gy_
            lFd = [self.deposit(st, lfd_p[d]) for d in range(3)]
            for d in range(3):
                lBt[d] = lBt[d] + self.deposit(st, lbt_p[d])
            dpump += sum(float(np.sum(lFd[d] * T["P"][d])) for d in range(3))
            lel = (lE[0] + lFd[0], lE[1] + lFd[1])
            lrho, lJ = self.solve_elb_T(lel, lBt)
            # sources rho, J, amu of (x, u)
            r_ = self.gather(lrho, st)
            j_ = [self.gather(lJ[d], st) for d in range(3)]
            a_ = [self.gather(lamu[m], st) for m in range(4)]
            ux, uy, uz = u
            lun[0] = lun[0] + q * (j_[0] + a_[0] * ux + a_[1] * uy + a_[2] * uz)
            lun[1] = lun[1] + q * (j_[1] - a_[0] * uy + a_[1] * ux + a_[3] * uz)
            lun[2] = lun[2] + q * (j_[2] + a_[2] * ux + a_[3] * uy)
            am = (0.5 * (ux * ux - uy * uy), ux * uy, uz * ux, uz * uy)
            gx_, gy_ = self.gather_grad(lrho, st)
            dx_, dy_ = q * gx_, q * gy_
            for d in range(3):
                gx_, gy_ = self.gather_grad(lJ[d], st)
                dx_, dy_ = dx_ + q * u[d] * gx_, dy_ + q * u[d] * gy_
            for m in range(4):
                gx_, gy_ = self.gather_grad(lamu[m], st)
                dx_, dy_ = dx_ + q * am[m] * gx_, dy_ + q * am[m] * gy_
            lx = lx + dx_
            ly = ly + dy_
            lu = lun
        return loss, np.stack(lu, axis=1), dpump


def loss_at(case, x, y, u, w, nsteps):
    return case.forward(x, y, u, w, nsteps, keep=False)[0]
