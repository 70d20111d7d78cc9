"""The straightforward FP64 single-rhs GPU solve, the denominator of the
"vs plain GPU solve" ratio: a direct restatement of GpuMatVec::apply
(DDA/GpuMatVec.cpp:144-431) and the BiCGStab loop (DDA/BicgStab.cpp:59-112)
with library building blocks and no fusion.

  matvec   scatter sqrt(cc) x into the zero-padded grid, cuFFT forward
           (torch.fft.fftn), the 3x3 D multiply on the full D (6 N complex,
           the reference layout), cuFFT inverse, gather, y = sqrt(cc) X + x;
  solver   one kernel per vector operation, dot products read back to the
           host every time (the reference's Pointer<T> blocking reads).

Benchmark infrastructure, not the product: the product path is
libdda_b200.so.
"""
import numpy as np


class PlainSolver:
    def __init__(self, mv, params, cc_sqrt, device="cuda"):
        import torch
        self.torch = torch
        gx, gy, gz = params.grid
        D = mv.dmatrix()  # [Gx][Gz][Gy][6] complex, reference units
        d = torch.from_numpy(np.ascontiguousarray(D.transpose(3, 0, 2, 1))).to(device)  # [6][Gx][Gy][Gz]
        self.D = d
        pos = params.geometry.positions.astype(np.int64)
        self.ix = torch.from_numpy(pos[:, 0]).to(device)
        self.iy = torch.from_numpy(pos[:, 1]).to(device)
        self.iz = torch.from_numpy(pos[:, 2]).to(device)
        mat = params.geometry.materials.astype(np.int64)
        ccs = np.asarray(cc_sqrt).reshape(-1, 3)[mat]  # [nv][3]
        self.ccs = torch.from_numpy(np.ascontiguousarray(ccs.T)).to(device)  # [3][nv]
        self.nv, self.nvs = params.nv, params.nvs
        self.grid = (gx, gy, gz)
        self.device = device

    def matvec(self, x):
        torch = self.torch
        nv, nvs = self.nv, self.nvs
        xv = x.view(3, nvs)[:, :nv]
        X = torch.zeros((3,) + self.grid, dtype=torch.complex128, device=self.device)
        for c in range(3):
            X[c, self.ix, self.iy, self.iz] = self.ccs[c] * xv[c]
        F = torch.fft.fftn(X, dim=(1, 2, 3))
        D = self.D
        Y = torch.empty_like(F)
        Y[0] = D[0] * F[0] + D[1] * F[1] + D[2] * F[2]
        Y[1] = D[1] * F[0] + D[3] * F[1] + D[4] * F[2]
        Y[2] = D[2] * F[0] + D[4] * F[1] + D[5] * F[2]
        Xr = torch.fft.ifftn(Y, dim=(1, 2, 3), norm="forward")
        out = torch.zeros_like(x).view(3, nvs)
        for c in range(3):
            out[c, :nv] = self.ccs[c] * Xr[c, self.ix, self.iy, self.iz] + xv[c]
        return out.view(-1)

    def solve(self, einc, eps, max_iter=10000):
        """BiCGStab as in DDA/BicgStab.cpp:59-112 (x0 = 0), host-side
        scalars; returns (P = sqrt(cc) x, iterations)."""
        torch = self.torch
        nv, nvs = self.nv, self.nvs
        e = torch.from_numpy(np.ascontiguousarray(einc)).to(self.device)
        b = torch.zeros_like(e).view(3, nvs)
        b[:, :nv] = self.ccs * e.view(3, nvs)[:, :nv]
        b = b.view(-1)
        bb = torch.vdot(b, b).real.item()
        x = torch.zeros_like(b)
        r = b.clone()
        rt = r.clone()
        p = torch.zeros_like(b)
        v = torch.zeros_like(b)
        rho_old = alpha = omega = 1.0 + 0j
        it = 0
        eps2 = eps * eps * bb
        while it < max_iter:
            rho = torch.vdot(rt, r).item()
            beta = (rho / rho_old) * (alpha / omega)
            p = r + beta * (p - omega * v)
            v = self.matvec(p)
            alpha = rho / torch.vdot(rt, v).item()
            s = r - alpha * v
            it += 1
            if torch.vdot(s, s).real.item() < eps2:
                x = x + alpha * p
                break
            t = self.matvec(s)
            omega = torch.vdot(t, s).item() / torch.vdot(t, t).real.item()
            x = x + alpha * p + omega * s
            r = s - omega * t
            rho_old = rho
            if torch.vdot(r, r).real.item() < eps2:
                break
        P = torch.zeros_like(x).view(3, nvs)
        P[:, :nv] = self.ccs * x.view(3, nvs)[:, :nv]
        return P.view(-1), it

    def solve_qmr(self, einc, eps, max_iter=10000):
        """QMR-CS as in DDA/QmrCs.cpp:58-168 (bilinear form sum a_i b_i,
        x0 = 0), host-side scalars; returns (P = sqrt(cc) x, iterations)."""
        torch = self.torch
        nv, nvs = self.nv, self.nvs
        e = torch.from_numpy(np.ascontiguousarray(einc)).to(self.device)
        b = torch.zeros_like(e).view(3, nvs)
        b[:, :nv] = self.ccs * e.view(3, nvs)[:, :nv]
        b = b.view(-1)
        bil = lambda a, c: torch.sum(a * c).item()  # noqa: E731
        nrm = lambda a: torch.vdot(a, a).real.item()  # noqa: E731
        bb = nrm(b)
        eps2 = eps * eps * bb
        x = torch.zeros_like(b)
        r = b.clone()
        inprod = bb
        beta = complex(np.sqrt(complex(bil(r, r))))
        omega_old, omega_new = 0.0, np.sqrt(inprod) / abs(beta)
        tautilda = omega_new * beta
        c_old = c_new = 1.0
        s_old = s_new = 0j
        v = r / beta
        vt = torch.zeros_like(b)
        p_old = torch.zeros_like(b)
        p_new = torch.zeros_like(b)
        it = 0
        while it < max_iter:
            A = self.matvec(v)
            alpha = bil(v, A)
            vt = A - alpha * v if it == 0 else vt * (-beta) - alpha * v + A
            ctmp3 = bil(vt, vt)
            rtmp2 = nrm(vt)
            ctmp1 = omega_old * beta
            ctmp2 = omega_new * alpha
            theta = np.conj(s_old) * ctmp1
            eta = c_old * c_new * ctmp1 + np.conj(s_new) * ctmp2
            zetatilda = c_new * ctmp2 - c_old * s_new * ctmp1
            beta = complex(np.sqrt(complex(ctmp3)))
            omega_old, omega_new = omega_new, np.sqrt(rtmp2) / abs(beta)
            zetaabs = np.sqrt(abs(zetatilda) ** 2 + rtmp2)
            rtmp3 = abs(zetatilda)
            zeta = zetaabs if rtmp3 < 1e-40 else zetaabs / rtmp3 * zetatilda
            c_old, c_new = c_new, rtmp3 / zetaabs
            s_old, s_new = s_new, omega_new * (beta / zeta)
            tau = c_new * tautilda
            tautilda = -s_new * tautilda
            if it == 0:
                p_new = v / zeta
            else:
                pn = v / zeta - (eta / zeta) * p_new
                if it > 1:
                    pn = pn - (theta / zeta) * p_old
                p_old, p_new = p_new, pn
            x = x + tau * p_new
            v, vt = vt / beta, v  # the new Lanczos vector; vt keeps the previous one
            r = r * abs(s_new) ** 2 + v * ((c_new / omega_new) * tautilda)
            it += 1
            if nrm(r) < eps2:
                break
        P = torch.zeros_like(x).view(3, nvs)
        P[:, :nv] = self.ccs * x.view(3, nvs)[:, :nv]
        return P.view(-1), it
