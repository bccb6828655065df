"""NumPy FP64 restatement of the JAX-ALFA per-timestep LES hot path.

TEST INFRASTRUCTURE ONLY.  This module is the checker for the CUDA path: only
``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline legs of
``bench.py`` may import it.  The product path (``jax_alfa_b200``) never calls
it and fails loudly when its CUDA library is missing.

Every method restates one reference function (cited as ``path:line`` inside
the reference project) with the reference's signature, so that the golden
vectors recorded from the reference (``tests/golden/make_golden.py``) can be
replayed call for call.  Arrays use the reference layout: real fields
(nx, ny, nz) C-order (z fastest); spectra (nx, ny//2+1, nz) complex; the
pressure system (nx, ny//2+1, nz+1).

Parity pinning: the reference cannot run with JAX here (not installed), so
its own sources were executed on a NumPy-backed stand-in for ``jax`` and the
resulting golden vectors are committed under ``tests/golden/``; the CPU tests
check this restatement against them.  The FFT provider behind ``jnp.fft`` in
the reference is jax/jaxlib (XLA: ducc on CPU, cuFFT on GPU; version
unpinned by the reference, ``docs/requirements.txt``); here and in the golden
runs it is NumPy's pocketfft.  Both compute the unnormalised forward DFT and
the 1/(n_x n_y)-normalised inverse of numpy.fft.rfft2 / irfft2 semantics.
"""
import math

import numpy as np

PI = math.pi          # src/config/DerivedVars.py:39

_FFT_WORKERS = None


def set_fft_workers(n):
    """Route the transforms through scipy.fft with ``n`` threads (used only to
    time the CPU baseline; None restores NumPy's single-threaded pocketfft,
    with which the golden vectors were recorded)."""
    global _FFT_WORKERS
    _FFT_WORKERS = n


def _rfft2(F):
    if _FFT_WORKERS:
        import scipy.fft
        return scipy.fft.rfft2(F, axes=(0, 1), workers=_FFT_WORKERS)
    return np.fft.rfft2(F, axes=(0, 1))


def _irfft2(F, shape):
    if _FFT_WORKERS:
        import scipy.fft
        return scipy.fft.irfft2(F, axes=(0, 1), s=shape, workers=_FFT_WORKERS)
    return np.fft.irfft2(F, axes=(0, 1), s=shape)
G = 9.81              # src/config/DerivedVars.py:40
VONK = 0.4            # src/config/DerivedVars.py:41


class AlfaOracle:
    """Config-bound restatement.  ``cfg`` holds the reference's Config.py
    option names (``jax_alfa_b200.cases``)."""

    # ------------------------------------------------------------------
    # Derived constants: src/config/DerivedVars.py:48-112,
    # src/initialization/Preprocess.py:44-62
    # ------------------------------------------------------------------
    def __init__(self, cfg):
        self.cfg = dict(cfg)
        c = self.cfg
        self.nx, self.ny, self.nz = int(c["nx"]), int(c["ny"]), int(c["nz"])
        nx, ny, nz = self.nx, self.ny, self.nz
        self.mx, self.my = int(1.5 * nx), int(1.5 * ny)
        self.nx_rfft, self.ny_rfft = nx // 2 + 1, ny // 2 + 1
        self.mx_rfft, self.my_rfft = self.mx // 2 + 1, self.my // 2 + 1
        self.u_scale = 1
        self.TH_scale = 1
        self.z_scale = c["l_x"] / (2 * PI)
        self.g_nondim = G * self.z_scale / (self.u_scale ** 2)
        self.f_coriolis_nondim = c["f_coriolis"] * (self.z_scale / self.u_scale)
        self.T_0_nondim = c["T_0"] / self.TH_scale
        self.inversion_nondim = c["inversion"] * (self.z_scale / self.TH_scale)
        self.qz_sfc = c["SensibleHeatFlux"] * np.ones((nx, ny)) / (self.u_scale * self.TH_scale)
        # moisture (DerivedVars.py:69-75)
        self.Q_scale = 1
        self.qm_sfc = c.get("MoistureFlux", 0.0) * np.ones((nx, ny)) / (self.u_scale * self.Q_scale)
        self.q_inversion_nondim = c.get("q_inversion", 0.0) * (self.z_scale / self.Q_scale)
        self.dx = 2 * PI / nx
        self.dy = 2 * PI / ny
        self.dz = (c["l_z"] / self.z_scale) / (nz - 1)
        self.idz = 1.0 / self.dz
        self.FGR = c["FGR"]
        self.L = self.FGR * (self.dx * self.dy * self.dz) ** (1 / 3)
        self.dt_nondim = c["dt"] * self.u_scale / self.z_scale
        self.nsteps = int(np.ceil(c["SimTime"] / c["dt"]))
        if self.FGR == 1:
            self.TFR, self.optDealias = 2, 1
        else:
            self.TFR, self.optDealias = np.sqrt(2), 0
        self.optSgs = c["optSgs"]
        if self.optSgs in (2, 4):
            self.Cs2_init, self.Cs2PrRatio_init = c["Cwl"], c["CwlPrRatio"]
        else:
            self.Cs2_init, self.Cs2PrRatio_init = c["Cs2"], c["Cs2PrRatio"]
        self.z_damping_nondim = c["z_damping"] / self.z_scale
        self.RelaxTime_nondim = c["RelaxTime"] * (self.u_scale / self.z_scale)
        self.Ugal = c["Ugal"]
        self.z0m, self.z0T = c["z0m"], c["z0T"]
        self.zTemperature = c.get("zTemperature", 0.0)

    # ------------------------------------------------------------------
    # src/initialization/Preprocess.py:73-161
    # ------------------------------------------------------------------
    def Wavenumber(self):
        nx, ny, nz = self.nx, self.ny, self.nz
        kx = np.fft.fftfreq(nx, 1 / nx)
        ky = np.fft.rfftfreq(ny, 1 / ny)
        kx[nx // 2] = 0.0
        ky[ny // 2] = 0.0
        kx2 = np.broadcast_to(kx[:, None, None], (nx, self.ny_rfft, nz))
        ky2 = np.broadcast_to(ky[None, :, None], (nx, self.ny_rfft, nz))
        return kx2, ky2

    def zeros3(self):
        return np.zeros((self.nx, self.ny, self.nz))

    def zeros3_fft(self):
        return np.zeros((self.nx, self.ny_rfft, self.nz), dtype=complex)

    # ------------------------------------------------------------------
    # src/operations/FFT.py:44-84
    # ------------------------------------------------------------------
    @staticmethod
    def FFT(F):
        return _rfft2(F)

    FFT_pad = FFT

    def _irfft2(self, F, shape):
        return _irfft2(F, shape)

    # ------------------------------------------------------------------
    # src/operations/Dealiasing.py:51-114.  Dealias1 copies the x-Nyquist
    # row twice (to kx=nx/2 and kx=mx-nx/2); Dealias2 drops both Nyquists
    # and rescales by 9/4, so a padded product of three factors comes back
    # scaled by 4/9 (the reference's behaviour, reproduced as is).
    # ------------------------------------------------------------------
    def Dealias1(self, F_fft, ZeRo3D_pad_fft=None):
        nxr, nyr = self.nx_rfft, self.ny_rfft
        P = np.zeros((self.mx, self.my_rfft) + F_fft.shape[2:], dtype=complex)
        P[:nxr, :nyr] = F_fft[:nxr, :nyr]
        P[self.mx - (nxr - 1):, :nyr] = F_fft[nxr - 1:, :nyr]
        return self._irfft2(P, (self.mx, self.my))

    def Dealias2(self, F_pad_fft, ZeRo3D_fft=None):
        nxr, nyr = self.nx_rfft, self.ny_rfft
        F = np.zeros((self.nx, nyr) + F_pad_fft.shape[2:], dtype=complex)
        F[:nxr - 1, :nyr - 1] = F_pad_fft[:nxr - 1, :nyr - 1]
        F[nxr:, :nyr - 1] = F_pad_fft[self.mx - (nxr - 2):, :nyr - 1]
        return (9.0 / 4.0) * self._irfft2(F, (self.nx, self.ny))

    # ------------------------------------------------------------------
    # src/operations/Filtering.py:50-165: sharp spectral cut-offs.  Kept:
    # kx in [0, c) U [nx-c+1, nx), ky in [0, cy); c from Python round().
    # ------------------------------------------------------------------
    def _truncate(self, F_fft, cx, cy):
        out = np.zeros_like(F_fft)
        out[:cx, :cy] = F_fft[:cx, :cy]
        out[self.nx - cx + 1:, :cy] = F_fft[self.nx - cx + 1:, :cy]
        return out

    def cutoffs(self):
        """(explicit, level-1, level-2) cut-offs in x and y."""
        inv2fgr = 1.0 / (2.0 * self.FGR)
        e = (round(self.nx * inv2fgr), round(self.ny * inv2fgr))
        l1 = (round(self.nx / (2 * self.FGR * self.TFR)), round(self.ny / (2 * self.FGR * self.TFR)))
        l2 = (round(self.nx / (2 * self.FGR * self.TFR * self.TFR)),
              round(self.ny / (2 * self.FGR * self.TFR * self.TFR)))
        return e, l1, l2

    def Filtering_Explicit(self, F_fft):
        (cx, cy), _, _ = self.cutoffs()
        Fn = self._truncate(F_fft, cx, cy)
        return self._irfft2(Fn, (self.nx, self.ny)), Fn

    def Filtering_Level1(self, F_fft):
        _, (cx, cy), _ = self.cutoffs()
        return self._irfft2(self._truncate(F_fft, cx, cy), (self.nx, self.ny))

    def Filtering_Level2(self, F_fft):
        _, _, (cx, cy) = self.cutoffs()
        return self._irfft2(self._truncate(F_fft, cx, cy), (self.nx, self.ny))

    # ------------------------------------------------------------------
    # src/operations/Derivatives.py:47-362
    # ------------------------------------------------------------------
    def Derivxy(self, F_fft, kxy2):
        return self._irfft2(1j * kxy2 * F_fft, (self.nx, self.ny))

    def Derivz_M(self, u, v, w, ustar, M_sfc_loc, fi2D_m, ZeRo3D=None):
        nz, idz = self.nz, self.idz
        dudz = np.zeros_like(u)
        dvdz = np.zeros_like(u)
        dwdz = np.zeros_like(u)
        dudz[:, :, 1:nz - 1] = np.diff(u[:, :, 0:nz - 1], axis=2) * idz
        dvdz[:, :, 1:nz - 1] = np.diff(v[:, :, 0:nz - 1], axis=2) * idz
        den = M_sfc_loc * VONK * 0.5 * self.dz
        dudz[:, :, 0] = fi2D_m * ustar * (u[:, :, 0] + self.Ugal) / den
        dvdz[:, :, 0] = fi2D_m * ustar * v[:, :, 0] / den
        dwdz[:, :, 0:nz - 1] = np.diff(w, axis=2) * idz
        dwdz[:, :, nz - 1] = 0.0
        return dudz, dvdz, dwdz

    def Derivz_TH(self, TH, ustar, qz_sfc, fi2D_h, ZeRo3D=None):
        dTHdz = np.zeros_like(TH)
        dTHdz[:, :, 1:self.nz] = np.diff(TH, axis=2) * self.idz
        dTHdz[:, :, 0] = fi2D_h * (-qz_sfc / ustar) / (VONK * 0.5 * self.dz)
        return dTHdz

    def Derivz_Generic_uvp(self, F, ZeRo3D=None):
        d = np.zeros_like(F)
        d[:, :, 1:self.nz] = np.diff(F, axis=2) * self.idz
        d[:, :, 0] = 0.0
        return d

    def Derivz_Generic_w(self, F, ZeRo3D=None):
        d = np.zeros_like(F)
        d[:, :, 0:self.nz - 1] = np.diff(F, axis=2) * self.idz
        d[:, :, self.nz - 1] = 0.0
        return d

    def velocityGradients(self, u, v, w, u_fft, v_fft, w_fft, kx2, ky2,
                          ustar, M_sfc_loc, MOSTfunctions, ZeRo3D=None):
        dudx, dvdx, dwdx = (self.Derivxy(u_fft, kx2), self.Derivxy(v_fft, kx2),
                            self.Derivxy(w_fft, kx2))
        dudy, dvdy, dwdy = (self.Derivxy(u_fft, ky2), self.Derivxy(v_fft, ky2),
                            self.Derivxy(w_fft, ky2))
        fi2D_m = MOSTfunctions[4]
        dudz, dvdz, dwdz = self.Derivz_M(u, v, w, ustar, M_sfc_loc, fi2D_m)
        return dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz

    def potentialTemperatureGradients(self, TH, kx2, ky2, ustar, qz_sfc,
                                      MOSTfunctions, ZeRo3D=None):
        T = self.FFT(TH)
        dTHdx = self.Derivxy(T, kx2)
        dTHdy = self.Derivxy(T, ky2)
        dTHdz = self.Derivz_TH(TH, ustar, qz_sfc, MOSTfunctions[5])
        return dTHdx, dTHdy, dTHdz

    def moistureGradients(self, Q, kx2, ky2, ustar, qm_sfc, MOSTfunctions, ZeRo3D=None):
        """``Derivatives.py:281-306``: the theta form with the moisture flux."""
        return self.potentialTemperatureGradients(Q, kx2, ky2, ustar, qm_sfc, MOSTfunctions)

    # ------------------------------------------------------------------
    # src/utilities/Utilities.py:41-241
    # ------------------------------------------------------------------
    @staticmethod
    def PlanarMean(F):
        return np.mean(F, axis=(0, 1))

    @staticmethod
    def StagGridAvg(F):
        return 0.5 * (F[:, :, :-1] + F[:, :, 1:])

    @staticmethod
    def Imfilter(x):
        """3x3 periodic box mean of every (x, y) plane; ``x`` is (nx, ny) or
        (nx, ny, nz) (planes filtered independently)."""
        p = np.pad(x, ((1, 1), (1, 1)) + ((0, 0),) * (x.ndim - 2), mode="wrap")
        n0, n1 = x.shape[0], x.shape[1]
        out = np.zeros_like(x)
        w = 1.0 / 9.0
        for a in range(3):
            for b in range(3):
                out = out + p[a:a + n0, b:b + n1] * w
        return out

    @staticmethod
    def Roots(coeffs, init_guess, tol=1e-6, max_iter=20):
        """Laguerre iteration of ``src/utilities/Utilities.py:123-241``,
        vectorised over any leading shape of ``init_guess`` (each element
        runs its own while-loop: it stops updating once converged).
        ``coeffs``: (..., deg+1) highest degree first, broadcast against
        ``init_guess``."""
        p = np.asarray(coeffs, dtype=complex)
        x = np.asarray(init_guess, dtype=complex) * np.ones(p.shape[:-1], dtype=complex)
        n = p.shape[-1] - 1
        dp = p[..., :-1] * np.arange(n, 0, -1)
        d2p = dp[..., :-1] * np.arange(n - 1, 0, -1)

        def horner(c, xv):
            y = np.zeros_like(xv)
            for j in range(c.shape[-1]):
                y = y * xv + c[..., j]
            return y

        eps = 1e-16 + 0j
        converged = np.zeros(x.shape, dtype=bool)
        it = 0
        while it < max_iter and not converged.all():
            active = ~converged
            f = horner(p, x)
            df = horner(dp, x)
            d2f = horner(d2p, x)
            fs = np.where(np.abs(f) < eps, eps, f)
            Gv = df / fs
            Hv = Gv ** 2 - d2f / fs
            disc = (n - 1) * (n * Hv - Gv ** 2)
            sq = np.sqrt(disc)
            d1, d2 = Gv + sq, Gv - sq
            den = np.where(np.abs(d1) > np.abs(d2), d1, d2)
            den = np.where(np.abs(den) < eps, eps, den)
            xn = x - n / den
            conv = (np.abs(xn - x) < tol * (1 + np.abs(x))) | (np.abs(f) < tol)
            x = np.where(active, xn, x)
            converged = np.where(active, conv, converged)
            it += 1
        return np.where(converged, x, np.nan + 0j)

    BETA_GUESSES = (0.5, 0.75, 1.0, 1.25, 1.5, 2.0, 3.0, 4.5)

    def ComputeBeta(self, ff, ee, dd, cc, bb, aa):
        """``ComputeBeta1`` (``src/subgridscale/DynamicSGS_LASDD_SM.py:53-95``)
        and ``ComputeBeta2`` (``DynamicSGS_ScalarLASDD_SM.py:54-96``): per
        level, Laguerre from 8 guesses; largest root with |Im|<1e-6 and
        0<Re<5, else 1."""
        coeffs = np.stack([ff, ee, dd, cc, bb, aa], axis=-1)[:, None, :]
        guesses = np.array(self.BETA_GUESSES)[None, :]
        r = self.Roots(coeffs, guesses)
        ok = (np.abs(r.imag) < 1e-6) & (r.real > 0) & (r.real < 5.0)
        vals = np.where(ok, r.real, -np.inf)
        best = vals.max(axis=1)
        return np.where(np.isfinite(best), best, 1.0)

    ComputeBeta1 = ComputeBeta
    ComputeBeta2 = ComputeBeta

    # ------------------------------------------------------------------
    # src/surface/SurfaceFlux.py:53-443 (dry variants)
    # ------------------------------------------------------------------
    @staticmethod
    def MOSTstable(zL):
        psi_m = 5.0 * zL
        psi_h = 5.0 * zL
        return psi_m, psi_h, 1.0 + psi_m, 1.0 + psi_h

    @staticmethod
    def MOSTunstable(zL):
        x = (1 - 15 * zL) ** 0.25
        psi_m = (-2 * np.log(0.5 * (1 + x)) - np.log(0.5 * (1 + x ** 2))
                 + 2 * np.arctan(x) - PI / 2)
        psi_h = -2 * np.log(0.5 * (1 + x ** 2))
        return psi_m, psi_h, 1.0 / x, (1.0 / x) ** 2

    def _z_ref_T(self):
        return self.zTemperature if self.zTemperature > 0.0 else self.z0T

    def _update_MOSTfunctions(self, ustar, qz_sfc_avg, TH_ref, psi_m, psi_m0, psi_h, psi_h0):
        invOB = -(VONK * self.g_nondim * qz_sfc_avg) / ((ustar ** 3) * TH_ref)
        most = self.MOSTstable if qz_sfc_avg <= 0 else self.MOSTunstable
        z1 = (0.5 * self.dz) * invOB
        z0 = (self.z0m / self.z_scale) * invOB
        zT = (self._z_ref_T() / self.z_scale) * invOB
        psi_m, psi_h, fi_m, fi_h = most(z1)
        psi_m0 = most(z0)[0]
        psi_h0 = most(zT)[1]
        return (psi_m, psi_m0, psi_h, psi_h0, fi_m, fi_h), invOB

    def _ustar(self, M, psi_m, psi_m0):
        denom_m = np.log(0.5 * self.dz * self.z_scale / self.z0m) + psi_m - psi_m0
        return np.maximum(VONK * M / denom_m, 1e-3)

    def _M_local(self, u, v):
        return np.sqrt((u[:, :, 0] + self.Ugal) ** 2 + v[:, :, 0] ** 2)

    def SurfaceFlux_HomogeneousConstantFlux(self, u, v, TH, MOST):
        one = np.ones((self.nx, self.ny))
        psi_m, psi_m0, psi_h, psi_h0 = MOST[:4]
        qavg = np.mean(self.qz_sfc)
        M = np.mean(self._M_local(u, v)) * one
        TH_ref = (np.mean(TH[:, :, 0]) + self.T_0_nondim) * one
        ustar = self._ustar(M, psi_m, psi_m0)
        MOST, invOB = self._update_MOSTfunctions(ustar, qavg, TH_ref, psi_m, psi_m0, psi_h, psi_h0)
        return M, ustar, qavg, invOB, MOST

    def SurfaceFlux_HeterogeneousConstantFlux(self, u, v, TH, MOST):
        psi_m, psi_m0, psi_h, psi_h0 = MOST[:4]
        qavg = np.mean(self.qz_sfc)
        M = self._M_local(u, v)
        TH_ref = TH[:, :, 0] + self.T_0_nondim
        ustar = self._ustar(M, psi_m, psi_m0)
        MOST, invOB = self._update_MOSTfunctions(ustar, qavg, TH_ref, psi_m, psi_m0, psi_h, psi_h0)
        return M, ustar, qavg, invOB, MOST

    def SurfaceFlux_HomogeneousVaryingFlux(self, u, v, TH, qz_t, MOST):
        one = np.ones((self.nx, self.ny))
        psi_m, psi_m0, psi_h, psi_h0 = MOST[:4]
        qavg = qz_t
        q2 = qz_t * one
        M = np.mean(self._M_local(u, v)) * one
        TH_ref = (np.mean(TH[:, :, 0]) + self.T_0_nondim) * one
        ustar = self._ustar(M, psi_m, psi_m0)
        MOST, invOB = self._update_MOSTfunctions(ustar, qavg, TH_ref, psi_m, psi_m0, psi_h, psi_h0)
        return M, ustar, q2, qavg, invOB, MOST

    def SurfaceFlux_HeterogeneousVaryingFlux(self, u, v, TH, qz_t, MOST):
        one = np.ones((self.nx, self.ny))
        psi_m, psi_m0, psi_h, psi_h0 = MOST[:4]
        qavg = qz_t
        q2 = qz_t * one
        M = self._M_local(u, v)
        TH_ref = TH[:, :, 0] + self.T_0_nondim
        ustar = self._ustar(M, psi_m, psi_m0)
        MOST, invOB = self._update_MOSTfunctions(ustar, qavg, TH_ref, psi_m, psi_m0, psi_h, psi_h0)
        return M, ustar, q2, qavg, invOB, MOST

    def _denom_h(self, psi_h, psi_h0):
        return np.log(0.5 * self.dz * self.z_scale / self._z_ref_T()) + psi_h - psi_h0

    def SurfaceFlux_HomogeneousPrescribedTemperature(self, u, v, TH, TH_s, MOST):
        one = np.ones((self.nx, self.ny))
        psi_m, psi_m0, psi_h, psi_h0 = MOST[:4]
        M = np.mean(self._M_local(u, v)) * one
        th_air = np.mean(TH[:, :, 0])
        TH_loc = (th_air + self.T_0_nondim) * one
        ustar = self._ustar(M, psi_m, psi_m0)
        q2 = ustar * VONK * (TH_s - th_air) * one / self._denom_h(psi_h, psi_h0)
        qavg = np.mean(q2)
        MOST, invOB = self._update_MOSTfunctions(ustar, qavg, TH_loc, psi_m, psi_m0, psi_h, psi_h0)
        return M, ustar, q2, qavg, invOB, MOST

    def SurfaceFlux_HeterogeneousPrescribedTemperature(self, u, v, TH, TH_s, MOST):
        psi_m, psi_m0, psi_h, psi_h0 = MOST[:4]
        M = self._M_local(u, v)
        th_air = TH[:, :, 0]
        ustar = self._ustar(M, psi_m, psi_m0)
        q2 = ustar * VONK * (TH_s - th_air) / self._denom_h(psi_h, psi_h0)
        qavg = np.mean(q2)
        TH_ref = (np.mean(th_air) + self.T_0_nondim) * np.ones((self.nx, self.ny))
        MOST, invOB = self._update_MOSTfunctions(ustar, qavg, TH_ref, psi_m, psi_m0, psi_h, psi_h0)
        return M, ustar, q2, qavg, invOB, MOST

    # src/surface/SurfaceFlux.py:447-504 (optMoistureSurfBC = 2)
    def _denom_q(self, psi_h, psi_h0):
        z = self.cfg.get("zMoisture", 0.0)
        zref = z if z > 0.0 else self.cfg["z0T"]
        return np.log(0.5 * self.dz * self.z_scale / zref) + psi_h - psi_h0

    def SurfaceMoistureFlux_HomogeneousPrescribedQ(self, Q, ustar, Q_sfc_t, MOST):
        one = np.ones((self.nx, self.ny))
        psi_h, psi_h0 = MOST[2], MOST[3]
        q_air = np.mean(Q[:, :, 0])
        return ustar * VONK * (Q_sfc_t - q_air) * one / self._denom_q(psi_h, psi_h0)

    def SurfaceMoistureFlux_HeterogeneousPrescribedQ(self, Q, ustar, Q_sfc_t, MOST):
        psi_h, psi_h0 = MOST[2], MOST[3]
        return ustar * VONK * (Q_sfc_t - Q[:, :, 0]) / self._denom_q(psi_h, psi_h0)

    # ------------------------------------------------------------------
    # src/pde/NSE_AdvectionTerms.py:65-155 (3/2-rule dealiased form)
    # ------------------------------------------------------------------
    def _pad(self, F):
        return self.Dealias1(self.FFT(F))

    def _unpad(self, P):
        return self.Dealias2(self.FFT(P))

    def _advect_xy(self, a1, a2, nz):
        """Rows of Cx/Cy: interior a1 + StagGridAvg(a2); k=0 uses a2[1]/2;
        top uses a2[nz-1] (``NSE_AdvectionTerms.py:113-116``)."""
        cc = np.zeros_like(a1)
        g = self.StagGridAvg(a2)
        cc[:, :, 1:nz - 1] = a1[:, :, 1:nz - 1] + g[:, :, 1:nz - 1]
        cc[:, :, 0] = a1[:, :, 0] + 0.5 * a2[:, :, 1]
        cc[:, :, nz - 1] = a1[:, :, nz - 1] + a2[:, :, nz - 1]
        return cc

    def Advection(self, u, v, w, dudy, dudz, dvdx, dvdz, dwdx, dwdy,
                  ZeRo3D=None, ZeRo3D_fft=None, ZeRo3D_pad=None, ZeRo3D_pad_fft=None):
        nz = self.nz
        if self.optDealias != 1:
            return self.Advection_NoDealias(u, v, w, dudy, dudz, dvdx, dvdz, dwdx, dwdy)
        up, vp, wp = self._pad(u), self._pad(v), self._pad(w)
        uy, uz = self._pad(dudy), self._pad(dudz)
        vx, vz = self._pad(dvdx), self._pad(dvdz)
        wx, wy = self._pad(dwdx), self._pad(dwdy)
        Cx = self._unpad(self._advect_xy(vp * (uy - vx), wp * (uz - wx), nz))
        Cy = self._unpad(self._advect_xy(up * (vx - uy), wp * (vz - wy), nz))
        a1 = np.zeros_like(up)
        a2 = np.zeros_like(up)
        ug, vg = self.StagGridAvg(up), self.StagGridAvg(vp)
        a1[:, :, 1:nz - 1] = ug[:, :, 0:nz - 2] * (wx[:, :, 1:nz - 1] - uz[:, :, 1:nz - 1])
        a2[:, :, 1:nz - 1] = vg[:, :, 0:nz - 2] * (wy[:, :, 1:nz - 1] - vz[:, :, 1:nz - 1])
        cc = a1 + a2
        cc[:, :, 0] = 0
        cc[:, :, nz - 1] = 0
        Cz = self._unpad(cc)
        return Cx, Cy, Cz

    def Advection_NoDealias(self, u, v, w, dudy, dudz, dvdx, dvdz, dwdx, dwdy, ZeRo3D=None):
        """``src/pde/NSE_AdvectionTerms.py:163-238``."""
        nz = self.nz
        Cx = self._advect_xy(v * (dudy - dvdx), w * (dudz - dwdx), nz)
        Cy = self._advect_xy(u * (dvdx - dudy), w * (dvdz - dwdy), nz)
        a1 = np.zeros_like(u)
        a2 = np.zeros_like(u)
        ug, vg = self.StagGridAvg(u), self.StagGridAvg(v)
        a1[:, :, 1:nz - 1] = ug[:, :, 0:nz - 2] * (dwdx[:, :, 1:nz - 1] - dudz[:, :, 1:nz - 1])
        a2[:, :, 1:nz - 1] = vg[:, :, 0:nz - 2] * (dwdy[:, :, 1:nz - 1] - dvdz[:, :, 1:nz - 1])
        Cz = a1 + a2
        Cz[:, :, 0] = 0
        Cz[:, :, nz - 1] = 0
        return Cx, Cy, Cz

    # src/pde/SCL_AdvectionTerms.py:57-150
    def _scalar_adv_rows(self, c1, c2):
        nz = self.nz
        cc = np.zeros_like(c1)
        cc[:, :, 0:nz - 1] = c1[:, :, 0:nz - 1] + self.StagGridAvg(c2)
        cc[:, :, nz - 1] = c1[:, :, nz - 1] + c2[:, :, nz - 1]
        return cc

    def ScalarAdvection(self, u, v, w, dsdx, dsdy, dsdz,
                        ZeRo3D=None, ZeRo3D_fft=None, ZeRo3D_pad=None, ZeRo3D_pad_fft=None):
        if self.optDealias != 1:
            return self._scalar_adv_rows(u * dsdx + v * dsdy, w * dsdz)
        up, vp, wp = self._pad(u), self._pad(v), self._pad(w)
        sx, sy, sz = self._pad(dsdx), self._pad(dsdy), self._pad(dsdz)
        return self._unpad(self._scalar_adv_rows(up * sx + vp * sy, wp * sz))

    # ------------------------------------------------------------------
    # src/pde/NSE_BuoyancyTerms.py:49-150 (dry: H = 0)
    # ------------------------------------------------------------------
    def _buoyancy(self, TH, H, by_mean):
        THv = (TH + self.T_0_nondim) * (1 + 0.61 * H)
        bar = self.PlanarMean(THv).reshape(1, 1, -1)
        nrm = (THv - bar) / (bar if by_mean else self.T_0_nondim)
        b = np.zeros_like(TH)
        b[:, :, 1:self.nz] = 0.5 * self.g_nondim * (nrm[:, :, 1:self.nz] + nrm[:, :, 0:self.nz - 1])
        b[:, :, 0] = 0.0
        return b

    def BuoyancyOpt1(self, TH, H, ZeRo3D=None):
        return self._buoyancy(TH, H, False)

    def BuoyancyOpt2(self, TH, H, ZeRo3D=None):
        return self._buoyancy(TH, H, True)

    # ------------------------------------------------------------------
    # src/subgridscale/StrainRates.py:56-368
    # ------------------------------------------------------------------
    @staticmethod
    def _smag(S11, S22, S33, S12, S13, S23):
        return np.sqrt(2 * (S11 ** 2 + S22 ** 2 + S33 ** 2 + 2 * S12 ** 2 + 2 * S13 ** 2 + 2 * S23 ** 2))

    def _uvp_strains(self, dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz):
        nz = self.nz
        uz, vz, wx, wy = (np.zeros_like(dudx) for _ in range(4))
        uz[:, :, 1:nz - 1] = self.StagGridAvg(dudz[:, :, 1:nz])
        vz[:, :, 1:nz - 1] = self.StagGridAvg(dvdz[:, :, 1:nz])
        wx[:, :, 1:nz - 1] = self.StagGridAvg(dwdx[:, :, 1:nz])
        wy[:, :, 1:nz - 1] = self.StagGridAvg(dwdy[:, :, 1:nz])
        uz[:, :, 0] = dudz[:, :, 0]
        vz[:, :, 0] = dvdz[:, :, 0]
        wx[:, :, 0] = 0.5 * dwdx[:, :, 1]
        wy[:, :, 0] = 0.5 * dwdy[:, :, 1]
        uz[:, :, nz - 1] = dudz[:, :, nz - 1]
        vz[:, :, nz - 1] = dvdz[:, :, nz - 1]
        wx[:, :, nz - 1] = dwdx[:, :, nz - 1]
        wy[:, :, nz - 1] = dwdy[:, :, nz - 1]
        S11, S22, S33 = dudx.copy(), dvdy.copy(), dwdz.copy()
        S12 = 0.5 * (dudy + dvdx)
        S13 = 0.5 * (uz + wx)
        S23 = 0.5 * (vz + wy)
        return S11, S22, S33, S12, S13, S23, self._smag(S11, S22, S33, S12, S13, S23)

    def StrainsUVPnodes_Dealias(self, dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz,
                                ZeRo3D=None, ZeRo3D_pad_fft=None):
        S = self._uvp_strains(dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz)
        P = tuple(self._pad(x) for x in S[:6])
        return S + P + (self._smag(*P),)

    def StrainsUVPnodes_NoDealias(self, dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz,
                                  ZeRo3D=None):
        return self._uvp_strains(dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz)

    def _w_strains(self, dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz):
        nz = self.nz
        ux, uy, vx, vy, wz = (np.zeros_like(dudx) for _ in range(5))
        ux[:, :, 1:nz - 1] = self.StagGridAvg(dudx[:, :, :nz - 1])
        uy[:, :, 1:nz - 1] = self.StagGridAvg(dudy[:, :, :nz - 1])
        vx[:, :, 1:nz - 1] = self.StagGridAvg(dvdx[:, :, :nz - 1])
        vy[:, :, 1:nz - 1] = self.StagGridAvg(dvdy[:, :, :nz - 1])
        uz, vz = dudz.copy(), dvdz.copy()
        wx, wy = dwdx.copy(), dwdy.copy()
        wz[:, :, 1:nz - 1] = self.StagGridAvg(dwdz[:, :, :nz - 1])
        ux[:, :, 0] = dudx[:, :, 0]
        uy[:, :, 0] = dudy[:, :, 0]
        vx[:, :, 0] = dvdx[:, :, 0]
        vy[:, :, 0] = dvdy[:, :, 0]
        wx[:, :, 0] = 0.5 * (dwdx[:, :, 0] + dwdx[:, :, 1])
        wy[:, :, 0] = 0.5 * (dwdy[:, :, 0] + dwdy[:, :, 1])
        wz[:, :, 0] = dwdz[:, :, 0]
        S11, S22, S33 = ux.copy(), vy.copy(), wz.copy()
        S12 = 0.5 * (uy + vx)
        S13 = 0.5 * (uz + wx)
        S23 = 0.5 * (vz + wy)
        return S11, S22, S33, S12, S13, S23

    def StrainsWnodes_Dealias(self, dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz,
                              ZeRo3D=None, ZeRo3D_pad_fft=None):
        S = self._w_strains(dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz)
        P = tuple(self._pad(x) for x in S)
        return P[4], P[5], self._smag(*S), self._smag(*P)

    def StrainsWnodes_NoDealias(self, dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz,
                                ZeRo3D=None):
        S = self._w_strains(dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz)
        return S[4], S[5], self._smag(*S)

    # ------------------------------------------------------------------
    # src/subgridscale/DynamicSGS_LASDD_SM.py:103-367
    # ------------------------------------------------------------------
    def _clip_ratio(self, num, den):
        """``Cs2_at_level_k`` (``DynamicSGS_LASDD_SM.py:103-130``) and
        ``Cs2PrRatio_at_level_k`` (``DynamicSGS_ScalarLASDD_SM.py:104-131``)
        for all levels at once."""
        nf = self.Imfilter(num)
        df = self.Imfilter(den)
        with np.errstate(divide="ignore", invalid="ignore"):
            r = nf / df
        bad = (np.abs(df) < 1e-10) | (r < 0) | (r > 1)
        return np.where(bad, 0.0, r)

    def _level1_level2(self, F):
        """Both test-filter levels of one field from one spectrum (the
        reference computes the same FFT once per level)."""
        Fh = self.FFT(F)
        return self.Filtering_Level1(Fh), self.Filtering_Level2(Fh)

    def LASDD(self, u, v, w, S11, S22, S33, S12, S13, S23, S, ZeRo3D=None):
        nz, L, TFR = self.nz, self.L, self.TFR
        u_, v_ = u.copy(), v.copy()
        w_ = np.zeros_like(w)
        w_[:, :, 1:nz - 1] = self.StagGridAvg(w[:, :, 1:nz])
        w_[:, :, 0] = 0.5 * w[:, :, 1]
        w_[:, :, nz - 1] = w[:, :, nz - 2]
        (u_h, u_d), (v_h, v_d), (w_h, w_d) = (self._level1_level2(x) for x in (u_, v_, w_))
        prods = (u_ ** 2, v_ ** 2, w_ ** 2, u_ * v_, u_ * w_, v_ * w_)
        ph = [self._level1_level2(x) for x in prods]
        Sij = (S11, S22, S33, S12, S13, S23)
        Sh = [self._level1_level2(x) for x in Sij]
        SSh = [self._level1_level2(S * x) for x in Sij]
        S_hat = self._smag(*(x[0] for x in Sh))
        S_hatd = self._smag(*(x[1] for x in Sh))
        hat1 = (u_h, v_h, w_h)
        hat2 = (u_d, v_d, w_d)
        pairs = ((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))
        Lij = [ph[i][0] - (hat1[a] ** 2 if a == b else hat1[a] * hat1[b]) for i, (a, b) in enumerate(pairs)]
        Qij = [ph[i][1] - (hat2[a] ** 2 if a == b else hat2[a] * hat2[b]) for i, (a, b) in enumerate(pairs)]

        def contract(A, B):
            return (A[0] * B[0] + A[1] * B[1] + A[2] * B[2]
                    + 2 * (A[3] * B[3] + A[4] * B[4] + A[5] * B[5]))

        def sq(A):
            return (A[0] ** 2 + A[1] ** 2 + A[2] ** 2 + 2 * (A[3] ** 2 + A[4] ** 2 + A[5] ** 2))

        S1 = [x[0] for x in Sh]
        S2 = [x[1] for x in Sh]
        SS1 = [x[0] for x in SSh]
        SS2 = [x[1] for x in SSh]
        PM = self.PlanarMean
        a1_t = contract(Lij, SS1)
        a1 = PM(2 * (L ** 2) * a1_t)
        a2 = PM(2 * (L ** 2) * contract(Qij, SS2))
        b1 = PM(2 * (L ** 2) * (TFR ** 2) * S_hat * contract(Lij, S1))
        b2 = PM(2 * (L ** 2) * (TFR ** 4) * S_hatd * contract(Qij, S2))
        c1 = PM((2 * L ** 2) ** 2 * sq(SS1))
        c2 = PM((2 * L ** 2) ** 2 * sq(SS2))
        d1 = PM((4 * L ** 4) * (TFR ** 4) * (S_hat ** 2) * sq(S1))
        d2 = PM((4 * L ** 4) * (TFR ** 8) * (S_hatd ** 2) * sq(S2))
        e1 = PM((8 * L ** 4) * (TFR ** 2) * S_hat * contract(S1, SS1))
        e2 = PM((8 * L ** 4) * (TFR ** 4) * S_hatd * contract(S2, SS2))
        aa = a1 * c2 - a2 * c1
        bb = a2 * e1 - b1 * c2
        cc = b2 * c1 - a1 * e2 - a2 * d1
        dd = b1 * e2 - b2 * e1
        ee = a1 * d2 + b2 * d1
        ff = -b1 * d2
        if self.optSgs in (1, 2):
            beta1 = self.ComputeBeta1(ff, ee, dd, cc, bb, aa)
        else:
            beta1 = np.ones(nz)
        b3 = beta1.reshape(1, 1, nz)
        T1 = 2 * L ** 2
        T2 = 2 * (TFR * L) ** 2
        Mij = [T1 * SS1[i] - T2 * b3 * S_hat * S1[i] for i in range(6)]
        LM = ((Lij[0] * Mij[0] + Lij[1] * Mij[1] + Lij[2] * Mij[2])
              + 2 * (Lij[3] * Mij[3] + Lij[4] * Mij[4] + Lij[5] * Mij[5]))
        MM = sq(Mij)
        Cs2_3D = self._clip_ratio(LM, MM)
        avg1 = self.PlanarMean(np.sqrt(Cs2_3D)) ** 2
        avg2 = self.PlanarMean(Cs2_3D)
        return (u_, v_, w_, u_h, v_h, w_h, u_d, v_d, w_d, S_hat, S_hatd,
                Cs2_3D, avg1, avg2, beta1)

    # ------------------------------------------------------------------
    # src/subgridscale/DynamicSGS_ScalarLASDD_SM.py:139-316
    # ------------------------------------------------------------------
    def ScalarLASDD(self, u_, v_, w_, u_hat, v_hat, w_hat, u_hatd, v_hatd, w_hatd,
                    TH, dTHdx, dTHdy, dTHdz, S, S_hat, S_hatd, ZeRo3D=None):
        nz, L, TFR = self.nz, self.L, self.TFR
        THz = np.zeros_like(TH)
        THz[:, :, 1:nz - 1] = self.StagGridAvg(dTHdz[:, :, 1:nz])
        THz[:, :, 0] = dTHdz[:, :, 0]
        THz[:, :, nz - 1] = dTHdz[:, :, nz - 1]
        T_h, T_d = self._level1_level2(TH)
        uT = [self._level1_level2(x * TH) for x in (u_, v_, w_)]
        G = (dTHdx, dTHdy, THz)
        Gf = [self._level1_level2(x) for x in G]
        SG = [self._level1_level2(S * x) for x in G]
        LT = [uT[0][0] - u_hat * T_h, uT[1][0] - v_hat * T_h, uT[2][0] - w_hat * T_h]
        QT = [uT[0][1] - u_hatd * T_d, uT[1][1] - v_hatd * T_d, uT[2][1] - w_hatd * T_d]
        G1 = [x[0] for x in Gf]
        G2 = [x[1] for x in Gf]
        SG1 = [x[0] for x in SG]
        SG2 = [x[1] for x in SG]
        PM = self.PlanarMean
        a2t = LT[0] * SG1[0] + LT[1] * SG1[1] + LT[2] * SG1[2]
        b2t = LT[0] * S_hat * G1[0] + LT[1] * S_hat * G1[1] + LT[2] * S_hat * G1[2]
        c2t = SG1[0] ** 2 + SG1[1] ** 2 + SG1[2] ** 2
        d2t = SG1[0] * S_hat * G1[0] + SG1[1] * S_hat * G1[1] + SG1[2] * S_hat * G1[2]
        e2t = (S_hat * G1[0]) ** 2 + (S_hat * G1[1]) ** 2 + (S_hat * G1[2]) ** 2
        a2 = PM((L ** 2) * a2t)
        b2 = PM((-L ** 2 * TFR ** 2) * b2t)
        c2 = PM((L ** 4) * c2t)
        d2 = PM((-2 * L ** 4 * TFR ** 2) * d2t)
        e2 = PM((L ** 4 * TFR ** 4) * e2t)
        a4 = PM((L ** 2) * (QT[0] * SG2[0] + QT[1] * SG2[1] + QT[2] * SG2[2]))
        b4 = PM((-L ** 2 * TFR ** 4) * (QT[0] * S_hatd * G2[0] + QT[1] * S_hatd * G2[1]
                                        + QT[2] * S_hatd * G2[2]))
        c4 = PM((L ** 4) * (SG2[0] ** 2 + SG2[1] ** 2 + SG2[2] ** 2))
        d4 = PM((-2 * L ** 4 * TFR ** 4) * (SG2[0] * S_hatd * G2[0] + SG2[1] * S_hatd * G2[1]
                                            + SG2[2] * S_hatd * G2[2]))
        e4 = PM((L ** 4 * TFR ** 8) * ((S_hatd * G2[0]) ** 2 + (S_hatd * G2[1]) ** 2
                                       + (S_hatd * G2[2]) ** 2))
        aa = a2 * c4 - a4 * c2
        bb = -a4 * d2 + b2 * c4
        cc = -c2 * b4 + a2 * d4 - a4 * e2
        dd = b2 * d4 - b4 * d2
        ee = a2 * e4 - b4 * e2
        ff = b2 * e4
        if self.optSgs in (1, 2):
            beta2 = self.ComputeBeta2(ff, ee, dd, cc, bb, aa)
        else:
            beta2 = np.ones(nz)
        b3 = beta2.reshape(1, 1, nz)
        T_up = (L ** 2) * a2t + (-L ** 2 * TFR ** 2) * b2t * b3
        T_dn = ((L ** 4) * c2t + (-2 * L ** 4 * TFR ** 2) * d2t * b3
                + (L ** 4 * TFR ** 4) * e2t * b3 ** 2)
        r3 = self._clip_ratio(T_up, T_dn)
        return r3, self.PlanarMean(r3), beta2

    # ------------------------------------------------------------------
    # Wong-Lilly base model (optSgs = 2, 4)
    # ------------------------------------------------------------------
    def _wl_coeffs(self, a1, a3, a6, a8):
        """Quintic coefficients (ff, ee, dd, cc, bb, aa) of the WL procedure
        from the four independent plane means
        (``DynamicSGS_LASDD_WL.py:262-277``, ``DynamicSGS_ScalarLASDD_WL.py:230-245``)."""
        TFR = self.TFR
        a2 = -(TFR ** (8 / 3)) * a1
        a4 = -2 * TFR ** (4 / 3) * a3
        a5 = TFR ** (8 / 3) * a3
        a7 = -TFR ** (4 / 3) * a6
        a9 = -2 * TFR ** (8 / 3) * a8
        a10 = TFR ** (16 / 3) * a8
        aa = a1 * a3 - a6 * a8
        bb = a1 * a4 - a7 * a8
        cc = a2 * a3 + a1 * a5 - a6 * a9
        dd = a2 * a4 - a7 * a9
        ee = a2 * a5 - a6 * a10
        ff = -a7 * a10
        return ff, ee, dd, cc, bb, aa

    def LASDD_WL(self, u, v, w, S11, S22, S33, S12, S13, S23, ZeRo3D=None):
        """``src/subgridscale/DynamicSGS_LASDD_WL.py:127-313``."""
        nz, L, TFR = self.nz, self.L, self.TFR
        u_, v_ = u.copy(), v.copy()
        w_ = np.zeros_like(w)
        w_[:, :, 1:nz - 1] = self.StagGridAvg(w[:, :, 1:nz])
        w_[:, :, 0] = 0.5 * w[:, :, 1]
        w_[:, :, nz - 1] = w[:, :, nz - 2]
        (u_h, u_d), (v_h, v_d), (w_h, w_d) = (self._level1_level2(x) for x in (u_, v_, w_))
        prods = (u_ ** 2, v_ ** 2, w_ ** 2, u_ * v_, u_ * w_, v_ * w_)
        ph = [self._level1_level2(x) for x in prods]
        Sh = [self._level1_level2(x) for x in (S11, S22, S33, S12, S13, S23)]
        S1 = [x[0] for x in Sh]
        S2 = [x[1] for x in Sh]
        S_hat = self._smag(*S1)
        S_hatd = self._smag(*S2)
        hat1 = (u_h, v_h, w_h)
        hat2 = (u_d, v_d, w_d)
        pairs = ((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))
        Lij = [ph[i][0] - (hat1[a] ** 2 if a == b else hat1[a] * hat1[b])
               for i, (a, b) in enumerate(pairs)]
        Qij = [ph[i][1] - (hat2[a] ** 2 if a == b else hat2[a] * hat2[b])
               for i, (a, b) in enumerate(pairs)]

        def contract(A, B):
            return (A[0] * B[0] + A[1] * B[1] + A[2] * B[2]
                    + 2 * (A[3] * B[3] + A[4] * B[4] + A[5] * B[5]))

        def sq(A):
            return (A[0] ** 2 + A[1] ** 2 + A[2] ** 2 + 2 * (A[3] ** 2 + A[4] ** 2 + A[5] ** 2))

        PM = self.PlanarMean
        a1 = PM(contract(Qij, S1))
        a3 = PM(sq(S1))
        a6 = PM(contract(Lij, S1))
        a8 = PM(sq(S2))
        if self.optSgs in (1, 2):
            beta1 = self.ComputeBeta1(*self._wl_coeffs(a1, a3, a6, a8))
        else:
            beta1 = np.ones(nz)
        b3 = beta1.reshape(1, 1, nz)
        T1 = 2 * L ** (4 / 3)
        T2 = 2 * (TFR * L) ** (4 / 3)
        Mij = [T1 * S1[i] - T2 * b3 * S2[i] for i in range(6)]
        LM = ((Lij[0] * Mij[0] + Lij[1] * Mij[1] + Lij[2] * Mij[2])
              + 2 * (Lij[3] * Mij[3] + Lij[4] * Mij[4] + Lij[5] * Mij[5]))
        MM = sq(Mij)
        Cwl_3D = self._clip_ratio(LM, MM)
        avg1 = self.PlanarMean(np.sqrt(Cwl_3D)) ** 2
        avg2 = self.PlanarMean(Cwl_3D)
        return (u_, v_, w_, u_h, v_h, w_h, u_d, v_d, w_d, S_hat, S_hatd,
                Cwl_3D, avg1, avg2, beta1)

    def ScalarLASDD_WL(self, u_, v_, w_, u_hat, v_hat, w_hat, u_hatd, v_hatd, w_hatd,
                       TH, dTHdx, dTHdy, dTHdz, ZeRo3D=None):
        """``src/subgridscale/DynamicSGS_ScalarLASDD_WL.py:130-275``."""
        nz, L, TFR = self.nz, self.L, self.TFR
        THz = np.zeros_like(TH)
        THz[:, :, 1:nz - 1] = self.StagGridAvg(dTHdz[:, :, 1:nz])
        THz[:, :, 0] = dTHdz[:, :, 0]
        THz[:, :, nz - 1] = dTHdz[:, :, nz - 1]
        T_h, T_d = self._level1_level2(TH)
        uT = [self._level1_level2(x * TH) for x in (u_, v_, w_)]
        Gf = [self._level1_level2(x) for x in (dTHdx, dTHdy, THz)]
        G1 = [x[0] for x in Gf]
        G2 = [x[1] for x in Gf]
        LT = [uT[0][0] - u_hat * T_h, uT[1][0] - v_hat * T_h, uT[2][0] - w_hat * T_h]
        QT = [uT[0][1] - u_hatd * T_d, uT[1][1] - v_hatd * T_d, uT[2][1] - w_hatd * T_d]
        PM = self.PlanarMean
        a1 = PM(QT[0] * G1[0] + QT[1] * G1[1] + QT[2] * G1[2])
        a3_t = G1[0] ** 2 + G1[1] ** 2 + G1[2] ** 2
        a3 = PM(a3_t)
        a6_t = LT[0] * G1[0] + LT[1] * G1[1] + LT[2] * G1[2]
        a6 = PM(a6_t)
        a8_t = G2[0] ** 2 + G2[1] ** 2 + G2[2] ** 2
        a8 = PM(a8_t)
        if self.optSgs in (1, 2):
            beta2 = self.ComputeBeta2(*self._wl_coeffs(a1, a3, a6, a8))
        else:
            beta2 = np.ones(nz)
        b3 = beta2.reshape(1, 1, nz)
        b6_t = LT[0] * G2[0] + LT[1] * G2[1] + LT[2] * G2[2]
        c36_t = G1[0] * G2[0] + G1[1] * G2[1] + G1[2] * G2[2]
        T_up = L ** (4 / 3) * (a6_t - TFR ** (4 / 3) * b3 * b6_t)
        T_dn = L ** (8 / 3) * (a3_t - 2 * TFR ** (4 / 3) * b3 * c36_t
                               + TFR ** (8 / 3) * b3 ** 2 * a8_t)
        r3 = self._clip_ratio(T_up, T_dn)
        return r3, self.PlanarMean(r3), beta2

    # ------------------------------------------------------------------
    # src/subgridscale/SGSStresses_SM.py:63-297
    # ------------------------------------------------------------------
    def Wall(self, u, v, M_sfc_loc, psi2D_m, psi2D_m0):
        denom = np.log(0.5 * self.dz * self.z_scale / self.z0m) + psi2D_m - psi2D_m0
        ustar = VONK * M_sfc_loc / denom
        txz = -(ustar ** 2) * (u[:, :, 0] + self.Ugal) / M_sfc_loc
        tyz = -(ustar ** 2) * v[:, :, 0] / M_sfc_loc
        return txz, tyz

    def StressesUVPnodes_Dealias(self, S11_pad, S22_pad, S33_pad, S12_pad, S_uvp_pad,
                                 Cs2_3D_pad, ZeRo3D_fft=None):
        pre = -2 * (self.L ** 2) * Cs2_3D_pad * S_uvp_pad
        out = []
        for s in (S11_pad, S22_pad, S33_pad, S12_pad):
            t = pre * s
            t[:, :, self.nz - 1] = 0
            out.append(self._unpad(t))
        return tuple(out)

    def StressesUVPnodes_NoDealias(self, S11, S22, S33, S12, S_uvp, Cs2_3D):
        pre = -2 * (self.L ** 2) * Cs2_3D * S_uvp
        out = []
        for s in (S11, S22, S33, S12):
            t = pre * s
            t[:, :, self.nz - 1] = 0
            out.append(t)
        return tuple(out)

    def _w_stress_interior(self, S13, S23, Sw, Cs2):
        nz = self.nz
        txz = np.zeros_like(Sw)
        tyz = np.zeros_like(Sw)
        pre = -2 * (self.L ** 2) * self.StagGridAvg(Cs2[:, :, :nz - 1]) * Sw[:, :, 1:nz - 1]
        txz[:, :, 1:nz - 1] = pre * S13[:, :, 1:nz - 1]
        tyz[:, :, 1:nz - 1] = pre * S23[:, :, 1:nz - 1]
        txz[:, :, nz - 1] = 0
        tyz[:, :, nz - 1] = 0
        return txz, tyz

    def StressesWnodes_Dealias(self, S13_pad, S23_pad, S_w_pad, Cs2_3D_pad,
                               u, v, M_sfc_loc, psi2D_m, psi2D_m0, ZeRo3D_fft=None):
        txz_p, tyz_p = self._w_stress_interior(S13_pad, S23_pad, S_w_pad, Cs2_3D_pad)
        txz, tyz = self._unpad(txz_p), self._unpad(tyz_p)
        wx, wy = self.Wall(u, v, M_sfc_loc, psi2D_m, psi2D_m0)
        txz[:, :, 0] = wx
        tyz[:, :, 0] = wy
        return txz, tyz

    def StressesWnodes_NoDealias(self, S13, S23, S_w, Cs2_3D, u, v, M_sfc_loc, psi2D_m, psi2D_m0):
        txz, tyz = self._w_stress_interior(S13, S23, S_w, Cs2_3D)
        wx, wy = self.Wall(u, v, M_sfc_loc, psi2D_m, psi2D_m0)
        txz[:, :, 0] = wx
        tyz[:, :, 0] = wy
        return txz, tyz

    # ------------------------------------------------------------------
    # src/subgridscale/ScalarSGSFluxes_SM.py:55-222
    # ------------------------------------------------------------------
    def ScalarFluxesUVPnodes_Dealias(self, dTHdx_pad, dTHdy_pad, S_pad, Cs2PrRatio_3D_pad,
                                     ZeRo3D_fft=None):
        pre = -2 * (self.L ** 2) * Cs2PrRatio_3D_pad * S_pad
        out = []
        for g in (dTHdx_pad, dTHdy_pad):
            q = pre * g
            q[:, :, self.nz - 1] = 0
            out.append(self._unpad(q))
        return tuple(out)

    def ScalarFluxesUVPnodes_NoDealias(self, dTHdx, dTHdy, S, Cs2PrRatio_3D):
        pre = -2 * (self.L ** 2) * Cs2PrRatio_3D * S
        qx, qy = pre * dTHdx, pre * dTHdy
        qx[:, :, self.nz - 1] = 0
        qy[:, :, self.nz - 1] = 0
        return qx, qy

    def _qz_interior(self, dTHdz, S, r):
        nz = self.nz
        q = np.zeros_like(S)
        q[:, :, 1:nz - 1] = (-2 * (self.L ** 2) * self.StagGridAvg(r[:, :, :nz - 1])
                             * S[:, :, 1:nz - 1] * dTHdz[:, :, 1:nz - 1])
        q[:, :, nz - 1] = 0
        return q

    def ScalarFluxesWnodes_Dealias(self, dTHdz_pad, S_pad, Cs2PrRatio_3D_pad, qz_sfc,
                                   ZeRo3D_fft=None):
        qz = self._unpad(self._qz_interior(dTHdz_pad, S_pad, Cs2PrRatio_3D_pad))
        qz[:, :, 0] = qz_sfc
        return qz

    def ScalarFluxesWnodes_NoDealias(self, dTHdz, S, Cs2PrRatio_3D, qz_sfc):
        qz = self._qz_interior(dTHdz, S, Cs2PrRatio_3D)
        qz[:, :, 0] = qz_sfc
        return qz

    # src/subgridscale/SGSStresses_WL.py:70-240 (tau = -2 L^(4/3) C_WL S_ij)
    def StressesUVPnodes_Dealias_WL(self, S11_pad, S22_pad, S33_pad, S12_pad, Cwl_3D_pad,
                                    ZeRo3D_fft=None):
        return tuple(self._unpad(t) for t in self._wl_uvp((S11_pad, S22_pad, S33_pad, S12_pad),
                                                           Cwl_3D_pad, -2 * (self.L ** (4 / 3))))

    def StressesUVPnodes_NoDealias_WL(self, S11, S22, S33, S12, Cwl_3D):
        return self._wl_uvp((S11, S22, S33, S12), Cwl_3D, -2 * (self.L ** (4 / 3)))

    def _wl_uvp(self, comps, C, c0):
        pre = c0 * C
        out = []
        for s in comps:
            t = pre * s
            t[:, :, self.nz - 1] = 0
            out.append(t)
        return tuple(out)

    def _wl_w(self, comps, C, c0):
        nz = self.nz
        pre = c0 * self.StagGridAvg(C[:, :, :nz - 1])
        out = []
        for s in comps:
            t = np.zeros_like(s)
            t[:, :, 1:nz - 1] = pre * s[:, :, 1:nz - 1]
            t[:, :, nz - 1] = 0
            out.append(t)
        return tuple(out)

    def StressesWnodes_Dealias_WL(self, S13_pad, S23_pad, Cwl_3D_pad, u, v, M_sfc_loc,
                                  psi2D_m, psi2D_m0, ZeRo3D_fft=None):
        txz_p, tyz_p = self._wl_w((S13_pad, S23_pad), Cwl_3D_pad, -2 * (self.L ** (4 / 3)))
        txz, tyz = self._unpad(txz_p), self._unpad(tyz_p)
        wx, wy = self.Wall(u, v, M_sfc_loc, psi2D_m, psi2D_m0)
        txz[:, :, 0] = wx
        tyz[:, :, 0] = wy
        return txz, tyz

    def StressesWnodes_NoDealias_WL(self, S13, S23, Cwl_3D, u, v, M_sfc_loc, psi2D_m, psi2D_m0):
        txz, tyz = self._wl_w((S13, S23), Cwl_3D, -2 * (self.L ** (4 / 3)))
        wx, wy = self.Wall(u, v, M_sfc_loc, psi2D_m, psi2D_m0)
        txz[:, :, 0] = wx
        tyz[:, :, 0] = wy
        return txz, tyz

    # src/subgridscale/ScalarSGSFluxes_WL.py:56-201 (q = -L^(4/3) (C_WL/Pr) grad)
    def ScalarFluxesUVPnodes_Dealias_WL(self, dTHdx_pad, dTHdy_pad, r_pad, ZeRo3D_fft=None):
        return tuple(self._unpad(q) for q in self._wl_uvp((dTHdx_pad, dTHdy_pad), r_pad,
                                                          -(self.L ** (4 / 3))))

    def ScalarFluxesUVPnodes_NoDealias_WL(self, dTHdx, dTHdy, r):
        return self._wl_uvp((dTHdx, dTHdy), r, -(self.L ** (4 / 3)))

    def ScalarFluxesWnodes_Dealias_WL(self, dTHdz_pad, r_pad, qz_sfc, ZeRo3D_fft=None):
        qz = self._unpad(self._wl_w((dTHdz_pad,), r_pad, -(self.L ** (4 / 3)))[0])
        qz[:, :, 0] = qz_sfc
        return qz

    def ScalarFluxesWnodes_NoDealias_WL(self, dTHdz, r, qz_sfc):
        qz = self._wl_w((dTHdz,), r, -(self.L ** (4 / 3)))[0]
        qz[:, :, 0] = qz_sfc
        return qz

    # ------------------------------------------------------------------
    # src/subgridscale/DynamicSGS_Main.py:85-478 and StaticSGS_Main.py:76-360
    # (SM variants optSgs 0, 1, 3; Wong-Lilly variants optSgs 2, 4)
    # ------------------------------------------------------------------
    @property
    def _wl(self):
        return self.optSgs in (2, 4)

    def DynamicSGS(self, dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz,
                   u, v, w, M_sfc_loc, psi2D_m, psi2D_m0,
                   ZeRo3D=None, ZeRo3D_fft=None, ZeRo3D_pad_fft=None):
        g = (dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz)
        wl = self._wl
        if self.optDealias == 1:
            (S11, S22, S33, S12, S13, S23, S_uvp,
             P11, P22, P33, P12, P13, P23, S_uvp_pad) = self.StrainsUVPnodes_Dealias(*g)
            if wl:
                las = self.LASDD_WL(u, v, w, S11, S22, S33, S12, S13, S23)
            else:
                las = self.LASDD(u, v, w, S11, S22, S33, S12, S13, S23, S_uvp)
            Cs2_3D = las[11]
            Cs2_pad = self._pad(Cs2_3D)
            if wl:
                txx, tyy, tzz, txy = self.StressesUVPnodes_Dealias_WL(P11, P22, P33, P12, Cs2_pad)
            else:
                txx, tyy, tzz, txy = self.StressesUVPnodes_Dealias(P11, P22, P33, P12, S_uvp_pad,
                                                                   Cs2_pad)
            W13, W23, S_w, S_w_pad = self.StrainsWnodes_Dealias(*g)
            if wl:
                txz, tyz = self.StressesWnodes_Dealias_WL(W13, W23, Cs2_pad, u, v, M_sfc_loc,
                                                          psi2D_m, psi2D_m0)
            else:
                txz, tyz = self.StressesWnodes_Dealias(W13, W23, S_w_pad, Cs2_pad, u, v, M_sfc_loc,
                                                       psi2D_m, psi2D_m0)
        else:
            S11, S22, S33, S12, S13, S23, S_uvp = self.StrainsUVPnodes_NoDealias(*g)
            S_uvp_pad = S_uvp
            if wl:
                las = self.LASDD_WL(u, v, w, S11, S22, S33, S12, S13, S23)
                Cs2_3D = las[11]
                txx, tyy, tzz, txy = self.StressesUVPnodes_NoDealias_WL(S11, S22, S33, S12, Cs2_3D)
            else:
                las = self.LASDD(u, v, w, S11, S22, S33, S12, S13, S23, S_uvp)
                Cs2_3D = las[11]
                txx, tyy, tzz, txy = self.StressesUVPnodes_NoDealias(S11, S22, S33, S12, S_uvp,
                                                                     Cs2_3D)
            W13, W23, S_w = self.StrainsWnodes_NoDealias(*g)
            S_w_pad = S_w
            if wl:
                txz, tyz = self.StressesWnodes_NoDealias_WL(W13, W23, Cs2_3D, u, v, M_sfc_loc,
                                                            psi2D_m, psi2D_m0)
            else:
                txz, tyz = self.StressesWnodes_NoDealias(W13, W23, S_w, Cs2_3D, u, v, M_sfc_loc,
                                                         psi2D_m, psi2D_m0)
        (u_, v_, w_, u_h, v_h, w_h, u_d, v_d, w_d, S_hat, S_hatd, _, avg1, avg2, beta1) = las
        return (txx, tyy, tzz, txy, txz, tyz, avg1, avg2, beta1, Cs2_3D,
                u_, v_, w_, u_h, v_h, w_h, u_d, v_d, w_d,
                S_uvp, S_uvp_pad, S_w, S_w_pad, S_hat, S_hatd)

    def DynamicSGSscalar(self, u_, v_, w_, u_hat, v_hat, w_hat, u_hatd, v_hatd, w_hatd,
                         S_uvp, S_uvp_pad, S_w, S_w_pad, S_uvp_hat, S_uvp_hatd,
                         TH, dTHdx, dTHdy, dTHdz, qz_sfc,
                         ZeRo3D=None, ZeRo3D_fft=None, ZeRo3D_pad_fft=None):
        if self._wl:
            r3, r1, beta2 = self.ScalarLASDD_WL(u_, v_, w_, u_hat, v_hat, w_hat, u_hatd, v_hatd,
                                                w_hatd, TH, dTHdx, dTHdy, dTHdz)
        else:
            r3, r1, beta2 = self.ScalarLASDD(u_, v_, w_, u_hat, v_hat, w_hat, u_hatd, v_hatd,
                                             w_hatd, TH, dTHdx, dTHdy, dTHdz, S_uvp, S_uvp_hat,
                                             S_uvp_hatd)
        qx, qy, qz = self.StaticSGSscalar(S_uvp, S_uvp_pad, S_w, S_w_pad, r3,
                                          dTHdx, dTHdy, dTHdz, qz_sfc)
        return qx, qy, qz, r3, r1, beta2

    def StaticSGS(self, dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz, Cs2_3D,
                  u, v, M_sfc_loc, psi2D_m, psi2D_m0,
                  ZeRo3D=None, ZeRo3D_fft=None, ZeRo3D_pad_fft=None):
        g = (dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz)
        wl = self._wl
        if self.optDealias == 1:
            (S11, S22, S33, S12, S13, S23, S_uvp,
             P11, P22, P33, P12, P13, P23, S_uvp_pad) = self.StrainsUVPnodes_Dealias(*g)
            Cs2_pad = self._pad(Cs2_3D)
            if wl:
                txx, tyy, tzz, txy = self.StressesUVPnodes_Dealias_WL(P11, P22, P33, P12, Cs2_pad)
            else:
                txx, tyy, tzz, txy = self.StressesUVPnodes_Dealias(P11, P22, P33, P12, S_uvp_pad,
                                                                   Cs2_pad)
            W13, W23, S_w, S_w_pad = self.StrainsWnodes_Dealias(*g)
            if wl:
                txz, tyz = self.StressesWnodes_Dealias_WL(W13, W23, Cs2_pad, u, v, M_sfc_loc,
                                                          psi2D_m, psi2D_m0)
            else:
                txz, tyz = self.StressesWnodes_Dealias(W13, W23, S_w_pad, Cs2_pad, u, v, M_sfc_loc,
                                                       psi2D_m, psi2D_m0)
        else:
            S11, S22, S33, S12, S13, S23, S_uvp = self.StrainsUVPnodes_NoDealias(*g)
            S_uvp_pad = S_uvp
            if wl:
                txx, tyy, tzz, txy = self.StressesUVPnodes_NoDealias_WL(S11, S22, S33, S12, Cs2_3D)
            else:
                txx, tyy, tzz, txy = self.StressesUVPnodes_NoDealias(S11, S22, S33, S12, S_uvp,
                                                                     Cs2_3D)
            W13, W23, S_w = self.StrainsWnodes_NoDealias(*g)
            S_w_pad = S_w
            if wl:
                txz, tyz = self.StressesWnodes_NoDealias_WL(W13, W23, Cs2_3D, u, v, M_sfc_loc,
                                                            psi2D_m, psi2D_m0)
            else:
                txz, tyz = self.StressesWnodes_NoDealias(W13, W23, S_w, Cs2_3D, u, v, M_sfc_loc,
                                                         psi2D_m, psi2D_m0)
        return txx, tyy, tzz, txy, txz, tyz, S_uvp, S_uvp_pad, S_w, S_w_pad

    def StaticSGSscalar(self, S_uvp, S_uvp_pad, S_w, S_w_pad, Cs2PrRatio_3D,
                        dTHdx, dTHdy, dTHdz, qz_sfc, ZeRo3D_fft=None, ZeRo3D_pad_fft=None):
        if self.optDealias == 1:
            gx, gy, gz = self._pad(dTHdx), self._pad(dTHdy), self._pad(dTHdz)
            rp = self._pad(Cs2PrRatio_3D)
            if self._wl:
                qx, qy = self.ScalarFluxesUVPnodes_Dealias_WL(gx, gy, rp)
                qz = self.ScalarFluxesWnodes_Dealias_WL(gz, rp, qz_sfc)
            else:
                qx, qy = self.ScalarFluxesUVPnodes_Dealias(gx, gy, S_uvp_pad, rp)
                qz = self.ScalarFluxesWnodes_Dealias(gz, S_w_pad, rp, qz_sfc)
        else:
            if self._wl:
                qx, qy = self.ScalarFluxesUVPnodes_NoDealias_WL(dTHdx, dTHdy, Cs2PrRatio_3D)
                qz = self.ScalarFluxesWnodes_NoDealias_WL(dTHdz, Cs2PrRatio_3D, qz_sfc)
            else:
                qx, qy = self.ScalarFluxesUVPnodes_NoDealias(dTHdx, dTHdy, S_uvp, Cs2PrRatio_3D)
                qz = self.ScalarFluxesWnodes_NoDealias(dTHdz, S_w, Cs2PrRatio_3D, qz_sfc)
        return qx, qy, qz

    # ------------------------------------------------------------------
    # src/pde/NSE_SGSTerms.py:55-249, src/pde/SCL_SGSTerms.py:55-219
    # ------------------------------------------------------------------
    def DivStress(self, txx, tyy, tzz, txy, txz, tyz, ZeRo3D, kx2, ky2):
        dxtxx = self.Derivxy(self.FFT(txx), kx2)
        dxtxy = self.Derivxy(self.FFT(txy), kx2)
        dxtxz = self.Derivxy(self.FFT(txz), kx2)
        dytyy = self.Derivxy(self.FFT(tyy), ky2)
        dytxy = self.Derivxy(self.FFT(txy), ky2)
        dytyz = self.Derivxy(self.FFT(tyz), ky2)
        dztxz = self.Derivz_Generic_w(txz)
        dztyz = self.Derivz_Generic_w(tyz)
        dztzz = self.Derivz_Generic_uvp(tzz)
        return (dxtxx + dytxy + dztxz, dxtxy + dytyy + dztyz, dxtxz + dytyz + dztzz)

    def DivStressDynamicSGS(self, dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz,
                            u, v, w, M_sfc_loc, MOSTfunctions,
                            ZeRo3D, ZeRo3D_fft, ZeRo3D_pad_fft, kx2, ky2):
        mom = self.DynamicSGS(dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz,
                              u, v, w, M_sfc_loc, MOSTfunctions[0], MOSTfunctions[1])
        divt = self.DivStress(*mom[0:6], None, kx2, ky2)
        return divt + (mom[6], mom[7], mom[8], mom[9], mom)

    def DivStressStaticSGS(self, dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz,
                           Cs2_3D, u, v, M_sfc_loc, MOSTfunctions,
                           ZeRo3D, ZeRo3D_fft, ZeRo3D_pad_fft, kx2, ky2):
        mom = self.StaticSGS(dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz, Cs2_3D,
                             u, v, M_sfc_loc, MOSTfunctions[0], MOSTfunctions[1])
        divt = self.DivStress(*mom[0:6], None, kx2, ky2)
        return divt + (mom,)

    def DivFlux(self, qx, qy, qz, ZeRo3D, kx2, ky2):
        return (self.Derivxy(self.FFT(qx), kx2) + self.Derivxy(self.FFT(qy), ky2)
                + self.Derivz_Generic_w(qz))

    def DivFluxDynamicSGS(self, dynamicSGSmomentum, TH, dTHdx, dTHdy, dTHdz, SHFX,
                          ZeRo3D, ZeRo3D_fft, ZeRo3D_pad_fft, kx2, ky2):
        qx, qy, qz, r3, r1, beta2 = self.DynamicSGSscalar(*dynamicSGSmomentum, TH,
                                                          dTHdx, dTHdy, dTHdz, SHFX)
        return qz, self.DivFlux(qx, qy, qz, None, kx2, ky2), r3, r1, beta2

    def DivFluxStaticSGS(self, staticSGSmomentum, Cs2PrRatio_3D, dTHdx, dTHdy, dTHdz, SHFX,
                         ZeRo3D, ZeRo3D_fft, ZeRo3D_pad_fft, kx2, ky2):
        qx, qy, qz = self.StaticSGSscalar(*staticSGSmomentum, Cs2PrRatio_3D,
                                          dTHdx, dTHdy, dTHdz, SHFX)
        return qz, self.DivFlux(qx, qy, qz, None, kx2, ky2)

    # ------------------------------------------------------------------
    # src/pde/NSE_AllTerms.py:48-104, src/pde/SCL_AllTerms.py:48-82
    # ------------------------------------------------------------------
    def RHS_Momentum(self, u, v, w, Ug, Vg, Cx, Cy, Cz, buoyancy, divtx, divty, divtz,
                     RayleighDampCoeff, RayleighDampCoeff_stag, Uadv, Vadv):
        f = self.f_coriolis_nondim
        ru = -Cx - divtx - f * (Vg - v)
        rv = -Cy - divty + f * (Ug - self.Ugal - u)
        rw = -Cz - divtz + buoyancy
        if self.cfg["optAdvection"] >= 1:
            ru = ru + Uadv
            rv = rv + Vadv
        if self.cfg["optDamping"] == 1:
            ub = self.PlanarMean(u).reshape(1, 1, -1)
            vb = self.PlanarMean(v).reshape(1, 1, -1)
            ru = ru - RayleighDampCoeff_stag * (u - ub)
            rv = rv - RayleighDampCoeff_stag * (v - vb)
            rw = rw - RayleighDampCoeff * w
        return ru, rv, rw

    def RHS_Scalar(self, TH, THAdvectionSum, divq, RayleighDampCoeff_stag, THadv):
        r = -THAdvectionSum - divq
        if self.cfg["optAdvection"] >= 1:
            r = r + THadv
        if self.cfg["optDamping"] == 1:
            r = r - RayleighDampCoeff_stag * (TH - self.PlanarMean(TH).reshape(1, 1, -1))
        return r

    def RHS_Moisture(self, Q, QAdvectionSum, divqm, RayleighDampCoeff_stag, Qadv):
        """``SCL_AllTerms.py:86-110``: Qadv is always added (zero when no
        forcing is prescribed)."""
        r = -QAdvectionSum - divqm + Qadv
        if self.cfg["optDamping"] == 1:
            r = r - RayleighDampCoeff_stag * (Q - self.PlanarMean(Q).reshape(1, 1, -1))
        return r

    # ------------------------------------------------------------------
    # src/pde/NSE_PressureTerms.py:55-335, NSE_PressureTerms_Thomas.py:74-292
    # ------------------------------------------------------------------
    def _pressure_coeffs(self):
        nx, nyr, nz, dz = self.nx, self.ny_rfft, self.nz, self.dz
        kr = np.where(np.arange(nx) < nx // 2, np.arange(nx), np.arange(nx) - nx).astype(float)
        kr2 = np.repeat(kr[:, None], nyr, axis=1)
        kc2 = np.repeat(np.arange(nyr, dtype=float)[None, :], nx, axis=0)
        a = np.ones(nz + 1) / (dz ** 2)
        c = np.ones(nz + 1) / (dz ** 2)
        a[0], a[nz] = 0, -1
        c[0], c[nz] = 1, 0
        bb = -(kr2 ** 2 + kc2 ** 2 + 2 / (dz ** 2))
        b = np.repeat(bb[:, :, None], nz + 1, axis=2)
        b[:, :, 0] = -1
        b[:, :, nz] = 1
        return kr2, kc2, a, b, c

    def PressureInit(self):
        return self._pressure_coeffs()

    @staticmethod
    def _thomas_factorize(a, b, c):
        bm = b.copy()
        N = b.shape[-1]
        m = np.zeros((N - 1,) + b.shape[:-1])
        for k in range(1, N):
            m[k - 1] = a[k] / bm[..., k - 1]
            bm[..., k] = bm[..., k] - m[k - 1] * c[k - 1]
        return bm, m

    @staticmethod
    def _thomas_solve(m, bm, c, d):
        N = d.shape[-1]
        d = d.copy()
        for k in range(1, N):
            d[..., k] = d[..., k] - m[k - 1] * d[..., k - 1]
        x = np.zeros_like(d)
        x[..., N - 1] = d[..., N - 1] / bm[..., N - 1]
        for k in range(N - 2, -1, -1):
            x[..., k] = (d[..., k] - c[k] * x[..., k + 1]) / bm[..., k]
        return x

    def ThomasPressureInit(self):
        kr2, kc2, a, b, c = self._pressure_coeffs()
        nz, dz = self.nz, self.dz
        b_safe = b.copy()
        b_safe[0, 0, 1:nz] = -(1.0 + 2.0 / dz ** 2)
        bt, mt = self._thomas_factorize(a, b_safe, c)
        return kr2, kc2, a, b, c, bt, mt

    def PressureRC(self, u, v, w, RHS_u, RHS_v, RHS_w, RHS_u_previous, RHS_v_previous,
                   RHS_w_previous, divtz, kr2_pressure, kc2_pressure):
        nx, nyr, nz, dz, dt = self.nx, self.ny_rfft, self.nz, self.dz, self.dt_nondim
        Rx = RHS_u - (1 / 3) * RHS_u_previous + (2 / (3 * dt)) * u
        Ry = RHS_v - (1 / 3) * RHS_v_previous + (2 / (3 * dt)) * v
        Rz = RHS_w - (1 / 3) * RHS_w_previous + (2 / (3 * dt)) * w
        fRx, fRy, fRz = self.FFT(Rx), self.FFT(Ry), self.FFT(Rz)
        RCr = np.zeros((nx, nyr, nz + 1))
        RCi = np.zeros((nx, nyr, nz + 1))
        fb = _rfft2(divtz[:, :, 0])
        ft = _rfft2(divtz[:, :, -1])
        RCr[:, :, 0] = -dz * fb.real
        RCi[:, :, 0] = -dz * fb.imag
        RCr[:, :, nz] = -dz * ft.real
        RCi[:, :, nz] = -dz * ft.imag
        kr = kr2_pressure[:, :, None]
        kc = kc2_pressure[:, :, None]
        hr = -kr * fRx[:, :, :-1].imag
        hr = hr - kc * fRy[:, :, :-1].imag
        hi = kr * fRx[:, :, :-1].real
        hi = hi + kc * fRy[:, :, :-1].real
        RCr[:, :, 1:nz] = hr + np.diff(fRz.real, axis=2) / dz
        RCi[:, :, 1:nz] = hi + np.diff(fRz.imag, axis=2) / dz
        return RCr, RCi, fRz.real.copy()

    def _pressure_from_modes(self, fp_real, fp_imag, RC_real, fRz_real):
        nz, dz = self.nz, self.dz
        zm = np.empty(nz)
        zm[0] = RC_real[0, 0, 0]
        zm[1:] = RC_real[0, 0, 0] + np.cumsum(fRz_real[0, 0, 1:nz] * dz)
        fp_real = fp_real.copy()
        fp_imag = fp_imag.copy()
        fp_real[0, 0] = zm
        fp_imag[0, 0] = 0.0
        p = self._irfft2(fp_real + 1j * fp_imag, (self.nx, self.ny))
        kx2, ky2 = self.Wavenumber()
        pf = self.FFT(p)
        return p, self.Derivxy(pf, kx2), self.Derivxy(pf, ky2), self.Derivz_Generic_uvp(p)

    def ThomasPressureSolve(self, RC_real, RC_imag, fRz_real, b_thomas, m_thomas, c_pressure):
        nxr, nyr = self.nx_rfft, self.ny_rfft
        Rr, Ri = RC_real.copy(), RC_imag.copy()
        for R in (Rr, Ri):
            R[0, 0, :] = 0.0
            R[nxr - 1, :, :] = 0.0
            R[:, nyr - 1, :] = 0.0
        xr = self._thomas_solve(m_thomas, b_thomas, c_pressure, Rr)
        xi = self._thomas_solve(m_thomas, b_thomas, c_pressure, Ri)
        return self._pressure_from_modes(xr[..., 1:], xi[..., 1:], RC_real, fRz_real)

    def PressureSolve(self, RC_real, RC_imag, fRz_real, a_pressure, b_pressure, c_pressure):
        """Dense per-mode solve (``optPressureSolver=0``): zero, x-Nyquist
        and y-Nyquist modes are skipped (left zero)."""
        nx, nyr, nz = self.nx, self.ny_rfft, self.nz
        fr = np.zeros((nx, nyr, nz))
        fi = np.zeros((nx, nyr, nz))
        for i in range(nx):
            for j in range(nyr):
                if (i == 0 and j == 0) or i == self.nx_rfft - 1 or j == nyr - 1:
                    continue
                A = (np.diag(b_pressure[i, j]) + np.diag(a_pressure[1:], -1)
                     + np.diag(c_pressure[:nz], 1))
                fr[i, j] = np.linalg.solve(A, RC_real[i, j])[1:]
                fi[i, j] = np.linalg.solve(A, RC_imag[i, j])[1:]
        return self._pressure_from_modes(fr, fi, RC_real, fRz_real)

    # ------------------------------------------------------------------
    # src/pde/NSE_TimeAdvancement.py:45-76, SCL_TimeAdvancement.py:46-71
    # ------------------------------------------------------------------
    def AB2_uvw(self, u, v, w, Ru, Rup, Rv, Rvp, Rw, Rwp):
        dt, nz = self.dt_nondim, self.nz
        un = u + dt * (1.5 * Ru - 0.5 * Rup)
        vn = v + dt * (1.5 * Rv - 0.5 * Rvp)
        wn = w + dt * (1.5 * Rw - 0.5 * Rwp)
        un[:, :, nz - 1] = un[:, :, nz - 2]
        vn[:, :, nz - 1] = vn[:, :, nz - 2]
        wn[:, :, nz - 1] = 0.0
        wn[:, :, 0] = 0.0
        return un, vn, wn

    def AB2_TH(self, TH, R, Rp):
        dt, nz = self.dt_nondim, self.nz
        t = TH + dt * (1.5 * R - 0.5 * Rp)
        t[:, :, nz - 1] = t[:, :, nz - 2] + self.inversion_nondim * self.dz
        return t

    def AB2_Q(self, Q, R, Rp):
        """``SCL_TimeAdvancement.py:79-99``."""
        dt, nz = self.dt_nondim, self.nz
        q = Q + dt * (1.5 * R - 0.5 * Rp)
        q[:, :, nz - 1] = q[:, :, nz - 2] + self.q_inversion_nondim * self.dz
        return q

    # ------------------------------------------------------------------
    # src/initialization/Initialization.py:58-460
    # ------------------------------------------------------------------
    def Initialize_RayleighDampingLayer(self):
        nx, ny, nz, dz = self.nx, self.ny, self.nz, self.dz
        inv = 1.0 / self.RelaxTime_nondim
        ztop = self.cfg["l_z"] / self.z_scale
        thick = ztop - self.z_damping_nondim

        def coeff(z):
            m = (z >= self.z_damping_nondim) & (z <= ztop)
            with np.errstate(divide="ignore", invalid="ignore"):
                val = 0.5 * inv * (1.0 - np.cos(PI * (z - self.z_damping_nondim) / thick))
            return np.where(m, val, 0.0)

        c1 = coeff(np.arange(nz) * dz)
        c2 = coeff((np.arange(nz) + 0.5) * dz)
        return (np.broadcast_to(c1.reshape(1, 1, nz), (nx, ny, nz)),
                np.broadcast_to(c2.reshape(1, 1, nz), (nx, ny, nz)))

    def initial_state(self, u, v, w, th):
        """``Initialize_uvw``/``Initialize_TH`` applied to dimensional fields
        (u total, theta absolute): u -= Ugal, theta -= T_0."""
        return (u - self.Ugal) / self.u_scale, v / self.u_scale, w / self.u_scale, th - self.T_0_nondim

    def surface_series(self, series_dim):
        """``Initialize_SurfaceBC`` non-dimensionalisation (``:151-158``)."""
        if self.cfg["optSurfBC"] == 1:
            return series_dim / (self.u_scale * self.TH_scale)
        return (series_dim - self.cfg["T_0"]) / self.TH_scale

    def geowind_series(self, Ug, Vg):
        """``Initialize_GeoWind_Varying`` non-dimensionalisation
        (``Initialization.py:241-244``): (nsteps+1, nz) rows / u_scale."""
        return np.asarray(Ug) / self.u_scale, np.asarray(Vg) / self.u_scale

    def adv_series(self, U, V, T):
        """``Initialize_AdvForcing`` non-dimensionalisation (``:305-314``)."""
        return (U * self.z_scale / self.u_scale ** 2, V * self.z_scale / self.u_scale ** 2,
                T * self.z_scale / (self.u_scale * self.TH_scale))


# ----------------------------------------------------------------------
# src/utilities/Statistics.py:47-380: plane-averaged statistics (dry:
# the moisture entries accumulate zeros)
# ----------------------------------------------------------------------
STATS_PROFILE_KEYS = ("U", "V", "W", "TH", "dUdz", "dVdz", "dTHdz",
                      "u2", "v2", "w2", "TH2", "uv", "uw", "vw", "uTH", "vTH", "wTH",
                      "txy", "txz", "tyz", "qz", "Cs2_1", "Cs2_2", "Cs2PrRatio",
                      "Beta1", "Beta2", "Q", "dQdz", "Q2", "wQ", "qHz")
STATS_SCALAR_KEYS = ("M_sfc", "ustar", "qz_sfc", "qm_sfc")


def InitializeStats(o, nz):
    """``Statistics.py:335-380``."""
    d = {k: np.zeros(nz) for k in STATS_PROFILE_KEYS}
    d.update({k: 0.0 for k in STATS_SCALAR_KEYS})
    d["Ugal"] = o.Ugal
    d["ZeRo1D"] = np.zeros(nz)
    return d


def ComputeStats(o, u, v, w, TH, Q, dudz, dvdz, dTHdz, dQdz, M_sfc_loc, ustar, qz_sfc_avg,
                 qm_sfc_avg, txy, txz, tyz, qz, qHz_q, Cs2_1D_avg1, Cs2_1D_avg2, Cs2PrRatio_1D,
                 beta1_1D, beta2_1D, StatsDict, ResetFlag):
    """``Statistics.py:47-328`` with the reference's argument order; a dry run
    passes None (zeros) for Q, dQdz, qHz_q and qm_sfc_avg."""
    nz = o.nz
    if ResetFlag == 1:
        return InitializeStats(o, nz) | {"Ugal": StatsDict["Ugal"]}
    us, ts, zs = o.u_scale, o.TH_scale, o.z_scale
    Ugal = StatsDict["Ugal"]
    m = lambda f: np.mean(f, axis=(0, 1))
    mU = (m(u) + Ugal) * us
    mV = m(v) * us
    mW = m(w) * us
    mTH_anom = m(TH)
    mTH = (mTH_anom + o.T_0_nondim) * ts
    new = {}
    new["U"], new["V"], new["W"], new["TH"] = mU, mV, mW, mTH
    new["dUdz"] = m(dudz) * (us / zs)
    new["dVdz"] = m(dvdz) * (us / zs)
    new["dTHdz"] = m(dTHdz) * (ts / zs)
    uf = u + Ugal - mU
    vf = v - mV
    wf = w - mW
    Tf = TH - mTH_anom
    new["u2"] = m(uf ** 2) * us ** 2
    new["v2"] = m(vf ** 2) * us ** 2
    new["w2"] = m(wf ** 2) * us ** 2
    new["TH2"] = m(Tf ** 2) * ts ** 2
    new["uv"] = m(uf * vf) * us ** 2
    new["uTH"] = m(uf * Tf) * (us * ts)
    new["vTH"] = m(vf * Tf) * (us * ts)
    u_st = np.zeros_like(u)
    v_st = np.zeros_like(v)
    T_st = np.zeros_like(TH)
    u_st[:, :, 1:nz] = o.StagGridAvg(u)
    v_st[:, :, 1:nz] = o.StagGridAvg(v)
    T_st[:, :, 1:nz] = o.StagGridAvg(TH)
    u_st[:, :, 0] = u[:, :, 0] + Ugal
    v_st[:, :, 0] = v[:, :, 0]
    T_st[:, :, 0] = TH[:, :, 0]
    mu_st = (m(u_st) + Ugal) * us
    mv_st = m(v_st) * us
    mw_st = m(w) * us
    mT_st = m(T_st) * ts
    usf = u_st + Ugal - mu_st
    vsf = v_st - mv_st
    wsf = w - mw_st
    Tsf = T_st - mT_st
    new["uw"] = m(usf * wsf) * us ** 2
    new["vw"] = m(vsf * wsf) * us ** 2
    new["wTH"] = m(wsf * Tsf) * (us * ts)
    new["txy"] = m(txy) * us ** 2
    new["txz"] = m(txz) * us ** 2
    new["tyz"] = m(tyz) * us ** 2
    new["qz"] = m(qz) * (us * ts)
    new["Cs2_1"], new["Cs2_2"], new["Cs2PrRatio"] = Cs2_1D_avg1, Cs2_1D_avg2, Cs2PrRatio_1D
    new["Beta1"], new["Beta2"] = beta1_1D, beta2_1D
    if Q is None:
        for k in ("Q", "dQdz", "Q2", "wQ", "qHz"):
            new[k] = np.zeros(nz)
    else:  # Statistics.py:166-168, 199-201, 231-256, 275 (Q_scale = 1)
        qs = o.Q_scale
        mQ = m(Q) * qs
        new["Q"] = mQ
        new["dQdz"] = m(dQdz) * (qs / zs)
        new["Q2"] = m((Q - mQ / qs) ** 2) * qs ** 2
        Q_st = np.zeros_like(Q)
        Q_st[:, :, 1:nz] = o.StagGridAvg(Q)
        Q_st[:, :, 0] = Q[:, :, 0]
        mQ_st = m(Q_st) * qs
        new["wQ"] = m(wsf * (Q_st - mQ_st / qs)) * (us * qs)
        new["qHz"] = m(qHz_q) * (us * qs)
    new["M_sfc"] = np.mean(M_sfc_loc)
    new["ustar"] = np.sqrt(np.mean(ustar ** 2)) * us
    new["qz_sfc"] = qz_sfc_avg * us * ts
    new["qm_sfc"] = 0.0 if qm_sfc_avg is None else qm_sfc_avg * us * o.Q_scale
    out = {k: StatsDict[k] + new[k] for k in STATS_PROFILE_KEYS + STATS_SCALAR_KEYS}
    out["Ugal"] = Ugal
    out["ZeRo1D"] = StatsDict["ZeRo1D"]
    return out


class OracleRun:
    """The time loop of ``src/Main.py:46-541`` on the oracle (dry, optSgs 0-4,
    constant or time/height-varying geostrophic wind).  ``step()`` advances one iteration
    and keeps the same state variables Main.py keeps between iterations."""

    def __init__(self, cfg, u, v, w, th, surface_series=None, adv=None, geowind=None,
                 Q=None, moisture_series=None):
        """Q: the initial specific humidity (kg/kg, as Initialize_Q loads it)
        when optMoisture >= 1; moisture_series: the non-dimensional
        Initialize_MoistureSurfaceBC series (optMoistureSurfBC >= 1); adv may
        carry a fourth, Qadv, series."""
        o = self.o = AlfaOracle(cfg)
        self.cfg = o.cfg
        self.kx2, self.ky2 = o.Wavenumber()
        if cfg["optPressureSolver"] == 1:
            (self.kr2, self.kc2, self.a_p, self.b_p, self.c_p,
             self.b_thomas, self.m_thomas) = o.ThomasPressureInit()
        else:
            self.kr2, self.kc2, self.a_p, self.b_p, self.c_p = o.PressureInit()
        self.u, self.v, self.w, self.TH = o.initial_state(u, v, w, th)
        shp = (o.nx, o.ny, o.nz)
        self.Ug = cfg["Ug2"] * np.ones(shp) / o.u_scale
        self.Vg = cfg["Vg2"] * np.ones(shp) / o.u_scale
        self.Rd, self.Rd_stag = o.Initialize_RayleighDampingLayer()
        self.RHS_prev = [np.zeros(shp) for _ in range(4)]
        z2 = np.zeros((o.nx, o.ny))
        self.MOST = (z2.copy(), z2.copy(), z2.copy(), z2.copy(), 1.0 + z2, 1.0 + z2)
        self.surface = surface_series
        self.adv = adv
        self.geowind = geowind  # non-dimensional (Ug, Vg) rows when optGeoWind >= 1
        self.moist = int(cfg.get("optMoisture", 0)) >= 1
        if self.moist:  # Main.py:71-76
            self.Q = np.array(Q, dtype=np.float64)
            self.RHS_prev.append(np.zeros(shp))
            self.moisture_series = moisture_series
        self.Cs2_3D = o.Cs2_init * np.ones(shp)
        self.Cs2PrRatio_3D = o.Cs2PrRatio_init * np.ones(shp)
        self.iteration = int(cfg["istep"])
        self.istep = int(cfg["istep"])
        self.CFLmax = 0.0
        self.last = {}
        nz = o.nz  # coefficient profiles start at zero (Main.py:141-145)
        self.Cs2_1D_avg1, self.Cs2_1D_avg2, self.Cs2PrRatio_1D = (np.zeros(nz) for _ in range(3))
        self.beta1_1D, self.beta2_1D = np.zeros(nz), np.zeros(nz)

    def step(self):
        o, it, c = self.o, self.iteration, self.cfg
        nz = o.nz
        zero3 = None
        if it > self.istep:
            self.RHS_prev = list(self.RHS)
        if c.get("optGeoWind", 0) >= 1:  # Main.py:170-174
            GU, GV = self.geowind
            self.Ug = np.broadcast_to(GU[it - 1].reshape(1, 1, nz), self.u.shape)
            self.Vg = np.broadcast_to(GV[it - 1].reshape(1, 1, nz), self.u.shape)
        Qadv = np.zeros(self.u.shape)
        if c["optAdvection"] >= 1:
            U, V, T = self.adv[:3]
            Uadv = np.broadcast_to(U[it - 1].reshape(1, 1, nz), self.u.shape)
            Vadv = np.broadcast_to(V[it - 1].reshape(1, 1, nz), self.u.shape)
            THadv = np.broadcast_to(T[it - 1].reshape(1, 1, nz), self.u.shape)
            if self.moist and len(self.adv) > 3:
                Qadv = np.broadcast_to(self.adv[3][it - 1].reshape(1, 1, nz), self.u.shape)
        else:
            Uadv = Vadv = THadv = np.zeros(self.u.shape)
        u, u_fft = o.Filtering_Explicit(o.FFT(self.u))
        v, v_fft = o.Filtering_Explicit(o.FFT(self.v))
        w, w_fft = o.Filtering_Explicit(o.FFT(self.w))
        TH, _ = o.Filtering_Explicit(o.FFT(self.TH))
        if self.moist:
            Q, _ = o.Filtering_Explicit(o.FFT(self.Q))
        if c["optSurfBC"] == 0:
            f = (o.SurfaceFlux_HomogeneousConstantFlux if c["optSurfFlux"] == 0
                 else o.SurfaceFlux_HeterogeneousConstantFlux)
            M, ustar, qavg, invOB, self.MOST = f(u, v, TH, self.MOST)
            qz_step = o.qz_sfc
        else:
            val = self.surface[it - 1]
            if c["optSurfBC"] == 1:
                f = (o.SurfaceFlux_HomogeneousVaryingFlux if c["optSurfFlux"] == 0
                     else o.SurfaceFlux_HeterogeneousVaryingFlux)
            else:
                f = (o.SurfaceFlux_HomogeneousPrescribedTemperature if c["optSurfFlux"] == 0
                     else o.SurfaceFlux_HeterogeneousPrescribedTemperature)
            M, ustar, qz_step, qavg, invOB, self.MOST = f(u, v, TH, val, self.MOST)
        if self.moist:  # Main.py:253-267
            mb = c.get("optMoistureSurfBC", 0)
            if mb == 0:
                qm_step = o.qm_sfc
            elif mb == 1:
                qm_step = self.moisture_series[it - 1] * np.ones((o.nx, o.ny))
            else:
                fq = (o.SurfaceMoistureFlux_HomogeneousPrescribedQ if c["optSurfFlux"] == 0
                      else o.SurfaceMoistureFlux_HeterogeneousPrescribedQ)
                qm_step = fq(Q, ustar, self.moisture_series[it - 1], self.MOST)
        grads = o.velocityGradients(u, v, w, u_fft, v_fft, w_fft, self.kx2, self.ky2,
                                    ustar, M, self.MOST)
        dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz = grads
        dTHdx, dTHdy, dTHdz = o.potentialTemperatureGradients(TH, self.kx2, self.ky2, ustar,
                                                              qz_step, self.MOST)
        Cx, Cy, Cz = o.Advection(u, v, w, dudy, dudz, dvdx, dvdz, dwdx, dwdy)
        THadvsum = o.ScalarAdvection(u, v, w, dTHdx, dTHdy, dTHdz)
        if self.moist:
            dQdx, dQdy, dQdz = o.moistureGradients(Q, self.kx2, self.ky2, ustar, qm_step,
                                                   self.MOST)
            Qadvsum = o.ScalarAdvection(u, v, w, dQdx, dQdy, dQdz)
        H = Q if self.moist else np.zeros(u.shape)
        buoy = o.BuoyancyOpt1(TH, H) if c["optBuoyancy"] == 0 else o.BuoyancyOpt2(TH, H)
        dyn = 1 <= o.optSgs <= 4 and (it == self.istep or it % c["dynamicSGS_call_time"] == 0)
        if dyn:
            (divtx, divty, divtz, self.Cs2_1D_avg1, self.Cs2_1D_avg2, self.beta1_1D,
             self.Cs2_3D, mom) = o.DivStressDynamicSGS(*grads, u, v, w, M, self.MOST,
                                                       zero3, zero3, zero3, self.kx2, self.ky2)
            qz, divq, self.Cs2PrRatio_3D, self.Cs2PrRatio_1D, self.beta2_1D = \
                o.DivFluxDynamicSGS(mom[10:], TH, dTHdx, dTHdy, dTHdz, qz_step,
                                    zero3, zero3, zero3, self.kx2, self.ky2)
            strains = mom[19:23]
        else:
            divtx, divty, divtz, mom = o.DivStressStaticSGS(
                *grads, self.Cs2_3D, u, v, M, self.MOST, zero3, zero3, zero3, self.kx2, self.ky2)
            qz, divq = o.DivFluxStaticSGS(mom[6:], self.Cs2PrRatio_3D, dTHdx, dTHdy, dTHdz,
                                          qz_step, zero3, zero3, zero3, self.kx2, self.ky2)
            strains = mom[6:]
        if self.moist:  # Main.py:358-369, 444-453: heat's Cs2PrRatio and strains
            qHz_q, divqm = o.DivFluxStaticSGS(strains, self.Cs2PrRatio_3D, dQdx, dQdy, dQdz,
                                              qm_step, zero3, zero3, zero3, self.kx2, self.ky2)
        Ru, Rv, Rw = o.RHS_Momentum(u, v, w, self.Ug, self.Vg, Cx, Cy, Cz, buoy,
                                    divtx, divty, divtz, self.Rd, self.Rd_stag, Uadv, Vadv)
        RT = o.RHS_Scalar(TH, THadvsum, divq, self.Rd_stag, THadv)
        if self.moist:
            RQ = o.RHS_Moisture(Q, Qadvsum, divqm, self.Rd_stag, Qadv)
        RCr, RCi, fRz = o.PressureRC(u, v, w, Ru, Rv, Rw, *self.RHS_prev[:3], divtz,
                                     self.kr2, self.kc2)
        if c["optPressureSolver"] == 1:
            p, dpdx, dpdy, dpdz = o.ThomasPressureSolve(RCr, RCi, fRz, self.b_thomas,
                                                        self.m_thomas, self.c_p)
        else:
            p, dpdx, dpdy, dpdz = o.PressureSolve(RCr, RCi, fRz, self.a_p, self.b_p, self.c_p)
        Ru, Rv, Rw = Ru - dpdx, Rv - dpdy, Rw - dpdz
        self.RHS = [Ru, Rv, Rw, RT] + ([RQ] if self.moist else [])
        if it == self.istep:
            self.RHS_prev = list(self.RHS)
        self.u, self.v, self.w = o.AB2_uvw(u, v, w, Ru, self.RHS_prev[0], Rv, self.RHS_prev[1],
                                           Rw, self.RHS_prev[2])
        self.TH = o.AB2_TH(TH, RT, self.RHS_prev[3])
        if self.moist:
            self.Q = o.AB2_Q(Q, RQ, self.RHS_prev[4])
            self.last.update(Q_filtered=Q, dQdz=dQdz, qHz_q=qHz_q, qm_sfc_step=qm_step)
        self.p = p
        cfl = max(np.max(np.abs(self.u)) * o.dt_nondim / o.dx,
                  np.max(np.abs(self.v)) * o.dt_nondim / o.dy,
                  np.max(np.abs(self.w)) * o.dt_nondim / o.dz)
        self.CFL = cfl
        self.CFLmax = max(self.CFLmax, cfl)
        self.ustar, self.M_sfc_loc, self.qz_sfc_avg = ustar, M, qavg
        self.last.update(dudz=grads[6], dvdz=grads[7], dTHdz=dTHdz, txy=mom[3], txz=mom[4],
                         tyz=mom[5], qz=qz, grads=grads)
        self.iteration += 1
        return self

    def stats_sample(self, StatsDict):
        """ComputeStats with the arguments Main.py:550-558 passes after this
        iteration."""
        L = self.last
        moist = self.moist
        return ComputeStats(self.o, self.u, self.v, self.w, self.TH,
                            self.Q if moist else None, L["dudz"], L["dvdz"], L["dTHdz"],
                            L["dQdz"] if moist else None, self.M_sfc_loc, self.ustar,
                            float(self.qz_sfc_avg),
                            float(np.mean(L["qm_sfc_step"])) if moist else None,
                            L["txy"], L["txz"], L["tyz"], L["qz"],
                            L["qHz_q"] if moist else None, self.Cs2_1D_avg1,
                            self.Cs2_1D_avg2, self.Cs2PrRatio_1D, self.beta1_1D, self.beta2_1D,
                            StatsDict, 0)
