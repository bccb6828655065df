"""The reference's time loop, statement for statement, on the libalfa
function-level API.

``MainLoop`` restates the loop body of the reference's ``src/Main.py:156-541``
(dry, constant geostrophic wind, optSgs in {0, 1, 3}) calling the
reference-named functions of ``jax_alfa_b200.api.Alfa`` instead of the JAX
ones: it is what the reference's driver looks like with libalfa dropped in
behind its function boundary.  The host holds only what Main.py holds
between calls; every array stays on the device, and, as in Main.py, the
only per-step host traffic is the forcing row going in and the CFL check
coming out (``Main.py:534-540``).
"""
import numpy as np
import torch

from .api import Alfa


class MainLoop:
    def __init__(self, cfg, u, v, w, th, surface_series=None, adv_series=None, api=None):
        a = self.a = api or Alfa(cfg)
        self.cfg = cfg
        dev = a.device
        z = a.derived.z_scale
        self.istep = int(cfg["istep"])
        self.iteration = self.istep
        N = a.N
        # Main.py:46-52 / Initialize_uvw / Initialize_TH (host arrays in)
        tt = lambda x: torch.as_tensor(np.ascontiguousarray(x, dtype=np.float64)).to(dev)
        self.u = tt(np.asarray(u) - cfg["Ugal"])
        self.v, self.w = tt(v), tt(w)
        self.TH = tt(np.asarray(th) - cfg["T_0"])
        self.kx2, self.ky2 = a.Wavenumber()
        self.Ug = torch.full((a.nz,), float(cfg["Ug2"]), dtype=torch.float64, device=dev)
        self.Vg = torch.full((a.nz,), float(cfg["Vg2"]), dtype=torch.float64, device=dev)
        zeros = lambda s: torch.zeros(s, dtype=torch.float64, device=dev)
        self.RHS_prev = [zeros(N) for _ in range(4)]
        H = a.H
        self.MOST = (zeros(H), zeros(H), zeros(H), zeros(H), zeros(H) + 1.0, zeros(H) + 1.0)
        wl = int(cfg["optSgs"]) in (2, 4)  # DerivedVars.py:101-106
        self.Cs2_3D = zeros(N) + cfg["Cwl" if wl else "Cs2"]
        self.Cs2PrRatio_3D = zeros(N) + cfg["CwlPrRatio" if wl else "Cs2PrRatio"]
        self.qz_sfc = zeros(H) + cfg["SensibleHeatFlux"]
        self.zero_prof = zeros(a.nz)
        # series stay on the host (pinned); one row goes to the device per step
        self.adv = None
        if adv_series is not None:
            self.adv = torch.from_numpy(np.stack([x * z for x in adv_series], axis=1).astype(np.float64)).pin_memory()
        self.sfc = None
        if surface_series is not None:
            s = np.asarray(surface_series, dtype=np.float64)
            self.sfc = s if cfg["optSurfBC"] == 1 else s - cfg["T_0"]
        self.CFLmax = 0.0
        self.h2d_bytes = 0
        self.d2h_bytes = 0

    def step(self):
        a, c, it = self.a, self.cfg, self.iteration
        if it > self.istep:
            self.RHS_prev = self.RHS
        if self.adv is not None:
            row = self.adv[it - 1].to(a.device, non_blocking=True)
            self.h2d_bytes += row.numel() * 8
            Uadv, Vadv, THadv = row[0], row[1], row[2]
        else:
            Uadv = Vadv = THadv = self.zero_prof
        u, u_fft = a.Filtering_Explicit(a.FFT(self.u))
        v, v_fft = a.Filtering_Explicit(a.FFT(self.v))
        w, w_fft = a.Filtering_Explicit(a.FFT(self.w))
        TH, _ = a.Filtering_Explicit(a.FFT(self.TH))
        if c["optSurfBC"] == 0:
            f = (a.SurfaceFlux_HomogeneousConstantFlux if c["optSurfFlux"] == 0
                 else a.SurfaceFlux_HeterogeneousConstantFlux)
            M, ustar, qz_avg, invOB, self.MOST = f(u, v, TH, self.MOST)
            qz_step = self.qz_sfc
        else:
            val = float(self.sfc[it - 1])
            if c["optSurfBC"] == 1:
                f = (a.SurfaceFlux_HomogeneousVaryingFlux if c["optSurfFlux"] == 0
                     else a.SurfaceFlux_HeterogeneousVaryingFlux)
            else:
                f = (a.SurfaceFlux_HomogeneousPrescribedTemperature if c["optSurfFlux"] == 0
                     else a.SurfaceFlux_HeterogeneousPrescribedTemperature)
            M, ustar, qz_step, qz_avg, invOB, self.MOST = f(u, v, TH, val, self.MOST)
        grads = a.velocityGradients(u, v, w, u_fft, v_fft, w_fft, self.kx2, self.ky2, ustar, M,
                                    self.MOST)
        dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz = grads
        dTHdx, dTHdy, dTHdz = a.potentialTemperatureGradients(TH, self.kx2, self.ky2, ustar,
                                                              qz_step, self.MOST)
        Cx, Cy, Cz = a.Advection(u, v, w, dudy, dudz, dvdx, dvdz, dwdx, dwdy)
        THAdvectionSum = a.ScalarAdvection(u, v, w, dTHdx, dTHdy, dTHdz)
        buoyancy = a.BuoyancyOpt1(TH) if c["optBuoyancy"] == 0 else a.BuoyancyOpt2(TH)
        if 1 <= c["optSgs"] <= 4 and (it == self.istep or it % c["dynamicSGS_call_time"] == 0):
            (divtx, divty, divtz, self.Cs2_1D_avg1, self.Cs2_1D_avg2, self.beta1_1D,
             self.Cs2_3D, mom) = a.DivStressDynamicSGS(*grads, u, v, w, M, self.MOST)
            qz, divq, self.Cs2PrRatio_3D, self.Cs2PrRatio_1D, self.beta2_1D = \
                a.DivFluxDynamicSGS(mom[10:], TH, dTHdx, dTHdy, dTHdz, qz_step)
        else:
            divtx, divty, divtz, mom = a.DivStressStaticSGS(*grads, self.Cs2_3D, u, v, M, self.MOST)
            qz, divq = a.DivFluxStaticSGS(mom[6:], self.Cs2PrRatio_3D, dTHdx, dTHdy, dTHdz, qz_step)
        RHS_u, RHS_v, RHS_w = a.RHS_Momentum(u, v, w, self.Ug, self.Vg, Cx, Cy, Cz, buoyancy,
                                             divtx, divty, divtz, None, None, Uadv, Vadv)
        RHS_TH = a.RHS_Scalar(TH, THAdvectionSum, divq, None, THadv)
        RC_real, RC_imag, fRz_real = a.PressureRC(u, v, w, RHS_u, RHS_v, RHS_w,
                                                  *self.RHS_prev[:3], divtz)
        p, dpdx, dpdy, dpdz = a.ThomasPressureSolve(RC_real, RC_imag, fRz_real)
        RHS_u, RHS_v, RHS_w = a.AddPressureGradient(RHS_u, RHS_v, RHS_w, dpdx, dpdy, dpdz)
        self.RHS = [RHS_u, RHS_v, RHS_w, RHS_TH]
        if it == self.istep:
            self.RHS_prev = list(self.RHS)
        self.u, self.v, self.w = a.AB2_uvw(u, v, w, RHS_u, self.RHS_prev[0], RHS_v,
                                           self.RHS_prev[1], RHS_w, self.RHS_prev[2])
        self.TH = a.AB2_TH(TH, RHS_TH, self.RHS_prev[3])
        self.p = p
        # CFL check on the host, as Main.py:534-540 does every step
        cfl = float(a.CFL(self.u, self.v, self.w).cpu().max())
        self.d2h_bytes += 24
        self.CFL = cfl
        self.CFLmax = max(self.CFLmax, cfl)
        self.iteration += 1
        return self
