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
    def __init__(self, cfg, u, v, w, th, surface_series=None, adv_series=None, api=None,
                 geowind_series=None, Q=None, moisture_series=None):
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
            self.adv = torch.from_numpy(np.stack([x * z for x in adv_series[:3]], axis=1).astype(np.float64)).pin_memory()
        self.sfc = None
        if surface_series is not None:
            s = np.asarray(surface_series, dtype=np.float64)
            self.sfc = s if cfg["optSurfBC"] == 1 else s - cfg["T_0"]
        # moisture (Main.py:71-76): Q in kg/kg; the moisture surface series
        # and Qadv (a fourth adv_series entry) non-dimensionalised with
        # u_scale = Q_scale = 1
        self.moist = int(cfg.get("optMoisture", 0)) >= 1
        if self.moist:
            self.Q = tt(Q)
            self.RHS_prev.append(zeros(N))
            self.qm_sfc = zeros(H) + float(cfg.get("MoistureFlux", 0.0))
            self.msfc = (None if moisture_series is None
                         else np.asarray(moisture_series, dtype=np.float64))
            self.qadv = None
            if adv_series is not None and len(adv_series) > 3:
                self.qadv = torch.from_numpy(np.asarray(adv_series[3] * z, dtype=np.float64)).pin_memory()
        self.geo = None  # Main.py:84-86, 170-174 (u_scale = 1)
        if int(cfg.get("optGeoWind", 0)) >= 1:
            if geowind_series is None:
                raise ValueError("optGeoWind >= 1 needs geowind_series (Ug, Vg)")
            self.geo = torch.from_numpy(np.stack([np.asarray(x, dtype=np.float64)
                                                  for x in geowind_series], axis=1)).pin_memory()
        self.CFLmax = 0.0
        self.h2d_bytes = 0
        self.d2h_bytes = 0

    def step(self):
        a, c, it = self.a, self.cfg, self.iteration
        if it > self.istep:
            self.RHS_prev = self.RHS
        if self.geo is not None:
            row = self.geo[it - 1].to(a.device, non_blocking=True)
            self.h2d_bytes += row.numel() * 8
            self.Ug, self.Vg = row[0], row[1]
        if self.adv is not None:
            row = self.adv[it - 1].to(a.device, non_blocking=True)
            self.h2d_bytes += row.numel() * 8
            Uadv, Vadv, THadv = row[0], row[1], row[2]
        else:
            Uadv = Vadv = THadv = self.zero_prof
        Qadv = self.zero_prof
        if self.moist and self.qadv is not None:
            Qadv = self.qadv[it - 1].to(a.device, non_blocking=True)
            self.h2d_bytes += Qadv.numel() * 8
        u, u_fft = a.Filtering_Explicit(a.FFT(self.u))
        v, v_fft = a.Filtering_Explicit(a.FFT(self.v))
        w, w_fft = a.Filtering_Explicit(a.FFT(self.w))
        TH, _ = a.Filtering_Explicit(a.FFT(self.TH))
        if self.moist:
            Q, _ = a.Filtering_Explicit(a.FFT(self.Q))
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
        if self.moist:  # Main.py:253-267
            mb = int(c.get("optMoistureSurfBC", 0))
            if mb == 0:
                qm_step = self.qm_sfc
            elif mb == 1:
                qm_step = torch.full(a.H, float(self.msfc[it - 1]), dtype=torch.float64,
                                     device=a.device)
            else:
                fq = (a.SurfaceMoistureFlux_HomogeneousPrescribedQ if c["optSurfFlux"] == 0
                      else a.SurfaceMoistureFlux_HeterogeneousPrescribedQ)
                qm_step = fq(Q, ustar, float(self.msfc[it - 1]), self.MOST)
        grads = a.velocityGradients(u, v, w, u_fft, v_fft, w_fft, self.kx2, self.ky2, ustar, M,
                                    self.MOST)
        dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz = grads
        dTHdx, dTHdy, dTHdz = a.potentialTemperatureGradients(TH, self.kx2, self.ky2, ustar,
                                                              qz_step, self.MOST)
        Cx, Cy, Cz = a.Advection(u, v, w, dudy, dudz, dvdx, dvdz, dwdx, dwdy)
        THAdvectionSum = a.ScalarAdvection(u, v, w, dTHdx, dTHdy, dTHdz)
        H = None
        if self.moist:
            dQdx, dQdy, dQdz = a.moistureGradients(Q, self.kx2, self.ky2, ustar, qm_step,
                                                   self.MOST)
            QAdvectionSum = a.ScalarAdvection(u, v, w, dQdx, dQdy, dQdz)
            H = Q
        buoyancy = a.BuoyancyOpt1(TH, H) if c["optBuoyancy"] == 0 else a.BuoyancyOpt2(TH, H)
        if 1 <= c["optSgs"] <= 4 and (it == self.istep or it % c["dynamicSGS_call_time"] == 0):
            (divtx, divty, divtz, self.Cs2_1D_avg1, self.Cs2_1D_avg2, self.beta1_1D,
             self.Cs2_3D, mom) = a.DivStressDynamicSGS(*grads, u, v, w, M, self.MOST)
            qz, divq, self.Cs2PrRatio_3D, self.Cs2PrRatio_1D, self.beta2_1D = \
                a.DivFluxDynamicSGS(mom[10:], TH, dTHdx, dTHdy, dTHdz, qz_step)
            strains = mom[19:23]
        else:
            divtx, divty, divtz, mom = a.DivStressStaticSGS(*grads, self.Cs2_3D, u, v, M, self.MOST)
            qz, divq = a.DivFluxStaticSGS(mom[6:], self.Cs2PrRatio_3D, dTHdx, dTHdy, dTHdz, qz_step)
            strains = mom[6:]
        if self.moist:  # Main.py:358-369, 444-453
            qHz_q, divqm = a.DivFluxStaticSGS(strains, self.Cs2PrRatio_3D, dQdx, dQdy, dQdz,
                                              qm_step)
        RHS_u, RHS_v, RHS_w = a.RHS_Momentum(u, v, w, self.Ug, self.Vg, Cx, Cy, Cz, buoyancy,
                                             divtx, divty, divtz, None, None, Uadv, Vadv)
        RHS_TH = a.RHS_Scalar(TH, THAdvectionSum, divq, None, THadv)
        if self.moist:
            RHS_Q = a.RHS_Moisture(Q, QAdvectionSum, divqm, None, Qadv)
        RC_real, RC_imag, fRz_real = a.PressureRC(u, v, w, RHS_u, RHS_v, RHS_w,
                                                  *self.RHS_prev[:3], divtz)
        p, dpdx, dpdy, dpdz = a.ThomasPressureSolve(RC_real, RC_imag, fRz_real)
        RHS_u, RHS_v, RHS_w = a.AddPressureGradient(RHS_u, RHS_v, RHS_w, dpdx, dpdy, dpdz)
        self.RHS = [RHS_u, RHS_v, RHS_w, RHS_TH] + ([RHS_Q] if self.moist else [])
        if it == self.istep:
            self.RHS_prev = list(self.RHS)
        self.u, self.v, self.w = a.AB2_uvw(u, v, w, RHS_u, self.RHS_prev[0], RHS_v,
                                           self.RHS_prev[1], RHS_w, self.RHS_prev[2])
        self.TH = a.AB2_TH(TH, RHS_TH, self.RHS_prev[3])
        if self.moist:
            self.Q = a.AB2_Q(Q, RHS_Q, self.RHS_prev[4])
        self.p = p
        # CFL check on the host, as Main.py:534-540 does every step
        cfl = float(a.CFL(self.u, self.v, self.w).cpu().max())
        self.d2h_bytes += 24
        self.CFL = cfl
        self.CFLmax = max(self.CFLmax, cfl)
        self.iteration += 1
        return self
