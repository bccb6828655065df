"""Host-side mirror of the reference's function-level API on libalfa.

``Alfa(cfg)`` binds one configuration (the reference's Config.py option names,
see ``jax_alfa_b200.cases``) to a libalfa context.  Its methods carry the
names, argument order and return tuples of the functions the reference's
``src/Main.py`` calls, operate on torch CUDA tensors in the reference layout
(fields (nx, ny, nz) float64 z-fastest, spectra (nx, ny//2+1, nz)
complex128) and launch on torch's current stream.  Static arguments the
reference threads through (kx2, ky2, ZeRo* scratch, pressure factors,
Rayleigh arrays) are accepted for signature compatibility and taken from the
context.  PyTorch provides device memory and streams only; all arithmetic is
in libalfa's kernels.

``Simulation`` drives the whole step (``alfa_step``) with the state resident
on the device.
"""
import ctypes
import os

import numpy as np
import torch

from . import _lib

F64 = torch.float64
C128 = torch.complex128

CONFIG_KEYS = [f for f, _ in _lib.AlfaConfig._fields_]
OPTIONAL_KEYS = ("optGeoWind", "optMoisture", "optMoistureSurfBC", "MoistureFlux", "zMoisture",
                 "q_inversion")
PRECISIONS = {"fp64": _lib.FP64, "fp32": _lib.FP32, "mixed": _lib.MIXED}


def precision_of(cfg):
    """alfa_config.precision of a config: its "precision" entry ("fp64",
    "fp32", "mixed" or the ALFA_* integer), else the reference's own switch
    use_double_precision (ConfigLoader.py:150-151): True -> FP64, False ->
    FP32."""
    p = cfg.get("precision")
    if p is None:
        return _lib.FP64 if cfg.get("use_double_precision", True) else _lib.FP32
    if isinstance(p, str):
        if p.lower() not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}, not {p!r}")
        return PRECISIONS[p.lower()]
    return int(p)


def make_config(cfg):
    """alfa_config from a reference-style config dict.  The Wong-Lilly models
    (optSgs 2, 4) start from Cwl / CwlPrRatio, as DerivedVars.py:101-103 does."""
    c = _lib.AlfaConfig()
    for k in CONFIG_KEYS:
        if k == "precision":
            c.precision = precision_of(cfg)
            continue
        # options newer than the original Config.py default to off / zero
        # (ConfigLoader.py:77-124)
        v = cfg.get(k, 0) if k in OPTIONAL_KEYS else cfg[k]
        setattr(c, k, int(v) if isinstance(getattr(c, k), int) else float(v))
    if int(cfg["optSgs"]) in (2, 4):
        c.Cs2 = float(cfg.get("Cwl", cfg["Cs2"]))
        c.Cs2PrRatio = float(cfg.get("CwlPrRatio", cfg["Cs2PrRatio"]))
    return c


class Alfa:
    def __init__(self, cfg, device=None):
        if not torch.cuda.is_available():
            raise _lib.AlfaError("libalfa needs a CUDA device (no CPU path)")
        self.lib = _lib.load()
        self.cfg = dict(cfg)
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        ctx = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            rc = self.lib.alfa_create(ctypes.byref(make_config(cfg)), ctypes.byref(ctx))
        if rc != 0:
            msg = self.lib.alfa_last_error(None)
            raise _lib.AlfaError(f"alfa_create failed ({rc}): {msg.decode() if msg else ''}")
        self.ctx = ctx
        d = _lib.AlfaDerived()
        self.lib.alfa_get_derived(ctx, ctypes.byref(d))
        self.derived = d
        self.nx, self.ny, self.nz = cfg["nx"], cfg["ny"], cfg["nz"]
        self.mx, self.my = d.mx, d.my
        self.nx_rfft, self.ny_rfft = d.nx_rfft, d.ny_rfft

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.alfa_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    TUNE_SHAPES = ("y pad", "x pad", "x unpad", "y unpad", "x derivative", "y derivative",
                   "x filter+derivative", "y filter+derivative")
    TUNE_VARIANTS = ("default", "compile-time", "radix-8", "radix-4", "ascending",
                     "tensor-core", "two-lane")

    def autotune(self, reps=5):
        """Time every line-pass variant of the step's pass shapes and keep the
        fastest one whose outputs equal the default's (alfa_autotune); for a
        mixed-precision context the split-BF16 tensor-core pass is a candidate
        too, at a tolerance of 5e-5 of the output's largest value.
        Returns a list of dicts, one per candidate."""
        cap = 64
        buf = (_lib.AlfaTuneEntry * cap)()
        n = ctypes.c_int(0)
        self._call("alfa_autotune", int(reps), buf, cap, ctypes.byref(n))
        torch.cuda.synchronize(self.device)
        out, shape, last = [], -1, None
        for e in buf[:min(n.value, cap)]:
            key = (e.axis, e.n_in, e.n_out, e.outputs, e.map)
            if key != last:
                shape, last = shape + 1, key
            out.append({"shape": self.TUNE_SHAPES[shape], "axis": e.axis, "n_in": e.n_in,
                        "n_out": e.n_out, "outputs": e.outputs, "map": e.map,
                        "variant": self.TUNE_VARIANTS[e.variant], "ms": e.ms,
                        "equal": bool(e.equal), "chosen": bool(e.chosen)})
        return out

    def tune_shapes(self):
        """The eight line-pass shapes of a step, in autotune's order, as the
        dicts set_line_variant takes."""
        nx, ny = int(self.cfg["nx"]), int(self.cfg["ny"])
        mx, my = 3 * nx // 2, 3 * ny // 2
        rows = [(1, ny, my, 4, 1), (0, nx, mx, 4, 1), (0, mx, nx, 5, 1), (1, my, ny, 5, 1),
                (0, nx, nx, 2, 1), (1, ny, ny, 2, 1), (0, nx, nx, 1, 2), (1, ny, ny, 1, 2)]
        return [{"shape": name, "axis": a, "n_in": i, "n_out": o, "map": m, "outputs": n}
                for name, (a, i, o, m, n) in zip(self.TUNE_SHAPES, rows)]

    def set_line_variant(self, shape, variant):
        """Make `variant` (a TUNE_VARIANTS name) the one the step uses for a
        pass shape of autotune's list (a dict with axis, n_in, n_out, map
        and outputs), without timing (alfa_set_line_variant)."""
        self._call("alfa_set_line_variant", int(shape["axis"]), int(shape["n_in"]),
                   int(shape["n_out"]), int(shape["map"]), int(shape["outputs"]),
                   self.TUNE_VARIANTS.index(variant))

    TC_MAPS = {"identity": 0, "truncate": 1, "derivative": 2, "truncate+derivative": 3,
               "pad": 4, "unpad": 5}

    def tc_line_apply(self, X, map="derivative", n_out=None, scale=None, cut=0):
        """scale * M X on the tensor cores in split BF16 (alfa_tc_line_apply):
        X an (n_in, ncols) float32 CUDA tensor of lines stored as rows; M the
        line map's operator; scale defaults to 1 / n_out, the FP64 passes'
        normalisation of the unnormalised inverse transform."""
        m = self.TC_MAPS[map]
        n_in = X.shape[0]
        ncols = X[0].numel()
        if n_out is None:
            n_out = {4: 3 * n_in // 2, 5: 2 * n_in // 3}.get(m, n_in)
        if scale is None:
            scale = 1.0 / n_out
        Y = torch.empty((n_out,) + tuple(X.shape[1:]), dtype=torch.float32, device=self.device)
        self._call("alfa_tc_line_apply", m, int(cut), int(n_in), int(n_out), float(scale),
                   int(ncols), self._p(X, tuple(X.shape), torch.float32),
                   self._p(Y, tuple(Y.shape), torch.float32))
        return Y

    # ---------------------------------------------------------------- plumbing
    def _call(self, name, *args):
        self.lib.alfa_set_stream(self.ctx, ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream))
        rc = getattr(self.lib, name)(self.ctx, *args)
        if rc != 0:
            raise _lib.AlfaError(f"{name} failed ({rc}): {self.lib.alfa_last_error(self.ctx).decode()}")

    def _p(self, t, shape=None, dtype=F64):
        if not isinstance(t, torch.Tensor):
            raise TypeError("expected a torch tensor")
        if t.device != self.device or t.dtype != dtype or not t.is_contiguous():
            raise ValueError(f"expected contiguous {dtype} on {self.device}, got {t.dtype} "
                             f"on {t.device} (contiguous={t.is_contiguous()})")
        if shape is not None and tuple(t.shape) != tuple(shape):
            raise ValueError(f"expected shape {tuple(shape)}, got {tuple(t.shape)}")
        return ctypes.c_void_p(t.data_ptr())

    def _pp(self, tensors, shapes=None):
        arr = (ctypes.c_void_p * len(tensors))()
        for i, t in enumerate(tensors):
            arr[i] = None if t is None else self._p(t, None if shapes is None else shapes[i]).value
        return arr

    def _new(self, shape, dtype=F64):
        return torch.empty(shape, dtype=dtype, device=self.device)

    @property
    def N(self):
        return (self.nx, self.ny, self.nz)

    @property
    def S(self):
        return (self.nx, self.ny_rfft, self.nz)

    @property
    def P(self):
        return (self.mx, self.my, self.nz)

    @property
    def H(self):
        return (self.nx, self.ny)

    @property
    def Q(self):
        """Shape of the reference's ``*_pad`` SGS slots: padded with FGR = 1,
        the unpadded field itself otherwise (``DynamicSGS_Main.py`` passes
        ``S_uvp_pad = S_uvp`` on the no-dealias branch)."""
        return self.P if int(self.cfg.get("FGR", 1)) == 1 else self.N

    def _f(self, t):
        return self._p(t, self.N)

    def _prof(self, a):
        """(nz) profile of a horizontally uniform argument (the reference
        passes broadcast (nx, ny, nz) arrays) or of an (nz) tensor.  The
        result may be a new tensor: hold it in a variable while its pointer
        is in use (a freed temporary's memory is reused by the next one)."""
        if isinstance(a, torch.Tensor) and a.dim() == 3:
            a = a[0, 0, :]
        return torch.as_tensor(a, dtype=F64, device=self.device).contiguous().reshape(self.nz)

    # ------------------------------------------------------------- operations
    def Wavenumber(self):
        """Preprocess.py:73-102 (for signature compatibility)."""
        kx = torch.fft.fftfreq(self.nx, 1 / self.nx, dtype=F64)
        ky = torch.fft.rfftfreq(self.ny, 1 / self.ny, dtype=F64)
        kx[self.nx // 2] = 0
        ky[self.ny // 2] = 0
        kx2 = kx[:, None, None].expand(self.nx, self.ny_rfft, self.nz).to(self.device)
        ky2 = ky[None, :, None].expand(self.nx, self.ny_rfft, self.nz).to(self.device)
        self._kx2, self._ky2 = kx2, ky2
        return kx2, ky2

    def FFT(self, F):
        out = self._new(self.S, C128)
        self._call("alfa_FFT", self._f(F), self._p(out, dtype=C128))
        return out

    def FFT_pad(self, F_pad):
        out = self._new((self.mx, self.my // 2 + 1, self.nz), C128)
        self._call("alfa_FFT_pad", self._p(F_pad, self.P), self._p(out, dtype=C128))
        return out

    def Dealias1(self, F_fft, ZeRo3D_pad_fft=None):
        out = self._new(self.P)
        self._call("alfa_Dealias1", self._p(F_fft, self.S, C128), self._p(out))
        return out

    def Dealias2(self, F_pad_fft, ZeRo3D_fft=None):
        out = self._new(self.N)
        self._call("alfa_Dealias2", self._p(F_pad_fft, (self.mx, self.my // 2 + 1, self.nz), C128),
                   self._p(out))
        return out

    def Filtering_Explicit(self, F_fft):
        F = self._new(self.N)
        Fn = self._new(self.S, C128)
        self._call("alfa_Filtering_Explicit", self._p(F_fft, self.S, C128), self._p(F),
                   self._p(Fn, dtype=C128))
        return F, Fn

    def Filtering_Level1(self, F_fft):
        F = self._new(self.N)
        self._call("alfa_Filtering_Level1", self._p(F_fft, self.S, C128), self._p(F))
        return F

    def Filtering_Level2(self, F_fft):
        F = self._new(self.N)
        self._call("alfa_Filtering_Level2", self._p(F_fft, self.S, C128), self._p(F))
        return F

    def _axis(self, kxy2):
        if isinstance(kxy2, (int, np.integer)):
            return int(kxy2)
        if isinstance(kxy2, str):
            return {"x": 0, "y": 1}[kxy2]
        if kxy2 is getattr(self, "_kx2", None):
            return 0
        if kxy2 is getattr(self, "_ky2", None):
            return 1
        k = torch.as_tensor(kxy2)
        # kx2 varies along axis 0, ky2 along axis 1
        return 0 if k.shape[0] > 1 and bool((k[1:2, 0, 0] != k[0:1, 0, 0]).any()) else 1

    def Derivxy(self, F_fft, kxy2):
        out = self._new(self.N)
        self._call("alfa_Derivxy", self._p(F_fft, self.S, C128), self._axis(kxy2), self._p(out))
        return out

    def velocityGradients(self, u, v, w, u_fft, v_fft, w_fft, kx2, ky2, ustar, M_sfc_loc,
                          MOSTfunctions, ZeRo3D=None):
        out = [self._new(self.N) for _ in range(9)]
        self._call("alfa_velocityGradients", self._f(u), self._f(v), self._f(w),
                   self._p(u_fft, self.S, C128), self._p(v_fft, self.S, C128),
                   self._p(w_fft, self.S, C128), self._p(ustar, self.H), self._p(M_sfc_loc, self.H),
                   self._p(MOSTfunctions[4], self.H), self._pp(out))
        return tuple(out)

    def potentialTemperatureGradients(self, TH, kx2, ky2, ustar, qz_sfc, MOSTfunctions,
                                      ZeRo3D=None):
        out = [self._new(self.N) for _ in range(3)]
        self._call("alfa_potentialTemperatureGradients", self._f(TH), self._p(ustar, self.H),
                   self._p(qz_sfc, self.H), self._p(MOSTfunctions[5], self.H), self._pp(out))
        return tuple(out)

    def moistureGradients(self, Q, kx2, ky2, ustar, qm_sfc, MOSTfunctions, ZeRo3D=None):
        out = [self._new(self.N) for _ in range(3)]
        self._call("alfa_moistureGradients", self._f(Q), self._p(ustar, self.H),
                   self._p(qm_sfc, self.H), self._p(MOSTfunctions[5], self.H), self._pp(out))
        return tuple(out)

    def Derivz_Generic_uvp(self, F, ZeRo3D=None):
        out = self._new(self.N)
        self._call("alfa_Derivz_Generic_uvp", self._f(F), self._p(out))
        return out

    def Derivz_Generic_w(self, F, ZeRo3D=None):
        out = self._new(self.N)
        self._call("alfa_Derivz_Generic_w", self._f(F), self._p(out))
        return out

    def PlanarMean(self, F):
        out = self._new((self.nz,))
        self._call("alfa_PlanarMean", self._f(F), self._p(out))
        return out

    def Imfilter(self, F):
        """Utilities.py:87-115 applied to every (x, y) plane of a field."""
        out = self._new(self.N)
        self._call("alfa_Imfilter", self._f(F), self._p(out))
        return out

    def ComputeBeta1(self, ff, ee, dd, cc, bb, aa):
        co = torch.stack([torch.as_tensor(x, dtype=F64, device=self.device)
                          for x in (ff, ee, dd, cc, bb, aa)]).contiguous()
        n = co.shape[1]
        out = self._new((n,))
        self._call("alfa_ComputeBeta", self._p(co), n, self._p(out))
        return out

    ComputeBeta2 = ComputeBeta1

    # ---------------------------------------------------------------- surface
    def _surface(self, name, u, v, TH, MOST, sfc_val=None):
        M, us, inv = self._new(self.H), self._new(self.H), self._new(self.H)
        q2 = self._new(self.H)
        qavg = self._new(())
        mo = [self._new(self.H) for _ in range(6)]
        mi = self._pp(list(MOST), [self.H] * 6)
        if sfc_val is None:
            self._call(name, self._f(u), self._f(v), self._f(TH), mi, self._p(M), self._p(us),
                       self._p(qavg), self._p(inv), self._pp(mo))
            return M, us, qavg, inv, tuple(mo)
        self._call(name, self._f(u), self._f(v), self._f(TH), ctypes.c_double(float(sfc_val)), mi,
                   self._p(M), self._p(us), self._p(q2), self._p(qavg), self._p(inv), self._pp(mo))
        return M, us, q2, qavg, inv, tuple(mo)

    def SurfaceFlux_HomogeneousConstantFlux(self, u, v, TH, MOSTfunctions):
        return self._surface("alfa_SurfaceFlux_HomogeneousConstantFlux", u, v, TH, MOSTfunctions)

    def SurfaceFlux_HeterogeneousConstantFlux(self, u, v, TH, MOSTfunctions):
        return self._surface("alfa_SurfaceFlux_HeterogeneousConstantFlux", u, v, TH, MOSTfunctions)

    def SurfaceFlux_HomogeneousVaryingFlux(self, u, v, TH, qz_sfc_t, MOSTfunctions):
        return self._surface("alfa_SurfaceFlux_HomogeneousVaryingFlux", u, v, TH, MOSTfunctions,
                             qz_sfc_t)

    def SurfaceFlux_HeterogeneousVaryingFlux(self, u, v, TH, qz_sfc_t, MOSTfunctions):
        return self._surface("alfa_SurfaceFlux_HeterogeneousVaryingFlux", u, v, TH, MOSTfunctions,
                             qz_sfc_t)

    def SurfaceFlux_HomogeneousPrescribedTemperature(self, u, v, TH, TH_sfc_t, MOSTfunctions):
        return self._surface("alfa_SurfaceFlux_HomogeneousPrescribedTemperature", u, v, TH,
                             MOSTfunctions, TH_sfc_t)

    def SurfaceFlux_HeterogeneousPrescribedTemperature(self, u, v, TH, TH_sfc_t, MOSTfunctions):
        return self._surface("alfa_SurfaceFlux_HeterogeneousPrescribedTemperature", u, v, TH,
                             MOSTfunctions, TH_sfc_t)

    # -------------------------------------------------------------------- pde
    def Advection(self, u, v, w, dudy, dudz, dvdx, dvdz, dwdx, dwdy, ZeRo3D=None, ZeRo3D_fft=None,
                  ZeRo3D_pad=None, ZeRo3D_pad_fft=None):
        out = [self._new(self.N) for _ in range(3)]
        self._call("alfa_Advection", *[self._f(x) for x in (u, v, w, dudy, dudz, dvdx, dvdz, dwdx,
                                                              dwdy)], *[self._p(x) for x in out])
        return tuple(out)

    def ScalarAdvection(self, u, v, w, dsdx, dsdy, dsdz, ZeRo3D=None, ZeRo3D_fft=None,
                        ZeRo3D_pad=None, ZeRo3D_pad_fft=None):
        out = self._new(self.N)
        self._call("alfa_ScalarAdvection", *[self._f(x) for x in (u, v, w, dsdx, dsdy, dsdz)],
                   self._p(out))
        return out

    def BuoyancyOpt1(self, TH, H=None, ZeRo3D=None):
        """H: the specific humidity (THv = (TH + T_0)(1 + 0.61 H)) or None."""
        out = self._new(self.N)
        self._call("alfa_BuoyancyOpt1", self._f(TH), None if H is None else self._f(H),
                   self._p(out))
        return out

    def BuoyancyOpt2(self, TH, H=None, ZeRo3D=None):
        out = self._new(self.N)
        self._call("alfa_BuoyancyOpt2", self._f(TH), None if H is None else self._f(H),
                   self._p(out))
        return out

    def SurfaceMoistureFlux_HomogeneousPrescribedQ(self, Q, ustar, Q_sfc_t, MOSTfunctions):
        return self._moisture_surface("alfa_SurfaceMoistureFlux_HomogeneousPrescribedQ", Q,
                                      ustar, Q_sfc_t, MOSTfunctions)

    def SurfaceMoistureFlux_HeterogeneousPrescribedQ(self, Q, ustar, Q_sfc_t, MOSTfunctions):
        return self._moisture_surface("alfa_SurfaceMoistureFlux_HeterogeneousPrescribedQ", Q,
                                      ustar, Q_sfc_t, MOSTfunctions)

    def _moisture_surface(self, name, Q, ustar, Q_sfc_t, MOST):
        out = self._new(self.H)
        self._call(name, self._f(Q), self._p(ustar, self.H), ctypes.c_double(float(Q_sfc_t)),
                   self._pp(list(MOST), [self.H] * 6), self._p(out))
        return out

    def RHS_Moisture(self, Q, QAdvectionSum, divqm, RayleighDampCoeff_stag=None, Qadv=None):
        out = self._new(self.N)
        Qa = torch.zeros(self.nz, dtype=F64, device=self.device) if Qadv is None else self._prof(Qadv)
        self._call("alfa_RHS_Moisture", self._f(Q), self._f(QAdvectionSum), self._f(divqm),
                   self._p(Qa), self._p(out))
        return out

    def AB2_Q(self, Q, RHS_Q, RHS_Q_previous):
        out = self._new(self.N)
        self._call("alfa_AB2_Q", self._f(Q), self._f(RHS_Q), self._f(RHS_Q_previous),
                   self._p(out))
        return out

    def InitializeStats(self, ZeRo1D=None):
        """``Statistics.py:335-380``."""
        nz = self.nz
        return stats_to_dict(np.zeros(len(STATS_PROFILE_KEYS) * nz + len(STATS_SCALAR_KEYS)),
                             nz, float(self.cfg["Ugal"]))

    def ComputeStats(self, u, v, w, TH, Q, dudz, dvdz, dTHdz, dQdz, M_sfc_loc, ustar,
                     qz_sfc_avg, qm_sfc_avg, txy, txz, tyz, qz, qHz_q, Cs2_1D_avg1,
                     Cs2_1D_avg2, Cs2PrRatio_1D, beta1_1D, beta2_1D, StatsDict, ResetFlag,
                     ZeRo3D=None):
        """``Statistics.py:47-328``.  A dry sample passes None for Q, dQdz,
        qm_sfc_avg and qHz_q (the reference passes zeros)."""
        if ResetFlag == 1:
            d = self.InitializeStats()
            d["Ugal"] = StatsDict["Ugal"]
            return d
        nz = self.nz
        acc = dict_to_stats(StatsDict, nz, self.device)
        scal = lambda x: torch.as_tensor(x, dtype=F64, device=self.device).reshape(1).contiguous()
        q = scal(qz_sfc_avg)
        moist = Q is not None
        qm = scal(0.0 if qm_sfc_avg is None else qm_sfc_avg) if moist else None
        profs = [self._prof(x) for x in (Cs2_1D_avg1, Cs2_1D_avg2, Cs2PrRatio_1D, beta1_1D,
                                         beta2_1D)]
        opt = lambda x: self._f(x) if moist else None
        self._call("alfa_ComputeStats", self._f(u), self._f(v), self._f(w), self._f(TH),
                   opt(Q), self._f(dudz), self._f(dvdz), self._f(dTHdz), opt(dQdz),
                   self._p(M_sfc_loc, self.H), self._p(ustar, self.H), self._p(q),
                   None if qm is None else self._p(qm), self._f(txy), self._f(txz),
                   self._f(tyz), self._f(qz), opt(qHz_q), *[self._p(x) for x in profs],
                   self._p(acc))
        return stats_to_dict(acc, nz, StatsDict["Ugal"])

    def _mom25(self):
        return [None if 6 <= i <= 9 else self._new(self.Q if i in (20, 22) else self.N)
                for i in range(25)]

    def DivStressDynamicSGS(self, dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz,
                            u, v, w, M_sfc_loc, MOSTfunctions, ZeRo3D=None, ZeRo3D_fft=None,
                            ZeRo3D_pad_fft=None, kx2=None, ky2=None):
        g = self._pp([dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz], [self.N] * 9)
        divt = [self._new(self.N) for _ in range(3)]
        a1, a2, b1 = self._new((self.nz,)), self._new((self.nz,)), self._new((self.nz,))
        cs2 = self._new(self.N)
        mom = self._mom25()
        self._call("alfa_DivStressDynamicSGS", g, self._f(u), self._f(v), self._f(w),
                   self._p(M_sfc_loc, self.H), self._p(MOSTfunctions[0], self.H),
                   self._p(MOSTfunctions[1], self.H), *[self._p(x) for x in divt], self._p(a1),
                   self._p(a2), self._p(b1), self._p(cs2), self._pp(mom))
        mom[6], mom[7], mom[8], mom[9] = a1, a2, b1, cs2
        return (*divt, a1, a2, b1, cs2, tuple(mom))

    def DivFluxDynamicSGS(self, dynamicSGSmomentum, TH, dTHdx, dTHdy, dTHdz, SHFX, ZeRo3D=None,
                          ZeRo3D_fft=None, ZeRo3D_pad_fft=None, kx2=None, ky2=None):
        m = list(dynamicSGSmomentum)
        shapes = [self.Q if i in (10, 12) else self.N for i in range(15)]
        qz, divq, r3 = self._new(self.N), self._new(self.N), self._new(self.N)
        r1, b2 = self._new((self.nz,)), self._new((self.nz,))
        self._call("alfa_DivFluxDynamicSGS", self._pp(m, shapes), self._f(TH), self._f(dTHdx),
                   self._f(dTHdy), self._f(dTHdz), self._p(SHFX.contiguous(), self.H), self._p(qz),
                   self._p(divq), self._p(r3), self._p(r1), self._p(b2))
        return qz, divq, r3, r1, b2

    def DivStressStaticSGS(self, dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz, Cs2_3D,
                           u, v, M_sfc_loc, MOSTfunctions, ZeRo3D=None, ZeRo3D_fft=None,
                           ZeRo3D_pad_fft=None, kx2=None, ky2=None):
        g = self._pp([dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz], [self.N] * 9)
        divt = [self._new(self.N) for _ in range(3)]
        mom = [self._new(self.Q if i in (7, 9) else self.N) for i in range(10)]
        self._call("alfa_DivStressStaticSGS", g, self._f(Cs2_3D), self._f(u), self._f(v),
                   self._p(M_sfc_loc, self.H), self._p(MOSTfunctions[0], self.H),
                   self._p(MOSTfunctions[1], self.H), *[self._p(x) for x in divt], self._pp(mom))
        return (*divt, tuple(mom))

    def DivFluxStaticSGS(self, staticSGSmomentum, Cs2PrRatio_3D, dTHdx, dTHdy, dTHdz, SHFX,
                         ZeRo3D=None, ZeRo3D_fft=None, ZeRo3D_pad_fft=None, kx2=None, ky2=None):
        m = list(staticSGSmomentum)
        qz, divq = self._new(self.N), self._new(self.N)
        self._call("alfa_DivFluxStaticSGS", self._pp(m, [self.N, self.Q, self.N, self.Q]),
                   self._f(Cs2PrRatio_3D), self._f(dTHdx), self._f(dTHdy), self._f(dTHdz),
                   self._p(SHFX.contiguous(), self.H), self._p(qz), self._p(divq))
        return qz, divq

    def RHS_Momentum(self, u, v, w, Ug, Vg, Cx, Cy, Cz, buoyancy, divtx, divty, divtz,
                     RayleighDampCoeff=None, RayleighDampCoeff_stag=None, Uadv=None, Vadv=None):
        out = [self._new(self.N) for _ in range(3)]
        z = torch.zeros(self.nz, dtype=F64, device=self.device)
        Ua = z if Uadv is None else self._prof(Uadv)
        Va = z if Vadv is None else self._prof(Vadv)
        ug, vg = self._prof(Ug), self._prof(Vg)
        self._call("alfa_RHS_Momentum", self._f(u), self._f(v), self._f(w),
                   self._p(ug), self._p(vg),
                   *[self._f(x) for x in (Cx, Cy, Cz, buoyancy, divtx, divty, divtz)],
                   self._p(Ua), self._p(Va), *[self._p(x) for x in out])
        return tuple(out)

    def RHS_Scalar(self, TH, THAdvectionSum, divq, RayleighDampCoeff_stag=None, THadv=None):
        out = self._new(self.N)
        Ta = torch.zeros(self.nz, dtype=F64, device=self.device) if THadv is None else self._prof(THadv)
        self._call("alfa_RHS_Scalar", self._f(TH), self._f(THAdvectionSum), self._f(divq),
                   self._p(Ta), self._p(out))
        return out

    def PressureRC(self, u, v, w, RHS_u, RHS_v, RHS_w, RHS_u_previous, RHS_v_previous,
                   RHS_w_previous, divtz, kr2_pressure=None, kc2_pressure=None):
        R = (self.nx, self.ny_rfft, self.nz + 1)
        RCr, RCi, fRz = self._new(R), self._new(R), self._new(self.S)
        self._call("alfa_PressureRC", *[self._f(x) for x in (u, v, w, RHS_u, RHS_v, RHS_w,
                                                              RHS_u_previous, RHS_v_previous,
                                                              RHS_w_previous, divtz)],
                   self._p(RCr), self._p(RCi), self._p(fRz))
        return RCr, RCi, fRz

    def ThomasPressureSolve(self, RC_real, RC_imag, fRz_real, b_thomas=None, m_thomas=None,
                            c_pressure=None):
        R = (self.nx, self.ny_rfft, self.nz + 1)
        out = [self._new(self.N) for _ in range(4)]
        self._call("alfa_ThomasPressureSolve", self._p(RC_real, R), self._p(RC_imag, R),
                   self._p(fRz_real, self.S), *[self._p(x) for x in out])
        return tuple(out)

    def AddPressureGradient(self, RHS_u, RHS_v, RHS_w, dpdx, dpdy, dpdz):
        """Main.py:498-500 (RHS_i - dp/dx_i), returning new tensors."""
        out = [x.clone() for x in (RHS_u, RHS_v, RHS_w)]
        self._call("alfa_AddPressureGradient", *[self._p(x) for x in out], self._f(dpdx),
                   self._f(dpdy), self._f(dpdz))
        return tuple(out)

    def CFL(self, u, v, w):
        """Main.py:534-537: (CFLx, CFLy, CFLz) on the device."""
        out = self._new((3,))
        self._call("alfa_CFL", self._f(u), self._f(v), self._f(w), self._p(out))
        return out

    def AB2_uvw(self, u, v, w, RHS_u, RHS_u_previous, RHS_v, RHS_v_previous, RHS_w,
                RHS_w_previous):
        out = [self._new(self.N) for _ in range(3)]
        self._call("alfa_AB2_uvw", *[self._f(x) for x in (u, v, w, RHS_u, RHS_u_previous, RHS_v,
                                                           RHS_v_previous, RHS_w, RHS_w_previous)],
                   *[self._p(x) for x in out])
        return tuple(out)

    def AB2_TH(self, TH, RHS_TH, RHS_TH_previous):
        out = self._new(self.N)
        self._call("alfa_AB2_TH", self._f(TH), self._f(RHS_TH), self._f(RHS_TH_previous),
                   self._p(out))
        return out


MLP_NPARAM = 4994


class Learned:
    """The learned SGS coefficient network attached to a Simulation
    (alfa_mlp_*): collect samples of the dynamic procedure, train, infer,
    and step with the network judged by the procedure."""

    def __init__(self, sim, capacity=200_000, seed=0):
        self.sim = sim
        a = sim.alfa
        self.lib = a.lib
        self._sync()
        h = ctypes.c_void_p()
        rc = self.lib.alfa_mlp_create(a.ctx, int(capacity), int(seed), ctypes.byref(h))
        if rc != 0:
            raise _lib.AlfaError(f"alfa_mlp_create failed ({rc}): "
                                 f"{self.lib.alfa_last_error(a.ctx).decode()}")
        self.h = h
        self.report = _lib.AlfaMlpReport()

    def _sync(self):
        a = self.sim.alfa
        a.lib.alfa_set_stream(a.ctx, ctypes.c_void_p(torch.cuda.current_stream(a.device).cuda_stream))

    def _chk(self, rc, what):
        if rc != 0:
            a = self.sim.alfa
            raise _lib.AlfaError(f"{what} failed ({rc}): {self.lib.alfa_last_error(a.ctx).decode()}")

    def collect(self, npoints):
        self._sync()
        self._chk(self.lib.alfa_mlp_collect(self.h, int(npoints)), "alfa_mlp_collect")

    def train(self, epochs, batch=1024, lr=1e-3):
        self._sync()
        loss = ctypes.c_double()
        self._chk(self.lib.alfa_mlp_train(self.h, int(epochs), int(batch), float(lr),
                                          ctypes.byref(loss)), "alfa_mlp_train")
        return loss.value

    def loss_grad(self, X, T, norm):
        a = self.sim.alfa
        X, T, norm = (torch.as_tensor(v, dtype=torch.float32, device=a.device).contiguous()
                      for v in (X, T, norm))
        g = torch.empty(MLP_NPARAM, dtype=torch.float32, device=a.device)
        l = torch.empty(1, dtype=torch.float32, device=a.device)
        self._sync()
        self._chk(self.lib.alfa_mlp_loss_grad(self.h, X.data_ptr(), T.data_ptr(), norm.data_ptr(),
                                              int(X.shape[0]), g.data_ptr(), l.data_ptr()),
                  "alfa_mlp_loss_grad")
        return float(l.item()), g.cpu().numpy()

    def params(self):
        a = self.sim.alfa
        P = torch.empty(MLP_NPARAM, dtype=torch.float32, device=a.device)
        nm = torch.empty(24, dtype=torch.float32, device=a.device)
        self._sync()
        self._chk(self.lib.alfa_mlp_get_params(self.h, P.data_ptr(), nm.data_ptr()),
                  "alfa_mlp_get_params")
        return P.cpu().numpy(), nm.cpu().numpy()

    def set_params(self, P, norm=None):
        a = self.sim.alfa
        P = torch.as_tensor(P, dtype=torch.float32, device=a.device).contiguous()
        nm = None if norm is None else torch.as_tensor(norm, dtype=torch.float32,
                                                       device=a.device).contiguous()
        self._sync()
        self._chk(self.lib.alfa_mlp_set_params(self.h, P.data_ptr(),
                                               None if nm is None else nm.data_ptr()),
                  "alfa_mlp_set_params")
        torch.cuda.current_stream(a.device).synchronize()

    def features(self):
        a = self.sim.alfa
        X = torch.empty((a.nx, a.ny, a.nz, 10), dtype=torch.float32, device=a.device)
        self._sync()
        self._chk(self.lib.alfa_mlp_features(self.h, X.data_ptr()), "alfa_mlp_features")
        return X

    def infer(self):
        a = self.sim.alfa
        c = a._new(a.N)
        b = a._new(a.N)
        self._sync()
        self._chk(self.lib.alfa_mlp_infer(self.h, c.data_ptr(), b.data_ptr()), "alfa_mlp_infer")
        return c, b

    def step(self, n, judge_every=20, tol=0.05, refresh_points=0, refresh_epochs=0):
        self._sync()
        self._chk(self.lib.alfa_step_learned(self.h, int(n), int(judge_every), float(tol),
                                             int(refresh_points), int(refresh_epochs),
                                             ctypes.byref(self.report)), "alfa_step_learned")
        return {k: getattr(self.report, k) for k, _ in self.report._fields_}

    def close(self):
        if getattr(self, "h", None):
            self.lib.alfa_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Ensemble:
    """Independent simulations (any grid sizes) advanced together: every step
    of all members is one CUDA graph launch (alfa_ensemble_*)."""

    def __init__(self, sims):
        self.sims = list(sims)
        self.lib = _lib.load()
        for s in self.sims:  # their setup work must be done first
            torch.cuda.current_stream(s.alfa.device).synchronize()
        arr = (ctypes.c_void_p * len(self.sims))(*[s.alfa.ctx.value for s in self.sims])
        h = ctypes.c_void_p()
        rc = self.lib.alfa_ensemble_create(arr, len(self.sims), ctypes.byref(h))
        if rc != 0:
            raise _lib.AlfaError(f"alfa_ensemble_create failed ({rc})")
        self.h = h

    def step(self, n=1):
        rc = self.lib.alfa_ensemble_step(self.h, int(n))
        if rc != 0:
            raise _lib.AlfaError(f"alfa_ensemble_step failed ({rc}): "
                                 f"{self.lib.alfa_ensemble_error(self.h).decode()}")
        return self

    def set_stream(self, stream):
        """Order later steps on a torch CUDA stream (alfa_ensemble_set_stream),
        so that events recorded on it time them; None stops.  The stream must
        not be the legacy default stream (its null handle means stop)."""
        if stream is not None and stream.cuda_stream == 0:
            raise ValueError("Ensemble.set_stream needs a created stream, not the default one")
        h = ctypes.c_void_p(stream.cuda_stream if stream is not None else None)
        if self.lib.alfa_ensemble_set_stream(self.h, h) != 0:
            raise _lib.AlfaError("alfa_ensemble_set_stream failed")
        return self

    def sync(self):
        if self.lib.alfa_ensemble_sync(self.h) != 0:
            raise _lib.AlfaError("ensemble synchronisation failed")
        return self

    def states(self):
        self.sync()
        return [s.state() for s in self.sims]

    def close(self):
        if getattr(self, "h", None):
            self.lib.alfa_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ----------------------------------------------------------------------
# Statistics (src/utilities/Statistics.py:47-380) and output writers
# (src/Main.py:588-635), on the GPU accumulator of alfa_ComputeStats
# ----------------------------------------------------------------------
STATS_PROFILE_KEYS = ("U", "V", "W", "TH", "dUdz", "dVdz", "dTHdz",
                      "u2", "v2", "w2", "TH2", "uv", "uw", "vw", "uTH", "vTH", "wTH",
                      "txy", "txz", "tyz", "qz", "Cs2_1", "Cs2_2", "Cs2PrRatio",
                      "Beta1", "Beta2", "Q", "dQdz", "Q2", "wQ", "qHz")
STATS_SCALAR_KEYS = ("M_sfc", "ustar", "qz_sfc", "qm_sfc")


def stats_to_dict(acc, nz, Ugal):
    """Accumulator (ALFA_STATS_LEN(nz) doubles) -> the reference's StatsDict."""
    a = acc.detach().cpu().numpy() if isinstance(acc, torch.Tensor) else np.asarray(acc)
    d = {k: a[i * nz:(i + 1) * nz].copy() for i, k in enumerate(STATS_PROFILE_KEYS)}
    base = len(STATS_PROFILE_KEYS) * nz
    d.update({k: float(a[base + j]) for j, k in enumerate(STATS_SCALAR_KEYS)})
    d["Ugal"] = Ugal
    d["ZeRo1D"] = np.zeros(nz)
    return d


def dict_to_stats(d, nz, device):
    """The reference's StatsDict -> accumulator tensor on ``device``."""
    acc = np.zeros(len(STATS_PROFILE_KEYS) * nz + len(STATS_SCALAR_KEYS))
    for i, k in enumerate(STATS_PROFILE_KEYS):
        acc[i * nz:(i + 1) * nz] = np.asarray(d[k], dtype=np.float64)
    base = len(STATS_PROFILE_KEYS) * nz
    for j, k in enumerate(STATS_SCALAR_KEYS):
        acc[base + j] = float(d[k])
    return torch.as_tensor(acc, dtype=F64, device=device)


def write_statistics(out_dir, iteration, StatsDict, SampleCounter):
    """``Main.py:588-603``: the averages over SampleCounter samples saved as
    ALFA_Statistics_Iteration_<iteration>.npz (Ugal and ZeRo1D as they are)."""
    out = {}
    for k, v in StatsDict.items():
        out[k] = v if k in ("Ugal", "ZeRo1D") else np.asarray(v) / SampleCounter
    path = os.path.join(out_dir, f"ALFA_Statistics_Iteration_{iteration}.npz")
    np.savez(path, **out)
    return path


def write_3d_fields(out_dir, iteration, u, v, w, TH, Ugal, T_0_nondim):
    """``Main.py:620-635``: u with Ugal added back, TH absolute, saved as
    ALFA_3DFields_Iteration_<iteration>.npz."""
    h = lambda t: t.detach().cpu().numpy() if isinstance(t, torch.Tensor) else np.asarray(t)
    path = os.path.join(out_dir, f"ALFA_3DFields_Iteration_{iteration}.npz")
    np.savez(path, u=h(u) + Ugal, v=h(v), w=h(w), TH=h(TH) + T_0_nondim)
    return path


def load_geowind(path, cfg):
    """The geostrophic wind series of a GeoWind ``.npz`` file, (Ug, Vg) of
    shape (nsteps+1, nz) in m/s, with the checks and the per-level linear
    interpolation of compact profiles of ``Initialize_GeoWind_Varying``
    (``Initialization.py:163-246``).  Raises ValueError as the reference
    does on a mismatched dt, option, length or nz."""
    d = np.load(path)
    dt, nz = float(cfg["dt"]), int(cfg["nz"])
    nsteps = int(np.ceil(cfg["SimTime"] / dt))  # DerivedVars.py:90
    if abs(float(d["dt_geo"]) - dt) > 1e-6:
        raise ValueError(f"GeoWind file dt_geo={float(d['dt_geo']):.6f} s does not match "
                         f"Config dt={dt:.6f} s")
    if int(d["optGeoWind"]) != int(cfg["optGeoWind"]):
        raise ValueError("GeoWind file optGeoWind does not match Config optGeoWind")
    if "Ug_series" in d and "Vg_series" in d:
        Ug, Vg = np.asarray(d["Ug_series"]), np.asarray(d["Vg_series"])
        if Ug.shape[0] != nsteps + 1:
            raise ValueError(f"GeoWind series length {Ug.shape[0]} != nsteps+1={nsteps + 1}")
        if Ug.shape[1] != nz:
            raise ValueError(f"GeoWind nz={Ug.shape[1]} != Config nz={nz}")
        return Ug, Vg
    t, Up, Vp = np.asarray(d["t_profile"]), np.asarray(d["Ug_profile"]), np.asarray(d["Vg_profile"])
    if Up.shape[1] != nz:
        raise ValueError(f"GeoWind nz={Up.shape[1]} != Config nz={nz}")
    tt = np.arange(nsteps + 1) * dt
    if tt[0] < t[0] - 1e-6 or tt[-1] > t[-1] + 1e-6:
        raise ValueError("GeoWind compact profiles do not cover the configured simulation interval")
    Ug = np.stack([np.interp(tt, t, Up[:, k]) for k in range(nz)], axis=1)
    Vg = np.stack([np.interp(tt, t, Vp[:, k]) for k in range(nz)], axis=1)
    return Ug, Vg


class Simulation:
    """The reference's time loop (``src/Main.py:156-541``) run by libalfa
    with the state on the device.  Fields in: dimensional (u total incl.
    Ugal, theta absolute) as the reference's input files hold them."""

    def __init__(self, cfg, u, v, w, th, surface_series=None, adv_series=None, device=None,
                 geowind_series=None, Q=None, moisture_series=None):
        """optMoisture = 1 takes Q (kg/kg, as Initialize_Q loads it),
        moisture_series (the MoistureSurfaceBC data series when
        optMoistureSurfBC >= 1) and, with optAdvection, an optional fourth
        adv_series entry Qadv (kg/kg s^-1)."""
        self.alfa = Alfa(cfg, device)
        a = self.alfa
        z = a.derived.z_scale
        dev = a.device
        tt = lambda x: torch.as_tensor(np.ascontiguousarray(x), dtype=F64).to(dev)
        self._call = a._call
        # keep the device copies alive until the (asynchronous) call is enqueued
        fields = (tt(u) - cfg["Ugal"], tt(v), tt(w), tt(th) - cfg["T_0"])
        self._call("alfa_init_state", *[a._f(x) for x in fields])
        torch.cuda.current_stream(dev).synchronize()
        del fields
        nrows = 0
        ptr = lambda x: None if x is None else np.ascontiguousarray(x, dtype=np.float64).ctypes.data_as(_lib.c_double_p)
        keep = []
        U = V = T = S = None
        if adv_series is not None:
            U, V, T = [np.ascontiguousarray(x * z, dtype=np.float64) for x in adv_series[:3]]
            nrows = U.shape[0]
            keep += [U, V, T]
        if surface_series is not None:
            s = np.asarray(surface_series, dtype=np.float64)
            S = np.ascontiguousarray(s if cfg["optSurfBC"] == 1 else s - cfg["T_0"])
            nrows = max(nrows, S.shape[0]) if adv_series is None else nrows
            keep.append(S)
        if U is not None and S is not None and S.shape[0] != U.shape[0]:
            raise ValueError("series lengths differ")
        self._call("alfa_set_series", ptr(U), ptr(V), ptr(T), ptr(S), nrows)
        if int(cfg.get("optGeoWind", 0)) >= 1:
            if geowind_series is None:
                raise ValueError("optGeoWind >= 1 needs geowind_series (Ug, Vg)")
            # non-dimensional = m/s / u_scale, u_scale = 1 (Initialization.py:241-244)
            Ug, Vg = [np.ascontiguousarray(x, dtype=np.float64) for x in geowind_series]
            if Ug.shape != Vg.shape or Ug.ndim != 2 or Ug.shape[1] != a.nz:
                raise ValueError("geowind_series: Ug, Vg must both be (nrows, nz)")
            self._call("alfa_set_geowind_series", ptr(Ug), ptr(Vg), Ug.shape[0])
        self.moist = int(cfg.get("optMoisture", 0)) >= 1
        if self.moist:
            if Q is None:
                raise ValueError("optMoisture >= 1 needs the initial humidity Q")
            q = tt(Q)
            self._call("alfa_init_moisture", a._f(q))
            torch.cuda.current_stream(dev).synchronize()
            # Initialize_AdvForcing / Initialize_MoistureSurfaceBC (u_scale = Q_scale = 1)
            Qa = (np.ascontiguousarray(adv_series[3] * z, dtype=np.float64)
                  if adv_series is not None and len(adv_series) > 3 else None)
            Ms = None
            if int(cfg.get("optMoistureSurfBC", 0)) >= 1:
                if moisture_series is None:
                    raise ValueError("optMoistureSurfBC >= 1 needs moisture_series")
                Ms = np.ascontiguousarray(moisture_series, dtype=np.float64)
            rows = [x.shape[0] for x in (Qa, Ms) if x is not None]
            if len(set(rows)) > 1:
                raise ValueError("moisture series lengths differ")
            self._call("alfa_set_moisture_series", ptr(Qa), ptr(Ms), rows[0] if rows else 0)

    def step(self, n=1, graph=False):
        """n steps; graph=True replays captured CUDA graphs (alfa_step_graph),
        on a stream of this simulation's own."""
        if not graph:
            self._call("alfa_step", int(n))
            return self
        if getattr(self, "_gstream", None) is None:
            self._gstream = torch.cuda.Stream(self.alfa.device)
        cur = torch.cuda.current_stream(self.alfa.device)
        self._gstream.wait_stream(cur)
        with torch.cuda.stream(self._gstream):
            self._call("alfa_step_graph", int(n))
        cur.wait_stream(self._gstream)
        return self

    def autotune(self, reps=5):
        """Alfa.autotune on this simulation's context (between steps)."""
        return self.alfa.autotune(reps)

    def set_line_variant(self, shape, variant):
        """Alfa.set_line_variant on this simulation's context."""
        self.alfa.set_line_variant(shape, variant)
        return self

    def reset(self, u, v, w, th, Q=None):
        """Start again from new initial fields (dimensional, as the
        constructor takes them; torch CPU tensors, pinned for asynchronous
        copies, or arrays): Main.py's state at iteration istep.  Series and
        captured step graphs are kept."""
        a = self.alfa
        cfg = a.cfg
        dev = a.device

        def dev_copy(x):
            t = x if isinstance(x, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(x))
            return t.to(dev, dtype=F64, non_blocking=True)
        fields = (dev_copy(u) - cfg["Ugal"], dev_copy(v), dev_copy(w), dev_copy(th) - cfg["T_0"])
        self._call("alfa_init_state", *[a._f(x) for x in fields])
        if self.moist:
            if Q is None:
                raise ValueError("optMoisture >= 1 needs the initial humidity Q")
            q = dev_copy(Q)
            self._call("alfa_init_moisture", a._f(q))
        # the copies stay referenced until the stream has consumed them
        self._reset_keep = fields + ((q,) if self.moist else ())
        return self

    def state(self):
        a = self.alfa
        out = [a._new(a.N) for _ in range(5)]
        self._call("alfa_get_state", *[a._p(x) for x in out])
        st = dict(zip(("u", "v", "w", "TH", "p"), out))
        if self.moist:
            st["Q"] = a._new(a.N)
            self._call("alfa_get_moisture", a._p(st["Q"]))
        return st

    def stats_sample(self, acc=None):
        """Add this iteration's statistics sample (Main.py:547-558) to the
        accumulator ``acc`` (a new zeroed one if None) and return it."""
        a = self.alfa
        if acc is None:
            acc = torch.zeros(len(STATS_PROFILE_KEYS) * a.nz + len(STATS_SCALAR_KEYS),
                              dtype=F64, device=a.device)
        self._call("alfa_stats_sample", a._p(acc))
        return acc

    def checkpoint(self):
        """Everything the time loop carries between iterations, as one device
        tensor (alfa_save_checkpoint)."""
        a = self.alfa
        buf = torch.empty(int(a.lib.alfa_checkpoint_doubles(a.ctx)), dtype=F64, device=a.device)
        self._call("alfa_save_checkpoint", a._p(buf))
        return buf

    def restore(self, buf):
        """Continue from a checkpoint() of a run with the same configuration."""
        a = self.alfa
        n = int(a.lib.alfa_checkpoint_doubles(a.ctx))
        buf = torch.as_tensor(buf, dtype=F64).to(a.device).contiguous()
        if buf.numel() != n:
            raise ValueError(f"checkpoint holds {buf.numel()} values, this configuration {n}")
        self._call("alfa_load_checkpoint", a._p(buf))
        return self

    def save(self, path):
        """checkpoint() written to an .npz file (key "checkpoint", plus the grid)."""
        a = self.alfa
        np.savez(path, checkpoint=self.checkpoint().cpu().numpy(),
                 grid=np.array([a.nx, a.ny, a.nz]))
        return path

    def load(self, path):
        z = np.load(path)
        return self.restore(torch.as_tensor(z["checkpoint"]))

    def diag(self):
        d = _lib.AlfaDiag()
        a = self.alfa
        a.lib.alfa_set_stream(a.ctx, ctypes.c_void_p(torch.cuda.current_stream(a.device).cuda_stream))
        rc = a.lib.alfa_get_diag(a.ctx, ctypes.byref(d))
        if rc != 0:
            raise _lib.AlfaError(a.lib.alfa_last_error(a.ctx).decode())
        return {k: getattr(d, k) for k, _ in d._fields_}
