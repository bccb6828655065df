"""Test infrastructure only (never imported by the product path): a NumPy
FP64 restatement of the learned-coefficient network of
``jax_alfa_b200/csrc/alfa_mlp.cu`` -- its input features, its forward pass,
its loss and the loss gradient by backpropagation -- used to check the GPU
training kernels (gradients) and feature kernel.  The network has no
counterpart in the reference; the features are built from the reference's
strain rates (``StrainRates.py:56-141``, staggering as StrainsUVPnodes) and
scalar gradient (the THz of ``DynamicSGS_ScalarLASDD_SM.py:182-185``)."""
import numpy as np

NIN, NH = 10, 64
SIZES = [("W1", (NH, NIN)), ("b1", (NH,)), ("W2", (NH, NH)), ("b2", (NH,)),
         ("W3", (2, NH)), ("b3", (2,))]
NPARAM = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(p):
    out, off = {}, 0
    for name, shp in SIZES:
        n = int(np.prod(shp))
        out[name] = np.asarray(p[off:off + n], dtype=np.float64).reshape(shp)
        off += n
    return out


def pack(d):
    return np.concatenate([d[name].ravel() for name, _ in SIZES])


def _bounded(ri):
    return ri / (1.0 + np.abs(ri))


def features(o, grads, dTHdz, with_scales=False):
    """(nx, ny, nz, 10) features at uvp nodes from velocityGradients' nine
    fields and dTHdz (w nodes); with_scales also returns |S| and
    uz^2 + vz^2, the denominators of the ratio features."""
    dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz = [np.asarray(g, np.float64)
                                                            for g in grads]
    nz = o.nz
    uz, vz, wx, wy = (np.zeros_like(dudx) for _ in range(4))
    uz[:, :, 0], vz[:, :, 0] = dudz[:, :, 0], dvdz[:, :, 0]
    wx[:, :, 0], wy[:, :, 0] = 0.5 * dwdx[:, :, 1], 0.5 * dwdy[:, :, 1]
    uz[:, :, nz - 1], vz[:, :, nz - 1] = dudz[:, :, nz - 1], dvdz[:, :, nz - 1]
    wx[:, :, nz - 1], wy[:, :, nz - 1] = dwdx[:, :, nz - 1], dwdy[:, :, nz - 1]
    sl, sr = slice(1, nz - 1), slice(2, nz)
    uz[:, :, sl] = 0.5 * (dudz[:, :, sl] + dudz[:, :, sr])
    vz[:, :, sl] = 0.5 * (dvdz[:, :, sl] + dvdz[:, :, sr])
    wx[:, :, sl] = 0.5 * (dwdx[:, :, sl] + dwdx[:, :, sr])
    wy[:, :, sl] = 0.5 * (dwdy[:, :, sl] + dwdy[:, :, sr])
    s11, s22, s33 = dudx, dvdy, dwdz
    s12 = 0.5 * (dudy + dvdx)
    s13 = 0.5 * (uz + wx)
    s23 = 0.5 * (vz + wy)
    S = np.sqrt(2 * (s11 ** 2 + s22 ** 2 + s33 ** 2 + 2 * s12 ** 2 + 2 * s13 ** 2 + 2 * s23 ** 2))
    iS = 1.0 / (S + 1e-30)
    T = np.asarray(dTHdz, np.float64)
    thz = T.copy()
    thz[:, :, sl] = 0.5 * (T[:, :, sl] + T[:, :, sr])
    z = (np.arange(nz) + 0.5) * o.dz / o.L
    f = [np.log(o.L * o.L * S + 1e-12), s11 * iS, s22 * iS, s33 * iS, s12 * iS, s13 * iS,
         s23 * iS, thz, np.broadcast_to(z, S.shape),
         _bounded((o.g_nondim / o.T_0_nondim) * thz / (uz * uz + vz * vz + 1e-12))]
    F = np.stack(f, axis=-1)
    return (F, S, uz * uz + vz * vz) if with_scales else F


def loss_and_grad(p, X, T, norm):
    """Mean over samples and both outputs of the squared error in normalised
    units, and its gradient (packed like the parameters)."""
    P = unpack(p)
    norm = np.asarray(norm, np.float64)
    x = (np.asarray(X, np.float64) - norm[:NIN]) / norm[NIN + 2:2 * NIN + 2]
    t = (np.asarray(T, np.float64) - norm[NIN:NIN + 2]) / norm[2 * NIN + 2:]
    n = x.shape[0]
    a1 = x @ P["W1"].T + P["b1"]
    h1 = np.tanh(a1)
    a2 = h1 @ P["W2"].T + P["b2"]
    h2 = np.tanh(a2)
    y = h2 @ P["W3"].T + P["b3"]
    d = y - t
    loss = np.sum(d * d) / (2 * n)
    dy = 2 * d / (2 * n)
    g = {"W3": dy.T @ h2, "b3": dy.sum(0)}
    dh2 = (dy @ P["W3"]) * (1 - h2 ** 2)
    g["W2"] = dh2.T @ h1
    g["b2"] = dh2.sum(0)
    dh1 = (dh2 @ P["W2"]) * (1 - h1 ** 2)
    g["W1"] = dh1.T @ x
    g["b1"] = dh1.sum(0)
    return loss, pack(g)
