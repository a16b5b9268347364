"""Host side of the learned return map (an MLP in place of the Drucker-Prager projection).

Data: (trial, projected) pairs recorded by the fused kernel
(`Context.harvest_begin/harvest_end`, 8 floats per record).  Training runs on
the GPU through the library's own kernels (icempm_mlp_grad: forward, loss and
backward; icempm_mlp_adam); inference and the exact-map fallback through
icempm_return_map_learned.  torch only holds device memory and streams.

    feats(trial)          x = (log s1, log s2, log Jp, log thickness)
    targets(trial, proj)  y = (log s1'/s1, log s2'/s2, log Jp'/Jp)
    Norm                  per-feature mean / std of x and y (norm[14])
"""
import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import capi

NPARAM = 4675
IN, HID, OUT = 4, 64, 3


def feats(trial):
    return np.log(np.asarray(trial[:, :4], np.float64))


def targets(trial, proj):
    return np.log(np.asarray(proj[:, :3], np.float64)) - np.log(np.asarray(trial[:, :3], np.float64))


@dataclass
class Norm:
    x_mean: np.ndarray
    x_std: np.ndarray
    y_mean: np.ndarray
    y_std: np.ndarray

    @staticmethod
    def fit(x, y):
        def ms(a):
            m = a.mean(0)
            s = a.std(0)
            return m, np.where(s > 1e-12 * np.maximum(np.abs(m), 1.0), s, 1.0)
        xm, xs = ms(x)
        ym, ys = ms(y)
        return Norm(xm, xs, ym, ys)

    def vector(self):
        return np.concatenate([self.x_mean, self.x_std, self.y_mean, self.y_std]).astype(np.float32)


def init_params(seed=0):
    """Uniform fan-in initialisation of W1, W2, W3; zero biases."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM, np.float32)
    k = 0
    for fan_out, fan_in in ((HID, IN), (HID, HID), (OUT, HID)):
        b = 1.0 / np.sqrt(fan_in)
        p[k:k + fan_out * fan_in] = rng.uniform(-b, b, fan_out * fan_in)
        k += fan_out * fan_in + fan_out
    return p


def _ptr(t):
    return C.c_void_p(t.data_ptr())


class Trainer:
    """Adam on the library's kernels.  x, y: standardised float32 arrays."""

    def __init__(self, params=None, lr=2e-3, seed=0):
        import torch
        self.torch = torch
        self.L = capi.load()
        self.dev = torch.device("cuda")
        p = init_params(seed) if params is None else np.asarray(params, np.float32)
        self.P = torch.from_numpy(p.copy()).to(self.dev)
        self.G = torch.zeros(NPARAM, device=self.dev)
        self.M = torch.zeros(NPARAM, device=self.dev)
        self.V = torch.zeros(NPARAM, device=self.dev)
        self.loss = torch.zeros(1, device=self.dev)
        self.t = 0
        self.lr = lr

    def stream(self):
        return C.c_void_p(self.torch.cuda.current_stream().cuda_stream)

    def grad(self, x, y):
        """Loss and gradient of one batch (device tensors), without a step."""
        self.G.zero_()
        self.loss.zero_()
        capi.check(self.L.icempm_mlp_grad(_ptr(self.P), _ptr(x), _ptr(y), int(x.shape[0]), _ptr(self.G),
                                          _ptr(self.loss), self.stream()))
        return float(self.loss.item()), self.G.cpu().numpy()

    def fit(self, x, y, epochs=10, batch=65536, seed=0, lr_decay=0.7):
        """Minibatch Adam over the whole set each epoch; returns the mean loss per epoch."""
        torch = self.torch
        xd = torch.from_numpy(np.ascontiguousarray(x, np.float32)).to(self.dev)
        yd = torch.from_numpy(np.ascontiguousarray(y, np.float32)).to(self.dev)
        n = xd.shape[0]
        gen = torch.Generator(device=self.dev)
        gen.manual_seed(seed)
        history = []
        for ep in range(epochs):
            perm = torch.randperm(n, device=self.dev, generator=gen)
            tot = torch.zeros(1, device=self.dev)
            nb = 0
            for s in range(0, n, batch):
                idx = perm[s:s + batch]
                xb = xd[idx].contiguous()
                yb = yd[idx].contiguous()
                self.G.zero_()
                self.loss.zero_()
                capi.check(self.L.icempm_mlp_grad(_ptr(self.P), _ptr(xb), _ptr(yb), int(xb.shape[0]), _ptr(self.G),
                                                  _ptr(self.loss), self.stream()))
                self.t += 1
                capi.check(self.L.icempm_mlp_adam(_ptr(self.P), _ptr(self.G), _ptr(self.M), _ptr(self.V), self.t,
                                                  float(self.lr), self.stream()))
                tot += self.loss
                nb += 1
            history.append(float(tot.item()) / nb)
            self.lr *= lr_decay ** (1.0 / max(1, epochs // 4))
        return history

    def params(self):
        return self.P.cpu().numpy()


def forward(params, x):
    """FP32 forward of standardised inputs (icempm_mlp_forward)."""
    import torch
    L = capi.load()
    P = torch.from_numpy(np.asarray(params, np.float32)).cuda()
    xd = torch.from_numpy(np.ascontiguousarray(x, np.float32)).cuda()
    yd = torch.zeros((xd.shape[0], OUT), device="cuda")
    capi.check(L.icempm_mlp_forward(_ptr(P), _ptr(xd), int(xd.shape[0]), _ptr(yd),
                                    C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    return yd.cpu().numpy()


def exact_map(prms, trial, fp64=True, repeat=1):
    """The exact return map on trial states [n, 4] (device kernel); returns
    (projected [n, 4], device ms per call)."""
    import torch
    L = capi.load()
    td = torch.from_numpy(np.ascontiguousarray(trial[:, :4], np.float32)).cuda()
    od = torch.zeros_like(td)
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    capi.check(L.icempm_return_map_exact(C.byref(prms), _ptr(td), int(td.shape[0]), _ptr(od), int(fp64), st))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(repeat):
        capi.check(L.icempm_return_map_exact(C.byref(prms), _ptr(td), int(td.shape[0]), _ptr(od), int(fp64), st))
    e1.record()
    torch.cuda.synchronize()
    return od.cpu().numpy(), e0.elapsed_time(e1) / repeat


def learned_map(prms, params, norm, trial, tol=1e-4, repeat=1):
    """The learned map with exact fallback on trial states [n, 4]; returns
    (projected [n, 4] with column 3 = 0 exact / 1 network / 2 fallback,
    fallback count of one call, device ms per call)."""
    import torch
    L = capi.load()
    td = torch.from_numpy(np.ascontiguousarray(trial[:, :4], np.float32)).cuda()
    od = torch.zeros_like(td)
    P = torch.from_numpy(np.asarray(params, np.float32)).cuda()
    nv = torch.from_numpy(norm.vector()).cuda()
    fb = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    args = lambda: (C.byref(prms), _ptr(P), _ptr(nv), _ptr(td), int(td.shape[0]), float(tol), _ptr(od), _ptr(fb), st)
    capi.check(L.icempm_return_map_learned(*args()))
    torch.cuda.synchronize()
    nfb = int(fb.item())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(repeat):
        capi.check(L.icempm_return_map_learned(*args()))
    e1.record()
    torch.cuda.synchronize()
    return od.cpu().numpy(), nfb, e0.elapsed_time(e1) / repeat


def train(records, epochs=30, batch=1024, lr=3e-3, seed=0):
    """Standardisation and network fitted to harvested records [n, 8]
    (trial 0..3, projected 4..6); returns (params, Norm, loss history)."""
    x = feats(records[:, :4])
    y = targets(records[:, :4], records[:, 4:7])
    norm = Norm.fit(x, y)
    xs = ((x - norm.x_mean) / norm.x_std).astype(np.float32)
    ys = ((y - norm.y_mean) / norm.y_std).astype(np.float32)
    tr = Trainer(lr=lr, seed=seed)
    hist = tr.fit(xs, ys, epochs=epochs, batch=batch, seed=seed)
    return tr.params(), norm, hist


class StepNetwork:
    """A trained network on the device for a context's step path
    (Context.set_learned_map): holds the FP32 parameters and the
    normalisation in device memory for as long as the context uses them."""

    def __init__(self, params, norm: Norm):
        import torch
        self.P = torch.from_numpy(np.asarray(params, np.float32).copy()).cuda()
        self.N = torch.from_numpy(norm.vector()).cuda()

    def attach(self, ctx, tol):
        ctx.set_learned_map(C.c_void_p(self.P.data_ptr()), C.c_void_p(self.N.data_ptr()), tol)

    @staticmethod
    def detach(ctx):
        ctx.set_learned_map(None, None, 1.0)
