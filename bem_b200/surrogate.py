"""Learned surrogate of the BEM perturbation field: an MLP (rho, z) -> (E_rho, E_z).

Network: 2 inputs -> 4 hidden layers of 128 (SiLU) -> 2 outputs; BF16 weights
and activations, FP32 accumulation and FP32 master weights.  The three
128 x 128 layers run on the tensor cores through spt_mlp_gemm (tcgen05, TMEM
accumulators); the first and last layers, the loss, the bias sums and Adam
are the library's own CUDA-core kernels.  Nothing here calls a library GEMM
or autograd: torch only holds the buffers.

Inputs are surface-normal coordinates -- the log distance to the profile
and the arclength position of the closest profile point (the stage kernel
finds that point anyway for the reference's on-surface rule) -- and the
outputs are the normal and tangential field components scaled by the local
|sigma| and a per-log-distance RMS table, so every output is O(1) from the
surface to z_handoff.

Training data: points at log-uniform distances (1 nm ... 1 mm, capped at the
blend region) along the outward normal of uniformly chosen points of the
profile's z >= 0 part, labelled by the float64 BEM evaluator (spt_bem_field).
"""

import ctypes
import math

import numpy as np

from . import _lib

WIDTH = 128
PARAM_SHAPES = [("W1", (WIDTH, 2)), ("b1", (WIDTH,)), ("W2", (WIDTH, WIDTH)), ("b2", (WIDTH,)),
                ("W3", (WIDTH, WIDTH)), ("b3", (WIDTH,)), ("W4", (WIDTH, WIDTH)), ("b4", (WIDTH,)),
                ("W5", (2, WIDTH)), ("b5", (2,))]
N_SCALE_BINS = 64


def _torch():
    import torch
    return torch


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _check(rc, what):
    if rc != 0:
        raise _lib.SptError(f"{what} failed ({rc})")


class FieldSurrogate:
    """Parameters (flat FP32 master buffer + BF16 copy + BF16-rounded FP32
    copy) and the surface-normal frame of the surrogate.

    Inputs: u1 = log distance d to the profile (normalised over
    [D_MIN, D_MAX]) and u2 = arclength position s of the closest profile
    point (normalised over the z >= 0 part).  Outputs: the field's components
    along the closest segment's outward normal and unit tangent, divided by
    (|sigma(s)| + 1e-3 max|sigma|) * g(d), g a per-log-distance RMS table."""

    D_MIN, D_MAX = 1e-10, 1e-3

    def __init__(self, profile, sigma, s_end, scale_table, device="cuda", seed=0):
        torch = _torch()
        self.device = torch.device(device)
        self.profile = np.asarray(profile, dtype=np.float64)
        self.sigma = np.asarray(sigma, dtype=np.float64)
        tan = self.profile[1:] - self.profile[:-1]
        self.seg_len = np.linalg.norm(tan, axis=-1)
        self.s_start = np.concatenate([[0.0], np.cumsum(self.seg_len)])[:-1]
        self.s_end = float(s_end)
        self.sig_floor = 1e-3 * np.abs(self.sigma).max()
        self.scale_table = np.asarray(scale_table, dtype=np.float64)
        self.offsets = {}
        o = 0
        for name, shape in PARAM_SHAPES:
            self.offsets[name] = (o, shape)
            o += int(np.prod(shape))
        self.n_params = o
        rng = np.random.default_rng(seed)
        flat = np.zeros(o, dtype=np.float32)
        for name, shape in PARAM_SHAPES:
            off, _ = self.offsets[name]
            if name.startswith("W"):
                fan_in = shape[1]
                flat[off:off + int(np.prod(shape))] = rng.normal(0.0, math.sqrt(2.0 / fan_in), int(np.prod(shape)))
        self.p = torch.as_tensor(flat, device=self.device)
        self.p16 = self.p.to(torch.bfloat16)
        self.pr = self.p16.float()

    def view(self, buf, name):
        off, shape = self.offsets[name]
        return buf[off:off + int(np.prod(shape))].view(*shape)

    # ---- frame, features and scale --------------------------------------------
    def frame(self, seg):
        tan = self.profile[seg + 1] - self.profile[seg]
        unit = tan / self.seg_len[seg][:, None]
        nrm = np.stack([-unit[:, 1], unit[:, 0]], -1)
        return nrm, unit

    def features(self, seg, t, d):
        s = (self.s_start[seg] + t * self.seg_len[seg]) / self.s_end
        ld = np.log(np.clip(d, self.D_MIN, self.D_MAX))
        u1 = 2.0 * (ld - math.log(self.D_MIN)) / (math.log(self.D_MAX) - math.log(self.D_MIN)) - 1.0
        u2 = 2.0 * s - 1.0
        return np.stack([u1, u2], -1).astype(np.float32)

    def log_scale_table(self):
        return np.log(self.scale_table)

    def scale(self, seg, t, d):
        sig = np.abs(self.sigma[seg] + t * (self.sigma[seg + 1] - self.sigma[seg])) + self.sig_floor
        ld = np.log(np.clip(d, self.D_MIN, self.D_MAX))
        pos = (ld - math.log(self.D_MIN)) / (math.log(self.D_MAX) - math.log(self.D_MIN)) * (N_SCALE_BINS - 1)
        g = np.exp(np.interp(pos, np.arange(N_SCALE_BINS), np.log(self.scale_table)))
        return sig * g

    def closest(self, rho, z):
        """Closest profile segment, parameter and distance of each point
        (bem/axisymmetric.py:341-389)."""
        prof = self.profile
        best = np.full(rho.shape, np.inf)
        seg = np.zeros(rho.shape, dtype=np.int64)
        tb = np.zeros(rho.shape)
        for j in range(len(prof) - 1):
            ab = prof[j + 1] - prof[j]
            t = np.clip(((rho - prof[j, 0]) * ab[0] + (z - prof[j, 1]) * ab[1]) / (ab @ ab), 0.0, 1.0)
            d2 = (rho - prof[j, 0] - t * ab[0]) ** 2 + (z - prof[j, 1] - t * ab[1]) ** 2
            better = d2 < best
            best = np.where(better, d2, best)
            seg = np.where(better, j, seg)
            tb = np.where(better, t, tb)
        return seg, tb, np.sqrt(best)

    # ---- inference (standalone, batched) -------------------------------------
    def predict(self, rho, z):
        """E_rho, E_z at points (numpy), through the library's kernels."""
        torch = _torch()
        rho = np.asarray(rho, dtype=np.float64)
        z = np.asarray(z, dtype=np.float64)
        seg, t, d = self.closest(rho, z)
        x = self.features(seg, t, d)
        n = len(x)
        npad = ((n + 127) // 128) * 128
        xb = torch.zeros((npad, 2), dtype=torch.float32, device=self.device)
        xb[:n] = torch.as_tensor(x, device=self.device)
        y = forward(self, xb)[:n].cpu().numpy().astype(np.float64)
        sc = self.scale(seg, t, d)
        nrm, unit = self.frame(seg)
        en, et = y[:, 0] * sc, y[:, 1] * sc
        return en * nrm[:, 0] + et * unit[:, 0], en * nrm[:, 1] + et * unit[:, 1]

    def state(self):
        return dict(params=self.p.cpu().numpy(), profile=self.profile, sigma=self.sigma, s_end=self.s_end,
                    scale_table=self.scale_table)

    @classmethod
    def from_state(cls, st, device="cuda"):
        torch = _torch()
        m = cls(st["profile"], st["sigma"], float(st["s_end"]), st["scale_table"], device=device)
        m.p = torch.as_tensor(np.asarray(st["params"], dtype=np.float32), device=m.device)
        m.p16 = m.p.to(torch.bfloat16)
        m.pr = m.p16.float()
        return m

    def params_dict(self):
        return {name: self.view(self.p, name).cpu().numpy() for name, _ in PARAM_SHAPES}


class _Work:
    """Activation and gradient buffers for a batch of n samples."""

    def __init__(self, n, device, n_params):
        torch = _torch()
        f32, b16 = torch.float32, torch.bfloat16
        self.n = n
        self.z = [torch.empty((n, WIDTH), dtype=f32, device=device) for _ in range(4)]
        self.h = [torch.empty((n, WIDTH), dtype=b16, device=device) for _ in range(4)]
        self.d = [torch.empty((n, WIDTH), dtype=b16, device=device) for _ in range(4)]
        self.y = torch.empty((n, 2), dtype=f32, device=device)
        self.g = torch.zeros(n_params, dtype=f32, device=device)
        self.loss = torch.zeros(1, dtype=f32, device=device)
        self.split = max(1, min(64, n // 128))
        while n % (self.split * 64):
            self.split -= 1
        self.part = torch.empty((self.split, WIDTH, WIDTH), dtype=f32, device=device)


def _gemm(A, a_mn, lda, B, b_mn, ldb, M, N, K, epi, C=None, ldc=WIDTH, bias=None, Z=None, H=None, split=1,
          split_stride=0, stream=None):
    g = _lib.SptGemmArgs()
    g.M, g.N, g.K = M, N, K
    g.a_mn, g.b_mn, g.epi, g.split_k = a_mn, b_mn, epi, split
    g.lda, g.ldb, g.ldc, g.split_stride = lda, ldb, ldc, split_stride
    g.A, g.B = A.data_ptr(), B.data_ptr()
    g.C = None if C is None else C.data_ptr()
    g.bias = None if bias is None else bias.data_ptr()
    g.Z = None if Z is None else Z.data_ptr()
    g.H = None if H is None else H.data_ptr()
    _check(_lib.lib().spt_mlp_gemm(ctypes.byref(g), stream), "spt_mlp_gemm")


def _stream():
    torch = _torch()
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def forward(model, x, work=None, target=None, inv_batch=None):
    """Forward pass of a batch x [n, 2] (n a multiple of 128) -> y [n, 2].
    With a target: also the loss and the last-layer gradients into work.g."""
    n = x.shape[0]
    if work is None:
        work = _Work(n, model.device, model.n_params)
    st = _stream()
    L = _lib.lib()
    v = lambda buf, name: model.view(buf, name)
    _check(L.spt_mlp_first_layer(_ptr(x), n, _ptr(v(model.pr, "W1")), _ptr(v(model.p, "b1")), _ptr(work.z[0]),
                                 _ptr(work.h[0]), st), "first_layer")
    for l in (2, 3, 4):
        _gemm(work.h[l - 2], 0, WIDTH, v(model.p16, f"W{l}"), 0, WIDTH, n, WIDTH, WIDTH, _lib.EPI_BIAS_SILU,
              C=work.z[l - 1], bias=v(model.p, f"b{l}"), H=work.h[l - 1], stream=st)
    g = work.g
    _check(L.spt_mlp_last_layer(_ptr(work.h[3]), _ptr(work.z[3]), n, _ptr(v(model.pr, "W5")), _ptr(v(model.p, "b5")),
                                _ptr(work.y), _ptr(target), float(inv_batch or 0.0), _ptr(work.d[3]),
                                _ptr(v(g, "W5")) if target is not None else None,
                                _ptr(v(g, "b5")) if target is not None else None,
                                _ptr(work.loss) if target is not None else None, st), "last_layer")
    return work.y


def backward(model, x, work):
    """Gradients of the loss into work.g (after forward(..., target=...))."""
    st = _stream()
    L = _lib.lib()
    n = work.n
    g = work.g
    v = lambda buf, name: model.view(buf, name)
    for l in (4, 3, 2):
        d = work.d[l - 1]
        _check(L.spt_mlp_colsum(_ptr(d), n, None, _ptr(v(g, f"b{l}")), None, st), "colsum")
        # dW_l[out][in] = sum_s d[s][out] h_{l-1}[s][in]: both operands MN-major, split over samples
        _gemm(d, 1, WIDTH, work.h[l - 2], 1, WIDTH, WIDTH, WIDTH, n, _lib.EPI_STORE, C=work.part, split=work.split,
              split_stride=WIDTH * WIDTH, stream=st)
        _check(L.spt_mlp_reduce_splits(_ptr(work.part), work.split, WIDTH * WIDTH, _ptr(v(g, f"W{l}")), st),
               "reduce")
        # d_{l-1} = (d_l W_l) * SiLU'(z_{l-1}): W_l read as (n = in, k = out), MN-major
        _gemm(d, 0, WIDTH, v(model.p16, f"W{l}"), 1, WIDTH, n, WIDTH, WIDTH, _lib.EPI_DSILU, Z=work.z[l - 2],
              H=work.d[l - 2], stream=st)
    _check(L.spt_mlp_colsum(_ptr(work.d[0]), n, _ptr(x), _ptr(v(g, "b1")), _ptr(v(g, "W1")), st), "colsum1")


def adam_step(model, work, m, vv, lr, step, beta1=0.9, beta2=0.999, eps=1e-8):
    _check(_lib.lib().spt_mlp_adam(_ptr(model.p), _ptr(work.g), _ptr(m), _ptr(vv), model.n_params, float(lr),
                                   beta1, beta2, eps, int(step), _ptr(model.p16), _ptr(model.pr), _stream()),
           "adam")


def sample_points(geometry, n, rng, d_min=1e-9, d_max=1e-3, apex_weight=0.5):
    """Training points around the z >= 0 part of a BEM profile: a point on a
    segment (half of them uniform in arclength, half uniform over segment
    index, which favours the finely meshed apex), offset along the outward
    normal by a log-uniform distance; kept if z >= 0, outside the conductor,
    below z_handoff.  Returns rho, z, seg, t, d."""
    prof = geometry.profile
    up = np.nonzero((prof[:-1, 1] >= 0) & (prof[1:, 1] >= 0))[0]
    lens = np.linalg.norm(prof[up + 1] - prof[up], axis=-1)
    cdf = np.cumsum(lens) / lens.sum()
    out = [[] for _ in range(5)]
    got = 0
    while got < n:
        m = 2 * (n - got) + 1024
        by_len = rng.uniform(0, 1, m) >= apex_weight
        pick = np.where(by_len, np.searchsorted(cdf, rng.uniform(0, 1, m)), rng.integers(0, len(up), m))
        s = up[np.minimum(pick, len(up) - 1)]
        t = rng.uniform(0, 1, m)
        p = prof[s] + t[:, None] * (prof[s + 1] - prof[s])
        tan = prof[s + 1] - prof[s]
        nrm = np.stack([-tan[:, 1], tan[:, 0]], -1)
        nrm /= np.linalg.norm(nrm, axis=-1, keepdims=True)
        d = np.exp(rng.uniform(np.log(d_min), np.log(d_max), m))
        q = p + d[:, None] * nrm
        rho, z = q[:, 0], q[:, 1]
        ok = (z >= 0) & (z < geometry.z_handoff) & (rho >= 0)
        if geometry.kind == _lib.GEOM_POST_BEM:
            rk = geometry.R
            ok &= ~(((rho <= rk) & (z <= geometry.L)) | (rho * rho + (z - geometry.L) ** 2 <= rk * rk))
        for lst, arr in zip(out, (rho, z, s, t, d)):
            lst.append(arr[ok])
        got += int(ok.sum())
    return tuple(np.concatenate(lst)[:n] for lst in out)


def label(geometry, rho, z, chunk=1 << 18):
    """float64 BEM perturbation field at (rho, 0, z) via spt_bem_field."""
    from .engine import bem_field
    tables = geometry.bem_tables()
    out = []
    for a in range(0, len(rho), chunk):
        pts = np.stack([rho[a:a + chunk], np.zeros(len(rho[a:a + chunk])), z[a:a + chunk]], -1)
        e = bem_field(tables, pts).cpu().numpy()
        out.append(np.stack([e[:, 0], e[:, 2]], -1))
    return np.concatenate(out)


def train(geometry, n_points=2_000_000, steps=20_000, batch=8192, lr=1e-3, seed=4, device="cuda", log_every=0,
          data=None):
    """Train the surrogate for a BEM geometry with the library's kernels.
    data = (rho, z, seg, t, d, E) skips sampling and labelling."""
    torch = _torch()
    rng = np.random.default_rng(seed)
    if data is None:
        rho, z, seg, t, d = sample_points(geometry, n_points, rng)
        E = label(geometry, rho, z)
    else:
        rho, z, seg, t, d, E = data
    prof = geometry.profile
    up = (prof[:-1, 1] >= 0) & (prof[1:, 1] >= 0)
    s_end = float(np.linalg.norm(prof[1:] - prof[:-1], axis=-1)[up].sum())
    model = FieldSurrogate(prof, geometry.sigma, s_end, np.ones(N_SCALE_BINS), device=device, seed=seed)
    nrm, unit = model.frame(seg)
    en = E[:, 0] * nrm[:, 0] + E[:, 1] * nrm[:, 1]
    et = E[:, 0] * unit[:, 0] + E[:, 1] * unit[:, 1]
    sig = model.scale(seg, t, d)  # |sigma| part only (table is still ones)
    ld = np.log(np.clip(d, model.D_MIN, model.D_MAX))
    pos = (ld - math.log(model.D_MIN)) / (math.log(model.D_MAX) - math.log(model.D_MIN)) * (N_SCALE_BINS - 1)
    b = np.clip(np.rint(pos).astype(int), 0, N_SCALE_BINS - 1)
    mag2 = (en * en + et * et) / (sig * sig)
    table = np.ones(N_SCALE_BINS)
    filled = np.zeros(N_SCALE_BINS, dtype=bool)
    for k in range(N_SCALE_BINS):
        sel = b == k
        if sel.any():
            table[k] = math.sqrt(mag2[sel].mean())
            filled[k] = True
    idx = np.arange(N_SCALE_BINS)
    table = np.exp(np.interp(idx, idx[filled], np.log(table[filled])))
    model.scale_table = table
    x = model.features(seg, t, d)
    sc = model.scale(seg, t, d)
    y = np.stack([en / sc, et / sc], -1).astype(np.float32)
    n = (len(x) // batch) * batch
    X = torch.as_tensor(x[:n], device=model.device)
    Y = torch.as_tensor(y[:n], device=model.device)
    work = _Work(batch, model.device, model.n_params)
    m = torch.zeros(model.n_params, dtype=torch.float32, device=model.device)
    vv = torch.zeros_like(m)
    gen = torch.Generator(device=model.device)
    gen.manual_seed(seed)
    perm = torch.randperm(n, generator=gen, device=model.device)
    losses = []
    pos_b = 0
    for step in range(1, steps + 1):
        if pos_b + batch > n:
            perm = torch.randperm(n, generator=gen, device=model.device)
            pos_b = 0
        idx = perm[pos_b:pos_b + batch]
        pos_b += batch
        xb, yb = X[idx].contiguous(), Y[idx].contiguous()
        work.g.zero_()
        work.loss.zero_()
        forward(model, xb, work, target=yb, inv_batch=1.0 / batch)
        backward(model, xb, work)
        lr_t = lr * 0.5 * (1.0 + math.cos(math.pi * (step - 1) / steps))
        adam_step(model, work, m, vv, lr_t, step)
        if log_every and (step % log_every == 0 or step == 1):
            losses.append((step, float(work.loss.item())))
    model.train_log = losses
    return model
