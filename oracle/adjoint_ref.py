"""FP64 restatement of bandpass + centroid refinement at fixed peaks.

TEST INFRASTRUCTURE ONLY: the checker of libgt's gt_adjoint_* entry points.
Nothing in the product imports this module.

The forward is the real-valued form of the locate path at a fixed walk
(gpu-tracking/src/shaders/preprocess_rows.wgsl:14-53 and
preprocess_cols.wgsl:14-61 for the bandpass, centers.wgsl:23-109 for the
centroid, walk_cols.wgsl:69-73 for the final position):

    a_i  = exp(-i^2 / (2 s)) / sum_j exp(-j^2 / (2 s)),  i = -k//2 .. k//2
    G    = sum_ij a_i a_j I(u + i, v + j)           taps outside the frame skipped
    B    = sum_ij I(refl(u + i), refl(v + j)) / kk   refl(x) = -x-1 | 2n-x-1
    P    = max(G - B, 0)
    mass = sum_circle P,  y = up + sum i P / mass,  x = vp + sum j P / mass

with s = noise_size and kk = k^2.  ``kk`` may be passed as a real number to
differentiate through the relaxation of smoothing_size (box normalisation
1/k^2 continuous in k, window and taps fixed).

Three checkers live here: central finite differences of the FP64 forward,
a torch float64 autograd gradient of the same forward, and the
linear-propagation uncertainty from that gradient.
"""
import numpy as np


def circle(rc):
    """Centroid circle offsets in the loop order of centers.wgsl (i outer, j
    inner), mask i^2 + j^2 <= r^2 evaluated in f32 as the shader does."""
    out = []
    r2 = np.float32(rc) * np.float32(rc)
    for i in range(-rc, rc + 1):
        for j in range(-rc, rc + 1):
            if np.float32(i) * np.float32(i) + np.float32(j) * np.float32(j) <= r2:
                out.append((i, j))
    return np.array(out, dtype=np.int64).reshape(-1, 2)


def taps(k, s):
    kr = k // 2
    i = np.arange(-kr, kr + 1, dtype=np.float64)
    w = np.exp(-i * i / (2.0 * s))
    return w / w.sum()


def _refl(x, n):
    x = np.where(x < 0, -x - 1, x)
    return np.where(x >= n, 2 * n - x - 1, x)


class Particle:
    """Index tables of one walk record: for each circle pixel, the Gaussian
    taps that fall inside the frame and the reflected box taps."""

    def __init__(self, rec, H, W, diameter, k):
        self.t, self.ul, self.vl, self.up, self.vp = (int(v) for v in rec)
        self.H, self.W = H, W
        self.rc = (diameter - 1) // 2
        self.border = diameter // 2
        self.kr = k // 2
        self.interior = not (self.ul - self.border < 0 or self.ul + self.border >= H or
                             self.vl - self.border < 0 or self.vl + self.border >= W)
        c = circle(self.rc)
        self.ci, self.cj = c[:, 0].astype(np.float64), c[:, 1].astype(np.float64)
        kr = self.kr
        o = np.arange(-kr, kr + 1)
        pu = (self.ul + c[:, 0])[:, None, None] + o[None, :, None]
        pv = (self.vl + c[:, 1])[:, None, None] + o[None, None, :]
        pu, pv = np.broadcast_arrays(pu, pv)
        self.gin = (pu >= 0) & (pu < H) & (pv >= 0) & (pv < W)
        self.g_lin = np.where(self.gin, np.clip(pu, 0, H - 1) * W + np.clip(pv, 0, W - 1), 0)
        self.b_lin = _refl(pu, H) * W + _refl(pv, W)
        self.ti = np.broadcast_to(o[None, :, None], pu.shape)
        self.tj = np.broadcast_to(o[None, None, :], pu.shape)

    def residual(self, frame, s, k, kk=None):
        """G - B at the circle pixels (FP64)."""
        a = taps(k, s)
        kk = float(k * k) if kk is None else float(kk)
        f = frame.reshape(-1)
        wg = a[self.ti + self.kr] * a[self.tj + self.kr] * self.gin
        G = (wg * f[self.g_lin]).sum(axis=(1, 2))
        B = f[self.b_lin].sum(axis=(1, 2)) / kk
        return G - B

    def refine(self, frame, s, k, kk=None):
        if not self.interior:
            return np.array([self.up, self.vp, 0.0])
        P = np.maximum(self.residual(frame, s, k, kk), 0.0)
        m = P.sum()
        return np.array([self.up + (self.ci * P).sum() / m, self.vp + (self.cj * P).sum() / m, m])

    def window(self):
        """Frame pixels (rows, cols) that the particle's bandpass reads."""
        R = self.rc + self.kr
        r = np.arange(self.ul - R, self.ul + R + 1)
        c = np.arange(self.vl - R, self.vl + R + 1)
        r = r[(r >= 0) & (r < self.H)]
        c = c[(c >= 0) & (c < self.W)]
        return r, c


def refine(frames, walk, diameter, s, k, kk=None):
    """(n, 3) y, x, mass of every walk record (FP64)."""
    T, H, W = frames.shape
    f64 = frames.astype(np.float64)
    out = np.empty((len(walk), 3))
    for q, rec in enumerate(walk):
        pt = Particle(rec, H, W, diameter, k)
        out[q] = pt.refine(f64[pt.t], s, k, kk)
    return out


def clip_margin(frames, walk, diameter, s, k):
    """Per particle, the smallest |G - B| over its circle: where this is tiny
    an FP32 and an FP64 evaluation may disagree about the clip."""
    T, H, W = frames.shape
    f64 = frames.astype(np.float64)
    out = np.full(len(walk), np.inf)
    for q, rec in enumerate(walk):
        pt = Particle(rec, H, W, diameter, k)
        if pt.interior:
            out[q] = np.abs(pt.residual(f64[pt.t], s, k)).min()
    return out


def fd_pixels(frames, walk, upstream, diameter, s, k, npix=32, h=1e-3, seed=0):
    """Central differences (step h) of L = sum_q upstream[q] . refine[q] with
    respect to ``npix`` random pixels of each particle's window.  Returns
    (t, row, col, dL/dI) samples; perturbed pixels affect every particle
    whose window contains them, all of which enter L."""
    T, H, W = frames.shape
    f64 = frames.astype(np.float64)
    parts = [Particle(rec, H, W, diameter, k) for rec in walk]
    rng = np.random.default_rng(seed)
    R = parts[0].rc + parts[0].kr if parts else 0
    samples = []
    for pt in parts:
        r, c = pt.window()
        for _ in range(npix):
            u, v = int(rng.choice(r)), int(rng.choice(c))
            near = [q for q, o in enumerate(parts)
                    if o.t == pt.t and abs(o.ul - u) <= R and abs(o.vl - v) <= R]
            img = f64[pt.t].copy()
            img[u, v] += h
            lp = sum(float(upstream[q] @ parts[q].refine(img, s, k)) for q in near)
            img[u, v] -= 2 * h
            lm = sum(float(upstream[q] @ parts[q].refine(img, s, k)) for q in near)
            samples.append((pt.t, u, v, (lp - lm) / (2 * h)))
    return samples


def fd_params(frames, walk, upstream, diameter, s, k, h=1e-3):
    """Central differences of L with respect to noise_size and to the
    relaxed smoothing_size (kk = k^2 continuous)."""
    def L(s_, kk_):
        return float((upstream * refine(frames, walk, diameter, s_, k, kk_)).sum())
    ds = (L(s + h, None) - L(s - h, None)) / (2 * h)
    dk = (L(s, (k + h) ** 2) - L(s, (k - h) ** 2)) / (2 * h)
    return ds, dk


def torch_reference(frames, walk, upstream, diameter, s, k):
    """dL/dframes, dL/ds, dL/dk by torch float64 autograd of the dense
    restatement (whole-frame bandpass, then the centroid at each walk)."""
    import torch

    T, H, W = frames.shape
    I = torch.tensor(frames, dtype=torch.float64, requires_grad=True)
    st = torch.tensor(float(s), dtype=torch.float64, requires_grad=True)
    kt = torch.tensor(float(k), dtype=torch.float64, requires_grad=True)
    kr = k // 2
    i = torch.arange(-kr, kr + 1, dtype=torch.float64)
    w = torch.exp(-i * i / (2.0 * st))
    a = w / w.sum()
    # Gaussian: zero padding
    x = I.unsqueeze(1)
    g = torch.nn.functional.conv2d(x, a.view(1, 1, 1, -1), padding=(0, kr))
    g = torch.nn.functional.conv2d(g, a.view(1, 1, -1, 1), padding=(kr, 0)).squeeze(1)
    # box: single reflection including the edge pixel
    ri = torch.tensor(_refl(np.arange(-kr, H + kr), H))
    ci = torch.tensor(_refl(np.arange(-kr, W + kr), W))
    xp = I[:, ri][:, :, ci]
    ones = torch.ones(1, 1, 2 * kr + 1, 2 * kr + 1, dtype=torch.float64)
    b = torch.nn.functional.conv2d(xp.unsqueeze(1), ones).squeeze(1) / (kt * kt)
    P = torch.clamp(g - b, min=0.0)
    c = circle((diameter - 1) // 2)
    ci_t = torch.tensor(c[:, 0], dtype=torch.float64)
    cj_t = torch.tensor(c[:, 1], dtype=torch.float64)
    up = torch.tensor(upstream, dtype=torch.float64)
    L = torch.zeros((), dtype=torch.float64)
    border = diameter // 2
    for q, (t, ul, vl, u_, v_) in enumerate(np.asarray(walk, dtype=np.int64)):
        if ul - border < 0 or ul + border >= H or vl - border < 0 or vl + border >= W:
            continue
        vals = P[t, ul + c[:, 0], vl + c[:, 1]]
        m = vals.sum()
        y = u_ + (ci_t * vals).sum() / m
        xx = v_ + (cj_t * vals).sum() / m
        L = L + up[q, 0] * y + up[q, 1] * xx + up[q, 2] * m
    L.backward()
    return I.grad.numpy(), float(st.grad), float(kt.grad)


def uncertainty(frames, walk, diameter, s, k, gain=1.0, read_noise=0.0):
    """(n, 3) standard deviations of y, x, mass by linear propagation of
    var(I) = gain * max(I, 0) + read_noise^2 through the FP64 Jacobian."""
    out = np.zeros((len(walk), 3))
    var = gain * np.maximum(frames.astype(np.float64), 0.0) + read_noise ** 2
    for q in range(len(walk)):
        for o in range(3):
            up = np.zeros((len(walk), 3))
            up[q, o] = 1.0
            g, _, _ = torch_reference(frames[walk[q, 0]:walk[q, 0] + 1],
                                      np.array([[0, *walk[q, 1:]]]), up[q:q + 1], diameter, s, k)
            out[q, o] = np.sqrt((g[0] ** 2 * var[walk[q, 0]]).sum())
    return out
