"""Learned repose proposal: a small conv net proposes per-edge outflows.

The network (4 -> 32 -> 32 -> 32 -> 4 channels, 3x3 kernels, ReLU between,
no bias so that a flat surface proposes nothing) reads the height drop along
the east, north, north-east and north-west edges of every cell (scaled by
L * tan(repose)) and outputs one transfer per edge.  The transfers are applied
in flux form -- on a fixed-point grid in whole height quanta, so the total
volume stays exact -- and the plain relaxation sweep then finishes until every
face slope is within the tolerance: the plain sweep is both the fallback and
the judge.  The reference has no counterpart (its repose relaxation is the
plain sweep, slope_model.py:273-343, alone).

Every convolution (forward, data gradient and weight gradient) runs in the
library's tensor-core kernels (``sb_learned_conv`` / ``sb_learned_wgrad``).
PyTorch only holds device buffers and the Adam optimizer state.
"""

from __future__ import annotations

import ctypes as C
import math
import time
from dataclasses import dataclass
import numpy as np

from . import _lib

LAYERS = ((16, 32), (32, 32), (32, 32), (32, 16))   # padded channel counts
REAL = ((4, 32), (32, 32), (32, 32), (32, 4))       # channels that carry data


def _torch():
    import torch  # PyTorch holds buffers and optimizer state only
    return torch


def _ok(rc: int, what: str) -> None:
    if rc != _lib.SB_OK:
        msg = _lib.load().sb_learned_last_error()
        text = msg.decode(errors="replace") if msg else f"{what} failed with status {rc}"
        if rc in (_lib.SB_ERR_BAD_ARG, _lib.SB_ERR_CAPACITY):
            raise ValueError(text)
        raise _lib.B200DeviceError(text)


def pack_index(cin: int, cout: int) -> np.ndarray:
    """Packed position -> flat index of W[3, 3, cin, cout]: one block per tap
    (dy, dx), each the canonical K-major operand with rows n = co and k = ci
    (8 x 16-byte core matrices, (n/8, k/8) blocks of 128 bytes)."""
    block = cout * cin
    idx = np.empty(9 * block, dtype=np.int64)
    n = np.arange(cout)[:, None]
    k = np.arange(cin)[None, :]
    off = ((n >> 3) * (cin >> 3) + (k >> 3)) * 64 + (n & 7) * 8 + (k & 7)  # in elements
    for tap in range(9):
        idx[tap * block + off] = (tap * cin + k) * cout + n
    return idx


def flip_transpose(w):
    """Data-gradient weights: W'[dy, dx, co, ci] = W[2-dy, 2-dx, ci, co]."""
    return w.flip(0).flip(1).permute(0, 1, 3, 2).contiguous()


class ReposeNet:
    """The proposal network's FP32 master weights and their packed BF16 forms."""

    def __init__(self, device: int = 0, seed: int = 0, weights=None) -> None:
        torch = _torch()
        self.device = torch.device("cuda", device)
        gen = torch.Generator().manual_seed(seed)
        self.weights = []
        for li, ((ci, co), (ri, ro)) in enumerate(zip(LAYERS, REAL)):
            w = torch.zeros(3, 3, ci, co)
            if weights is not None:
                w.copy_(torch.as_tensor(np.asarray(weights[li]), dtype=torch.float32))
            else:
                std = math.sqrt(2.0 / (9 * ri)) * (0.1 if li == len(LAYERS) - 1 else 1.0)
                w[:, :, :ri, :ro] = torch.randn(3, 3, ri, ro, generator=gen) * std
            self.weights.append(w.to(self.device))
        self._fwd_idx = [torch.as_tensor(pack_index(ci, co), device=self.device)
                         for ci, co in LAYERS]
        self._bwd_idx = [torch.as_tensor(pack_index(co, ci), device=self.device)
                         for ci, co in LAYERS]
        self.status = torch.zeros(1, dtype=torch.int32, device=self.device)

    def packed(self):
        torch = _torch()
        return [w.reshape(-1)[i].to(torch.bfloat16) for w, i in zip(self.weights, self._fwd_idx)]

    def packed_backward(self):
        torch = _torch()
        return [flip_transpose(w).reshape(-1)[i].to(torch.bfloat16)
                for w, i in zip(self.weights, self._bwd_idx)]

    def numpy_weights(self):
        return [w.detach().cpu().numpy().astype(np.float64) for w in self.weights]

    def save(self, path) -> None:
        np.savez(path, *[w.cpu().numpy() for w in self.weights])

    @classmethod
    def load(cls, path, device: int = 0) -> "ReposeNet":
        with np.load(path) as z:
            ws = [z[f"arr_{i}"] for i in range(len(LAYERS))]
        return cls(device=device, weights=ws)


def conv_rows(b: int, h: int, w: int) -> int:
    """Rows per CTA: about one wave of 4 resident CTAs on each of 148 SMs."""
    tiles = (w + 127) // 128
    return int(min(32, max(4, -(-b * h * tiles // (148 * 4)))))


def conv(x, wpk, cin: int, cout: int, *, relu: bool, out_f32: bool | int = False, mask=None,
         status=None, stream=None, rows: int | None = None):
    """One tensor-core 3x3 convolution of a BF16 NHWC tensor [B, H, W, cin].

    ``out_f32``: False -> BF16 output of all channels; True -> FP32, all
    channels; an int k -> FP32, the first k channels only."""
    torch = _torch()
    b, h, w, c = x.shape
    rows = conv_rows(b, h, w) if rows is None else int(rows)
    if c != cin:
        raise ValueError(f"[soilb200] conv input has {c} channels, expected {cin}")
    nf = (cout if out_f32 is True else int(out_f32)) if out_f32 is not False else 0
    out = torch.empty(b, h, w, nf if nf else cout,
                      dtype=torch.float32 if nf else torch.bfloat16, device=x.device)
    st = stream if stream is not None else torch.cuda.current_stream(x.device).cuda_stream
    _ok(_lib.load().sb_learned_conv(x.data_ptr(), out.data_ptr(), wpk.data_ptr(),
                                    mask.data_ptr() if mask is not None else None, b, h, w, cin,
                                    cout, int(relu), nf, rows,
                                    status.data_ptr() if status is not None else None, st),
        "conv")
    return out


def wgrad(x, g, cin: int, cout: int, *, status=None, stream=None, rows: int = 16):
    """dW[3, 3, cin, cout] (f32) from a layer input x and its output gradient g."""
    torch = _torch()
    b, h, w, _ = x.shape
    nctas = ((w + 127) // 128) * ((h + rows - 1) // rows) * b
    part = torch.empty(nctas * 3 * 128 * cout, dtype=torch.float32, device=x.device)
    dw = torch.empty(3, 3, cin, cout, dtype=torch.float32, device=x.device)
    st = stream if stream is not None else torch.cuda.current_stream(x.device).cuda_stream
    _ok(_lib.load().sb_learned_wgrad(x.data_ptr(), g.data_ptr(), part.data_ptr(), part.numel(),
                                     dw.data_ptr(), b, h, w, cin, cout, rows,
                                     status.data_ptr() if status is not None else None, st),
        "wgrad")
    return dw


def network_forward(net: ReposeNet, feat, packed=None, stream=None):
    """Activations (inputs of layers 1..3) and the f32 fluxes [B, H, W, 4]."""
    packed = packed or net.packed()
    acts = []
    a = feat
    for li, (ci, co) in enumerate(LAYERS):
        last = li == len(LAYERS) - 1
        if li > 0:
            acts.append(a)
        a = conv(a, packed[li], ci, co, relu=not last, out_f32=4 if last else False,
                 status=net.status, stream=stream)
    return acts, a


def network_forward_fused(net: ReposeNet, feat, packed=None, stream=None, rows: int = 0):
    """The f32 fluxes [B, H, W, 4] of the whole network in one kernel
    (inference: no activations are kept).  Equal bit for bit to
    ``network_forward``'s output; ``rows`` = rows per CTA (0: about one wave)."""
    torch = _torch()
    packed = packed or net.packed()
    b, h, w, c = feat.shape
    if c != LAYERS[0][0]:
        raise ValueError(f"[soilb200] features have {c} channels, expected {LAYERS[0][0]}")
    flux = torch.empty(b, h, w, 4, dtype=torch.float32, device=feat.device)
    st = stream if stream is not None else torch.cuda.current_stream(feat.device).cuda_stream
    _ok(_lib.load().sb_learned_forward(feat.data_ptr(), flux.data_ptr(), packed[0].data_ptr(),
                                       packed[1].data_ptr(), packed[2].data_ptr(),
                                       packed[3].data_ptr(), b, h, w, int(rows),
                                       net.status.data_ptr(), st), "forward")
    return flux


def features_f64(heights, dx: float, dy: float, tan_crit: float):
    """BF16 features [B, H, W, 16] of float64 device heights [B, H, W]."""
    torch = _torch()
    b, h, w = heights.shape
    feat = torch.empty(b, h, w, 16, dtype=torch.bfloat16, device=heights.device)
    _ok(_lib.load().sb_learned_features_f64(heights.data_ptr(), feat.data_ptr(), b, h, w, dx, dy,
                                            tan_crit,
                                            torch.cuda.current_stream(heights.device).cuda_stream),
        "features")
    return feat


def loss_and_grads(net: ReposeNet, feat, target_dh, dx: float, dy: float, tan_crit: float,
                   norm: float):
    """Loss sum((dH - target)^2) * norm and the weight gradients (all on the GPU)."""
    torch = _torch()
    b, h, w, _ = feat.shape
    packed = net.packed()
    acts, flux = network_forward(net, feat, packed)
    resid = torch.empty(b, h, w, dtype=torch.float32, device=feat.device)
    dflux = torch.empty(b, h, w, 16, dtype=torch.bfloat16, device=feat.device)
    nblk = int(_lib.load().sb_learned_loss_blocks(b, h, w))
    part = torch.empty(nblk, dtype=torch.float64, device=feat.device)
    st = torch.cuda.current_stream(feat.device).cuda_stream
    _ok(_lib.load().sb_learned_loss(flux.data_ptr(), target_dh.data_ptr(), resid.data_ptr(),
                                    dflux.data_ptr(), part.data_ptr(), b, h, w, dx, dy, tan_crit,
                                    float(norm), st), "loss")
    back = net.packed_backward()
    grads = [None] * len(LAYERS)
    g = dflux
    layer_in = [feat] + acts
    for li in range(len(LAYERS) - 1, -1, -1):
        ci, co = LAYERS[li]
        grads[li] = wgrad(layer_in[li], g, ci, co, status=net.status)
        if li > 0:
            # data gradient: flipped/transposed weights, masked by the ReLU of this layer's input
            g = conv(g, back[li], co, ci, relu=False, mask=layer_in[li], status=net.status)
    return float(part.sum().item()), grads, flux


@dataclass
class TrainStats:
    steps: int
    first_loss: float
    last_loss: float
    seconds: float


def train(net: ReposeNet, pre: np.ndarray, post: np.ndarray, *, dx: float, dy: float,
          critical_angle_deg: float, steps: int = 200, batch: int = 16, lr: float = 2e-3,
          seed: int = 0) -> TrainStats:
    """Adam on pairs (pre, post) [N, H, W] float64 from the plain relaxation."""
    torch = _torch()
    dev = net.device
    tan_crit = float(np.tan(np.deg2rad(critical_angle_deg)))
    pre_t = torch.as_tensor(np.asarray(pre, dtype=np.float64), device=dev)
    tgt_t = torch.as_tensor(np.asarray(post, dtype=np.float64) - np.asarray(pre, dtype=np.float64),
                            device=dev).to(torch.float32)
    n, h, w = pre_t.shape
    scale = tan_crit * dx
    norm = 1.0 / (scale * scale * batch * h * w)
    params = [torch.nn.Parameter(wt.clone()) for wt in net.weights]
    opt = torch.optim.Adam(params, lr=lr)
    masks = []
    for (ci, co), (ri, ro) in zip(LAYERS, REAL):
        m = torch.zeros(3, 3, ci, co, device=dev)
        m[:, :, :ri, :ro] = 1.0
        masks.append(m)
    rng = np.random.default_rng(seed)
    first = last = float("nan")
    t0 = time.perf_counter()
    for step in range(steps):
        sel = torch.as_tensor(rng.choice(n, size=min(batch, n), replace=False), device=dev)
        feat = features_f64(pre_t[sel].contiguous(), dx, dy, tan_crit)
        loss, grads, _ = loss_and_grads(net, feat, tgt_t[sel].contiguous(), dx, dy, tan_crit, norm)
        for p, g, m in zip(params, grads, masks):
            p.grad = g * m
        opt.step()
        for wt, p in zip(net.weights, params):
            wt.copy_(p.detach())
        if step == 0:
            first = loss
        last = loss
    torch.cuda.synchronize(dev)
    if int(net.status.item()) != 0:
        raise _lib.B200DeviceError("[soilb200] a bounded device wait gave up in a conv kernel")
    return TrainStats(steps, first, last, time.perf_counter() - t0)


# The proposal schedule the bench and the gain test use: four full-size and
# four half-size rounds with 5 plain sweeps after each; a surface that is not
# at the tolerance 20 sweeps later (a long run-out) gets six full and six
# half rounds more, 2 sweeps after each (tuned on the post-cut config-1
# surfaces of seeds 1 and 6-9; seeds 2-5 were kept for checking).
SCHEDULE = dict(scales=(1.0, 1.0, 1.0, 1.0, 0.5, 0.5, 0.5, 0.5), plain_between=5,
                check_sweeps=20, extra_scales=(1.0,) * 6 + (0.5,) * 6, extra_between=2)
PLAIN = dict(scales=())  # the plain sweep alone


class LearnedRelaxation:
    """Learned proposal rounds on a fixed-point grid's resident b_eff, then the
    plain sweep to the tolerance."""

    def __init__(self, grid, net: ReposeNet, critical_angle_deg: float,
                 fused: bool = True) -> None:
        torch = _torch()
        self.fused = bool(fused)  # False: one launch per layer (the training path's kernels)
        if grid.precision != "fx32":
            raise ValueError("[soilb200] the learned proposal runs on fx32 grids")
        self.grid = grid
        self.net = net
        self.tan_crit = float(np.tan(np.deg2rad(critical_angle_deg)))
        ny, nx = grid.shape
        dev = net.device
        self._feat = torch.empty(1, ny, nx, 16, dtype=torch.bfloat16, device=dev)
        self._tq = torch.empty(ny * nx * 4, dtype=torch.int32, device=dev)
        self._packed = net.packed()
        self._stream = grid.stream_handle()
        # buffers made during a proposal belong to the grid's stream, so the
        # allocator never hands them out while that stream still reads them
        self._torch_stream = torch.cuda.ExternalStream(self._stream, device=dev)
        torch.cuda.current_stream(dev).synchronize()

    def propose(self, rounds: int = 1, scale: float = 1.0) -> None:
        """``rounds`` proposals; each moves ``scale`` times the network's
        transfer (flux * tan_crit * dx * scale per edge, still limited to half
        the height difference and rounded toward zero to whole quanta)."""
        torch = _torch()
        lib = _lib.load()
        if not scale > 0.0:
            raise ValueError("[soilb200] the proposal scale must be positive")
        with torch.cuda.stream(self._torch_stream):
            for _ in range(rounds):
                _lib.check(self.grid.ctx, lib.sb_learned_features(self.grid.ctx,
                                                                  self._feat.data_ptr(),
                                                                  self.tan_crit), "features")
                if self.fused:
                    flux = network_forward_fused(self.net, self._feat, self._packed,
                                                 stream=self._stream)
                else:
                    _, flux = network_forward(self.net, self._feat, self._packed,
                                              stream=self._stream)
                # the transfer is flux * tan * dx, so the scale rides on tan
                _lib.check(self.grid.ctx, lib.sb_learned_apply(self.grid.ctx, flux.data_ptr(),
                                                               self._tq.data_ptr(),
                                                               self.tan_crit * scale), "apply")

    def relax(self, tolerance_m: float, max_iterations: int = 20000, rounds: int = 1,
              spacing=None, plain_between: int = 0, scales=None, check_sweeps: int = 0,
              extra_scales=None, extra_between: int = 0):
        """Learned rounds, then relax_critical_slope sweeps to the tolerance.

        With ``plain_between`` > 0 each proposal is followed by that many plain
        sweeps (the proposal moves material over the network's receptive
        field, the sweeps resolve what it left); the whole schedule is queued
        on the grid's stream without host round trips, and only the final
        sweeps to the tolerance report back.  ``scales`` (one positive factor
        per round, default 1.0 each) damps later proposals, whose full-size
        transfers overshoot once the surface is near repose.

        ``check_sweeps`` > 0 adapts the schedule to the surface: after the
        rounds, at most that many plain sweeps run; a surface that has not
        reached the tolerance by then (one whose run-out is long) gets the
        further proposal rounds ``extra_scales`` (``extra_between`` sweeps
        after each) before the sweeps to the tolerance.  Returns the final
        RelaxStats, with ``iterations`` counting every sweep queued (the
        interleaved calls as an upper bound: they stop early when already
        converged)."""
        rounds = max(0, int(rounds))
        scales = [1.0] * rounds if scales is None else [float(x) for x in scales]
        if len(scales) != rounds:
            raise ValueError("[soilb200] scales needs one factor per proposal round")
        extra = [float(x) for x in (extra_scales or ())]
        s0, s1 = spacing if spacing is not None else (self.grid.dy, self.grid.dx)
        lib = _lib.load()

        def sweeps(count: int):
            p = _lib.RelaxParams(float(s0), float(s1), self.tan_crit, float(tolerance_m),
                                 int(max(count, 1)), 0)
            _lib.check(self.grid.ctx, lib.sb_relax_sweeps(self.grid.ctx, p), "relax")

        def full(limit: int):
            p = _lib.RelaxParams(float(s0), float(s1), self.tan_crit, float(tolerance_m),
                                 int(limit), 0)
            st = _lib.RelaxStats()
            _lib.check(self.grid.ctx, lib.sb_relax_full(self.grid.ctx, p, st), "relax")
            return st

        done = 0
        for sc in scales:
            self.propose(1, sc)
            if plain_between > 0:
                sweeps(plain_between)
                done += plain_between
        if check_sweeps > 0 and extra:
            st = full(check_sweeps)
            done += int(st.iterations)
            if st.converged:
                st.iterations = done
                return st
            for sc in extra:
                self.propose(1, sc)
                if extra_between > 0:
                    sweeps(extra_between)
                    done += extra_between
        st = full(max_iterations)
        st.iterations = int(st.iterations) + done
        return st

    def relax_scheduled(self, tolerance_m: float, schedule=None, max_iterations: int = 400000,
                        spacing=None):
        """``relax`` with a whole proposal schedule (a dict with the keys of
        ``SCHEDULE``, the default); ``schedule={"scales": ()}`` gives the plain
        sweep alone."""
        s = SCHEDULE if schedule is None else schedule
        scales = tuple(s.get("scales", ()))
        if not scales:
            return self.relax(tolerance_m, max_iterations=max_iterations, rounds=0,
                              spacing=spacing)
        return self.relax(tolerance_m, max_iterations=max_iterations, rounds=len(scales),
                          spacing=spacing, plain_between=int(s.get("plain_between", 0)),
                          scales=scales, check_sweeps=int(s.get("check_sweeps", 0)),
                          extra_scales=tuple(s.get("extra_scales", ())),
                          extra_between=int(s.get("extra_between", 0)))
