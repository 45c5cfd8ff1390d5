"""Learned Davidson preconditioner (no counterpart in the reference).

Replaces the diagonal preconditioner of pdvdson (source/tools/pdvdson.py:275-278)
by a per-symmetry-block correction

    c_i = r_i * alpha_b / (|diag_i - e| + sigma_b),   (log alpha_b, log sigma_b) = MLP(features_b)

where b is the (N, Sz) block of the packed wavefunction that element i belongs
to and features_b summarise the residual and the shifted diagonal inside the
block.  The MLP (3 layers, width 256, BF16 weights, FP32 accumulation) runs on
the GPU through hand-written forward/backward/Adam kernels (csrc/mlp.cu).
It is trained on pairs the solver produces itself: for every Davidson
iteration k of a dot, the residual r_k and, once the dot has converged to x*,
the exact correction direction t_k = x* - (x*.x_k) x_k; the loss is
1 - cos^2(c(r_k), t_k) (Davidson adds span{c}: the sign of c is irrelevant).
Untrained, or not better than Jacobi on held-out pairs, the fallback is the reference's
Jacobi formula (alpha = 1, sigma = 1e-4).  The preconditioner only changes the
search directions, never the Rayleigh-Ritz eigenvalue.
"""
import math

import numpy
import torch

from . import native
from .native import check

NFEAT = 8
HIDDEN = 256
NOUT = 2
YCLAMP = 30.0     # range of the network outputs log(alpha), log(sigma) used by the correction


def _stream(dev):
    return torch.cuda.current_stream(dev).cuda_stream


def block_index(layout, device):
    """Element -> block id (position of the block in packed order) for a layout."""
    idx = numpy.empty(layout.size, dtype=numpy.int32)
    for b, blk in enumerate(layout.idx_allowed):
        o = int(layout.ioff[blk])
        idx[o:o + int(layout.ndim[blk])] = b
    return torch.from_numpy(idx).to(device), len(layout.idx_allowed)


def features(r, d, e, blk, nblk, it=0):
    """Per-block features [nblk, NFEAT] (float32) from residual r and diagonal d."""
    dev = r.device
    blk64 = blk.long()
    sh = (d - e).abs() + 1e-12
    cnt = torch.zeros(nblk, dtype=torch.float64, device=dev).index_add_(0, blk64, torch.ones_like(sh))
    lsh = torch.log(sh)
    mean_l = torch.zeros(nblk, dtype=torch.float64, device=dev).index_add_(0, blk64, lsh) / cnt
    mn = torch.full((nblk,), 1e300, dtype=torch.float64, device=dev).scatter_reduce_(0, blk64, sh, "amin")
    mx = torch.zeros(nblk, dtype=torch.float64, device=dev).scatter_reduce_(0, blk64, sh, "amax")
    neg = torch.zeros(nblk, dtype=torch.float64, device=dev).index_add_(0, blk64, ((d - e) < 0).double()) / cnt
    rn2 = torch.zeros(nblk, dtype=torch.float64, device=dev).index_add_(0, blk64, r * r)
    rtot = torch.sqrt(rn2.sum()) + 1e-300
    f = torch.stack([mean_l, torch.log(mn), torch.log(mx), neg,
                     0.5 * torch.log(rn2 / (rtot * rtot) * nblk + 1e-30), torch.log(cnt),
                     torch.full_like(cnt, math.log(float(rtot))), torch.full_like(cnt, it / 20.0)], dim=1)
    return f.float().contiguous()


class MLP(object):
    """Weights (FP32 master + BF16 working copies) and the native kernels."""

    def __init__(self, device, seed=0):
        self.device = device
        g = torch.Generator().manual_seed(seed)
        shapes = {"W1": (HIDDEN, NFEAT), "b1": (HIDDEN,), "W2": (HIDDEN, HIDDEN), "b2": (HIDDEN,),
                  "W3": (NOUT, HIDDEN), "b3": (NOUT,)}
        self.p = {}
        for k, s in shapes.items():
            if k.startswith("W"):
                w = torch.randn(s, generator=g) * (1.0 / math.sqrt(s[1]))
                if k == "W3":
                    w *= 0.01          # start close to the output bias (the Jacobi fallback)
            else:
                w = torch.zeros(s)
            self.p[k] = w.float().to(device).contiguous()
        # output bias: alpha = 1, sigma = 1e-4 -> the reference's preconditioner
        self.p["b3"][:] = torch.tensor([0.0, math.log(1e-4)], device=device)
        self.bf = {k: self.p[k].to(torch.bfloat16).contiguous() for k in ("W1", "W2", "W3")}
        self.m = {k: torch.zeros_like(v) for k, v in self.p.items()}
        self.v = {k: torch.zeros_like(v) for k, v in self.p.items()}
        self.step = 0

    def forward(self, X):
        B = X.shape[0]
        H1 = torch.empty((B, HIDDEN), dtype=torch.float32, device=self.device)
        H2 = torch.empty_like(H1)
        Y = torch.empty((B, NOUT), dtype=torch.float32, device=self.device)
        p, bf = self.p, self.bf
        check(native.lib().qc_mlp_forward(B, NFEAT, X.data_ptr(), bf["W1"].data_ptr(), p["b1"].data_ptr(),
                                          bf["W2"].data_ptr(), p["b2"].data_ptr(), bf["W3"].data_ptr(),
                                          p["b3"].data_ptr(), H1.data_ptr(), H2.data_ptr(), Y.data_ptr(),
                                          _stream(self.device)), "qc_mlp_forward")
        return Y, H1, H2

    def backward(self, X, H1, H2, dY):
        g = {k: torch.zeros_like(v) for k, v in self.p.items()}
        check(native.lib().qc_mlp_backward(X.shape[0], NFEAT, X.data_ptr(), self.bf["W2"].data_ptr(),
                                           self.bf["W3"].data_ptr(), H1.data_ptr(), H2.data_ptr(),
                                           dY.contiguous().data_ptr(), g["W1"].data_ptr(), g["b1"].data_ptr(),
                                           g["W2"].data_ptr(), g["b2"].data_ptr(), g["W3"].data_ptr(),
                                           g["b3"].data_ptr(), _stream(self.device)), "qc_mlp_backward")
        return g

    def adam(self, grads, lr=1e-3, scale=1.0):
        self.step += 1
        lib = native.lib()
        for k, w in self.p.items():
            wb = self.bf[k].data_ptr() if k in self.bf else None
            check(lib.qc_adam_step(w.numel(), w.data_ptr(), wb, grads[k].data_ptr(), self.m[k].data_ptr(),
                                   self.v[k].data_ptr(), lr, 0.9, 0.999, 1e-8, self.step, scale,
                                   _stream(self.device)), "qc_adam_step")


def correction(r, d, e, blk, Y):
    """c = r * alpha_b / (|d - e| + sigma_b) on the device (qc_precond_apply)."""
    c = torch.empty_like(r)
    check(native.lib().qc_precond_apply(r.numel(), r.data_ptr(), d.data_ptr(), float(e), blk.data_ptr(),
                                        Y.data_ptr(), c.data_ptr(), _stream(r.device)), "qc_precond_apply")
    return c


def loss_and_grad(r, d, e, blk, nblk, Y, t):
    """1 - cos^2(c, t) and dL/dY (per block) for c = correction(r, d, e, blk, Y).  Davidson
    adds span{c} to its subspace, so only the direction of c up to sign matters: the loss is
    sign-invariant (1 - cos would push a correct direction of the opposite sign away)."""
    blk64 = blk.long()
    Yd = Y.double()
    inside = ((Yd > -YCLAMP) & (Yd < YCLAMP)).double()          # clamp(Y): zero gradient outside
    Yd = Yd.clamp(-YCLAMP, YCLAMP)
    alpha = torch.exp(Yd[:, 0])[blk64]
    sigma = torch.exp(Yd[:, 1])[blk64]
    den = (d - e).abs() + sigma
    c = r * alpha / den
    nc = torch.linalg.norm(c) + 1e-300
    nt = torch.linalg.norm(t) + 1e-300
    cos = torch.dot(c, t) / (nc * nt)
    dc = -2.0 * cos * (t / (nc * nt) - cos * c / (nc * nc))
    g_la = torch.zeros(nblk, dtype=torch.float64, device=r.device).index_add_(0, blk64, dc * c)
    g_ls = torch.zeros(nblk, dtype=torch.float64, device=r.device).index_add_(0, blk64, -dc * c * sigma / den)
    return float(1.0 - cos * cos), (torch.stack([g_la, g_ls], dim=1) * inside).float().contiguous()


class LearnedPreconditioner(object):
    """Davidson preconditioner callable + the training-pair collector."""

    def __init__(self, device, seed=0, train_sweeps=0, epochs=30):
        """train_sweeps > 0: collect (residual, exact correction) pairs during that many
        sweeps (end_sweep() counts them), then train on the GPU and switch the network on."""
        self.device = torch.device(device)
        self.net = MLP(self.device, seed)
        self.enabled = False         # Jacobi fallback until trained
        self.train_sweeps = int(train_sweeps)
        self.epochs = int(epochs)
        self.sweeps = 0
        self.train_info = None
        self.blk = None
        self.nblk = 0
        self.it = 0
        self.pairs = []              # (r, d, e, blk, nblk, t) on the device
        self.collect = False
        self.max_pairs = 400
        self._dot = []
        self.history = []
        if self.train_sweeps > 0:
            self.collect = True

    def end_sweep(self):
        """Schedule hook: after train_sweeps sweeps of collected pairs, train on the GPU and
        switch the network on only if it beats Jacobi on held-out pairs (every fifth pair,
        not trained on) by at least 5 %; otherwise the Jacobi fallback stays."""
        self.sweeps += 1
        if self.train_sweeps > 0 and self.sweeps == self.train_sweeps:
            self.collect = False
            import time as _t
            t0 = _t.time()
            held = self.pairs[4::5]
            train = [p for i, p in enumerate(self.pairs) if i % 5 != 4]
            self.pairs = train
            losses = self.train(epochs=self.epochs)
            self.pairs = held
            jac, mod = self.jacobi_loss(), self.model_loss()
            self.enabled = bool(held) and mod < 0.95 * jac
            self.train_info = {"pairs": len(train), "held_out": len(held), "epochs": self.epochs,
                               "train_s": round(_t.time() - t0, 2),
                               "loss_first": losses[0] if losses else None,
                               "loss_last": losses[-1] if losses else None,
                               "held_out_loss_jacobi": jac, "held_out_loss_network": mod}
            self.pairs = []              # the device copies are not needed any more

    def summary(self):
        return {"enabled": self.enabled, "trained_after_sweeps": self.train_sweeps, "train": self.train_info}

    # -- per dot
    def set_layout(self, layout):
        self.blk, self.nblk = block_index(layout, self.device)
        self.it = 0
        self._dot = []

    def __call__(self, r, diag, e, x):
        self.it += 1
        jac = r / ((diag - e).abs() + 1e-4)
        if not self.enabled:
            return jac
        X = features(r, diag, float(e), self.blk, self.nblk, self.it)
        Y, _, _ = self.net.forward(X)
        c = correction(r.contiguous(), diag.contiguous(), float(e), self.blk, Y)
        # Davidson uses only the direction: the correction gets the Jacobi step's norm, so a
        # network scale that collapsed (or blew up) cannot drop the new direction below the
        # orthogonalisation threshold; a non-finite correction falls back to Jacobi
        nc = torch.linalg.norm(c)
        if not bool(torch.isfinite(nc)) or float(nc) == 0.0:
            return jac
        return c * (torch.linalg.norm(jac) / nc)

    # -- training-pair collection (Davidson record hook)
    def record(self, r, diag, e, x):
        if self.collect and len(self.pairs) + len(self._dot) < self.max_pairs:
            self._dot.append((r.clone(), diag, float(e), x.clone(), self.it))

    def end_dot(self, xstar):
        """Turn the recorded iterations of the finished dot into (residual, exact correction) pairs."""
        xs = xstar / torch.linalg.norm(xstar)
        for (r, d, e, x, it) in self._dot:
            t = xs - torch.dot(xs, x) * x
            if float(torch.linalg.norm(t)) > 1e-10:
                self.pairs.append((r, d, e, self.blk, self.nblk, t, it))
        self._dot = []

    # -- training on the GPU
    def train(self, epochs=30, lr=2e-3):
        if not self.pairs:
            return []
        losses = []
        for ep in range(epochs):
            tot = 0.0
            for (r, d, e, blk, nblk, t, it) in self.pairs:
                X = features(r, d, e, blk, nblk, it)
                Y, H1, H2 = self.net.forward(X)
                L, dY = loss_and_grad(r, d, e, blk, nblk, Y, t)
                if not (math.isfinite(L) and bool(torch.isfinite(dY).all())):
                    continue                 # a pair the current network cannot score: no step
                g = self.net.backward(X, H1, H2, dY)
                self.net.adam(g, lr=lr)
                tot += L
            losses.append(tot / len(self.pairs))
        self.history += losses
        return losses

    def jacobi_loss(self):
        """Mean loss of the Jacobi fallback on the collected pairs (the baseline)."""
        tot = 0.0
        for (r, d, e, blk, nblk, t, it) in self.pairs:
            Y = torch.zeros((nblk, 2), dtype=torch.float32, device=self.device)
            Y[:, 1] = math.log(1e-4)
            L, _ = loss_and_grad(r, d, e, blk, nblk, Y, t)
            tot += L
        return tot / max(1, len(self.pairs))

    def model_loss(self):
        tot = 0.0
        for (r, d, e, blk, nblk, t, it) in self.pairs:
            Y, _, _ = self.net.forward(features(r, d, e, blk, nblk, it))
            L, _ = loss_and_grad(r, d, e, blk, nblk, Y, t)
            tot += L
        return tot / max(1, len(self.pairs))
