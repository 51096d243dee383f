"""Learned warm start for batched Newton solves.

A multilayer perceptron maps each scenario's loads (P and Q at every bus) and
its PV voltage setpoints to a starting state: Va at the PV and PQ buses and
Vm at the PQ buses, in the Jacobian-row order the engine's warm entry point
reads (``NewtonSolver.solve_batch_warm_device``).  Newton then runs from that
prediction to the same tolerance as from a flat start; scenarios that do not
converge within the iteration cap are solved again from the flat start.

The network is trained on solutions the engine itself produces, with the
engine's own BF16 kernels (include/cupf_mlp.h): tcgen05 GEMMs with fused
bias + GELU epilogues for the forward pass, GELU-derivative epilogues and
transposed GEMMs for the backward pass, and Adam on FP32 master weights.
torch only allocates the buffers.  Layer widths are padded to multiples of
128 (the GEMM tile); padded rows and columns stay exactly zero.

nominal_state() is the model-free alternative: every scenario starts from the
converged nominal-load state, which is what the 10,000-bus gradient case uses.
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np

from . import _capi

EPI_F32, EPI_BIAS_F32, EPI_BIAS_GELU, EPI_DGELU = 0, 1, 2, 3


def _round_up(x: int, m: int) -> int:
    return (x + m - 1) // m * m


def _ptr(t) -> C.c_void_p:
    return C.c_void_p(t.data_ptr())


class MLP:
    """Dense GELU network with BF16 weights and activations, FP32 accumulation,
    FP32 master weights (Adam).  All compute goes through the mlp_* kernels.

    Hidden layers: a_{l+1} = gelu(a_l W_l^T + b_l).  With skip=True the output
    layer reads [a_L | x] (the last hidden activation next to the standardized
    input), so the dominant, nearly linear part of the load-to-state map has a
    direct path and the GELU stack learns the nonlinear remainder.

    Inference evaluates the output layer with split weights, W = hi + lo with
    hi = bf16(W) and lo = bf16(W - hi), in one GEMM (mlp_gemm_bf16_split).
    Rounding the output weights to bf16 alone adds independent noise to every
    bus's predicted angle; Newton's mismatch sees that noise across every
    branch, while the network's smooth, large-scale error costs it little."""

    def __init__(self, n_in: int, n_out: int, hidden: int = 1024, layers: int = 3, seed: int = 0,
                 device=None, skip: bool = True):
        import torch

        if hidden % 128:
            raise ValueError("hidden width must be a multiple of 128")
        self.lib = _capi.load()
        self.torch = torch
        self.dev = torch.device(device or "cuda")
        self.n_in, self.n_out, self.hidden, self.layers, self.skip = n_in, n_out, hidden, layers, skip
        self.k0, self.no = _round_up(n_in, 128), _round_up(n_out, 128)
        self.cat_w = hidden + (self.k0 if skip else 0)   # width of the output layer's input
        self.dims_in = [self.k0] + [hidden] * (layers - 1) + [self.cat_w]
        self.dims_out = [hidden] * layers + [self.no]
        gen = torch.Generator().manual_seed(seed)
        self.W, self.b, self.W16, self.WT16, self.mW, self.vW, self.mb, self.vb = [], [], [], [], [], [], [], []
        for i in range(layers + 1):
            d_in, d_out = self.dims_in[i], self.dims_out[i]
            real_out = n_out if i == layers else hidden
            w = torch.zeros(d_out, d_in)
            if i == 0:
                w[:, :n_in] = torch.randn(d_out, n_in, generator=gen) * math.sqrt(2.0 / n_in)
            elif i < layers:
                w[:] = torch.randn(d_out, d_in, generator=gen) * math.sqrt(2.0 / hidden)
            else:
                fan = hidden + (n_in if skip else 0)
                w[:real_out, :hidden] = torch.randn(real_out, hidden, generator=gen) * math.sqrt(1.0 / fan)
                if skip:
                    w[:real_out, hidden:hidden + n_in] = torch.randn(real_out, n_in, generator=gen) * math.sqrt(1.0 / fan)
            w = w.to(self.dev)
            self.W.append(w)
            self.b.append(torch.zeros(d_out, device=self.dev))
            self.W16.append(w.to(torch.bfloat16).contiguous())
            self.WT16.append(torch.empty(d_in, d_out, dtype=torch.bfloat16, device=self.dev))
            self.mW.append(torch.zeros_like(w))
            self.vW.append(torch.zeros_like(w))
            self.mb.append(torch.zeros(d_out, device=self.dev))
            self.vb.append(torch.zeros(d_out, device=self.dev))
        self._refresh_transposes()
        self.step = 0
        self._bufs: dict[tuple, dict] = {}
        self.split_out = True        # inference: output layer with hi + lo weights
        self.Wsplit16 = None         # [no, 2 cat_w] bf16: [hi | lo] of the fp32 output weights
        self._split_stale = True

    # -- low-level wrappers --
    def _stream(self):
        return C.c_void_p(self.torch.cuda.current_stream(self.dev).cuda_stream)

    def _check(self, rc: int) -> None:
        if rc:
            raise RuntimeError("mlp kernel: " + self.lib.mlp_last_error().decode())

    def gemm(self, A, B, out, epi: int, bias=None, aux=None) -> None:
        """out = epilogue(A B^T); A [M, K], B [N, K], out [M, N]: 2-D views with unit column stride."""
        M, K = A.shape
        N = B.shape[0]
        for t in (A, B, out) + ((aux,) if aux is not None else ()):
            if t.stride(1) != 1:
                raise ValueError("gemm operands need unit column stride")
        self._check(self.lib.mlp_gemm_bf16(_ptr(A), A.stride(0), _ptr(B), B.stride(0), M, N, K, epi, _ptr(out),
                                           out.stride(0), _ptr(bias) if bias is not None else None,
                                           _ptr(aux) if aux is not None else None,
                                           aux.stride(0) if aux is not None else 0, self._stream()))

    def gemm_split(self, A, Wsplit, out, bias) -> None:
        """out = A (W_hi + W_lo)^T + bias, fp32; Wsplit [N, 2K] holds [hi | lo]."""
        M, K = A.shape
        N = Wsplit.shape[0]
        if Wsplit.shape[1] != 2 * K or A.stride(1) != 1 or Wsplit.stride(1) != 1 or out.stride(1) != 1:
            raise ValueError("gemm_split: need A [M, K] and Wsplit [N, 2K] with unit column stride")
        self._check(self.lib.mlp_gemm_bf16_split(_ptr(A), A.stride(0), _ptr(Wsplit), Wsplit.stride(0), M, N, K,
                                                 EPI_BIAS_F32, _ptr(out), out.stride(0), _ptr(bias), self._stream()))

    def _build_split(self) -> None:
        t = self.torch
        W = self.W[self.layers]
        hi = W.to(t.bfloat16)
        lo = (W - hi.float()).to(t.bfloat16)
        self.Wsplit16 = t.cat([hi, lo], dim=1).contiguous()
        self._split_stale = False

    def set_output_layer(self, W, b) -> None:
        """Replace the output layer's first n_out rows (fp32 W [n_out, d_in],
        b [n_out]); refreshes the bf16 copies and the split weights."""
        L = self.layers
        self.W[L][: self.n_out].copy_(W)
        self.b[L][: self.n_out].copy_(b)
        self.W16[L].copy_(self.W[L].to(self.torch.bfloat16))
        self._refresh_transposes()
        self._build_split()

    def transpose(self, a, out) -> None:
        r, c = a.shape
        self._check(self.lib.mlp_transpose_bf16(_ptr(a), a.stride(0), _ptr(out), r, c, self._stream()))

    def _refresh_transposes(self) -> None:
        for i in range(1, self.layers + 1):
            self.transpose(self.W16[i], self.WT16[i])

    def buffers(self, B: int, slot: int = 0) -> dict:
        """Activation and gradient buffers for batch B; independent sets per
        slot let two inferences be in flight at once (HostPipeline)."""
        if B % 128:
            raise ValueError("batch must be a multiple of 128")
        key = (B, slot)
        if key not in self._bufs:
            t, d = self.torch, self.dev
            bf = t.bfloat16
            H, L = self.hidden, self.layers
            cat = t.zeros(B, self.cat_w if self.skip else H, dtype=bf, device=d)
            xbuf = cat[:, H:] if self.skip else t.zeros(B, self.k0, dtype=bf, device=d)
            acts = [t.empty(B, H, dtype=bf, device=d) for _ in range(L - 1)] + [cat[:, :H]]
            h = {"cat": cat, "x": xbuf, "a": acts,
                 "z": [t.empty(B, H, dtype=bf, device=d) for _ in range(L)],
                 "p": t.empty(B, self.no, device=d),
                 "gp": t.empty(B, self.no, dtype=bf, device=d),
                 "g": [t.empty(B, H, dtype=bf, device=d) for _ in range(2)],
                 "gT": t.empty(max(self.no, H), B, dtype=bf, device=d),
                 "actT": t.empty(max(self.dims_in), B, dtype=bf, device=d),
                 "gW": [t.empty(self.dims_out[i], self.dims_in[i], device=d) for i in range(L + 1)],
                 "gb": [t.empty(self.dims_out[i], device=d) for i in range(L + 1)],
                 "loss": t.zeros(1, device=d)}
            self._bufs[key] = h
        return self._bufs[key]

    def _layer_input(self, h: dict, i: int):
        if i == 0:
            return h["x"]
        if i == self.layers:
            return h["cat"] if self.skip else h["a"][-1]
        return h["a"][i - 1]

    # -- passes --
    def hidden_layers(self, h: dict, keep_pre: bool = True) -> None:
        """The GELU layers on the standardized features in h['x']; the output
        layer's input is then _layer_input(h, layers)."""
        for i in range(self.layers):
            self.gemm(self._layer_input(h, i), self.W16[i], h["a"][i], EPI_BIAS_GELU, bias=self.b[i],
                      aux=h["z"][i] if keep_pre else None)

    def forward(self, h: dict, keep_pre: bool = True):
        """Forward pass on the standardized features in h['x']; fp32 [B, no]
        outputs.  keep_pre=True (training) stores the GELU pre-activations
        the backward pass reads and uses the bf16 output weights the
        gradients are taken for; keep_pre=False (inference) stores none and
        evaluates the output layer with split weights when split_out is set."""
        self.hidden_layers(h, keep_pre)
        L = self.layers
        if not keep_pre and self.split_out:
            if self._split_stale:
                self._build_split()
            self.gemm_split(self._layer_input(h, L), self.Wsplit16, h["p"], self.b[L])
        else:
            self.gemm(self._layer_input(h, L), self.W16[L], h["p"], EPI_BIAS_F32, bias=self.b[L])
        return h["p"]

    def backward(self, h: dict, target) -> None:
        """Gradients of the mean-squared error against target (fp32 [B, n_out])
        into h['gW'] / h['gb']; the loss accumulates into h['loss']."""
        B = h["p"].shape[0]
        self._check(self.lib.mlp_mse_grad(_ptr(h["p"]), self.no, _ptr(target), self.n_out, B, _ptr(h["gp"]),
                                          _ptr(h["loss"]), self._stream()))
        g = h["gp"]
        H = self.hidden
        for i in range(self.layers, -1, -1):
            d_out, d_in = self.dims_out[i], self.dims_in[i]
            act = self._layer_input(h, i)
            gT = h["gT"][:d_out]
            actT = h["actT"][:d_in]
            self.transpose(g, gT)
            self.transpose(act, actT)
            self.gemm(gT, actT, h["gW"][i], EPI_F32)                    # dW = g^T act
            self._check(self.lib.mlp_col_sum_bf16(_ptr(g), B, d_out, _ptr(h["gb"][i]), self._stream()))
            if i > 0:
                gn = h["g"][i % 2]
                # (g W)[:, hidden part] * gelu'(z): the rows of W^T that multiply a_{i-1}
                self.gemm(g, self.WT16[i][:H], gn, EPI_DGELU, aux=h["z"][i - 1])
                g = gn

    def adam(self, h: dict, lr: float, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8,
             wd: float = 0.0) -> None:
        """One Adam step from the gradients in buffer set h; refreshes the bf16
        weights and their transposes."""
        self.step += 1
        for i in range(self.layers + 1):
            self._check(self.lib.mlp_adam(_ptr(self.W[i]), _ptr(h["gW"][i]), _ptr(self.mW[i]), _ptr(self.vW[i]),
                                          _ptr(self.W16[i]), self.W[i].numel(), lr, b1, b2, eps, self.step, wd,
                                          self._stream()))
            self._check(self.lib.mlp_adam(_ptr(self.b[i]), _ptr(h["gb"][i]), _ptr(self.mb[i]), _ptr(self.vb[i]),
                                          None, self.b[i].numel(), lr, b1, b2, eps, self.step, 0.0, self._stream()))
        self._refresh_transposes()

    def train_step(self, h: dict, target, lr: float) -> None:
        """Forward, backward and Adam on the features already standardized in h['x']."""
        self.forward(h)
        self.backward(h, target)
        self.adam(h, lr)

    def standardize(self, h: dict, raw, mean, inv_std) -> None:
        x = h["x"]
        self._check(self.lib.mlp_standardize(_ptr(raw), _ptr(mean), _ptr(inv_std), _ptr(x), x.stride(0),
                                             raw.shape[0], self.n_in, self.k0, self._stream()))

    def load_features(self, h: dict, sbus, sgen, extra, mean, inv_std) -> None:
        """Standardized features of Sbus (complex128 [B, n]) straight into h['x']
        (mlp_load_features: loads sgen - S, then the fixed extra inputs); the
        rows past B repeat the last scenario."""
        x = h["x"]
        if sbus.stride(1) != 1:
            sbus = sbus.contiguous()
        B, n = sbus.shape
        self._check(self.lib.mlp_load_features(_ptr(sbus), sbus.stride(0), _ptr(sgen), _ptr(extra), n, extra.numel(),
                                               _ptr(mean), _ptr(inv_std), _ptr(x), x.stride(0), B, x.shape[0],
                                               self.k0, self._stream()))

    def error_flag(self) -> int:
        v = C.c_int32(0)
        self._check(self.lib.mlp_error_flag(C.byref(v), 1))
        return v.value


def nominal_state(solver, grid, tol: float = 1e-10, max_iter: int = 20, device=None):
    """The converged state of the grid's nominal-load case (Sbus = grid.sbus,
    from its flat start), complex128 [n_bus] on the device.  Started from it,
    a scenario near nominal load needs fewer Newton steps than from the flat
    start: the model-free warm start for grids too large to train a network
    for.  Raises if the nominal case does not converge."""
    import torch

    import cupf

    dev = torch.device(device or "cuda")
    S = torch.tensor(grid.sbus[None, :], device=dev)
    V0 = torch.tensor(grid.v0[None, :], device=dev)
    V, fm, _ = solver.solve_batch_device(S, V0, config=cupf.NRConfig(tolerance=tol, max_iter=max_iter))
    if not bool((fm <= tol).all()):
        raise RuntimeError("warm start: the nominal-load case did not converge")
    return V[0].clone()


class WarmStart:
    """Warm-start predictor for one grid (features: P and Q loads at every bus
    and the PV setpoints; outputs: the Newton unknowns in Jacobian-row order)."""

    def __init__(self, grid, hidden: int = 1024, layers: int = 3, seed: int = 0, device=None, skip: bool = True):
        import torch

        self.torch = torch
        self.g = grid
        self.dev = torch.device(device or "cuda")
        self.n_pvpq = grid.pv.size + grid.pq.size
        self.n_in = 2 * grid.n_bus + grid.pv.size
        self.n_out = self.n_pvpq + grid.pq.size
        self.mlp = MLP(self.n_in, self.n_out, hidden, layers, seed, self.dev, skip=skip)
        self.pvpq = torch.tensor(np.concatenate([grid.pv, grid.pq]), dtype=torch.long, device=self.dev)
        self.pq = torch.tensor(grid.pq, dtype=torch.long, device=self.dev)
        self.vm_pv = torch.tensor(np.abs(grid.v0[grid.pv]), dtype=torch.float32, device=self.dev)
        self.sgen = torch.tensor(grid.sgen, device=self.dev)
        self.v0 = torch.tensor(grid.v0, device=self.dev)
        self.x_mean = self.x_istd = self.y_mean = self.y_std = None
        self.va_ref = None  # angles of the nominal-load solution: the unwrapping reference
        self.history: list[float] = []

    # -- data --
    def features(self, sbus):
        """Raw features fp32 [B, n_in] from Sbus (complex128 [B, n]): load = Sgen - Sbus."""
        t = self.torch
        load = self.sgen[None, :] - sbus
        B = sbus.shape[0]
        return t.cat([load.real.float(), load.imag.float(), self.vm_pv[None, :].expand(B, -1)], dim=1).contiguous()

    def targets(self, V):
        """Newton unknowns of solved states V [B, n]: Va at the PV+PQ buses and
        Vm at the PQ buses.  Bus angles on a large grid span more than 2 pi, so
        each angle is unwrapped to within pi of the nominal-load solution's
        (Newton only sees V = Vm e^{j Va}, so any 2 pi offset is harmless)."""
        t = self.torch
        va = t.angle(V)
        if self.va_ref is not None:
            va = self.va_ref[None, :] + t.remainder(va - self.va_ref[None, :] + math.pi, 2 * math.pi) - math.pi
        return t.cat([va[:, self.pvpq], t.abs(V)[:, self.pq]], dim=1).float().contiguous()

    def set_reference(self, solver, tol: float = 1e-10, max_iter: int = 20) -> None:
        """Solve the nominal-load case once; its angles anchor the unwrapping."""
        self.vref = nominal_state(solver, self.g, tol, max_iter, self.dev)
        self.va_ref = self.torch.angle(self.vref)

    def generate(self, solver, n: int, lo: float = 0.7, hi: float = 1.3, seed: int = 12345, tol: float = 1e-10,
                 max_iter: int = 20, chunk: int = 8192, keep_all: bool = False):
        """Solve n seeded scenarios with the engine; returns (features,
        targets, keep) as CUDA tensors.  keep marks the converged solutions on
        the regular branch (every PQ magnitude within 0.1 pu and every angle
        within 2.5 rad of the nominal-load solution); unless keep_all, only
        those rows are returned.  A heavily loaded scenario can converge to a
        far solution, which would only teach the network outliers."""
        import cupf

        t = self.torch
        cfg = cupf.NRConfig(tolerance=tol, max_iter=max_iter)
        if self.va_ref is None:
            self.set_reference(solver, tol, max_iter)
        ref = self.targets(self.vref[None, :])[0]
        rng = np.random.default_rng(seed)
        xs, ys, ks = [], [], []
        for c0 in range(0, n, chunk):
            m = min(chunk, n - c0)
            f = rng.uniform(lo, hi, size=(m, self.g.n_bus))
            S = t.tensor(self.g.sgen[None, :] - f * self.g.sload[None, :], device=self.dev)
            V, fm, _ = solver.solve_batch_device(S, self.v0[None, :].expand(m, -1).contiguous(), config=cfg)
            y = self.targets(V)
            dev = (y - ref[None, :]).abs()
            keep = (fm <= tol) & (dev[:, : self.n_pvpq].amax(1) <= 2.5) & (dev[:, self.n_pvpq:].amax(1) <= 0.1)
            x = self.features(S)
            if not keep_all:
                x, y = x[keep], y[keep]
            xs.append(x)
            ys.append(y)
            ks.append(keep)
        return t.cat(xs), t.cat(ys), t.cat(ks)

    # -- training --
    def fit(self, X, Y, epochs: int = 10, batch: int = 1024, lr: float = 1e-3, lr_min: float = 1e-5,
            seed: int = 0, log=None, refit: bool = True):
        """Adam on the mean-squared error of the standardized targets (cosine
        learning rate from lr to lr_min), then, with refit, the output layer
        solved in closed form on the trained hidden features
        (refit_output)."""
        t = self.torch
        self.x_mean = X.mean(0)
        self.x_istd = 1.0 / X.std(0).clamp_min(1e-6)
        self.y_mean = Y.mean(0)
        self.y_std = Y.std(0).clamp_min(1e-9)
        Yn = ((Y - self.y_mean) / self.y_std).contiguous()
        n = X.shape[0] // batch * batch
        steps = epochs * (n // batch)
        h = self.mlp.buffers(batch)
        gen = t.Generator(device=self.dev).manual_seed(seed)
        s = 0
        t0 = time.perf_counter()
        for ep in range(epochs):
            perm = t.randperm(X.shape[0], generator=gen, device=self.dev)[:n]
            h["loss"].zero_()
            for k in range(0, n, batch):
                idx = perm[k:k + batch]
                self.mlp.standardize(h, X[idx].contiguous(), self.x_mean, self.x_istd)
                lr_s = lr_min + 0.5 * (lr - lr_min) * (1 + math.cos(math.pi * s / max(1, steps)))
                self.mlp.train_step(h, Yn[idx].contiguous(), lr_s)
                s += 1
            loss = float(h["loss"].item()) / (n // batch)
            self.history.append(loss)
            if not math.isfinite(loss):
                raise RuntimeError(f"warm-start training diverged at epoch {ep}")
            if log:
                log(f"epoch {ep}: loss {loss:.3e} ({time.perf_counter() - t0:.1f} s)")
        if self.mlp.error_flag():
            raise RuntimeError("warm-start GEMM reported a wait timeout")
        if refit:
            self.refit_output(X, Y)
        return self.history

    def refit_output(self, X, Y, ridge: float = 1e-6, chunk: int = 8192) -> None:
        """Least-squares output layer on the trained hidden features.

        The hidden layers (the project's kernels, bf16) map every training
        row to the output layer's input a = [a_L | x]; the output layer is
        then the ridge solution of min ||[a 1] [W^T; b] - Y_std||^2.  The
        normal equations are accumulated in FP64 by the project's Gram
        kernel chunk by chunk (mlp_gram_f64) and solved by its blocked
        Cholesky (mlp_cholesky_solve_f64), ridge = ridge x the mean diagonal.
        Adam's stochastic steps leave independent per-output noise in W that
        the exact minimiser does not have; set_output_layer installs the
        result as split weights for inference."""
        t = self.torch
        mlp = self.mlp
        if self.y_mean is None:
            raise RuntimeError("refit_output: fit the network first")
        L = mlp.layers
        h = mlp.buffers(chunk)
        n = X.shape[0]
        p = mlp.dims_in[L]
        D = p + 1
        q = self.n_out
        AtA = t.zeros(D, D, dtype=t.float64, device=self.dev)
        AtY = t.zeros(D, q, dtype=t.float64, device=self.dev)
        stream = mlp._stream()
        lib = mlp.lib
        for c0 in range(0, n, chunk):
            m = min(chunk, n - c0)
            xb = X[c0:c0 + m]
            if m < chunk:
                xb = t.cat([xb, xb[-1:].expand(chunk - m, -1)])
            mlp.standardize(h, xb.contiguous(), self.x_mean, self.x_istd)
            mlp.hidden_layers(h, keep_pre=False)
            A = mlp._layer_input(h, L)
            Ys = ((Y[c0:c0 + m] - self.y_mean) / self.y_std).float().contiguous()
            rc = lib.mlp_gram_f64(_ptr(A), A.stride(0), 0, _ptr(Ys), Ys.stride(0), 0, m, p, q, _ptr(AtA),
                                  AtA.stride(0), _ptr(AtY), AtY.stride(0), stream)
            if rc:
                raise RuntimeError("refit_output: " + lib.mlp_refit_last_error().decode())
        if mlp.error_flag():
            raise RuntimeError("warm-start GEMM reported a wait timeout")
        info = t.zeros(1, dtype=t.int32, device=self.dev)
        rc = lib.mlp_cholesky_solve_f64(_ptr(AtA), AtA.stride(0), D, _ptr(AtY), AtY.stride(0), q, ridge, _ptr(info),
                                        stream)
        if rc:
            raise RuntimeError("refit_output: " + lib.mlp_refit_last_error().decode())
        if int(info.item()) != 0:
            raise RuntimeError(f"refit_output: the normal equations are not positive definite "
                               f"(pivot {int(info.item()) - 1})")
        sol = AtY
        if not bool(t.isfinite(sol).all()):
            raise RuntimeError("refit_output: the least-squares solve is not finite")
        mlp.set_output_layer(sol[:-1].T.float(), sol[-1].float())

    # -- checkpoints --
    def save(self, path) -> None:
        """Write the trained predictor to an .npz file: the network's FP32
        weights and biases, the input and output standardization, the
        unwrapping reference and the grid's shape (checked on load).  The bf16
        copies, transposes and split output weights are rebuilt on load."""
        if self.y_mean is None:
            raise RuntimeError("WarmStart.save: fit the network first")
        m = self.mlp
        arrays = {f"W{i}": m.W[i].cpu().numpy() for i in range(m.layers + 1)}
        arrays.update({f"b{i}": m.b[i].cpu().numpy() for i in range(m.layers + 1)})
        for k in ("x_mean", "x_istd", "y_mean", "y_std", "va_ref"):
            arrays[k] = getattr(self, k).cpu().numpy()
        arrays["vref"] = self.vref.cpu().numpy()
        arrays["shape"] = np.array([self.g.n_bus, self.g.pv.size, self.g.pq.size, self.n_in, self.n_out, m.hidden,
                                    m.layers, int(m.skip)], dtype=np.int64)
        np.savez(path, **arrays)

    def load(self, path) -> None:
        """Restore a predictor written by save() for this grid and network
        shape (ValueError when they differ); ready for predict/solve."""
        t = self.torch
        d = np.load(path)
        m = self.mlp
        want = np.array([self.g.n_bus, self.g.pv.size, self.g.pq.size, self.n_in, self.n_out, m.hidden, m.layers,
                         int(m.skip)], dtype=np.int64)
        if not np.array_equal(d["shape"], want):
            raise ValueError(f"WarmStart.load: checkpoint shape {d['shape'].tolist()} does not match "
                             f"this grid and network {want.tolist()}")
        for i in range(m.layers + 1):
            m.W[i].copy_(t.from_numpy(d[f"W{i}"]))
            m.b[i].copy_(t.from_numpy(d[f"b{i}"]))
            m.W16[i].copy_(m.W[i].to(t.bfloat16))
        m._refresh_transposes()
        m._build_split()
        for k in ("x_mean", "x_istd", "y_mean", "y_std", "va_ref"):
            setattr(self, k, t.from_numpy(d[k]).to(self.dev))
        self.vref = t.from_numpy(d["vref"]).to(self.dev)

    # -- inference --
    def predict_standardized(self, sbus, slot: int = 0):
        """Network output fp32 [B rounded up to 128, no], still standardized
        (state = out * y_std + y_mean on the first n_out columns): the
        features are built from Sbus by one kernel and no pre-activations
        are kept.  The output lives in the buffers of `slot` until the next
        prediction into that slot."""
        Bp = _round_up(sbus.shape[0], 128)
        h = self.mlp.buffers(Bp, slot)
        self.mlp.load_features(h, sbus, self.sgen, self.vm_pv, self.x_mean, self.x_istd)
        return self.mlp.forward(h, keep_pre=False)

    def predict(self, sbus):
        """Predicted Newton unknowns fp32 [B, n_out]."""
        B = sbus.shape[0]
        out = self.predict_standardized(sbus)
        return (out[:B, : self.n_out] * self.y_std + self.y_mean).contiguous()

    def solve(self, solver, sbus, config=None, pred=None):
        """Warm-started batched solve with flat-start fallback.  Returns
        (V, final_mismatch, iterations_warm, n_fallback).  pred: this batch's
        predict_standardized output when it was computed beforehand (on
        another stream, ordered before this call's stream)."""
        import cupf

        cfg = config or cupf.NRConfig()
        if pred is None:
            pred = self.predict_standardized(sbus)
        V, fm, it = solver.solve_batch_warm_device(sbus, self.v0, pred, config=cfg, pred_scale=self.y_std,
                                                   pred_shift=self.y_mean)
        if solver.last_all_converged:  # known from the solve itself: no extra synchronisation
            return V, fm, it, 0
        # (a non-finite prediction only makes its scenario fail and fall back)
        bad = (fm > cfg.tolerance).nonzero().flatten()
        nb = int(bad.numel())
        if nb:
            Sb = sbus[bad].contiguous()
            Vb, fmb, _ = solver.solve_batch_device(Sb, self.v0[None, :].expand(nb, -1).contiguous(), config=cfg)
            V[bad] = Vb
            fm[bad] = fmb
        return V, fm, it, nb
