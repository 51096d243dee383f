"""Warm-start network kernels (include/cupf_mlp.h) on the GPU: the tcgen05
GEMM and its epilogues against torch fp32 products, a full training step's
gradients against the CPU oracle (oracle/mlp_oracle.py), training
convergence, and the warm start's iteration savings on a real grid."""
import numpy as np
import pytest

from conftest import gpu_available, max_dv_vs_oracle

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]


@pytest.fixture(scope="module")
def torch():
    import torch
    return torch


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


# 128 x 64 tiles below 148 tiles of 128 x 128; 128 x 224 tiles when those fill
# 80-100 % of the SMs in one wave (1024 x 3712: 8 x 17 tiles, the last column
# tile partial); else 128 x 128 tiles two per SM
@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (256, 384, 1024), (384, 128, 4480), (1280, 2048, 320),
                                   (1024, 3712, 1024)])
def test_gemm_f32_matches_torch(torch, M, N, K):
    from cupf.warm_start import MLP, EPI_F32, EPI_BIAS_F32

    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    bias = torch.randn(N, device="cuda", generator=g)
    net = MLP(64, 64, hidden=128, layers=1)
    out = torch.empty(M, N, device="cuda")
    net.gemm(A, B, out, EPI_F32)
    ref = A.float() @ B.float().T
    assert _rel(out.cpu().numpy(), ref.cpu().numpy()) < 1e-5
    net.gemm(A, B, out, EPI_BIAS_F32, bias=bias)
    assert _rel(out.cpu().numpy(), (ref + bias).cpu().numpy()) < 1e-5
    assert net.error_flag() == 0


@pytest.mark.parametrize("M,N,K", [(128, 128, 256), (1280, 2048, 320), (1024, 3712, 320)])
def test_gemm_wait_timeout_reports_and_recovers(torch, M, N, K):
    """The GEMM's bounded waits, made to run out on the host's request (the
    producer issues no tile loads, the wait limit is 1,000 polls): the kernel
    returns, raises the error flag and marks its outputs NaN; the context
    stays usable, and the next GEMM with the normal limit is exact again."""
    from cupf.warm_start import MLP, EPI_F32

    g = torch.Generator(device="cuda").manual_seed(7)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    net = MLP(64, 64, hidden=128, layers=1)
    lib = net.lib
    out = torch.zeros(M, N, device="cuda")
    assert net.error_flag() == 0
    assert lib.mlp_set_wait_test(1000, 1) == 0
    try:
        net.gemm(A, B, out, EPI_F32)
        torch.cuda.synchronize()
    finally:
        assert lib.mlp_set_wait_test(1 << 22, 0) == 0
    assert net.error_flag() == 1  # read and reset
    assert bool(torch.isnan(out).all())
    net.gemm(A, B, out, EPI_F32)
    ref = A.float() @ B.float().T
    assert _rel(out.cpu().numpy(), ref.cpu().numpy()) < 1e-5
    assert net.error_flag() == 0
    assert lib.mlp_set_wait_test(0, 0) == 1  # a limit must be positive


def test_gemm_gelu_epilogues(torch):
    from cupf.warm_start import MLP, EPI_BIAS_GELU, EPI_DGELU
    from oracle.mlp_oracle import gelu, gelu_grad

    M, N, K = 256, 256, 512
    g = torch.Generator(device="cuda").manual_seed(7)
    A = (0.1 * torch.randn(M, K, device="cuda", generator=g)).to(torch.bfloat16)
    B = (0.1 * torch.randn(N, K, device="cuda", generator=g)).to(torch.bfloat16)
    bias = 0.1 * torch.randn(N, device="cuda", generator=g)
    net = MLP(64, 64, hidden=128, layers=1)
    out = torch.empty(M, N, dtype=torch.bfloat16, device="cuda")
    aux = torch.empty(M, N, dtype=torch.bfloat16, device="cuda")
    net.gemm(A, B, out, EPI_BIAS_GELU, bias=bias, aux=aux)
    z = (A.double() @ B.double().T + bias.double()).cpu().numpy()
    assert np.abs(aux.float().cpu().numpy() - z).max() <= 1e-2 * np.abs(z).max()
    assert np.abs(out.float().cpu().numpy() - gelu(z)).max() <= 1e-2 * np.abs(gelu(z)).max()
    out2 = torch.empty(M, N, dtype=torch.bfloat16, device="cuda")
    net.gemm(A, B, out2, EPI_DGELU, aux=aux)
    acc = (A.double() @ B.double().T).cpu().numpy()
    ref = acc * gelu_grad(aux.double().cpu().numpy())
    assert np.abs(out2.float().cpu().numpy() - ref).max() <= 1e-2 * np.abs(ref).max()


@pytest.mark.parametrize("skip", [False, True])
def test_training_step_gradients_match_oracle(torch, skip):
    """One forward + backward of a 2-hidden-layer network: every weight and
    bias gradient against the CPU oracle (same bf16 rounding points)."""
    from cupf.warm_start import MLP
    from oracle import mlp_oracle as mo

    n_in, n_out, B = 200, 150, 128
    net = MLP(n_in, n_out, hidden=256, layers=2, seed=3, skip=skip)
    rng = np.random.default_rng(0)
    x = np.zeros((B, net.k0))
    x[:, :n_in] = rng.standard_normal((B, n_in))
    x = mo.bf16(x)
    y = rng.standard_normal((B, n_out))
    h = net.buffers(B)
    h["x"].copy_(torch.tensor(x, dtype=torch.float32, device="cuda").to(torch.bfloat16))
    yt = torch.tensor(y, dtype=torch.float32, device="cuda")
    for i in range(len(net.b)):
        net.b[i].copy_(0.05 * torch.randn(net.b[i].shape, device="cuda"))
    net.forward(h)
    h["loss"].zero_()
    net.backward(h, yt)
    Ws = [w16.double().cpu().numpy() for w16 in net.W16]
    bs = [b.double().cpu().numpy() for b in net.b]
    p, loss, dWs, dbs = mo.forward_backward(x, Ws, bs, y, n_out, skip=skip)
    assert _rel(h["p"].cpu().numpy(), p) < 1e-3
    assert abs(float(h["loss"].item()) - loss) <= 1e-3 * loss
    for i in range(len(dWs)):
        assert _rel(h["gW"][i].cpu().numpy(), dWs[i]) < 2e-2, i
        assert _rel(h["gb"][i].cpu().numpy(), dbs[i]) < 2e-2, i
    assert net.error_flag() == 0


def test_training_reduces_loss(torch):
    from cupf.warm_start import MLP

    n_in, n_out, B = 128, 64, 256
    net = MLP(n_in, n_out, hidden=256, layers=2, seed=1)
    g = torch.Generator(device="cuda").manual_seed(5)
    T = torch.randn(n_out, n_in, device="cuda", generator=g) / n_in ** 0.5
    X = torch.randn(B * 8, n_in, device="cuda", generator=g)
    Y = torch.tanh(X @ T.T)
    h = net.buffers(B)
    losses = []
    for step in range(300):
        k = (step % 8) * B
        h["x"][:, :n_in] = X[k:k + B].to(torch.bfloat16)
        h["loss"].zero_()
        net.train_step(h, Y[k:k + B].contiguous(), 2e-3)
        losses.append(float(h["loss"].item()))
    assert np.mean(losses[-20:]) < 0.1 * np.mean(losses[:5])


def test_warm_start_saves_newton_iterations(torch, oracle):
    """Trained on engine solutions of a 118-bus grid (load scaling 0.7-1.3),
    the network's starting point needs fewer Newton iterations than the flat
    start on held-out scenarios, and every scenario from either start lies
    within 1e-8 of the FP64 oracle solved to 1e-12."""
    import cupf
    from cupf import grids as G
    from cupf.warm_start import WarmStart

    g = G.grid_118()
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    o.compute = cupf.ComputePolicy.Mixed
    o.custom.serial_nd = True
    s = cupf.NewtonSolver(o)
    s.initialize(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, g.pv, g.pq)
    ws = WarmStart(g, hidden=256, layers=2, seed=0)
    X, Y, _ = ws.generate(s, 16384, seed=1)
    ws.fit(X, Y, epochs=40, batch=512, lr=2e-3)
    rng = np.random.default_rng(99)
    f = rng.uniform(0.7, 1.3, size=(512, g.n_bus))
    S = torch.tensor(g.sgen[None, :] - f * g.sload[None, :], device="cuda")
    cfg = cupf.NRConfig(tolerance=1e-8, max_iter=10)
    Vf, fmf, itf = s.solve_batch_device(S, ws.v0[None, :].expand(512, -1).contiguous(), config=cfg)
    Vw, fmw, itw, nfb = ws.solve(s, S, cfg)
    assert bool((fmw <= 1e-8).all()) and bool((fmf <= 1e-8).all())
    assert itw < itf, (itw, itf)
    V0 = np.repeat(g.v0[None, :], 512, axis=0)
    for V in (Vw, Vf):
        dv = max_dv_vs_oracle(oracle, g, S.cpu().numpy(), V0, V.cpu().numpy())
        assert dv.max() <= 1e-8, float(dv.max())


def test_warm_start_2000_full_batch_matches_oracle(torch, oracle):
    """The headline configuration's warm start: the bench's network shape
    (loads and PV setpoints -> 3 x 1,024 GELU -> 3,598, input skip, output
    layer refit and evaluated with split weights), trained here on a smaller
    set (16,384 engine-solved scenarios, 12 epochs), then run on the full
    1,024-scenario U(0.8, 1.2) batch of the 2,000-bus grid.  Every scenario
    converges to 1e-8 and lies within 1e-8 of the FP64 oracle, and the warm
    start needs fewer Newton iterations than the flat start."""
    import cupf
    from cupf import grids as G
    from cupf.warm_start import WarmStart

    g = G.grid_2000()
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    o.compute = cupf.ComputePolicy.Mixed
    o.custom.serial_nd = True
    o.use_cuda_graph = True
    s = cupf.NewtonSolver(o)
    s.initialize(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, g.pv, g.pq)
    ws = WarmStart(g, hidden=1024, layers=3, seed=0)
    X, Y, _ = ws.generate(s, 16384, lo=0.7, hi=1.3, seed=777)
    ws.fit(X, Y, epochs=12, batch=1024, lr=2e-3)
    B = 1024
    S_h = g.scenarios(B, seed=9100)
    S = torch.tensor(S_h, device="cuda")
    cfg = cupf.NRConfig(tolerance=1e-8, max_iter=10)
    Vw, fmw, itw, nfb = ws.solve(s, S, cfg)
    V0 = g.flat_start(B)
    Vf, fmf, itf = s.solve_batch_device(S, torch.tensor(V0, device="cuda"), config=cfg)
    assert bool((fmw <= 1e-8).all()) and bool((fmf <= 1e-8).all())
    assert itw < itf, (itw, itf)
    dv = max_dv_vs_oracle(oracle, g, S_h, V0, Vw.cpu().numpy())
    assert dv.size == B and dv.max() <= 1e-8, (int(dv.argmax()), float(dv.max()))


def test_warm_entry_point_exact_prediction_and_failed_row(torch):
    """pf_solve_batch_warm_device: seeded with the exact solution a scenario
    converges at the first norm evaluation; a non-finite prediction only fails
    its own scenario (final mismatch inf), the rest of the batch converges."""
    import cupf
    from cupf import grids as G

    g = G.grid_118()
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    o.compute = cupf.ComputePolicy.FP64
    o.custom.serial_nd = True
    s = cupf.NewtonSolver(o)
    s.initialize(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, g.pv, g.pq)
    B = 40
    S = torch.tensor(g.scenarios(B, seed=4), device="cuda")
    v0 = torch.tensor(g.v0, device="cuda")
    cfg = cupf.NRConfig(tolerance=1e-10, max_iter=20)
    V, fm, it = s.solve_batch_device(S, v0[None, :].expand(B, -1).contiguous(), config=cfg)
    assert bool((fm <= 1e-10).all())
    pvpq = torch.tensor(np.concatenate([g.pv, g.pq]), device="cuda")
    pq = torch.tensor(g.pq, device="cuda")
    pred = torch.cat([torch.angle(V)[:, pvpq], torch.abs(V)[:, pq]], 1).float().contiguous()
    cfg8 = cupf.NRConfig(tolerance=1e-5, max_iter=10)
    Vw, fmw, itw = s.solve_batch_warm_device(S, v0, pred, config=cfg8)
    assert itw == 1 and bool((fmw <= 1e-5).all())
    # the same prediction given standardized, with its scale and shift
    mean, std = pred.mean(0), pred.std(0).clamp_min(1e-6)
    z = ((pred - mean) / std).contiguous()
    Vz, fmz, itz = s.solve_batch_warm_device(S, v0, z, config=cfg8, pred_scale=std.contiguous(),
                                            pred_shift=mean.contiguous())
    assert itz == 1 and bool((fmz <= 1e-5).all()) and s.last_all_converged
    pred[3, 5] = float("nan")
    Vw, fmw, itw = s.solve_batch_warm_device(S, v0, pred, config=cfg8)
    assert np.isinf(fmw[3].item())
    assert not s.last_all_converged  # a failed scenario is never reported as converged
    ok = torch.ones(B, dtype=torch.bool, device="cuda")
    ok[3] = False
    assert bool((fmw[ok] <= 1e-5).all())


def test_load_features_match_the_torch_features(torch):
    """mlp_load_features builds, from Sbus, exactly the standardized bf16
    inputs that the torch feature path plus mlp_standardize produce."""
    from cupf import grids as G
    from cupf.warm_start import WarmStart

    g = G.grid_118()
    ws = WarmStart(g, hidden=128, layers=1, seed=0)
    B = 100  # padded to 128 inside; the padding rows repeat the last scenario
    S = torch.tensor(g.scenarios(B, seed=7), device="cuda")
    raw = ws.features(S)
    ws.x_mean = raw.mean(0)
    ws.x_istd = 1.0 / raw.std(0).clamp_min(1e-6)
    h = ws.mlp.buffers(128)
    ref = torch.cat([raw, raw[-1:].expand(28, -1)]).contiguous()
    ws.mlp.standardize(h, ref, ws.x_mean, ws.x_istd)
    a = h["x"].clone()
    h["x"].zero_()
    ws.mlp.load_features(h, S, ws.sgen, ws.vm_pv, ws.x_mean, ws.x_istd)
    assert torch.equal(h["x"], a)


def test_device_entry_points_follow_the_callers_stream(torch):
    """The prediction is written by work still queued on torch's default stream
    (behind a GPU sleep) when the warm solve is called: the engine must run on
    that same stream (handle 0 = legacy default stream), not on a private one."""
    import cupf
    from cupf import grids as G

    g = G.grid_118()
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    o.compute = cupf.ComputePolicy.Mixed
    o.custom.serial_nd = True
    s = cupf.NewtonSolver(o)
    s.initialize(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, g.pv, g.pq)
    B = 64
    S = torch.tensor(g.scenarios(B, seed=8), device="cuda")
    v0 = torch.tensor(g.v0, device="cuda")
    V, fm, _ = s.solve_batch_device(S, v0[None, :].expand(B, -1).contiguous(),
                                    config=cupf.NRConfig(tolerance=1e-11, max_iter=20))
    pvpq = torch.tensor(np.concatenate([g.pv, g.pq]), device="cuda")
    pq = torch.tensor(g.pq, device="cuda")
    exact = torch.cat([torch.angle(V)[:, pvpq], torch.abs(V)[:, pq]], 1).float().contiguous()
    pred = torch.full_like(exact, float("nan"))
    torch.cuda.synchronize()
    assert torch.cuda.current_stream().cuda_stream == 0
    torch.cuda._sleep(20_000_000)  # keep the default stream busy
    pred.copy_(exact)              # queued behind the sleep
    Vw, fmw, itw = s.solve_batch_warm_device(S, v0, pred, config=cupf.NRConfig(tolerance=1e-6, max_iter=10))
    assert bool((fmw <= 1e-6).all()) and itw <= 2


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (256, 384, 5504), (1024, 3712, 1024), (1024, 3712, 5504)])
def test_split_gemm_carries_the_fp32_weights(torch, M, N, K):
    """mlp_gemm_bf16_split: A (W_hi + W_lo)^T + bias within fp32 accumulation
    of the fp64 product with the fp32 weights, where the bf16 weights alone
    are off by their rounding."""
    import ctypes as C
    from cupf.warm_start import MLP, EPI_BIAS_F32, EPI_BIAS_GELU, _ptr

    g = torch.Generator(device="cuda").manual_seed(M + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    W = torch.randn(N, K, device="cuda", generator=g) / K ** 0.5
    bias = torch.randn(N, device="cuda", generator=g)
    hi = W.to(torch.bfloat16)
    Ws = torch.cat([hi, (W - hi.float()).to(torch.bfloat16)], 1).contiguous()
    net = MLP(64, 64, hidden=128, layers=1)
    out = torch.empty(M, N, device="cuda")
    net.gemm_split(A, Ws, out, bias)
    ref = (A.double() @ W.double().T + bias.double()).cpu().numpy()
    err_split = _rel(out.cpu().numpy(), ref)
    net.gemm(A, hi, out, EPI_BIAS_F32, bias=bias)
    err_bf16 = _rel(out.cpu().numpy(), ref)
    # hi + lo carries W to within 2^-16 relative per weight (about 5e-6 rms)
    assert err_split < 3e-5 and err_bf16 > 30 * err_split, (err_split, err_bf16)
    assert net.error_flag() == 0
    rc = net.lib.mlp_gemm_bf16_split(_ptr(A), K, _ptr(Ws), 2 * K, M, N, K, EPI_BIAS_GELU, _ptr(out), N, _ptr(bias),
                                     C.c_void_p(0))
    assert rc != 0 and b"fp32 epilogues" in net.lib.mlp_last_error()


@pytest.mark.parametrize("a_type", [0, 1])
def test_gram_kernel_matches_numpy(torch, a_type):
    """mlp_gram_f64: [A|1]^T [A|1] (upper triangle) and [A|1]^T Y accumulated
    in FP64 from bf16 (or fp32) A and fp32 Y, sizes off the 128 tiles, added
    to what the outputs hold; against numpy in FP64 on the same values."""
    from cupf import _capi

    lib = _capi.load()
    rng = np.random.default_rng(21)
    n, p, q = 1000, 300, 77
    dt = torch.bfloat16 if a_type == 0 else torch.float32
    A = torch.tensor(rng.standard_normal((n, p + 5)), dtype=torch.float32, device="cuda").to(dt)
    Y = torch.tensor(rng.standard_normal((n, q)), dtype=torch.float32, device="cuda")
    AtA = torch.full((p + 1, p + 1), 2.0, dtype=torch.float64, device="cuda")
    AtY = torch.full((p + 1, q), -1.0, dtype=torch.float64, device="cuda")
    ptr = lambda t: t.data_ptr()  # noqa: E731
    assert lib.mlp_gram_f64(ptr(A), A.stride(0), a_type, ptr(Y), Y.stride(0), 0, n, p, q, ptr(AtA), AtA.stride(0),
                            ptr(AtY), AtY.stride(0), None) == 0
    Ah = np.hstack([A[:, :p].double().cpu().numpy(), np.ones((n, 1))])
    ref = Ah.T @ Ah + 2.0
    got = AtA.cpu().numpy()
    iu = np.triu_indices(p + 1)
    assert np.abs(got[iu] - ref[iu]).max() <= 1e-12 * np.abs(ref).max()
    assert (got[np.tril_indices(p + 1, -1)] == 2.0).all()  # the lower triangle is left alone
    refy = Ah.T @ Y.double().cpu().numpy() - 1.0
    assert np.abs(AtY.cpu().numpy() - refy).max() <= 1e-12 * np.abs(refy).max()


@pytest.mark.parametrize("D,q", [(300, 77), (64, 1), (129, 200)])
def test_cholesky_solve_matches_numpy(torch, D, q):
    """mlp_cholesky_solve_f64: (M + ridge) X = R for an SPD M given by its
    upper triangle (64-column panels, a ragged last panel), against numpy;
    a matrix that is not positive definite reports its pivot."""
    from cupf import _capi

    lib = _capi.load()
    rng = np.random.default_rng(D + q)
    G = rng.standard_normal((D + 20, D))
    M = G.T @ G
    R = rng.standard_normal((D, q))
    Md = torch.tensor(np.triu(M) + np.tril(np.full((D, D), 7.0), -1), dtype=torch.float64, device="cuda")
    Rd = torch.tensor(R, dtype=torch.float64, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    ridge = 1e-6
    assert lib.mlp_cholesky_solve_f64(Md.data_ptr(), Md.stride(0), D, Rd.data_ptr(), Rd.stride(0), q, ridge,
                                      info.data_ptr(), None) == 0
    assert int(info.item()) == 0
    d = np.diag(M)
    Mr = M + np.eye(D) * ridge * d[d > 0].mean()
    X = np.linalg.solve(Mr, R)
    assert np.abs(Rd.cpu().numpy() - X).max() <= 1e-9 * np.abs(X).max()
    bad = torch.tensor(np.triu(M) - np.eye(D) * (2 * np.abs(M).sum()), dtype=torch.float64, device="cuda")
    Rd = torch.tensor(R, dtype=torch.float64, device="cuda")
    assert lib.mlp_cholesky_solve_f64(bad.data_ptr(), bad.stride(0), D, Rd.data_ptr(), Rd.stride(0), q, 0.0,
                                      info.data_ptr(), None) == 0
    assert int(info.item()) == 1  # the first pivot is already negative


def test_refit_output_solves_the_least_squares_problem(torch):
    """refit_output: the output layer equals the FP64 ridge solution on the
    hidden features the network's own kernels compute (the project's Gram
    and Cholesky kernels against numpy), lowers the training error, and
    inference evaluates it through the split weights."""
    import cupf
    from cupf import grids as G
    from cupf.warm_start import WarmStart

    g = G.grid_118()
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    o.compute = cupf.ComputePolicy.Mixed
    o.custom.serial_nd = True
    s = cupf.NewtonSolver(o)
    s.initialize(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, g.pv, g.pq)
    ws = WarmStart(g, hidden=128, layers=2, seed=0)
    X, Y, _ = ws.generate(s, 3000, seed=5)
    ws.fit(X, Y, epochs=5, batch=512, lr=2e-3, refit=False)
    net, L = ws.mlp, ws.mlp.layers
    n = X.shape[0]
    Bp = (n + 127) // 128 * 128
    h = net.buffers(Bp)
    net.standardize(h, torch.cat([X, X[-1:].expand(Bp - n, -1)]).contiguous(), ws.x_mean, ws.x_istd)
    net.hidden_layers(h, keep_pre=False)
    A = np.hstack([net._layer_input(h, L)[:n].double().cpu().numpy(), np.ones((n, 1))])
    T = ((Y - ws.y_mean) / ws.y_std).double().cpu().numpy()
    AtA = A.T @ A
    d = np.diag(AtA)
    AtA[np.diag_indices_from(AtA)] += 1e-6 * d[d > 0].mean()
    sol = np.linalg.solve(AtA, A.T @ T)
    before = float(((net.forward(h)[:n, : ws.n_out].double().cpu().numpy() - T) ** 2).mean())
    ws.refit_output(X, Y)
    Wr = net.W[L][: ws.n_out].double().cpu().numpy()
    assert np.abs(Wr - sol[:-1].T).max() <= 1e-5 * np.abs(sol).max()
    assert np.abs(net.b[L][: ws.n_out].double().cpu().numpy() - sol[-1]).max() <= 1e-5 * np.abs(sol).max()
    p = net.forward(h, keep_pre=False)[:n, : ws.n_out].double().cpu().numpy()
    exact = A @ sol
    # split weights: within 2^-16 |w| per weight; a 4x margin for fp32 rounding
    assert (np.abs(p - exact) <= 2.0 ** -14 * (np.abs(A) @ np.abs(sol)) + 1e-6).all()
    assert float(((p - T) ** 2).mean()) < before



def test_host_pipeline_matches_serial_solves(torch):
    """cupf.streaming.HostPipeline: batches of different sizes from pinned
    host memory, uploads and downloads overlapped with the solves, give the
    results of solving each batch alone, bit for bit; a shared output buffer
    ends with the last batch's results."""
    import cupf
    from cupf import grids as G
    from cupf.streaming import HostPipeline

    g = G.grid_118()
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    o.compute = cupf.ComputePolicy.Mixed
    o.use_cuda_graph = True
    o.custom.serial_nd = True
    s = cupf.NewtonSolver(o)
    s.initialize(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, g.pv, g.pq)
    cfg = cupf.NRConfig(tolerance=1e-8, max_iter=10)
    v0 = torch.tensor(g.v0, device="cuda")
    sizes = [64, 33, 64, 7, 100]
    ins = [torch.tensor(g.scenarios(b, seed=40 + i)).pin_memory() for i, b in enumerate(sizes)]

    def solve(s_dev):
        v, fm, _ = s.solve_batch_device(s_dev, v0[None, :].expand(s_dev.shape[0], -1).contiguous(), config=cfg)
        return v, fm

    V_out = [torch.empty(b, g.n_bus, dtype=torch.complex128).pin_memory() for b in sizes]
    fm_out = [torch.empty(b, dtype=torch.float64).pin_memory() for b in sizes]
    HostPipeline(solve).run(ins, V_out, fm_out)
    for i, b in enumerate(sizes):
        v, fm = solve(ins[i].cuda())
        assert torch.equal(V_out[i], v.cpu()) and torch.equal(fm_out[i], fm.cpu())
        assert bool((fm_out[i] <= 1e-8).all())
    shared = torch.empty(64, g.n_bus, dtype=torch.complex128).pin_memory()
    fms = [torch.empty(64, dtype=torch.float64).pin_memory() for _ in range(3)]
    HostPipeline(solve).run([ins[0], ins[2], ins[0]], [shared] * 3, fms)
    assert torch.equal(shared, V_out[0])


@pytest.mark.parametrize("lanes", [2, 3])
def test_host_pipeline_with_concurrent_solve_lanes(torch, lanes):
    """HostPipeline with several solve lanes (one solver handle, stream and
    worker thread each; batches round-robin): every batch's results equal the
    batch solved alone, bit for bit, in batch order, whatever the lane."""
    import cupf
    from cupf import grids as G
    from cupf.streaming import HostPipeline

    g = G.grid_500()
    cfg = cupf.NRConfig(tolerance=1e-8, max_iter=10)
    v0 = torch.tensor(g.v0, device="cuda")
    solvers = []
    for _ in range(lanes):
        o = cupf.NewtonOptions()
        o.backend = cupf.BackendKind.CUDA
        o.use_cuda_graph = True
        o.custom.serial_nd = True
        s = cupf.NewtonSolver(o)
        s.initialize(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, g.pv, g.pq)
        solvers.append(s)

    def make(s):
        def solve(s_dev):
            v, fm, _ = s.solve_batch_device(s_dev, v0[None, :].expand(s_dev.shape[0], -1).contiguous(), config=cfg)
            return v, fm
        return solve
    sizes = [96, 64, 33, 96, 7, 128, 64]
    ins = [torch.tensor(g.scenarios(b, seed=70 + i)).pin_memory() for i, b in enumerate(sizes)]
    V_out = [torch.empty(b, g.n_bus, dtype=torch.complex128).pin_memory() for b in sizes]
    fm_out = [torch.empty(b, dtype=torch.float64).pin_memory() for b in sizes]
    HostPipeline([make(s) for s in solvers]).run(ins, V_out, fm_out)
    ref = make(solvers[0])
    for i in range(len(sizes)):
        v, fm = ref(ins[i].cuda())
        assert torch.equal(V_out[i], v.cpu()) and torch.equal(fm_out[i], fm.cpu()), i


def test_host_pipeline_overlaps_the_warm_start_network(torch):
    """HostPipeline with a prepare stage: the next batch's network inference
    runs on its own stream into its own slot's buffers while the current
    batch solves; every batch equals its serial warm-started solve, bit for
    bit."""
    import cupf
    from cupf import grids as G
    from cupf.streaming import HostPipeline
    from cupf.warm_start import WarmStart

    g = G.grid_118()
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    o.compute = cupf.ComputePolicy.Mixed
    o.use_cuda_graph = True
    o.custom.serial_nd = True
    s = cupf.NewtonSolver(o)
    s.initialize(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, g.pv, g.pq)
    ws = WarmStart(g, hidden=256, layers=2, seed=0)
    X, Y, _ = ws.generate(s, 4096, seed=2)
    ws.fit(X, Y, epochs=5, batch=512, lr=2e-3)
    cfg = cupf.NRConfig(tolerance=1e-8, max_iter=10)
    sizes = [128, 100, 128, 128, 60]
    ins = [torch.tensor(g.scenarios(b, seed=70 + i)).pin_memory() for i, b in enumerate(sizes)]
    V_out = [torch.empty(b, g.n_bus, dtype=torch.complex128).pin_memory() for b in sizes]
    fm_out = [torch.empty(b, dtype=torch.float64).pin_memory() for b in sizes]
    pipe = HostPipeline(lambda sd, p: ws.solve(s, sd, cfg, pred=p)[:2],
                        prepare=lambda sd, j: ws.predict_standardized(sd, slot=j))
    pipe.run(ins, V_out, fm_out)
    for i in range(len(sizes)):
        v, fm, _, _ = ws.solve(s, ins[i].cuda(), cfg)
        assert torch.equal(V_out[i], v.cpu()) and torch.equal(fm_out[i], fm.cpu())
        assert bool((fm_out[i] <= 1e-8).all())


def test_host_pipeline_hands_failures_to_the_caller(torch):
    """A solve that raises in the pipeline's worker thread, or a prepare that
    raises in the caller's thread, ends run() with that exception; nothing
    is left waiting."""
    from cupf.streaming import HostPipeline

    ins = [torch.ones(32, 8, dtype=torch.complex128).pin_memory() * (i + 1) for i in range(5)]
    V_out = [torch.empty(32, 8, dtype=torch.complex128).pin_memory() for _ in range(5)]
    fm_out = [torch.empty(32, dtype=torch.float64).pin_memory() for _ in range(5)]
    calls = []

    def solve(sd):
        calls.append(1)
        if len(calls) == 2:
            raise RuntimeError("solve failed")
        return sd * 2, sd.real[:, 0].clone()

    with pytest.raises(RuntimeError, match="solve failed"):
        HostPipeline(solve).run(ins, V_out, fm_out)
    assert torch.equal(V_out[0], ins[0] * 2)

    def prepare(sd, slot):
        if float(sd.real[0, 0]) == 2.0:
            raise ValueError("prepare failed")
        return slot

    with pytest.raises(ValueError, match="prepare failed"):
        HostPipeline(lambda sd, st: (sd * 3, sd.real[:, 0].clone()), prepare=prepare).run(ins, V_out, fm_out)
    # and a clean run after both
    HostPipeline(lambda sd: (sd * 4, sd.real[:, 0].clone())).run(ins, V_out, fm_out)
    assert all(torch.equal(V_out[i], ins[i] * 4) for i in range(5))


def test_warm_start_checkpoint_round_trip(torch, tmp_path):
    """WarmStart.save / load: a predictor restored into a freshly built one
    (different initial weights) predicts bit for bit what the trained one
    does; a checkpoint of another network shape is refused."""
    import cupf
    from cupf import grids as G
    from cupf.warm_start import WarmStart

    g = G.grid_118()
    o = cupf.NewtonOptions()
    o.backend = cupf.BackendKind.CUDA
    o.custom.serial_nd = True
    s = cupf.NewtonSolver(o)
    s.initialize(g.indptr, g.indices, g.data, g.n_bus, g.n_bus, g.pv, g.pq)
    ws = WarmStart(g, hidden=128, layers=2, seed=0)
    X, Y, _ = ws.generate(s, 2048, seed=3)
    ws.fit(X, Y, epochs=3, batch=512, lr=2e-3)
    path = tmp_path / "warm118.npz"
    ws.save(path)
    S = torch.tensor(g.scenarios(256, seed=12), device="cuda")
    ref = ws.predict(S).clone()
    fresh = WarmStart(g, hidden=128, layers=2, seed=5)
    fresh.load(path)
    assert torch.equal(fresh.predict(S), ref)
    cfg = cupf.NRConfig(tolerance=1e-8, max_iter=10)
    Va, fa, ia, _ = ws.solve(s, S, cfg)
    Vb, fb, ib, _ = fresh.solve(s, S, cfg)
    assert ia == ib and torch.equal(Va, Vb)
    other = WarmStart(g, hidden=256, layers=2, seed=0)
    with pytest.raises(ValueError):
        other.load(path)
