"""The surrogate's tensor-core kernels (tcgen05 BF16 GEMM with fused epilogues, loss / bias /
split-K / Adam kernels) against numpy: GEMM variants, full-network gradients against the float64
CPU reference (tests/mlp_reference.py) on the same BF16 weights, and a training run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from tests.mlp_reference import forward as ref_forward, loss_and_grads  # noqa: E402
from xyce_b200 import surrogate as S  # noqa: E402


def _bf(a):
    return torch.as_tensor(a, dtype=torch.float32).to(torch.bfloat16)


def _np(t):
    return t.float().cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("M,N,K,tile_n,splits", [(256, 128, 64, 128, 1), (384, 128, 128, 128, 1),
                                                 (128, 16, 128, 16, 1), (200, 100, 48, 128, 1),
                                                 (128, 128, 1024, 128, 4), (16, 128, 4096, 128, 8)])
def test_gemm_f32_matches_numpy(M, N, K, tile_n, splits):
    rng = np.random.default_rng(M + N + K)
    A = _bf(rng.standard_normal((M, K))).cuda()
    B = _bf(rng.standard_normal((N, K))).cuda()
    k = S._Lib(torch, torch.device("cuda", 0))
    part = torch.zeros(splits * M * N, dtype=torch.float32, device="cuda")
    used = k.gemm(A, B, M, N, K, K, K, S.EPI_F32, tile_n, C32=part, ldc=N, splits=splits)
    torch.cuda.synchronize()
    k.check_err()
    C = part.view(-1, M, N)[:used].sum(0).cpu().numpy().astype(np.float64)
    ref = _np(A) @ _np(B).T
    assert np.allclose(C, ref, rtol=1e-5, atol=1e-4 * np.abs(ref).max()), np.abs(C - ref).max()


def test_gemm_epilogues_match_numpy():
    rng = np.random.default_rng(3)
    M, N, K = 256, 128, 128
    A = _bf(rng.standard_normal((M, K)) * 0.3).cuda()
    B = _bf(rng.standard_normal((N, K)) * 0.3).cuda()
    bias = torch.as_tensor(rng.standard_normal(N), dtype=torch.float32, device="cuda")
    k = S._Lib(torch, torch.device("cuda", 0))
    Z = torch.zeros(M, N, dtype=torch.bfloat16, device="cuda")
    H = torch.zeros_like(Z)
    HT = torch.zeros(N, M, dtype=torch.bfloat16, device="cuda")
    k.gemm(A, B, M, N, K, K, K, S.EPI_BIAS_SILU, 128, bias=bias, Z=Z, H=H, HT=HT, ldc=N, ldt=M)
    acc = _np(A) @ _np(B).T + bias.cpu().numpy()
    zr = acc
    hr = zr / (1 + np.exp(-zr))
    assert np.allclose(_np(Z), zr, rtol=1e-2, atol=1e-2)
    assert np.allclose(_np(H), hr, rtol=1e-2, atol=1e-2)
    assert np.array_equal(_np(HT), _np(H).T)
    D = torch.zeros_like(Z)
    DT = torch.zeros_like(HT)
    k.gemm(A, B, M, N, K, K, K, S.EPI_SILU_BACK, 128, Zin=Z, H=D, HT=DT, ldc=N, ldt=M)
    z = _np(Z)
    s = 1 / (1 + np.exp(-z))
    dr = (_np(A) @ _np(B).T) * s * (1 + z * (1 - s))
    assert np.allclose(_np(D), dr, rtol=2e-2, atol=2e-2 * np.abs(dr).max())
    assert np.array_equal(_np(DT), _np(D).T)
    Y = torch.zeros(M, 16, dtype=torch.float32, device="cuda")
    B16 = _bf(rng.standard_normal((16, K))).cuda()
    k.gemm(A, B16, M, 16, K, K, K, S.EPI_BIAS_F32, 16, C32=Y, bias=bias, ldc=16)
    yr = _np(A) @ _np(B16).T + bias.cpu().numpy()[:16]
    torch.cuda.synchronize()
    k.check_err()
    assert np.allclose(Y.cpu().numpy(), yr, rtol=1e-5, atol=1e-4)


def test_network_gradients_match_cpu_reference():
    rng = np.random.default_rng(11)
    net = S.SurrogateMLP(seed=5, max_batch=1024)
    n = 1000
    X = rng.uniform(-1, 1, (n, S.N_IN))
    T = rng.standard_normal((n, S.N_OUT))
    Xq = X.astype(np.float32).astype(np.float64)  # the inputs as the kernels see them (FP32)
    Bp = 1024
    net._load_inputs(X)
    net.T[:n] = torch.as_tensor(T, dtype=torch.float32, device="cuda")
    net._forward(Bp)
    net.backward(n, Bp)
    torch.cuda.synchronize()
    net.k.check_err()
    params = net.parameters_numpy()
    y_ref, _ = ref_forward(params, Xq)
    y = net.Y[:n, :S.N_OUT].double().cpu().numpy()
    assert np.abs(y - y_ref).max() <= 0.05 * np.abs(y_ref).max() + 1e-3
    _, grads = loss_and_grads(params, Xq, T)
    for l, (o, i) in enumerate(net.dims):
        gw = net.gW[l][:o, :i].double().cpu().numpy()
        gb = net.gb[l][:o].double().cpu().numpy()
        for got, ref in ((gw, grads[l][0]), (gb, grads[l][1])):
            rel = np.linalg.norm(got - ref) / max(np.linalg.norm(ref), 1e-30)
            assert rel < 0.05, (l, rel)


def test_training_reduces_loss():
    rng = np.random.default_rng(2)
    net = S.SurrogateMLP(seed=1, max_batch=8192)
    W = rng.standard_normal((S.N_OUT, S.N_IN))
    cfg = S.AdamConfig(lr=3e-3)
    losses = []
    for it in range(300):
        X = rng.uniform(-1, 1, (8192, S.N_IN))
        T = np.tanh(X @ W.T) + 0.1 * X[:, :1] ** 2
        losses.append(float(net.train_step(X, T, cfg)))
    torch.cuda.synchronize()
    net.k.check_err()
    assert losses[-1] < 0.05 * losses[0], (losses[0], losses[-1])


def test_bsim4_surrogate_trains_on_fp64_samples_and_warm_start_keeps_exact_answer():
    """FP64 kernel samples -> tensor-core training -> held-out error vs FP64; then a transient of a
    BSIM4 gate netlist with and without the surrogate warm start: the exact FP64 loads make the
    converged evaluations, so the waveforms agree to the Newton tolerance."""
    from tests.parity import family_inputs
    from xyce_b200 import MosfetDevice, netlist
    from xyce_b200.transient import GpuTransient, NewtonParams

    sur = S.BsimSurrogate(seed=0)
    rep = sur.train(n_samples=2_000_000, epochs=4, batch=16384)
    for typ in ("nmos", "pmos"):
        assert rep[typ]["Id"]["rel_median"] < 0.35, rep[typ]["Id"]
    c = netlist.random_logic(300, seed=3, n_inputs=8)
    rowptr, colind = netlist.jacobian_pattern(c)
    cards, im, nd, params = family_inputs(c, None)
    tight = NewtonParams(max_iter=40, rhs_tol=1e-9, delta_x_tol=1e-3, abs_tol=1e-9, rel_tol=1e-6,
                         update_weights_each_iter=False)
    waves = []
    for warm in (False, True):
        fam = MosfetDevice(cards, im, nd, params, (rowptr, colind), c.n_unknowns, level=14)
        g = GpuTransient(c, fam, rowptr, colind)
        g.predictor = "linear"
        if warm:
            g.surrogate = S.SurrogateLoads(sur, fam, c.mos_type, c.mos_nodes, c.mos_w, c.mos_l)
        g.dcop()
        _, w = g.run(0.3e-9, 10e-12, params=tight, record=np.arange(c.n_nodes))
        if warm:
            assert g.stats.surrogate_loads > 0
        waves.append(w)
        g.close()
        fam.close()
    assert np.abs(waves[0] - waves[1]).max() < 1e-9


def test_fused_forward_matches_layer_by_layer():
    """The one-launch fused inference kernel against the layer-by-layer GEMM path, on a trained-ish
    network (a few Adam steps so the weights are not the initial ones)."""
    rng = np.random.default_rng(8)
    net = S.SurrogateMLP(seed=4, max_batch=70000)
    for _ in range(5):
        X = rng.uniform(-1, 1, (4096, S.N_IN))
        net.train_step(X, np.tanh(X @ rng.standard_normal((S.N_IN, S.N_OUT))), S.AdamConfig(lr=1e-2))
    n = 66_000  # not a multiple of the 128-row tile
    X = rng.uniform(-1, 1, (n, S.N_IN))
    ref = net.forward(X).clone()
    net._load_inputs(X)
    net.Y.zero_()
    got = net.forward_fused(n)
    torch.cuda.synchronize()
    net.k.check_err()
    assert torch.allclose(got, ref, rtol=1e-5, atol=1e-5), (got - ref).abs().max()
