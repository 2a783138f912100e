"""
Surrogate MLP: the numpy oracle checked by finite differences (CPU), then
the tensor-core forward, backward and weight-gradient kernels checked
against the oracle, and a short training run (GPU).
"""

import numpy as np
import pytest

from oracle import mlp_ref


def _random_net(rng, scale=0.5, nin=16, hid=256):
    W = [rng.normal(0, scale/np.sqrt(nin if l == 0 else hid), (hid, nin if l == 0 else hid))
         for l in range(4)]
    W[0][:, 15:] = 0.0
    b = [rng.normal(0, 0.1, hid) for _ in range(4)]
    w_out = rng.normal(0, 1/np.sqrt(hid), hid)
    return W, b, w_out, 0.3


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    hid = 8
    W = [rng.normal(0, 0.5, (hid, 16 if l == 0 else hid)) for l in range(4)]
    b = [rng.normal(0, 0.1, hid) for _ in range(4)]
    w_out = rng.normal(0, 0.5, hid)
    x = rng.normal(0, 1, (5, 16))
    dout = rng.normal(0, 1, 5)

    def f(W, b, w_out, b_out):
        out, _, _ = mlp_ref.forward(x, W, b, w_out, b_out, emulate_bf16=False)
        return float(dout @ out)
    out, zs, hs = mlp_ref.forward(x, W, b, w_out, 0.2, emulate_bf16=False)
    dW, db, dwo, dbo = mlp_ref.backward(x, W, w_out, dout, zs, hs, emulate_bf16=False)
    eps = 1e-6
    for l in range(4):
        for (i, j) in [(0, 0), (3, 5), (hid - 1, 2)]:
            Wp = [w.copy() for w in W]
            Wp[l][i, j] += eps
            Wm = [w.copy() for w in W]
            Wm[l][i, j] -= eps
            fd = (f(Wp, b, w_out, 0.2) - f(Wm, b, w_out, 0.2))/(2*eps)
            assert abs(fd - dW[l][i, j]) < 1e-6*max(1, abs(fd))
        bp = [v.copy() for v in b]
        bp[l][1] += eps
        bm = [v.copy() for v in b]
        bm[l][1] -= eps
        fd = (f(W, bp, w_out, 0.2) - f(W, bm, w_out, 0.2))/(2*eps)
        assert abs(fd - db[l][1]) < 1e-6*max(1, abs(fd))
    wp = w_out.copy()
    wp[2] += eps
    wm = w_out.copy()
    wm[2] -= eps
    fd = (f(W, b, wp, 0.2) - f(W, b, wm, 0.2))/(2*eps)
    assert abs(fd - dwo[2]) < 1e-6
    assert abs(dbo - dout.sum()) < 1e-12


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2**-8, 1.0 + 2**-7, -3.14159, 1e-3])
    r = mlp_ref.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2**-7
    assert abs(r[3] + 3.140625) < 1e-12


def _gpu_net(rng):
    import torch
    from sasmodels_b200.surrogate import MLP
    net = MLP(seed=1)
    W, b, w_out, b_out = _random_net(rng)
    net.load_state({"W": [w.astype(np.float32) for w in W],
                    "b": [v.astype(np.float32) for v in b],
                    "w_out": w_out.astype(np.float32),
                    "b_out": np.array([b_out], np.float32)})
    return net, W, b, w_out, b_out


def _inputs(rng, n, n_pad):
    """Features as the compensated pair the kernels take: hi, lo (device)
    and their float64 sum (host)."""
    import torch
    x = np.zeros((n_pad, 16))
    x[:n, :11] = rng.uniform(-1, 1, (n, 11))
    hi = mlp_ref.bf16(x)
    lo = mlp_ref.bf16(x - hi)
    return (torch.as_tensor(hi, dtype=torch.bfloat16, device="cuda"),
            torch.as_tensor(lo, dtype=torch.bfloat16, device="cuda"), hi + lo, hi)


@pytest.mark.gpu
def test_tc_forward_matches_oracle(cuda):
    rng = np.random.default_rng(3)
    net, W, b, w_out, b_out = _gpu_net(rng)
    n, n_pad = 300, 384
    x, xlo, xh, _ = _inputs(rng, n, n_pad)
    out = net.forward(x, xlo, n)
    net.stream.synchronize()
    assert net.errors() == 0
    got = out.cpu().numpy()[:n]
    ref, _, _ = mlp_ref.forward(xh[:n], [mlp_ref.bf16(w) for w in W],
                                [np.float32(v).astype(np.float64) for v in b],
                                np.float32(w_out).astype(np.float64), np.float32(b_out))
    # the oracle rounds every stored value as the kernel does; what remains
    # is FP32 accumulation order and the fast exp/divide of SiLU, which move
    # a rounding decision of the compensated activations now and then
    err = np.abs(got - ref).max()/np.abs(ref).max()
    assert err < 2e-3, err
    # an FP64 forward without BF16 storage differs only at BF16 precision
    exact, _, _ = mlp_ref.forward(xh[:n], W, b, w_out, b_out, emulate_bf16=False)
    assert np.abs(got - exact).max()/np.abs(exact).max() < 5e-2


@pytest.mark.gpu
def test_tc_gradients_match_oracle(cuda):
    import torch
    rng = np.random.default_rng(4)
    net, W, b, w_out, b_out = _gpu_net(rng)
    n, n_pad = 500, 512
    x, xlo, xh, xhi = _inputs(rng, n, n_pad)
    y = torch.as_tensor(rng.normal(0, 1, n_pad), dtype=torch.float32, device="cuda")
    loss, dW, db, dwo, dbo = net.gradients(x, xlo, y, n)
    net.stream.synchronize()
    assert net.errors() == 0
    Wf = [np.float32(w).astype(np.float64) for w in W]
    bf = [np.float32(v).astype(np.float64) for v in b]
    wof = np.float32(w_out).astype(np.float64)
    out, zs, hs = mlp_ref.forward(xh, Wf, bf, wof, np.float32(b_out))
    yv = y.cpu().numpy().astype(np.float64)
    dout = np.zeros(n_pad)
    dout[:n] = 2*(out[:n] - yv[:n])/n
    # the layer-0 weight gradient uses the high half of the inputs
    rW, rb, rwo, rbo = mlp_ref.backward(xhi, Wf, wof, dout, zs, hs)
    for l in range(4):
        nb = 16 if l == 0 else 256
        g = dW[l].cpu().numpy().reshape(net.splits, 256, nb).sum(axis=0)
        rel = np.linalg.norm(g - rW[l])/np.linalg.norm(rW[l])
        assert rel < 2e-3, (l, rel)
        rel = np.linalg.norm(db[l].cpu().numpy() - rb[l])/np.linalg.norm(rb[l])
        assert rel < 2e-3, (l, "bias", rel)
    rel = np.linalg.norm(dwo.cpu().numpy() - rwo)/np.linalg.norm(rwo)
    assert rel < 2e-3
    assert abs(float(dbo.item()) - rbo) < 1e-3*max(1, abs(rbo))
    assert abs(float(loss.item()) - np.mean((out[:n] - yv[:n])**2)) < 2e-3*np.mean((out[:n] - yv[:n])**2)


@pytest.mark.gpu
def test_tc_training_reduces_loss(cuda):
    """Fit a smooth function of the 7 inputs; the loss must fall by >10x."""
    import torch
    from sasmodels_b200.surrogate import MLP
    rng = np.random.default_rng(5)
    net = MLP(seed=2)
    n = n_pad = 4096
    xs = np.zeros((n, 16))
    xs[:, :7] = rng.uniform(-1, 1, (n, 7))
    target = np.sin(2*xs[:, 0]) + xs[:, 1]*xs[:, 5] - 0.5*xs[:, 3]**2
    hi = mlp_ref.bf16(xs)
    x = torch.as_tensor(hi, dtype=torch.bfloat16, device="cuda")
    xlo = torch.as_tensor(mlp_ref.bf16(xs - hi), dtype=torch.bfloat16, device="cuda")
    y = torch.as_tensor(target, dtype=torch.float32, device="cuda")
    first = None
    for step in range(300):
        loss = net.train_step(x, xlo, y, n, lr=2e-3)
        if first is None:
            net.stream.synchronize()
            first = float(loss.item())
    net.stream.synchronize()
    last = float(loss.item())
    assert net.errors() == 0
    assert last < first/10, (first, last)


@pytest.mark.gpu
@pytest.mark.parametrize("n, blocks", [(300, 0), (5000, 3), (128*300 + 17, 0)])
def test_tc_infer_matches_forward(cuda, n, blocks):
    """The persistent pipelined inference kernel computes the training
    forward's outputs (same MMAs in the same order; the output dot is summed
    in two halves), for ragged n, several tiles per CTA and one tile per CTA."""
    from sasmodels_b200.surrogate import pad128
    rng = np.random.default_rng(11)
    net, W, b, w_out, b_out = _gpu_net(rng)
    n_pad = pad128(n)
    x, xlo, xh, _ = _inputs(rng, n, n_pad)
    # the kernels run on net.stream: synchronise before reading or copying
    fwd = net.forward(x, xlo, n)
    net.stream.synchronize()
    a = fwd.cpu().numpy()[:n].copy()
    inf = net.infer(x, xlo, n, blocks=blocks)
    net.stream.synchronize()
    assert net.errors() == 0
    c = inf.cpu().numpy()[:n]
    np.testing.assert_allclose(c, a, rtol=1e-5, atol=1e-5*np.abs(a).max())
    ref, _, _ = mlp_ref.forward(xh[:min(n, 2000)], [mlp_ref.bf16(w) for w in W],
                                [np.float32(v).astype(np.float64) for v in b],
                                np.float32(w_out).astype(np.float64), np.float32(b_out))
    assert np.abs(c[:len(ref)] - ref).max()/np.abs(ref).max() < 2e-3


@pytest.mark.gpu
@pytest.mark.parametrize("n, blocks", [(1, 0), (300, 0), (5000, 3), (128*300 + 17, 0),
                                       (128*1000, 1)])
def test_tc_serve_matches_infer(cuda, n, blocks):
    """The overlapped inference kernel (its own MMA warp, two TMEM
    accumulators, layer l+1's MMAs under layer l's epilogue) gives the
    outputs of mlp_infer: the hidden activations are computed identically,
    only the output dot is summed in four partial sums per row.  Cases: one
    row, one tile per CTA, many tiles per CTA (every barrier phase wraps
    many times), one CTA for 1000 tiles."""
    import torch
    from sasmodels_b200.surrogate import pad128
    rng = np.random.default_rng(17)
    net, W, b, w_out, b_out = _gpu_net(rng)
    n_pad = pad128(n)
    x, xlo, xh, _ = _inputs(rng, n, n_pad)
    inf = net.infer(x, xlo, n)
    net.stream.synchronize()
    a = inf.cpu().numpy()[:n].copy()
    net._infer_out.fill_(float("nan"))
    torch.cuda.synchronize()
    srv = net.serve(x, xlo, n, blocks=blocks)
    net.stream.synchronize()
    assert net.errors() == 0
    c = srv.cpu().numpy()
    assert np.isfinite(c[:n]).all()
    np.testing.assert_allclose(c[:n], a, rtol=1e-5, atol=1e-6*np.abs(a).max())
    # rows beyond n are not written
    assert np.isnan(c[n:n_pad]).all()
    ref, _, _ = mlp_ref.forward(xh[:min(n, 2000)], [mlp_ref.bf16(w) for w in W],
                                [np.float32(v).astype(np.float64) for v in b],
                                np.float32(w_out).astype(np.float64), np.float32(b_out))
    assert np.abs(c[:len(ref)] - ref).max()/np.abs(ref).max() < 2e-3


@pytest.mark.gpu
def test_tc_infer_tracks_training(cuda):
    """The weight image is refreshed after training steps."""
    import torch
    from sasmodels_b200.surrogate import pad128
    rng = np.random.default_rng(12)
    net, *_ = _gpu_net(rng)
    n = 1000
    x, xlo, _, _ = _inputs(rng, n, pad128(n))
    y = torch.as_tensor(rng.normal(size=pad128(n)), dtype=torch.float32, device="cuda")
    def host(t):
        net.stream.synchronize()
        return t.cpu().numpy()[:n].copy()
    before = host(net.infer(x, xlo, n))
    net.train_step(x, xlo, y, n, 1e-2)
    after = host(net.infer(x, xlo, n))
    fwd = host(net.forward(x, xlo, n))
    assert not np.array_equal(before, after)
    np.testing.assert_allclose(after, fwd, rtol=1e-5, atol=1e-5*np.abs(fwd).max())


@pytest.mark.gpu
def test_tc_pipelined_training_kernels_match(cuda):
    """The pipelined forward (with z/h planes), the overlapped forward that
    training uses, and the pipelined backward give the planes of the
    one-CTA-per-tile training kernels bit for bit (same MMAs in the same
    order, same epilogue arithmetic)."""
    import ctypes as ct
    import torch
    from sasmodels_b200.surrogate import HID, pad128
    rng = np.random.default_rng(13)
    net, *_ = _gpu_net(rng)
    n = 3000
    n_pad = pad128(n)
    x, xlo, _, _ = _inputs(rng, n, n_pad)
    net._scratch(n_pad)
    lib, st = net.lib, net.stream.cuda_stream
    bf = dict(dtype=torch.bfloat16, device="cuda")
    z1, h1, z2, h2 = [torch.zeros(4*n_pad*HID, **bf) for _ in range(4)]
    o1 = torch.zeros(n_pad, dtype=torch.float32, device="cuda")
    o2 = torch.zeros_like(o1)
    net._check(lib.sasb200_mlp_forward(n, n_pad, x.data_ptr(), xlo.data_ptr(), net._ptrs(net.Wb),
                                       net._ptrs(net.b), net.w_out.data_ptr(),
                                       net.b_out.data_ptr(), o1.data_ptr(), z1.data_ptr(),
                                       h1.data_ptr(), net.err.data_ptr(), st), "forward")
    net._pack()
    net._check(lib.sasb200_mlp_infer(n, n_pad, x.data_ptr(), xlo.data_ptr(), net.img.data_ptr(),
                                     net._ptrs(net.b), net.w_out.data_ptr(),
                                     net.b_out.data_ptr(), o2.data_ptr(), z2.data_ptr(),
                                     h2.data_ptr(), net.err.data_ptr(), 5, st), "infer")
    dout = torch.as_tensor(rng.normal(size=n_pad), dtype=torch.float32, device="cuda")
    d1, d2 = torch.zeros_like(z1), torch.zeros_like(z1)
    net._check(lib.sasb200_mlp_backward(n, n_pad, net._ptrs(net.WTb), net.w_out.data_ptr(),
                                        dout.data_ptr(), z1.data_ptr(), d1.data_ptr(),
                                        net.err.data_ptr(), st), "backward")
    net._check(lib.sasb200_mlp_backward_p(n, n_pad, net.img_t.data_ptr(), net.w_out.data_ptr(),
                                          dout.data_ptr(), z2.data_ptr(), d2.data_ptr(),
                                          net.err.data_ptr(), 7, st), "backward_p")
    net.stream.synchronize()
    assert net.errors() == 0
    assert torch.equal(z1, z2) and torch.equal(h1, h2)
    assert torch.equal(d1, d2)
    # the overlapped kernel writes the same planes (the training forward);
    # several tiles per CTA so its barrier phases wrap
    z3, h3 = torch.zeros_like(z1), torch.zeros_like(h1)
    o3 = torch.zeros_like(o1)
    net._check(lib.sasb200_mlp_serve(n, n_pad, x.data_ptr(), xlo.data_ptr(), net.img.data_ptr(),
                                     net._ptrs(net.b), net.w_out.data_ptr(),
                                     net.b_out.data_ptr(), o3.data_ptr(), z3.data_ptr(),
                                     h3.data_ptr(), net.err.data_ptr(), 5, st), "serve")
    net.stream.synchronize()
    assert net.errors() == 0
    assert torch.equal(z1, z3) and torch.equal(h1, h3)
    torch.testing.assert_close(o3[:n], o1[:n], rtol=1e-5, atol=1e-6*float(o1[:n].abs().max()))


@pytest.mark.gpu
def test_tc_data_parallel_replicas(cuda):
    """Two replicas each taking half of a global batch, their gradients
    averaged as the data-parallel all-reduce does, give the full batch's
    gradients, and both replicas apply the same update bit for bit."""
    import torch
    n, half = 2048, 1024
    a, *_ = _gpu_net(np.random.default_rng(21))
    b, *_ = _gpu_net(np.random.default_rng(21))
    full, *_ = _gpu_net(np.random.default_rng(21))
    rng = np.random.default_rng(22)
    x, xlo, _, _ = _inputs(rng, n, n)
    y = torch.as_tensor(rng.normal(0, 1, n), dtype=torch.float32, device="cuda")
    g_full = full.reduced_gradients(x, xlo, y, n)
    g_b = b.reduced_gradients(x[half:], xlo[half:], y[half:], half)
    b.stream.synchronize()
    seen = {}

    def reduce(grads):
        for t, u in zip(grads, g_b):
            t.add_(u).div_(2.0)
        seen["grads"] = grads
    loss = a.train_step(x[:half], xlo[:half], y[:half], half, 1e-3, reduce=reduce)
    a.stream.synchronize()
    b.apply_gradients(seen["grads"][1:], 1e-3, 1)
    b.stream.synchronize()
    full.stream.synchronize()
    assert a.errors() == 0 and b.errors() == 0 and full.errors() == 0
    for u, v in zip(seen["grads"], g_full):
        rel = (torch.linalg.norm(u - v)/torch.linalg.norm(v)).item()
        assert rel < 1e-4, rel
    assert abs(loss.item() - g_full[0].item()) < 1e-5*abs(g_full[0].item())
    for p, q in zip(a.params, b.params):
        assert torch.equal(p, q)
    for p, q in zip(a.Wb + a.WTb, b.Wb + b.WTb):
        assert torch.equal(p, q)


@pytest.mark.gpu
def test_training_graph_replays_the_eager_steps(cuda):
    """A training step captured as a CUDA graph (batch gather by index
    buffer, learning-rate schedule and Adam bias corrections advanced on the
    device) updates the weights as the eager steps with the host-computed
    schedule do."""
    import math
    import torch
    from sasmodels_b200.surrogate import MLP, WARMUP_STEPS
    rng = np.random.default_rng(21)
    B, n, total, lr = 1024, 1024*6, 7, 3e-3
    x = torch.as_tensor(mlp_ref.bf16(np.c_[rng.uniform(-1, 1, (n, 7)), np.zeros((n, 9))]),
                        dtype=torch.bfloat16, device="cuda")
    xlo = torch.zeros_like(x)
    y = torch.as_tensor(rng.normal(0, 1, n), dtype=torch.float32, device="cuda")
    idx = [torch.as_tensor(rng.permutation(n)[:B], device="cuda") for _ in range(total)]
    eager, graphed = MLP(seed=4), MLP(seed=4)
    losses_e, losses_g = [], []
    for s in range(total):
        rate = lr*min(1.0, (s + 1)/WARMUP_STEPS)*0.5*(1 + math.cos(math.pi*s/total))
        with torch.cuda.stream(eager.stream):
            xb, xlb, yb = x.index_select(0, idx[s]), xlo.index_select(0, idx[s]), y.index_select(0, idx[s])
        loss = eager.train_step(xb, xlb, yb, B, rate)
        eager.stream.synchronize()          # the loss is computed on the net's stream
        losses_e.append(float(loss.item()))
    rate0 = lr*min(1.0, 1/WARMUP_STEPS)
    with torch.cuda.stream(graphed.stream):
        xb, xlb, yb = x.index_select(0, idx[0]), xlo.index_select(0, idx[0]), y.index_select(0, idx[0])
    loss = graphed.train_step(xb, xlb, yb, B, rate0)
    graphed.stream.synchronize()
    losses_g.append(float(loss.item()))
    g = graphed.capture_training(x, xlo, y, B, lr, total, 1, warmup=WARMUP_STEPS)
    for s in range(1, total):
        loss = g.step(idx[s])
        graphed.stream.synchronize()
        losses_g.append(float(loss.item()))
    eager.stream.synchronize()
    assert eager.errors() == 0 and graphed.errors() == 0
    assert graphed.step_count == eager.step_count == total
    np.testing.assert_allclose(losses_g, losses_e, rtol=1e-5)
    for a, b in zip(graphed.params, eager.params):
        a, b = a.cpu().numpy(), b.cpu().numpy()
        assert np.abs(a - b).max() <= 1e-5*max(np.abs(b).max(), 1e-3)
    # the weight images of inference are refreshed after graph steps
    out_g = graphed.serve(x[:B], xlo[:B], B)
    out_e = eager.serve(x[:B], xlo[:B], B)
    graphed.stream.synchronize()
    eager.stream.synchronize()
    np.testing.assert_allclose(out_g.cpu().numpy(), out_e.cpu().numpy(), rtol=1e-4, atol=1e-5)


@pytest.mark.gpu
@pytest.mark.parametrize("rows", [1, 63, 1000, 8192])
def test_col_sums(cuda, rows):
    """Column sums of a bf16 matrix (plain and row-weighted), the bias and
    output-layer gradients of training, against float64 sums."""
    import torch
    from sasmodels_b200.surrogate import _lib
    lib = _lib()
    rng = np.random.default_rng(rows)
    M = mlp_ref.bf16(rng.normal(0, 1, (rows, 256)))
    v = rng.normal(0, 1, rows).astype(np.float32)
    Md = torch.as_tensor(M, dtype=torch.bfloat16, device="cuda")
    vd = torch.as_tensor(v, device="cuda")
    part = torch.empty(lib.sasb200_col_sum_parts(rows)*256, dtype=torch.float32, device="cuda")
    out = torch.empty(256, dtype=torch.float32, device="cuda")
    for weights in (None, vd):
        st = torch.cuda.current_stream().cuda_stream
        assert lib.sasb200_col_sums(rows, 256, Md.data_ptr(),
                                    weights.data_ptr() if weights is not None else None,
                                    part.data_ptr(), out.data_ptr(), st) == 0
        torch.cuda.synchronize()
        want = (M*(v[:, None].astype(np.float64) if weights is not None else 1.0)).sum(axis=0)
        scale = np.abs(M).sum(axis=0)*(np.abs(v).max() if weights is not None else 1.0)
        assert np.all(np.abs(out.cpu().numpy() - want) <= 1e-5*scale)
