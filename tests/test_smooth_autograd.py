"""The smoothed F2M bound as a differentiable function (no reference counterpart).

A `torch.autograd.Function` whose forward calls `f2m_smoothed_bound_fwd` and
whose backward calls `f2m_smoothed_bound_bwd` with the upstream gradient, both
through the C ABI, lives here in the test harness only.  The checks:

* `torch.autograd.gradcheck` of that Function on two small jittered-lattice
  instances (coordinates on a 2^-20 grid, step 2^-10, so every perturbed
  coordinate is exact in FP32 and the kNN graph provably does not change);
* the CUDA gradient against central differences (step 1e-4) of the CUDA
  forward on 128 seeded points, x and y, at the defaults of the differentiated
  configuration: 10,000 uniform FP32 points, N = 30, tau = 1e-3, 100 steps --
  and against the FP64 host gradient of the oracle on every coordinate;
* dL/dc_e exported by `f2m_smoothed_bound_bwd_edges` against the oracle's, and
  its node sums (2 at a stationary u: the smoothed x is a fractional 2-matching).

Central differences only make sense where the graph is locally constant, so
the perturbed points are those whose neighbour lists (and the lists they
belong to) keep a margin of several steps at the N-th / (N+1)-th distance.
"""
import numpy as np
import pytest

from f2m_b200 import synth

TAU = 1e-3


def _margins(x, y, N):
    """Per point i: how far its distances may move before a kNN list changes
    (moving i by h along one axis moves each of its distances by at most h).
    Its own list changes when its N-th and (N+1)-th neighbours swap (half
    their gap, both may move); the list of another point j, whose N-th and
    (N+1)-th distances are r_N <= r_N+1, loses i (in it) when d(i,j) passes
    r_N+1 and gains i (outside it) when d(i,j) drops below r_N.  Brute force
    in FP64 over chunks."""
    p = np.stack([x.astype(np.float64), y.astype(np.float64)], 1)
    n = len(p)
    kth = np.zeros((n, 2))  # N-th and (N+1)-th neighbour distance of each point
    chunk = 1024
    for s in range(0, n, chunk):
        d = np.sqrt(((p[s:s + chunk, None, :] - p[None, :, :]) ** 2).sum(-1))
        d[np.arange(d.shape[0]), np.arange(s, s + d.shape[0])] = np.inf
        part = np.partition(d, (N - 1, N), axis=1)
        kth[s:s + chunk] = part[:, [N - 1, N]]
    margin = (kth[:, 1] - kth[:, 0]) / 2  # own list
    for s in range(0, n, chunk):
        d = np.sqrt(((p[s:s + chunk, None, :] - p[None, :, :]) ** 2).sum(-1))
        d[np.arange(d.shape[0]), np.arange(s, s + d.shape[0])] = np.inf
        inside = d <= kth[None, :, 0]
        m = np.where(inside, kth[None, :, 1] - d, d - kth[None, :, 0]).min(axis=1)
        margin[s:s + chunk] = np.minimum(margin[s:s + chunk], m)
    return margin


@pytest.fixture(scope="module")
def torch():
    return pytest.importorskip("torch")


def _function(torch):
    class SmoothedBound(torch.autograd.Function):
        """L[b] of each instance from the (n, 2) FP64 coordinate tensor; the
        device computes in FP32 coordinates with FP64 accumulation."""

        @staticmethod
        def forward(fctx, xy, offs, top_k, params, f2m_ctx):
            a = xy.detach().cpu().numpy()
            x, y = a[:, 0].astype(np.float32), a[:, 1].astype(np.float32)
            L = f2m_ctx.smoothed_bound(offs, x, y, top_k, params=params)
            fctx.save_for_backward(xy)
            fctx.args = (offs, top_k, params, f2m_ctx)
            return torch.from_numpy(L)

        @staticmethod
        def backward(fctx, gL):
            (xy,) = fctx.saved_tensors
            offs, top_k, params, f2m_ctx = fctx.args
            a = xy.detach().cpu().numpy()
            x, y = a[:, 0].astype(np.float32), a[:, 1].astype(np.float32)
            _, gx, gy = f2m_ctx.smoothed_bound(offs, x, y, top_k, params=params, grad=True,
                                               dL=gL.detach().cpu().numpy().astype(np.float64))
            g = np.stack([gx.astype(np.float64), gy.astype(np.float64)], 1)
            return torch.from_numpy(g), None, None, None, None

    return SmoothedBound


@pytest.mark.gpu
def test_autograd_function_passes_gradcheck(ctx, torch):
    import f2m_b200
    N, eps = 8, 2.0 ** -10
    xs, ys, offs = [], [], [0]
    for seed in (26, 33):  # seeds whose kNN margins exceed 3 steps
        x, y = synth.jittered_lattice(40, seed)
        # on a 2^-20 grid: x +- eps stays exact in FP32 (|x| < 8)
        x = (np.round(x.astype(np.float64) * 2 ** 20) / 2 ** 20).astype(np.float32)
        y = (np.round(y.astype(np.float64) * 2 ** 20) / 2 ** 20).astype(np.float32)
        assert _margins(x, y, N).min() > 3 * eps, "pick another seed: a kNN list could change"
        xs.append(x)
        ys.append(y)
        offs.append(offs[-1] + len(x))
    offs = np.array(offs, np.int64)
    xy = torch.tensor(np.stack([np.concatenate(xs), np.concatenate(ys)], 1).astype(np.float64),
                      requires_grad=True)
    # The device takes edge costs in FP32, so each cost carries a rounding of
    # about 3e-8 that a central difference divides by its step: at a step of
    # 2^-13 that noise is ~1e-3 of the gradient, at 2^-10 ~1e-4.  tau 5e-2
    # keeps the step's O(eps^2 / tau^2) truncation near 4e-4.
    p = f2m_b200.default_smooth_params(tau=5e-2, iters=40)
    F = _function(torch)
    assert torch.autograd.gradcheck(lambda t: F.apply(t, offs, N, p, ctx), (xy,), eps=eps,
                                    atol=1e-3, rtol=5e-3)
    # the upstream gradient reaches the device: d(3 L0 + 0.5 L1)
    L = F.apply(xy, offs, N, p, ctx)
    (3.0 * L[0] + 0.5 * L[1]).backward()
    _, gx, gy = ctx.smoothed_bound(offs, xy.detach().numpy()[:, 0].astype(np.float32),
                                   xy.detach().numpy()[:, 1].astype(np.float32), N, params=p,
                                   grad=True, dL=np.array([3.0, 0.5]))
    assert np.array_equal(xy.grad.numpy()[:, 0], gx.astype(np.float64))
    assert np.array_equal(xy.grad.numpy()[:, 1], gy.astype(np.float64))


@pytest.mark.gpu
def test_gradient_at_config4_defaults_vs_central_differences_and_fp64_host(ctx):
    """10,000 FP32 points uniform in [0,1)^2, N = 30, tau = 1e-3, 100 steps:
    central differences (step 1e-4) of the CUDA forward on 128 seeded points
    (x and y: 256 coordinates), and the FP64 host gradient everywhere.

    At tau = 1e-3 a step of 1e-4 moves a logistic argument by up to 0.1, so
    the central difference carries an O(h^2) truncation of up to about 1%;
    the same difference at step 2e-4 gives the Richardson extrapolation,
    which removes that term and must agree to 2e-3."""
    from oracle import oracle as O
    import f2m_b200
    N, h = 30, 1e-4
    x, y = synth.config4(4)
    p = f2m_b200.default_smooth_params()  # tau 1e-3, 100 steps, damping 0.5
    assert p.tau == TAU and p.iters == 100
    offs = np.array([0, len(x)], np.int64)
    L0, gx, gy = ctx.smoothed_bound(offs, x, y, N, params=p, grad=True)
    safe = np.nonzero(_margins(x, y, N) > 6 * h)[0]  # both steps keep the graph
    rng = np.random.default_rng(128)
    pts = rng.choice(safe, 128, replace=False)

    def central(arr, i, hh):
        pp, mm = arr.copy(), arr.copy()
        pp[i] = np.float32(arr[i] + hh)
        mm[i] = np.float32(arr[i] - hh)
        xp, yp = (pp, y) if arr is x else (x, pp)
        xm, ym = (mm, y) if arr is x else (x, mm)
        Lp = ctx.smoothed_bound(offs, xp, yp, N, params=p)[0]
        Lm = ctx.smoothed_bound(offs, xm, ym, N, params=p)[0]
        half = (float(pp[i]) - float(mm[i])) / 2  # the FP32 step actually taken
        return (Lp - Lm) / (2 * half), half

    for i in pts:
        for arr, g in ((x, gx), (y, gy)):
            f1, s1 = central(arr, i, h)
            f2, s2 = central(arr, i, 2 * h)
            rich = (s2 * s2 * f1 - s1 * s1 * f2) / (s2 * s2 - s1 * s1)
            scale = max(1.0, abs(float(g[i])))
            assert abs(f1 - float(g[i])) <= 2e-2 * scale, (int(i), f1, float(g[i]))
            assert abs(rich - float(g[i])) <= 2e-3 * scale, (int(i), rich, f1, float(g[i]))
    # FP64 host gradient of the same computation, every coordinate
    Lo, dx, dy, _ = O.smooth_bound(x, y, N, tau=p.tau, iters=p.iters, omega=p.damping,
                                   newton_max=p.newton_max, grad=True)
    assert abs(L0[0] - Lo) <= 1e-9 * abs(Lo)
    scale = max(np.abs(dx).max(), np.abs(dy).max())
    assert np.abs(gx - dx).max() <= 1e-5 * scale
    assert np.abs(gy - dy).max() <= 1e-5 * scale


@pytest.mark.gpu
def test_edge_cost_gradient_matches_oracle_and_sums_to_two(ctx):
    """dL/dc_e through the C ABI against the oracle's per-edge value, and at a
    stationary u (tau = 1e-2, 400 steps) its sum over each point's edges is 2."""
    from oracle import oracle as O
    import f2m_b200
    x, y = synth.config4(11, 600)
    N = 10
    offs = np.array([0, len(x)], np.int64)
    for tau, iters, up in ((1e-3, 60, 1.0), (1e-2, 400, 2.5)):
        p = f2m_b200.default_smooth_params(tau=tau, iters=iters)
        L, gx, gy, (a, b, c, dc) = ctx.smoothed_bound_edges(offs, x, y, N, params=p,
                                                           dL=np.array([up]))
        row, nbr, co = O.smooth_graph(x, y, N)
        _, _, _, dco = O.smooth_bound(x, y, N, tau=tau, iters=iters, grad=True)
        ref = {}
        for v in range(len(x)):
            for k in range(row[v], row[v + 1]):
                if nbr[k] > v:
                    ref[(v, int(nbr[k]))] = (co[k], dco[k])
        assert len(ref) == len(a)
        for e in range(len(a)):
            cr, dr = ref[(int(a[e]), int(b[e]))]
            assert c[e] == cr
            assert abs(dc[e] - up * dr) <= 1e-6 * up
        if iters == 400:
            deg = np.zeros(len(x))
            np.add.at(deg, a, dc / up)
            np.add.at(deg, b, dc / up)
            assert np.allclose(deg, 2.0, atol=1e-6)
            assert np.all(dc >= -1e-9) and np.all(dc <= up * (1 + 1e-9))
    with pytest.raises(f2m_b200.F2MError) as e:
        import ctypes
        m = ctypes.c_int64()
        gx = np.zeros(len(x), np.float32)
        gy = np.zeros(len(x), np.float32)
        L = np.zeros(1)
        ctx._check(f2m_b200.lib().f2m_smoothed_bound_bwd_edges(
            ctx.handle, 1, f2m_b200._ptr(offs), f2m_b200._ptr(x), f2m_b200._ptr(y), N,
            ctypes.byref(p), None, f2m_b200._ptr(L), f2m_b200._ptr(gx), f2m_b200._ptr(gy), 5,
            ctypes.byref(m), None, None, None, None))
    assert e.value.status == f2m_b200.ERR_CAPACITY and m.value > 5


def test_margin_helper_flags_a_tie():
    """The margin helper sees an exact tie at the N-th distance (zero margin)."""
    x = np.array([0, 1, -1, 0, 0, 3, 5, 7], np.float32)
    y = np.array([0, 0, 0, 1, -1, 3, 5, 7], np.float32)
    assert _margins(x, y, 3).min() == 0.0
