"""The learned limiter's tensor-core MLP kernels (through the C ABI) against the numpy oracle: logits, loss and every
parameter's gradient (BF16 MMA inputs, FP32 accumulation; tolerance 2e-3 relative to the largest entry, the size of
BF16 rounding of the accumulated terms), two training steps giving the same bits, and a loss that falls under Adam."""
import numpy as np
import pytest

from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu


def data(n, seed=0):
    rng = np.random.default_rng(seed)
    x = M.bf16(rng.uniform(-1, 1, (n, M.IN)).astype(np.float32))
    t = rng.uniform(0, 1, (n, M.USED)).astype(np.float32)
    w = (rng.uniform(0, 1, (n, M.USED)) > 0.2).astype(np.float32)
    return x, t, w


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-30))


def test_forward_and_gradient_match_oracle(cuda):
    import torch

    from luna_cpp_b200.learned import LimiterMLP, init_params

    n = 1000  # not a multiple of the 64-row block: padded rows must add nothing
    x, t, w = data(n)
    p = init_params(3)
    p[M.B3:M.PARAMS] = 0.3
    net = LimiterMLP(p)
    xd = torch.tensor(x, device="cuda").to(torch.bfloat16)
    logits = net.forward(xd).cpu().numpy()
    want, _ = M.forward(p, x)
    assert rel(logits, want) < 2e-3
    scale = 1.0 / w.sum()
    loss = net.gradient(xd, torch.tensor(t, device="cuda"), torch.tensor(w, device="cuda"), scale).item()
    g = net.grad.cpu().numpy().copy()
    want_loss, want_g = M.loss_and_grad(p, x, t, w, scale)
    assert abs(loss - want_loss) <= 2e-3 * abs(want_loss)
    for name, a, b in (("W1", M.W1, M.B1), ("b1", M.B1, M.W2), ("W2", M.W2, M.B2), ("b2", M.B2, M.W3), ("W3", M.W3, M.B3),
                       ("b3", M.B3, M.PARAMS)):
        assert rel(g[a:b], want_g[a:b]) < 2e-3, name
    net.gradient(xd, torch.tensor(t, device="cuda"), torch.tensor(w, device="cuda"), scale)
    assert np.array_equal(net.grad.cpu().numpy(), g)


def test_adam_lowers_the_loss(cuda):
    import torch

    from luna_cpp_b200.learned import LimiterMLP

    n = 4096
    rng = np.random.default_rng(1)
    x = M.bf16(rng.uniform(-1, 1, (n, M.IN)).astype(np.float32))
    # A learnable target: a smooth function of the first features.
    t = (0.5 + 0.4 * np.tanh(x[:, :M.USED] - 0.5 * x[:, M.USED:2 * M.USED])).astype(np.float32)
    w = np.ones((n, M.USED), np.float32)
    net = LimiterMLP(seed=2)
    xd, td, wd = (torch.tensor(x, device="cuda").to(torch.bfloat16), torch.tensor(t, device="cuda"), torch.tensor(w, device="cuda"))
    first = net.gradient(xd, td, wd).item()
    for _ in range(300):
        net.gradient(xd, td, wd)
        net.adam(lr=3e-3)
    last = net.gradient(xd, td, wd).item()
    assert last < 0.2 * first


def test_factor_path_reproduces_the_plain_limiter(cuda):
    """The learned path with the factors min(alpha, 1) (the min-factor form of the limiter) gives the plain sweep's
    limited gradients to rounding, and the same step."""
    from conftest import jittered_mesh
    from luna_cpp_b200 import hydro
    from luna_cpp_b200.problems import rough_state

    mesh = jittered_mesh(16)
    q0 = rough_state(mesh.n_cells) * mesh.volume[:, None]
    plain = hydro.FiniteVolume(mesh)
    plain.set_state(q0)
    factors = hydro.FiniteVolume(mesh)
    factors.set_limiter("factors")
    factors.set_state(q0)
    dt = plain.time_step(0.3)
    assert abs(factors.time_step(0.3) - dt) <= 1e-14 * dt
    gp, gf = plain.gradients(), factors.gradients()
    assert np.max(np.abs(gp - gf)) <= 1e-10 * np.max(np.abs(gp))
    plain.step(dt)
    factors.step(dt)
    qp, qf = plain.get_state(), factors.get_state()
    assert np.max(np.abs(qp - qf)) / np.max(np.abs(qp)) < 1e-12


def test_learned_limiter_keeps_face_values_in_range(cuda):
    """Any network output keeps the slope within [0, alpha]: the limited face-centroid values stay within the
    neighbours' range (checked on the CPU from the sweep's own inputs)."""
    import torch

    from conftest import jittered_mesh
    from luna_cpp_b200 import hydro
    from luna_cpp_b200.learned import LimiterMLP
    from luna_cpp_b200.problems import rough_state

    mesh = jittered_mesh(12)
    q0 = rough_state(mesh.n_cells) * mesh.volume[:, None]
    fv = hydro.FiniteVolume(mesh)
    fv.set_state(q0)
    feats, alpha, g0 = fv.limiter_inputs()
    net = LimiterMLP(seed=5)
    fv.set_limiter("learned", net.params)
    fv.set_state(q0)
    fv.time_step(0.3)
    g = fv.gradients()
    alpha = alpha.cpu().numpy()
    g0 = g0.cpu().numpy()
    logits = net.forward(feats).cpu().numpy()
    phi = alpha * (1 / (1 + np.exp(-logits[:, :5])))
    want = g0.reshape(-1, 5, 3) * phi[:, :, None]
    assert np.max(np.abs(g.reshape(-1, 5, 3) - want)) <= 1e-6 * np.max(np.abs(want)) + 1e-300
    assert np.all(phi >= 0) and np.all(phi <= alpha + 1e-7)


def test_learned_limiter_leaves_round_off_cells_at_factor_one(cuda):
    """In a step the network runs only on the cells whose slopes are not round-off (compact rows); the others keep the
    factor 1, as the plain limiter does there. On the point blast most cells are round-off (alpha = 1 for every
    variable in the dense inputs); the step's gradients are g0 there and g0 alpha sigmoid(logits) elsewhere."""
    from conftest import jittered_mesh
    from luna_cpp_b200 import hydro
    from luna_cpp_b200.learned import LimiterMLP
    from luna_cpp_b200.problems import point_blast

    mesh = jittered_mesh(16)
    q0 = point_blast(mesh)
    fv = hydro.FiniteVolume(mesh)
    fv.set_state(q0)
    feats, alpha, g0 = fv.limiter_inputs()
    net = LimiterMLP(seed=3)
    fv.set_limiter("learned", net.params)
    fv.set_state(q0)
    fv.time_step(0.3)
    g = fv.gradients().reshape(-1, 5, 3)
    alpha = alpha.cpu().numpy()
    round_off = np.all(alpha == 1.0, axis=1)
    assert round_off.sum() > mesh.n_cells // 2 and (~round_off).sum() > 0
    logits = net.forward(feats).cpu().numpy()
    phi = np.where(round_off[:, None], 1.0, alpha * (1 / (1 + np.exp(-logits[:, :5]))))
    want = g0.cpu().numpy().reshape(-1, 5, 3) * phi[:, :, None]
    assert np.max(np.abs(g - want)) <= 1e-6 * np.max(np.abs(want)) + 1e-300


@pytest.mark.parametrize("n", [1, 127, 128, 129, 300_000])
def test_tensor_core_forward_tiles(cuda, n):
    """The tcgen05 forward (tiles of 128 rows, a grid-stride loop once the rows outnumber 296 tiles) against the numpy
    oracle at row counts around a tile and at many tiles a CTA."""
    import torch

    from luna_cpp_b200.learned import LimiterMLP, init_params

    x, _, _ = data(n, seed=n % 97)
    p = init_params(7)
    net = LimiterMLP(p)
    logits = net.forward(torch.tensor(x, device="cuda").to(torch.bfloat16)).cpu().numpy()
    want, _ = M.forward(p, x)
    assert logits.shape == (n, M.OUT)
    assert rel(logits, want) < 2e-3


def test_tensor_core_wait_that_runs_out_reports_a_timeout(cuda):
    """The bounded MMA-completion wait made to run out (no polls allowed): luna_mlp_forward returns LUNA_ETIMEOUT, the
    CTAs still wait for their MMAs in flight (full bound) and free tensor memory, and the context stays usable: the next
    forward with the default limit matches the oracle. Nothing faults or hangs: the MMAs complete; only the first wait
    is told to give up."""
    import ctypes

    import torch

    from luna_cpp_b200 import hydro
    from luna_cpp_b200.learned import LimiterMLP, init_params

    lib = hydro.lib()
    x, _, _ = data(1000, seed=5)
    p = init_params(3)
    net = LimiterMLP(p)
    feats = torch.tensor(x, device="cuda").to(torch.bfloat16)
    logits = torch.empty((1000, M.OUT), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    previous = lib.luna_mlp_set_wait_limit(0)
    try:
        status = lib.luna_mlp_forward(ctypes.c_void_p(net.params.data_ptr()), ctypes.c_void_p(feats.data_ptr()), 1000,
                                      ctypes.c_void_p(logits.data_ptr()), ctypes.c_void_p(stream))
    finally:
        lib.luna_mlp_set_wait_limit(previous)
    assert status == 5, (status, lib.luna_last_error())  # LUNA_ETIMEOUT
    assert b"gave up" in lib.luna_last_error()
    want, _ = M.forward(p, x)
    assert rel(net.forward(feats).cpu().numpy(), want) < 2e-3
