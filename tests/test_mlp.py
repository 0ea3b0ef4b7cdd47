"""Warm-start MLP: the oracle's backward pass against central differences (CPU) and the
tensor-core kernels against the oracle (GPU).

Bars: FP64 analytic gradient within 1e-4 relative of central differences (step 1e-5); GPU forward
outputs within 2e-3 relative (max-norm) of the oracle, which rounds to BF16 at the same
points as the kernels; GPU gradients within 5e-3 relative (norm-wise per parameter
block); AdamW update within 1e-6 of the oracle's given the same gradient."""
import numpy as np
import pytest

from oracle import mlp_oracle as mo


def test_oracle_backward_matches_finite_differences():
    for seed in (0, 1, 2):
        assert mo.fd_check(seed=seed, h=1e-5) < 1e-4
    assert mo.fd_check(seed=3, n=17, h=1e-5) < 1e-4


def test_bf16_rounding_helper():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5e-3, 65504.0])
    r = mo.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == 1.0 + 2 ** -7
    assert abs(r[3] - x[3]) <= 2 ** -8 * abs(x[3])


def test_product_init_matches_oracle_init():
    from dissolve_tp import mlp
    assert np.array_equal(mlp.initial_params(3), mo.init_params(3))
    assert mlp.P == mo.P


def _random_setup(seed, rows):
    rng = np.random.default_rng(seed)
    p = mo.init_params(seed).astype(np.float64)
    p[mo.OFF_B1:mo.OFF_W2] = rng.normal(0, 0.2, mo.H)
    p[mo.OFF_B2:mo.OFF_W3] = rng.normal(0, 0.2, mo.H)
    p[mo.OFF_B3] = 0.1
    p = p.astype(np.float32)
    X = rng.normal(0, 1, (rows, mo.IN))
    X[:, 7] = 1.0
    X[:, mo.NFEAT:] = 0.0
    X = mo.bf16(X)
    T = rng.normal(0, 1, rows).astype(np.float32)
    return p, X, T


@pytest.mark.gpu
@pytest.mark.parametrize("rows", [64, 1000, 20011])
def test_gpu_gradient_matches_oracle(cuda_device, rows):
    import torch

    from dissolve_tp.mlp import WarmStartMLP
    p, X, T = _random_setup(7, rows)
    m = WarmStartMLP(cuda_device, capacity_rows=rows)
    m.params.copy_(torch.from_numpy(p))
    m.X[:rows].copy_(torch.from_numpy(X.astype(np.float32)).to(torch.bfloat16))
    m.T[:rows].copy_(torch.from_numpy(T))
    m.rows = rows
    g, loss = m.gradient(0, rows)
    g = g.cpu().numpy().astype(np.float64)
    lo, go = mo.loss_and_grad(p, X, T.astype(np.float64))
    assert abs(float(loss.item()) - lo) <= 2e-3 * lo
    blocks = {"W1": (mo.OFF_W1, mo.OFF_B1), "b1": (mo.OFF_B1, mo.OFF_W2),
              "W2": (mo.OFF_W2, mo.OFF_B2), "b2": (mo.OFF_B2, mo.OFF_W3),
              "w3": (mo.OFF_W3, mo.OFF_B3), "b3": (mo.OFF_B3, mo.P)}
    for name, (a, b) in blocks.items():
        err = np.linalg.norm(g[a:b] - go[a:b]) / max(np.linalg.norm(go[a:b]), 1e-30)
        assert err < 5e-3, (name, err)
    # determinism: same inputs -> same gradient bits
    g2, _ = m.gradient(0, rows)
    assert np.array_equal(g2.cpu().numpy().astype(np.float64), g)


@pytest.mark.gpu
def test_gpu_adamw_step_matches_oracle(cuda_device):
    import torch

    from dissolve_tp.mlp import WarmStartMLP
    rows = 5000
    p, X, T = _random_setup(11, rows)
    m = WarmStartMLP(cuda_device, capacity_rows=rows)
    m.params.copy_(torch.from_numpy(p))
    m.X[:rows].copy_(torch.from_numpy(X.astype(np.float32)).to(torch.bfloat16))
    m.T[:rows].copy_(torch.from_numpy(T))
    m.rows = rows
    g, _ = m.gradient(0, rows)
    g = g.cpu().numpy().astype(np.float64)
    m.train(steps=1, batch_rows=rows, lr=1e-3, wd=1e-4)
    # train() uses a cosine schedule: lr at step 0 is the full lr
    po, _, _ = mo.adamw(p.astype(np.float64), np.zeros(mo.P), np.zeros(mo.P), g, 1, 1e-3)
    assert np.abs(m.params.cpu().numpy() - po).max() < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("base", ["previous", "extrapolate"])
def test_gpu_forward_from_fields_matches_oracle(cuda_device, base):
    import torch

    from dissolve_tp.mlp import WarmStartMLP
    rng = np.random.default_rng(5)
    V, S, ld = 3001, 3, 4
    U = rng.uniform(0, 1, (V, S))
    Up = U + rng.normal(0, 0.05, (V, S))
    phi = rng.normal(0, 1, V)
    ng = np.abs(rng.normal(1, 0.2, V))
    D, k = [1.0, 1.0, 2.6], [0.5, 0.0, 0.2]
    m = WarmStartMLP(cuda_device, base=base)
    m.mean = np.array([0.0, 1.0, 0.5, 0.5, 0.0, 0.3, 0.2, 0.0, 0.1, -0.1])
    m.istd = np.array([1.0, 5.0, 3.0, 3.0, 20.0, 2.0, 4.0, 1.0, 0.5, 2.0])
    m.sigma = 0.01
    Ud = torch.zeros((V, ld), dtype=torch.float64, device=cuda_device)
    Upd = torch.zeros_like(Ud)
    Ud[:, :S] = torch.from_numpy(U)
    Upd[:, :S] = torch.from_numpy(Up)
    phid = torch.from_numpy(phi).to(cuda_device)
    ngd = torch.from_numpy(ng).to(cuda_device)
    oU, oDU = rng.normal(0, 2, (V, S)), rng.normal(0, 0.5, (V, S))
    ops = []
    for o in (oU, oDU):
        t = torch.zeros((V, ld), dtype=torch.float64, device=cuda_device)
        t[:, :S] = torch.from_numpy(o)
        ops.append(t)
    y = m.predict(Ud, Upd, S, ld, D, k, phid, ngd, ops=ops).cpu().numpy().astype(np.float64)
    X = mo.features(U, Up, phi, ng, np.log(D), k, m.mean, m.istd, oU, oDU)
    yo, _ = mo.forward(m.params.cpu().numpy(), X)
    assert np.abs(y - yo).max() <= 2e-3 * np.abs(yo).max()
    x = torch.zeros_like(Ud)
    m.predict(Ud, Upd, S, ld, D, k, phid, ngd, x_out=x, ops=ops)
    b = 2.0 * U - Up if base == "extrapolate" else U
    xo = b + m.sigma * yo.reshape(V, S)
    assert np.abs(x[:, :S].cpu().numpy() - xo).max() <= 2e-3 * m.sigma * np.abs(yo).max() + 1e-12
    # the tensor-core inference never gave up waiting (the call's own status word)
    assert not m.timed_out()
    # training target: (u^{n+1} - base) / sigma, rounded to FP32
    Un1 = U + rng.normal(0, 0.02, (V, S))
    Un1d = torch.zeros_like(Ud)
    Un1d[:, :S] = torch.from_numpy(Un1)
    m.add_pairs([(Upd, Ud, Un1d)], S, ld, D, k, phid, ngd, ops=[ops])
    To = ((Un1 - b) / m.sigma).reshape(-1)
    assert np.abs(m.T[: V * S].cpu().numpy() - To).max() <= 1e-6 * np.abs(To).max()


@pytest.mark.gpu
def test_learned_guess_reduces_iterations(cuda_device):
    """Train on one trajectory, evaluate on another: same tolerance, fewer iterations."""
    from dissolve_tp import mlp
    from dissolve_tp.mesh import kuhn_cube
    from dissolve_tp.transport import BatchedTransport
    m = kuhn_cube(16, 0.2, seed=0)
    rng = np.random.default_rng(1)
    coef = np.exp(0.3 * rng.standard_normal(m.n_cells))
    D, K, dt = (1.0, 1.0, 2.6), (0.5, 0.0, 0.2), 0.02
    u_eval = np.random.default_rng(2).uniform(0, 1, (m.n_verts, 3))
    runs = {}
    for guess in ("previous", "learned"):
        tr = BatchedTransport(m, coef, D, K, dt, rtol=1e-8, inner_fp32=True)
        if guess == "learned":
            mlp.attach_trained_predictor(tr, m, coef, u_eval, D, K, dt, train_steps=10,
                                         epochs=300)
        tr.set_state(u_eval)
        its = []
        for _ in range(8):
            r = tr.step()
            assert r["converged"], r
            its.append(r["iterations"])
        runs[guess] = (its, tr.state())
    prev, learned = runs["previous"], runs["learned"]
    assert sum(learned[0][1:]) < sum(prev[0][1:]), (prev[0], learned[0])
    # the guess only changes the iteration count: both solves meet the same tolerance
    assert np.linalg.norm(learned[1] - prev[1]) / np.linalg.norm(prev[1]) < 1e-7


@pytest.mark.gpu
@pytest.mark.parametrize("with_bc,n_dirs", [(False, 2), (False, 6), (True, 3), (True, 5)])
def test_guess_projection_matches_galerkin_solve(cuda_device, with_bc, n_dirs):
    """tp_guess_project against the Galerkin solve done with scipy on the same operator;
    the projected guess is never worse than u^n in the energy norm."""
    import ctypes

    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    import torch

    from dissolve_tp import _lib
    from dissolve_tp._lib import call
    from dissolve_tp.device import ptr, stream_handle
    from dissolve_tp.mesh import face_dofs, kuhn_cube
    from dissolve_tp.transport import BatchedTransport
    m = kuhn_cube(8, 0.2, seed=0)
    coef = np.exp(0.3 * np.random.default_rng(1).standard_normal(m.n_cells))
    D, K, S = (1.0, 1.0, 2.6), (0.5, 0.0, 0.2), 3
    bcv = [1.0, 0.5, 0.2]
    bc = face_dofs(m, 0, "min") if with_bc else None
    tr = BatchedTransport(m, coef, D, K, 0.02, bc_dofs=bc, bc_values=bcv if with_bc else None)
    rng = np.random.default_rng(3)
    U = rng.uniform(0, 1, (m.n_verts, S))
    if with_bc:
        U[bc] = bcv
    tr.set_state(U)
    tr.assemble_operator()
    tr.assemble_rhs()
    dn = [rng.normal(0, 0.02 * (k + 1), U.shape) for k in range(n_dirs)]
    dirs = []
    for a in dn:
        t = torch.zeros_like(tr.U)
        t[:, :S] = torch.from_numpy(a)
        dirs.append(t)
    opU, _ = tr.operator_images(tr.U, tr.U)
    x = torch.zeros_like(tr.U)
    work = torch.empty(int(_lib.lib.tp_guess_project_workspace_doubles()), dtype=torch.float64,
                       device=cuda_device)
    arr = (ctypes.c_void_p * n_dirs)(*[ptr(d) for d in dirs])
    call("tp_guess_project", ctypes.byref(tr.stiff_op.struct), ptr(tr.D64), ptr(tr.bc_mask),
         ptr(tr.solver.b), ptr(tr.U), ptr(opU), n_dirs, arr, None, ptr(x), ptr(work),
         stream_handle())
    xg = x.cpu().numpy()
    n = m.n_verts
    Km = sp.csr_matrix((tr.K64.cpu().numpy(), tr.dm.indices[: tr.dm.nnz].cpu().numpy(),
                        tr.dm.indptr.cpu().numpy()), shape=(n, n))
    dg = tr.D64.cpu().numpy()
    b = tr.solver.b.cpu().numpy()
    free = np.ones(n, bool)
    if with_bc:
        free[bc] = False
    for s in range(S):
        A = (D[s] * Km + sp.diags(dg[:, s])).tocsr()
        AF = A[free][:, free]
        u = U[:, s]
        ds = [np.where(free, a[:, s], 0.0) for a in dn]
        r0 = (b[:, s] - A @ u)[free]
        Ad = [(A @ d)[free] for d in ds]
        G = np.array([[di[free] @ Aj for Aj in Ad] for di in ds])
        c = np.linalg.solve(0.5 * (G + G.T), [di[free] @ r0 for di in ds])
        xr = np.where(free, u + sum(ci * di for ci, di in zip(c, ds)), b[:, s])
        assert np.abs(xg[:, s] - xr).max() <= 1e-9 * np.abs(xr).max(), s
        # energy norm of the free-row error against the exact solution
        xs = u.copy()
        xs[free] = spla.spsolve(AF.tocsc(), b[free, s] - (A[free][:, ~free] @ u[~free]
                                                          if with_bc else 0.0))
        e_new, e_old = (xg[:, s] - xs)[free], (u - xs)[free]
        assert e_new @ (AF @ e_new) <= e_old @ (AF @ e_old) * (1 + 1e-12)
    # a repeated direction is dropped (its pivot vanishes), the result is unchanged
    arr2 = (ctypes.c_void_p * 2)(ptr(dirs[0]), ptr(dirs[0]))
    x1, x2 = torch.zeros_like(x), torch.zeros_like(x)
    arr1 = (ctypes.c_void_p * 1)(ptr(dirs[0]))
    call("tp_guess_project", ctypes.byref(tr.stiff_op.struct), ptr(tr.D64), ptr(tr.bc_mask),
         ptr(tr.solver.b), ptr(tr.U), ptr(opU), 1, arr1, None, ptr(x1), ptr(work),
         stream_handle())
    call("tp_guess_project", ctypes.byref(tr.stiff_op.struct), ptr(tr.D64), ptr(tr.bc_mask),
         ptr(tr.solver.b), ptr(tr.U), ptr(opU), 2, arr2, None, ptr(x2), ptr(work),
         stream_handle())
    assert torch.equal(x1, x2)
    if not with_bc:
        # every other direction's image supplied precomputed: same guess to rounding
        x3 = torch.zeros_like(x)
        imgs = [tr.operator_images(tr.U + d, tr.U, fresh=True)[1] for d in dirs]
        iarr = (ctypes.c_void_p * n_dirs)(*[ptr(im) if k % 2 == 0 else None
                                            for k, im in enumerate(imgs)])
        call("tp_guess_project", ctypes.byref(tr.stiff_op.struct), ptr(tr.D64), None,
             ptr(tr.solver.b), ptr(tr.U), ptr(opU), n_dirs, arr, iarr, ptr(x3), ptr(work),
             stream_handle())
        assert (x3 - x).abs().max().item() <= 1e-9 * x.abs().max().item()


@pytest.mark.gpu
def test_inference_wait_runs_out_then_recovers(cuda_device):
    """Tensor-core waits that run out (the test hook issues no MMA and commits nothing, so
    no mbarrier phase ever completes) end the inference with its status word set and its
    rows untouched, and free the tensor memory: the next launch predicts normally."""
    import ctypes

    import torch

    from dissolve_tp import _lib
    from dissolve_tp.mlp import WarmStartMLP
    rng = np.random.default_rng(9)
    V, S, ld = 2000, 3, 4
    Ud = torch.zeros((V, ld), dtype=torch.float64, device=cuda_device)
    Ud[:, :S] = torch.from_numpy(rng.uniform(0, 1, (V, S)))
    Upd = Ud + 0.01
    D, k = [1.0, 1.0, 2.6], [0.5, 0.0, 0.2]
    m = WarmStartMLP(cuda_device)
    m.sigma = 0.01
    want = torch.zeros_like(Ud)
    m.predict(Ud, Upd, S, ld, D, k, x_out=want)
    assert not m.timed_out()
    x = torch.full_like(Ud, 7.0)
    _lib.call("tp_mlp_set_wait_limit", 1 << 12, 1)
    try:
        m.predict(Ud, Upd, S, ld, D, k, x_out=x)
        assert m.timed_out()
        assert torch.all(x == 7.0)
    finally:
        _lib.call("tp_mlp_set_wait_limit", 0, 0)
    flag = ctypes.c_int(-1)
    _lib.call("tp_mlp_tensor_status", ctypes.byref(flag), None)
    assert flag.value == 1  # sticky since load
    m.predict(Ud, Upd, S, ld, D, k, x_out=x)
    assert not m.timed_out()
    assert torch.equal(x[:, :S], want[:, :S])


@pytest.mark.gpu
@pytest.mark.parametrize("engine", ["cgt", "pipe"])
def test_network_adds_to_the_projection_in_the_early_steps(cuda_device, monkeypatch, engine):
    """Ablation of the learned guess on the 32^3 version of the benchmarked workload: the
    energy-norm projection over past step increments with the trained network's correction
    as one more direction needs fewer CG iterations over steps 2-6 than the same projection
    without the network (the network's own gain), and than the previous-step guess of the
    reference (numerics/solvers.py:367).  Every solve runs to the same tolerance, so the
    guess changes the iteration count only.  With the Chronopoulos-Gear engine ("cgt"),
    which keeps its direction across the FP64 refreshes, the projection alone also beats
    the previous-step guess; the pipelined engine ("pipe") restarts at every refresh, so
    its iteration count moves in whole refresh cycles (a factor 1e3 of the residual each)
    and a modestly better start often saves none: only the network's direction moves it."""
    from dissolve_tp import mlp
    from dissolve_tp.mesh import kuhn_cube
    from dissolve_tp.transport import BatchedTransport
    monkeypatch.setenv("DISSOLVE_PCG_PIPE", "1" if engine == "pipe" else "0")
    m = kuhn_cube(32, 0.2, seed=0)
    coef = np.exp(0.3 * np.random.default_rng(1).standard_normal(m.n_cells))
    u0 = np.random.default_rng(2).uniform(0, 1, (m.n_verts, 3))
    D, kk, dt = (1.0, 1.0, 2.6), (0.5, 0.0, 0.2), 0.02
    tr = BatchedTransport(m, coef, D, kk, dt, rtol=1e-8, inner_fp32=True)
    assert mlp.attach_trained_predictor(tr, m, coef, u0, D, kk, dt, train_steps=6, epochs=200)
    its, states = {}, {}
    for name, guess in (("previous", "previous"), ("projection", "project"),
                        ("projection_and_network", "learned")):
        tr.guess = guess
        tr.set_state(u0)
        res = [tr.step() for _ in range(6)]
        assert all(r["converged"] for r in res)
        its[name] = sum(int(r["iterations"]) for r in res[1:])
        states[name] = tr.state()
    assert tr.solver.engine()["pipelined"] == (engine == "pipe")
    assert its["projection_and_network"] <= 0.98 * its["projection"], its
    assert its["projection_and_network"] < its["previous"], its
    if engine == "cgt":
        assert its["projection"] < its["previous"], its
    ref = states["previous"]
    for name in ("projection", "projection_and_network"):
        assert np.linalg.norm(states[name] - ref) / np.linalg.norm(ref) < 1e-7
