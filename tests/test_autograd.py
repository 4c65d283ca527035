"""The differentiable solve (basilisk_b200.autograd) against central finite
differences and against a dense FP64 torch.linalg.solve of the same discrete
operator.  The relative tolerance of every gradient comparison is 1e-6."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-6


def dense_operator(n, alpha, lam, delta, periodic, dirichlet):
    """L as a dense n^2 x n^2 torch matrix (2D), differentiable in alpha and
    lam: (L a)_p = lam_p a_p + sum_f alpha_f (a_nb - a_p)/Delta^2; a
    homogeneous Dirichlet boundary face adds -2 alpha_f/Delta^2 to the
    diagonal, a Neumann one nothing."""
    import torch
    N = n * n
    dev = alpha[0].device
    rows, cols, vals = [], [], []
    idx = torch.arange(N, device=dev).reshape(n, n)
    inv = 1.0 / delta ** 2
    for d in range(2):
        a = alpha[d]
        for f in range(n + 1):
            sl = [slice(None), slice(None)]
            sl[d] = f
            af = a[tuple(sl)] * inv                       # n values along the other axis
            if periodic[d]:
                if f == n:
                    continue
                p = idx.select(d, (f - 1) % n)
                q = idx.select(d, f)
            else:
                p = idx.select(d, f - 1) if f >= 1 else None
                q = idx.select(d, f) if f <= n - 1 else None
            if p is not None and q is not None:
                rows += [p, p, q, q]; cols += [p, q, q, p]; vals += [-af, af, -af, af]
            else:
                c = p if p is not None else q
                if dirichlet:
                    rows.append(c); cols.append(c); vals.append(-2.0 * af)
    r = torch.cat(rows); c = torch.cat(cols); v = torch.cat(vals)
    L = torch.zeros(N * N, dtype=torch.float64, device=dev)
    L = L.index_add(0, r * N + c, v).reshape(N, N)
    if lam is not None:
        L = L + torch.diag(lam.reshape(-1))
    return L


def make_problem(n_depth, periodic, dirichlet, lam, precision="fp64", tol=1e-13):
    from basilisk_b200.autograd import Problem
    bc = {} if periodic == (0, 1) else {s: ("dirichlet" if dirichlet else "neumann", 0.0)
                                         for s in range(4) if s // 2 not in periodic}
    return Problem(2, n_depth, periodic=periodic, bc=bc, tolerance=tol, precision=precision,
                   alpha=True, lam=lam)


def random_inputs(n, seed, lam=True):
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    b = torch.randn(n, n, generator=g, dtype=torch.float64).cuda()
    kx = torch.randn(n + 1, n, generator=g, dtype=torch.float64).cuda() * 0.5
    ky = torch.randn(n, n + 1, generator=g, dtype=torch.float64).cuda() * 0.5
    la = (-1.0 - torch.rand(n, n, generator=g, dtype=torch.float64).cuda()) if lam else None
    aobs = torch.randn(n, n, generator=g, dtype=torch.float64).cuda()
    return b, kx, ky, la, aobs


@pytest.mark.parametrize("case", ["dirichlet", "periodic_helmholtz", "neumann_helmholtz"])
def test_gradient_matches_dense_solve(case):
    """32x32: gradients of 0.5|a - a_obs|^2 in b, alpha and lambda against
    autograd through a dense torch.linalg.solve."""
    import torch
    from basilisk_b200.autograd import solve
    depth, n = 5, 32
    periodic = (0, 1) if case == "periodic_helmholtz" else ()
    prob = make_problem(depth, periodic, case == "dirichlet", lam=True)
    b, kx, ky, la, aobs = random_inputs(n, 1)
    if case == "dirichlet":
        la = la * 0.0 - 0.0                          # Poisson
    ax, ay = torch.exp(kx), torch.exp(ky)
    if periodic:
        ax = ax.clone(); ay = ay.clone()
        ax[n] = ax[0]; ay[:, n] = ay[:, 0]           # face n is the image of face 0
    ins = [t.clone().requires_grad_(True) for t in (b, ax, ay, la)]
    a = solve(prob, ins[0], alpha=[ins[1], ins[2]], lam=ins[3])
    loss = 0.5 * ((a - aobs) ** 2).sum()
    g_ours = torch.autograd.grad(loss, ins)
    ref = [t.clone().requires_grad_(True) for t in (b, ax, ay, la)]
    L = dense_operator(n, [ref[1], ref[2]], ref[3], 1.0 / n, (0 in periodic, 1 in periodic),
                       case == "dirichlet")
    ad = torch.linalg.solve(L, ref[0].reshape(-1)).reshape(n, n)
    assert torch.allclose(a.detach(), ad.detach(), rtol=0, atol=1e-9 * ad.abs().max().item())
    loss_d = 0.5 * ((ad - aobs) ** 2).sum()
    g_ref = torch.autograd.grad(loss_d, ref)
    for name, go, gr in zip(("b", "alpha_x", "alpha_y", "lambda"), g_ours, g_ref):
        if periodic and name == "alpha_x":
            go, gr = go[:n], gr[:n]
        if periodic and name == "alpha_y":
            go, gr = go[:, :n], gr[:, :n]
        err = (go - gr).abs().max().item() / gr.abs().max().item()
        assert err < RTOL, (name, err)
    prob.close()


def test_singular_periodic_poisson_matches_pinned_dense_solve():
    """32x32 periodic pure Poisson (lambda = 0, L singular): b with a non-zero
    mean and a loss that is not invariant under a + const.  The reference
    map is the zero-mean solution of the zero-mean projection of b, i.e. a
    dense solve of (L + J/N) a = b - mean(b), J the all-ones matrix (it
    pins mean(a) = 0 and is regular); gradients in b and alpha agree to
    1e-6 relative."""
    import torch
    from basilisk_b200.autograd import solve
    depth, n = 5, 32
    prob = make_problem(depth, (0, 1), False, lam=False)
    assert prob.singular
    b, kx, ky, _, aobs = random_inputs(n, 7, lam=False)
    b = b + 0.3                                       # incompatible as given
    ax, ay = torch.exp(kx), torch.exp(ky)
    ax[n] = ax[0]; ay[:, n] = ay[:, 0]
    ins = [t.clone().requires_grad_(True) for t in (b, ax, ay)]
    a = solve(prob, ins[0], alpha=[ins[1], ins[2]])
    assert abs(a.mean().item()) < 1e-12 * a.abs().max().item()
    loss = 0.5 * ((a - aobs) ** 2).sum() + (a * aobs).sum()
    g_ours = torch.autograd.grad(loss, ins)
    ref = [t.clone().requires_grad_(True) for t in (b, ax, ay)]
    L = dense_operator(n, [ref[1], ref[2]], None, 1.0 / n, (True, True), False)
    N = n * n
    Lp = L + torch.full((N, N), 1.0 / N, dtype=torch.float64, device=L.device)
    bz = ref[0] - ref[0].mean()
    ad = torch.linalg.solve(Lp, bz.reshape(-1)).reshape(n, n)
    assert torch.allclose(a.detach(), ad.detach(), rtol=0, atol=1e-9 * ad.abs().max().item())
    loss_d = 0.5 * ((ad - aobs) ** 2).sum() + (ad * aobs).sum()
    g_ref = torch.autograd.grad(loss_d, ref)
    for name, go, gr in zip(("b", "alpha_x", "alpha_y"), g_ours, g_ref):
        if name == "alpha_x":
            go, gr = go[:n], gr[:n]
        if name == "alpha_y":
            go, gr = go[:, :n], gr[:, :n]
        err = (go - gr).abs().max().item() / gr.abs().max().item()
        assert err < RTOL, (name, err)
    prob.close()


def test_unconverged_solve_raises():
    """A solve that cannot reach its tolerance within NITERMAX cycles raises
    instead of returning an unconverged field."""
    import torch
    from basilisk_b200 import _lib
    from basilisk_b200.autograd import solve
    prob = make_problem(4, (), True, lam=False, tol=1e-30)
    b, kx, ky, _, _ = random_inputs(16, 8, lam=False)
    with pytest.raises(_lib.BMGError) as e:
        solve(prob, b, alpha=[torch.exp(kx), torch.exp(ky)])
    assert e.value.status == _lib.ENOTCONV
    prob.close()


def test_gradient_matches_central_differences():
    """Directional derivatives in b, kappa (alpha = exp(kappa) on faces) and
    lambda against central differences with h = 1e-6."""
    import torch
    from basilisk_b200.autograd import solve
    depth, n = 4, 16
    prob = make_problem(depth, (), True, lam=True)
    b, kx, ky, la, aobs = random_inputs(n, 2)

    def loss_of(b, kx, ky, la):
        a = solve(prob, b, alpha=[torch.exp(kx), torch.exp(ky)], lam=la)
        return 0.5 * ((a - aobs) ** 2).sum()

    ins = [t.clone().requires_grad_(True) for t in (b, kx, ky, la)]
    loss0 = loss_of(*ins)
    grads = torch.autograd.grad(loss0, ins)
    g = torch.Generator(device="cpu").manual_seed(3)
    h = 1e-6
    # a central difference of an FP64 loss carries a cancellation error of
    # about eps |loss| / h on top of the O(h^2) truncation error
    noise = 8 * np.finfo(np.float64).eps * abs(loss0.item()) / h
    for k in range(4):
        v = torch.randn(ins[k].shape, generator=g, dtype=torch.float64).cuda()
        plus = [t.detach().clone() for t in ins]
        minus = [t.detach().clone() for t in ins]
        plus[k] += h * v
        minus[k] -= h * v
        with torch.no_grad():
            fd = (loss_of(*plus) - loss_of(*minus)).item() / (2 * h)
        an = (grads[k] * v).sum().item()
        assert abs(fd - an) <= RTOL * abs(an) + noise, (k, fd, an, noise)
    prob.close()


def test_batch_and_mixed_form():
    """A batch of 4 periodic instances (alpha = exp(kappa), b zero-mean): the
    batched gradient equals the per-instance gradients, and the mixed form's
    gradients agree with FP64 to 1e-6."""
    import torch
    from basilisk_b200.autograd import solve
    depth, n, B = 6, 64, 4
    probs = {p: make_problem(depth, (0, 1), False, lam=False, precision=p, tol=1e-12)
             for p in ("fp64", "mixed")}
    g = torch.Generator(device="cpu").manual_seed(4)
    b = torch.randn(B, n, n, generator=g, dtype=torch.float64).cuda()
    b = b - b.mean(dim=(1, 2), keepdim=True)
    kx = torch.randn(B, n + 1, n, generator=g, dtype=torch.float64).cuda() * 0.3
    ky = torch.randn(B, n, n + 1, generator=g, dtype=torch.float64).cuda() * 0.3
    kx[:, n] = kx[:, 0]; ky[:, :, n] = ky[:, :, 0]
    aobs = torch.randn(B, n, n, generator=g, dtype=torch.float64).cuda()
    out = {}
    for p, prob in probs.items():
        ins = [t.clone().requires_grad_(True) for t in (b, kx, ky)]
        a = solve(prob, ins[0], alpha=[torch.exp(ins[1]), torch.exp(ins[2])])
        a = a - a.mean(dim=(1, 2), keepdim=True)
        loss = 0.5 * ((a - aobs) ** 2).sum()
        out[p] = torch.autograd.grad(loss, ins)
    for k in range(3):
        err = (out["mixed"][k] - out["fp64"][k]).abs().max() / out["fp64"][k].abs().max()
        assert err.item() < RTOL, (k, err.item())
    # instance 2 alone gives the batch's slice
    ins = [t[2].clone().requires_grad_(True) for t in (b, kx, ky)]
    a = solve(probs["fp64"], ins[0], alpha=[torch.exp(ins[1]), torch.exp(ins[2])])
    a = a - a.mean()
    loss = 0.5 * ((a - aobs[2]) ** 2).sum()
    one = torch.autograd.grad(loss, ins)
    for k in range(3):
        assert torch.allclose(one[k], out["fp64"][k][2], rtol=0,
                              atol=1e-9 * one[k].abs().max().item())
    for prob in probs.values():
        prob.close()


def test_checkpointed_chain():
    """Implicit diffusion steps a_{k+1} = solve(-a_k/dt) with lambda = -1/dt:
    the gradient with a checkpoint every 3 steps equals the plain one."""
    import torch
    from basilisk_b200.autograd import solve, chain
    depth, n, dt = 5, 32, 1e-3
    prob = make_problem(depth, (0, 1), False, lam=True, tol=1e-12)
    g = torch.Generator(device="cpu").manual_seed(5)
    a0 = torch.randn(n, n, generator=g, dtype=torch.float64).cuda()
    ax = torch.full((n + 1, n), 1e-2, dtype=torch.float64, device="cuda")
    ay = torch.full((n, n + 1), 1e-2, dtype=torch.float64, device="cuda")
    lam = torch.full((n, n), -1.0 / dt, dtype=torch.float64, device="cuda")

    def step(a):
        return solve(prob, -a / dt, alpha=[ax, ay], lam=lam)

    grads = []
    for every in (1, 3):
        x = a0.clone().requires_grad_(True)
        y = chain(step, x, 7, every=every)
        loss = (y ** 2).sum()
        grads.append(torch.autograd.grad(loss, x)[0])
    assert torch.allclose(grads[0], grads[1], rtol=0, atol=1e-12 * grads[0].abs().max().item())
    prob.close()


def test_lanes_give_the_single_lane_results():
    """A batch of 6 periodic instances on a Problem with 3 lanes (three grids,
    three streams, three host threads) gives the single-lane solutions and
    gradients bit for bit."""
    import torch
    from basilisk_b200.autograd import solve
    depth, n, B = 6, 64, 6
    g = torch.Generator(device="cpu").manual_seed(12)
    b = torch.randn(B, n, n, generator=g, dtype=torch.float64).cuda()
    kx = torch.randn(B, n + 1, n, generator=g, dtype=torch.float64).cuda() * 0.3
    ky = torch.randn(B, n, n + 1, generator=g, dtype=torch.float64).cuda() * 0.3
    kx[:, n] = kx[:, 0]; ky[:, :, n] = ky[:, :, 0]
    aobs = torch.randn(B, n, n, generator=g, dtype=torch.float64).cuda()
    out = {}
    for lanes in (1, 3):
        from basilisk_b200.autograd import Problem
        prob = Problem(2, depth, periodic=(0, 1), tolerance=1e-12, alpha=True, lanes=lanes)
        ins = [t.clone().requires_grad_(True) for t in (b, kx, ky)]
        a = solve(prob, ins[0], alpha=[torch.exp(ins[1]), torch.exp(ins[2])])
        loss = 0.5 * ((a - aobs) ** 2).sum()
        out[lanes] = (a.detach(), torch.autograd.grad(loss, ins))
        prob.close()
    assert torch.equal(out[1][0], out[3][0])
    for k in range(3):
        assert torch.equal(out[1][1][k], out[3][1][k]), k
