"""The hand-written adjoint against forward-mode dual numbers of the same
discrete program (the CPU checker), central differences, and the plain path.

Tolerance of the gradient checks: 1e-6 relative (Float64)."""
import numpy as np
import pytest

import conftest
from _oracle import oracle_adjoint_dual
from scenarios import adjoint_problem

cbm = conftest.cbm
pytestmark = pytest.mark.gpu


def small_problem(abi, N=400, steps=60, seed=31):
    L = (N / 0.128) ** (1 / 3)  # the density of the 65536-agent problem in [0,80]^3
    kw, x0, star = adjoint_problem(abi, N=N, L=L, seed=seed, steps=steps)
    return kw, x0, star


def target_for(abi, kw, x0, star, steps):
    k, a, rho = star
    fw = cbm.Adjoint(abi.make_config(**dict(kw, k_rep=k, k_att=a, r_rep=rho, r_att=1.5 * rho,
                                            cell_edge=max(kw["cell_edge"], 1.5 * rho))))
    return fw.forward(x0, steps)


def test_forward_map_is_the_plain_path(gpu_lib, abi):
    kw, x0, _ = small_problem(abi, N=800, steps=50)
    adj = cbm.Adjoint(abi.make_config(**kw))
    xT = adj.forward(x0, 50)
    g = cbm.Context(abi.make_config(**kw))
    g.upload(dict(x=x0[0], y=x0[1], z=x0[2]))
    g.step(50)
    s = g.download()
    for d, k in enumerate("xyz"):
        np.testing.assert_array_equal(xT[d], s[k])


def test_gradients_match_dual_numbers(gpu_lib, abi):
    steps = 60
    kw, x0, star = small_problem(abi, steps=steps)
    tgt = target_for(abi, kw, x0, star, steps)
    adj = cbm.Adjoint(abi.make_config(**kw))
    res = adj.run(x0, tgt, steps, checkpoint_every=20)
    seeds = [(5, 0), (17, 1), (123, 2), (321, 0), (399, 1)]
    loss, g, dx = oracle_adjoint_dual(abi, abi.make_config(**kw), x0, tgt, steps, seeds=seeds)
    assert abs(res["loss"] - loss) <= 1e-10 * abs(loss)
    np.testing.assert_allclose(res["dtheta"], g, rtol=1e-6)
    scale = max(np.max(np.abs(d)) for d in res["dx0"])
    for s, (i, ax) in enumerate(seeds):
        assert abs(res["dx0"][ax][i] - dx[s]) <= 1e-6 * scale


def test_checkpoint_interval_does_not_change_the_gradient(gpu_lib, abi):
    steps = 45
    kw, x0, star = small_problem(abi, N=300, steps=steps, seed=33)
    tgt = target_for(abi, kw, x0, star, steps)
    adj = cbm.Adjoint(abi.make_config(**kw))
    ref = adj.run(x0, tgt, steps, checkpoint_every=1)
    for K in (7, 20, 45, 100):
        r = adj.run(x0, tgt, steps, checkpoint_every=K)
        assert r["loss"] == ref["loss"]
        np.testing.assert_array_equal(r["dtheta"], ref["dtheta"])
        for d in range(3):
            np.testing.assert_array_equal(r["dx0"][d], ref["dx0"][d])


def test_gradient_matches_central_differences(gpu_lib, abi):
    steps = 30
    kw, x0, star = small_problem(abi, N=200, steps=steps, seed=35)
    tgt = target_for(abi, kw, x0, star, steps)
    res = cbm.Adjoint(abi.make_config(**kw)).run(x0, tgt, steps, checkpoint_every=10)
    for q, name in enumerate(("k_rep", "k_att", "r_rep")):
        h = 1e-6 * kw[name]

        def loss_at(v):
            over = {name: v}
            if name == "r_rep":
                over["r_att"] = kw["r_att"]  # the cutoff is held fixed in the derivative
            a = cbm.Adjoint(abi.make_config(**dict(kw, **over)))
            return a.run(x0, tgt, steps, checkpoint_every=10, want_dx0=False)["loss"]

        fd = (loss_at(kw[name] + h) - loss_at(kw[name] - h)) / (2 * h)
        assert abs(fd - res["dtheta"][q]) <= 1e-5 * abs(res["dtheta"][q]), (name, fd, res["dtheta"][q])
