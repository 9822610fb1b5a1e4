"""GPU tests of the learned warm start: the network kernels against the FP64 restatement in
oracle/mlp_oracle.py (gradient, Adam, initialisation, tensor-core inference), the fallback to the
reference warm start, and the ablation on a stiff workload (a resting 10 x 40 x 10 column).

Bars: gradient within 1e-4 (relative, per parameter block) of the FP64 gradient, the FP32
accumulation over up to 4096 samples being the only difference; Adam updates within 2 % of the
learning rate per parameter; inference within 2e-3 (relative to the output norm) of the same
arithmetic with BF16 inputs, weights and activations, and within 3e-2 of FP64; initialisation
bit-exact."""
import numpy as np
import pytest

from oracle import mlp_oracle as M
from splishsplash_for_cuda_b200 import _capi
from splishsplash_for_cuda_b200.dfsph import DFSPHCUDA
from splishsplash_for_cuda_b200.scene import column_scene, synthetic_scene
from tests._compare import assert_field

pytestmark = pytest.mark.gpu


def _net():
    return DFSPHCUDA(synthetic_scene(1, counts=(6, 6, 6)))


def _case(n, seed=0, pscale=0.3):
    rng = np.random.default_rng(seed)
    p = (rng.normal(size=M.N_PARAMS) * pscale).astype(np.float32)
    s = rng.uniform(0.5, 2.0, size=M.N_IN).astype(np.float32)
    x = rng.normal(size=(n, M.N_IN)).astype(np.float32)
    x[:, 5:] = 0.0
    t = rng.normal(size=(n, M.N_OUT)).astype(np.float32)
    return p, s, x, t


BLOCKS = [(M.W1, M.B1), (M.B1, M.W2), (M.W2, M.B2), (M.B2, M.W3), (M.W3, M.B3), (M.B3, M.N_PARAMS)]


def test_mlp_init_matches_oracle(cuda_lib):
    d = _net()
    for seed in (1, 99):
        d.mlp_reset(seed)
        assert np.array_equal(d.mlp_params(), M.init_params(seed))
    assert d.get_param("mlp_ready") == 0


@pytest.mark.parametrize("n", [1, 127, 1000, 4096])
def test_mlp_gradient_matches_oracle(cuda_lib, n):
    p, s, x, t = _case(n, seed=n)
    d = _net()
    d.set_mlp_params(p)
    d.set_mlp_scales(s, np.ones(2, np.float32))
    g, loss = d.mlp_gradient(x, t)
    lo, go = M.loss_and_grad(p, s, x, t)
    assert abs(loss - lo) <= 1e-5 * lo
    for a, b in BLOCKS:
        ref = go[a:b]
        err = np.linalg.norm(g[a:b] - ref) / max(np.linalg.norm(ref), 1e-30)
        assert err < 1e-4, (a, b, err)


def test_mlp_adam_matches_oracle(cuda_lib):
    p, s, x, t = _case(1000, seed=5)
    d = _net()
    d.set_mlp_params(p)
    d.set_mlp_scales(s, np.ones(2, np.float32))
    lr = 1e-3
    d.mlp_train(x, t, iters=3, learning_rate=lr)
    got = d.mlp_params().astype(np.float64)
    q, m, v = p.astype(np.float64), np.zeros(M.N_PARAMS), np.zeros(M.N_PARAMS)
    for k in range(1, 4):
        _, g = M.loss_and_grad(q.astype(np.float32), s, x, t)
        q, m, v = M.adam(q, m, v, g, lr, k)
    assert np.abs(got - q).max() <= 0.02 * lr
    moved = got - p
    assert np.linalg.norm(moved - (q - p)) <= 1e-2 * np.linalg.norm(q - p)


@pytest.mark.parametrize("n", [16, 129, 1000, 40001, 65536])
def test_mlp_tensor_core_forward(cuda_lib, n):
    """tcgen05 inference (tiles of 128 particles; partial last tiles) against the same arithmetic in
    NumPy. (Inside the solver, 262,144 particles give 2048 tiles on at most 592 persistent CTAs: the
    ablation test below runs that path.)"""
    p, s, x, _ = _case(n, seed=11)
    d = _net()
    d.set_mlp_params(p)
    d.set_mlp_scales(s, np.ones(2, np.float32))
    d.status(clear=True)
    y = d.mlp_forward(x)
    assert d.status() & _capi.ST_MMA_TIMEOUT == 0
    yb = M.forward_bf16(p, s, x)
    y64 = M.forward(p, s, x)
    assert np.linalg.norm(y - yb) <= 2e-3 * np.linalg.norm(yb)
    assert np.linalg.norm(y - y64) <= 3e-2 * np.linalg.norm(y64)


def test_mlp_training_reduces_loss(cuda_lib):
    rng = np.random.default_rng(3)
    x = rng.normal(size=(4096, M.N_IN)).astype(np.float32)
    x[:, 5:] = 0
    t = np.stack([np.tanh(x[:, 0] - 0.5 * x[:, 3]), 0.3 * x[:, 1] * x[:, 4]], axis=1).astype(np.float32)
    d = _net()
    d.mlp_reset(4)
    _, l0 = d.mlp_gradient(x, t)
    d.mlp_train(x, t, iters=300, learning_rate=3e-3)
    _, l1 = d.mlp_gradient(x, t)
    assert l1 < 0.2 * l0


def _run(scene, steps, learned, **kw):
    d = DFSPHCUDA(scene)
    if learned:
        d.set_learned_warm_start(True, **kw)
    its, itv, warm, st_bits = [], [], [], 0
    for _ in range(steps):
        st = d.step()
        its.append(st.iterations)
        itv.append(st.iterations_v)
        warm.append(st.warm_start)
        st_bits |= st.status
    return d, np.array(its), np.array(itv), np.array(warm), st_bits


def test_learned_mode_is_plain_before_training(cuda_lib):
    """With no trained network the learned mode runs the reference warm start: bit-identical states."""
    s = column_scene(counts=(8, 20, 8), time_step=0.002)
    a, ia, va, _, _ = _run(s, 30, False)
    b, ib, vb, wb, _ = _run(s, 30, True, train_interval=0)
    assert np.array_equal(ia, ib) and np.array_equal(va, vb) and not wb.any()
    assert np.array_equal(a.positions(), b.positions())
    assert np.array_equal(a.velocities(), b.velocities())


def test_fallback_restores_reference_warm_start(cuda_lib):
    """A network that predicts the largest pressure everywhere loses every probe once the fluid
    settles (its over-pressure shows as expansion, r < 0, in sum |r|): the step falls back to the
    reference warm start and the states stay bit-identical to the plain mode. (A candidate can tie
    the plain one, e.g. a divergence candidate while no particle has a positive source, or before
    any contact with the floor: the tie keeps the learned one, which then changes nothing.)"""
    s = column_scene(counts=(8, 20, 8), time_step=0.002)
    a, ia, va, _, _ = _run(s, 30, False)
    d = DFSPHCUDA(s)
    d.set_learned_warm_start(True, train_interval=0)
    p = np.zeros(M.N_PARAMS, np.float32)
    p[M.B3:] = -50.0
    d.set_mlp_params(p)
    d.set_mlp_scales(np.ones(8, np.float32), np.ones(2, np.float32))
    ib, vb = [], []
    for _ in range(30):
        st = d.step()
        ib.append(st.iterations)
        vb.append(st.iterations_v)
        assert st.warm_start & 2 == 0
    assert d.get_param("learned_solves_p") == 30 and d.get_param("learned_kept_p") == 0
    assert d.get_param("learned_solves_v") == 30
    assert np.array_equal(ia, ib) and np.array_equal(va, vb)
    assert np.array_equal(a.positions(), d.positions())


def test_learned_warm_start_cuts_iterations_on_stiff_column(cuda_lib):
    """Ablation: same scene, same tolerance, reference warm start vs learned warm start. Both solve
    every step to the tolerance; after the column settles the learned one needs >= 30 % fewer
    pressure iterations."""
    s = column_scene(counts=(10, 40, 10), time_step=0.002, max_error=0.01)
    steps = 300
    p, ip, vp, _, bits_p = _run(s, steps, False)
    d, il, vl, wl, bits_l = _run(s, steps, True, train_interval=25)
    assert bits_l & (_capi.ST_PRESSURE_NOT_CONVERGED | _capi.ST_NONFINITE) == 0
    assert np.isfinite(d.positions()).all()
    win = slice(150, steps)
    mp, ml = ip[win].mean(), il[win].mean()
    print(f"pressure iterations plain {mp:.2f} learned {ml:.2f}; divergence {vp[win].mean():.2f} "
          f"{vl[win].mean():.2f}; learned kept p {d.get_param('learned_kept_p'):.0f}/"
          f"{d.get_param('learned_solves_p'):.0f} v {d.get_param('learned_kept_v'):.0f}/"
          f"{d.get_param('learned_solves_v'):.0f}; trainings {d.get_param('mlp_trainings'):.0f} "
          f"loss {d.get_param('mlp_loss'):.3g}")
    assert ml <= 0.7 * mp
    assert d.get_param("mlp_trainings") >= 10
    # Same fluid: mean density and the column top within a few percent of the plain run.
    rp, rl = p.field("density").astype(np.float64), d.field("density").astype(np.float64)
    assert abs(rl.mean() - rp.mean()) <= 0.05 * rp.mean()
    assert abs(d.positions()[:, 1].max() - p.positions()[:, 1].max()) <= 0.25 * p.positions()[:, 1].max()


def test_gate_off_phases_run_the_plain_passes(cuda_lib):
    """With a margin no solve reaches, the cost gate keeps the learned passes off after its first
    probe window: the run is bit-identical to the plain mode, the network never trains, and every
    step is counted as a plain step."""
    s = column_scene(counts=(8, 20, 8), time_step=0.002)
    a, ia, va, _, _ = _run(s, 60, False)
    d, ib, vb, wb, _ = _run(s, 60, True, gate=True, gate_period=20, gate_window=4, gate_recheck=10,
                            gate_margin=1e9)
    assert np.array_equal(ia, ib) and np.array_equal(va, vb) and not wb.any()
    assert np.array_equal(a.positions(), d.positions()) and np.array_equal(a.velocities(), d.velocities())
    assert d.get_param("gate_learned_steps") == 0 and d.get_param("gate_plain_steps") == 60
    assert d.get_param("mlp_trainings") == 0
    assert d.get_param("gate_last_excess") >= 0.0


def test_gate_turns_learned_passes_on_for_stiff_column(cuda_lib):
    """Once the column has settled its plain solver needs ~20 pressure iterations above the minimum:
    the gate runs the learned passes between its probe windows and keeps most of the iteration cut.
    (While the column still falls the plain solver sits near the minimum, so the first probes keep
    the learned passes off for a few re-check periods.)"""
    s = column_scene(counts=(10, 40, 10), time_step=0.002, max_error=0.01)
    steps = 300
    _, ip, _, _, _ = _run(s, steps, False)
    d, ig, _, wg, bits = _run(s, steps, True, train_interval=25, gate=True, gate_period=100, gate_window=5,
                              gate_recheck=20)
    assert bits & (_capi.ST_PRESSURE_NOT_CONVERGED | _capi.ST_NONFINITE) == 0
    assert d.get_param("gate_last_excess") >= 1.0
    learned_steps, plain_steps = d.get_param("gate_learned_steps"), d.get_param("gate_plain_steps")
    assert learned_steps + plain_steps == steps and learned_steps >= steps // 2
    win = slice(150, steps)
    assert ig[win].mean() <= 0.75 * ip[win].mean()


def test_gate_parameters_and_divergence_off(cuda_lib):
    """Gate parameters are validated and read back; with the divergence solver off the gate measures
    the pressure solve alone, and a gated-off run is still bit-identical to the plain mode."""
    s = column_scene(counts=(8, 20, 8), time_step=0.002)
    d = DFSPHCUDA(s)
    for key, bad in (("gate_period", 0), ("gate_window", 0), ("gate_recheck", 0), ("gate_margin", -1)):
        with pytest.raises(_capi.DfsphError) as e:
            d.set_param(key, bad)
        assert e.value.code == _capi.DFSPH_E_INVALID
    d.set_learned_warm_start(True, gate=True, gate_period=7, gate_window=3, gate_recheck=5, gate_margin=1e9)
    assert (d.get_param("learned_gate"), d.get_param("gate_period"), d.get_param("gate_window"),
            d.get_param("gate_recheck"), d.get_param("gate_margin")) == (1, 7, 3, 5, 1e9)
    assert d.get_param("gate_last_excess") == -1.0
    a = DFSPHCUDA(s)
    for x in (a, d):
        x.setEnableDivergenceSolver(False)
    for _ in range(20):
        sa, sd = a.step(), d.step()
        assert sa.iterations == sd.iterations and sd.iterations_v == 0 and sd.warm_start == 0
    assert np.array_equal(a.positions(), d.positions())
    assert d.get_param("gate_plain_steps") == 20 and d.get_param("gate_last_excess") >= 0.0


def _oracle_features(o, needed_p, needed_v):
    """The five network inputs of the density + alpha pass, restated from the oracle's fields:
    (rho - rho0)/rho0, rho_dot * alpha, neighbours / 64, and the previous step's needed kappa and
    kappa_v (solver.cu density_alpha_kernel)."""
    counts, _ = o.get_neighbors()
    rho0 = o.scene.config.density0
    return np.stack([(o.field("density") - rho0) / rho0, o.field("density_adv") * o.field("factor"),
                     counts.sum(axis=1) / 64.0, needed_p, needed_v], axis=1)


def test_features_match_oracle(cuda_lib):
    """The warm-start network's inputs written by the density + alpha pass, against the oracle on
    the same state: step 1 of a scene with random velocities (+-0.5 m/s), and step 2, whose last two
    inputs are the coefficients step 1 needed. The learned mode runs with the network's correction
    fixed at zero, which makes its first step the plain step (the oracle's). Bars: the neighbour count
    exactly; (rho - rho0)/rho0 within 1e-5 relative (floored at 1e-3 of its largest value); rho_dot *
    alpha and the needed coefficients within 2^-8 relative, floored the same way: the network rounds
    its inputs to BF16 (2^-8 relative), and these are sums of velocity differences that cancel after
    a solve, where FP32 itself errs by ~1e-3 (measured 1.5e-3 on rho_dot * alpha at step 2)."""
    from oracle import Oracle

    s = synthetic_scene(1, counts=(14, 14, 14))
    rng = np.random.default_rng(7)
    s.fluid_velocity = rng.uniform(-0.5, 0.5, size=s.fluid.shape).astype(np.float32)
    d = DFSPHCUDA(s)
    d.set_learned_warm_start(True, train_interval=0)
    d.set_param("learned_base_only", 1)
    o = Oracle(s, 64)
    zeros = np.zeros(s.n_fluid)
    for step in (1, 2):
        if step == 1:
            o.neighbors()
            o.density_alpha(True)
            ref = _oracle_features(o, zeros, zeros)
            o2 = Oracle(s, 64)
            ro = o2.step()
        else:
            need_p, need_v = o2.field("kappa_needed"), o2.field("kappa_v_needed")
            assert np.abs(need_p).max() > 0 and np.abs(need_v).max() > 0
            o2.neighbors()
            o2.density_alpha(True)
            ref = _oracle_features(o2, need_p, need_v)
        st = d.step()
        if step == 1:
            assert st.iterations == ro["iterations"] and st.iterations_v == ro["iterations_v"]
        got = d.field("features").astype(np.float64)
        assert got.shape == (s.n_fluid, 5)
        assert np.array_equal(got[:, 2], ref[:, 2]), step
        assert_field(f"feature 0 step {step}", got[:, 0], ref[:, 0], 1e-5, 1e-3)
        for k in (1, 3, 4):
            assert_field(f"feature {k} step {step}", got[:, k], ref[:, k], 2.0 ** -8, 1e-3)


def test_network_contribution_ablation(cuda_lib):
    """Three arms on the stiff resting column, same scene and tolerance: the reference warm start,
    the needed-coefficient base with the network's correction fixed at zero, and the online-trained
    network on top of that base. Every solve converges in every arm; the base alone cuts the
    pressure iterations by >= 30 %; the trained network's own contribution (base minus trained
    iterations) is measured and must not cost more than 10 % of the base's iterations."""
    s = column_scene(counts=(10, 40, 10), time_step=0.002, max_error=0.01)
    steps = 300
    _, ip, _, _, bp = _run(s, steps, False)
    db = DFSPHCUDA(s)
    db.set_learned_warm_start(True, train_interval=25)
    db.set_param("learned_base_only", 1)
    ib, bb = [], 0
    for _ in range(steps):
        st = db.step()
        ib.append(st.iterations)
        bb |= st.status
    ib = np.array(ib)
    dl, il, _, _, bl = _run(s, steps, True, train_interval=25)
    for bits in (bp, bb, bl):
        assert bits & (_capi.ST_PRESSURE_NOT_CONVERGED | _capi.ST_NONFINITE) == 0
    assert db.get_param("mlp_trainings") == 0 and dl.get_param("mlp_trainings") >= 10
    win = slice(150, steps)
    mp, mb, ml = ip[win].mean(), ib[win].mean(), il[win].mean()
    print(f"pressure iterations: plain {mp:.2f}, base (network output 0) {mb:.2f}, trained {ml:.2f}; "
          f"network contribution {mb - ml:+.2f} iterations/step ({(mb - ml) / mb:+.1%} of the base)")
    assert mb <= 0.7 * mp
    assert ml <= 1.1 * mb
