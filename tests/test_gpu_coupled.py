"""Coupled gyroid step (interface reaction, 3-species solve, level-set advance) on the GPU
against the oracle's coupled step (per-species FP64 assembly + direct solve).

Bars after 3 steps: FP64 inner (rtol 1e-10) within 1e-9 relative L2 per species, FP32
inner + FP64 refinement (rtol 1e-8) within 1e-7; the level set within 1e-12 absolute;
the plain FP64 form within 1e-7 of the fast form; the learned guess changes only the
iteration count (solutions within 1e-7 of the previous-step guess)."""
import math

import numpy as np
import pytest

from oracle import oracle as orc

pytestmark = pytest.mark.gpu

N, DT = 6, 0.02
D_S, K_S = (1.0, 1.0, 2.6), (0.5, 0.0, 0.2)


def _inputs():
    from dissolve_tp.coupled import gyroid_inputs
    return gyroid_inputs(N, 0.15)


def _oracle_steps(m, phi, coef, U, steps, eps):
    return orc.gyroid_steps(m.coords, m.cells, phi, coef, U, steps, DT, eps, D_S, K_S)


@pytest.mark.parametrize("fp32,rtol,bar", [(False, 1e-10, 1e-9), (True, 1e-8, 1e-7)])
def test_coupled_step_matches_oracle(cuda_device, fp32, rtol, bar):
    from dissolve_tp.coupled import GyroidStep
    m, phi, coef, u0 = _inputs()
    h = 2 * math.pi / N
    g = GyroidStep(m, phi, coef, dt=DT, rtol=rtol, inner_fp32=fp32, h=h)
    g.set_state(u0)
    for _ in range(3):
        assert g.step()["converged"]
    Uo, phio = _oracle_steps(m, phi, coef, u0, 3, 1.5 * h)
    U = g.state()
    for s in range(3):
        assert np.linalg.norm(U[:, s] - Uo[:, s]) / np.linalg.norm(Uo[:, s]) < bar, s
    # phi moves by dt rate gain c_Cl per step: it inherits 1e-4 of the solution's error
    assert np.abs(g.phi.cpu().numpy() - phio).max() < (1e-12 if not fp32 else 1e-10)


def test_plain_form_matches_fast_form(cuda_device):
    from dissolve_tp.coupled import GyroidStep, GyroidStepPlain
    m, phi, coef, u0 = _inputs()
    h = 2 * math.pi / N
    g = GyroidStep(m, phi, coef, dt=DT, rtol=1e-8, h=h)
    p = GyroidStepPlain(m, phi, coef, dt=DT, rtol=1e-8, h=h)
    g.set_state(u0)
    p.set_state(u0)
    for _ in range(3):
        assert g.step()["converged"]
        assert all(r["converged"] for r in p.step())
    a, b = g.state(), p.state()
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-7


def test_learned_guess_only_changes_iterations(cuda_device):
    from dissolve_tp.coupled import GyroidStep
    m, phi, coef, u0 = _inputs()
    h = 2 * math.pi / N
    runs = {}
    for guess in ("previous", "learned"):
        g = GyroidStep(m, phi, coef, dt=DT, rtol=1e-8, h=h)
        g.set_state(u0)
        if guess == "learned":
            g.train_predictor(12, every=2, epochs=100)
        else:
            for _ in range(12):
                g.step()
        its = []
        for _ in range(4):
            r = g.step()
            assert r["converged"]
            its.append(r["iterations"])
        runs[guess] = g.state()
    a, b = runs["learned"], runs["previous"]
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-7


def test_graph_replay_matches_eager_steps(cuda_device):
    """The coupled step with the learned guess captured once in a CUDA graph and replayed:
    the same iteration counts and states as the same steps run eagerly (the increment
    history shifts in fixed buffers, so the replay sees the new history each time)."""
    import torch

    from dissolve_tp.coupled import GyroidStep
    m, phi, coef, u0 = _inputs()
    runs = {}
    for mode in ("eager", "graph"):
        g = GyroidStep(m, phi, coef, dt=DT)
        g.set_state(u0)
        g.train_predictor(12, every=3, epochs=100, seed=5)
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            for _ in range(2):
                g.step(sync=False)
        torch.cuda.current_stream().wait_stream(s)
        its = []
        if mode == "graph":
            # capture records the step without running it; each replay runs one step
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph):
                g.step(sync=False)
            for _ in range(5):
                graph.replay()
                its.append(g.tr.solver.result()["iterations"])
            del graph
        else:
            for _ in range(5):
                its.append(g.step()["iterations"])
        runs[mode] = (its, g.state())
    assert runs["graph"][0] == runs["eager"][0], runs
    # the captured step keeps the set of directions whose stiffness images were known at
    # capture (the eager steps gain more as they go): the guesses differ by rounding and
    # both solves stop at rtol 1e-8
    a, b = runs["graph"][1], runs["eager"][1]
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-8
