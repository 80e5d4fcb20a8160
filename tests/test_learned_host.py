"""Host logic of the learned corrector guess (no GPU): the per-step plan
(LearnedGuess._plan) that the host-driven step and its graph form both
follow -- use the guess while its latest measured error is below the gate,
re-measure every `recheck` steps while gated off, measure every step while
gated on or training online, and nothing when disabled."""

from dnsjax_b200.learned import LearnedGuess


def guess(gate=0.9, recheck=8, train_iters=0, enabled=True):
    g = LearnedGuess.__new__(LearnedGuess)  # the plan needs no network or flow
    g.gate, g.recheck, g.train_iters, g.enabled = gate, recheck, train_iters, enabled
    g.last_rel, g._since = None, 0
    return g


def run(g, rels, n):
    """n steps; a measured step's error is taken from rels in turn.
    Returns (used, measured) per step."""
    out = []
    it = iter(rels)
    for _ in range(n):
        use, measure, since = g._plan()
        g._since = since
        if measure:
            g.last_rel = next(it)
        out.append((use, measure))
    return out


def test_first_step_uses_and_measures():
    assert run(guess(), [0.5], 1) == [(True, True)]


def test_gated_on_measures_every_step():
    steps = run(guess(), [0.5, 0.4, 0.3], 3)
    assert steps == [(True, True)] * 3


def test_gated_off_rechecks_every_recheck_steps():
    # the first measurement turns the guess off; it is measured again at
    # steps 1 + 8, 1 + 16 ... while it stays above the gate
    steps = run(guess(recheck=8), [1.5] * 10, 20)
    measured = [i for i, (_, m) in enumerate(steps) if m]
    assert measured == [0, 8, 16]
    assert [u for u, _ in steps] == [True] + [False] * 19


def test_gated_off_then_back_on():
    # off after the first measurement; the recheck three steps later is
    # below the gate, so the guess is used (and measured) from the next step
    steps = run(guess(recheck=3), [2.0, 0.5, 0.4, 0.3], 6)
    assert steps == [(True, True), (False, False), (False, False), (False, True),
                     (True, True), (True, True)]


def test_no_gate_uses_always_and_measures_only_when_training():
    assert run(guess(gate=None), [], 4) == [(True, False)] * 4
    assert run(guess(gate=None, train_iters=2), [1.0] * 4, 4) == [(True, True)] * 4


def test_disabled_neither_uses_nor_measures():
    assert run(guess(enabled=False), [], 5) == [(False, False)] * 5


def test_plan_is_pure():
    g = guess()
    g.last_rel, g._since = 1.5, 3
    a = g._plan()
    b = g._plan()
    assert a == b and g._since == 3
