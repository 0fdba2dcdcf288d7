"""Schedules an app registers itself (khz_app_register): validation on the host, no GPU needed.
Every index the device engine would follow must be in range, or the call fails with KHZ_ERR_ARG
and names the first bad field."""
import pytest

from openkhuzdulgraph_b200 import khz
from openkhuzdulgraph_b200.khz import AND, N, S, SUB, level, schedule, term


def _err(runs, mult=(1,)):
    with pytest.raises(khz.KhzError) as e:
        khz.register_app(runs, list(mult))
    assert e.value.status == 1
    return str(e.value)


def test_valid_schedules_get_fresh_ids():
    star = schedule(4, [level(term(N(0))), level(term(N(0), gt=[1]))], [term(N(0), gt=[2])])
    a = khz.register_app([star], [1])
    b = khz.register_app([star], [1])
    assert a >= 12 and b == a + 1
    assert khz.num_counts(a) == 1 and khz.lib().khz_app_multiplicity(a, 0) == 1
    four_cycle = schedule(4, [level(term(N(0), gt=[0])), level(term(N(1), gt=[0], ne=[0, 1]))],
                          [term(AND(N(0), 2), gt=[1], ne=[0, 1, 2])])
    fused = schedule(3, [level(term(N(0)))],
                     [term(AND(N(0), 1), gt=[1], counter=0, guard=(0, 1)), term(SUB(N(0), 1), ne=[1], counter=1)])
    c = khz.register_app([four_cycle, fused], [1, 2])
    assert khz.num_counts(c) == 2 and khz.lib().khz_app_multiplicity(c, 1) == 2


def test_invalid_schedules_are_rejected():
    ok1 = level(term(N(0)))
    assert "level 1" in _err([schedule(4, [level(term(N(1))), ok1], [term(N(0))])])
    assert "not materialised" in _err([schedule(4, [ok1, level(term(S(2)))], [term(N(0))])])
    assert "not yet matched" in _err([schedule(4, [ok1, level(term(AND(N(0), 2)))], [term(N(0))])])
    assert "not yet matched" in _err([schedule(3, [ok1], [term(N(2))])])
    assert "filter" in _err([schedule(3, [ok1], [term(N(0), gt=[2])])])
    assert "counter" in _err([schedule(3, [ok1], [term(N(0), counter=1)])])
    assert "pattern size" in _err([schedule(6, [ok1], [term(N(0))])])
    assert "cached set" in _err([schedule(4, [ok1, level(term(N(1)), cached=S(4))], [term(N(0))])])
    assert "multiplicity" in _err([schedule(3, [ok1], [term(N(0))])], mult=(0,))
    assert "num_runs" in _err([], mult=(1,))


def test_level_sets_materialised_bounded_only_when_every_use_allows():
    """Both forms register; the engine keeps a level set's members below the level's bound when a
    later use filters below it (checked on the device by the GPU schedule tests)."""
    bounded = schedule(4, [level(term(N(0), gt=[0])), level(term(AND(N(0), 1), gt=[1]))],
                       [term(AND(S(2), 2), gt=[2])])
    unbounded = schedule(4, [level(term(N(0), gt=[0])), level(term(AND(N(0), 1), gt=[1]))],
                         [term(AND(S(2), 2), gt=[0])])
    assert khz.register_app([bounded], [1]) != khz.register_app([unbounded], [1])
