"""The Python Coupling mirror (coupling.rs:150-283): defaults, declarations,
group lookup and the serde JSON form of the reference's own unit tests."""
import pytest


def test_default_couples_everything(fh):
    c = fh.Coupling.all_pairs()
    assert c.is_all_pairs() and c.is_trivial()
    assert c.couples("a", "b")
    assert c.group_of(7) == fh.DEFAULT_GROUP
    assert c.to_json() == {}


def test_truncation_and_declarations(fh):
    c = fh.Coupling.truncated(["a", "b"])
    assert not c.is_all_pairs()
    assert c.couples("a", "a") and not c.couples("a", "b")
    d = fh.Coupling.truncated(["a", "b", "c"]).coupled("a", "b")
    assert d.couples("a", "b") and d.couples("b", "a") and not d.couples("a", "c")
    short = fh.Coupling.truncated(["b"])
    assert short.group_names(3) == ["b", ""]


def test_json_round_trip(fh):
    c = fh.Coupling.truncated(["a", "b"]).coupled("a", "b")
    assert fh.Coupling.from_json(c.to_json()) == c
    assert fh.Coupling.from_json({}) == fh.Coupling.all_pairs()
    with pytest.raises(fh.InvalidArgument):
        fh.Coupling.from_json({"typo": 1})
