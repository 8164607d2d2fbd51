"""The C ABI without a GPU: the library loads, exports every entry point include/*.h declares, and its spec parser
(host code) follows the reference's grammar and exit codes (src/cheese.cu:1149-1226)."""
import ctypes as C
import re
from pathlib import Path

import pytest

import cheese_b200 as cz
from conftest import ROOT, spec_text


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        src = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^\s*[A-Za-z_][\w\s\*]*?\b(cz_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_entry_point():
    lib = cz.lib()
    names = declared_functions()
    assert {"cz_spec_parse", "cz_search", "cz_engine_create"} <= names
    for n in names:
        assert hasattr(lib, n), n
    assert set(cz.SIGNATURES) >= names


def test_version_names_the_architecture():
    assert b"sm_100a" in cz.lib().cz_version()


def test_parse_reference_spec():
    s = cz.Spec(spec_text("toffoli"))
    assert (s.n, s.gates) == (3, 27) and s.depth >= 1
    assert s.names[0] == "L_cx_0_1" and s.names[-1] == "L_z_2"
    s2 = cz.Spec(spec_text("cs"))
    assert (s2.n, s2.gates) == (2, 16)


@pytest.mark.parametrize("text,rc,msg", [
    ("hello 1\n", 2, "not a spec"),
    ("", 2, "not a spec"),
    ("cheese-spec 1\nn 3\nbogus 1\n", 2, "unknown spec field bogus"),
    ("cheese-spec 1\nmode qudit\n", 2, "unsupported mode qudit"),
    ("cheese-spec 1\nn 5\ntarget 0\nend\n", 3, "not built"),
])
def test_parse_errors_follow_reference_codes(text, rc, msg):
    with pytest.raises(cz.SpecError) as e:
        cz.Spec(text)
    assert e.value.rc == rc
    assert msg in str(e.value)


def test_too_many_gates_is_a_spec_error():
    with pytest.raises(cz.SpecError) as e:
        cz.Spec("cheese-spec 1\nn 3\ngates 65\n")
    assert e.value.rc == 2 and "too many gates" in str(e.value)


def test_state_specs_are_parsed():
    # a state-target spec: parsed (grammar, start rows, goal rows and goal bounds) and flagged
    s = cz.Spec(spec_text("cs-states"))
    assert s.states
    with pytest.raises(cz.SpecError) as e:      # a states header without its start / goal blocks
        cz.Spec(spec_text("cs").replace("mode unitary", "mode states"))
    assert e.value.rc == 2 and "states spec incomplete" in str(e.value)


def test_cuts_outside_the_register_are_refused():
    """a cut naming a qubit outside the register (or twice) is refused on the host: the device never indexes with it"""
    t = spec_text("toffoli")
    head, tail = t[:t.index("cuts ")], t[t.index("cxtable"):]
    for cuts, msg in (("cuts 3\n1 0\n1 1\n1 3\n", "cut acts outside the register"), ("cuts 1\n2 0 0\n", "bad cut"),
                      ("cuts 1\n1 -1\n", "bad cut")):
        with pytest.raises(cz.SpecError) as e:
            cz.Spec(head + cuts + tail)
        assert e.value.rc == 2 and msg in str(e.value)
    cz.Spec(head + "cuts 3\n1 0\n1 1\n1 2\n" + tail)


def test_state_goal_info_must_cover_every_pair():
    """the goal lines (sde, nullity, one Schmidt rank per cut) must cover every pair and cut the device reads"""
    t = spec_text("cs-states")
    short = t.replace("goal 2\n0 0 1\n0 0 1\n", "goal 1\n0 0 1\n")
    assert short != t
    with pytest.raises(cz.SpecError) as e:
        cz.Spec(short)
    assert e.value.rc == 2 and "states spec incomplete" in str(e.value)
