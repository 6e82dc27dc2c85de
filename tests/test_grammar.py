"""The host mirror of ProtoMol's force grammar (factory/ForceFactory.cpp:
133-200) for the switching functions and algorithms beyond the benchmark
path: the parse of each line and the C-ABI switch it becomes (no device
needed)."""
import pytest

from protomol_b200 import ForceFactory
from protomol_b200 import _lib as L
from protomol_b200.engine import _switch


def test_cmpcncn_line_keeps_its_four_parameters():
    kws, alg, sws, p = ForceFactory.parse(
        "LennardJones Coulomb -algorithm NonbondedCutoff -switchingFunction ComplimentCnCn "
        "-switchon 2 -switchoff 5 -cutoff 7 -n 3 -switchingFunction ComplimentCnCn "
        "-switchon 1 -switchoff 4 -cutoff 7 -n 4 -cutoff 7")
    assert kws == ["LennardJones", "Coulomb"] and alg == "NonbondedCutoff"
    assert sws[0] == {"kind": "ComplimentCnCn", "switchon": 2.0, "switchoff": 5.0,
                      "cutoff": 7.0, "n": 3.0}
    assert sws[1]["switchoff"] == 4.0 and sws[1]["n"] == 4.0
    assert p == {"cutoff": 7.0}
    w = _switch(sws[0]["kind"], sws[0]["cutoff"], sws[0]["switchon"], sws[0]["switchoff"],
                sws[0]["n"])
    assert w.kind == L.SW_CMPCNCN and (w.cutoff, w.switchon, w.switchoff, w.order) == \
        (7.0, 2.0, 5.0, 3.0)


@pytest.mark.parametrize("name,base", [("ComplementC1", L.SW_C1), ("ComplementC2", L.SW_C2),
                                       ("ComplementCn", L.SW_CN)])
def test_complement_switch_is_a_flag_on_its_function(name, base):
    w = _switch(name, 6.0, 4.0)
    assert w.kind == base | L.SW_COMPLEMENT
    assert _switch(name[len("Complement"):], 6.0, 4.0).kind == base


def test_lattice_sum_and_scpism_lines():
    kws, alg, sws, p = ForceFactory.parse(
        "Coulomb -algorithm NonbondedFull -switchingFunction C1 -cutoff 8 -cutoff 8")
    assert alg == "NonbondedFull" and sws == [{"kind": "C1", "cutoff": 8.0}] and p["cutoff"] == 8.0
    kws, alg, sws, p = ForceFactory.parse(
        "CoulombSCPISM -algorithm NonbondedCutoff -switchingFunction C2 -switchon 0 "
        "-cutoff 12 -cutoff 12 -D 60")
    assert kws == ["CoulombSCPISM"] and p == {"cutoff": 12.0, "d": 60.0}
    kws, alg, sws, p = ForceFactory.parse(
        "BornSelf -algorithm NonbondedCutoff -switchingFunction Cutoff -bornswitch 2 "
        "-cutoff 4.5 -cutoff 4.5 -D 60")
    assert kws == ["BornSelf"] and sws == [{"kind": "Cutoff", "cutoff": 4.5}]
    assert p == {"bornswitch": 2.0, "cutoff": 4.5, "d": 60.0}


def test_unknown_switch_is_rejected():
    with pytest.raises(KeyError):
        _switch("Quartic", 8.0)
