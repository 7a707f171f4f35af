"""The algorithmic bytes behind bench.py's roofline, array by array: the
compulsory FP64 traffic at the four dependency boundaries of a cycle, and
this build's own traffic beside it."""
import bytes_model as b


def test_algorithmic_phases():
    assert b.phase_bytes() == {"force": 152, "nodal": 128, "kinematics": 176, "eos": 196}
    assert b.step_bytes() == 652


def test_this_build():
    # corner forces: 24 doubles written per element by force, read by nodal;
    # nodelist, links and boundary masks come from the element position
    assert b.phase_bytes(b.THIS_BUILD) == {"force": 288, "nodal": 296, "kinematics": 144,
                                           "eos": 168}
    assert b.step_bytes(b.THIS_BUILD) == 896
