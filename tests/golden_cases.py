"""Case definitions of the committed golden fixtures (tests/golden/*.npz)."""
from canard_b200 import cases


def golden_case(name):
    if name == "tgv16_step3":
        return cases.tgv(16), 3
    if name == "curv4_step2":
        return cases.curvilinear_4block(24, 16, 14), 2
    raise KeyError(name)
