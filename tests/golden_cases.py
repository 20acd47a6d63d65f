"""Case definitions of the committed golden fixtures (tests/golden/*.npz and
the state digests in tests/golden/digests.json)."""
from canard_b200 import cases

# state digests: (case, steps) frozen as SHA-256 of each block's FP64 state
DIGEST_CASES = ["tgv16_step1", "tgv16_step10", "tgv16_step100", "curv4_step10", "toy_step10",
                "validation_split_step8", "toy_split_step4"]


def golden_case(name):
    if name == "tgv16_step3":
        return cases.tgv(16), 3
    if name == "curv4_step2":
        return cases.curvilinear_4block(24, 16, 14), 2
    if name.startswith("tgv16_step"):
        return cases.tgv(16), int(name.rsplit("step", 1)[1])
    if name == "curv4_step10":
        return cases.curvilinear_4block(24, 16, 14), 10
    if name == "toy_step10":
        return cases.reference_toy(16, 14, 12), 10
    if name == "validation_split_step8":
        return cases.decompose(cases.reference_validation(26, 26, 12), [(2, 2, 1)]), 8
    if name == "toy_split_step4":
        return cases.decompose(cases.reference_toy(26, 26, 12), [(2, 2, 1)] * 6), 4
    raise KeyError(name)
